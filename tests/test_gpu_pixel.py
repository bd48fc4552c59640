"""GPU parity of the per-pixel CUDA path (through the C ABI) against the oracle.

Tolerances (stated here, checked below):
  * rays: bit-exact against the oracle's closed-form camera (both FP64, unfused).
  * plain settings (midpoint init, 8 evaluations, eps 1e-6) against the FP64
    oracle running the same method: hit/miss agreement >= 99.99%, and on rays
    that hit the same patch, relative t error <= 1e-4 and (u,v) error <= 1e-3.
  * reference settings (bilinear guess, 7 evaluations, eps 1e-4) against the
    reference's own outputs (golden fixtures): hit/miss agreement >= 99.9%,
    same patch >= 99.5%, relative t error <= 1e-3 (eps 1e-4 is a loose stop:
    two FP32 runs may stop on different iterates within the tolerance).
  * the hull test never changes a result: outputs with and without it are
    identical.
"""
import numpy as np
import pytest

from conftest import golden_rays, golden_surfaces, load_golden
from parity import compare, gpu_rays, to_numpy

pytestmark = pytest.mark.gpu

FIXTURES = ["heightfield", "torus", "sphere", "mixed4"]


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


def oracle_patches(oracle_mod, surfaces):
    P = oracle_mod.decompose_scene(surfaces, f64=False)
    P.cp64 = P.cp.astype(np.float64)  # the FP64 oracle solves the same (float) patches
    return P


@pytest.mark.parametrize("spp", [1, 4])
def test_camera_rays_bit_exact(nrt_gpu, oracle_mod, spp):
    from nrt import scenes

    cam = scenes.heightfield_scene(0, 96, 64, spp).camera
    cam.seed = 7
    g = [a.cpu().numpy() for a in nrt_gpu.camera_rays(cam)]
    o = oracle_mod.camera_rays(cam).arrays()
    for a, b in zip(g, o):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_heightfield_plain_vs_fp64(nrt_gpu, oracle_mod):
    """The small height-field scene (25 patches, 256x256) with the plain settings."""
    from nrt import scenes

    sc = scenes.heightfield_scene(0)
    P = oracle_patches(oracle_mod, sc.surfaces)
    bvh = oracle_mod.build_bvh(oracle_mod.patch_boxes(P))
    rays = oracle_mod.camera_rays(sc.camera)
    ref64 = oracle_mod.intersect(P, bvh, rays, init_mode=0, max_iter=8, eps=1e-6, f64=True)
    scene = nrt_gpu.Scene(sc.surfaces)
    for opts in [nrt_gpu.default_opts(), nrt_gpu.default_opts(fp64_final=1, cond_fp64=1e4)]:
        out = to_numpy(scene.intersect(gpu_rays(rays), opts))
        st = compare(out, ref64.patch, ref64.t, ref64.u, ref64.v)
        assert st["agree"] >= 0.9999, st
        assert st["same_patch"] >= 0.999, st
        assert st["t_rel_max"] <= 1e-4, st
        assert st["uv_abs_max"] <= 1e-3, st


@pytest.mark.parametrize("name", FIXTURES)
def test_reference_mode_vs_reference_outputs(nrt_gpu, oracle_mod, name):
    g = load_golden(name)
    surfaces = golden_surfaces(g)
    rays = golden_rays(g)
    order = g["bvh_order"]
    slot = g["ref_hit_slot"]
    ref_patch = np.where(slot >= 0, order[np.maximum(slot, 0)], -1)
    scene = nrt_gpu.Scene(surfaces)
    out = to_numpy(scene.intersect(gpu_rays(rays), nrt_gpu.reference_opts()))
    st = compare(out, ref_patch, g["ref_t"].astype(np.float64), g["ref_u"], g["ref_v"])
    assert st["agree"] >= 0.999, st
    assert st["same_patch"] >= 0.995, st
    assert st.get("t_rel_max", 0.0) <= 1e-3, st


@pytest.mark.parametrize("name", FIXTURES)
def test_hull_cull_changes_nothing(nrt_gpu, name):
    g = load_golden(name)
    scene = nrt_gpu.Scene(golden_surfaces(g))
    rays = gpu_rays(golden_rays(g))
    for base in [nrt_gpu.default_opts(), nrt_gpu.reference_opts()]:
        for sched in (nrt_gpu.SCHED_PIXEL, nrt_gpu.SCHED_WAVEFRONT):
            a = to_numpy(scene.intersect(rays, base.replace(schedule=sched)))
            for level in (1, 2, 3, 4):
                b = to_numpy(scene.intersect(rays, base.replace(hull_cull=level, schedule=sched)))
                for k in ("patch", "t", "u", "v", "iters"):
                    assert np.array_equal(a[k], b[k]), (k, sched, level)


def test_counters_and_empty_launch(nrt_gpu):
    import torch

    from nrt import scenes

    sc = scenes.heightfield_scene(0, 64, 64)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    scene.enable_counters(True)
    out = scene.intersect(rays, nrt_gpu.default_opts(hull_cull=1))
    c = scene.counters()
    hits = int((out["patch"] >= 0).sum())
    assert c["rays"] == 64 * 64 and c["hits"] == hits and c["errors"] == 0
    assert c["patch_candidates"] >= c["patch_culled"] + c["newton_solves"]
    assert c["newton_solves"] == int(out["tests"].sum())
    empty = [torch.empty(0, device="cuda") for _ in range(6)]
    r = scene.intersect(empty, nrt_gpu.default_opts())
    assert r["patch"].numel() == 0
