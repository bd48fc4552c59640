"""GPU parity of the wavefront schedule (through the C ABI).

Tolerances:
  * against the per-pixel schedule with the same options: identical hit/miss
    on >= 99.99% of rays, the same patch on >= 99.9% of rays both hit (the two
    may pick different patches only on exact ties), identical (bit-equal) t, u,
    v where they pick the same patch.
  * against the FP64 oracle (same method): hit/miss agreement >= 99.99%,
    relative t error <= 1e-4 and (u,v) error <= 1e-3 on same-patch hits.
"""
import numpy as np
import pytest

from conftest import golden_rays, golden_surfaces, load_golden
from parity import compare, gpu_rays, to_numpy

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


def same_as_pixel(nrt_gpu, scene, rays, base):
    a = to_numpy(scene.intersect(rays, base.replace(schedule=nrt_gpu.SCHED_PIXEL)))
    b = to_numpy(scene.intersect(rays, base.replace(schedule=nrt_gpu.SCHED_WAVEFRONT)))
    hit_a, hit_b = a["patch"] >= 0, b["patch"] >= 0
    assert (hit_a == hit_b).mean() >= 0.9999
    both = hit_a & hit_b
    same = both & (a["patch"] == b["patch"])
    assert same.sum() >= 0.999 * both.sum()
    for k in ("t", "u", "v", "iters"):
        assert np.array_equal(a[k][same], b[k][same]), k
    return a, b


@pytest.mark.parametrize("name", ["heightfield", "torus", "sphere", "mixed4"])
def test_wavefront_matches_pixel_on_fixtures(nrt_gpu, name):
    g = load_golden(name)
    scene = nrt_gpu.Scene(golden_surfaces(g))
    rays = gpu_rays(golden_rays(g))
    for base in [nrt_gpu.default_opts(), nrt_gpu.default_opts(hull_cull=1, fp64_final=1, cond_fp64=1e4),
                 nrt_gpu.reference_opts(), nrt_gpu.reference_opts(hull_cull=1)]:
        same_as_pixel(nrt_gpu, scene, rays, base)


def test_wavefront_many_surfaces_vs_fp64(nrt_gpu, oracle_mod):
    """16 mixed-degree surfaces, 320x180x2 jittered rays, against the FP64 oracle."""
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(16, seed=5, width=320, height=180, spp=2)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    opts = nrt_gpu.default_opts(hull_cull=1, fp64_final=1, cond_fp64=1e4, schedule=nrt_gpu.SCHED_WAVEFRONT)
    out = to_numpy(scene.intersect(rays, opts))
    P = oracle_mod.decompose_scene(sc.surfaces, f64=False)
    P.cp64 = P.cp.astype(np.float64)
    nb, lf, cnt, order, used = nrt_gpu.build_bvh_binary(nrt_gpu.patch_bounds(P.cp, P.off, P.deg),
                                                        nrt_gpu.BVH_BINNED_SAH)
    r_np = oracle_mod.Rays(*[a.cpu().numpy() for a in rays])
    ref = oracle_mod.intersect(P, oracle_mod.BinaryBVH(nb, lf, cnt, order, used), r_np, 0, 8, 1e-6, f64=True)
    st = compare(out, ref.patch, ref.t, ref.u, ref.v)
    assert st["hit_rate"] > 0.3, st
    assert st["agree"] >= 0.9999, st
    assert st["t_rel_max"] <= 1e-4, st
    assert st["uv_abs_p999"] <= 1e-3, st
    same_as_pixel(nrt_gpu, scene, rays, opts)


def test_wavefront_chunks_and_overflow(nrt_gpu):
    """Small chunks (many passes) and rays with more candidates than a list
    holds (per-pixel fallback) give the per-pixel results."""
    import torch

    from nrt import scenes

    # 48 stacked parallel bilinear sheets: a ray along z crosses all of them
    cp, off, deg = [], [], []
    for k in range(48):
        z = 0.1 * k
        for (x, y) in [(0, 0), (0, 1), (1, 0), (1, 1)]:
            cp.append([x, y, z, 1.0])
        off.append(4 * k)
        deg.append([1, 1])
    cp = np.array(cp, np.float32)
    scene = nrt_gpu.Scene(patches=(cp, np.array(off, np.int32), np.array(deg, np.int32)), wavefront_chunk=100)
    n = 1000
    rng = np.random.default_rng(0)
    o = np.stack([rng.uniform(0.05, 0.95, n), rng.uniform(0.05, 0.95, n), np.full(n, -1.0)], 1).astype(np.float32)
    d = np.tile(np.array([[0.0, 0.0, 1.0]], np.float32), (n, 1))
    d[::2] = np.array([0.05, 0.02, 1.0]) / np.linalg.norm([0.05, 0.02, 1.0])
    rays = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (o[:, 0], o[:, 1], o[:, 2], d[:, 0], d[:, 1], d[:, 2])]
    a, b = same_as_pixel(nrt_gpu, scene, rays, nrt_gpu.default_opts(hull_cull=1))
    near = a["patch"] == 0  # the nearest sheet, at z = 0
    assert near.mean() > 0.9
    np.testing.assert_allclose(a["t"][near], 1.0 / d[near, 2], rtol=1e-6)
    sc = scenes.heightfield_scene(0, 64, 48)
    scene = nrt_gpu.Scene(sc.surfaces, wavefront_chunk=777)
    same_as_pixel(nrt_gpu, scene, nrt_gpu.camera_rays(sc.camera), nrt_gpu.default_opts(hull_cull=1, fp64_final=1))


def test_clip_cull_changes_nothing(nrt_gpu):
    """The oriented-box and exact hull culls (levels 3, 4) on 16 random mixed-degree surfaces, where
    most (ray, patch) candidates that reach Newton have no root: bit-identical
    hits to no cull at all, and more candidates culled than the levels below."""
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(16, seed=5, width=320, height=180, spp=2)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    W = nrt_gpu.SCHED_WAVEFRONT
    culled = {}
    base = to_numpy(scene.intersect(rays, nrt_gpu.default_opts(schedule=W)))
    for level in (1, 2, 3, 4):
        scene.enable_counters(True)
        b = to_numpy(scene.intersect(rays, nrt_gpu.default_opts(schedule=W, hull_cull=level)))
        c = scene.counters()
        scene.enable_counters(False)
        culled[level] = c["patch_culled"]
        assert c["errors"] == 0
        for k in ("patch", "t", "u", "v", "iters"):
            assert np.array_equal(base[k], b[k]), (k, level)
    assert culled[4] > culled[3] > culled[2] > culled[1] > 0, culled


def test_tuning_changes_nothing_and_autotune(nrt_gpu):
    """Launch shapes (graph or host-driven rounds, grid sizes, rays per pass,
    the staged top of the tree) change no result bit; the autotuner picks one
    of them."""
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(16, seed=5, width=320, height=180, spp=2)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    opts = nrt_gpu.default_opts(hull_cull=3, fp64_final=1, cond_fp64=1e4, schedule=nrt_gpu.SCHED_WAVEFRONT)
    scene.enable_counters(True)
    base = to_numpy(scene.intersect(rays, opts))
    c0 = scene.counters()
    assert c0["rounds"] > 1 and c0["kernel_launches"] > c0["rounds"]
    # (set_tuning keeps the fields a variant leaves out: the staged-top variants come before the quota
    # variants, so that they run with the default quotas and their per-ray test counts can be compared)
    for kw in [dict(graph=2), dict(graph=1, step_blocks=37, scatter_blocks=11, class_blocks=5),
               dict(graph=1, chunk=10007), dict(graph=2, chunk=4096), dict(graph=1, stage_nodes=341),
               dict(graph=2, stage_nodes=85), dict(graph=1, stage_nodes=1), dict(graph=1, quota0=8, quota_max=8),
               dict(graph=2, quota0=1, quota_max=1), dict(graph=1, quota0=2, quota_max=4)]:
        scene.set_tuning(**kw)
        b = to_numpy(scene.intersect(rays, opts))
        c = scene.counters()
        for k in ("patch", "t", "u", "v", "iters") + (() if "quota0" in kw else ("tests",)):
            assert np.array_equal(base[k], b[k]), (k, kw)
        assert c["hits"] == c0["hits"], kw
        if "quota0" not in kw:  # the round quotas change which candidates are pruned, not the hits
            assert c["newton_evals"] == c0["newton_evals"], kw
    scene.set_tuning(chunk=1 << 23, quota0=1, quota_max=8)
    scene.enable_counters(False)
    t, ms = scene.autotune(rays, opts, reps=1)
    assert ms > 0 and t["graph"] in (1, 2) and t["step_blocks"] > 0
    assert scene.tuning() == t
    b = to_numpy(scene.intersect(rays, opts))
    for k in ("patch", "t", "u", "v", "iters"):
        assert np.array_equal(base[k], b[k]), k


def test_refined_torus(nrt_gpu, oracle_mod):
    """The exact torus after the reference's curvature refinement (C = 4, as
    src/core/main.cpp:100-102): both schedules agree with each other and with
    the FP64 oracle on the refined patches."""
    from nrt import scenes

    sc = scenes.analytic_scene("torus", 192, 108)
    surf = nrt_gpu.refine(sc.surfaces[0], 4.0)
    scene = nrt_gpu.Scene([surf])
    rays = nrt_gpu.camera_rays(sc.camera)
    opts = nrt_gpu.default_opts(hull_cull=3, fp64_final=1, cond_fp64=1e4, schedule=nrt_gpu.SCHED_WAVEFRONT)
    out = to_numpy(scene.intersect(rays, opts))
    same_as_pixel(nrt_gpu, scene, rays, opts.replace(hull_cull=1))
    P = oracle_mod.decompose_scene([surf], f64=False)
    P.cp64 = P.cp.astype(np.float64)
    ref = oracle_mod.intersect(P, oracle_mod.build_bvh(oracle_mod.patch_boxes(P)),
                               oracle_mod.Rays(*[a.cpu().numpy() for a in rays]), 0, 8, 1e-6, f64=True)
    st = compare(out, ref.patch, ref.t, ref.u, ref.v)
    assert st["hit_rate"] > 0.02 and st["agree"] >= 0.9999, st
    assert st["t_rel_max"] <= 1e-4, st


@pytest.mark.parametrize("name", ["heightfield", "torus", "sphere", "mixed4"])
def test_flat_skip_both_schedules(nrt_gpu, name):
    """Flat-skip at 2 px with the reference's settings (golden fixture flat2px,
    made by the reference's own code): the per-pixel kernel and the wavefront
    agree with each other (the wavefront accepts a flat guess even when a
    nearer hit is already known, where the per-pixel kernel would run Newton
    on that patch; both keep the nearest), and both agree with the reference's
    outputs on >= 99.9 % of hit/miss decisions, on the patch for >= 99 % of
    rays both hit, with relative t differences <= 1e-2 at the 99th percentile
    (an accepted flat guess is a pixel-level approximation; different trees
    and visiting orders accept different guesses)."""
    g = load_golden(name)
    scene = nrt_gpu.Scene(golden_surfaces(g))
    rays = gpu_rays(golden_rays(g))
    c = g["camera"]
    cam_k = float(0.5 * c[11] / np.tan(np.radians(c[9]) / 2.0))
    base = nrt_gpu.reference_opts(flat_threshold=2.0, cam_k=cam_k)
    scene.enable_counters(True)
    a = to_numpy(scene.intersect(rays, base))
    skips_pixel = scene.counters()["flat_skips"]
    b = to_numpy(scene.intersect(rays, base.replace(schedule=nrt_gpu.SCHED_WAVEFRONT)))
    skips_wf = scene.counters()["flat_skips"]
    scene.enable_counters(False)
    if name in ("heightfield", "mixed4"):  # the torus and sphere fixtures are not flat enough at 2 px
        assert skips_pixel > 0 and skips_wf > 0
    hit_a, hit_b = a["patch"] >= 0, b["patch"] >= 0
    assert (hit_a == hit_b).mean() >= 0.999
    slot = g["flat2px_hit_slot"]
    order = g["bvh_order"]
    ref_patch = np.where(slot >= 0, order[np.maximum(slot, 0)], -1)
    for out in (a, b):
        st = compare(out, ref_patch, g["flat2px_t"].astype(np.float64))
        both = (out["patch"] >= 0) & (ref_patch >= 0)
        rel = np.abs(out["t"][both] - g["flat2px_t"][both]) / np.abs(g["flat2px_t"][both])
        print(name, st["agree"], st["same_patch"], np.quantile(rel, 0.99) if rel.size else None)
        assert st["agree"] >= 0.999 and st["same_patch"] >= 0.99, st
        assert rel.size == 0 or np.quantile(rel, 0.99) <= 1e-2
