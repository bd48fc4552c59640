"""The device scene builder (NRT_BVH_BINNED_SAH_DEVICE: decomposition, patch
boxes, binned SAH, 4-wide collapse and per-slot packing as kernels) against
the host builder (NRT_BVH_BINNED_SAH).

Bar: the two device arenas are equal byte for byte, the only tolerated
difference being a float zero stored with the other sign (a min or max that
met both +0 and -0 may keep either); intersection through the two scenes
returns bit-identical hits (patch, t, u, v) on both schedules.

Scenes: the mixed-degree lattice (64 surfaces, about 10k patches: the SAH's
block-per-node kernel runs on its top levels), 256 surfaces (about 60k
patches), the torus and the sphere, the torus after curvature refinement
(C = 4), 32 degree-7 patches with weights over four decades and collapsed
edges, and patches with a zero weight (NaN points), a negative weight, a net
collapsed to one point and a flat net, each also with 8 patches per leaf."""
import numpy as np
import pytest

from parity import to_numpy

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


def arena_diff(a, b):
    """Number of 32-bit words that differ only in the sign of a zero; fails on any other difference."""
    assert a.shape == b.shape
    wa, wb = a.view(np.uint32), b.view(np.uint32)
    d = wa != wb
    if d.any():
        x, y = wa[d], wb[d]
        signed_zero = ((x | y) == 0x80000000) & ((x & y) == 0)
        bad = np.flatnonzero(d)[~signed_zero]
        assert bad.size == 0, f"{bad.size} arena words differ, first at byte {4 * bad[0]}"
    return int(d.sum())


def same_scene(nrt_gpu, make, rays=None, max_leaf=1):
    host = make(nrt_gpu.BVH_BINNED_SAH, max_leaf)
    dev = make(nrt_gpu.BVH_BINNED_SAH_DEVICE, max_leaf)
    ih, idv = host.info(), dev.info()
    assert ih == idv, (ih, idv)
    arena_diff(host.arena(), dev.arena())
    sh, sd = host.patch_table(), dev.patch_table()
    assert np.array_equal(sh[0], sd[0]) and np.array_equal(sh[1], sd[1])
    if rays is not None:
        for sched in (nrt_gpu.SCHED_PIXEL, nrt_gpu.SCHED_WAVEFRONT):
            opts = nrt_gpu.default_opts(hull_cull=3, schedule=sched)
            a, b = to_numpy(host.intersect(rays, opts)), to_numpy(dev.intersect(rays, opts))
            for k in ("patch", "t", "u", "v"):
                assert np.array_equal(a[k], b[k]), (sched, k)
            assert (a["patch"] >= 0).mean() > 0.01
    return ih


def surface_maker(nrt_gpu, surfaces):
    return lambda builder, max_leaf: nrt_gpu.Scene(surfaces, builder=builder, max_leaf=max_leaf)


@pytest.mark.parametrize("name", ["mixed64", "wave256"])
def test_lattice_scenes(nrt_gpu, name):
    from nrt import scenes

    sc = scenes.mixed_degree_scene() if name == "mixed64" else scenes.wavefront_scene()
    cam = scenes.Camera(sc.camera.eye, sc.camera.look, sc.camera.up, sc.camera.fov_deg, 480, 270, 1, 7)
    info = same_scene(nrt_gpu, surface_maker(nrt_gpu, sc.surfaces), nrt_gpu.camera_rays(cam))
    assert info["n_patches"] > 4096  # the block-per-node SAH kernel ran


@pytest.mark.parametrize("kind", ["torus", "sphere", "refined_torus"])
def test_analytic(nrt_gpu, kind):
    from nrt import scenes

    sc = scenes.analytic_scene("sphere" if kind == "sphere" else "torus", 192, 108)
    surfs = [nrt_gpu.refine(sc.surfaces[0], 4.0)] if kind == "refined_torus" else sc.surfaces
    for max_leaf in (1, 4):
        same_scene(nrt_gpu, surface_maker(nrt_gpu, surfs), nrt_gpu.camera_rays(sc.camera), max_leaf)


def patch_maker(nrt_gpu, cp, off, deg):
    return lambda builder, max_leaf: nrt_gpu.Scene(patches=(cp, off, deg), builder=builder, max_leaf=max_leaf)


def test_precision_patches(nrt_gpu):
    from nrt import scenes

    cp, off, deg = scenes.precision_patches()
    rays = nrt_gpu.camera_rays(scenes.precision_camera(640, 360))
    same_scene(nrt_gpu, patch_maker(nrt_gpu, cp, off, deg), rays)


def test_degenerate_patches(nrt_gpu):
    """Zero weight (NaN points and a NaN box corner), negative weight,
    coincident points, a flat net, duplicated patches; 1 and 8 per leaf."""
    import torch
    from test_gpu_edge_cases import edge_patches, edge_rays

    cp, off, deg = edge_patches()
    # five copies of the set, shifted, plus duplicates of two patches
    n_pts = cp.shape[0]
    cps, offs, degs = [], [], []
    for k in range(5):
        c = cp.copy()
        c[:, 1] += 1.5 * k * c[:, 3]
        cps.append(c)
        offs.append(off + k * n_pts)
        degs.append(deg)
    cps = np.concatenate(cps)
    offs = np.concatenate(offs + [off[:2], off[:2]])
    degs = np.concatenate(degs + [deg[:2], deg[:2]])
    o, d = edge_rays()
    rays = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (*o.T, *d.T)]
    for max_leaf in (1, 8):
        same_scene(nrt_gpu, patch_maker(nrt_gpu, cps, offs, degs), rays, max_leaf)


def test_leaf_limit_error(nrt_gpu):
    """Nine patches with the same box cannot be split: both builders refuse
    the scene the same way (a leaf above 8 patches)."""
    from test_gpu_edge_cases import edge_patches

    cp, off, deg = edge_patches()
    offs = np.repeat(off[:1], 9)
    degs = np.repeat(deg[:1], 9, axis=0)
    msgs = []
    for builder in (nrt_gpu.BVH_BINNED_SAH, nrt_gpu.BVH_BINNED_SAH_DEVICE):
        with pytest.raises(nrt_gpu.NrtError) as e:
            nrt_gpu.Scene(patches=(cp, offs, degs), builder=builder)
        assert e.value.status == 3
        msgs.append(str(e.value))
    assert msgs[0] == msgs[1] and "limit 8" in msgs[0]
