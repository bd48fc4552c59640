"""Edge cases through the C ABI on the GPU: rays with NaN or infinite
components, zero and axis-aligned directions, rays starting inside patches;
patches with a zero or a negative weight, a net collapsed to one point and a
net flat in a plane; ray counts of 1, 31, 33 and an odd size across wavefront
passes.  Every schedule (per-pixel kernel, wavefront in the CUDA graph, with
host-driven rounds, the no-allocation entry point) must report no device
error, give the same hit/miss decision on every ray and bit-identical t, u, v
where it hits the same patch; rays with a NaN component miss."""
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


def edge_patches():
    rng = np.random.default_rng(3)
    cps, off, deg = [], [], []

    def add(pts, p, q):
        off.append(sum(len(c) for c in cps))
        cps.append(np.asarray(pts, np.float32))
        deg.append((p, q))

    for k in range(6):  # bicubic bumps on a row
        g = np.linspace(0, 1, 4)
        X, Y = np.meshgrid(g, g, indexing="ij")
        Z = 0.2 * rng.normal(size=X.shape)
        w = rng.uniform(0.5, 2.0, X.shape)
        P = np.stack([(X + 1.2 * k) * w, Y * w, Z * w, w], -1).reshape(-1, 4)
        if k == 1:
            P[5] = 0.0          # a zero weight (and zero homogeneous point)
        if k == 2:
            P[6] *= -1.0        # a negative weight (same dehomogenised point)
        if k == 3:
            P[:, :3] = P[:, 3:4] * np.array([1.2 * k + 0.5, 0.5, 0.0])  # all points coincident
        if k == 4:
            P[:, 2] = 0.0       # flat in the plane z = 0
        add(P, 3, 3)
    return np.concatenate(cps), np.array(off, np.int32), np.array(deg, np.int32)


def edge_rays(n_cam=4000, seed=1):
    rng = np.random.default_rng(seed)
    o = np.stack([rng.uniform(-0.5, 7.5, n_cam), rng.uniform(-0.2, 1.2, n_cam), np.full(n_cam, -3.0)], 1)
    d = np.stack([rng.normal(0, 0.05, n_cam), rng.normal(0, 0.05, n_cam), np.ones(n_cam)], 1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    nan, inf = np.nan, np.inf
    special_o = [[0.5, 0.5, -3], [nan, 0.5, -3], [0.5, 0.5, -3], [0.5, 0.5, -3], [inf, 0, 0], [1.5, 0.5, 0.0],
                 [2.5, 0.5, 0.0], [0.5, 0.5, -3], [4.1, 0.4, -1], [5.3, 0.3, 1.0]]
    special_d = [[0, 0, 1], [0, 0, 1], [nan, 0, 1], [0, 0, 0], [0, 0, 1], [0, 0, 1],
                 [1, 0, 0], [0, 0, -1], [0, 0, 1], [0, 0, -1]]
    o = np.concatenate([o, np.array(special_o)]).astype(np.float32)
    d = np.concatenate([d, np.array(special_d)]).astype(np.float32)
    return o, d


def run_all(nrt_gpu, scene, rays, opts):
    import torch

    res = {}
    scene.enable_counters(True)
    for name, o, tune in [("pixel", opts, None), ("graph", opts.replace(schedule=nrt_gpu.SCHED_WAVEFRONT), 1),
                          ("host", opts.replace(schedule=nrt_gpu.SCHED_WAVEFRONT), 2)]:
        if tune:
            scene.set_tuning(graph=tune)
        res[name] = to_numpy(scene.intersect(rays, o))
        assert scene.counters()["errors"] == 0, name
    n = rays[0].numel()
    out = {k: torch.empty(n, dtype=torch.int32 if k == "patch" else torch.float32, device="cuda")
           for k in ("patch", "t", "u", "v")}
    from nrt.lib import HitsC, RaysC, _ptr, _check, lib
    import ctypes as C

    r = RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
    h = HitsC(_ptr(out["patch"]), _ptr(out["t"]), _ptr(out["u"]), _ptr(out["v"]), None, None, None)
    _check(lib().nrt_intersect_noalloc(scene.handle, C.byref(r), n, C.byref(opts), C.byref(h), None))
    res["noalloc"] = to_numpy(out)
    scene.enable_counters(False)
    return res


def check_same(res):
    a = res["pixel"]
    for name, b in res.items():
        hit_a, hit_b = a["patch"] >= 0, b["patch"] >= 0
        assert np.array_equal(hit_a, hit_b), name
        same = hit_a & (a["patch"] == b["patch"])
        assert same.sum() >= 0.999 * hit_a.sum(), name
        for k in ("t", "u", "v"):
            assert np.array_equal(a[k][same], b[k][same]), (name, k)


@pytest.mark.parametrize("hull", [0, 3])
def test_degenerate_patches_and_rays(nrt_gpu, hull):
    import torch

    cp, off, deg = edge_patches()
    scene = nrt_gpu.Scene(patches=(cp, off, deg))
    o, d = edge_rays()
    rays = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in (o[:, 0], o[:, 1], o[:, 2], d[:, 0], d[:, 1], d[:, 2])]
    for opts in (nrt_gpu.default_opts(hull_cull=hull, fp64_final=1, cond_fp64=1e4),
                 nrt_gpu.reference_opts(hull_cull=min(hull, 1))):
        res = run_all(nrt_gpu, scene, rays, opts)
        check_same(res)
        nan_ray = np.isnan(o).any(1) | np.isnan(d).any(1)
        assert (res["graph"]["patch"][nan_ray] == -1).all()
        assert (res["pixel"]["patch"] >= 0).mean() > 0.3


@pytest.mark.parametrize("n", [1, 31, 33, 100003])
def test_ragged_ray_counts(nrt_gpu, n):
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(4, seed=9, width=400, height=300, spp=1)
    scene = nrt_gpu.Scene(sc.surfaces, wavefront_chunk=40000)
    rays = [a[:n].contiguous() for a in nrt_gpu.camera_rays(sc.camera)]
    res = run_all(nrt_gpu, scene, rays, nrt_gpu.default_opts(hull_cull=3, fp64_final=1))
    check_same(res)
