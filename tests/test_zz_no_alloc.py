"""nrt_intersect_noalloc: intersection for callers that cannot allocate GPU
memory while they run (fixed-budget real-time loops, code under a memory pool
that owns the device).  Its scratch is a fixed array inside libnrt.so, so the
test checks that it returns what nrt_intersect's wavefront schedule returns,
with the tolerance of the other wavefront tests (identical hit/miss on
>= 99.99% of rays, same patch on >= 99.9% of rays both hit, bit-equal t, u, v
where the patch is the same), on two calls in a row (the second one runs on the
array the first left behind).  The ray batch is larger than one pass through
the array, so the passes are exercised too.  The property the entry point
exists for is checked as well: after a warm-up call, a further call leaves the
device's free memory (cudaMemGetInfo) exactly where it was.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    L = nrt.lib()
    L.nrt_intersect_noalloc.argtypes = [C.c_void_p, C.POINTER(nrt.lib_module.RaysC), C.c_int64,
                                        C.POINTER(nrt.IntersectOpts), C.POINTER(nrt.lib_module.HitsC), C.c_void_p]
    return nrt


def call_noalloc(nrt_gpu, scene, rays, opts):
    import torch

    lm = nrt_gpu.lib_module
    n = rays[0].numel()
    out = {"patch": torch.full((n,), -7, dtype=torch.int32, device="cuda"),
           "t": torch.empty(n, dtype=torch.float32, device="cuda"),
           "u": torch.empty(n, dtype=torch.float32, device="cuda"),
           "v": torch.empty(n, dtype=torch.float32, device="cuda"),
           "iters": torch.empty(n, dtype=torch.int32, device="cuda")}
    r = lm.RaysC(*[C.c_void_p(a.data_ptr()) for a in rays])
    h = lm.HitsC(*[C.c_void_p(out[k].data_ptr()) for k in ("patch", "t", "u", "v", "iters")], None, None)
    st = nrt_gpu.lib().nrt_intersect_noalloc(scene.handle, C.byref(r), n, C.byref(opts), C.byref(h),
                                             C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, nrt_gpu.lib().nrt_last_error().decode()
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def assert_same(a, b):
    hit_a, hit_b = a["patch"] >= 0, b["patch"] >= 0
    assert (hit_a == hit_b).mean() >= 0.9999
    both = hit_a & hit_b
    same = both & (a["patch"] == b["patch"])
    assert same.sum() >= 0.999 * both.sum()
    for k in ("t", "u", "v", "iters"):
        assert np.array_equal(a[k][same], b[k][same]), k


def test_noalloc_matches_wavefront_twice(nrt_gpu):
    import torch

    from nrt import scenes

    sc = scenes.surfaces_grid_scene(16, seed=5, width=400, height=240, spp=2)  # 192,000 rays
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    cam_k = float(sc.camera.cam_k)
    for opts in [nrt_gpu.default_opts(fp64_final=1, cond_fp64=1e4, schedule=nrt_gpu.SCHED_WAVEFRONT),
                 nrt_gpu.reference_opts(hull_cull=1, schedule=nrt_gpu.SCHED_WAVEFRONT),
                 nrt_gpu.reference_opts(flat_threshold=2.0, cam_k=cam_k, schedule=nrt_gpu.SCHED_WAVEFRONT)]:
        ref = {k: v.cpu().numpy() for k, v in scene.intersect(rays, opts).items()}
        assert (ref["patch"] >= 0).mean() > 0.3
        first = call_noalloc(nrt_gpu, scene, rays, opts)
        free_before = torch.cuda.mem_get_info()[0]
        second = call_noalloc(nrt_gpu, scene, rays, opts)
        free_after = torch.cuda.mem_get_info()[0]
        assert free_after == free_before, (free_before, free_after)
        assert_same(ref, first)
        assert_same(ref, second)
