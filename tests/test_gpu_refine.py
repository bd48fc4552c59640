"""Curvature refinement on the GPU (nrt_refine_surface_device) against the
reference's own curvatureRefinementU / curvatureRefinementV
(src/math/nurbs.h:289-486): bit-exact control points and knots on the golden
fixture (tests/golden/refine.npz, made from oracle/_ref), equal to the host
refinement (nrt_refine_surface) on random nets refined to a few hundred
points per side, and
the size query of the entry point (outputs too small: sizes returned, nothing
written)."""
import ctypes as C
import time

import numpy as np
import pytest

from test_refine_cpu import golden_refine_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


def same_surface(a, b):
    return ((a.n, a.m) == (b.n, b.m) and np.array_equal(a.cp.view(np.uint32), b.cp.view(np.uint32))
            and np.array_equal(a.U.view(np.uint32), b.U.view(np.uint32))
            and np.array_equal(a.V.view(np.uint32), b.V.view(np.uint32)))


def test_device_refine_bit_exact_vs_golden(nrt_gpu):
    cases = list(golden_refine_cases())
    assert len(cases) == 8
    for name, s, c, g in cases:
        r = nrt_gpu.refine_device(s, c)
        key = f"{name}_C{c:g}"
        assert (r.n, r.m) == tuple(int(x) for x in g[key + "_nm"]), key
        assert np.array_equal(r.cp.view(np.uint32), g[key + "_cp"].view(np.uint32)), key
        assert np.array_equal(r.U, g[key + "_U"]) and np.array_equal(r.V, g[key + "_V"]), key


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_device_refine_equals_host_large(nrt_gpu, seed):
    from nrt import scenes

    rng = np.random.default_rng(seed)
    s = scenes.random_surface(rng, (0.0, 0.0, 0.0), (2, 5), (12, 16), 1.0)
    for c in (4.0, 12.0):  # refined nets of a few hundred points per side
        t0 = time.perf_counter()
        h = nrt_gpu.refine(s, c)
        t1 = time.perf_counter()
        d = nrt_gpu.refine_device(s, c)
        t2 = time.perf_counter()
        print(f"seed {seed} C {c:g}: {s.n + 1}x{s.m + 1} -> {h.n + 1}x{h.m + 1} points; host {1e3 * (t1 - t0):.1f} ms, "
              f"device {1e3 * (t2 - t1):.1f} ms (with its set-up and copies)")
        assert h.n > s.n and h.m > s.m
        assert same_surface(h, d), (seed, c)


def test_device_refine_size_query(nrt_gpu):
    from nrt import scenes

    s = scenes.heightfield_scene(0).surfaces[0]
    L = nrt_gpu.lib()
    st, keep = nrt_gpu.lib_module._surface_struct(s)
    n, m = C.c_int(-1), C.c_int(-1)
    rc = L.nrt_refine_surface_device(C.byref(st), 4.0, 0, None, 0, None, 0, None, 0, C.byref(n), C.byref(m))
    assert rc == 1 and (n.value, m.value) == (nrt_gpu.refine(s, 4.0).n, nrt_gpu.refine(s, 4.0).m)
    r = nrt_gpu.refine_device(s, 0.0)  # C <= 0: unchanged
    assert same_surface(r, s)
