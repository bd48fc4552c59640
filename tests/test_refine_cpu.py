"""Curvature-driven refinement (nrt_refine_surface, host C++) against the
reference's own curvatureRefinementU / curvatureRefinementV
(src/math/nurbs.h:289-486): bit-exact control points and knots on the golden
fixture (tests/golden/refine.npz, made by tests/golden/make_golden.py from
oracle/_ref), and live against oracle/_ref over the reference's sweep of
constants where that library is built.  Knot insertion preserves the surface:
the refined surface evaluated in FP64 matches the original within 1e-5 (float
control points), and a constant <= 0 changes nothing."""
import numpy as np
import pytest

from conftest import load_golden


@pytest.fixture(scope="module")
def nrt_mod():
    import nrt

    nrt.lib()
    return nrt


def golden_refine_cases():
    from nrt.scenes import Surface

    g = load_golden("refine")
    names = sorted({k.split("_")[0] for k in g})
    for name in names:
        n, m, p, q = (int(x) for x in g[f"{name}_nmpq"])
        s = Surface(g[f"{name}_cp"], g[f"{name}_U"], g[f"{name}_V"], n, m, p, q)
        for c in g[f"{name}_C"]:
            yield name, s, float(c), g


def test_refine_bit_exact_vs_golden(nrt_mod):
    cases = list(golden_refine_cases())
    assert len(cases) == 8
    for name, s, c, g in cases:
        r = nrt_mod.refine(s, c)
        key = f"{name}_C{c:g}"
        assert (r.n, r.m) == tuple(int(x) for x in g[key + "_nm"]), key
        assert np.array_equal(r.cp.view(np.uint32), g[key + "_cp"].view(np.uint32)), key
        assert np.array_equal(r.U, g[key + "_U"]) and np.array_equal(r.V, g[key + "_V"]), key


def test_refine_live_vs_reference(nrt_mod, oracle_mod):
    from nrt import scenes

    if not oracle_mod.ref_available(7):
        pytest.skip("oracle/_ref not built")
    for s in (scenes.torus_surface(), scenes.sphere_surface(), scenes.heightfield_scene(3).surfaces[0]):
        for c in (1.0, 2.0, 4.0, 8.0, 16.0):
            r = nrt_mod.refine(s, c)
            cp, U, V, n, m = oracle_mod.ref_refine(s, c)
            assert (r.n, r.m) == (n, m)
            assert np.array_equal(r.cp.view(np.uint32), cp.view(np.uint32))
            assert np.array_equal(r.U, U) and np.array_equal(r.V, V)


def test_refine_preserves_surface(nrt_mod, oracle_mod):
    from nrt import scenes

    rng = np.random.default_rng(0)
    for s in (scenes.torus_surface(), scenes.heightfield_scene(0).surfaces[0]):
        r = nrt_mod.refine(s, 4.0)
        assert r.n > s.n and r.m > s.m
        for u, v in rng.uniform(0.0, 1.0, (50, 2)):
            a = oracle_mod.surface_point(s, float(u), float(v))
            b = oracle_mod.surface_point(r, float(u), float(v))
            assert np.abs(a - b).max() <= 1e-5 * (1 + np.abs(a).max())
        # more, smaller patches after refinement
        assert np.prod(nrt_mod.decompose(r)[2]) > np.prod(nrt_mod.decompose(s)[2])


def test_refine_zero_constant_is_identity(nrt_mod):
    from nrt import scenes

    s = scenes.torus_surface()
    for c in (0.0, -1.0):
        r = nrt_mod.refine(s, c)
        assert (r.n, r.m) == (s.n, s.m)
        assert np.array_equal(r.cp, s.cp) and np.array_equal(r.U, s.U) and np.array_equal(r.V, s.V)
