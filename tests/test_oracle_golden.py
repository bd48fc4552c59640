"""Pin the oracle restatement against the reference's own outputs.

The fixtures in tests/golden/ were produced by the reference's own code
(tests/golden/make_golden.py runs oracle/_ref).  Decomposition, BVH and the
FP32 traversal+Newton must reproduce them bit for bit; the closed-form camera
agrees with the reference's matrix camera to a few ulps.
"""
import numpy as np
import pytest

from conftest import golden_rays, golden_surfaces, load_golden

FIXTURES = ["heightfield", "torus", "sphere", "mixed4"]


@pytest.mark.parametrize("name", FIXTURES)
def test_decomposition_bit_exact(oracle_mod, name):
    g = load_golden(name)
    for k, s in enumerate(golden_surfaces(g)):
        cp, cp64, ranges, _ = oracle_mod.decompose(s)
        assert np.array_equal(cp.view(np.uint32), g[f"surf{k}_patch_cp"].view(np.uint32))
        assert np.array_equal(ranges, g[f"surf{k}_patch_ranges"])
        # the FP64 decomposition is the same surface to float rounding
        scale = np.abs(cp).max()
        assert np.abs(cp64 - cp).max() <= 4e-6 * scale


@pytest.mark.parametrize("name", FIXTURES)
def test_bvh_bit_exact(oracle_mod, name):
    g = load_golden(name)
    P = oracle_mod.decompose_scene(golden_surfaces(g), f64=False)
    bvh = oracle_mod.build_bvh(oracle_mod.patch_boxes(P))
    M = g["bvh_box"].shape[0]
    assert np.array_equal(bvh.box[:M], g["bvh_box"])
    assert np.array_equal(bvh.lf[:M], g["bvh_lf"])
    assert np.array_equal(bvh.cnt[:M], g["bvh_cnt"])
    assert np.array_equal(bvh.order, g["bvh_order"])


@pytest.mark.parametrize("name", FIXTURES)
def test_camera_rays_close(oracle_mod, name):
    from nrt.scenes import Camera

    g = load_golden(name)
    c = g["camera"]
    cam = Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), int(c[10]), int(c[11]))
    mine = oracle_mod.camera_rays(cam)
    ref = golden_rays(g)
    for a, b in zip(mine.arrays(), ref.arrays()):
        assert np.abs(a - b).max() <= 4e-7


@pytest.mark.parametrize("name", FIXTURES)
@pytest.mark.parametrize("tag,init,eps,iters,flat", [("ref", 1, 1e-4, 7, 0.0), ("plain", 0, 1e-6, 8, 0.0),
                                                     ("flat2px", 1, 1e-4, 7, 2.0)])
def test_intersect_bit_exact(oracle_mod, name, tag, init, eps, iters, flat):
    g = load_golden(name)
    P = oracle_mod.decompose_scene(golden_surfaces(g), f64=False)
    bvh = oracle_mod.BinaryBVH(g["bvh_box"], g["bvh_lf"], g["bvh_cnt"], g["bvh_order"], g["bvh_box"].shape[0])
    rays = golden_rays(g)
    c = g["camera"]
    cam_k = 0.5 * c[11] / np.tan(np.radians(c[9]) / 2.0)
    # the oracle indexes delta by BVH slot, like the reference (intersect.cu:104)
    H = oracle_mod.intersect(P, bvh, rays, init_mode=init, max_iter=iters, eps=eps, delta=g["delta_bvh_order"],
                             flat_threshold=flat, cam_k=cam_k, geo=True)
    slot = g[f"{tag}_hit_slot"]
    ref_patch = np.where(slot >= 0, bvh.order[np.maximum(slot, 0)], -1)
    assert np.array_equal(H.patch, ref_patch)
    hit = slot >= 0
    assert np.array_equal(H.t[hit].view(np.uint32), g[f"{tag}_t"][hit].view(np.uint32))
    assert np.array_equal(H.u[hit], g[f"{tag}_u"][hit])
    assert np.array_equal(H.v[hit], g[f"{tag}_v"][hit])
    assert np.array_equal(H.geo[hit], g[f"{tag}_geo"][hit])
    assert (H.newton_total, H.skip_total) == tuple(int(x) for x in g[f"{tag}_counts"])


@pytest.mark.parametrize("name", ["heightfield", "mixed4"])
def test_decomposition_preserves_surface(oracle_mod, name):
    """Each Bezier patch evaluated at local (s,t) equals the NURBS surface at the
    mapped global parameter (Algorithm A4.3, nurbs.h:66-92)."""
    g = load_golden(name)
    rng = np.random.default_rng(5)
    for s in golden_surfaces(g):
        cp, cp64, ranges, (nu, nv) = oracle_mod.decompose(s)
        piece = (s.p + 1) * (s.q + 1)
        for k in rng.choice(nu * nv, size=min(8, nu * nv), replace=False):
            u0, u1, v0, v1 = (float(x) for x in ranges[k])
            for _ in range(4):
                a, b = rng.uniform(0, 1, 2)
                H = oracle_mod.patch_eval_f64(cp64[k * piece:(k + 1) * piece], s.p, s.q, a, b)[0]
                P = H[:3] / H[3]
                Q = oracle_mod.surface_point(s, u0 + a * (u1 - u0), v0 + b * (v1 - v0))
                assert np.abs(P - Q).max() < 1e-10 * max(1.0, np.abs(Q).max())
