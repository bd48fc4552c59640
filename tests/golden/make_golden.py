"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs oracle/_ref/libnrt_ref_it{7,8}.so -- the reference's host-compilable
functions (getPatch, buildBVH, the camera, getRayPlanes, intersectBound,
biliniearRay, newtonRhapson), compiled from the reference sources by
``make -C oracle ref`` -- on small seeded scenes and stores inputs and outputs
as .npz files.  The tests then pin this project's oracle restatement against
these files without needing the reference at test time.

Usage (needs the reference sources at build time of oracle/_ref):
    NRT_REFERENCE=<reference checkout> make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "rt-nurbs_b200"))

import oracle as O  # noqa: E402
from nrt import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def small_mixed_scene():
    """Four surfaces of degree (2..5) with 9-12 point nets and random knots
    (multiplicity 1-2), placed side by side; 96x64 pixel-centre rays."""
    return scenes.surfaces_grid_scene(4, seed=11, width=96, height=64, spp=1, relief=0.4, deg_range=(2, 5),
                                      net_range=(9, 12), name="mixed4")


def fixture(scene, name):
    rec = {}
    P_parts = []
    for k, s in enumerate(scene.surfaces):
        cp, ranges = O.ref_decompose(s)
        rec[f"surf{k}_cp"] = s.cp
        rec[f"surf{k}_U"] = s.U
        rec[f"surf{k}_V"] = s.V
        rec[f"surf{k}_nmpq"] = np.array([s.n, s.m, s.p, s.q], np.int32)
        rec[f"surf{k}_patch_cp"] = cp
        rec[f"surf{k}_patch_ranges"] = ranges
        P_parts.append(cp)
    rec["n_surfaces"] = np.array(len(scene.surfaces), np.int32)
    # Patches as the oracle's flat set (the decomposition above is bit-exact with it).
    P = O.decompose_scene(scene.surfaces, f64=False)
    assert np.array_equal(np.concatenate(P_parts).view(np.uint32), P.cp.view(np.uint32))
    bvh = O.ref_build_bvh(P)
    rec["bvh_box"], rec["bvh_lf"], rec["bvh_cnt"], rec["bvh_order"] = bvh.box, bvh.lf, bvh.cnt, bvh.order
    cam = scene.camera
    rays = O.ref_camera_rays(cam)
    rec["camera"] = np.array(list(cam.eye) + list(cam.look) + list(cam.up) + [cam.fov_deg, cam.width, cam.height],
                             np.float64)
    for nm, arr in zip(("ox", "oy", "oz", "dx", "dy", "dz"), rays.arrays()):
        rec["ray_" + nm] = arr
    Pb = P.subset(bvh.order)
    delta = O.patch_delta(Pb)
    rec["delta_bvh_order"] = delta
    # Reference settings (bilinear guess, 7 iterations, eps 1e-4) and the
    # plain settings (midpoint, 8 iterations, eps 1e-6), flat-skip off; plus one
    # flat-skip run at 2 px so the skip branch has a fixture too.
    runs = [("ref", True, 1e-4, 7, 0.0), ("plain", False, 1e-6, 8, 0.0), ("flat2px", True, 1e-4, 7, 2.0)]
    for tag, bil, eps, it, flat in runs:
        h, t, u, v, g, nc, sc = O.ref_intersect(Pb, bvh, rays, bilinear_init=bil, eps=eps, iters=it, delta=delta,
                                                flat_threshold=flat, cam_k=cam.cam_k, geo=True)
        rec[f"{tag}_hit_slot"], rec[f"{tag}_t"], rec[f"{tag}_u"], rec[f"{tag}_v"] = h, t, u, v
        rec[f"{tag}_geo"] = g
        rec[f"{tag}_counts"] = np.array([nc, sc], np.int64)
        print(f"{name}/{tag}: {P.n} patches, {rays.n} rays, hit rate {np.mean(h >= 0):.4f}, newton {nc}, skip {sc}")
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **rec)


def main():
    if not (O.ref_available(7) and O.ref_available(8)):
        raise SystemExit("oracle/_ref not built: run `make -C oracle ref` where the reference sources exist")
    fixture(scenes.heightfield_scene(0, width=64, height=64), "heightfield")
    fixture(scenes.analytic_scene("torus", 96, 54), "torus")
    fixture(scenes.analytic_scene("sphere", 96, 54), "sphere")
    fixture(small_mixed_scene(), "mixed4")
    refine_fixture()


def refine_surfaces():
    """Surfaces and refinement constants of the refinement fixture: the exact
    torus and sphere at the reference's own sweep values, the height field, and
    one random mixed-degree surface with fewer v than u points."""
    rnd = scenes.random_surface(np.random.default_rng(4), (0.0, 0.0, 0.0), (2, 5), (9, 12), 0.4)
    return [("torus", scenes.torus_surface(), (1.0, 4.0, 16.0)), ("sphere", scenes.sphere_surface(), (2.0, 8.0)),
            ("heightfield", scenes.heightfield_scene(0).surfaces[0], (2.0, 4.0)), ("random", rnd, (4.0,))]


def refine_fixture():
    """The reference's curvature refinement (curvatureRefinementU then V) of each
    surface at each constant: refine.npz."""
    rec = {}
    for name, s, cs in refine_surfaces():
        rec[f"{name}_cp"], rec[f"{name}_U"], rec[f"{name}_V"] = s.cp, s.U, s.V
        rec[f"{name}_nmpq"] = np.array([s.n, s.m, s.p, s.q], np.int32)
        rec[f"{name}_C"] = np.array(cs, np.float32)
        for c in cs:
            cp, U, V, n, m = O.ref_refine(s, c)
            rec[f"{name}_C{c:g}_cp"], rec[f"{name}_C{c:g}_U"], rec[f"{name}_C{c:g}_V"] = cp, U, V
            rec[f"{name}_C{c:g}_nm"] = np.array([n, m], np.int32)
    np.savez_compressed(os.path.join(OUT, "refine.npz"), **rec)


if __name__ == "__main__":
    main()
