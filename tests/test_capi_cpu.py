"""C-ABI checks that need no GPU: the library loads, exports every symbol of
include/nrt.h, and its host-side pipeline (decomposition, patch bounds, BVH
builders) matches the reference's outputs in the golden fixtures."""
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden_surfaces, load_golden

FIXTURES = ["heightfield", "torus", "sphere", "mixed4"]


@pytest.fixture(scope="module")
def nrt_mod():
    import nrt

    nrt.lib()
    return nrt


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "nrt.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(nrt_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header(nrt_mod):
    import ctypes

    L = ctypes.CDLL(nrt_mod.lib_path())
    syms = header_symbols()
    assert len(syms) >= 15
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


# The reference's C++ entry points (include/nrt_compat.h) under their mangled
# names, as the reference's own declarations (src/gpu/intersect.h:9-13,
# src/gpu/generateRaysKernel.h:6) name them.
COMPAT_SYMBOLS = [
    "_Z25calculateIntersectWrapperRN8SoAQueue9ray_queueEP7BVHNodeP11bezierPatchP18surfaceInteractioniiffPfPyS9_",
    "_Z20calculateRaysWrapperRN8SoAQueue9ray_queueE10projectionR13camera_config",
]


def test_library_exports_reference_entry_points(nrt_mod):
    """libnrt.so defines the reference's two C++ entry points; where the program
    built on the reference's own headers exists (oracle/_ref/compat_driver), the
    symbols it needs are exactly these."""
    import ctypes
    import subprocess

    L = ctypes.CDLL(nrt_mod.lib_path())
    assert all(hasattr(L, s) for s in COMPAT_SYMBOLS)
    drv = os.path.join(ROOT, "oracle", "_ref", "compat_driver")
    if os.path.exists(drv):
        undef = subprocess.run(["nm", "-u", drv], capture_output=True, text=True, check=True).stdout
        wanted = sorted(w for w in undef.split() if "Wrapper" in w)
        assert wanted == sorted(COMPAT_SYMBOLS), wanted


def test_version_and_opts(nrt_mod):
    assert b"nrt" in nrt_mod.lib().nrt_version()
    d = nrt_mod.default_opts()
    assert (d.init_mode, d.max_iter, d.eps, d.hull_cull) == (0, 8, np.float32(1e-6), 0)
    r = nrt_mod.reference_opts()
    assert (r.init_mode, r.max_iter, r.eps) == (1, 7, np.float32(1e-4))


@pytest.mark.parametrize("name", FIXTURES)
def test_decompose_bit_exact_vs_reference(nrt_mod, name):
    g = load_golden(name)
    for k, s in enumerate(golden_surfaces(g)):
        cp, ranges, _ = nrt_mod.decompose(s)
        assert np.array_equal(cp.view(np.uint32), g[f"surf{k}_patch_cp"].view(np.uint32))
        assert np.array_equal(ranges, g[f"surf{k}_patch_ranges"])


def test_decompose_high_degree(nrt_mod, oracle_mod):
    """Degrees above the reference's cap of 4 (up to 7) decompose and agree
    with the oracle restatement bit for bit."""
    from nrt import scenes

    for p, q in [(5, 5), (7, 6), (6, 7), (7, 7), (1, 7), (2, 1)]:
        rng = np.random.default_rng(p * 10 + q)
        n, m = p + 5, q + 4
        cp = np.empty(((n + 1) * (m + 1), 4), np.float32)
        cp[:, :3] = rng.normal(size=((n + 1) * (m + 1), 3))
        cp[:, 3] = rng.uniform(0.5, 2.0, (n + 1) * (m + 1))
        cp[:, :3] *= cp[:, 3:]
        s = scenes.Surface(cp, scenes._random_knots(rng, n, p), scenes._random_knots(rng, m, q), n, m, p, q)
        cpn, ranges, (nu, nv) = nrt_mod.decompose(s)
        ocp, _, orng, (onu, onv) = oracle_mod.decompose(s, f64=False)
        assert (nu, nv) == (onu, onv) and nu * nv > 1
        assert np.array_equal(cpn.view(np.uint32), ocp.view(np.uint32))
        assert np.array_equal(ranges, orng)


@pytest.mark.parametrize("name", FIXTURES)
def test_bounds_and_exact_bvh_vs_reference(nrt_mod, oracle_mod, name):
    g = load_golden(name)
    P = oracle_mod.decompose_scene(golden_surfaces(g), f64=False)
    boxes = nrt_mod.patch_bounds(P.cp, P.off, P.deg)
    assert np.array_equal(boxes, oracle_mod.patch_boxes(P))
    nb, lf, cnt, order, used = nrt_mod.build_bvh_binary(boxes, nrt_mod.BVH_EXACT_SAH)
    M = g["bvh_box"].shape[0]
    assert np.array_equal(nb[:M], g["bvh_box"])
    assert np.array_equal(lf[:M], g["bvh_lf"])
    assert np.array_equal(cnt[:M], g["bvh_cnt"])
    assert np.array_equal(order, g["bvh_order"])


def _check_bvh_invariants(nb, lf, cnt, order, used, boxes):
    N = boxes.shape[0]
    assert sorted(order.tolist()) == list(range(N))
    seen = np.zeros(N, bool)
    stack = [0]
    while stack:
        i = stack.pop()
        if cnt[i] > 0:
            for s in range(lf[i], lf[i] + cnt[i]):
                seen[s] = True
                b = boxes[order[s]]
                assert np.all(nb[i, :3] <= b[:3]) and np.all(nb[i, 3:] >= b[3:])
        else:
            for c in (lf[i], lf[i] + 1):
                assert c < used
                assert np.all(nb[i, :3] <= nb[c, :3]) and np.all(nb[i, 3:] >= nb[c, 3:])
                stack.append(c)
    assert seen.all()


def test_binned_bvh_invariants(nrt_mod, oracle_mod):
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(8, seed=2, width=8, height=8, spp=1)
    P = oracle_mod.decompose_scene(sc.surfaces, f64=False)
    boxes = nrt_mod.patch_bounds(P.cp, P.off, P.deg)
    _check_bvh_invariants(*nrt_mod.build_bvh_binary(boxes, nrt_mod.BVH_BINNED_SAH), boxes)
    _check_bvh_invariants(*nrt_mod.build_bvh_binary(boxes[:1], nrt_mod.BVH_BINNED_SAH), boxes[:1])
    # identical boxes cannot be split
    same = np.repeat(boxes[:1], 5, axis=0)
    nb, lf, cnt, order, used = nrt_mod.build_bvh_binary(same, nrt_mod.BVH_BINNED_SAH)
    assert used == 1 and cnt[0] == 5


def test_invalid_inputs_report_errors(nrt_mod):
    from nrt import scenes

    s = scenes.heightfield_scene().surfaces[0]
    bad = scenes.Surface(s.cp, s.U, s.V, s.n, s.m, 9, s.q)
    with pytest.raises(nrt_mod.NrtError, match="degree"):
        nrt_mod.decompose(bad)
    U = s.U.copy()
    U[5], U[6] = U[6], U[5] + 0.5
    with pytest.raises(nrt_mod.NrtError, match="non-decreasing"):
        nrt_mod.decompose(scenes.Surface(s.cp, U, s.V, s.n, s.m, s.p, s.q))
    U = s.U.copy()
    U[s.p] = 0.5 * U[s.p + 1]
    with pytest.raises(nrt_mod.NrtError, match="clamped"):
        nrt_mod.decompose(scenes.Surface(s.cp, U, s.V, s.n, s.m, s.p, s.q))
    assert nrt_mod.lib().nrt_decompose(None, None, None, None, None) == 1


def _binned_sah_restated(boxes, max_leaf=1):
    """The 32-bin SAH as the builders define it (csrc/scene_math.h), restated
    in numpy float32, one rounding per operation: centroid bounds, bins per
    axis with a positive extent, cost nL*halfArea(L) + nR*halfArea(R) with the
    first minimum in (axis, bin) order, a stable partition, children numbered
    as a depth-first stack allocates them."""
    f = np.float32
    N = boxes.shape[0]
    lo, hi = boxes[:, :3].astype(f), boxes[:, 3:].astype(f)
    cen = (f(0.5) * (lo + hi)).astype(f)

    def half_area(b_lo, b_hi):
        ex, ey, ez = f(b_hi[0] - b_lo[0]), f(b_hi[1] - b_lo[1]), f(b_hi[2] - b_lo[2])
        return f(f(f(ex * ey) + f(ey * ez)) + f(ez * ex))

    def sah_bin(c, l, s):
        v = f(f(c - l) * s)
        return (int(v) if v < f(32) else 31) if v >= f(0) else 0

    M = 2 * N - 1
    nb = np.zeros((M, 6), f)
    lf = np.zeros(M, np.uint32)
    cnt = np.zeros(M, np.uint32)
    order = np.arange(N, dtype=np.int32)
    nb[0, :3], nb[0, 3:] = lo.min(0), hi.max(0)
    cnt[0] = N
    used, todo = 1, [0]
    while todo:
        node = todo.pop()
        first, count = int(lf[node]), int(cnt[node])
        if count <= max_leaf:
            continue
        ids = order[first:first + count]
        clo, chi = cen[ids].min(0), cen[ids].max(0)
        ext = (chi - clo).astype(f)
        scale = [f(f(32) / ext[a]) if ext[a] > 0 else f(0) for a in range(3)]
        best = (np.inf, -1, 0)
        bins = {}
        for a in range(3):
            if not ext[a] > 0:
                continue
            bl = np.full((32, 3), np.inf, f); bh = np.full((32, 3), -np.inf, f); bc = np.zeros(32, int)
            for i in ids:
                b = sah_bin(cen[i, a], clo[a], scale[a])
                bc[b] += 1; bl[b] = np.minimum(bl[b], lo[i]); bh[b] = np.maximum(bh[b], hi[i])
            bins[a] = (bl, bh, bc)
            rlo, rhi, n = np.full(3, np.inf, f), np.full(3, -np.inf, f), 0
            ra, rc = [None] * 32, [0] * 32
            for k in range(31, 0, -1):
                rlo, rhi, n = np.minimum(rlo, bl[k]), np.maximum(rhi, bh[k]), n + bc[k]
                ra[k], rc[k] = half_area(rlo, rhi), n
            llo, lhi, n = np.full(3, np.inf, f), np.full(3, -np.inf, f), 0
            for k in range(31):
                llo, lhi, n = np.minimum(llo, bl[k]), np.maximum(lhi, bh[k]), n + bc[k]
                if n == 0 or rc[k + 1] == 0:
                    continue
                c = f(f(f(n) * half_area(llo, lhi)) + f(f(rc[k + 1]) * ra[k + 1]))
                if c < best[0]:
                    best = (c, a, k + 1)
        _, axis, split = best
        if axis < 0:
            continue
        left = np.array([sah_bin(cen[i, axis], clo[axis], scale[axis]) < split for i in ids])
        nl = int(left.sum())
        if nl == 0 or nl == count:
            continue
        order[first:first + count] = np.concatenate([ids[left], ids[~left]])
        L, R = used, used + 1
        used += 2
        bl, bh, _ = bins[axis]
        lf[L], cnt[L], lf[R], cnt[R] = first, nl, first + nl, count - nl
        nb[L] = np.concatenate([bl[:split].min(0), bh[:split].max(0)])
        nb[R] = np.concatenate([bl[split:].min(0), bh[split:].max(0)])
        lf[node], cnt[node] = L, 0
        todo += [L, R]
    return nb, lf, cnt, order, used


@pytest.mark.parametrize("n_surfaces,seed", [(3, 4), (8, 2)])
def test_binned_bvh_matches_restatement(nrt_mod, oracle_mod, n_surfaces, seed):
    """The host binned builder equals the numpy restatement node for node and
    slot for slot (the device builder is compared with the host builder on
    the GPU, byte for byte), and so does the oracle's C builder that the
    reference arm of the bench uses."""
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(n_surfaces, seed=seed, width=8, height=8, spp=1)
    P = oracle_mod.decompose_scene(sc.surfaces, f64=False)
    boxes = nrt_mod.patch_bounds(P.cp, P.off, P.deg)
    got = nrt_mod.build_bvh_binary(boxes, nrt_mod.BVH_BINNED_SAH)
    ref = _binned_sah_restated(boxes)
    assert got[4] == ref[4]
    used = got[4]
    assert np.array_equal(got[3], ref[3])
    assert np.array_equal(got[1][:used], ref[1][:used]) and np.array_equal(got[2][:used], ref[2][:used])
    assert np.array_equal(got[0][:used], ref[0][:used])
    orc = oracle_mod.build_bvh_binned(oracle_mod.patch_boxes(P))
    assert orc.used == used and np.array_equal(orc.order, ref[3])
    assert np.array_equal(orc.lf[:used], ref[1][:used]) and np.array_equal(orc.cnt[:used], ref[2][:used])
    assert np.array_equal(orc.box[:used], ref[0][:used])


def test_ctypes_mirrors_match_header(tmp_path):
    """Every struct of include/nrt.h that the ctypes binding (nrt/lib.py)
    mirrors has the same size and the same field offsets: a C program built on
    the header with the system compiler prints sizeof and offsetof for each
    mirrored field.  A field added on one side only would make the library
    read or write past the caller's struct."""
    import ctypes
    import shutil
    import subprocess

    from nrt import lib_module as L

    if not shutil.which("gcc"):
        pytest.skip("no C compiler")
    mirrors = {"nrt_nurbs_surface": L.NurbsSurface, "nrt_build_opts": L.BuildOpts, "nrt_scene_info": L.SceneInfo,
               "nrt_rays": L.RaysC, "nrt_hits": L.HitsC, "nrt_intersect_opts": L.IntersectOpts,
               "nrt_wavefront_tuning": L.Tuning, "nrt_counters": L.Counters, "nrt_train_opts": L.TrainOpts,
               "nrt_camera": L.CameraC}
    src = ["#include <stdio.h>", "#include <stddef.h>", '#include "nrt.h"', "int main(void) {"]
    for cname, cls in mirrors.items():
        src.append(f'printf("{cname} . %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            src.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src += ["return 0;", "}"]
    c_file, exe = tmp_path / "layout.c", tmp_path / "layout"
    c_file.write_text("\n".join(src) + "\n")
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(c_file)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, field, value = line.split()
        got[(cname, field)] = int(value)
    for cname, cls in mirrors.items():
        assert got[(cname, ".")] == ctypes.sizeof(cls), (cname, got[(cname, ".")], ctypes.sizeof(cls))
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)
