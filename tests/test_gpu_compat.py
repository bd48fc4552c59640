"""The reference's own C++ entry points served by libnrt.so (GPU).

oracle/_ref/compat_driver is a program compiled against the reference's
headers (src/gpu/intersect.h, src/gpu/generateRaysKernel.h) and linked against
rt-nurbs_b200/lib/libnrt.so; it follows the reference's benchmark
(src/core/benchmark.cpp:122-204): getPatch, buildBVH, managed copies of
nodes, patches, rebased control points and flatness, calculateRaysWrapper,
idx_interact preset to -1, calculateIntersectWrapper (twice: the second call
runs on the cached scene and must give the same bytes).  Its outputs are
compared with the reference's own outputs on the golden fixtures (its host
code, oracle/_ref, committed in tests/golden/):

  * rays: bit-identical to the reference camera's;
  * idx_interact[i] = i exactly where the pixel hits, -1 elsewhere; wo = -d;
  * against the reference's hits, with the reference's settings (flat-skip
    off, and at 2 px): hit/miss agreement >= 99.9 %, t within 1e-4 relative
    on >= 99.5 % of the rays both hit, (u, v) within 1e-3 on >= 99.5 % (the
    bilinear guess is decided by rounding noise, so a few rays take another
    root, as between the reference's own host and GPU builds).
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden_surfaces, load_golden

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "oracle", "_ref", "compat_driver")
FIXTURES = ["heightfield", "torus", "sphere", "mixed4"]
SI = np.dtype([("t_hit", "<f4"), ("wo", "<f4", 3), ("uv", "<f4", 2), ("dpdu", "<f4", 3), ("dpdv", "<f4", 3),
               ("dndu", "<f4", 3), ("dndv", "<f4", 3)])


@pytest.fixture(scope="module")
def driver():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(DRIVER):
        pytest.skip("oracle/_ref/compat_driver is built only where the reference sources are present")
    return DRIVER


def run_driver(drv, g, flat, tmp_path):
    cam = g["camera"]
    W, H = int(cam[10]), int(cam[11])
    inp, out = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        surfs = golden_surfaces(g)
        np.array([len(surfs)], np.int32).tofile(f)
        for s in surfs:
            np.array([s.n, s.m, s.p, s.q], np.int32).tofile(f)
            np.ascontiguousarray(s.cp, np.float32).tofile(f)
            np.ascontiguousarray(s.U, np.float32).tofile(f)
            np.ascontiguousarray(s.V, np.float32).tofile(f)
        cam[:10].astype(np.float32).tofile(f)
        np.array([W, H], np.int32).tofile(f)
        np.array([flat], np.float32).tofile(f)
        delta = g["delta_bvh_order"].astype(np.float32)
        np.array([delta.size], np.int32).tofile(f)
        delta.tofile(f)
    r = subprocess.run([drv, str(inp), str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr[-2000:])
    n = W * H
    raw = np.fromfile(out, np.uint8)
    at = 0

    def take(dtype, count):
        nonlocal at
        a = raw[at:at + np.dtype(dtype).itemsize * count].view(dtype)
        at += np.dtype(dtype).itemsize * count
        return a

    idx = take(np.int32, n)
    si = take(SI, n)
    rays = [take(np.float32, n) for _ in range(6)]
    counts = take(np.uint64, 2)
    n_patches = int(take(np.int32, 1)[0])
    return idx, si, rays, counts, n_patches, r.stderr


@pytest.mark.parametrize("name", FIXTURES)
def test_reference_program_links_and_matches(driver, name, tmp_path):
    g = load_golden(name)
    for tag, flat in (("ref", 0.0), ("flat2px", 2.0)):
        idx, si, rays, counts, n_patches, err = run_driver(driver, g, flat, tmp_path)
        n = idx.size
        assert n_patches == g["bvh_order"].size
        for k, a in zip(("ox", "oy", "oz", "dx", "dy", "dz"), rays):
            assert np.array_equal(a.view(np.uint32), g["ray_" + k].view(np.uint32)), k
        hit = idx != -1
        assert np.array_equal(idx[hit], np.nonzero(hit)[0]), "idx_interact must be the pixel index on a hit"
        d = np.stack(rays[3:], 1)
        assert np.array_equal(si["wo"][hit], -d[hit])
        ref_hit = g[f"{tag}_hit_slot"] >= 0
        agree = float((hit == ref_hit).mean())
        both = hit & ref_hit
        t_ref = g[f"{tag}_t"][both].astype(np.float64)
        rel = np.abs(si["t_hit"][both] - t_ref) / np.abs(t_ref)
        duv = np.maximum(np.abs(si["uv"][both, 0] - g[f"{tag}_u"][both]),
                         np.abs(si["uv"][both, 1] - g[f"{tag}_v"][both]))
        geo = g[f"{tag}_geo"][both]
        dp = np.abs(np.concatenate([si["dpdu"][both], si["dpdv"][both]], 1) - geo[:, 3:9])
        dp_rel = dp.max(1) / (np.abs(geo[:, 3:9]).max(1) + 1e-30)
        print(f"{name}/{tag}: hits {hit.mean():.4f}, agreement {agree:.5f}, t rel <= 1e-4 on "
              f"{(rel <= 1e-4).mean():.5f}, uv <= 1e-3 on {(duv <= 1e-3).mean():.5f}, newton {counts[0]}, "
              f"skips {counts[1]} (reference: {g[f'{tag}_counts'].tolist()})")
        assert agree >= 0.999, agree
        assert (rel <= 1e-4).mean() >= 0.995
        assert (duv <= 1e-3).mean() >= 0.995
        assert (dp_rel <= 1e-3).mean() >= 0.995
        assert counts[0] > 0
        if g[f"{tag}_counts"][1] > 0:
            assert counts[1] > 0, "flat-skip accepted nothing where the reference accepted guesses"
        else:
            assert counts[1] == 0
