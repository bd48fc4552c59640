"""Output stage: the PPM writer on the host (CPU), and on the GPU the
framebuffers of nrt_shade and the per-ray error measures of nrt_compare_hits
against numpy restatements of their definitions (hit mask exact; normal map
and errors within 1e-5)."""
import numpy as np
import pytest

from parity import to_numpy


@pytest.fixture(scope="module")
def nrt_mod():
    import nrt

    nrt.lib()
    return nrt


def test_write_ppm(nrt_mod, tmp_path):
    W, H = 7, 3
    rng = np.random.default_rng(0)
    r, g, b = (rng.uniform(-0.2, 1.2, W * H).astype(np.float32) for _ in range(3))
    path = tmp_path / "img.ppm"
    nrt_mod.write_ppm(path, W, H, r, g, b)
    data = path.read_bytes()
    head = b"P6\n7 3\n255\n"
    assert data.startswith(head) and len(data) == len(head) + 3 * W * H
    px = np.frombuffer(data[len(head):], np.uint8).reshape(-1, 3)
    want = (np.clip(np.stack([r, g, b], 1), 0, 1) * np.float32(255.999)).astype(np.uint8)
    assert np.array_equal(px, want)
    with pytest.raises(nrt_mod.NrtError):
        nrt_mod.write_ppm(tmp_path / "missing_dir" / "x.ppm", W, H, r, g, b)


@pytest.mark.gpu
def test_shade_and_compare(nrt_mod):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from nrt import scenes

    sc = scenes.heightfield_scene(0, 128, 96)
    scene = nrt_mod.Scene(sc.surfaces)
    rays = nrt_mod.camera_rays(sc.camera)
    hits = scene.intersect(rays, nrt_mod.default_opts(hull_cull=1, fp64_final=1), geom=True)
    h = to_numpy(hits)
    hit = h["patch"] >= 0
    r, g, b = (x.cpu().numpy() for x in nrt_mod.shade(hits, 0))
    assert np.array_equal(r, hit.astype(np.float32)) and not g.any() and not b.any()
    rgb = np.stack([x.cpu().numpy() for x in nrt_mod.shade(hits, 1)], 1)
    geo = h["geom"].astype(np.float64)
    nrm = np.cross(geo[:, 6:9], geo[:, 3:6])
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-300)
    want = np.where(hit[:, None], (nrm + 1) * 0.5, 0.0)
    assert np.abs(rgb - want).max() <= 1e-5
    # the other schedule: no error at all; a shifted hit set: the definition
    other = scene.intersect(rays, nrt_mod.default_opts(hull_cull=3, fp64_final=1, schedule=nrt_mod.SCHED_WAVEFRONT),
                            geom=True)
    cam_k = sc.camera.cam_k
    px, deg, mm = (x.cpu().numpy() for x in nrt_mod.compare_hits(rays, hits, other, cam_k))
    assert not mm.any() and np.nanmax(px) <= 1e-3 and np.nanmax(deg) <= 1e-3
    shifted = {k: v.clone() for k, v in hits.items()}
    shifted["t"] *= 1.001
    shifted["patch"][::50] = -1
    px, deg, mm = (x.cpu().numpy() for x in nrt_mod.compare_hits(rays, hits, shifted, cam_k))
    s = shifted["patch"].cpu().numpy() >= 0
    assert np.array_equal(mm.astype(bool), hit != s)
    both = hit & s
    d = np.stack([a.cpu().numpy() for a in rays[3:]], 1)
    want_px = np.abs(h["t"] * 0.001) * np.linalg.norm(d, axis=1) * cam_k / h["t"]
    assert np.allclose(px[both], want_px[both], rtol=1e-3, atol=1e-6)
    assert np.isnan(px[~both]).all() and np.nanmax(deg) <= 1e-3
