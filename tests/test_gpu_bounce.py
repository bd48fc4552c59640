"""GPU bounce-ray generation (nrt_generate_bounce_rays) through the C ABI,
against a numpy restatement of its definition on the same hits.

Tolerances: compaction order exact (the hit rays in ray order); origins and
directions within 2e-5 absolute (float32 normal, square roots and the
hardware sine/cosine); every direction in the hemisphere of the normal that
faces the incoming ray; over ~100k bounces the mean cosine to the normal is
2/3 (cosine-weighted) within 0.01.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


def pcg(x):
    x = (x.astype(np.uint64) * 747796405 + 2891336453) & 0xFFFFFFFF
    w = (((x >> ((x >> 28) + 4)) ^ x) * 277803737) & 0xFFFFFFFF
    return ((w >> 22) ^ w) & 0xFFFFFFFF


def test_bounce_rays_match_definition(nrt_gpu):
    from nrt import scenes

    sc = scenes.surfaces_grid_scene(16, seed=5, width=320, height=180, spp=2)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    hits = scene.intersect(rays, nrt_gpu.default_opts(hull_cull=3, fp64_final=1, schedule=nrt_gpu.SCHED_WAVEFRONT),
                           geom=True)
    seed, offset = 1234, 1e-4
    out, src, m = nrt_gpu.bounce_rays(rays, hits, seed=seed, offset=offset)
    patch = hits["patch"].cpu().numpy()
    idx = np.nonzero(patch >= 0)[0]
    assert m == idx.size > 10000
    assert np.array_equal(src.cpu().numpy(), idx)
    g = hits["geom"].cpu().numpy()[idx].astype(np.float64)
    d_in = np.stack([a.cpu().numpy()[idx] for a in rays[3:]], 1).astype(np.float64)
    S, Su, Sv = g[:, 0:3], g[:, 3:6], g[:, 6:9]
    nrm = np.cross(Sv, Su)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    flip = np.sum(nrm * d_in, 1) > 0
    nrm[flip] *= -1
    sgn = np.where(nrm[:, 2] >= 0, 1.0, -1.0)
    a = -1.0 / (sgn + nrm[:, 2])
    b = nrm[:, 0] * nrm[:, 1] * a
    t1 = np.stack([1 + sgn * nrm[:, 0] ** 2 * a, sgn * b, -sgn * nrm[:, 0]], 1)
    t2 = np.stack([b, sgn + nrm[:, 1] ** 2 * a, -nrm[:, 1]], 1)
    h = pcg(np.uint64(seed) ^ pcg(idx.astype(np.uint64)))
    r1 = (h >> 8).astype(np.float64) / 16777216.0
    r2 = (pcg(h) >> 8).astype(np.float64) / 16777216.0
    rad, phi = np.sqrt(r1), 2 * np.pi * r2
    w = rad[:, None] * np.cos(phi)[:, None] * t1 + rad[:, None] * np.sin(phi)[:, None] * t2 + \
        np.sqrt(np.maximum(0, 1 - r1))[:, None] * nrm
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    o = S + offset * nrm
    got_o = np.stack([x.cpu().numpy() for x in out[:3]], 1)
    got_d = np.stack([x.cpu().numpy() for x in out[3:]], 1)
    assert np.abs(got_o - o).max() <= 2e-5
    assert np.abs(got_d - w).max() <= 2e-5
    cosn = np.sum(got_d * nrm, 1)
    assert cosn.min() >= -1e-6
    assert abs(cosn.mean() - 2.0 / 3.0) <= 0.01, cosn.mean()
    # the bounce batch intersects like any other
    hb = scene.intersect(out, nrt_gpu.default_opts(hull_cull=3, schedule=nrt_gpu.SCHED_WAVEFRONT))
    assert (hb["patch"] >= 0).float().mean().item() > 0.05
