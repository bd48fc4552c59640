"""Parity of the timed configurations against the FP64 oracle, at the sizes
the bench times them (through the C ABI).

  * the bench workload: 64 surfaces of degree 2-5 (13,078 Bezier patches),
    1920x1080x4 = 8,294,400 rays, the bench's options (wavefront, oriented-box
    cull, FP64 escalation and final step); every 16th ray (518,400) is traced
    by the FP64 oracle (the same method in double, OpenMP);
  * the batched-wavefront scene: 256 surfaces (52,936 patches), 2048x2048x4 =
    2^24 primary rays, then the depth-1 cosine-weighted bounce rays of every
    hit; every 32nd primary ray and every 24th bounce ray against the oracle;
  * the learned-init wavefront on the bench workload (the committed network,
    two evaluations from its guess before the plain fallback), same sample.

Tolerance (the stated target): hit/miss agreement >= 99.99 % with the FP64
oracle; the same root (same patch, coinciding exact roots) on >= 99.9 % of
the rays both hit; every reported hit a genuine root (>= 99.99 % refine to
one) with relative t error <= 1e-4 against that exact root (or an absolute
error within one FP32 ulp of the ray origin's largest coordinate, the finest
the hit point o + t d can be stored: bounce rays that reach the next patch of
a crease end at t ~ 1e-6 of their origin), and (u, v) within
1e-4 at the 99.9th percentile.  t is measured against the exact root, not
against the oracle's own t: the oracle stops at |r1|+|r2| < 1e-6, which on a
short or grazing ray is more than 1e-4 of t.  The t bound holds for every hit
whose ray crosses the surface at more than 0.6 degrees (|cos| >= 1e-2 between
ray and normal); at near-tangent crossings t is ill-conditioned (two crossings
merge; even the FP64 exact root is only good to the square root of its
residual there), so those are counted, at most 2e-5 of the hits above 1e-4,
and the 99.99th percentile over all hits stays <= 1e-4.
"""
import numpy as np
import pytest

from parity import compare, crossing_cos, root_stats, to_numpy

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


def bench_opts(nrt_gpu, **kw):
    return nrt_gpu.default_opts(hull_cull=3, fp64_final=1, cond_fp64=1e4, schedule=nrt_gpu.SCHED_WAVEFRONT, **kw)


def oracle_scene(oracle_mod, surfaces):
    P = oracle_mod.decompose_scene(surfaces, f64=False)
    P.cp64 = P.cp.astype(np.float64)  # the oracle runs the same (float) patches in double
    return P, oracle_mod.build_bvh_binned(oracle_mod.patch_boxes(P))


def check_sample(oracle_mod, P, bvh, rays_np, got, idx, label):
    sub_np = [np.ascontiguousarray(a[idx]) for a in rays_np]
    ref = oracle_mod.intersect(P, bvh, oracle_mod.Rays(*sub_np), 0, 8, 1e-6, f64=True)
    g = {k: v[idx] for k, v in got.items() if k in ("patch", "t", "u", "v")}
    st = compare(g, ref.patch, ref.t, ref.u, ref.v)
    st.update(root_stats(oracle_mod, P, sub_np, g, ref, crossing_cos(sub_np, got["geom"][idx])))
    print(label, {k: (round(v, 8) if isinstance(v, float) else v) for k, v in st.items()})
    assert st["hit_rate"] > 0.2, st
    assert st["agree"] >= 0.9999, st
    assert st["same_root"] >= 0.999, st
    assert st["genuine"] >= 0.9999, st
    assert st["t_err_max"] <= 1e-4, st
    assert st["t_err_tangent"] <= 2e-5 * st["both"] and st["t_err_p9999"] <= 1e-4, st
    assert st["uv_err_p999"] <= 1e-4, st
    return st


def test_bench_workload_vs_fp64(nrt_gpu, oracle_mod):
    from nrt import learned, scenes

    sc = scenes.mixed_degree_scene(1)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    n = rays[0].numel()
    assert n == 1920 * 1080 * 4
    rays_np = [a.cpu().numpy() for a in rays]
    P, bvh = oracle_scene(oracle_mod, sc.surfaces)
    idx = np.arange(0, n, 16)
    got = to_numpy(scene.intersect(rays, bench_opts(nrt_gpu), geom=True, extra=False))
    check_sample(oracle_mod, P, bvh, rays_np, got, idx, "bench workload, plain-init wavefront:")
    mlp, _ = learned.load_or_train()
    scene.set_mlp(mlp)
    got_l = to_numpy(scene.intersect(rays, bench_opts(nrt_gpu, init_mode=nrt_gpu.INIT_LEARNED, learned_iters=2),
                                     geom=True, extra=False))
    check_sample(oracle_mod, P, bvh, rays_np, got_l, idx, "bench workload, learned-init wavefront:")
    scene.close()


def test_batched_scene_and_bounces_vs_fp64(nrt_gpu, oracle_mod):
    import torch

    from nrt import scenes

    sc = scenes.wavefront_scene(3)
    scene = nrt_gpu.Scene(sc.surfaces)
    rays = nrt_gpu.camera_rays(sc.camera)
    n = rays[0].numel()
    assert n == 1 << 24
    out = scene.intersect(rays, bench_opts(nrt_gpu), geom=True, extra=False)
    got = to_numpy(out)
    P, bvh = oracle_scene(oracle_mod, sc.surfaces)
    rays_np = [a.cpu().numpy() for a in rays]
    check_sample(oracle_mod, P, bvh, rays_np, got, np.arange(0, n, 32), "256 surfaces, primary rays:")
    del rays_np
    b_rays, _, m = nrt_gpu.bounce_rays(rays, out, seed=17, offset=1e-4)
    assert m > 0.3 * n
    b_out = to_numpy(scene.intersect(b_rays, bench_opts(nrt_gpu), geom=True, extra=False))
    b_np = [a.cpu().numpy() for a in b_rays]
    torch.cuda.synchronize()
    check_sample(oracle_mod, P, bvh, b_np, b_out, np.arange(0, m, 24), "256 surfaces, depth-1 bounces:")
    scene.close()
