"""GPU tests of the learned initial guess (hand-written BF16 tensor-core MLP).

Tolerances:
  * forward pass against the CPU oracle with the same BF16 rounding points:
    |y_gpu - y_oracle| <= 2e-2 * (1 + |y|) (FP32 vs FP64 accumulation and the
    hardware tanh of the inference SiLU may move an activation by one BF16 step);
  * gradients: ||g_gpu - g_oracle|| <= 2e-2 ||g_oracle||, and every
    component within 5e-2 * max|g| of the oracle;
  * training on plain-Newton pairs collected on smooth height-field surfaces
    (where the features determine the root well) lowers the loss at least 3x;
  * the learned guess (with plain Newton as the fallback) keeps hit/miss
    agreement with the FP64 oracle >= 99.9% and needs fewer Newton evaluations
    per converged solve than the midpoint guess.
"""
import numpy as np
import pytest

from parity import compare, to_numpy

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nrt_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nrt

    nrt.lib()
    return nrt


@pytest.fixture(scope="module")
def mlp_oracle():
    from oracle import mlp_oracle

    return mlp_oracle


def random_theta(rng, M):
    theta = np.zeros(M.N_PARAMS)
    W1, b1, W2, b2, W3, b3 = M.unpack(np.arange(M.N_PARAMS))
    parts = [rng.normal(0, 0.4, (64, 12)), rng.normal(0, 0.1, 64), rng.normal(0, 0.15, (64, 64)),
             rng.normal(0, 0.1, 64), rng.normal(0, 0.15, (2, 64)), rng.normal(0.5, 0.1, 2)]
    return M.pack(parts).astype(np.float32)


def test_forward_matches_oracle(nrt_gpu, mlp_oracle):
    import torch

    rng = np.random.default_rng(1)
    theta = random_theta(rng, mlp_oracle)
    mlp = nrt_gpu.Mlp(seed=3)
    mlp.set_params(theta)
    assert np.array_equal(mlp.params(), theta)
    X = rng.uniform(-2, 2, (1000, 12)).astype(np.float32)
    y = mlp.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    ref, _ = mlp_oracle.forward(theta.astype(np.float64), X.astype(np.float64))
    assert np.all(np.abs(y - ref) <= 2e-2 * (1 + np.abs(ref))), np.abs(y - ref).max()
    assert np.abs(y - ref).mean() < 2e-3


def test_gradients_match_oracle(nrt_gpu, mlp_oracle):
    import torch

    rng = np.random.default_rng(2)
    theta = random_theta(rng, mlp_oracle)
    mlp = nrt_gpu.Mlp(seed=4)
    mlp.set_params(theta)
    for n in (32, 517):
        X = rng.uniform(-2, 2, (n, 12)).astype(np.float32)
        T = rng.uniform(0, 1, (n, 2)).astype(np.float32)
        loss, g = mlp.gradients(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
        ref_loss, ref = mlp_oracle.loss_and_grad(theta.astype(np.float64), X.astype(np.float64), T.astype(np.float64))
        assert abs(loss - ref_loss) <= 1e-2 * ref_loss
        assert np.linalg.norm(g - ref) <= 2e-2 * np.linalg.norm(ref)
        assert np.all(np.abs(g - ref) <= 5e-2 * np.abs(ref).max())


def test_train_save_load(nrt_gpu, tmp_path):
    import torch

    from nrt import scenes

    feats, targs = [], []
    for seed in (21, 22, 23, 24):
        sc = scenes.heightfield_scene(seed, 256, 256, 1)
        scene = nrt_gpu.Scene(sc.surfaces)
        rays = nrt_gpu.camera_rays(sc.camera)
        feat, targ, total = scene.collect_training_data(rays, nrt_gpu.default_opts(schedule=nrt_gpu.SCHED_WAVEFRONT),
                                                        capacity=32 * rays[0].numel())
        assert feat.shape[0] == total > 5000
        conv = targ[:, 0] >= 0  # converged solves; the others carry (-1, -1)
        assert torch.isfinite(feat).all() and conv.sum() > 5000
        assert ((targ[conv] >= 0) & (targ[conv] <= 1)).all() and (targ[~conv] == -1).all()
        feats.append(feat[conv])
        targs.append(targ[conv])
    feat, targ = torch.cat(feats).contiguous(), torch.cat(targs).contiguous()
    mlp = nrt_gpu.Mlp(seed=5)
    losses = mlp.train(feat, targ, epochs=12, batch=256, lr=1e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < losses[0] / 3, losses
    path = tmp_path / "init.mlp"
    mlp.save(path)
    back = nrt_gpu.Mlp.load(path)
    assert np.array_equal(back.params(), mlp.params())
    a = mlp.forward(feat[:2048]).cpu().numpy()
    b = back.forward(feat[:2048]).cpu().numpy()
    assert np.array_equal(a, b)
    raw = bytearray(path.read_bytes())
    raw[100] ^= 0xFF
    bad = tmp_path / "bad.mlp"
    bad.write_bytes(bytes(raw))
    with pytest.raises(nrt_gpu.NrtError, match="checksum"):
        nrt_gpu.Mlp.load(bad)


def test_learned_init_gain_and_agreement(nrt_gpu, oracle_mod):
    """Trained on height-field seeds 1..60, evaluated on the unseen seed 0: hit
    agreement with the FP64 oracle (plain method) stays, and converged solves
    need fewer Newton evaluations than from the midpoint guess."""
    from nrt import learned, scenes

    feat, targ = learned.collect(400_000, verbose=False,
                                 which=[scenes.heightfield_scene(s, 256, 256, 1) for s in range(1, 61)])
    mlp = nrt_gpu.Mlp(seed=6)
    mlp.train(feat, targ, epochs=20, batch=4096, lr=1e-3, seed=2)
    test = scenes.heightfield_scene(0, 512, 512, 1)
    scene = nrt_gpu.Scene(test.surfaces)
    scene.set_mlp(mlp)
    rays = nrt_gpu.camera_rays(test.camera)
    W = nrt_gpu.SCHED_WAVEFRONT
    plain = nrt_gpu.default_opts(hull_cull=2, schedule=W)
    learned_opts = nrt_gpu.default_opts(hull_cull=2, schedule=W, init_mode=nrt_gpu.INIT_LEARNED, learned_iters=6)
    scene.enable_counters(True)
    a = to_numpy(scene.intersect(rays, plain))
    b = to_numpy(scene.intersect(rays, learned_opts))
    cb = scene.counters()
    assert 0 < cb["learned_solves"] <= cb["newton_solves"]
    P = oracle_mod.decompose_scene(test.surfaces, f64=False)
    P.cp64 = P.cp.astype(np.float64)
    bvh = oracle_mod.build_bvh(oracle_mod.patch_boxes(P))
    r_np = oracle_mod.Rays(*[x.cpu().numpy() for x in rays])
    ref = oracle_mod.intersect(P, bvh, r_np, 0, 8, 1e-6, f64=True)
    st_plain = compare(a, ref.patch, ref.t, ref.u, ref.v)
    st_learn = compare(b, ref.patch, ref.t, ref.u, ref.v)
    assert st_plain["agree"] >= 0.9999, st_plain
    assert st_learn["agree"] >= 0.999, st_learn
    assert st_learn["t_rel_max"] <= 1e-4, st_learn
    plain_evals = a["iters"][a["patch"] >= 0].mean()
    learned_evals = b["iters"][b["patch"] >= 0].mean()
    assert learned_evals < 0.9 * plain_evals, (learned_evals, plain_evals)
