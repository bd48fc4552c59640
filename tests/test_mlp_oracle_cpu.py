"""The MLP's CPU oracle (oracle/mlp_oracle.py) against finite differences, and
its parameter layout against the C ABI's."""
import numpy as np

from oracle import mlp_oracle as M


def test_param_count_matches_abi():
    import nrt

    assert M.N_PARAMS == int(nrt.lib().nrt_mlp_param_count()) == 5122


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    theta = rng.normal(0, 0.3, M.N_PARAMS)
    X = rng.normal(0, 1, (16, 12))
    T = rng.uniform(0, 1, (16, 2))
    loss, g = M.loss_and_grad(theta, X, T, emulate=False)
    idx = rng.choice(M.N_PARAMS, 60, replace=False)
    h = 1e-6
    for k in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (M.loss_and_grad(tp, X, T, emulate=False)[0] - M.loss_and_grad(tm, X, T, emulate=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, g[k])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005, 3.1415926, -2.5e-3, 65504.0])
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even
    assert r[2] == 1.0078125
    assert abs(r[3] - 3.140625) < 1e-12
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8)
