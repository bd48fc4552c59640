"""CPU oracle of the learned-initial-guess MLP (TEST INFRASTRUCTURE ONLY).

12 -> 64 -> 64 -> 2 with SiLU, mean squared error on (u, v).  Computed in
float64 with the same BF16 rounding points as the CUDA kernels (operands of
every tensor-core product are rounded to bfloat16; accumulation, biases,
activations before rounding, and bias gradients stay in higher precision), so
the GPU forward pass and gradients can be checked tightly.

Parameter order (the C ABI's nrt_mlp_get_params): W1[64][12], b1[64],
W2[64][64], b2[64], W3[2][64], b3[2]; W[n][k] is the weight from input k to
output n.
"""
import numpy as np

N_IN, N_HID, N_OUT = 12, 64, 2
SIZES = [(N_HID, N_IN), (N_HID,), (N_HID, N_HID), (N_HID,), (N_OUT, N_HID), (N_OUT,)]
N_PARAMS = sum(int(np.prod(s)) for s in SIZES)


def bf16(x):
    """Round float64 values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(theta):
    out, at = [], 0
    for s in SIZES:
        k = int(np.prod(s))
        out.append(np.asarray(theta[at:at + k], np.float64).reshape(s))
        at += k
    return out


def pack(parts):
    return np.concatenate([np.asarray(p, np.float64).ravel() for p in parts])


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(theta, X, emulate=True):
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    Xb = r(X)
    Z1 = Xb @ r(W1).T + b1
    H1 = r(silu(Z1))
    Z2 = H1 @ r(W2).T + b2
    H2 = r(silu(Z2))
    Y = H2 @ r(W3).T + b3
    return Y, (Xb, Z1, H1, Z2, H2)


def loss_and_grad(theta, X, T, emulate=True):
    """Mean over rows of sum((Y - T)^2) and its gradient w.r.t. theta."""
    W1, b1, W2, b2, W3, b3 = unpack(theta)
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    B = X.shape[0]
    Y, (Xb, Z1, H1, Z2, H2) = forward(theta, X, emulate)
    loss = float(np.sum((Y - T) ** 2) / B)
    dY = 2.0 * (Y - T) / B
    dYb = r(dY)
    gW3 = dYb.T @ H2
    gb3 = dY.sum(0)
    dH2 = dYb @ r(W3)
    dZ2 = dH2 * dsilu(Z2)
    dZ2b = r(dZ2)
    gW2 = dZ2b.T @ H1
    gb2 = dZ2.sum(0)
    dH1 = dZ2b @ r(W2)
    dZ1 = dH1 * dsilu(Z1)
    dZ1b = r(dZ1)
    gW1 = dZ1b.T @ Xb
    gb1 = dZ1.sum(0)
    return loss, pack([gW1, gb1, gW2, gb2, gW3, gb3])


def adam_step(theta, m, v, g, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v
