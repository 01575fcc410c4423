"""FP64 NumPy restatement of the con2prim start-point network (test
infrastructure): the same layers, SiLU, loss weights and BF16 rounding
points as the device kernels, so that their forward pass and gradients can
be checked on the CPU."""
import numpy as np

W1, B1, W2, B2, W3, B3 = 0, 256, 320, 4416, 4480, 4672
LOSS_W = np.array([1.0, 4.0, 1.0])


def bf16(x):
    """Round float32 values to bfloat16 (nearest, ties to even), as float64."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P, rnd=True):
    r = bf16 if rnd else (lambda a: np.asarray(a, dtype=np.float64))
    P = np.asarray(P, dtype=np.float32 if rnd else np.float64)
    return (r(P[W1:B1]).reshape(64, 4), P[B1:W2].astype(np.float64),
            r(P[W2:B2]).reshape(64, 64), P[B2:W3].astype(np.float64),
            r(P[W3:B3]).reshape(3, 64), P[B3:B3 + 3].astype(np.float64))


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(P, X, rnd=True):
    """rnd=False drops the BF16 rounding (for finite-difference checks)."""
    r = bf16 if rnd else (lambda a: np.asarray(a, dtype=np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(P, rnd)
    x = r(X)
    z1 = x @ w1.T + b1
    h1 = r(silu(z1))
    z2 = h1 @ w2.T + b2
    h2 = r(silu(z2))
    y = h2 @ w3.T + b3
    return y, (x, z1, h1, z2, h2)


def loss_and_grad(P, X, Y, rnd=True):
    """Mean weighted squared error over the samples and its gradient (the
    rounding is straight-through, as in the device backward pass)."""
    w1, b1, w2, b2, w3, b3 = unpack(P, rnd)
    y, (x, z1, h1, z2, h2) = forward(P, X, rnd)
    n = len(X)
    e = y - np.asarray(Y, dtype=np.float64)
    loss = float((LOSS_W * e * e).sum() / n)
    dy = 2.0 * LOSS_W * e / n
    g = np.zeros(len(P))
    g[W3:B3] = (dy.T @ h2).reshape(-1)
    g[B3:B3 + 3] = dy.sum(0)
    dz2 = (dy @ w3) * silu_grad(z2)
    g[W2:B2] = (dz2.T @ h1).reshape(-1)
    g[B2:W3] = dz2.sum(0)
    dz1 = (dz2 @ w2) * silu_grad(z1)
    g[W1:B1] = (dz1.T @ x).reshape(-1)
    g[B1:W2] = dz1.sum(0)
    return loss, g
