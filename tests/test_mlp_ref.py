"""The CPU restatement of the start-point network checks itself: its
backward pass against central finite differences (FP64, no rounding), and
its BF16 rounding against the definition."""
import numpy as np

import mlp_ref as M


def _params(rng):
    P = np.zeros(4675)
    P[M.W1:M.B1] = rng.normal(0, 0.5, 256)
    P[M.B1:M.W2] = rng.normal(0, 0.1, 64)
    P[M.W2:M.B2] = rng.normal(0, 0.15, 4096)
    P[M.B2:M.W3] = rng.normal(0, 0.1, 64)
    P[M.W3:M.B3] = rng.normal(0, 0.15, 192)
    P[M.B3:] = rng.normal(0, 0.1, 3)
    return P


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(5)
    P = _params(rng)
    X = rng.normal(0, 1, (40, 4))
    Y = rng.uniform(0, 1, (40, 3))
    _, g = M.loss_and_grad(P, X, Y, rnd=False)
    idx = np.concatenate([rng.choice(np.arange(a, b), min(6, b - a), replace=False)
                          for a, b in ((M.W1, M.B1), (M.B1, M.W2), (M.W2, M.B2), (M.B2, M.W3),
                                       (M.W3, M.B3), (M.B3, 4675))])
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (M.loss_and_grad(Pp, X, Y, rnd=False)[0] - M.loss_and_grad(Pm, X, Y, rnd=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, -3.14159, 0.0, 1e-30,
                  1.0 + 2 ** -8 + 2 ** -12], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # a tie goes to the even mantissa
    assert r[2] == 1.0 + 2 ** -7  # below half an ulp (2^-7): down
    assert r[6] == 1.0 + 2 ** -7  # above half an ulp: up
    assert abs(r[3] + 3.140625) < 1e-12 and r[4] == 0.0
    u = r.astype(np.float32).view(np.uint32)
    assert np.all(u & 0xFFFF == 0)
