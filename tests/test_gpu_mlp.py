"""The learned con2prim start point on the device: the training kernels'
gradient and the tensor-core forward pass against the FP64 CPU restatement
(tests/mlp_ref.py), and what a trained network gains -- fewer root-find
iterations at the tight tolerance -- while the step stays within 1e-8 of the
tight oracle (the reference's algorithm with only the tolerance changed).

Tolerances: the device accumulates in FP32 and rounds activations to BF16,
so its gradient and outputs match the FP64 restatement (which rounds at the
same points) to about 1e-3 of their norms; the fields, which the FP64 Newton
finishes to |dv| < 1e-13, to 1e-8 relative."""
import numpy as np
import pytest

import mlp_ref as M
import pyoracle as P
from helpers import gpu_state_as_oracle
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
TIGHT = 1e-13


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    p = np.zeros(4675, dtype=np.float32)
    p[M.W1:M.B1] = rng.normal(0, 0.6, 256)
    p[M.B1:M.W2] = rng.normal(0, 0.1, 64)
    p[M.W2:M.B2] = rng.normal(0, 0.15, 4096)
    p[M.B2:M.W3] = rng.normal(0, 0.1, 64)
    p[M.W3:M.B3] = rng.normal(0, 0.15, 192)
    p[M.B3:] = rng.normal(0, 0.1, 3)
    return p


def _data(seed, n):
    rng = np.random.default_rng(seed)
    X = np.stack([rng.uniform(-1, 0.7, n), rng.uniform(0, 1, n), rng.uniform(0, 0.1, n),
                  (rng.uniform(0, 1, n) < 0.05).astype(float)], 1).astype(np.float32)
    Y = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    return X, Y


def test_gpu_mlp_gradient_matches_cpu_restatement():
    import torch
    from vhlle_b200.capi import Mlp
    m = Mlp(seed=3)
    p = _rand_params(11)
    m.set_params(p)
    X, Y = _data(12, 300)  # 3 blocks, the last one partial
    g, loss = m.grad(torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda())
    lr, gr = M.loss_and_grad(p, X, Y)
    assert abs(loss - lr) <= 1e-4 * abs(lr)
    for a, b in ((M.W1, M.B1), (M.B1, M.W2), (M.W2, M.B2), (M.B2, M.W3), (M.W3, M.B3), (M.B3, 4675)):
        err = np.linalg.norm(g[a:b] - gr[a:b]) / np.linalg.norm(gr[a:b])
        assert err < 3e-3, (a, b, err)
    m.close()


def test_gpu_mlp_forward_matches_cpu_restatement():
    import torch
    from vhlle_b200.capi import Mlp
    m = Mlp(seed=4)
    p = _rand_params(21)
    m.set_params(p)
    X, _ = _data(22, 1000 + 7)  # not a multiple of 16
    y = m.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    yr, _ = M.forward(p, X)
    err = np.abs(y - yr).max() / np.abs(yr).max()
    assert err < 5e-3, err
    m.close()


def _iters_per_call(setup, mlp, nsteps):
    from vhlle_b200.capi import GpuHydro
    d = GpuHydro(setup)
    d.set_con2prim(TIGHT)
    if mlp is not None:
        d.set_con2prim_guess(mlp)
    d.step(2)
    d.con2prim_stats(True)
    d.step(nsteps)
    calls, iters = d.con2prim_stats(False)
    st = d.get_state()
    d.close()
    return iters / calls, st


def test_gpu_mlp_trained_guess_saves_iterations_within_tolerance():
    import torch
    from vhlle_b200.capi import GpuHydro, Mlp
    setup = W.small_glauber3d(33, 17, seed=41, b=6.0)
    # training data: every cell state of several snapshots of the event
    d = GpuHydro(setup)
    cap = 64 * setup.grid.ncells
    X = torch.empty((cap, 4), dtype=torch.float32, device="cuda")
    Y = torch.empty((cap, 3), dtype=torch.float32, device="cuda")
    n = 0
    for k in range(8):
        d.step(2)
        n += d.mlp_samples(X[n:], Y[n:])
    d.close()
    assert n > 10000
    X, Y = X[:n].contiguous(), Y[:n].contiguous()
    m = Mlp(seed=7)
    losses = m.train(X, Y, batch=4096, epochs=40, lr=3e-3, seed=9)
    assert losses[-1] < losses[0] / 5, losses
    pred = m.forward(X).cpu().numpy()
    v_err = np.abs(pred[:, 1] - Y[:, 1].cpu().numpy())
    assert np.median(v_err) < 0.05

    base, _ = _iters_per_call(setup, None, 4)
    untrained = Mlp(seed=8)
    raw, _ = _iters_per_call(setup, untrained, 4)
    guided, st = _iters_per_call(setup, m, 4)
    print("iterations per root find: start 0.5 %.3f, untrained %.3f, trained %.3f"
          % (base, raw, guided))
    assert guided < base
    # the guided step against the tight oracle after the same 6 steps
    o = P.OracleRun(setup, tol=TIGHT)
    o.step(6)
    got, exp = gpu_state_as_oracle(st), o.get_state()
    for k in exp:
        a = np.asarray(got[k], dtype=np.float64).reshape(-1)
        b = np.asarray(exp[k], dtype=np.float64).reshape(-1)
        scale = np.abs(b).max()
        ok = np.abs(a - b) <= 1e-8 * np.maximum(np.abs(a), np.abs(b)) + 1e-12 * scale
        assert ok.all(), (k, np.argwhere(~ok)[:5])
    m.close()
    untrained.close()
