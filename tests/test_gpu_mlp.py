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


def _iters_per_call(setup, mlp, nsteps, method=0):
    from vhlle_b200.capi import GpuHydro
    d = GpuHydro(setup)
    d.set_con2prim(TIGHT)
    d.set_con2prim_method(method)
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
    slope, st_s = _iters_per_call(setup, None, 4, method=1)
    guided_slope, st_gs = _iters_per_call(setup, m, 4, method=1)
    print("iterations per root find: start 0.5 %.3f, untrained %.3f, trained %.3f; "
          "table slope: start 0.5 %.3f, trained %.3f" % (base, raw, guided, slope, guided_slope))
    assert guided < base
    # the EoS's own slope converges quadratically inside a table cell; the
    # trained start point saves iterations on top of it
    assert slope < 0.7 * base and guided_slope < slope
    # every guided / table-slope step against the tight oracle after the
    # same 6 steps
    o = P.OracleRun(setup, tol=TIGHT)
    o.step(6)
    exp = o.get_state()
    for state in (st, st_s, st_gs):
        _within_tight(gpu_state_as_oracle(state), exp)
    m.close()
    untrained.close()


def _within_tight(got, exp):
    for k in exp:
        a = np.asarray(got[k], dtype=np.float64).reshape(-1)
        b = np.asarray(exp[k], dtype=np.float64).reshape(-1)
        scale = np.abs(b).max()
        ok = np.abs(a - b) <= 1e-8 * np.maximum(np.abs(a), np.abs(b)) + 1e-12 * scale
        assert ok.all(), (k, np.argwhere(~ok)[:5])


@pytest.mark.parametrize("case", [
    ("glauber_nb_25x25x13", lambda: W.glauber3d_nb_setup(25, 25, 13, eos=W.nb_table(200, 20)), 8),
    ("glauber_nb_chiral_17x17x9", lambda: W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos()), 6),
    ("gubser_31x31", lambda: W.gubser_setup(nx=31, ny=31), 10),
], ids=lambda c: c[0])
def test_gpu_table_slope_within_tight_oracle(case):
    """VH_C2P_TABLE_SLOPE on the (e, nb) table, the chiral EoS and the
    conformal gas: the step stays within 1e-8 of the tight oracle and takes
    no more iterations than the reference's constant slope."""
    from vhlle_b200.capi import GpuHydro, VhError
    _, fac, n = case
    setup = fac()
    d = GpuHydro(setup)
    with pytest.raises(VhError):
        d.set_con2prim_method(1)  # needs a tight tolerance first
    d.set_con2prim(TIGHT)
    d.set_con2prim_method(1)
    with pytest.raises(VhError):
        d.set_con2prim(1e-5)  # and keeps it
    d.con2prim_stats(True)
    d.step(n)
    c, it = d.con2prim_stats(False)
    o = P.OracleRun(setup, tol=TIGHT)
    o.step(n)
    _within_tight(gpu_state_as_oracle(d.get_state()), o.get_state())
    d.close()
    r = GpuHydro(setup)
    r.set_con2prim(TIGHT)
    r.con2prim_stats(True)
    r.step(n)
    c0, it0 = r.con2prim_stats(False)
    r.close()
    print("iterations per root find: constant slope %.3f, table slope %.3f" % (it0 / c0, it / c))
    assert it / c <= it0 / c0 + 1e-9
