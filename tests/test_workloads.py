"""Host-side input generation: EoS table file format, seeded ICs."""
import math
import os

import numpy as np

from vhlle_b200 import workloads as W


def test_eos1f_file_roundtrip_is_exact(tmp_path):
    t = W.make_cs2_table(ne=50, nn=3, mub_slope=0.2)
    f = os.path.join(tmp_path, "t.dat")
    t.write_eos1f(f)
    u = W.EosTable.read_eos1f(f)
    for k in ("egrid", "ngrid", "p", "T", "mub"):
        assert np.array_equal(getattr(t, k), getattr(u, k)), k


def test_cs2_table_is_thermodynamically_sane():
    t = W.make_cs2_table()
    e, p, T = t.egrid, t.p[:t.ne], t.T[:t.ne]
    assert np.all(np.diff(e) > 0) and np.all(np.diff(p) > 0) and np.all(np.diff(T) > 0)
    cs2 = np.gradient(p, e)
    assert np.allclose(cs2[5:-5], W.cs2_model(e[5:-5]), rtol=2e-3, atol=2e-4)
    # Stefan-Boltzmann anchor at the top of the table
    assert math.isclose(T[-1], (e[-1] / W.CONF_CNST) ** 0.25, rel_tol=1e-12)
    # s = (e + p)/T increases with e
    assert np.all(np.diff((e + p) / T) > 0)


def test_glauber_ic_is_seeded_and_deterministic():
    a = W.small_glauber3d(21, 9, seed=3)
    b = W.small_glauber3d(21, 9, seed=3)
    c = W.small_glauber3d(21, 9, seed=4)
    assert np.array_equal(a.Q, b.Q)
    assert not np.array_equal(a.Q, c.Q)
    assert a.Q[0].max() == 50.0 * a.tau0  # peak e = 50 GeV/fm^3 at rest


def test_gubser_ic_has_the_grid_symmetry():
    # x_i = xmin + i*dx is symmetric only to rounding, hence allclose
    s = W.gubser_setup()
    Q = s.Q.reshape(7, s.grid.ny, s.grid.nx)
    assert np.allclose(Q[0], Q[0][::-1, :], rtol=1e-12) and np.allclose(Q[0], Q[0][:, ::-1], rtol=1e-12)
    assert np.allclose(Q[1], -Q[1][:, ::-1], rtol=1e-12, atol=1e-300)
    assert np.allclose(Q[0], Q[0].T, rtol=1e-12)


def test_full_size_configs_have_the_stated_shapes():
    g = W.glauber3d_setup().grid
    assert (g.nx, g.ny, g.nz) == (101, 101, 51) and g.ncells == 520251
    assert math.isclose(g.dx, 0.3) and math.isclose(g.dz, 0.3)
    g1 = W.gubser_setup().grid
    assert (g1.nx, g1.ny, g1.nz) == (101, 101, 1) and math.isclose(g1.dx, 0.1)


def test_batch_events_shape_and_physics():
    evs = W.batch_events(8)
    bs = np.random.default_rng(W.BATCH_SEED0).uniform(0, 12, 8)
    for k, s in enumerate(evs):
        g = s.grid
        assert 61 <= g.nx <= 121 and g.nx == g.ny and g.nx % 2 == 1
        assert g.nz == W.BATCH_NZ[k % 4]
        assert s.zetaSparam == 5 and s.tr["etaS0"] == 0.12 and s.tr["zetaS0"] == 0.05
        assert s.tr["zetaSPeakT"] == 0.175 and s.tr["zetaSWidthT"] == 0.02
        assert s.viscous
        nt = 121 - 2 * int(round(30 * bs[k] / 12))
        assert g.nx == nt
        assert np.asarray(s.Q).shape == (7, g.ncells)
        assert np.isfinite(np.asarray(s.Q)).all() and np.asarray(s.Q)[0].max() > 0
    # the same event regardless of how many are generated
    assert np.array_equal(np.asarray(W.batch_event(5).Q), np.asarray(evs[5].Q))
