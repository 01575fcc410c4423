"""The driver-loop pieces around performStep -- the eta-CFL substeps
(src/main.cpp:405-419) and the one-shot x2 transverse grid resize
(expandGrid2x, src/main.cpp:246-271, Cell::importVars src/cll.cpp:54-68) --
in the C restatement against the reference compiled from its own sources:
bit-for-bit, including the grid coordinates the resize derives."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states
from vhlle_b200 import workloads as W

needs_ref = pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")


def test_substep_rule_counts():
    lib = P.oracle_lib()
    # dtau / n > tau * deta doubles n
    assert lib.or_substeps(0.05, 1.0, -5., 5., 101) == 1      # deta 0.1
    assert lib.or_substeps(0.05, 0.3, -5., 5., 101) == 2      # 0.03 < 0.05 <= 0.06
    assert lib.or_substeps(0.05, 0.1, -5., 5., 101) == 8      # 0.01 -> 0.00625
    assert lib.or_substeps(0.05, 0.5, -7.5, 7.5, 1) == 1      # nz = 1: deta = inf
    # exactly equal is not "greater": no halving
    assert lib.or_substeps(0.25, 1.0, 0., 1., 5) == 1
    assert lib.or_substeps(0.25, 1.0, 0., 1., 6) == 2


def _drive(run, setup, nloops, dtau, tau_resize):
    """main.cpp's loop without the output calls: substeps, then the
    one-shot resize once tau >= tau_resize.  Returns the substep counts."""
    g = setup.grid
    counts, resized = [], False
    for _ in range(nloops):
        counts.append(run.advance(dtau, g.etamin, g.etamax, g.nz))
        if run.tau_now >= tau_resize and not resized:
            assert run.resize2x() == 1
            resized = True
    return counts, resized


@needs_ref
@pytest.mark.parametrize("case", [
    # tau0 = 0.05: tau * deta starts below dtau, so the first loops substep
    ("glauber_17x17x9_tau005", lambda: W.small_glauber3d(17, 9, tau0=0.05, dt=0.1), 0.1, 8, 0.3),
    ("glauber_16x16x7_even", lambda: W.small_glauber3d(16, 7, tau0=0.04, dt=0.1, b=4.0), 0.1, 7,
     0.2),
], ids=lambda c: c[0])
def test_substeps_and_resize_equal_reference(case):
    name, fac, dtau, nloops, tres = case
    setup = fac()
    o, r = P.OracleRun(setup), P.RefRun(setup)
    co, ro = _drive(o, setup, nloops, dtau, tres)
    cr, rr = _drive(r, setup, nloops, dtau, tres)
    assert co == cr and ro and rr
    assert max(co) > 1, "case must exercise substeps"
    assert o.tau_now == r.tau_now
    assert o.dt == r.dtau
    assert np.array_equal(o.grid_coords(), r.grid_coords())
    bad = compare_states(o.get_state(), r.get_state())
    assert not bad, bad
    # the totals after the resize follow the new grid
    to, tr_ = o.totals(), r.totals()
    for k in P.TOTALS:
        assert to[k] == tr_[k] or (np.isnan(to[k]) and np.isnan(tr_[k])), k
    r.close()


@needs_ref
def test_resize_refuses_asymmetric_grid():
    setup = W.small_glauber3d(13, 5)
    g = setup.grid
    setup.grid = W.Grid(g.nx, g.ny, g.nz, g.xmin + 1.0, g.xmax + 1.0, g.ymin, g.ymax, g.etamin,
                        g.etamax)
    o, r = P.OracleRun(setup), P.RefRun(setup)
    before = o.get_state()
    assert o.resize2x() == 0 and r.resize2x() == 0
    assert not compare_states(o.get_state(), before)
    assert np.array_equal(o.grid_coords(), r.grid_coords())
    r.close()


@needs_ref
def test_resize_2d_grid_coordinates_follow_reference():
    """nz = 1: dz = inf, so getZ(0) = etamin + 0*inf is NaN in the reference
    and the resized grid carries NaN eta bounds; the restatement keeps that."""
    setup = W.gubser_setup(nx=21, ny=21)
    o, r = P.OracleRun(setup), P.RefRun(setup)
    o.step(2)
    r.step(2)
    assert o.resize2x() == 1 and r.resize2x() == 1
    go, gr = o.grid_coords(), r.grid_coords()
    assert np.isnan(go[4]) and np.isnan(gr[4])
    same = (go == gr) | (np.isnan(go) & np.isnan(gr))
    assert same.all(), (go, gr)
    assert o.step(3) == 0
    r.step(3)
    bad = compare_states(o.get_state(), r.get_state())
    assert not bad, bad
    r.close()
