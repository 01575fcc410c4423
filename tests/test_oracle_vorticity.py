"""The oracle's vorticity (Hydro::enableVorticity) pinned against the
reference: the d_mu beta_nu that ISformal stores in every cell
(src/hdo.cpp:381-611,682-727, one matrix carried through the cell loop) and
the beta.dat lines of Fluid::outputSurface (src/fld.cpp:606-831), from
golden fixtures written by the compiled reference, and live."""
import os

import numpy as np
import pytest

import pyoracle as P
from make_golden import load_vorticity_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REC_RTOL = 1e-12  # beta.dat holds 15 significant digits
CASES = ("vorticity_glauber_21x21x11_b9", "vorticity_glauber_nb_17x17x9",
         "vorticity_glauber_nb_chiral_17x17x9")


def beta_columns(rec, beta):
    """The 33 beta.dat columns from an oracle record and its dbeta row."""
    return np.concatenate([rec[:, :16], beta, rec[:, 27:28]], axis=1)


def rec_close(a, b, rtol=REC_RTOL):
    return np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + 1e-300


@pytest.mark.parametrize("name", CASES)
def test_oracle_dbeta_equals_reference_fixture(name):
    setup, nsteps, counts, beta_rec, db_first, db_last = load_vorticity_case(
        os.path.join(GOLDEN, name + ".npz"))
    o = P.OracleRun(setup, vorticity=True)
    got = []
    for k in range(nsteps):
        assert o.step(1) == 0
        if k == 0:
            assert np.array_equal(o.dbeta, db_first, equal_nan=True)
        rec, _, beta = o.surface_beta()
        assert len(rec) == counts[k], k
        got.append(beta_columns(rec, beta))
    assert np.array_equal(o.dbeta, db_last, equal_nan=True)
    got = np.concatenate(got)
    assert got.shape == beta_rec.shape
    ok = rec_close(got, beta_rec)
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], beta_rec[~ok][:5])
    # the table-EoS fixtures reach the [-100, 100] clamp of Cell::setDbeta;
    # every fixture has elements on the surface
    if "chiral" not in name:
        assert (np.abs(db_first) == 100.).any() or (np.abs(db_last) == 100.).any()
    assert sum(counts) > 50


def test_vorticity_leaves_the_evolution_unchanged():
    """dbeta only feeds beta.dat: the fields after the steps are the same
    bits with vorticity on and off."""
    setup, nsteps, *_ = load_vorticity_case(os.path.join(GOLDEN, CASES[1] + ".npz"))
    a = P.OracleRun(setup, vorticity=True)
    b = P.OracleRun(setup)
    a.step(nsteps)
    b.step(nsteps)
    sa, sb = a.get_state(), b.get_state()
    for k in sa:
        assert np.array_equal(sa[k], sb[k], equal_nan=True), k


@pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")
def test_oracle_dbeta_equals_reference_live_with_resize():
    """Live against the reference, through a x2 resize (the new fluid's
    cells start from zero dbeta, src/main.cpp:257-265)."""
    from vhlle_b200 import workloads as W

    setup = W.small_glauber3d(17, 9, b=4.0, seed=11)
    o = P.OracleRun(setup, vorticity=True)
    r = P.RefRun(setup)
    r.enable_vorticity()
    try:
        for k in range(5):
            if k == 2:
                assert o.resize2x() == 1 and r.resize2x() == 1
                assert np.array_equal(o.dbeta, r.get_dbeta())
            o.step(1)
            r.step(1)
            assert np.array_equal(o.dbeta, r.get_dbeta(), equal_nan=True), k
    finally:
        r.close()
