"""The C restatement (oracle) against the golden fixtures that the compiled
reference generated (tests/golden/make_golden.py): bit-for-bit."""
import glob
import os

import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states
from make_golden import load_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# end-state fixtures (the surface_*, corona_* and vorticity_* fixtures hold
# freeze-out and beta.dat records instead)
CASES = sorted(p for p in glob.glob(os.path.join(GOLDEN, "*_*x*.npz"))
               if not os.path.basename(p).startswith(("surface_", "corona_", "vorticity_")))


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
def test_oracle_matches_reference_fixture(path):
    setup, nsteps, tau_end, expect = load_case(path)
    o = P.OracleRun(setup)
    err = o.step(nsteps)
    assert err == 0
    assert o.tau_now == tau_end
    bad = compare_states(o.get_state(), expect)
    assert not bad, bad


@pytest.fixture(scope="module")
def known():
    return np.load(os.path.join(GOLDEN, "known_answers.npz"))


def _setup_for(kind, z):
    from vhlle_b200 import workloads as W
    if kind == "conf":
        return W.gubser_setup(nx=5, ny=5)
    s = W.small_glauber3d(5, 5)
    s.eos = W.EosTable(kind=1, egrid=z["keos_table_egrid"], ngrid=z["keos_table_ngrid"],
                       p=z["keos_table_p"], T=z["keos_table_T"], mub=z["keos_table_mub"])
    return s


@pytest.mark.parametrize("kind", ["conf", "table"])
def test_oracle_transform_pv_known_answers(known, kind):
    o = P.OracleRun(_setup_for(kind, known))
    got = o.transform_pv(known["kpv_Q"])
    assert np.array_equal(got, known["kpv_%s" % kind], equal_nan=True)


@pytest.mark.parametrize("kind", ["conf", "table"])
def test_oracle_eos_known_answers(known, kind):
    o = P.OracleRun(_setup_for(kind, known))
    e, nb = known["keos_%s_in" % kind]
    pT, s = o.eos_eval(e, nb)
    assert np.array_equal(pT, known["keos_%s_out" % kind])
    assert np.array_equal(s, known["keos_%s_s" % kind])


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p) for p in CASES])
def test_oracle_totals_match_reference_fixture(path):
    from make_golden import load_totals
    setup, nsteps, tau_end, expect = load_case(path)
    tot_ref, line, nelem = load_totals(path)
    o = P.OracleRun(setup)
    o.step(nsteps)
    tot = o.totals()
    for k in tot_ref:  # nz = 1 gives 0 * dz = NaN, in the reference too
        assert tot[k] == tot_ref[k] or (np.isnan(tot[k]) and np.isnan(tot_ref[k])), k
    # and the 6-digit line the reference printed: tau E Efull nbSurf S ...
    printed = [float(x) for x in line.split()]
    assert printed[0] == pytest.approx(tau_end, rel=1e-5)
    for val, k in ((printed[1], "E"), (printed[2], "Efull"), (printed[4], "S")):
        assert val == pytest.approx(tot[k], rel=1e-5, abs=1e-6, nan_ok=True), k
