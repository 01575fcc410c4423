"""The C restatement against the reference compiled from its own sources
(oracle/_ref), on fresh seeded inputs, step by step: bit-for-bit."""
import numpy as np
import pytest

import pyoracle as P
from helpers import TRANSPORT_VARIANTS, compare_states, transport_inputs, transport_variant
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")


@pytest.mark.parametrize("case", [
    ("gubser_31x31", lambda: W.gubser_setup(nx=31, ny=31), 12),
    ("glauber_25x25x13_b9", lambda: W.small_glauber3d(25, 13, b=9.0, seed=99), 8),
    ("glauber_21x21x11_eta02", lambda: W.small_glauber3d(21, 11, seed=7, etaS=0.2, epeak=20.0), 8),
    ("glauber_nb_21x21x11", lambda: W.glauber3d_nb_setup(21, 21, 11), 6),
], ids=lambda c: c[0])
def test_oracle_equals_reference_every_step(case):
    name, fac, n = case
    setup = fac()
    o, r = P.OracleRun(setup), P.RefRun(setup)
    for s in range(n):
        assert o.step(1) == 0
        r.step(1)
        assert o.tau_now == r.tau_now
        bad = compare_states(o.get_state(), r.get_state())
        assert not bad, (s, bad)
    r.close()


@pytest.mark.parametrize("variant", TRANSPORT_VARIANTS, ids=lambda v: "%sSparam%d" % v)
def test_transport_forms_equal_reference_every_step(variant):
    setup = transport_variant(*variant)
    o, r = P.OracleRun(setup), P.RefRun(setup)
    for s in range(6):
        assert o.step(1) == 0
        r.step(1)
        bad = compare_states(o.get_state(), r.get_state())
        assert not bad, (s, bad)
    st = o.get_state()
    # the form is exercised: shear everywhere, bulk for the zeta forms
    assert np.abs(st["pi"]).max() > 0.1
    assert (np.abs(st["Pi"]).max() > 0.1) == (variant[0] == "zeta")
    r.close()


@pytest.mark.parametrize("variant", TRANSPORT_VARIANTS + [("eta", 0)],
                         ids=lambda v: "%sSparam%d" % v)
def test_transport_coefficients_equal_reference(variant):
    """TransportCoeff::getEta + getTau on 1e5 random points: bit-for-bit."""
    setup = transport_variant(*variant)
    if variant == ("eta", 0):
        setup.zetaSparam = 0
    inp = transport_inputs()
    r = P.RefRun(setup)
    a, b = P.OracleRun(setup).transport_eval(inp), r.transport_eval(inp)
    r.close()
    assert np.array_equal(a, b, equal_nan=True)
    assert np.abs(a[:, 0]).max() > 0 and np.abs(a[:, 2]).max() > 0


def test_reference_rejects_the_oracle_only_zeta_bump():
    with pytest.raises(ValueError):
        P.RefRun(W.large_event_setup(0, 9, 9, 5, eos=W.nb_table(20, 4)))


def test_transform_pv_random_states_equal_reference():
    rng = np.random.default_rng(7)
    n = 3000
    Q = np.zeros((n, 7))
    Q[:, 0] = 10 ** rng.uniform(-6, 3, n)
    v = rng.uniform(0, 1.2, n)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    Q[:, 1:4] = d * (v * Q[:, 0])[:, None]
    Q[:, 4] = rng.uniform(0, 0.1, n) * Q[:, 0]
    for setup in (W.gubser_setup(nx=5, ny=5), W.small_glauber3d(5, 5)):
        o, r = P.OracleRun(setup), P.RefRun(setup)
        assert np.array_equal(o.transform_pv(Q), r.transform_pv(Q), equal_nan=True)
        r.close()
