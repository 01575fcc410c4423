"""The C restatement against the reference compiled from its own sources
(oracle/_ref), on fresh seeded inputs, step by step: bit-for-bit."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")


@pytest.mark.parametrize("case", [
    ("gubser_31x31", lambda: W.gubser_setup(nx=31, ny=31), 12),
    ("glauber_25x25x13_b9", lambda: W.small_glauber3d(25, 13, b=9.0, seed=99), 8),
    ("glauber_21x21x11_eta02", lambda: W.small_glauber3d(21, 11, seed=7, etaS=0.2, epeak=20.0), 8),
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
