"""EoSAZH (src/eoAZH.cpp, the driver's eosType 2: six EoSAZHaux tables, p,
T and muB below and above the first table's e range, scaled down by e/emin
below it) in the oracle against the reference's own class, compiled from
its sources and reading the six files from eos/azhydro0p2 as it does: the
lookup bit for bit (both table sets, below, beyond and at their edges,
negative baryon density, where muB extrapolates from the first nb cell),
and steps of an event with baryon charge on that EoS bit for bit, with its
freeze-out records.  The tables are synthetic (workloads.azh_eos_table) in
the reference's file format: the azhydro0p2 files are not in the reference
tree."""
import os
import tempfile

import numpy as np
import pytest

import pyoracle as P
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.skipif(not P.ref_available(), reason="compiled reference not present")


def _setup(n=17, nz=9):
    return W.glauber3d_nb_setup(n, n, nz, eos=W.azh_eos_table())


def test_azh_lookup_equals_reference():
    s = _setup(5, 5)
    rng = np.random.default_rng(5)
    n = 20000
    edges = np.array([0.01, 2.01, 2.0, 152.0, 0.005, 1e-12, 500.0])
    e = np.concatenate([10 ** rng.uniform(-4, 2.6, n - 300), -rng.uniform(0, 1, 100),
                        np.zeros(100), 0.01 + 0.005 * rng.integers(0, 401, 93), edges])
    nb = rng.uniform(-0.7, 0.7, len(e))
    nb[::9] = 0.0
    nb[::13] = 0.01 * rng.integers(0, 51, len(nb[::13]))
    pts = np.column_stack([e, nb, np.zeros_like(e), np.zeros_like(e)])
    ref = P.RefRun(s).eos_full(pts)
    got = P.OracleRun(s).eos_full(pts)
    same = (got == ref) | (np.isnan(got) & np.isnan(ref))
    assert same.all(), np.argwhere(~same)[:5]
    # all three branches and a signed muB were reached
    assert (e < 0.01).any() and ((e > 0.01) & (e < 2.01)).any() and (e > 2.01).any()
    assert (ref[:, 2] < 0).any() and (ref[:, 2] > 0).any()


def test_azh_event_equals_reference():
    s = _setup()
    o, r = P.OracleRun(s), P.RefRun(s)
    for step in range(4):
        assert o.step(1) == 0
        r.step(1)
        a, b = o.get_state(), r.get_state()
        for k in a:
            assert np.array_equal(a[k], b[k], equal_nan=True), (step, k)
    with tempfile.TemporaryDirectory() as d:
        n, _ = r.output_surface(d, extend=True)
        rec = P.read_freezeout(os.path.join(d, "freezeout.dat.unfinished"), extend=True)
    ro, _ = o.surface(cap=400000)
    assert len(ro) == n > 50
    ok = np.abs(ro - rec) <= 1e-13 * np.maximum(np.abs(ro), np.abs(rec)) + 1e-300
    assert ok.all(), np.argwhere(~ok)[:5]
