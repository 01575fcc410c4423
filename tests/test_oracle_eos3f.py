"""EoS3f (src/eo3.cpp: the (e, nb, nq, ns) table with one n grid for the
three charges) in the oracle against the reference's own class, compiled
from its sources: the lookup at general charges bit for bit (inside the
table, beyond its edges, e below the grid and negative, where the reference
extrapolates), and steps of an event with baryon charge on that EoS bit for
bit, with the freeze-out records' mu_Q column.  The table is synthetic
(workloads.eos3f_table) in the reference's file format: no EoS3f table is
in the reference tree."""
import os
import tempfile

import numpy as np
import pytest

import pyoracle as P
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.skipif(not P.ref_available(), reason="compiled reference not present")


def _setup(n=17, nz=9):
    return W.glauber3d_nb_setup(n, n, nz, eos=W.eos3f_table())


def test_eos3f_lookup_equals_reference():
    s = _setup(5, 5)
    rng = np.random.default_rng(3)
    n = 20000
    e = np.concatenate([10 ** rng.uniform(-5, 3.3, n - 400), -rng.uniform(0, 1, 200),
                        np.zeros(100), s.eos.egrid[rng.integers(0, s.eos.ne, 100)]])
    ch = rng.uniform(-0.5, 0.5, (len(e), 3))
    ch[::7] = 0.0
    ch[::11, 0] = s.eos.ngrid[rng.integers(0, s.eos.nn, len(ch[::11]))]
    pts = np.column_stack([e, ch])
    ref = P.RefRun(s).eos_full(pts)
    got = P.OracleRun(s).eos_full(pts)
    same = (got == ref) | (np.isnan(got) & np.isnan(ref))
    assert same.all(), np.argwhere(~same)[:5]
    assert np.abs(ref[:, 3]).max() > 0.01 and np.abs(ref[:, 4]).max() > 0.01


def test_eos3f_event_equals_reference():
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
    col = {c: k for k, c in enumerate(P.SURF_COLS)}
    assert np.abs(rec[:, col["muq"]]).max() > 1e-5
