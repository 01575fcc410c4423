"""EoSCMFe (src/eoCMFe.cpp, the driver's eosType 4: two uniform (e, nb)
tables of the CMF model, 1501 x 501 and 4001 x 401, with EPS_CUTOFF and a
NaN-entry fallback) in the oracle against the reference's own class,
compiled from its sources and reading eos/cmfe_small.dat and eos/cmfe.dat
as it does: the lookup bit for bit (both tables, below the cutoff, in the
NaN hole, beyond both tables, negative baryon density), and steps of an
event with baryon charge on that EoS bit for bit, with its freeze-out
records.  The tables are synthetic (workloads.cmfe_eos_table) in the
reference's file format: the CMF tables are not in the reference tree."""
import os
import tempfile

import numpy as np
import pytest

import pyoracle as P
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.skipif(not P.ref_available(), reason="compiled reference not present")


@pytest.fixture(scope="module")
def tables(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("cmfe"))
    eos = W.cmfe_eos_table()
    eos.write_cmfe(d)
    return eos, d


def test_cmfe_lookup_equals_reference(tables):
    eos, d = tables
    s = W.glauber3d_nb_setup(5, 5, 5, eos=eos)
    rng = np.random.default_rng(7)
    n = 30000
    e = np.concatenate([10 ** rng.uniform(-3, 2.3, n - 300), -rng.uniform(0, 1, 100),
                        np.zeros(100), rng.uniform(0.015, 0.025, 100)])
    nb = np.concatenate([rng.uniform(-0.5, 6.5, n - 3000), rng.uniform(4.9, 5.6, 3000)])
    nb[::9] = 0.0
    pts = np.column_stack([e, nb, np.zeros_like(e), np.zeros_like(e)])
    ref = P.RefRun(s, eos_file=d).eos_full(pts)
    got = P.OracleRun(s).eos_full(pts)
    same = (got == ref) | (np.isnan(got) & np.isnan(ref))
    assert same.all(), np.argwhere(~same)[:5]
    eps0, n0 = W.CMFE_EPS0, W.CMFE_N0
    small = (e < 15 * eps0 / 1000.0) & (nb < 5 * n0) & (e >= 2e-2)
    big = ~small & (e < 0.8 * eps0) & (nb < 40.0 * n0) & (e >= 2e-2)
    hole = big & (nb > 36.0 * n0) & (e < 40.0 * eps0 / 1000.0)
    assert small.sum() > 100 and big.sum() > 100 and hole.sum() > 10
    assert (ref[hole, 0] == 0).all() and (ref[~hole & big, 0] > 0).any()


def test_cmfe_event_equals_reference(tables):
    eos, d = tables
    s = W.glauber3d_nb_setup(17, 17, 9, eos=eos)
    o, r = P.OracleRun(s), P.RefRun(s, eos_file=d)
    for step in range(4):
        assert o.step(1) == 0
        r.step(1)
        a, b = o.get_state(), r.get_state()
        for k in a:
            assert np.array_equal(a[k], b[k], equal_nan=True), (step, k)
    with tempfile.TemporaryDirectory() as t:
        n, _ = r.output_surface(t, extend=True)
        rec = P.read_freezeout(os.path.join(t, "freezeout.dat.unfinished"), extend=True)
    ro, _ = o.surface(cap=400000)
    assert len(ro) == n > 50
    ok = np.abs(ro - rec) <= 1e-13 * np.maximum(np.abs(ro), np.abs(rec)) + 1e-300
    assert ok.all(), np.argwhere(~ok)[:5]
