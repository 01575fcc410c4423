"""The oracle's EoSChiral (the reference's default EoS, src/eoChiral.cpp)
pinned against the reference: its lookups over every region and edge from a
fixture of the reference's own outputs, and (live, where the compiled
reference is present) its freeze-out records with muS."""
import os
import tempfile

import numpy as np
import pytest

import pyoracle as P
from make_golden import chiral_digest
from vhlle_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_chiral_eos_equals_reference_answers():
    z = np.load(os.path.join(GOLDEN, "chiral_known_answers.npz"))
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos())
    assert chiral_digest(setup.eos) == str(z["eos_digest"])
    got = P.OracleRun(setup).eos6(z["e"], z["nb"])
    exp = z["out"]
    same = (got == exp) | (np.isnan(got) & np.isnan(exp))
    assert same.all(), (np.argwhere(~same)[:5], got[~same][:5], exp[~same][:5])
    # the fixture covers the three regions, the p clamp and a nonzero muS
    e, nb = z["e"], z["nb"]
    assert ((e < 1.46) & (nb < 0.3)).sum() > 1000 and (e >= 146).sum() > 100
    assert (exp[:, 0] == 0).sum() > 10 and (np.abs(exp[:, 3]) > 0).sum() > 1000


@pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")
def test_oracle_chiral_surface_equals_reference_live():
    """The corona at tau0 and three steps' freeze-out records (muS in
    column 15) equal the reference's freezeout.dat (15 digits)."""
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos())
    o, r = P.OracleRun(setup), P.RefRun(setup)
    try:
        with tempfile.TemporaryDirectory() as d:
            n, _ = r.output_corona(d, extend=True)
            rec = [o.corona()[0]]
            assert len(rec[0]) == n
            for _ in range(3):
                o.step(1)
                r.step(1)
                rec.append(o.surface()[0])
                r.output_surface(d, extend=True)
            ref = P.read_freezeout(os.path.join(d, "freezeout.dat.unfinished"), extend=True)
    finally:
        r.close()
    got = np.concatenate(rec)
    assert got.shape == ref.shape and len(got) > 100
    ok = np.abs(got - ref) <= 1e-12 * np.maximum(np.abs(got), np.abs(ref)) + 1e-300
    assert ok.all(), np.argwhere(~ok)[:5]
    assert (np.abs(got[:, 15]) > 0).any()
