"""The device EoSChiral (vh_eos kind VH_EOS_CHIRAL, the reference's default
EoS, src/eoChiral.cpp) against the reference's own lookups (fixture) and
the oracle: lookups bit for bit over every region and edge, a viscous
baryon-charge event's fields bit for bit, and its corona and freeze-out
records (muS in column 15) within the surface tests' 1e-12."""
import os

import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def rec_close(a, b, rtol=1e-12):
    return np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + 1e-300


def test_gpu_chiral_eos_equals_reference_answers():
    from vhlle_b200.capi import GpuHydro
    z = np.load(os.path.join(GOLDEN, "chiral_known_answers.npz"))
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos())
    d = GpuHydro(setup)
    got = d.eos6(z["e"], z["nb"])
    exp = z["out"]
    same = (got == exp) | (np.isnan(got) & np.isnan(exp))
    assert same.all(), (np.argwhere(~same)[:5], got[~same][:5], exp[~same][:5])
    d.close()


def test_gpu_chiral_event_equals_oracle():
    from vhlle_b200.capi import GpuHydro
    setup = W.glauber3d_nb_setup(25, 25, 13, eos=W.chiral_eos())
    o, d = P.OracleRun(setup), GpuHydro(setup)
    rc, _ = d.corona()
    ro, _ = o.corona()
    assert len(rc) == len(ro) and rec_close(rc, ro).all()
    n_rec = 0
    for k in range(4):
        o.step(1)
        d.step(1)
        bad = compare_states(gpu_state_as_oracle(d.get_state()), o.get_state())
        assert not bad, (k, bad)
        rd, info = d.surface()
        ro, acc = o.surface()
        assert len(rd) == len(ro) and info["nsusp"] == int(acc["nsusp"]), k
        assert rec_close(rd, ro).all(), (k, np.argwhere(~rec_close(rd, ro))[:5])
        n_rec += len(rd)
        assert (np.abs(rd[:, 15]) > 0).any() or len(rd) == 0
    assert n_rec > 100
    d.close()
