"""The EoSCMFe kind on the device (VH_EOS_CMFE) against the oracle, itself
equal bit for bit to the reference's compiled eoCMFe.cpp
(tests/test_oracle_cmfe_eos.py): the lookup over both tables, the cutoff,
the NaN hole and beyond, the steps of an event with baryon charge (bit for
bit) and its freeze-out records (1e-12 relative, as every record)."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eos():
    return W.cmfe_eos_table()


def test_gpu_cmfe_lookup_equals_oracle(eos):
    s = W.glauber3d_nb_setup(5, 5, 5, eos=eos)
    rng = np.random.default_rng(8)
    e = np.concatenate([10 ** rng.uniform(-3, 2.3, 8000), -rng.uniform(0, 1, 50), np.zeros(20),
                        rng.uniform(0.015, 0.025, 50)])
    nb = rng.uniform(-0.5, 6.5, len(e))
    h = capi.GpuHydro(s, upload=False)
    got = h.eos6(e, nb)  # p, T, muB, muS, EoS::p, EoS::s
    h.close()
    o = P.OracleRun(s)
    assert np.array_equal(got, o.eos6(e, nb), equal_nan=True)


def test_gpu_cmfe_event_equals_oracle(eos):
    from test_gpu_surface import rec_close
    s = W.glauber3d_nb_setup(25, 25, 13, eos=eos)
    o, d = P.OracleRun(s), capi.GpuHydro(s)
    for step in range(5):
        assert o.step(1) == 0
        d.step(1)
        bad = compare_states(gpu_state_as_oracle(d.get_state()), o.get_state())
        assert not bad, (step, bad)
    ro, _ = o.surface(cap=400000)
    rd, info = d.surface()
    assert len(ro) == info["nelements"] > 50
    ok = rec_close(rd, ro)
    assert ok.all(), np.argwhere(~ok)[:5]
    with pytest.raises(capi.VhError):
        d.set_con2prim(1e-13)
        d.set_con2prim_method(1)
    d.close()
