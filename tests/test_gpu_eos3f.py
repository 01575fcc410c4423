"""The EoS3f kind on the device (VH_EOS_TABLE3) against the oracle, itself
equal bit for bit to the reference's compiled eo3.cpp
(tests/test_oracle_eos3f.py): the lookup, the steps of an event with baryon
charge (bit for bit) and its freeze-out records with the mu_Q column
(1e-12 relative, as every record)."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_gpu_eos3f_lookup_equals_oracle():
    s = W.glauber3d_nb_setup(5, 5, 5, eos=W.eos3f_table())
    rng = np.random.default_rng(4)
    e = np.concatenate([10 ** rng.uniform(-5, 3.3, 5000), -rng.uniform(0, 1, 50), np.zeros(20)])
    nb = rng.uniform(-0.5, 0.5, len(e))
    h = capi.GpuHydro(s, upload=False)
    got = h.eos6(e, nb)  # p, T, muB, muS, EoS::p, EoS::s
    h.close()
    o = P.OracleRun(s)
    full = o.eos_full(np.column_stack([e, nb, np.zeros_like(e), np.zeros_like(e)]))
    assert np.array_equal(got[:, 0], full[:, 0]) and np.array_equal(got[:, 1], full[:, 1])
    assert np.array_equal(got[:, 2], full[:, 2]) and np.array_equal(got[:, 3], full[:, 4])
    assert np.array_equal(got, o.eos6(e, nb), equal_nan=True)


def test_gpu_eos3f_event_equals_oracle():
    from test_gpu_surface import rec_close
    s = W.glauber3d_nb_setup(25, 25, 13, eos=W.eos3f_table())
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
    col = {c: k for k, c in enumerate(P.SURF_COLS)}
    assert np.abs(rd[:, col["muq"]]).max() > 1e-5
    with pytest.raises(capi.VhError):
        d.set_con2prim(1e-13)
        d.set_con2prim_method(1)
    d.close()
