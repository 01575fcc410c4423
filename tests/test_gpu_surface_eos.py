"""The freeze-out EoS on the device (vh_set_surface_eos: Fluid's eosH, which
outputSurface and outputCorona swap in, src/fld.cpp:540-542, 885-887) set to
EoSHadron (VH_EOS_HADRON, src/eoHadron.cpp) or EoSSmash (VH_EOS_SMASH,
src/eoSmash.cpp) against the oracle, itself equal bit for bit to the
reference's classes (tests/test_oracle_hadron_eos.py):
the corona and the surface records within 1e-12 relative (EoSHadron takes
logarithms, which the device may round differently from the C library in
the last bit), the totals within 1e-10; the hydro evolution is untouched."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _close(a, b, rtol):
    return np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + 1e-300


@pytest.mark.parametrize("name", ["hadron", "smash"])
def test_gpu_surface_eos_equals_oracle(name):
    h = {"hadron": W.hadron_eos_table, "smash": W.smash_eos_table}[name]()
    s = W.glauber3d_nb_setup(33, 33, 17, eos=W.nb_table(200, 20))
    o, d = P.OracleRun(s, surface_eos=h), capi.GpuHydro(s)
    d.set_surface_eos(h)
    oc, _ = o.corona()
    dc, _ = d.corona()
    assert len(oc) == len(dc) > 0
    assert _close(dc, oc, 1e-12).all()
    for step in range(4):
        assert o.step(1) == 0
        d.step(1)
        ro, acc = o.surface(cap=400000)
        rd, info = d.surface()
        assert len(ro) == info["nelements"] > 0 and int(acc["nsusp"]) == info["nsusp"], step
        ok = _close(rd, ro, 1e-12)
        assert ok.all(), (step, np.argwhere(~ok)[:5])
    t_o, t_d = o.totals(), d.totals()
    for k in t_o:
        assert _close(np.array(t_d[k]), np.array(t_o[k]), 1e-10), (k, t_d[k], t_o[k])
    assert not compare_states(gpu_state_as_oracle(d.get_state()), o.get_state())
    # back to the hydro EoS
    d.set_surface_eos(None)
    o2 = P.OracleRun(s)
    o2.step(4)
    r2, _ = o2.surface(cap=400000)
    rd2, _ = d.surface()
    assert _close(rd2, r2, 1e-12).all()
    d.close()


@pytest.mark.parametrize("name", ["hadron", "smash"])
def test_gpu_hadron_eos_is_only_a_surface_eos(name):
    h = {"hadron": W.hadron_eos_table, "smash": W.smash_eos_table}[name]()
    s = W.glauber3d_nb_setup(9, 9, 5, eos=h)
    with pytest.raises(capi.VhError):
        capi.GpuHydro(s)
