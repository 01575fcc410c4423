"""The freeze-out EoS on the device (vh_set_surface_eos: Fluid's eosH, which
outputSurface and outputCorona swap in, src/fld.cpp:540-542, 885-887) set to
EoSHadron (VH_EOS_HADRON, src/eoHadron.cpp) or EoSSmash (VH_EOS_SMASH,
src/eoSmash.cpp) against the oracle, itself equal bit for bit to the
reference's classes (tests/test_oracle_hadron_eos.py):
the corona and the surface records within 1e-12 relative, with the
allowances of test_gpu_surface.rec_close_scaled after steps (a near-zero
dSigma component cancels, and gamma^2 multiplies a last-bit difference of
the device's cosh/sinh/log/tanh in transformToLab), the totals within
1e-10; the hydro evolution is untouched."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from test_gpu_surface import rec_close_scaled
from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _close(a, b, rtol):
    return np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + 1e-300


def _report(a, b, ok):
    """The failing records: index, column, both values, u^0."""
    bad = np.argwhere(~ok)[:6]
    return [(int(i), int(c), float(a[i, c]), float(b[i, c]), float(a[i, 8])) for i, c in bad]


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
        ok = rec_close_scaled(rd, ro)
        assert ok.all(), (step, _report(rd, ro, ok))
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
    ok = rec_close_scaled(rd2, r2)
    assert ok.all(), _report(rd2, r2, ok)
    d.close()


@pytest.mark.parametrize("name", ["hadron", "smash"])
def test_gpu_hadron_eos_is_only_a_surface_eos(name):
    h = {"hadron": W.hadron_eos_table, "smash": W.smash_eos_table}[name]()
    s = W.glauber3d_nb_setup(9, 9, 5, eos=h)
    with pytest.raises(capi.VhError):
        capi.GpuHydro(s)
