"""vh_step_host (the step with the state in host memory, its copies
overlapping the kernels) against vh_step with the state resident on the
device: after every step the host arrays hold what the resident run
downloads, bit for bit, with page-locked arrays (the captured graph with its
copy branches) and with ordinary ones (the upload / step / download
sequence), on a viscous event (the relaxation-stage copies), the same with
vorticity on, and an ideal one (every copy at the end), with surface calls
between the steps."""
import numpy as np
import pytest

from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
STATE_IO = ("Q", "pi", "piH", "Pi", "PiH", "m", "viscCorrCut")


@pytest.mark.parametrize("pinned", [True, False])
@pytest.mark.parametrize("case", ["viscous", "ideal", "vorticity"])
def test_gpu_step_host_equals_resident(case, pinned):
    setup = (W.gubser_setup(nx=41, ny=41) if case == "ideal"
             else W.small_glauber3d(33, 17, seed=11, b=6.0))
    a, b = capi.GpuHydro(setup), capi.GpuHydro(setup)
    if case == "vorticity":
        a.enable_vorticity()
        b.enable_vorticity()
    try:
        host = (b.pinned_state(STATE_IO) if pinned else
                {k: np.zeros((capi.STATE_NCOMP[k], b.N)) for k in STATE_IO})
        st = b.get_state(STATE_IO)
        for k in STATE_IO:
            host[k][:] = st[k]
        for n in range(1, 9):
            a.step(1)
            b.step_host(host)
            ref = a.get_state(STATE_IO)
            for k in STATE_IO:
                assert np.array_equal(host[k], ref[k]), (n, k)
            assert a.tau == b.tau
            if n % 3 == 0:
                assert a.surface()[1] == b.surface()[1]
        assert (host["Q"][0] > 0).any() and (host["m"] > 0).any()
        if case != "ideal":
            assert np.abs(host["pi"]).max() > 0
        if case == "vorticity":
            assert np.array_equal(a.get_dbeta(), b.get_dbeta())
    finally:
        a.close()
        b.close()


def test_gpu_step_host_refused_while_a_surface_is_pending():
    setup = W.small_glauber3d(17, 9)
    h = capi.GpuHydro(setup)
    try:
        host = {k: np.zeros((capi.STATE_NCOMP[k], h.N)) for k in STATE_IO}
        h.step(1)
        h.surface_begin()
        with pytest.raises(capi.VhError):
            h.step_host(host)
        h.surface_end()
    finally:
        h.close()
