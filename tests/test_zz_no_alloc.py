"""vh_step_noalloc: the allocation-free step for callers that cannot let a
library allocate device memory (their memory is reserved by their own pool
or by another framework's allocator, or allocation is forbidden inside their
time loop).  The caller owns every array; the test allocates them with
torch, as such a caller would with its own allocator, and checks two calls
in a row against the regular context-based step (vh_create / vh_step) with
the parity tolerance of the other GPU tests: 1e-12 relative, and then bit
for bit.

This file is named to be collected last, so that a run stopping at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from helpers import compare_states
from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu

FIELDS = capi.STATE_FIELDS


def _device_state(torch, setup):
    N = setup.grid.ncells
    Q = np.ascontiguousarray(setup.Q, dtype=np.float64).reshape(7, N)
    host = {
        "Q": Q, "Qh": np.zeros((7, N)), "Qprev": Q.copy(), "pi": np.zeros((10, N)),
        "piH": np.zeros((10, N)), "Pi": np.zeros((1, N)), "PiH": np.zeros((1, N)),
        "m": np.repeat(np.asarray(setup.m, dtype=np.float64).reshape(1, N), 3, 0),
        "viscCorrCut": np.ones((1, N)),
    }
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in host.items()}


def _device_eos(torch, eos):
    d = capi.VhEos()
    d.kind = eos.kind
    d.conf_cnst = eos.conf_cnst
    keep = []
    if eos.kind == 1:
        keep = [torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
                for a in (eos.egrid, eos.ngrid, eos.p, eos.T, eos.mub)]
        d.ne, d.nn = len(eos.egrid), len(eos.ngrid)
        dp = ctypes.POINTER(ctypes.c_double)
        d.egrid, d.ngrid, d.p, d.T, d.mub = (ctypes.cast(t.data_ptr(), dp) for t in keep)
    if eos.kind == 2:  # EoSChiral: both tables' planes on the device
        dp = ctypes.POINTER(ctypes.c_double)
        for k, a in enumerate(eos.aux):
            ts = [torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()
                  for x in (a.p, a.T, a.mub, a.mus)]
            keep += ts
            x = d.aux[k]
            x.ne, x.nn, x.emin, x.emax, x.nmin, x.nmax = a.ne, a.nn, a.emin, a.emax, a.nmin, a.nmax
            x.p, x.T, x.mub, x.mus = (ctypes.cast(t.data_ptr(), dp) for t in ts)
    return d, keep


def _noalloc_step(L, setup, eos_d, dev, tau):
    g = setup.grid
    grid = capi.VhGrid(g.nx, g.ny, g.nz, *g.bounds())
    tr = capi.make_trcoeff(setup)
    view = capi.VhStateView()
    for k, t in dev.items():
        setattr(view, k, t.data_ptr())
    bits = ctypes.c_uint(123)
    st = L.vh_step_noalloc(ctypes.byref(grid), ctypes.byref(eos_d), ctypes.byref(tr), tau,
                           setup.dt, ctypes.byref(view), None, ctypes.byref(bits))
    return st, bits.value


@pytest.mark.parametrize("make", [lambda: W.small_glauber3d(21, 11),
                                  lambda: W.gubser_setup(nx=31, ny=31),
                                  lambda: W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos())],
                         ids=["viscous_21x21x11", "gubser_31x31", "chiral_nb_17x17x9"])
def test_noalloc_step_matches_the_context_step_twice(make):
    torch = pytest.importorskip("torch")
    setup = make()
    L = capi.lib()
    # the set-up a caller does before reserving its own memory pool
    assert L.vh_noalloc_prepare(0) == capi.VH_OK, L.vh_noalloc_last_error().decode()
    ref = capi.GpuHydro(setup)
    dev = _device_state(torch, setup)
    eos_d, keep = _device_eos(torch, setup.eos)
    torch.cuda.synchronize()
    tau = setup.tau0
    for call in range(2):
        ref.step(1)
        ref.sync()
        expect = ref.get_state()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st, bits = _noalloc_step(L, setup, eos_d, dev, tau)
        assert st == capi.VH_OK, L.vh_noalloc_last_error().decode()
        # after vh_noalloc_prepare the call takes no device memory at all
        assert torch.cuda.mem_get_info()[0] == free_before, call
        assert bits == 0
        tau = tau + setup.dt
        assert ref.tau == tau
        got = {k: t.cpu().numpy() for k, t in dev.items()}
        bad = compare_states(got, expect, FIELDS, rtol=1e-12)
        assert not bad, (call, bad)
        bad = compare_states(got, expect, FIELDS)
        assert not bad, (call, bad)
    ref.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    setup = W.small_glauber3d(41, 21)  # 35301 cells > 32768
    L = capi.lib()
    eos_d, keep = _device_eos(torch, setup.eos)
    dev = _device_state(torch, W.small_glauber3d(5, 5))  # never touched: rejected first
    st, bits = _noalloc_step(L, setup, eos_d, dev, setup.tau0)
    assert st == capi.VH_ERR_ARG
    assert b"VH_NOALLOC_MAX_CELLS" in L.vh_noalloc_last_error()
