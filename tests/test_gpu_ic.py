"""The device initial-state builder (vh_init_glauber) against the host
generator every workload uses (workloads.glauber_profile + glauber3d_setup:
the same participants, the same smearing sum in participant order, the same
normalisation, cut and Cell::setPrimVar at rest, the last pinned to the
reference's own function by tests/test_ic_entry.py).

Tolerance: the device's exp is correctly rounded, NumPy's is within an ulp,
so each smeared term may differ in its last bit: the conserved fields agree
to 1e-14 relative (sums of a few hundred terms), the vacuum mask exactly
except at cells within 1e-12 of the cut; the steps from the device-built
state then match the host-built ones to 1e-10."""
import time

import numpy as np
import pytest

from vhlle_b200 import capi
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device_ic(setup, seed, b, epeak=50.0, nb_peak=0.0, ecut=1e-3):
    h = capi.GpuHydro(setup, upload=False)
    _, _, eta = setup.grid.coords()
    H = W.eta_profile(eta) if setup.grid.nz > 1 else np.ones(1)
    h.init_glauber(W.glauber_participants(seed, b), H, epeak=epeak, ecut=ecut, nb_peak=nb_peak)
    return h


def _check_ic(st, setup):
    Q = setup.Q.reshape(7, -1)
    near_cut = np.abs(Q[0] / setup.tau0 - 1e-3) <= 1e-12
    got = st["Q"]
    for k in range(7):
        a, b = got[k][~near_cut], Q[k][~near_cut]
        ok = np.abs(a - b) <= 1e-14 * np.maximum(np.abs(a), np.abs(b))
        assert ok.all(), (k, np.argwhere(~ok)[:5])
    return near_cut


@pytest.mark.parametrize("case", [
    ("glauber_101x101x51", dict(seed=20260001, b=7.0), lambda: W.glauber3d_setup()),
    ("glauber_nb_41x41x21", dict(seed=20260001, b=7.0, nb_peak=0.3),
     lambda: W.glauber3d_nb_setup(41, 41, 21, eos=W.nb_table(200, 20))),
    ("large_61x61x31_b3", dict(seed=20265000, b=3.0, epeak=80.0, nb_peak=0.3),
     lambda: W.large_event_setup(0, 61, 61, 31, eos=W.nb_table(200, 20))),
], ids=lambda c: c[0])
def test_device_ic_equals_host_generator(case):
    _, kw, fac = case
    setup = fac()
    h = _device_ic(setup, **kw)
    st = h.get_state()
    near_cut = _check_ic(st, setup)
    m = (setup.Q.reshape(7, -1)[0] > 0).astype(float)
    assert np.array_equal(st["m"][0][~near_cut], m[~near_cut])
    assert np.array_equal(st["Qprev"], st["Q"]) and not st["pi"].any()
    assert (st["viscCorrCut"] == 1).all() and (st["Q"][0] > 0).sum() > 1000
    h.close()


def test_device_ic_evolves_like_the_host_ic():
    """Ten viscous steps from the device-built state and from the host one."""
    setup = W.small_glauber3d(33, 17, seed=11, b=6.0)
    a = _device_ic(setup, seed=11, b=6.0)
    b = capi.GpuHydro(setup)
    a.step(10)
    b.step(10)
    sa, sb = a.get_state(("Q", "pi", "Pi")), b.get_state(("Q", "pi", "Pi"))
    for k in sa:
        scale = np.abs(sb[k]).max()
        ok = np.abs(sa[k] - sb[k]) <= 1e-10 * np.maximum(np.abs(sa[k]), np.abs(sb[k])) + 1e-12 * scale
        assert ok.all(), (k, np.argwhere(~ok)[:5])
    a.close()
    b.close()


def test_device_ic_builds_the_event_set_faster_than_the_host():
    """The event-by-event set's first 32 events (2+1D and 3D) built on the
    device (participants from the host stream) against the host generator:
    the same states, in less time."""
    t0 = time.perf_counter()
    evs = W.batch_events(32)
    t_host = time.perf_counter() - t0
    hs = [capi.GpuHydro(s, upload=False) for s in evs]
    bs = np.random.default_rng(W.BATCH_SEED0).uniform(0.0, 12.0, 32)
    t0 = time.perf_counter()
    for k, (h, s) in enumerate(zip(hs, evs)):
        _, _, eta = s.grid.coords()
        H = W.eta_profile(eta) if s.grid.nz > 1 else np.ones(1)
        h.init_glauber(W.glauber_participants(W.BATCH_SEED0 + k, float(bs[k])), H)
    t_dev = time.perf_counter() - t0
    print("32 events: host generator %.3f s, device builder %.3f s" % (t_host, t_dev))
    for h, s in zip(hs, evs):
        _check_ic(h.get_state(("Q",)), s)
        h.close()
    assert t_dev < t_host
