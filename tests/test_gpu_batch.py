"""Events advanced together (vh_batch: one CUDA graph per driver-loop
iteration, every event an independent branch, or stage-batched: one launch
per stage over a work table of every event's blocks; online autotuning of
the launch configuration) equal the same events advanced one by one with
the substep block and the resize (vh_advance, vh_resize2x): bit for bit."""
import numpy as np
import pytest

from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _events():
    return [
        (W.small_glauber3d(17, 9, seed=1, tau0=0.05, dt=0.1), 0.3),
        (W.small_glauber3d(21, 11, seed=2, b=9.0, tau0=0.1, dt=0.1), 0.6),
        (W.gubser_setup(nx=21, ny=21), 1.1),
        (W.small_glauber3d(13, 7, seed=3, tau0=0.3, dt=0.1), 10.0),
        (W.small_glauber3d(25, 5, seed=4, tau0=0.05, dt=0.1), 0.45),
    ]


def test_gpu_batch_equals_events_alone():
    from vhlle_b200.capi import Batch, GpuHydro
    nit = 24
    alone = []
    for setup, tres in _events():
        h = GpuHydro(setup)
        g = setup.grid
        resized = False
        for _ in range(nit):
            h.advance(setup.dt, g.etamin, g.etamax, g.nz)
            if h.tau >= tres and not resized:
                assert h.resize2x() == 1
                resized = True
        h.sync()
        alone.append((h.tau, h.dtau, h.grid_coords(), h.get_state()))
        h.close()

    evs = _events()
    hs = [GpuHydro(s) for s, _ in evs]
    b = Batch(hs)
    for k, (s, tres) in enumerate(evs):
        g = s.grid
        b.set_driver(k, s.dt, g.etamin, g.etamax, g.nz, tres)
    b.tune(True)
    nmax = [b.advance() for _ in range(nit)]
    assert b.sync() == 0
    assert max(nmax) > 1  # substeps happened
    info = b.info()
    assert info["captures"] >= 3 and info["nstreams"] in (0, 1, 4, 8, 16, 32)
    for k, h in enumerate(hs):
        tau, dt, gc, st = alone[k]
        assert h.tau == tau and h.dtau == dt, k
        gb = h.grid_coords()
        assert ((gb == gc) | (np.isnan(gb) & np.isnan(gc))).all(), k
        bad = compare_states(h.get_state(), st)
        assert not bad, (k, bad)
    b.close()
    for h in hs:
        h.close()


def _viscous_events():
    """3D events with substeps and resizes at different times, and 2+1D
    events of the batch set: every one viscous on an EoS1f table, so the
    stage-batched form is open to them."""
    return [
        (W.small_glauber3d(17, 9, seed=1, tau0=0.05, dt=0.1), 0.3),
        (W.small_glauber3d(21, 11, seed=2, b=9.0, tau0=0.1, dt=0.1), 0.6),
        (W.small_glauber3d(13, 7, seed=3, tau0=0.3, dt=0.1), 10.0),
        (W.small_glauber3d(25, 5, seed=4, tau0=0.05, dt=0.1), 0.45),
    ] + [(s, s.tau0 + 0.3) for s in W.batch_events(3, nz=1)]


def _alone(evs, nit, mlp=None):
    from vhlle_b200.capi import GpuHydro
    out = []
    for setup, tres in evs:
        h = GpuHydro(setup)
        if mlp is not None:
            h.set_con2prim_guess(mlp)
        g = setup.grid
        resized = False
        for _ in range(nit):
            h.advance(setup.dt, g.etamin, g.etamax, g.nz)
            if h.tau >= tres and not resized:
                assert h.resize2x() == 1
                resized = True
        h.sync()
        out.append((h.tau, h.dtau, h.grid_coords(), h.get_state()))
        h.close()
    return out


@pytest.mark.parametrize("with_mlp", [False, True], ids=["plain", "learned_guess"])
def test_gpu_stage_batched_equals_events_alone(with_mlp):
    """The stage-batched form (vh_batch_set_mode(b, 1)): per substep index
    one launch per stage over every event's blocks, events with fewer
    substeps dropping out of the later tables; with and without a learned
    start point attached to every context."""
    from vhlle_b200.capi import Batch, GpuHydro, Mlp
    nit = 16
    mlp = Mlp(seed=3) if with_mlp else None
    alone = _alone(_viscous_events(), nit, mlp)
    evs = _viscous_events()
    hs = [GpuHydro(s) for s, _ in evs]
    for h in hs:
        if mlp is not None:
            h.set_con2prim_guess(mlp)
    b = Batch(hs)
    for k, (s, tres) in enumerate(evs):
        g = s.grid
        b.set_driver(k, s.dt, g.etamin, g.etamax, g.nz, tres)
    b.set_mode(True)
    nmax = [b.advance() for _ in range(nit)]
    assert b.sync() == 0
    assert max(nmax) > 1 and b.info()["nstreams"] == 0
    for k, h in enumerate(hs):
        tau, dt, gc, st = alone[k]
        assert h.tau == tau and h.dtau == dt, k
        gb = h.grid_coords()
        assert ((gb == gc) | (np.isnan(gb) & np.isnan(gc))).all(), k
        bad = compare_states(h.get_state(), st)
        assert not bad, (k, bad)
    b.close()
    for h in hs:
        h.close()
    if mlp is not None:
        mlp.close()


def test_gpu_stage_batched_needs_one_class():
    """Events of different viscosity (the ideal Gubser flow beside viscous
    ones) cannot share stage launches: set_mode(True) is refused and the
    tuner keeps to the branch form."""
    from vhlle_b200.capi import Batch, GpuHydro, VhError
    hs = [GpuHydro(W.small_glauber3d(13, 5)), GpuHydro(W.gubser_setup(nx=21, ny=21))]
    b = Batch(hs)
    with pytest.raises(VhError):
        b.set_mode(True)
    b.close()
    for h in hs:
        h.close()


def test_gpu_batch_rejects_bad_input():
    from vhlle_b200.capi import Batch, GpuHydro, VhError
    h = GpuHydro(W.small_glauber3d(11, 5))
    with pytest.raises(VhError):
        Batch([h, h])
    h.close()


def test_gpu_zeta_bump_event_against_oracle():
    """A batch event with the zeta/s bump (zetaSparam 5) against the oracle.
    The bump uses exp, where the device and glibc may differ in the last bit;
    the oracle alone, with the bump height moved by one ulp, differs from
    itself by ~1e-16 of each field's scale after 5 steps (more at the vacuum
    edge later on).  Tolerance: 1e-10 relative plus 1e-12 of the field's
    largest magnitude, after one step and after five."""
    import pyoracle as P
    from vhlle_b200.capi import GpuHydro
    setup = W.batch_event(1, nz=9)
    o, d = P.OracleRun(setup), GpuHydro(setup)

    def check():
        got, exp = gpu_state_as_oracle(d.get_state()), o.get_state()
        for k in exp:
            a = np.asarray(got[k], dtype=np.float64).reshape(-1)
            b = np.asarray(exp[k], dtype=np.float64).reshape(-1)
            scale = np.abs(b).max()
            ok = np.abs(a - b) <= 1e-10 * np.maximum(np.abs(a), np.abs(b)) + 1e-12 * scale
            assert ok.all(), (k, np.argwhere(~ok)[:5])
        return exp

    o.step(1)
    d.step(1)
    check()
    o.step(4)
    d.step(4)
    exp = check()
    assert np.abs(exp["Pi"]).max() > 0  # the bump drives bulk pressure
    d.close()


def test_gpu_batch_of_c3_events_runs_and_tunes():
    from vhlle_b200.capi import Batch, GpuHydro
    evs = W.batch_events(12)
    hs = [GpuHydro(s) for s in evs]
    b = Batch(hs)
    for k, s in enumerate(evs):
        g = s.grid
        b.set_driver(k, s.dt, g.etamin, g.etamax, g.nz, 4.0)
    b.tune(True)
    b.advance(20)
    assert b.sync() == 0
    assert all(abs(h.tau - (0.5 + 20 * 0.05)) < 1e-12 for h in hs)
    b.close()
    for h in hs:
        h.close()
