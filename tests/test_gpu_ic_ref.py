"""The device builders of the reference's initial-state modules
(vh_init_glissando, vh_init_trento, vh_init_gubser, vh_init_table,
vh_init_urqmd) against the C restatement and the compiled reference modules
(IcGlissando, IcTrento, ICGubser, IC, IcPartUrqmd: src/icGlissando.cpp,
src/icTrento.cpp, src/icGubser.cpp, src/ic.cpp, src/icPartUrqmd.cpp), on
seeded synthetic inputs in the modules' file formats.

The device evaluates exp and pow correctly rounded (crm::exp_cr, pow_cr):
against the oracle's crmath arm every cell is bit-identical (Q, Qprev, m, the
zeroed viscous fields) and so are the normalisations; against the reference
(the C library's exp and pow, which misround about one pow call in a
thousand by one ulp) the conserved fields agree to 1e-14 relative, the fill
fractions exactly."""
import time

import numpy as np
import pytest

from oracle import pyoracle as P
from vhlle_b200 import capi
from vhlle_b200 import ic_files as F
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu

GLISSANDO_SETUPS = ("LHC276", "RHIC200", "LHC5020", "RHIC62", "AFTER72", "RHIC27")
TRENTO_SETUPS = ("LHC276", "RHIC200", "LHC5020", "RHIC62", "RHIC27")


@pytest.fixture(scope="module")
def grid_setup():
    return W.glauber3d_setup(nx=31, ny=31, nz=11, xmax=12.0, etamax=6.0)


def _device(setup, init):
    h = capi.GpuHydro(setup, upload=False)
    try:
        out = init(h)
        return h.get_state(), out
    finally:
        h.close()


def _equal_oracle(st, o):
    assert np.array_equal(st["Q"], o["Q"])
    assert np.array_equal(st["Qprev"], o["Qprev"])
    assert np.array_equal(st["m"], o["m"])
    for k in ("Qh", "pi", "piH", "Pi", "PiH"):
        assert not st[k].any(), k
    assert (st["viscCorrCut"] == 1.0).all()


def _close_ref(st, r, rtol=1e-14):
    Q = r["Q"]
    scale = np.maximum(np.abs(Q).max(axis=1, keepdims=True), 1e-300)
    assert np.all(np.abs(st["Q"] - Q) <= rtol * np.maximum(np.abs(Q), 1e-3 * scale))
    assert np.array_equal(st["m"][0], r["m"])


@pytest.mark.parametrize("name", GLISSANDO_SETUPS)
def test_gpu_glissando_equals_oracle_and_reference(name, grid_setup, tmp_path):
    path = str(tmp_path / "sources.txt")
    F.write_glissando(path, F.synthetic_glissando_events(3, seed=5))
    ev = F.read_glissando(path)
    su = capi.ic_setup(capi.IC_GLISSANDO, name)
    st, norms = _device(grid_setup, lambda h: h.init_glissando(ev, su))
    o, on = P.oracle_ic(grid_setup, 5, ev, su, crmath=True)
    assert norms == on
    _equal_oracle(st, o)
    if P.ref_available():
        ref = P.RefRun(grid_setup)
        try:
            _close_ref(st, ref.ic(5, path, name))
        finally:
            ref.close()


@pytest.mark.parametrize("name", TRENTO_SETUPS)
def test_gpu_trento_equals_oracle_and_reference(name, grid_setup, tmp_path):
    path = str(tmp_path / "trento.dat")
    F.write_trento(path, F.synthetic_trento_events(2, seed=7, n=60))
    ev = F.read_trento(path)
    su = capi.ic_setup(capi.IC_TRENTO, name)
    st, norms = _device(grid_setup, lambda h: h.init_trento(ev, su))
    o, on = P.oracle_ic(grid_setup, 7, ev, su, crmath=True)
    assert norms == on
    _equal_oracle(st, o)
    if P.ref_available():
        ref = P.RefRun(grid_setup)
        try:
            _close_ref(st, ref.ic(7, path, name))
        finally:
            ref.close()


def test_gpu_gubser_equals_oracle_and_reference(grid_setup):
    st, _ = _device(grid_setup, lambda h: h.init_gubser())
    o, _ = P.oracle_ic(grid_setup, 4, crmath=True)
    _equal_oracle(st, o)
    if P.ref_available():
        ref = P.RefRun(grid_setup)
        try:
            _close_ref(st, ref.ic(4))
        finally:
            ref.close()


@pytest.mark.parametrize("gv", [1, 0])
def test_gpu_table_equals_oracle_and_reference(gv, grid_setup, tmp_path):
    path = str(tmp_path / "table.dat")
    F.synthetic_song_table().write(path)
    tab = F.read_song_table(path)
    factor = 1.0 if gv == 1 else 8.0
    st, _ = _device(grid_setup, lambda h: h.init_table(tab, factor, gv))
    o, _ = P.oracle_ic(grid_setup, 2, tab, factor=factor, glauber_var=gv, crmath=True)
    _equal_oracle(st, o)
    if P.ref_available():
        ref = P.RefRun(grid_setup)
        try:
            _close_ref(st, ref.ic(2, path, "", factor, gv))
        finally:
            ref.close()


@pytest.mark.parametrize("Rgt,Rgz", [(1.0, 1.0), (0.8, 0.0)])
def test_gpu_urqmd_equals_oracle_and_reference(Rgt, Rgz, grid_setup, tmp_path):
    """IcPartUrqmd (icModel 3): the per-cell transformPV amplifies the
    smearing's last-bit exp differences, hence 1e-13 against the
    reference."""
    path = str(tmp_path / "particles.txt")
    F.write_urqmd(path, F.synthetic_urqmd_events(3, seed=5, nmean=300))
    ev = F.read_urqmd(path)
    st, _ = _device(grid_setup, lambda h: h.init_urqmd(ev, Rgt, Rgz))
    o, _ = P.oracle_ic(grid_setup, 3, ev, Rgt=Rgt, Rgz=Rgz, crmath=True)
    _equal_oracle(st, o)
    if P.ref_available():
        ref = P.RefRun(grid_setup)
        try:
            _close_ref(st, ref.ic(3, path, Rgt=Rgt, Rgz=Rgz), rtol=1e-13)
        finally:
            ref.close()


def test_gpu_glissando_full_grid_equals_oracle(tmp_path):
    """The 101x101x51 grid with 10 RHIC62 events (baryon density on): bit
    for bit the oracle's crmath arm; the device and reference times are
    printed."""
    setup = W.glauber3d_setup()
    path = str(tmp_path / "sources.txt")
    F.write_glissando(path, F.synthetic_glissando_events(10, seed=11))
    ev = F.read_glissando(path)
    su = capi.ic_setup(capi.IC_GLISSANDO, "RHIC62")
    h = capi.GpuHydro(setup, upload=False)
    try:
        h.init_glissando(ev, su)  # first call: module load
        t0 = time.perf_counter()
        norms = h.init_glissando(ev, su)
        t_dev = time.perf_counter() - t0
        st = h.get_state()
    finally:
        h.close()
    t0 = time.perf_counter()
    o, on = P.oracle_ic(setup, 5, ev, su, crmath=True)
    t_or = time.perf_counter() - t0
    assert norms == on
    _equal_oracle(st, o)
    msg = "IcGlissando 101x101x51, %d sources: device %.4f s, oracle %.2f s" % (
        len(ev.x), t_dev, t_or)
    if P.ref_available():
        ref = P.RefRun(setup)
        try:
            t0 = time.perf_counter()
            r = ref.ic(5, path, "RHIC62")
            msg += ", reference %.2f s" % (time.perf_counter() - t0)
            _close_ref(st, r)
        finally:
            ref.close()
    print(msg)


def test_gpu_urqmd_full_grid_equals_oracle(tmp_path):
    """IcPartUrqmd on the 101x101x51 grid, 10 events of ~400 particles,
    Rgt = Rgz = 1 (a 41 x 41 x 11 stencil per particle): bit for bit the
    oracle's crmath arm; the device and reference times are printed."""
    setup = W.glauber3d_setup()
    path = str(tmp_path / "particles.txt")
    F.write_urqmd(path, F.synthetic_urqmd_events(10, seed=13))
    ev = F.read_urqmd(path)
    h = capi.GpuHydro(setup, upload=False)
    try:
        h.init_urqmd(ev, 1.0, 1.0)  # first call: module load
        t0 = time.perf_counter()
        h.init_urqmd(ev, 1.0, 1.0)
        t_dev = time.perf_counter() - t0
        st = h.get_state()
    finally:
        h.close()
    o, _ = P.oracle_ic(setup, 3, ev, Rgt=1.0, Rgz=1.0, crmath=True)
    _equal_oracle(st, o)
    msg = "IcPartUrqmd 101x101x51, %d particles: device %.4f s" % (len(ev.id), t_dev)
    if P.ref_available():
        ref = P.RefRun(setup)
        try:
            t0 = time.perf_counter()
            r = ref.ic(3, path, Rgt=1.0, Rgz=1.0)
            msg += ", reference %.2f s" % (time.perf_counter() - t0)
            _close_ref(st, r, rtol=1e-13)
        finally:
            ref.close()
    print(msg)


def test_gpu_ic_refused_on_a_slab(grid_setup):
    h = capi.GpuHydro(grid_setup, upload=False)
    try:
        h.set_slab(2, grid_setup.grid.nz - 2, 4, grid_setup.grid.nz + 8)
        with pytest.raises(capi.VhError) as e:
            h.init_gubser()
        assert e.value.args[0].startswith("vhlle_b200 status %d" % capi.VH_ERR_STATE)
    finally:
        h.close()


@pytest.mark.parametrize("model", [5, 7, 4, 3])
def test_gpu_driver_builds_the_reference_ic(model, grid_setup, tmp_path):
    """vhlle_run with icModel 5 (IcGlissando), 7 (IcTrento), 4 (ICGubser) or
    3 (IcPartUrqmd, Rgt = Rgz = 1 by default):
    the initial state built on the device (the printed sNorm is the
    oracle's), then the corona at tau0 equals the oracle's on that state."""
    import dataclasses
    import subprocess
    from vhlle_b200 import build as B
    drv = B.build_driver()
    setup = grid_setup
    extra = dict(icModel=model, tauMax=setup.tau0 + setup.dt, eos1fFile=str(tmp_path / "eos.dat"))
    setup.eos.write_eos1f(str(tmp_path / "eos.dat"))
    args = []
    if model == 5:
        path = str(tmp_path / "sources.txt")
        F.write_glissando(path, F.synthetic_glissando_events(3, seed=5))
        o, norms = P.oracle_ic(setup, 5, F.read_glissando(path),
                               capi.ic_setup(capi.IC_GLISSANDO, "RHIC200"), crmath=True)
        args = ["-ISinput", path, "-system", "RHIC200"]
    elif model == 7:
        path = str(tmp_path / "trento.dat")
        F.write_trento(path, F.synthetic_trento_events(2, seed=7, n=60))
        o, norms = P.oracle_ic(setup, 7, F.read_trento(path),
                               capi.ic_setup(capi.IC_TRENTO, "RHIC62"), crmath=True)
        args = ["-ISinput", path, "-system", "RHIC62"]
    elif model == 3:
        path = str(tmp_path / "particles.txt")
        F.write_urqmd(path, F.synthetic_urqmd_events(3, seed=5, nmean=300))
        o, norms = P.oracle_ic(setup, 3, F.read_urqmd(path), Rgt=1.0, Rgz=1.0, crmath=True)
        args = ["-ISinput", path]
    else:
        o, norms = P.oracle_ic(setup, 4, crmath=True)
    params = str(tmp_path / "params.txt")
    W.write_params(params, setup, **extra)
    out = tmp_path / "out"
    run = subprocess.run([drv, "-params", params, *args, "-outputDir", str(out)],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr
    if model in (5, 7):
        assert "sNorm set to %.17g" % norms[0] in run.stdout, run.stdout[-1500:]
    ic_setup = dataclasses.replace(setup, Q=o["Q"], m=o["m"][0].copy())
    corona, _ = P.OracleRun(ic_setup).corona()
    assert "corona elements : %d" % len(corona) in run.stdout, run.stdout[-1500:]
