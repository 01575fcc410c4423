"""The device builders of the reference's initial-state modules
(vh_init_glissando, vh_init_trento, vh_init_gubser, vh_init_table) against
the C restatement and the compiled reference modules (IcGlissando, IcTrento,
ICGubser, IC: src/icGlissando.cpp, src/icTrento.cpp, src/icGubser.cpp,
src/ic.cpp), on seeded synthetic inputs in the modules' file formats.

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


def test_gpu_ic_refused_on_a_slab(grid_setup):
    h = capi.GpuHydro(grid_setup, upload=False)
    try:
        h.set_slab(2, grid_setup.grid.nz - 2, 4, grid_setup.grid.nz + 8)
        with pytest.raises(capi.VhError) as e:
            h.init_gubser()
        assert e.value.args[0].startswith("vhlle_b200 status %d" % capi.VH_ERR_STATE)
    finally:
        h.close()
