"""The device vorticity (vh_enable_vorticity) against the reference's own
outputs (golden fixtures) and the oracle: the d_mu beta_nu every cell
stores (bit-exact: ISformal's one matrix carried through the loop order,
src/hdo.cpp:381-611, 682-727) and the beta.dat values of the freeze-out
elements (src/fld.cpp:606-831; within 1e-12 relative plus a floor for
cancellation, since the device's cosh/sinh of the Milne-to-Cartesian
Jacobian may differ from the host library's in the last bit)."""
import os

import numpy as np
import pytest

import pyoracle as P
from make_golden import load_beta_header, load_vorticity_case, read_beta
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ("vorticity_glauber_21x21x11_b9", "vorticity_glauber_nb_17x17x9",
         "vorticity_glauber_nb_chiral_17x17x9")


def beta_columns(rec, beta):
    return np.concatenate([rec[:, :16], beta, rec[:, 27:28]], axis=1)


def beta_close(a, b, rtol=1e-12, floor=1e-13):
    """Relative rtol, plus floor x the row's largest d_i beta_j magnitude
    (the Jacobian's cosh^2 and sinh^2 terms cancel in some components)."""
    scale = np.maximum(np.abs(a[:, 16:32]).max(axis=1), np.abs(b[:, 16:32]).max(axis=1))[:, None]
    tol = rtol * np.maximum(np.abs(a), np.abs(b)) + floor * scale + 1e-300
    return np.abs(a - b) <= tol


@pytest.mark.parametrize("name", CASES)
def test_gpu_dbeta_equals_reference_fixture(name):
    from vhlle_b200.capi import GpuHydro
    setup, nsteps, counts, beta_rec, db_first, db_last = load_vorticity_case(
        os.path.join(GOLDEN, name + ".npz"))
    d = GpuHydro(setup)
    d.enable_vorticity()
    got = []
    for k in range(nsteps):
        d.step(1)
        if k == 0:
            db = d.get_dbeta()
            assert np.array_equal(db, db_first, equal_nan=True), np.argwhere(db != db_first)[:5]
        rec, info, beta = d.surface_beta()
        assert info["nelements"] == counts[k], k
        got.append(beta_columns(rec, beta))
    assert np.array_equal(d.get_dbeta(), db_last, equal_nan=True)
    got = np.concatenate(got)
    assert got.shape == beta_rec.shape
    ok = beta_close(got, beta_rec)
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], beta_rec[~ok][:5])
    d.close()


@pytest.mark.parametrize("case", [
    ("glauber_41x41x21", lambda: W.small_glauber3d(41, 21, seed=3, b=6.0), 5),
    ("glauber_nb_33x33x17", lambda: W.glauber3d_nb_setup(33, 33, 17, eos=W.nb_table(200, 20)), 4),
    # EoSChiral: the k_vort_T / k_vort_ops instantiations of the chiral class
    ("glauber_nb_chiral_25x25x13", lambda: W.glauber3d_nb_setup(25, 25, 13, eos=W.chiral_eos()), 4),
], ids=lambda c: c[0])
def test_gpu_dbeta_equals_oracle(case):
    """Every step's stored dbeta bit for bit, on events whose surface and
    vacuum edges put many cells next to vacuum and many rows unwritten."""
    from vhlle_b200.capi import GpuHydro
    _, fac, nsteps = case
    setup = fac()
    o, d = P.OracleRun(setup, vorticity=True), GpuHydro(setup)
    d.enable_vorticity()
    for k in range(nsteps):
        o.step(1)
        d.step(1)
        db = d.get_dbeta()
        bad = db != o.dbeta
        bad &= ~(np.isnan(db) & np.isnan(o.dbeta))
        assert not bad.any(), (k, np.argwhere(bad)[:5])
    assert np.count_nonzero(o.dbeta) > 1000
    # the evolution itself is the plain path's
    st = d.get_state()
    so = o.get_state()
    assert np.array_equal(st["Q"], so["Q"])
    d.close()


@pytest.mark.parametrize("chain", [0, 1])
def test_gpu_dbeta_ordered_walk_equals_oracle(chain):
    """With the chain limit at 0 or 1 every run of lone increments is folded
    by the ordered walk over loop positions: the same bits as the oracle."""
    from vhlle_b200.capi import GpuHydro
    setup = W.small_glauber3d(33, 17, seed=5, b=8.0)
    o, d = P.OracleRun(setup, vorticity=True), GpuHydro(setup)
    d.enable_vorticity()
    d._check(d.L.vh_vorticity_chain(d.h, chain))
    for k in range(4):
        o.step(1)
        d.step(1)
        db = d.get_dbeta()
        bad = (db != o.dbeta) & ~(np.isnan(db) & np.isnan(o.dbeta))
        assert not bad.any(), (k, np.argwhere(bad)[:5])
    d.close()


def test_gpu_vorticity_resize_and_toggle():
    """Zero dbeta after a x2 resize, as the reference's new Fluid; turning
    vorticity off keeps the stored values and the step's results."""
    from vhlle_b200.capi import GpuHydro
    setup = W.small_glauber3d(17, 9, b=4.0, seed=11)
    o, d = P.OracleRun(setup, vorticity=True), GpuHydro(setup)
    d.enable_vorticity()
    for k in range(4):
        if k == 2:
            assert o.resize2x() == 1 and d.resize2x() == 1
            assert not d.get_dbeta().any()
        o.step(1)
        d.step(1)
        assert np.array_equal(d.get_dbeta(), o.dbeta, equal_nan=True), k
    kept = d.get_dbeta()
    d.enable_vorticity(False)
    d.step(1)
    o.step(1)
    assert np.array_equal(d.get_dbeta(), kept)
    assert np.array_equal(d.get_state()["Q"], o.get_state()["Q"])
    d.close()


def test_gpu_beta_writer_matches_reference_text(tmp_path):
    """vh_surface_write_beta: the reference's header bytes (after vh_corona)
    and its beta.dat lines."""
    from vhlle_b200.capi import GpuHydro
    path = os.path.join(GOLDEN, CASES[0] + ".npz")
    setup, nsteps, counts, beta_rec, _, _ = load_vorticity_case(path)
    ncorona, header = load_beta_header(path)
    d = GpuHydro(setup)
    d.enable_vorticity()
    out = str(tmp_path / "beta.dat")
    c, _ = d.corona()
    assert len(c) == ncorona
    d.surface_write_beta(out, header=True)  # the header only: the corona has no beta lines
    for _ in range(nsteps):
        d.step(1)
        d.surface()
        d.surface_write_beta(out)
    with open(out, "rb") as f:
        assert f.read(len(header)) == header
    back = read_beta(out)
    assert back.shape == beta_rec.shape
    assert beta_close(back, beta_rec).all()
    with open(out) as f:
        lines = f.read().splitlines()
    assert len(lines[3]) == 24 * 33
    d.close()


def test_gpu_pipelined_surface_with_vorticity_equals_blocking():
    """With vorticity on, the pipelined surface call (on its own stream, from
    the copy of Q, Qprev, pi, Pi and dbeta it takes in stream order) gives
    the blocking call's records and beta.dat values bit for bit while the
    next step runs beside it."""
    import ctypes
    from vhlle_b200.capi import GpuHydro
    setup = W.small_glauber3d(33, 17, seed=11, b=6.0)
    a, b = GpuHydro(setup), GpuHydro(setup)
    a.enable_vorticity()
    b.enable_vorticity()
    pending, checked = None, 0
    for k in range(1, 10):
        a.step(1)
        b.step(1)
        if pending is not None:
            info = b.surface_end()
            rec0, info0, beta0 = pending
            assert info == info0, (k, info, info0)
            assert np.array_equal(b.surface_records(), rec0)
            n = info["nelements"]
            beta = np.zeros((n, 16))
            got = ctypes.c_long()
            b._check(b.L.vh_surface_beta(b.h, beta.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                         n, ctypes.byref(got)))
            assert got.value == n and np.array_equal(beta, beta0)
            checked += n
            pending = None
        if k % 2 == 0:
            pending = a.surface_beta()
            b.surface_begin()
    assert checked > 500
    a.close()
    b.close()
