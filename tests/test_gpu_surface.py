"""The device freeze-out surface (Cornelius 4D per hypercube and the element
records of Fluid::outputSurface, src/fld.cpp:606-842) against the
reference's own outputs (golden fixtures) and the oracle.

Tolerances: element counts, nsusp and the element order are exact; records
within 1e-12 relative (the fixtures hold the reference's 15-digit text, and
the device's cosh/sinh/log/tanh may differ from the host's in the last bit);
Cornelius centroids and normals on given hypercubes bit-exact; the summed
EtotSurf / nbSurf / vEff within 1e-10 of the sum of their magnitudes
(summation order differs)."""
import os

import numpy as np
import pytest

import pyoracle as P
from make_golden import load_surface_case
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REC_RTOL = 1e-12


def rec_close(a, b, rtol=REC_RTOL):
    return np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + 1e-300


def test_gpu_cornelius_equals_reference_cubes():
    from vhlle_b200.capi import cornelius4d
    z = np.load(os.path.join(GOLDEN, "cornelius_cubes.npz"))
    counts, cent, norm = cornelius4d(z["cubes"], z["dx"], float(z["e0"]))
    assert np.array_equal(counts, z["counts"])
    k = 0
    for i, n in enumerate(z["counts"]):
        assert np.array_equal(cent[i, :n], z["cent"][k:k + n]), i
        assert np.array_equal(norm[i, :n], z["norm"][k:k + n]), i
        k += n


def test_gpu_cornelius_equals_oracle_random():
    from vhlle_b200.capi import cornelius4d
    rng = np.random.default_rng(31)
    cubes = np.concatenate([rng.uniform(0, 1, (3000, 16)),
                            rng.choice([0.1, 0.9], (3000, 16)) + rng.uniform(-0.02, 0.02, (3000, 16)),
                            rng.choice([0.2, 0.5, 0.8], (2000, 16))])
    dx = np.array([0.05, 0.6, 0.6, 0.3])
    counts, cent, norm = cornelius4d(cubes, dx, 0.5)
    for i, c in enumerate(cubes):
        co, no = P.cornelius4d(c, dx, 0.5)
        if co is None:
            assert counts[i] == -1
            continue
        assert counts[i] == len(co), i
        assert np.array_equal(cent[i, :len(co)], co) and np.array_equal(norm[i, :len(co)], no), i


def test_gpu_surface_equals_reference_fixture():
    from vhlle_b200.capi import GpuHydro
    setup, nsteps, counts, rec, lines = load_surface_case(
        os.path.join(GOLDEN, "surface_glauber_21x21x11_b9.npz"))
    d = GpuHydro(setup)
    got = []
    for s in range(nsteps):
        d.step(1)
        r, info = d.surface()
        assert info["nelements"] == counts[s], s
        words = lines[s].split()
        assert int(words[7]) == info["nsusp"], s
        assert abs(info["EtotSurf"] - float(words[5])) <= 5e-6 * abs(info["EtotSurf"]) + 1e-9
        got.append(r)
    got = np.concatenate(got)
    ok = rec_close(got, rec)
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], rec[~ok][:5])
    d.close()


@pytest.mark.parametrize("case", [
    ("glauber_33x33x17", lambda: W.small_glauber3d(33, 17, seed=11, b=6.0), 6),
    ("gubser_2d_no_interior", lambda: W.gubser_setup(nx=21, ny=21), 2),
], ids=lambda c: c[0])
def test_gpu_surface_equals_oracle(case):
    from vhlle_b200.capi import GpuHydro
    name, fac, nsteps = case
    setup = fac()
    o, d = P.OracleRun(setup), GpuHydro(setup)
    sums = {"EtotSurf": 0., "nbSurf": 0., "vEff": 0.}
    mags = {"EtotSurf": 0., "nbSurf": 0., "vEff": 0.}
    for s in range(nsteps):
        o.step(1)
        d.step(1)
        ro, acc = o.surface()
        rd, info = d.surface()
        assert len(ro) == info["nelements"] and int(acc["nsusp"]) == info["nsusp"], s
        ok = rec_close(rd, ro)
        assert ok.all(), (s, np.argwhere(~ok)[:5])
        for k in sums:
            sums[k] += acc[k]
            mags[k] += np.abs(acc[k])
            assert abs(info[k] - sums[k]) <= 1e-10 * (mags[k] + 1e-30) + 1e-300, (k, info[k], sums[k])
    d.close()


def test_gpu_surface_full_size_event():
    """The 101x101x51 event after 3 steps: every element and the sums as
    the oracle's."""
    from vhlle_b200.capi import GpuHydro
    setup = W.glauber3d_setup()
    o, d = P.OracleRun(setup), GpuHydro(setup)
    o.step(3)
    d.step(3)
    ro, acc = o.surface(cap=2000000)
    rd, info = d.surface()
    assert len(ro) == info["nelements"] > 1000
    ok = rec_close(rd, ro)
    assert ok.all(), np.argwhere(~ok)[:5]
    assert int(acc["nsusp"]) == info["nsusp"]
    assert abs(info["EtotSurf"] - acc["EtotSurf"]) <= 1e-10 * abs(acc["EtotSurf"]) + 1e-6
    d.close()


def test_gpu_surface_writer_matches_reference_text(tmp_path):
    """vh_surface_write emits the reference's freezeout.dat layout."""
    from vhlle_b200.capi import GpuHydro
    setup, nsteps, counts, rec, lines = load_surface_case(
        os.path.join(GOLDEN, "surface_glauber_21x21x11_b9.npz"))
    d = GpuHydro(setup)
    path = str(tmp_path / "freezeout.dat")
    for _ in range(nsteps):
        d.step(1)
        d.surface()
        d.surface_write(path, extend=True)
    back = P.read_freezeout(path, extend=True)
    assert back.shape == rec.shape
    assert rec_close(back, rec, 1e-13).all()
    with open(path) as f:
        first = f.readline()
    assert len(first.rstrip("\n")) == 24 * 29
    d.close()


def _ripple_setup(n=81, nz=41, lam=4.0):
    """A smooth triply periodic level set e = e_f crossing most hypercubes of
    an 81x81x41 grid (about 200k elements), so that one surface call holds
    more straddling cubes than vh_surface's first buffers (64k cubes)."""
    g = W.Grid(n, n, nz, -15, 15, -15, 15, -7.5, 7.5)
    x, y, eta = g.coords()
    Z, Y, X = np.meshgrid(eta, y, x, indexing="ij")
    k = 2 * np.pi / lam
    e = 0.5 * (0.97 + 0.2 * (np.sin(k * X / g.dx) + np.sin(k * Y / g.dy) + np.sin(k * Z / g.dz + 0.3)))
    zero = np.zeros_like(e)
    Q = W.conserved_from_primitive(0.5, e, zero, zero, zero, zero, zero).reshape(7, -1)
    tr = dict(W.TR_DEFAULTS, etaS0=0.08, zetaS0=0.0)
    return W.Setup("ripple", g, W.make_cs2_table(), tr, 0, 0, 0.5, 0.05, 0.5, Q,
                   np.ones(g.ncells))


def test_gpu_surface_grows_past_first_capacity():
    """A call with more straddling cubes than the first buffers hold grows
    them and runs again; that call and the next (on the grown buffers) give
    the oracle's elements."""
    from vhlle_b200.capi import GpuHydro
    setup = _ripple_setup()
    o, d = P.OracleRun(setup), GpuHydro(setup)
    for s in range(2):
        o.step(1)
        d.step(1)
        ro, acc = o.surface(cap=4000000)
        rd, info = d.surface()
        assert len(ro) == info["nelements"] > 150000, s
        ok = rec_close(rd, ro)
        assert ok.all(), (s, np.argwhere(~ok)[:5])
        assert int(acc["nsusp"]) == info["nsusp"]
    d.close()


def test_gpu_pipelined_surface_past_capacity_loses_nothing():
    """A pipelined call (vh_surface_begin, the next step queued, then
    vh_surface_end) that finds more straddling cubes than the first buffers
    hold keeps its inputs on the device and runs again at surface_end: its
    elements are the oracle's at the call's tau, although the grid has
    moved on by then; the next pipelined call runs on the grown buffers."""
    from vhlle_b200.capi import GpuHydro
    setup = _ripple_setup()
    o, d = P.OracleRun(setup), GpuHydro(setup)
    for s in range(2):
        o.step(1)
        d.step(1)
        ro, acc = o.surface(cap=4000000)
        d.surface_begin()
        d.step(1)  # queued behind the call's pass; runs before surface_end waits
        info = d.surface_end()
        rd = d.surface_records()
        # the first call finds more than the first buffers' 128k elements
        assert len(ro) == info["nelements"] > (150000 if s == 0 else 100000), s
        ok = rec_close(rd, ro)
        assert ok.all(), (s, np.argwhere(~ok)[:5])
        assert int(acc["nsusp"]) == info["nsusp"]
        o.step(1)
    d.close()


def test_gpu_grid_changes_refused_while_surface_pending():
    """vh_resize2x, vh_upload_state and vh_enable_vorticity return
    VH_ERR_STATE between vh_surface_begin and vh_surface_end (the reference
    takes the old Fluid's surface before a resize replaces it); after the
    call ends they run."""
    from vhlle_b200.capi import GpuHydro, VhError
    setup = W.small_glauber3d(21, 11, b=9.0, seed=5)
    d = GpuHydro(setup)
    d.step(2)
    d.surface_begin()
    for call in (d.resize2x, d.upload_initial, lambda: d.enable_vorticity(True)):
        with pytest.raises(VhError) as e:
            call()
        assert e.value.status == 4 and "has not ended" in str(e.value)
    info = d.surface_end()
    o = P.OracleRun(setup)
    o.step(2)
    ro, _ = o.surface()
    assert info["nelements"] == len(ro)
    assert d.resize2x() == 1
    d.close()


@pytest.mark.parametrize("name", ["corona_glauber_41x41x21", "corona_glauber_nb_25x25x13"])
def test_gpu_corona_equals_reference_fixture(name, tmp_path):
    """vh_corona at tau0 against the reference's outputCorona: element
    count, records (15 printed digits, device cosh/sinh/log/tanh within the
    last bit) and EtotSurf; vh_surface_write then writes those records."""
    from make_golden import load_corona_case
    from vhlle_b200.capi import GpuHydro
    setup, n, rec, line = load_corona_case(os.path.join(GOLDEN, name + ".npz"))
    d = GpuHydro(setup)
    got, info = d.corona()
    assert info["nelements"] == n > 0 and info["nsusp"] == 0
    ok = rec_close(got, rec)
    assert ok.all(), np.argwhere(~ok)[:5]
    assert abs(info["EtotSurf"] - float(line.split()[5])) <= 5e-6 * abs(info["EtotSurf"])
    path = str(tmp_path / "freezeout.dat")
    d.surface_write(path, extend=True)
    assert rec_close(P.read_freezeout(path, extend=True), rec, 1e-13).all()
    d.close()


def rec_close_scaled(a, b, rtol=REC_RTOL, floor=1e-13):
    """rec_close with two allowances for the amplification of a last-bit
    difference between the device's cosh/sinh/log/tanh and the host
    library's (transformToLab, pi^{mu nu} to Cartesian components):
    an absolute floor of `floor` x the column's largest magnitude, for
    results that cancel near zero (e.g. Y = eta + ln((1+v)/(1-v))/2 close
    to 0), and a relative 1e-15 gamma^2 per element (gamma = u^0), since
    gamma = 1/sqrt(1 - v^2) multiplies a relative change of v by gamma^2
    (gamma ~ 160 in the corona's vacuum-edge cells after a few steps)."""
    scale = np.maximum(np.abs(a).max(axis=0), np.abs(b).max(axis=0))
    g2 = np.maximum(np.abs(a[:, 8]), np.abs(b[:, 8]))[:, None] ** 2
    tol = (rtol + 1e-15 * g2) * np.maximum(np.abs(a), np.abs(b)) + floor * scale + 1e-300
    return np.abs(a - b) <= tol


def _bad(a, b, ok):
    idx = np.argwhere(~ok)[:5]
    return [(int(i), int(j), float(a[i, j]), float(b[i, j])) for i, j in idx]


def test_gpu_corona_full_size_event_equals_oracle():
    """The 101x101x51 event's corona at tau0 and after 3 steps: every
    record, the sums, and EtotSurf / vEff carried into the next vh_surface."""
    from vhlle_b200.capi import GpuHydro
    setup = W.glauber3d_setup()
    o, d = P.OracleRun(setup), GpuHydro(setup)
    ro, acc = o.corona()
    rd, info = d.corona()
    assert len(ro) == info["nelements"] > 1000
    ok = rec_close(rd, ro)
    assert ok.all(), _bad(rd, ro, ok)
    for k in ("EtotSurf", "vEff"):
        assert abs(info[k] - acc[k]) <= 1e-10 * abs(acc[k]), k
    etot, veff = acc["EtotSurf"], acc["vEff"]
    o.step(3)
    d.step(3)
    ro, acc = o.corona()
    rd, info = d.corona()
    assert len(ro) == info["nelements"]
    ok = rec_close_scaled(rd, ro)
    assert ok.all(), _bad(rd, ro, ok)
    etot += acc["EtotSurf"]
    rs, accs = o.surface(cap=2000000)
    _, infos = d.surface()
    assert infos["nelements"] == len(rs)
    assert abs(infos["EtotSurf"] - (etot + accs["EtotSurf"])) <= 1e-10 * abs(etot) + 1e-8
    d.close()


def _records(d, n):
    import ctypes
    from vhlle_b200 import capi
    rec = np.zeros((n, capi.SURF_REC))
    if n:
        got = ctypes.c_long()
        d._check(d.L.vh_surface_records(d.h, rec.ctypes.data_as(capi._dp), n, ctypes.byref(got)))
    return rec


def test_gpu_surface_pipelined_equals_synchronous():
    """vh_surface_begin / vh_surface_end, with the next step enqueued
    between them, give what vh_surface gives on the same state: counts,
    nsusp, the carried EtotSurf / nbSurf / vEff and every record, bit for
    bit.  Out-of-order calls are refused."""
    from vhlle_b200.capi import GpuHydro, VhError
    setup = W.small_glauber3d(33, 17, seed=11, b=6.0)
    a, b = GpuHydro(setup), GpuHydro(setup)
    with pytest.raises(VhError):
        b.surface_end()
    expect = None
    n_checked = 0
    for k in range(1, 10):
        a.step(1)
        b.step(1)
        if expect is not None:
            info = b.surface_end()
            assert info == expect[1], (k, info, expect[1])
            assert np.array_equal(_records(b, info["nelements"]), expect[0])
            n_checked += info["nelements"]
            expect = None
        if k % 2 == 0:
            expect = a.surface()
            b.surface_begin()
            with pytest.raises(VhError):
                b.surface_begin()
            with pytest.raises(VhError):
                b.surface()
    with pytest.raises(VhError):  # the last call was collected in the loop
        b.surface_end()
    assert n_checked > 500
    a.close()
    b.close()
