"""The oracle's freeze-out surface (Cornelius 4D and the element loop of
Fluid::outputSurface, src/fld.cpp:544-842) pinned against the reference:
its Cornelius class on hypercubes (golden and live), and its freezeout.dat
records and printed counts over an evolving event (golden)."""
import os

import numpy as np
import pytest

import pyoracle as P
from make_golden import load_surface_case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
REC_RTOL = 1e-12  # the reference prints 15 significant digits


def rec_close(a, b, rtol=REC_RTOL):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.abs(a - b) <= rtol * np.maximum(np.abs(a), np.abs(b)) + 1e-300


def test_oracle_cornelius_equals_reference_fixture():
    z = np.load(os.path.join(GOLDEN, "cornelius_cubes.npz"))
    k = 0
    for cube, n in zip(z["cubes"], z["counts"]):
        c, nrm = P.cornelius4d(cube, z["dx"], float(z["e0"]))
        assert c is not None and len(c) == n
        assert np.array_equal(c, z["cent"][k:k + n])
        assert np.array_equal(nrm, z["norm"][k:k + n])
        k += n
    assert k == len(z["cent"])
    assert max(z["counts"]) >= 4  # ambiguous cubes with several elements are covered


@pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")
def test_oracle_cornelius_equals_reference_live():
    rng = np.random.default_rng(99)
    dx = np.array([0.1, 0.2, 0.25, 0.4])
    n_multi = 0
    for t in range(4000):
        if t % 2:
            cube = rng.choice([0.1, 1.0, 3.0], 16) * rng.uniform(0.98, 1.02, 16)
        else:
            cube = rng.lognormal(0, 1, 16)
        co, no = P.cornelius4d(cube, dx, 1.0)
        if co is None:
            continue
        cr, nr = P.cornelius4d(cube, dx, 1.0, reference=True)
        assert np.array_equal(co, cr) and np.array_equal(no, nr), t
        n_multi += len(co) > 1
    assert n_multi > 50


def test_oracle_surface_equals_reference_fixture():
    setup, nsteps, counts, rec, lines = load_surface_case(
        os.path.join(GOLDEN, "surface_glauber_21x21x11_b9.npz"))
    o = P.OracleRun(setup)
    got, etot = [], 0.0
    for s in range(nsteps):
        assert o.step(1) == 0
        r, acc = o.surface()
        assert len(r) == counts[s], s
        got.append(r)
        etot += acc["EtotSurf"]
        # printed: tau E Efull nbSurf S EtotSurf nelements nsusp ratio
        words = lines[s].split()
        assert int(words[6]) == counts[s] and int(words[7]) == int(acc["nsusp"])
        assert abs(etot - float(words[5])) <= 5e-6 * abs(etot) + 1e-9
    got = np.concatenate(got)
    assert got.shape == rec.shape
    ok = rec_close(got, rec)
    assert ok.all(), (np.argwhere(~ok)[:5], got[~ok][:5], rec[~ok][:5])
    assert sum(counts) > 500


CORONA_FIXTURES = ("corona_glauber_41x41x21", "corona_glauber_nb_25x25x13")


@pytest.mark.parametrize("name", CORONA_FIXTURES)
def test_oracle_corona_equals_reference_fixture(name):
    """Fluid::outputCorona at tau0 (src/fld.cpp:876-1089): element count,
    records (15 printed digits) and the printed EtotSurf."""
    from make_golden import load_corona_case
    setup, n, rec, line = load_corona_case(os.path.join(GOLDEN, name + ".npz"))
    ro, acc = P.OracleRun(setup).corona()
    assert len(ro) == n > 0
    ok = rec_close(ro, rec)
    assert ok.all(), np.argwhere(~ok)[:5]
    words = line.split()  # tau E Efull nbSurf S EtotSurf
    assert abs(acc["EtotSurf"] - float(words[5])) <= 5e-6 * abs(acc["EtotSurf"])
    assert acc["nsusp"] == 0


@pytest.mark.skipif(not P.ref_available(), reason="oracle/_ref not built here")
def test_oracle_corona_equals_reference_live():
    """The corona of a fresh event with baryon charge, after some steps (the
    reference calls it at tau0 only, but it is defined at any tau)."""
    import tempfile
    from vhlle_b200 import workloads as W
    setup = W.glauber3d_nb_setup(33, 33, 17, eos=W.nb_table(200, 20), seed=77, b=10.0)
    o, r = P.OracleRun(setup), P.RefRun(setup)
    o.step(3)
    r.step(3)
    ro, _ = o.corona()
    with tempfile.TemporaryDirectory() as d:
        n, _ = r.output_corona(d, extend=True)
        rr = P.read_freezeout(os.path.join(d, "freezeout.dat.unfinished"), extend=True)
    r.close()
    assert len(ro) == n == len(rr) > 0
    assert rec_close(ro, rr).all()
