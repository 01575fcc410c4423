"""Generates the golden fixtures in this directory from the reference itself.

Run from the repository root, where oracle/_ref/libvhlle_ref.so has been
built from the reference sources (``make -C oracle``):

    python tests/golden/make_golden.py

Each fixture is self-contained: the grid, EoS table, transport constants,
clock, initial state and the reference's state after ``nsteps`` calls of
Hydro::performStep.  A second set holds transformPV and EoS known answers.
The generator is the only thing that needs the reference; the fixtures are
committed so that tests on machines without it still pin the oracle and the
CUDA path.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from vhlle_b200 import workloads as W  # noqa: E402
import pyoracle as P  # noqa: E402

CASES = {
    # name: (setup factory, steps)
    "gubser_21x21": (lambda: W.gubser_setup(nx=21, ny=21), 5),
    "glauber_17x17x9": (lambda: W.small_glauber3d(17, 9), 4),
    "glauber_13x13x7_b3": (lambda: W.small_glauber3d(13, 7, b=3.0, seed=5, etaS=0.2), 6),
    # baryon charge on a 200 x 20 (e, nb) table
    "glauber_nb_17x17x9": (lambda: W.glauber3d_nb_setup(17, 17, 9, eos=W.nb_table(200, 20)), 5),
    # the large event's physics (shear + bulk + cross terms + nb) on a coarse
    # grid, with the reference's own zeta/s form 2 in place of the bump
    "large_21x21x11_zeta2": (lambda: large_with_zeta(21, 11, 2), 5),
    # baryon charge on the reference's default EoS, EoSChiral (its two
    # tables from workloads.chiral_eos)
    "glauber_nb_chiral_17x17x9": (lambda: W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos()), 5),
}


def chiral_digest(eos):
    """A fingerprint of a chiral EoS's tables (the fixtures hold it instead
    of the 26 MB of tables, which workloads.chiral_eos regenerates)."""
    import hashlib
    h = hashlib.sha256()
    for a in eos.aux:
        h.update(np.array([a.ne, a.nn, a.emin, a.emax, a.nmin, a.nmax]).tobytes())
        for x in (a.p, a.T, a.mub, a.mus):
            h.update(np.ascontiguousarray(x, dtype=np.float64).tobytes())
    return h.hexdigest()


def large_with_zeta(n, nz, zetaSparam):
    s = W.large_event_setup(0, n, n, nz, eos=W.nb_table(200, 20))
    s.zetaSparam = zetaSparam
    return s


def save_case(name, setup, nsteps):
    r = P.RefRun(setup)
    r.step(nsteps)
    st = r.get_state()
    tot = r.totals()
    with tempfile.TemporaryDirectory() as d:
        nelem, line = r.output_surface(d)
    g = setup.grid
    eos = setup.eos
    arrays = dict(
        grid_n=np.array([g.nx, g.ny, g.nz]), grid_b=np.array(g.bounds()),
        eos_kind=np.array(eos.kind), eos_cnst=np.array(eos.conf_cnst),
        tr=np.array(setup.tr_vector()), tr_params=np.array([setup.etaSparam, setup.zetaSparam]),
        clock=np.array([setup.tau0, setup.dt, setup.ecrit]), nsteps=np.array(nsteps),
        Q0=setup.Q, m0=setup.m, tau_end=np.array(r.tau_now),
        tot_ref=np.array([tot[k] for k in P.TOTALS]),
        surface_line=np.array(line), surface_nelements=np.array(nelem),
    )
    if eos.kind == 1:
        arrays.update(eos_egrid=eos.egrid, eos_ngrid=eos.ngrid, eos_p=eos.p, eos_T=eos.T,
                      eos_mub=eos.mub)
    if eos.kind == 2:
        arrays.update(eos_digest=np.array(chiral_digest(eos)))
    for k, v in st.items():
        arrays["out_" + k] = v
    r.close()
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


SURFACE_CASES = {
    # name: (setup factory, steps; Fluid::outputSurface after every step)
    "surface_glauber_21x21x11_b9": (lambda: W.small_glauber3d(21, 11, b=9.0, seed=5), 8),
}


def save_surface_case(name, setup, nsteps):
    """Per-step freeze-out elements as the reference writes them
    (freezeout.dat, extended records with e and nb) and the printed lines."""
    r = P.RefRun(setup)
    counts, lines = [], []
    with tempfile.TemporaryDirectory() as d:
        for _ in range(nsteps):
            r.step(1)
            n, line = r.output_surface(d, extend=True)
            counts.append(n)
            lines.append(line)
        r.close()
        rec = P.read_freezeout(os.path.join(d, "freezeout.dat.unfinished"), extend=True)
    g = setup.grid
    eos = setup.eos
    arrays = dict(
        grid_n=np.array([g.nx, g.ny, g.nz]), grid_b=np.array(g.bounds()),
        eos_kind=np.array(eos.kind), eos_cnst=np.array(eos.conf_cnst),
        tr=np.array(setup.tr_vector()), tr_params=np.array([setup.etaSparam, setup.zetaSparam]),
        clock=np.array([setup.tau0, setup.dt, setup.ecrit]), nsteps=np.array(nsteps),
        Q0=setup.Q, m0=setup.m, tau_end=np.array(0.0),
        surf_counts=np.array(counts), surf_rec=rec, surf_lines=np.array(lines),
    )
    if eos.kind == 1:
        arrays.update(eos_egrid=eos.egrid, eos_ngrid=eos.ngrid, eos_p=eos.p, eos_T=eos.T,
                      eos_mub=eos.mub)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


VORTICITY_CASES = {
    # name: (setup factory, steps); vorticity on, Fluid::outputSurface after
    # every step (beta.dat lines), the cells' dbeta after the first and the
    # last step
    "vorticity_glauber_21x21x11_b9": (lambda: W.small_glauber3d(21, 11, b=9.0, seed=5), 6),
    "vorticity_glauber_nb_17x17x9": (
        lambda: W.glauber3d_nb_setup(17, 17, 9, eos=W.nb_table(200, 20)), 4),
    # the same physics on the reference's default EoS, EoSChiral
    "vorticity_glauber_nb_chiral_17x17x9": (
        lambda: W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos()), 4),
}


def read_beta(path):
    """beta.dat element lines (src/fld.cpp:665-669,741-745,826-830): position,
    dSigma_mu, u^mu, T, muB, muQ, muS, the 16 Cartesian d_mu beta_nu, e."""
    rows = []
    with open(path) as f:
        for line in f:
            v = line.split()
            if v and not v[0].startswith("#"):
                rows.append([float(x) for x in v])
    return np.array(rows, dtype=np.float64).reshape(-1, 33)


def save_vorticity_case(name, setup, nsteps):
    r = P.RefRun(setup)
    r.enable_vorticity()
    counts, dbeta = [], []
    with tempfile.TemporaryDirectory() as d:
        # the driver's order (src/main.cpp:385-391): outputCorona at tau0,
        # then the beta.dat header with its element count
        ncorona, _ = r.output_corona(d)
        assert r.print_dbeta_header()
        for k in range(nsteps):
            r.step(1)
            if k in (0, nsteps - 1):
                dbeta.append(r.get_dbeta())
            n, _ = r.output_surface(d, extend=True)
            counts.append(n)
        r.close()
        beta = read_beta(os.path.join(d, "beta.dat"))
        with open(os.path.join(d, "beta.dat"), "rb") as f:
            header = b"".join(f.readline() for _ in range(3))
    assert beta.shape[0] == sum(counts)
    arrays = _setup_arrays(setup)
    arrays.update(nsteps=np.array(nsteps), surf_counts=np.array(counts), beta_rec=beta,
                  dbeta_first=dbeta[0], dbeta_last=dbeta[1], corona_count=np.array(ncorona),
                  beta_header=np.frombuffer(header, dtype=np.uint8))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def load_vorticity_case(path):
    """(Setup, steps, per-step element counts, beta.dat records [n][33],
    dbeta [16 N] after the first step, dbeta after the last step)."""
    z = np.load(path)
    setup = _setup_from(z, os.path.basename(path))
    return (setup, int(z["nsteps"]), z["surf_counts"], z["beta_rec"], z["dbeta_first"],
            z["dbeta_last"])


def load_beta_header(path):
    """(outputCorona's element count at tau0, the beta.dat header bytes)."""
    z = np.load(path)
    return int(z["corona_count"]), z["beta_header"].tobytes()


def _setup_from(z, name):
    nx, ny, nz = (int(v) for v in z["grid_n"])
    g = W.Grid(nx, ny, nz, *(float(v) for v in z["grid_b"]))
    if int(z["eos_kind"]) == 2:
        eos = W.chiral_eos()
        if chiral_digest(eos) != str(z["eos_digest"]):
            raise RuntimeError("workloads.chiral_eos no longer gives the fixture's tables")
    else:
        eos = W.EosTable(kind=1, egrid=z["eos_egrid"], ngrid=z["eos_ngrid"], p=z["eos_p"],
                         T=z["eos_T"], mub=z["eos_mub"])
    tr = dict(zip(W.TR_FIELDS, (float(v) for v in z["tr"])))
    tau0, dt, ecrit = (float(v) for v in z["clock"])
    return W.Setup(name, g, eos, tr, int(z["tr_params"][0]), int(z["tr_params"][1]), tau0, dt,
                   ecrit, z["Q0"], z["m0"])


CORONA_CASES = {
    # name: setup factory; Fluid::outputCorona at tau0
    "corona_glauber_41x41x21": lambda: W.small_glauber3d(41, 21),
    "corona_glauber_nb_25x25x13": lambda: W.glauber3d_nb_setup(25, 25, 13, eos=W.nb_table(200, 20)),
}


def _setup_arrays(setup):
    g = setup.grid
    eos = setup.eos
    arrays = dict(
        grid_n=np.array([g.nx, g.ny, g.nz]), grid_b=np.array(g.bounds()),
        eos_kind=np.array(eos.kind), eos_cnst=np.array(eos.conf_cnst),
        tr=np.array(setup.tr_vector()), tr_params=np.array([setup.etaSparam, setup.zetaSparam]),
        clock=np.array([setup.tau0, setup.dt, setup.ecrit]), Q0=setup.Q, m0=setup.m)
    if eos.kind == 1:
        arrays.update(eos_egrid=eos.egrid, eos_ngrid=eos.ngrid, eos_p=eos.p, eos_T=eos.T,
                      eos_mub=eos.mub)
    if eos.kind == 2:
        arrays.update(eos_digest=np.array(chiral_digest(eos)))
    return arrays


def save_corona_case(name, setup):
    """The corona elements the reference writes at tau0 (freezeout.dat,
    extended records with e and nb), its element count and printed line."""
    r = P.RefRun(setup)
    with tempfile.TemporaryDirectory() as d:
        n, line = r.output_corona(d, extend=True)
        r.close()
        rec = P.read_freezeout(os.path.join(d, "freezeout.dat.unfinished"), extend=True)
    assert n == len(rec)
    arrays = _setup_arrays(setup)
    arrays.update(corona_count=np.array(n), corona_rec=rec, corona_line=np.array(line))
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def load_corona_case(path):
    """(Setup, element count, records [n][29], printed line)."""
    z = np.load(path)
    nx, ny, nz = (int(v) for v in z["grid_n"])
    g = W.Grid(nx, ny, nz, *(float(v) for v in z["grid_b"]))
    eos = W.EosTable(kind=1, egrid=z["eos_egrid"], ngrid=z["eos_ngrid"], p=z["eos_p"],
                     T=z["eos_T"], mub=z["eos_mub"])
    tr = dict(zip(W.TR_FIELDS, (float(v) for v in z["tr"])))
    tau0, dt, ecrit = (float(v) for v in z["clock"])
    setup = W.Setup(os.path.basename(path), g, eos, tr, int(z["tr_params"][0]),
                    int(z["tr_params"][1]), tau0, dt, ecrit, z["Q0"], z["m0"])
    return setup, int(z["corona_count"]), z["corona_rec"], str(z["corona_line"])


def cornelius_cubes():
    """Hypercubes (random, near-binary and exact hits of the iso-value) with
    the reference Cornelius' elements."""
    rng = np.random.default_rng(2024)
    dx = np.array([0.05, 0.3, 0.3, 0.25])
    cubes, counts, cent, norm = [], [], [], []
    while len(cubes) < 1200:
        mode = len(cubes) % 4
        if mode == 0:
            c = rng.uniform(0, 1, 16)
        elif mode == 1:
            c = rng.choice([0.2, 0.8], 16) + rng.uniform(-0.01, 0.01, 16)
        elif mode == 2:
            c = rng.choice([0.2, 0.5, 0.8], 16)
        else:
            c = 0.5 + rng.normal(0, 0.3, 16) * (rng.uniform(0, 1, 16) < 0.5)
        co, _ = P.cornelius4d(c, dx, 0.5)  # the oracle first: skips cubes the reference exits on
        if co is None:
            continue
        cr, nr = P.cornelius4d(c, dx, 0.5, reference=True)
        cubes.append(c)
        counts.append(len(cr))
        cent.append(cr)
        norm.append(nr)
    np.savez_compressed(os.path.join(HERE, "cornelius_cubes.npz"), dx=dx, e0=np.array(0.5),
                        cubes=np.array(cubes), counts=np.array(counts),
                        cent=np.concatenate(cent), norm=np.concatenate(norm))


def load_surface_case(path):
    """(Setup, steps, per-step element counts, records [n][29], lines)."""
    z = np.load(path)
    nx, ny, nz = (int(v) for v in z["grid_n"])
    g = W.Grid(nx, ny, nz, *(float(v) for v in z["grid_b"]))
    eos = W.EosTable(kind=1, egrid=z["eos_egrid"], ngrid=z["eos_ngrid"], p=z["eos_p"],
                     T=z["eos_T"], mub=z["eos_mub"])
    tr = dict(zip(W.TR_FIELDS, (float(v) for v in z["tr"])))
    tau0, dt, ecrit = (float(v) for v in z["clock"])
    setup = W.Setup(os.path.basename(path), g, eos, tr, int(z["tr_params"][0]),
                    int(z["tr_params"][1]), tau0, dt, ecrit, z["Q0"], z["m0"])
    return setup, int(z["nsteps"]), z["surf_counts"], z["surf_rec"], [str(v) for v in z["surf_lines"]]


def chiral_points():
    """(e, nb) points over EoSChiral's three regions, their borders, the
    clamped table edges, negative e and nb, and the power law above."""
    rng = np.random.default_rng(12)
    e = np.concatenate([rng.uniform(-0.1, 1.6, 3000), rng.uniform(0, 160, 3000),
                        10 ** rng.uniform(-6, 5, 2000),
                        [0., -0., 1.46, 1.4599999999, 146., 145.99999999, 1e300, 0.146, 0.073,
                         np.inf, 1e-300]])
    nb = np.concatenate([rng.uniform(-0.05, 0.35, 3000), rng.uniform(-0.1, 6.5, 3000),
                         rng.uniform(0, 7, 2000),
                         [0., 0.3, 0.2999999999, 0., 5.999999, 6., 0., 0.15, -1e300, 0., 0.]])
    return e, nb


def chiral_known_answers():
    """EoSChiral (the reference's own class on workloads.chiral_eos's files)
    at chiral_points(): p, T, muB, muS, EoS::p, EoS::s."""
    e, nb = chiral_points()
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos())
    r = P.RefRun(setup)
    out = r.eos6(e, nb)
    r.close()
    np.savez_compressed(os.path.join(HERE, "chiral_known_answers.npz"), e=e, nb=nb, out=out,
                        eos_digest=np.array(chiral_digest(setup.eos)))


def known_answers():
    """transformPV / EoS known answers over regimes the step meets: empty
    (Q_t <= 0), at rest (M = 0), superluminal (M > Q_t), dilute, dense."""
    rng = np.random.default_rng(12345)
    n = 2000
    Qt = 10 ** rng.uniform(-5, 2.5, n)
    frac = np.concatenate([rng.uniform(0, 0.999, n - 400), rng.uniform(1.0, 1.3, 200),
                           np.zeros(100), rng.uniform(0, 0.5, 100)])
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1)[:, None]
    Q = np.zeros((n, 7))
    Q[:, 0] = Qt
    Q[:, 1:4] = dirs * (frac * Qt)[:, None]
    Q[:, 4] = Qt * rng.uniform(0, 0.02, n)
    Q[-50:, 0] = -np.abs(Q[-50:, 0])  # empty cells
    out = {"kpv_Q": Q}
    for kind, setup in (("conf", W.gubser_setup(nx=5, ny=5)), ("table", W.small_glauber3d(5, 5))):
        r = P.RefRun(setup)
        out["kpv_%s" % kind] = r.transform_pv(Q)
        e = 10 ** rng.uniform(-4.5, 3.2, 1000)
        nb = rng.uniform(0, 0.9, 1000)
        pT, s = r.eos_eval(e, nb)
        out["keos_%s_in" % kind] = np.stack([e, nb])
        out["keos_%s_out" % kind] = pT
        out["keos_%s_s" % kind] = s
        if kind == "table":
            ee = setup.eos
            out.update(keos_table_egrid=ee.egrid, keos_table_ngrid=ee.ngrid, keos_table_p=ee.p,
                       keos_table_T=ee.T, keos_table_mub=ee.mub)
        r.close()
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), **out)


def load_case(path):
    """Rebuilds the Setup and the expected end state from a fixture."""
    z = np.load(path)
    nx, ny, nz = (int(v) for v in z["grid_n"])
    g = W.Grid(nx, ny, nz, *(float(v) for v in z["grid_b"]))
    if int(z["eos_kind"]) == 1:
        eos = W.EosTable(kind=1, egrid=z["eos_egrid"], ngrid=z["eos_ngrid"], p=z["eos_p"],
                         T=z["eos_T"], mub=z["eos_mub"])
    elif int(z["eos_kind"]) == 2:
        eos = W.chiral_eos()
        if chiral_digest(eos) != str(z["eos_digest"]):
            raise RuntimeError("workloads.chiral_eos no longer gives the fixture's tables")
    else:
        eos = W.EosTable(kind=0, conf_cnst=float(z["eos_cnst"]))
    tr = dict(zip(W.TR_FIELDS, (float(v) for v in z["tr"])))
    tau0, dt, ecrit = (float(v) for v in z["clock"])
    setup = W.Setup(os.path.basename(path), g, eos, tr, int(z["tr_params"][0]),
                    int(z["tr_params"][1]), tau0, dt, ecrit, z["Q0"], z["m0"])
    expect = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return setup, int(z["nsteps"]), float(z["tau_end"]), expect


def load_totals(path):
    """The reference's interior totals after the fixture's steps, and the
    line Fluid::outputSurface printed (6 significant digits)."""
    z = np.load(path)
    return dict(zip(P.TOTALS, z["tot_ref"])), str(z["surface_line"]), int(z["surface_nelements"])


if __name__ == "__main__":
    if not P.ref_available():
        sys.exit("oracle/_ref/libvhlle_ref.so missing: run `make -C oracle` first")
    # with arguments, only the named fixtures are (re)written
    only = set(sys.argv[1:])
    for name, (fac, n) in CASES.items():
        if not only or name in only:
            save_case(name, fac(), n)
            print("wrote", name)
    for name, (fac, n) in SURFACE_CASES.items():
        if not only or name in only:
            save_surface_case(name, fac(), n)
            print("wrote", name)
    for name, (fac, n) in VORTICITY_CASES.items():
        if not only or name in only:
            save_vorticity_case(name, fac(), n)
            print("wrote", name)
    for name, fac in CORONA_CASES.items():
        if not only or name in only:
            save_corona_case(name, fac())
            print("wrote", name)
    if not only or "cornelius_cubes" in only:
        cornelius_cubes()
        print("wrote cornelius_cubes")
    if not only or "chiral_known_answers" in only:
        chiral_known_answers()
        print("wrote chiral_known_answers")
    if not only or "known_answers" in only:
        known_answers()
        print("wrote known_answers")
