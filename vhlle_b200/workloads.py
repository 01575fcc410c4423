"""Seeded synthetic inputs for the hydro step: grids, EoS tables, initial states.

Everything here runs once on the host, off the timed path.  The same FP64
arrays are handed to the CUDA path and to the CPU checkers, so the initial
state never has to be reproduced bit-for-bit by two implementations.

Workloads (sizes and physics as the benchmark configurations state them):
  * ``gubser``   Gubser flow, ideal, conformal EoS, 101x101x1 on [-5,5]^2,
                 tau0 = 1, dtau = 0.025.  The initial state follows the
                 reference's analytic Gubser IC (src/icGubser.cpp:17-62:
                 q = 1, t = 1, e = (...)^(4/3), transverse flow k(r)).
  * ``glauber3d`` 3D viscous single event, 101x101x51 on [-15,15]^2 x
                 [-7.5,7.5], tau0 = 0.5, dtau = 0.05, eta/s = 0.08,
                 zeta/s = 0, 2000-point log e-table from
                 c_s^2(e) = 1/3 - 0.18 exp(-(ln(e/0.45))^2/1.5); seeded
                 Monte-Carlo Glauber Pb+Pb (WS R = 6.62, a = 0.546, b = 7,
                 sigma_NN = 6.4 fm^2, 0.4 fm smearing, peak e = 50 GeV/fm^3,
                 plateau |eta_s| < 2.5 with Gaussian tails of width 1.0).
  * ``glauber3d_nb`` the same event with baryon charge: nb = 0.3 fm^-3 x
                 the same Glauber profile, a 2000 x 200 (e, nb) table over
                 nb in [0, 1] fm^-3 with mu_B = 1 GeV fm^3 x nb.
  * ``large_event`` 201x201x101 on [-20,20]^2 x [-10,10], tau0 = 0.4,
                 dtau = 0.02, b = 3 fm, peak e = 80 GeV/fm^3, eta/s = 0.08,
                 the zeta/s bump of the batch, baryon charge and the e x nb
                 table; a batch of 8 with seeds 20265000 + k.
  Smaller grids of the same physics come from the same functions with
  smaller nx, ny, nz.

The reference publishes no input files for these workloads (its data
repository is separate), so seeded synthetic inputs stand in for them.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional

import numpy as np

HBARC = 0.1973269804  # GeV fm
# conformal gas with g = 16 + 31.5 (src/eos.cpp:12 uses the same degeneracy)
CONF_DEG = 16.0 + 3.0 * 12.0 * (7.0 / 8.0)
CONF_CNST = 3.0 * CONF_DEG * math.pi ** 2 / 90.0 / HBARC ** 3  # e = cnst T^4

# transport-coefficient parameter order of TransportCoeff's constructor
# (src/trancoeff.h:14-20)
TR_FIELDS = ("etaS0", "zetaS0", "ah", "al", "aRho", "T0", "etaSMin",
             "etaSEpsilonMin", "etaSShiftMuB", "etaSScaleMuB",
             "zetaSPeakEpsilon", "zetaSScaleBeta", "zetaSSigmaMinus",
             "zetaSSigmaPlus")
# defaults of the reference driver (src/main.cpp:70-78)
TR_DEFAULTS = dict(etaS0=0.08, zetaS0=0.0, ah=0.0, al=0.0, aRho=0.0, T0=0.15,
                   etaSMin=0.08, etaSEpsilonMin=5.0, etaSShiftMuB=0.0,
                   etaSScaleMuB=0.0, zetaSPeakEpsilon=5.0,
                   zetaSScaleBeta=0.103, zetaSSigmaMinus=0.1,
                   zetaSSigmaPlus=0.1)


@dataclasses.dataclass
class Grid:
    nx: int
    ny: int
    nz: int
    xmin: float
    xmax: float
    ymin: float
    ymax: float
    etamin: float
    etamax: float
    # the eta cell size of a larger grid this one is a slab of (None: from
    # the bounds, as Fluid does)
    cell_dz: Optional[float] = None

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dx(self) -> float:  # src/fld.cpp:77-79
        return (self.xmax - self.xmin) / (self.nx - 1)

    @property
    def dy(self) -> float:
        return (self.ymax - self.ymin) / (self.ny - 1)

    @property
    def dz(self) -> float:
        if self.cell_dz:
            return self.cell_dz
        # nz = 1 gives an infinite cell, as the reference's FP64 division does
        span = self.etamax - self.etamin
        if self.nz == 1:
            return math.copysign(math.inf, span) if span != 0 else math.nan
        return span / (self.nz - 1)

    def bounds(self):
        return (self.xmin, self.xmax, self.ymin, self.ymax, self.etamin,
                self.etamax)

    def coords(self):
        """Cell-centre coordinates x[ix], y[iy], eta[iz] (Fluid::getX etc.)."""
        ix = np.arange(self.nx)
        iy = np.arange(self.ny)
        iz = np.arange(self.nz)
        with np.errstate(invalid="ignore"):
            return (self.xmin + ix * self.dx, self.ymin + iy * self.dy,
                    self.etamin + iz * self.dz)


@dataclasses.dataclass
class EosTable:
    """EoS descriptor.  kind 0: conformal gas; kind 1: EoS1f (e, nb) table
    with p/T/mub stored [ie + ne*inb] (src/eo1.cpp:21-45); kind 2: EoSChiral
    (src/eoChiral.cpp), `aux` = (chiralsmall, chiraleos) ChiralAux tables;
    kind 3: EoS3f (e, nb, nq, ns) table, one n grid for the three charges
    (src/eo3.cpp:21-91)."""
    kind: int
    conf_cnst: float = CONF_CNST
    egrid: Optional[np.ndarray] = None
    ngrid: Optional[np.ndarray] = None
    p: Optional[np.ndarray] = None
    T: Optional[np.ndarray] = None
    mub: Optional[np.ndarray] = None
    aux: Optional[tuple] = None
    # kind 3 (EoS3f): muQ and muS tables beside p, T, muB, all
    # [ie + ne*inb + ne*nn*inq + ne*nn*nn*ins], and the file's header
    # constants B, volex0, delta0, aaa, bbb
    muq: Optional[np.ndarray] = None
    mus: Optional[np.ndarray] = None
    header3: tuple = (0.0, 0.0, 0.0, 0.0, 0.0)
    # kind 4 (EoSHadron): (ne, nnb, nnq, e0, n0, logemin, logemax, lognmax),
    # the file's e, nb, nq value of every row, and the status table; p, T,
    # mub, muq, mus at [inq + nnq*inb + nnq*nnb*ie]
    hadron: Optional[tuple] = None
    hrows: Optional[np.ndarray] = None
    status: Optional[np.ndarray] = None
    # kind 5 (EoSSmash): (ne, nnb, nnq) and the uniform grids' values; p, T,
    # mub, muq, mus at [inq + nnq*inb + nnq*nnb*ie]
    smash: Optional[tuple] = None
    # kind 6 (EoSAZH): six tables p1, p2, T1, T2, mu1, mu2, each
    # (ne, nn, emin, nmin, de, dn, values[ie * nn + in])
    azh: Optional[tuple] = None

    def write_azh(self, directory: str) -> None:
        """directory/eos/azhydro0p2/aa{1,2}_{p,t,mb}.dat, the files EoSAZH
        reads from its working directory (src/eoAZH.cpp:110-117), in the
        EoSAZHaux format: ``nmin emin``, ``dn de nn-1 ne-1``, then the values
        with e outer and nb inner (src/eoAZH.cpp:31-50); 17 significant
        digits."""
        assert self.kind == 6
        d = os.path.join(directory, "eos", "azhydro0p2")
        os.makedirs(d, exist_ok=True)
        names = ("aa1_p", "aa2_p", "aa1_t", "aa2_t", "aa1_mb", "aa2_mb")
        for name, (ne, nn, emin, nmin, de, dn, v) in zip(names, self.azh):
            with open(os.path.join(d, name + ".dat"), "w") as f:
                f.write("%r %r\n%r %r %d %d\n" % (nmin, emin, dn, de, nn - 1, ne - 1))
                v = np.asarray(v, dtype=np.float64).reshape(ne, nn)
                for row in v:
                    f.write(" ".join("%r" % float(x) for x in row) + "\n")

    def write_cmfe(self, directory: str) -> None:
        """directory/eos/cmfe_small.dat and cmfe.dat, the files EoSCMFe reads
        from its working directory (src/eoCMFe.cpp:194-197): a header line,
        then 7 columns (e, n, T, p, s, mu_B, mu_S in the files' units) with e
        outer and n inner (src/eoCMFe.cpp:83-94), every value exact in 10
        decimals (a NaN written as nan)."""
        assert self.kind == 7
        os.makedirs(os.path.join(directory, "eos"), exist_ok=True)
        for name, cols, _ in _cmfe_tables():
            np.savetxt(os.path.join(directory, "eos", name), cols, fmt="%.10f",
                       header="e n T p s muB muS", comments="# ")

    def write_chiral(self, directory: str) -> None:
        """directory/eos/chiralsmall.dat and chiraleos.dat, the files
        EoSChiral reads from its working directory (src/eoChiral.cpp:153-156):
        8 columns (T, mu_q, e, p, n, s, mu_S, unused) with n outer and e
        inner, every value exact in 10 decimals."""
        assert self.kind == 2
        os.makedirs(os.path.join(directory, "eos"), exist_ok=True)
        for name, cols, _ in _chiral_tables():
            np.savetxt(os.path.join(directory, "eos", name), cols, fmt="%.10f")

    @property
    def ne(self) -> int:
        return 0 if self.egrid is None else len(self.egrid)

    @property
    def nn(self) -> int:
        return 0 if self.ngrid is None else len(self.ngrid)

    def write_eos1f(self, path: str) -> None:
        """Write the table in the reference's EoS1f text format: header
        ``emax e0 nmax n0 ne nn``, the e grid, the n grid, then ``p T mub``
        rows with ie outer and inb inner (src/eo1.cpp:24-43).  Values are
        written with 17 significant digits so that they read back exactly."""
        assert self.kind == 1
        ne, nn = self.ne, self.nn
        with open(path, "w") as f:
            f.write("%r %r %r %r %d %d\n" % (float(self.egrid[-1]), float(self.egrid[0]),
                                            float(self.ngrid[-1]), float(self.ngrid[0]), ne, nn))
            f.write(" ".join(repr(float(v)) for v in self.egrid) + "\n")
            f.write(" ".join(repr(float(v)) for v in self.ngrid) + "\n")
            for ie in range(ne):
                for inb in range(nn):
                    k = ie + ne * inb
                    f.write("%r %r %r\n" % (float(self.p[k]), float(self.T[k]), float(self.mub[k])))

    def write_eos3f(self, path: str) -> None:
        """Write the table in the reference's EoS3f text format: the header
        constants ``B volex0 delta0 aaa bbb``, ``emax e0 nmax n0 ne nn``, the
        e grid, the n grid, then ``p T mub muq mus`` rows with ie, inb, inq,
        ins nested outer to inner (src/eo3.cpp:24-85); 17 significant digits."""
        assert self.kind == 3
        ne, nn = self.ne, self.nn
        with open(path, "w") as f:
            f.write(" ".join(repr(float(v)) for v in self.header3) + "\n")
            f.write("%r %r %r %r %d %d\n" % (float(self.egrid[-1]), float(self.egrid[0]),
                                            float(self.ngrid[-1]), float(self.ngrid[0]), ne, nn))
            f.write(" ".join(repr(float(v)) for v in self.egrid) + "\n")
            f.write(" ".join(repr(float(v)) for v in self.ngrid) + "\n")
            idx = np.arange(ne * nn ** 3).reshape(nn, nn, nn, ne)  # [is][iq][ib][ie]
            order = idx.transpose(3, 2, 1, 0).reshape(-1)           # ie, ib, iq, is nesting
            cols = np.stack([self.p[order], self.T[order], self.mub[order], self.muq[order],
                             self.mus[order]], 1)
            f.write("\n".join(" ".join(repr(float(v)) for v in row) for row in cols) + "\n")

    def write_hadron(self, path: str) -> None:
        """Write the table in the reference's EoSHadron text format: the
        header ``ne nnb nnq e0 n0 logemin logemax lognmax``, then ``e nb nq p T
        mub muq mus status`` rows with ie, inb, inq nested outer to inner
        (src/eoHadron.cpp:13-40); 17 significant digits."""
        assert self.kind == 4
        ne, nnb, nnq, e0, n0, lo, hi, ln = self.hadron
        with open(path, "w") as f:
            f.write("%d %d %d %r %r %r %r %r\n" % (ne, nnb, nnq, e0, n0, lo, hi, ln))
            for k in range(ne * nnb * nnq):
                f.write("%r %r %r %r %r %r %r %r %d\n" % (
                    float(self.hrows[k, 0]), float(self.hrows[k, 1]), float(self.hrows[k, 2]),
                    float(self.p[k]), float(self.T[k]), float(self.mub[k]), float(self.muq[k]),
                    float(self.mus[k]), int(self.status[k])))

    def write_smash(self, path: str) -> None:
        """Write the table in the reference's EoSSmash text format: one header
        line, then ``e nb nq T p mub mus muq`` rows with ie, inb, inq nested
        outer to inner (src/eoSmash.cpp:30-43); 17 significant digits."""
        assert self.kind == 5
        (ne, nnb, nnq), (eg, bg, qg) = self.smash
        with open(path, "w") as f:
            f.write("# e nb nq T p muB muS muQ\n")
            for ie in range(ne):
                for inb in range(nnb):
                    for inq in range(nnq):
                        k = inq + nnq * inb + nnq * nnb * ie
                        f.write("%r %r %r %r %r %r %r %r\n" % (
                            float(eg[ie]), float(bg[inb]), float(qg[inq]), float(self.T[k]),
                            float(self.p[k]), float(self.mub[k]), float(self.mus[k]),
                            float(self.muq[k])))

    @staticmethod
    def read_eos1f(path: str) -> "EosTable":
        """Parse an EoS1f file the way the reference constructor does; values
        below 1e-18 in the pressure column read as 0 (src/eo1.cpp:42)."""
        with open(path) as f:
            tok = f.read().split()
        emax, e0, nmax, n0 = (float(t) for t in tok[:4])
        ne, nn = int(tok[4]), int(tok[5])
        pos = 6
        egrid = np.array([float(t) for t in tok[pos:pos + ne]]); pos += ne
        ngrid = np.array([float(t) for t in tok[pos:pos + nn]]); pos += nn
        p = np.zeros(ne * nn); T = np.zeros(ne * nn); mub = np.zeros(ne * nn)
        for ie in range(ne):
            for inb in range(nn):
                k = ie + ne * inb
                p[k] = float(tok[pos]); T[k] = float(tok[pos + 1]); mub[k] = float(tok[pos + 2])
                if p[k] < 1e-18:
                    p[k] = 0.0
                pos += 3
        return EosTable(kind=1, egrid=egrid, ngrid=ngrid, p=p, T=T, mub=mub)


@dataclasses.dataclass
class ChiralAux:
    """One EoSaux table as its constructor leaves it (src/eoChiral.cpp:48-80):
    uniform grids [emin, emax] x [nmin, nmax] (GeV/fm^3, fm^-3), p/T/mub/mus
    (GeV/fm^3, GeV) at [in * ne + ie]."""
    ne: int
    nn: int
    emin: float
    emax: float
    nmin: float
    nmax: float
    p: np.ndarray
    T: np.ndarray
    mub: np.ndarray
    mus: np.ndarray


# EoSChiral's table sizes and this generator's ranges in the files' units
# (e in e0 = 0.146 GeV/fm^3, n in n0 = 0.15 fm^-3): the small table covers
# e < 1.46 GeV/fm^3, nb < 0.3 fm^-3 and the big one e < 146, nb < 6, the
# regions EoSChiral::eos sends to them (src/eoChiral.cpp:153-170)
CHIRAL_TABLES = (("chiralsmall.dat", 201, 201, 10.0, 2.0), ("chiraleos.dat", 2001, 401, 1000.0, 40.0))


def _q(x):
    """Rounded to a multiple of 2^-10: exact in binary and in short decimal."""
    return np.round(np.asarray(x, dtype=np.float64) * 1024.0) / 1024.0


def _chiral_tables():
    """(file name, the file's 8 columns, ChiralAux) per EoSChiral table."""
    out = []
    for name, ne, nn, emax_f, nmax_f in CHIRAL_TABLES:
        e_f = _q(np.arange(ne) * (emax_f / (ne - 1)))
        n_f = _q(np.arange(nn) * (nmax_f / (nn - 1)))
        E, Nb = np.meshgrid(e_f, n_f)  # [in][ie]
        T_f = _q(20.0 + 140.0 * (E + 0.05) ** 0.25 * (1.0 - 0.1 * Nb / nmax_f))
        muq_f = _q(60.0 * Nb / (1.0 + 0.02 * E) + 0.5 * Nb ** 2)
        p_f = _q(E / 3.0 * (1.0 - 0.3 * np.exp(-E)) - 0.02 + 0.01 * Nb)
        s_f = _q((E + p_f) * 146.0 / T_f)
        mus_f = _q(15.0 * Nb / (1.0 + E))
        cols = np.stack([T_f, muq_f, E, p_f, Nb, s_f, mus_f, np.zeros_like(E)],
                        axis=-1).reshape(-1, 8)
        aux = ChiralAux(ne=ne, nn=nn, emin=e_f[0] * 0.146, emax=e_f[-1] * 0.146,
                        nmin=n_f[0] * 0.15, nmax=n_f[-1] * 0.15,
                        p=(p_f * 0.146).ravel(), T=(T_f / 1000.0).ravel(),
                        mub=(muq_f * (3.0 / 1000.0)).ravel(), mus=(mus_f / 1000.0).ravel())
        out.append((name, cols, aux))
    return out


def chiral_eos() -> EosTable:
    """A synthetic EoSChiral (the chiral model's tables are not in the
    reference tree): smooth T, mu_q, p, s, mu_S over each table's (e, n)
    grid in the file units (MeV, e0, n0), every value a multiple of 2^-10,
    converted as the reference's EoSaux constructor converts them (T / 1000,
    mu_q * (3 / 1000), mu_S / 1000, p * 0.146, grid ends * 0.146 and * 0.15),
    so that the files (write_chiral) and these arrays hold the same doubles."""
    return EosTable(kind=2, aux=tuple(t[2] for t in _chiral_tables()))


# EoSCMFe's table sizes (src/eoCMFe.cpp:194-197) and this generator's
# ranges in the files' units (e in EPS_0 / 1000 GeV/fm^3, n in N_0): the
# small table covers the region EoSCMFe::eos sends to it (e < 15, n < 5),
# the big one e < 800, n < 40
CMFE_TABLES = (("cmfe_small.dat", 1501, 501, 15.0, 5.0), ("cmfe.dat", 4001, 401, 800.0, 40.0))
CMFE_EPS0 = 146.51751415742 * 0.87326281
CMFE_N0 = 0.15891 * 0.87272727


def _cmfe_tables():
    """(file name, the file's 7 columns, ChiralAux) per EoSCMFe table; the
    big table has no model solution (NaN) where n > 36 N_0 and e < 40."""
    out = []
    for name, ne, nn, emax_f, nmax_f in CMFE_TABLES:
        e_f = _q(np.arange(ne) * (emax_f / (ne - 1)))
        n_f = _q(np.arange(nn) * (nmax_f / (nn - 1)))
        E, Nb = np.meshgrid(e_f, n_f, indexing="ij")  # [ie][in]
        T_f = _q(20.0 + 140.0 * (E / 10.0 + 0.05) ** 0.25 * (1.0 - 0.1 * Nb / nmax_f))
        p_f = _q(E / 3.0 * (1.0 - 0.3 * np.exp(-E / 10.0)) - 0.02 + 0.01 * Nb)
        s_f = _q((E + p_f) * 7.0 / T_f)
        mub_f = _q(300.0 * Nb / (1.0 + 0.02 * E))
        mus_f = _q(15.0 * Nb / (1.0 + E / 10.0))
        if nmax_f > 5.0:
            hole = (Nb > 36.0) & (E < 40.0)
            for a in (T_f, p_f, s_f, mub_f, mus_f):
                a[hole] = np.nan
        cols = np.stack([E, Nb, T_f, p_f, s_f, mub_f, mus_f], axis=-1).reshape(-1, 7)
        # EoSCMFeaux's conversions (src/eoCMFe.cpp:85-92), in the aux layout
        aux = ChiralAux(ne=ne, nn=nn, emin=e_f[0] * CMFE_EPS0 / 1000.0,
                        emax=e_f[-1] * CMFE_EPS0 / 1000.0, nmin=n_f[0] * CMFE_N0,
                        nmax=n_f[-1] * CMFE_N0,
                        p=np.ascontiguousarray((p_f * CMFE_EPS0 / 1000.0).T).ravel(),
                        T=np.ascontiguousarray((T_f / 1000.0).T).ravel(),
                        mub=np.ascontiguousarray((mub_f / 1000.0).T).ravel(),
                        mus=np.ascontiguousarray((mus_f / 1000.0).T).ravel())
        out.append((name, cols, aux))
    return out


def cmfe_eos_table() -> EosTable:
    """A synthetic EoSCMFe (the CMF model's tables are not in the reference
    tree): smooth T, p, s, mu_B, mu_S over each table's (e, n) grid in the
    file units (MeV, EPS_0 / 1000, N_0), every value a multiple of 2^-10,
    converted as the reference's EoSCMFeaux constructor converts them, so
    that the files (write_cmfe) and these arrays hold the same doubles."""
    return EosTable(kind=7, aux=tuple(t[2] for t in _cmfe_tables()))


def hadron_eos_table(ne: int = 101, nnb: int = 41, nnq: int = 21, e0: float = 1.0,
                     n0: float = 0.15, logemin: float = -6.9, logemax: float = 2.3,
                     lognmax: float = 2.5) -> EosTable:
    """A synthetic hadronic EoS in the reference's EoSHadron format (the
    freeze-out EoS the reference's driver loads by default): e on a log
    grid e0 exp(x), x uniform on [logemin, logemax]; nb and nq on the
    symmetric log mapping of src/eoHadron.cpp:91-112 (|n| = n0 exp(2|x| -
    lognmax) beyond the two innermost cells, linear inside), x uniform on
    [-lognmax, lognmax]; a resonance-gas-like p = 0.15 e + 0.4 nb^2, T =
    0.16 (e / 0.5)^0.2 - 0.01 nb^2, mu_B = 0.8 tanh(nb / 0.3), mu_Q = 0.1 nq,
    mu_S = 0.2 mu_B; the status is 1 (invalid) where |nb| > 1.5 fm^-3 and e
    < 0.02 GeV/fm^3."""
    dxe = (logemax - logemin) / (ne - 1)
    xe = logemin + dxe * np.arange(ne)
    e = e0 * np.exp(xe)

    def charge(nn):
        dx = (2.0 * lognmax) / (nn - 1)
        x = -lognmax + dx * np.arange(nn)
        amin = n0 * math.exp(2.0 * dx - lognmax)
        n = np.where(np.abs(x) >= dx, np.sign(x) * n0 * np.exp(2 * np.abs(x) - lognmax),
                     x / dx * amin)
        return n

    nb = charge(nnb)
    nq = charge(nnq)
    E = e[:, None, None]
    B = nb[None, :, None]
    Qc = nq[None, None, :]
    shape = (ne, nnb, nnq)
    p = np.broadcast_to(0.15 * E + 0.4 * B * B + 0 * Qc, shape)
    T = np.broadcast_to(0.16 * (E / 0.5) ** 0.2 - 0.01 * B * B + 0 * Qc, shape)
    mub = np.broadcast_to(0.8 * np.tanh(B / 0.3) + 0 * E + 0 * Qc, shape)
    muq = np.broadcast_to(0.1 * Qc + 0 * E + 0 * B, shape)
    mus = 0.2 * mub
    status = np.broadcast_to(((np.abs(B) > 1.5) & (E < 0.02)) + 0 * Qc, shape).astype(np.int32)
    rows = np.stack(np.broadcast_arrays(E, B, Qc), -1).reshape(-1, 3)
    flat = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)  # noqa: E731
    return EosTable(kind=4, p=flat(p), T=flat(T), mub=flat(mub), muq=flat(muq), mus=flat(mus),
                    hadron=(ne, nnb, nnq, e0, n0, logemin, logemax, lognmax), hrows=rows,
                    status=np.ascontiguousarray(status.reshape(-1)))


def smash_eos_table(ne: int = 101, nnb: int = 51, nnq: int = 51) -> EosTable:
    """A synthetic hadron-gas EoS in the reference's EoSSmash format (the
    driver's eosTypeHadron 1, read with ne x nnb x nnq = 101 x 51 x 51,
    src/main.cpp:308): uniform grids e in [0.01, 1.01] GeV/fm^3, nb and nq in
    [-0.5, 0.5] fm^-3; p = 0.14 e + 0.3 nb^2 + 0.05 nq^2, T = 0.12 + 0.05 e
    - 0.02 nb^2, mu_B = 0.9 nb, mu_Q = 0.2 nq, mu_S = 0.25 nb."""
    eg = 0.01 + 0.01 * np.arange(ne)
    bg = -0.5 + (1.0 / (nnb - 1)) * np.arange(nnb)
    qg = -0.5 + (1.0 / (nnq - 1)) * np.arange(nnq)
    E, B, Qc = np.meshgrid(eg, bg, qg, indexing="ij")
    flat = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)  # noqa: E731
    return EosTable(kind=5, p=flat(0.14 * E + 0.3 * B * B + 0.05 * Qc * Qc),
                    T=flat(0.12 + 0.05 * E - 0.02 * B * B), mub=flat(0.9 * B),
                    muq=flat(0.2 * Qc), mus=flat(0.25 * B), smash=((ne, nnb, nnq), (eg, bg, qg)))


def azh_eos_table(ne1: int = 401, ne2: int = 301, nn: int = 51) -> EosTable:
    """A synthetic EoS in the reference's EoSAZH format (eosType 2, six
    EoSAZHaux tables): the first set on e = 0.01 + 0.005 ie GeV/fm^3 (up to
    2.01), the second on e = 2 + 0.5 ie (up to 152), both on nb = 0.01 in
    fm^-3 (0 .. 0.5); p = e/3 - 0.15 e / (1 + e) + 0.05 nb^2 / (1 + e),
    T = 0.16 e^(1/4) (1 - 0.2 nb), mu_B = 0.8 nb / sqrt(0.3 + e).  Below the
    first set (e < 0.01) EoSAZH scales its first row by e / emin."""
    def fill(f, ne, emin, de):
        E, B = np.meshgrid(emin + de * np.arange(ne), 0.01 * np.arange(nn), indexing="ij")
        return np.ascontiguousarray(f(E, B), dtype=np.float64).reshape(-1)
    fp = lambda E, B: E / 3.0 - 0.15 * E / (1.0 + E) + 0.05 * B * B / (1.0 + E)  # noqa: E731
    fT = lambda E, B: 0.16 * E ** 0.25 * (1.0 - 0.2 * B)  # noqa: E731
    fm = lambda E, B: 0.8 * B / np.sqrt(0.3 + E)  # noqa: E731
    sets = ((ne1, 0.01, 0.005), (ne2, 2.0, 0.5))
    tabs = []
    for f in (fp, fT, fm):
        for ne, emin, de in sets:
            tabs.append((ne, nn, emin, 0.0, de, 0.01, fill(f, ne, emin, de)))
    return EosTable(kind=6, azh=tuple(tabs))


def eos3f_table(ne: int = 120, emin: float = 1e-4, emax: float = 1e3) -> EosTable:
    """A synthetic EoS3f table: ``ne`` log e-points (1e-4 .. 1e3 GeV/fm^3)
    and one n grid of 9 points on [-0.4, 0.4] fm^-3 (0 a node) for nb, nq
    and ns; p = c_s^2(e) e + 0.5 nb^2 + 0.25 nq^2 + 0.15 ns^2 with the
    c_s^2(e) of the other tables, T from the conformal-gas form, mu_B =
    1 GeV fm^3 nb, mu_Q = 0.5 GeV fm^3 nq + 0.05 GeV fm^3 nb, mu_S = 0.3 GeV fm^3 ns + 0.1 GeV
    fm^3 nb.  The header's B is 0, so the reference reads it without checking
    its constructor's arguments against it (src/eo3.cpp:26-51)."""
    egrid = np.exp(np.linspace(np.log(emin), np.log(emax), ne))
    ngrid = np.array([-0.4, -0.3, -0.2, -0.1, 0.0, 0.1, 0.2, 0.3, 0.4])
    nn = len(ngrid)
    E = egrid[None, None, None, :]
    nb = ngrid[None, None, :, None]
    nq = ngrid[None, :, None, None]
    ns = ngrid[:, None, None, None]
    p = cs2_model(E) * E + 0.5 * nb * nb + 0.25 * nq * nq + 0.15 * ns * ns
    T = 0.15120476935 * np.sqrt(np.sqrt(E)) + 0.0 * nb
    shape = (nn, nn, nn, ne)
    return EosTable(kind=3, egrid=egrid, ngrid=ngrid,
                    p=np.broadcast_to(p, shape).reshape(-1).copy(),
                    T=np.broadcast_to(T, shape).reshape(-1).copy(),
                    mub=np.broadcast_to(1.0 * nb + 0 * E, shape).reshape(-1).copy(),
                    muq=np.broadcast_to(0.5 * nq + 0.05 * nb + 0 * E, shape).reshape(-1).copy(),
                    mus=np.broadcast_to(0.3 * ns + 0.1 * nb + 0 * E, shape).reshape(-1).copy())


def cs2_model(e):
    """c_s^2(e) = 1/3 - 0.18 exp(-(ln(e/0.45))^2/1.5) of the 3D workloads."""
    e = np.asarray(e, dtype=np.float64)
    return 1.0 / 3.0 - 0.18 * np.exp(-np.log(e / 0.45) ** 2 / 1.5)


def make_cs2_table(ne: int = 2000, emin: float = 1e-4, emax: float = 1e3,
                   nn: int = 2, nbmax: float = 1.0, mub_slope: float = 0.0,
                   sub: int = 64) -> EosTable:
    """Log-spaced e-table with p and T integrated consistently from c_s^2(e).

    p(e) = p(emin) + int c_s^2 de with p(emin) = emin/3 (conformal at the low
    end, where c_s^2 -> 1/3), and d ln T = dp/(e+p) at mu_B = 0, anchored to
    the Stefan-Boltzmann gas of CONF_DEG degrees of freedom at emax.  The nb
    axis has ``nn`` points on [0, nbmax]; for nn = 2 and mub_slope = 0 the
    table is nb independent (the reference's EoS1f needs nn >= 2).  A nonzero
    ``mub_slope`` adds mu_B = mub_slope * nb (GeV per fm^-3) and the matching
    first-order pressure shift dp = nb * mu_B / 2 (thermodynamically
    consistent to that order)."""
    egrid = np.exp(np.linspace(math.log(emin), math.log(emax), ne))
    # fine composite Simpson integration between grid points
    p = np.empty(ne)
    lnT_rel = np.empty(ne)
    p[0] = emin / 3.0
    lnT_rel[0] = 0.0
    for i in range(1, ne):
        a, b = egrid[i - 1], egrid[i]
        xs = np.linspace(a, b, 2 * sub + 1)
        w = np.ones_like(xs); w[1:-1:2] = 4.0; w[2:-1:2] = 2.0
        h = (b - a) / (2 * sub)
        cs = cs2_model(xs)
        pseg = p[i - 1] + np.concatenate(([0.0], np.cumsum((cs[1:] + cs[:-1]) * 0.5 * np.diff(xs))))
        p[i] = p[i - 1] + h / 3.0 * np.sum(w * cs)
        lnT_rel[i] = lnT_rel[i - 1] + h / 3.0 * np.sum(w * cs / (xs + pseg))
    T_top = (emax / CONF_CNST) ** 0.25
    T = T_top * np.exp(lnT_rel - lnT_rel[-1])
    ngrid = np.linspace(0.0, nbmax, nn)
    P = np.empty(ne * nn); TT = np.empty(ne * nn); MU = np.empty(ne * nn)
    for inb in range(nn):
        nb = ngrid[inb]
        mu = mub_slope * nb
        P[inb * ne:(inb + 1) * ne] = p + 0.5 * nb * mu
        TT[inb * ne:(inb + 1) * ne] = T
        MU[inb * ne:(inb + 1) * ne] = mu
    return EosTable(kind=1, egrid=egrid, ngrid=ngrid, p=P, T=TT, mub=MU)


@dataclasses.dataclass
class Setup:
    """One hydro problem: grid, EoS, transport, clock and initial state."""
    name: str
    grid: Grid
    eos: EosTable
    tr: dict
    etaSparam: int
    zetaSparam: int
    tau0: float
    dt: float
    ecrit: float
    Q: np.ndarray          # [7][N] tau-weighted conserved variables
    m: np.ndarray          # [N] initial fill fraction (setAllM value)
    pi: Optional[np.ndarray] = None   # [10][N]
    Pi: Optional[np.ndarray] = None   # [N]

    @property
    def viscous(self) -> bool:  # TransportCoeff::isViscous, src/trancoeff.h:39-45
        t = self.tr
        return (t["etaS0"] > 0 or t["zetaS0"] > 0 or self.etaSparam > 0
                or self.zetaSparam > 0)

    def tr_vector(self):
        return [float(self.tr[k]) for k in TR_FIELDS]


def conserved_from_primitive(tau, e, p, nb, vx, vy, vz):
    """Cell::setPrimVar arithmetic (src/cll.cpp:222-241) on arrays."""
    gamma2 = 1.0 / (1 - vx * vx - vy * vy - vz * vz)
    v2 = vx * vx + vy * vy + vz * vz
    Q = np.zeros((7,) + np.shape(e))
    Q[0] = tau * (e + p * v2) * gamma2
    Q[1] = tau * (e + p) * vx * gamma2
    Q[2] = tau * (e + p) * vy * gamma2
    Q[3] = tau * (e + p) * vz * gamma2
    Q[4] = tau * nb * np.sqrt(gamma2)
    return Q


def gubser_setup(nx: int = 101, ny: int = 101, xmax: float = 5.0,
                 tau0: float = 1.0, dt: float = 0.025) -> Setup:
    """Gubser flow initial state on an nz = 1 grid (eta in [-0.5, 0.5], so
    that dz is finite), following src/icGubser.cpp:24-57."""
    g = Grid(nx, ny, 1, -xmax, xmax, -xmax, xmax, -0.5, 0.5)
    x, y, _ = g.coords()
    X, Y = np.meshgrid(x, y, indexing="xy")  # [iy][ix]
    t, q = 1.0, 1.0
    r = np.sqrt(X * X + Y * Y)
    k = 2. * q * q * t * r / (1. + q * q * t * t + q * q * r * r)
    e = 4. * q * q / (1. + 2. * q * q * (t * t + r * r) + (q * q * (t * t - r * r)) ** 2) / t
    e = np.where(e < 0., 0., e)
    e = e ** (4. / 3.)
    vx = X / (r + 1e-50) * k
    vy = Y / (r + 1e-50) * k
    vz = np.zeros_like(e)
    nb = np.zeros_like(e)
    p = e / 3.
    Q = conserved_from_primitive(tau0, e, p, nb, vx, vy, vz).reshape(7, -1)
    m = (e.reshape(-1) > 0).astype(np.float64)
    tr = dict(TR_DEFAULTS, etaS0=0.0, etaSMin=0.0)
    return Setup("gubser", g, EosTable(kind=0), tr, 0, 0, tau0, dt, 0.5, Q, m)


def _woods_saxon(rng, A, R, a):
    out = np.empty((A, 3))
    n = 0
    rmax = R + 10 * a
    while n < A:
        r = rng.uniform(0, rmax, size=4 * A)
        acc = rng.uniform(0, 1, size=4 * A) < (r * r / (rmax * rmax)) / (1 + np.exp((r - R) / a))
        r = r[acc]
        cth = rng.uniform(-1, 1, size=r.size)
        ph = rng.uniform(0, 2 * math.pi, size=r.size)
        sth = np.sqrt(1 - cth * cth)
        pts = np.stack([r * sth * np.cos(ph), r * sth * np.sin(ph), r * cth], 1)
        take = min(A - n, len(pts))
        out[n:n + take] = pts[:take]
        n += take
    return out


def glauber_participants(seed: int, b: float, A: int = 208, R: float = 6.62,
                         a: float = 0.546, sigma_nn: float = 6.4) -> np.ndarray:
    """Transverse positions [n][2] (fm) of the participants of one seeded
    MC-Glauber event: two Woods-Saxon nuclei at x = +-b/2, a nucleon
    participates when it comes within sqrt(sigma_NN / pi) of one of the
    other nucleus (nucleus A's participants first, in sampling order)."""
    rng = np.random.default_rng(seed)
    na = _woods_saxon(rng, A, R, a)
    nbn = _woods_saxon(rng, A, R, a)
    na[:, 0] += b / 2
    nbn[:, 0] -= b / 2
    d2 = ((na[:, None, 0] - nbn[None, :, 0]) ** 2 + (na[:, None, 1] - nbn[None, :, 1]) ** 2)
    hit = d2 < sigma_nn / math.pi
    return np.ascontiguousarray(np.concatenate([na[hit.any(1), :2], nbn[hit.any(0), :2]], 0))


def glauber_profile(seed: int, b: float, x: np.ndarray, y: np.ndarray,
                    A: int = 208, R: float = 6.62, a: float = 0.546,
                    sigma_nn: float = 6.4, smear: float = 0.4):
    """Participant density of one seeded MC-Glauber event on the (x, y) grid,
    normalised to a maximum of 1; returns (profile[iy][ix], n_participants)."""
    parts = glauber_participants(seed, b, A, R, a, sigma_nn)
    X, Y = np.meshgrid(x, y, indexing="xy")
    prof = np.zeros_like(X)
    for px, py in parts:
        prof += np.exp(-((X - px) ** 2 + (Y - py) ** 2) / (2 * smear * smear))
    if prof.max() > 0:
        prof /= prof.max()
    return prof, len(parts)


def eta_profile(eta, plateau=2.5, width=1.0):
    ae = np.abs(eta)
    return np.where(ae < plateau, 1.0, np.exp(-(ae - plateau) ** 2 / (2 * width * width)))


def glauber3d_setup(nx: int = 101, ny: int = 101, nz: int = 51,
                    xmax: float = 15.0, etamax: float = 7.5,
                    tau0: float = 0.5, dt: float = 0.05, seed: int = 20260001,
                    b: float = 7.0, epeak: float = 50.0, etaS: float = 0.08,
                    eos: Optional[EosTable] = None, ecut: float = 1e-3,
                    nb_peak: float = 0.0) -> Setup:
    """3D viscous single event (seeded MC-Glauber).  Cells whose energy
    density falls below ``ecut`` GeV/fm^3 start as vacuum (e = 0, m = 0), so
    the vacuum-front machinery (Fluid::updateM) is exercised as in real runs."""
    g = Grid(nx, ny, nz, -xmax, xmax, -xmax, xmax, -etamax, etamax)
    x, y, eta = g.coords()
    prof, _ = glauber_profile(seed, b, x, y)
    H = eta_profile(eta)
    e = epeak * H[:, None, None] * prof[None, :, :]  # [iz][iy][ix]
    e = np.where(e < ecut, 0.0, e)
    nb = nb_peak * H[:, None, None] * prof[None, :, :]
    nb = np.where(e > 0, nb, 0.0)
    zero = np.zeros_like(e)
    if eos is None:
        eos = make_cs2_table()
    # v = 0: Q_T = tau e and Q_NB = tau nb, independent of p
    Q = conserved_from_primitive(tau0, e, zero, nb, zero, zero, zero).reshape(7, -1)
    m = (e.reshape(-1) > 0).astype(np.float64)
    tr = dict(TR_DEFAULTS, etaS0=etaS, zetaS0=0.0)
    return Setup("glauber3d", g, eos, tr, 0, 0, tau0, dt, 0.5, Q, m)


def small_glauber3d(n: int = 17, nz: int = 9, seed: int = 20260001, **kw) -> Setup:
    """The 3D viscous physics on a reduced grid that the CPU checkers finish
    in seconds (same physical extent, coarser cells, smaller dt)."""
    kw.setdefault("dt", 0.05)
    kw.setdefault("xmax", 15.0)
    return glauber3d_setup(nx=n, ny=n, nz=nz, seed=seed, **kw)


# --------------------------------------------------------------- snapshots
SNAPSHOT_TAG = b"VHBSNAP1"
SNAPSHOT_FIELDS = (("Q", 7), ("Qh", 7), ("Qprev", 7), ("pi", 10), ("piH", 10), ("Pi", 1),
                   ("PiH", 1), ("m", 3), ("vcc", 1))


def write_snapshot(path: str, grid: Grid, tau: float, dt: float, state: dict) -> None:
    """Grid snapshot read by the C++ driver (Fluid::loadSnapshot): tag
    "VHBSNAP1", int32 nx ny nz 0, float64 bounds tau dt, then the planes
    Q Qh Qprev pi piH Pi PiH m vcc as raw float64 (component-major)."""
    N = grid.ncells
    with open(path, "wb") as f:
        f.write(SNAPSHOT_TAG)
        f.write(np.array([grid.nx, grid.ny, grid.nz, 0], dtype="<i4").tobytes())
        f.write(np.array(list(grid.bounds()) + [tau, dt], dtype="<f8").tobytes())
        for k, nc in SNAPSHOT_FIELDS:
            a = state.get(k)
            if a is None:
                a = np.ones(N) if k == "vcc" else np.zeros((nc, N))
            f.write(np.ascontiguousarray(a, dtype="<f8").reshape(nc, N).tobytes())


def read_snapshot(path: str):
    """(nx, ny, nz, bounds[6], tau, dt, state) of a snapshot file."""
    with open(path, "rb") as f:
        raw = f.read()
    if raw[:8] != SNAPSHOT_TAG:
        raise ValueError("not a grid snapshot: %s" % path)
    nx, ny, nz, _ = np.frombuffer(raw, dtype="<i4", count=4, offset=8)
    hdr = np.frombuffer(raw, dtype="<f8", count=8, offset=24)
    N = int(nx) * int(ny) * int(nz)
    off, state = 88, {}
    for k, nc in SNAPSHOT_FIELDS:
        state[k] = np.frombuffer(raw, dtype="<f8", count=nc * N, offset=off).reshape(nc, N).copy()
        off += nc * N * 8
    if off != len(raw):
        raise ValueError("snapshot size mismatch: %s" % path)
    return int(nx), int(ny), int(nz), hdr[:6].copy(), float(hdr[6]), float(hdr[7]), state


def initial_snapshot_state(setup: "Setup") -> dict:
    """The state an initial-condition model leaves in the cells: Q, Qprev = Q,
    m on all three axes, optional pi/Pi, other fields zero, vcc = 1."""
    N = setup.grid.ncells
    Q = np.array(setup.Q, dtype=np.float64).reshape(7, N)
    Q[:, Q[0] < 0] = 0.0  # Cell::setQ, src/cll.h:75-80
    m = np.repeat(np.asarray(setup.m, dtype=np.float64).reshape(1, N), 3, 0)
    st = dict(Q=Q, Qh=np.zeros((7, N)), Qprev=Q.copy(), m=m, vcc=np.ones((1, N)))
    if setup.pi is not None:
        st["pi"] = np.asarray(setup.pi, dtype=np.float64).reshape(10, N)
    if setup.Pi is not None:
        st["Pi"] = np.asarray(setup.Pi, dtype=np.float64).reshape(1, N)
    return st


def write_params(path: str, setup: "Setup", **extra) -> None:
    """A parameters file in the reference's "name value" format for the
    setup's grid, step and transport coefficients (src/main.cpp:83-156)."""
    g = setup.grid
    tr = dict(zip(TR_FIELDS, setup.tr_vector()))
    lines = ["! written by vhlle_b200.workloads.write_params",
             "nx %d" % g.nx, "ny %d" % g.ny, "nz %d" % g.nz,
             "xmin %r" % g.xmin, "xmax %r" % g.xmax, "ymin %r" % g.ymin, "ymax %r" % g.ymax,
             "etamin %r" % g.etamin, "etamax %r" % g.etamax,
             "tau0 %r" % setup.tau0, "dtau %r" % setup.dt, "e_crit %r" % setup.ecrit,
             "etaS %r" % tr["etaS0"], "zetaS %r" % tr["zetaS0"],
             "etaSparam %d" % setup.etaSparam, "zetaSparam %d" % setup.zetaSparam]
    for k in ("ah", "al", "aRho", "T0", "etaSMin", "etaSEpsilonMin", "etaSShiftMuB",
              "etaSScaleMuB", "zetaSPeakEpsilon", "zetaSScaleBeta", "zetaSSigmaMinus",
              "zetaSSigmaPlus"):
        lines.append("%s %r" % (k, tr[k]))
    for k, v in extra.items():
        lines.append("%s %s" % (k, v if isinstance(v, str) else repr(v)))
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# ------------------------------------------------- event-by-event batches
BATCH_SEED0 = 20263000
BATCH_NZ = (1, 21, 41, 61)


def batch_event(k: int, seed0: int = BATCH_SEED0, nz: Optional[int] = None,
                eos: Optional[EosTable] = None, etaS: float = 0.12, zeta_height: float = 0.05,
                zeta_peak_T: float = 0.175, zeta_width_T: float = 0.02, tau0: float = 0.5,
                dt: float = 0.05) -> Setup:
    """Event k of the event-by-event batch: seed seed0 + k; impact parameter
    uniform on [0, 12] fm from one seeded stream shared by the batch; the
    transverse grid sized to the event's extent (121 cells at b = 0 down to
    61 at b = 12, x, y in [-15, 15] * n / 121 fm); eta cells cycling through
    1, 21, 41, 61 (eta_s in [-7.5, 7.5], or [-0.5, 0.5] boost-invariant for
    one cell); eta/s = 0.12 and a zeta/s Gaussian bump in T (height 0.05 at
    T = 0.175 GeV, width 0.02 GeV: zetaSparam 5)."""
    bs = np.random.default_rng(seed0).uniform(0.0, 12.0, k + 1)
    b = float(bs[k])
    nt = 121 - 2 * int(round(30.0 * b / 12.0))
    nz = BATCH_NZ[k % len(BATCH_NZ)] if nz is None else nz
    xmax = 15.0 * nt / 121.0
    if nz > 1:
        s = glauber3d_setup(nt, nt, nz, xmax=xmax, etamax=7.5, tau0=tau0, dt=dt, seed=seed0 + k,
                            b=b, etaS=etaS, eos=eos)
    else:
        g = Grid(nt, nt, 1, -xmax, xmax, -xmax, xmax, -0.5, 0.5)
        x, y, _ = g.coords()
        prof, _ = glauber_profile(seed0 + k, b, x, y)
        e = 50.0 * prof[None, :, :]
        e = np.where(e < 1e-3, 0.0, e)
        zero = np.zeros_like(e)
        Q = conserved_from_primitive(tau0, e, zero, zero, zero, zero, zero).reshape(7, -1)
        m = (e.reshape(-1) > 0).astype(np.float64)
        tr = dict(TR_DEFAULTS, etaS0=etaS, zetaS0=0.0)
        s = Setup("glauber2d", g, eos or make_cs2_table(), tr, 0, 0, tau0, dt, 0.5, Q, m)
    s.name = "batch_event_%d" % k
    s.tr = dict(s.tr, zetaS0=zeta_height, zetaSPeakT=zeta_peak_T, zetaSWidthT=zeta_width_T)
    s.zetaSparam = 5
    return s


def batch_events(n: int = 256, seed0: int = BATCH_SEED0, **kw):
    """The first n events of the batch (one EoS table shared by all)."""
    eos = kw.pop("eos", None) or make_cs2_table()
    return [batch_event(k, seed0, eos=eos, **kw) for k in range(n)]


# ------------------------------------------------- baryon charge, large events
NB_PEAK = 0.3        # fm^-3, peak of the initial nb profile
NB_TABLE_MAX = 1.0   # fm^-3, top of the table's nb axis
MUB_SLOPE = 1.0      # GeV fm^3: mu_B = MUB_SLOPE * nb
LARGE_SEED0 = 20265000


def nb_table(ne: int = 2000, nn: int = 200) -> EosTable:
    """The e x nb table of the baryon-charge workloads: ``ne`` log e-points
    (1e-4 .. 1e3 GeV/fm^3, the same c_s^2(e) form) x ``nn`` nb-points on
    [0, 1] fm^-3, mu_B linear in nb."""
    return make_cs2_table(ne=ne, nn=nn, nbmax=NB_TABLE_MAX, mub_slope=MUB_SLOPE)


def glauber3d_nb_setup(nx: int = 101, ny: int = 101, nz: int = 51,
                       eos: Optional[EosTable] = None, **kw) -> Setup:
    """The 3D viscous event plus baryon charge: initial nb is the Glauber
    profile scaled to a peak of 0.3 fm^-3; the (e, nb) table is
    ``nb_table()`` unless ``eos`` is given."""
    kw.setdefault("nb_peak", NB_PEAK)
    s = glauber3d_setup(nx, ny, nz, eos=eos if eos is not None else nb_table(), **kw)
    s.name = "glauber3d_nb"
    return s


def with_zeta_bump(s: Setup, height: float = 0.05, peak_T: float = 0.175,
                   width_T: float = 0.02) -> Setup:
    """zeta/s = height exp(-(T - peak_T)^2 / (2 width_T^2)) (zetaSparam 5)."""
    s.tr = dict(s.tr, zetaS0=height, zetaSPeakT=peak_T, zetaSWidthT=width_T)
    s.zetaSparam = 5
    return s


def large_event_setup(k: int = 0, nx: int = 201, ny: int = 201, nz: int = 101,
                      eos: Optional[EosTable] = None, seed0: int = LARGE_SEED0,
                      **kw) -> Setup:
    """Event k of the large-event batch: 201x201x101 on [-20,20]^2 x
    [-10,10], tau0 = 0.4, dtau = 0.02, seed seed0 + k, b = 3 fm, peak
    e = 80 GeV/fm^3, eta/s = 0.08 plus the zeta/s bump (shear, bulk and their
    cross terms), baryon charge and the e x nb table.  Smaller nx, ny, nz
    keep the physical extent (coarser cells)."""
    kw.setdefault("xmax", 20.0)
    kw.setdefault("etamax", 10.0)
    kw.setdefault("tau0", 0.4)
    kw.setdefault("dt", 0.02)
    kw.setdefault("b", 3.0)
    kw.setdefault("epeak", 80.0)
    s = glauber3d_nb_setup(nx, ny, nz, eos=eos, seed=seed0 + k, **kw)
    s.name = "large_event_%d" % k
    return with_zeta_bump(s)
