"""The input files of the reference's initial-state modules, read the way the
modules read them, and seeded synthetic stand-ins of their content (the
generators' own outputs, GLISSANDO and TRENTO, are not in the reference
tree):

  * GLISSANDO source lists, one "x y c w" line per source, events separated
    by any line that does not parse (IcGlissando, src/icGlissando.cpp:130-160)
  * TRENTO event grids: an 11-line header (npart on line 3, grid-nsteps on
    line 10, grid-max on line 11) and n rows of n entropy values
    (IcTrento, src/icTrento.cpp:115-179)
  * the (x, y, value) table of s95p::loadSongIC (src/s95p.cpp:43-66)
  * UrQMD particle lists, one "tau x y eta mt px py rap id charge" line per
    particle, events separated as GLISSANDO's (IcPartUrqmd,
    src/icPartUrqmd.cpp:79-103)

The parsed forms feed vh_init_glissando, vh_init_trento, vh_init_table and
vh_init_urqmd (capi.GpuHydro.init_glissando / init_trento / init_table /
init_urqmd)."""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

GLISSANDO_MAX_SOURCES = 10000  # IcGlissando::NP, the reader's array size (src/icGlissando.h:24)


@dataclass
class GlissandoEvents:
    x: np.ndarray      # [nsrc] every event's sources in file order
    y: np.ndarray
    c: np.ndarray      # int32 codes, non-zero
    npart: np.ndarray  # int32 [nevents]

    @property
    def nevents(self) -> int:
        return len(self.npart)


def _parse_source(line: str):
    """`istringstream >> X >> Y >> C >> W` on one line: the four values, or
    None where the extraction fails (too few fields, a field that is not a
    number)."""
    t = line.split()
    if len(t) < 4:
        return None
    try:
        x, y = float(t[0]), float(t[1])
        c = int(t[2])
        float(t[3])
    except ValueError:
        return None
    return x, y, c


def read_glissando(path: str) -> GlissandoEvents:
    """The constructor's reading loop (src/icGlissando.cpp:130-160): sources
    with c != 0 are kept (binary-collision lines, c == 0, are dropped), and a
    line that does not parse ends an event that holds sources."""
    xs: List[float] = []
    ys: List[float] = []
    cs: List[int] = []
    npart: List[int] = []
    np_ev = 0
    with open(path) as f:
        lines = f.read().split("\n")
    # the reference's last getline at end of file yields an empty line,
    # which ends the last event when the file ends with a newline
    for line in lines:
        v = _parse_source(line)
        if v is not None:
            if v[2] != 0:
                xs.append(v[0])
                ys.append(v[1])
                cs.append(v[2])
                np_ev += 1
                if np_ev >= GLISSANDO_MAX_SOURCES:
                    raise ValueError("an event with more sources than the reader's arrays hold")
        elif np_ev > 0:
            npart.append(np_ev)
            np_ev = 0
    if not npart:
        raise ValueError("no GLISSANDO events in %s" % path)
    return GlissandoEvents(np.array(xs), np.array(ys), np.array(cs, dtype=np.int32),
                           np.array(npart, dtype=np.int32))


def write_glissando(path: str, events: List[np.ndarray]) -> None:
    """events: per event an array of rows (x, y, c, w); each event after a
    "# event k" line, which ends the one before."""
    with open(path, "w") as f:
        for k, rows in enumerate(events):
            f.write("# event %d\n" % k)
            for x, y, c, w in rows:
                f.write("%.10g %.10g %d %.6g\n" % (x, y, int(c), w))


def _nucleus(rng, A, R, a):
    """A nucleon positions (x, y) of a Woods-Saxon nucleus (rejection)."""
    out = []
    while len(out) < A:
        r = rng.uniform(0, R + 6 * a, 4 * A)
        keep = rng.uniform(0, 1, r.size) < r ** 2 / (R + 6 * a) ** 2 / (1 + np.exp((r - R) / a))
        out.extend(r[keep][: A - len(out)])
    r = np.array(out)
    ct = rng.uniform(-1, 1, A)
    ph = rng.uniform(0, 2 * math.pi, A)
    st = np.sqrt(1 - ct ** 2)
    return np.stack([r * st * np.cos(ph), r * st * np.sin(ph)], 1)


def synthetic_glissando_events(nevents: int, seed: int, A: int = 197, R: float = 6.38,
                               a: float = 0.535, sigma_nn: float = 4.2, bmax: float = 8.0):
    """Seeded Monte-Carlo Glauber events in the GLISSANDO source layout:
    wounded nucleons of nucleus A (c = +1) and B (c = -1) and, between them,
    binary-collision lines (c = 0, which the reader drops), w = 1."""
    rng = np.random.default_rng(seed)
    d2 = sigma_nn / math.pi
    events = []
    for _ in range(nevents):
        b = bmax * math.sqrt(rng.uniform(0.05, 1.0))
        pa = _nucleus(rng, A, R, a) + [b / 2, 0.0]
        pb = _nucleus(rng, A, R, a) - [b / 2, 0.0]
        dd = ((pa[:, None, :] - pb[None, :, :]) ** 2).sum(-1) <= d2
        wa, wb = dd.any(1), dd.any(0)
        rows = [(x, y, 1, 1.0) for x, y in pa[wa]]
        ia, ib = np.nonzero(dd)
        for i, j in list(zip(ia, ib))[: len(rows) // 3]:
            m = 0.5 * (pa[i] + pb[j])
            rows.append((m[0], m[1], 0, 1.0))
        rows += [(x, y, -1, 1.0) for x, y in pb[wb]]
        events.append(np.array(rows, dtype=object))
    return events


@dataclass
class TrentoEvents:
    grids: List[np.ndarray]  # per event [n][n] in file order (row iy, then ix)
    gmax: np.ndarray         # grid-max of each event
    npart: np.ndarray        # npart of each header

    @property
    def nevents(self) -> int:
        return len(self.grids)


TRENTO_HEADER = ("# event {k}\n# b     = {b:.6f}\n# npart = {npart}\n# mult  = {mult:.6f}\n"
                 "# e2    = 0.1\n# e3    = 0.1\n# e4    = 0.1\n# e5    = 0.1\n"
                 "# grid-step = {step:.6f}\n# grid-nsteps = {n}\n# grid-max = {gmax:.6f}\n")


def write_trento(path: str, ev: TrentoEvents, b: float = 5.0) -> None:
    with open(path, "w") as f:
        for k, g in enumerate(ev.grids):
            n = g.shape[0]
            f.write(TRENTO_HEADER.format(k=k, b=b, npart=int(ev.npart[k]), mult=float(g.sum()),
                                         step=2 * ev.gmax[k] / n, n=n, gmax=float(ev.gmax[k])))
            for row in g:
                f.write(" ".join("%.10e" % v for v in row) + "\n")


def read_trento(path: str) -> TrentoEvents:
    """The constructor's reading loop (src/icTrento.cpp:115-179): npart from
    column 9 of line 3, grid-nsteps from column 15 of line 10, grid-max from
    column 12 of line 11, then n*n values (row iy, then ix); an empty third
    line ends the file."""
    with open(path) as f:
        lines = f.read().split("\n")
    grids, gmax, npart = [], [], []
    i = 0
    while True:
        if i + 3 > len(lines) or lines[i + 2] == "":
            break
        npart.append(int(lines[i + 2][9:].split()[0]))
        n = int(lines[i + 9][15:].split()[0])
        gmax.append(float(lines[i + 10][12:].split()[0]))
        i += 11
        vals: List[float] = []
        while len(vals) < n * n:
            vals.extend(float(t) for t in lines[i].split())
            i += 1
        grids.append(np.array(vals[: n * n]).reshape(n, n))
    if not grids:
        raise ValueError("no TRENTO events in %s" % path)
    return TrentoEvents(grids, np.array(gmax), np.array(npart, dtype=np.int32))


def synthetic_trento_events(nevents: int, seed: int, n: int = 100, gmax: float = 10.0,
                            A: int = 208, R: float = 6.62, a: float = 0.546,
                            sigma_nn: float = 6.4, w: float = 0.5) -> TrentoEvents:
    """Seeded TRENTO-like events: the reduced thickness sqrt(T_A T_B) (p = 0)
    of the wounded nucleons' Gaussians of width w on the n x n grid over
    [-gmax, gmax]^2 (cell centres), npart their count."""
    rng = np.random.default_rng(seed)
    d2 = sigma_nn / math.pi
    step = 2 * gmax / n
    c = -gmax + step * (np.arange(n) + 0.5)
    X, Y = np.meshgrid(c, c)  # [iy][ix]
    grids, npart = [], []
    for _ in range(nevents):
        b = 8.0 * math.sqrt(rng.uniform(0.05, 1.0))
        pa = _nucleus(rng, A, R, a) + [b / 2, 0.0]
        pb = _nucleus(rng, A, R, a) - [b / 2, 0.0]
        dd = ((pa[:, None, :] - pb[None, :, :]) ** 2).sum(-1) <= d2
        wa, wb = pa[dd.any(1)], pb[dd.any(0)]

        def thick(p):
            t = np.zeros_like(X)
            for x, y in p:
                t += np.exp(-((X - x) ** 2 + (Y - y) ** 2) / (2 * w * w))
            return t / (2 * math.pi * w * w)

        grids.append(20.0 * np.sqrt(thick(wa) * thick(wb)))
        npart.append(len(wa) + len(wb))
    return TrentoEvents(grids, np.full(nevents, gmax), np.array(npart, dtype=np.int32))


@dataclass
class SongTable:
    x: np.ndarray    # [NX] as the loader keeps them
    y: np.ndarray    # [NY]
    val: np.ndarray  # [NX][NY] as read

    def write(self, path: str) -> None:
        with open(path, "w") as f:
            f.write("%d %d\n" % (len(self.x), len(self.y)))
            for ix, xv in enumerate(self.x):
                for iy, yv in enumerate(self.y):
                    f.write("%.10g %.10g %.12g\n" % (xv, yv, self.val[ix, iy]))


def read_song_table(path: str) -> SongTable:
    """s95p::loadSongIC's reading (src/s95p.cpp:50-60): NX NY, then NX*NY
    triplets x y value (ix outer); x[ix] keeps the last x read in its row and
    y[iy] the value read in the last row."""
    with open(path) as f:
        tok = f.read().split()
    NX, NY = int(tok[0]), int(tok[1])
    v = np.array([float(t) for t in tok[2:2 + 3 * NX * NY]]).reshape(NX, NY, 3)
    return SongTable(v[:, -1, 0].copy(), v[-1, :, 1].copy(), v[:, :, 2].copy())


def synthetic_song_table(nx: int = 101, ny: int = 101, xmax: float = 12.0,
                         s0: float = 60.0, r0: float = 4.0) -> SongTable:
    """An entropy-density table s0 (1 + exp((r - r0) / 0.6))^-1 on a uniform
    grid over [-xmax, xmax]^2, elliptic (x stretched by 0.8)."""
    x = np.linspace(-xmax, xmax, nx)
    y = np.linspace(-xmax, xmax, ny)
    X, Y = np.meshgrid(x, y, indexing="ij")
    r = np.sqrt((X / 0.8) ** 2 + Y ** 2)
    return SongTable(x, y, s0 / (1 + np.exp((r - r0) / 0.6)))


# ------------------------------------------------------ UrQMD particle lists
URQMD_MAX_PARTICLES = 10000  # IcPartUrqmd::NP (src/icPartUrqmd.h:11)


@dataclass
class UrqmdEvents:
    p: np.ndarray       # [n][8] tau, x, y, eta, mt, px, py, rap; every event in file order
    id: np.ndarray      # int32 [n] particle id
    charge: np.ndarray  # int32 [n]
    npart: np.ndarray   # int32 [nevents]

    @property
    def nevents(self) -> int:
        return len(self.npart)


def _parse_particle(line: str):
    """`istringstream >> Tau >> X >> Y >> Eta >> Mt >> Px >> Py >> Rap >> Id
    >> Charge` on one line, or None where it fails."""
    t = line.split()
    if len(t) < 10:
        return None
    try:
        v = [float(x) for x in t[:8]]
        return v, int(t[8]), int(t[9])
    except ValueError:
        return None


def read_urqmd(path: str) -> UrqmdEvents:
    """IcPartUrqmd's reading loop (src/icPartUrqmd.cpp:79-103): a line that
    parses is a particle, a line that does not ends an event that holds
    particles (the end of the file, after a last newline, too)."""
    rows, ids, ch, npart = [], [], [], []
    n = 0
    with open(path) as f:
        lines = f.read().split("\n")
    for line in lines:
        v = _parse_particle(line)
        if v is not None:
            rows.append(v[0])
            ids.append(v[1])
            ch.append(v[2])
            n += 1
            if n >= URQMD_MAX_PARTICLES:
                raise ValueError("an event with more particles than the reader's arrays hold")
        elif n > 0:
            npart.append(n)
            n = 0
    if not npart:
        raise ValueError("no particle events in %s" % path)
    return UrqmdEvents(np.array(rows).reshape(-1, 8), np.array(ids, dtype=np.int32),
                       np.array(ch, dtype=np.int32), np.array(npart, dtype=np.int32))


def write_urqmd(path: str, ev: UrqmdEvents) -> None:
    """One "tau x y eta mt px py rap id charge" line per particle, each
    event after a "# event k" line (which ends the one before)."""
    with open(path, "w") as f:
        base = 0
        for k, n in enumerate(ev.npart):
            f.write("# event %d\n" % k)
            for j in range(base, base + n):
                f.write(" ".join("%.10g" % v for v in ev.p[j]) + " %d %d\n" % (ev.id[j], ev.charge[j]))
            base += n


def synthetic_urqmd_events(nevents: int, seed: int, nmean: int = 400, tau0: float = 0.5,
                           R: float = 4.0) -> UrqmdEvents:
    """Seeded particle lists on the tau0 hypersurface: positions Gaussian in
    x, y (width R) and in eta (width 1.5), thermal-like transverse momenta,
    rapidities near eta, a nucleon / pion / kaon mix of ids and charges (a
    few baryons with |id| < 56 and charged mesons)."""
    rng = np.random.default_rng(seed)
    rows, ids, ch, npart = [], [], [], []
    for _ in range(nevents):
        n = int(rng.integers(nmean // 2, nmean + nmean // 2))
        x, y = rng.normal(0, R, n), rng.normal(0, R, n)
        eta = rng.normal(0, 1.5, n)
        m = rng.choice([0.938, 0.138, 0.494], n, p=[0.25, 0.6, 0.15])
        pt = rng.exponential(0.45, n)
        phi = rng.uniform(0, 2 * np.pi, n)
        px, py = pt * np.cos(phi), pt * np.sin(phi)
        mt = np.sqrt(m * m + pt * pt)
        rap = eta + rng.normal(0, 0.3, n)
        pid = np.where(m > 0.9, rng.choice([1, 17, -1], n, p=[0.7, 0.2, 0.1]),
                       np.where(m > 0.3, 106, 101))
        c = np.where(m > 0.9, np.where(pid > 0, 1, -1) * (rng.uniform(0, 1, n) < 0.4),
                     rng.choice([-1, 0, 1], n))
        rows.append(np.stack([np.full(n, tau0), x, y, eta, mt, px, py, rap], 1))
        ids.append(pid)
        ch.append(c)
        npart.append(n)
    return UrqmdEvents(np.concatenate(rows), np.concatenate(ids).astype(np.int32),
                       np.concatenate(ch).astype(np.int32), np.array(npart, dtype=np.int32))
