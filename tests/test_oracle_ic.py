"""The C restatement of the reference's initial-state modules
(oracle/vh_oracle_ic.c) against the modules themselves, compiled unmodified
into oracle/_ref: IcGlissando, IcTrento, ICGubser, IC over the s95p table and
IcPartUrqmd (icModel 5, 7, 4, 2, 3: src/main.cpp:324-366), on seeded synthetic inputs in
the modules' file formats (vhlle_b200/ic_files.py), every named setup.

With the C library's exp and pow (the reference's) the restatement is bit
for bit the reference: Q, Qprev and the fill fractions of every cell and the
two normalisations.  With the correctly rounded exp / pow of the CUDA path
(crmath) it differs only where the library misrounds, by a few ulps; the
CUDA builders are checked against that arm bit for bit (tests/
test_gpu_ic_ref.py).  The setup constants come from the library's own table
(vh_ic_setup_named), so agreement also pins that table to the reference."""
import os

import numpy as np
import pytest

from oracle import pyoracle as P
from vhlle_b200 import capi
from vhlle_b200 import ic_files as F
from vhlle_b200 import workloads as W

needs_ref = pytest.mark.skipif(not P.ref_available(), reason="compiled reference not built")

GLISSANDO_SETUPS = ("LHC276", "RHIC200", "LHC5020", "RHIC62", "AFTER72", "RHIC27")
TRENTO_SETUPS = ("LHC276", "RHIC200", "LHC5020", "RHIC62", "RHIC27")


@pytest.fixture(scope="module")
def grid_setup():
    return W.glauber3d_setup(nx=31, ny=31, nz=11, xmax=12.0, etamax=6.0)


@pytest.fixture(scope="module")
def ref(grid_setup):
    r = P.RefRun(grid_setup)
    yield r
    r.close()


def _same(o, r):
    assert np.array_equal(o["Q"], r["Q"])
    assert np.array_equal(o["Qprev"], r["Qprev"])
    assert np.array_equal(o["m"][0], r["m"])
    assert np.array_equal(o["m"][1], r["m"]) and np.array_equal(o["m"][2], r["m"])


def _close(a, b, rtol):
    scale = np.maximum(np.abs(b).max(axis=1, keepdims=True), 1e-300)
    assert np.all(np.abs(a - b) <= rtol * np.maximum(np.abs(b), 1e-3 * scale))


@needs_ref
def test_s95p_e_equals_reference(ref):
    rng = np.random.default_rng(1)
    s = np.concatenate([10 ** rng.uniform(-5, 3, 4000), [0.0, 1e-300, 5.0, 1e3]])
    lib = P.oracle_lib()
    r = ref.s95p_e(s)
    o = np.array([lib.or_s95p_e(v, 0) for v in s])
    assert np.array_equal(o, r)
    o1 = np.array([lib.or_s95p_e(v, 1) for v in s])
    assert np.all(np.abs(o1 - r) <= 1e-15 * np.abs(r))


@needs_ref
@pytest.mark.parametrize("name", GLISSANDO_SETUPS)
def test_glissando_oracle_equals_reference(name, grid_setup, ref, tmp_path):
    path = str(tmp_path / "sources.txt")
    F.write_glissando(path, F.synthetic_glissando_events(3, seed=5))
    ev = F.read_glissando(path)
    su = capi.ic_setup(capi.IC_GLISSANDO, name)
    r = ref.ic(5, path, name)
    o, norms = P.oracle_ic(grid_setup, 5, ev, su)
    _same(o, r)
    assert (r["Q"][0] > 0).sum() > 500  # matter on the grid
    if su["sNN"] < 100:
        assert (r["Q"][4] > 0).any() and norms[1] > 0
    o1, n1 = P.oracle_ic(grid_setup, 5, ev, su, crmath=True)
    _close(o1["Q"], r["Q"], 1e-14)
    assert np.array_equal(o1["m"], o["m"])
    assert abs(n1[0] - norms[0]) <= 1e-14 * norms[0]


@needs_ref
@pytest.mark.parametrize("name", TRENTO_SETUPS)
def test_trento_oracle_equals_reference(name, grid_setup, ref, tmp_path):
    path = str(tmp_path / "trento.dat")
    F.write_trento(path, F.synthetic_trento_events(2, seed=7, n=60))
    ev = F.read_trento(path)
    su = capi.ic_setup(capi.IC_TRENTO, name)
    r = ref.ic(7, path, name)
    o, norms = P.oracle_ic(grid_setup, 7, ev, su)
    _same(o, r)
    if su["sNN"] >= 2760:
        assert norms[0] == 1.0
    o1, _ = P.oracle_ic(grid_setup, 7, ev, su, crmath=True)
    _close(o1["Q"], r["Q"], 1e-14)


@needs_ref
def test_gubser_oracle_equals_reference(grid_setup, ref):
    r = ref.ic(4)
    o, _ = P.oracle_ic(grid_setup, 4)
    _same(o, r)
    assert np.array_equal(r["Q"], r["Qprev"]) and np.abs(r["Q"][1]).max() > 0
    o1, _ = P.oracle_ic(grid_setup, 4, crmath=True)
    _close(o1["Q"], r["Q"], 1e-14)


@needs_ref
@pytest.mark.parametrize("gv", [1, 0])
def test_table_oracle_equals_reference(gv, grid_setup, ref, tmp_path):
    path = str(tmp_path / "table.dat")
    F.synthetic_song_table().write(path)
    tab = F.read_song_table(path)
    factor = 1.0 if gv == 1 else 8.0
    r = ref.ic(2, path, "", factor, gv)
    o, _ = P.oracle_ic(grid_setup, 2, tab, factor=factor, glauber_var=gv)
    _same(o, r)
    assert (r["Q"][0] > 0).sum() > 100
    o1, _ = P.oracle_ic(grid_setup, 2, tab, factor=factor, glauber_var=gv, crmath=True)
    _close(o1["Q"], r["Q"], 1e-14)


@needs_ref
@pytest.mark.parametrize("Rgt,Rgz", [(1.0, 1.0), (0.8, 0.0)])
def test_urqmd_oracle_equals_reference(Rgt, Rgz, grid_setup, ref, tmp_path):
    """IcPartUrqmd (icModel 3), with the eta smearing and without it."""
    path = str(tmp_path / "particles.txt")
    F.write_urqmd(path, F.synthetic_urqmd_events(3, seed=5, nmean=300))
    ev = F.read_urqmd(path)
    r = ref.ic(3, path, Rgt=Rgt, Rgz=Rgz)
    o, _ = P.oracle_ic(grid_setup, 3, ev, Rgt=Rgt, Rgz=Rgz)
    _same(o, r)
    assert (r["Q"][0] > 0).sum() > 1000 and np.abs(r["Q"][1]).max() > 0
    assert (r["Q"][4] != 0).any() and (r["Q"][5] != 0).any()
    o1, _ = P.oracle_ic(grid_setup, 3, ev, Rgt=Rgt, Rgz=Rgz, crmath=True)
    _close(o1["Q"], r["Q"], 1e-13)


def test_glissando_reader_follows_the_reference_loop(tmp_path):
    """Binary-collision lines (c = 0) are dropped, a line that does not parse
    ends an event that holds sources, and the last event ends at the end of
    the file."""
    path = tmp_path / "g.txt"
    path.write_text("# header\n1 2 1 1\n3 4 0 1\n5 6 -1 1\nbad line\n\n7 8 2 0.5\n")
    ev = F.read_glissando(str(path))
    assert list(ev.npart) == [2, 1]
    assert list(ev.c) == [1, -1, 2] and list(ev.x) == [1.0, 5.0, 7.0]


def test_trento_reader_roundtrip(tmp_path):
    ev = F.synthetic_trento_events(2, seed=3, n=20)
    path = str(tmp_path / "t.dat")
    F.write_trento(path, ev)
    back = F.read_trento(path)
    assert list(back.npart) == list(ev.npart) and np.allclose(back.gmax, ev.gmax)
    for a, b in zip(back.grids, ev.grids):
        assert np.allclose(a, b, rtol=1e-10)
    with open(path) as f:
        head = f.read().split("\n")[:11]
    assert head[2][9:].split()[0] == str(ev.npart[0])
    assert head[9][15:].split()[0] == "20" and float(head[10][12:]) == ev.gmax[0]


def test_song_table_reader_roundtrip(tmp_path):
    tab = F.synthetic_song_table(nx=11, ny=7)
    path = str(tmp_path / "s.dat")
    tab.write(path)
    back = F.read_song_table(path)
    assert np.allclose(back.x, tab.x) and np.allclose(back.y, tab.y)
    assert np.allclose(back.val, tab.val, rtol=1e-11)


def test_ic_setup_names():
    for name in GLISSANDO_SETUPS:
        assert capi.ic_setup(capi.IC_GLISSANDO, name)["Rg"] == 0.4
    for name in TRENTO_SETUPS:
        assert capi.ic_setup(capi.IC_TRENTO, name)["sNN"] > 0
    with pytest.raises(ValueError):
        capi.ic_setup(capi.IC_TRENTO, "AFTER72")
    with pytest.raises(ValueError):
        capi.ic_setup(3, "LHC276")


def _cpp_readers(tmp_path):
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no C++ compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    libdir = os.path.join(root, "vhlle_b200")
    if not os.path.exists(os.path.join(libdir, "libvhlle_b200.so")):
        pytest.skip("library not built")
    exe = str(tmp_path / "ic_readers")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(root, "include"),
                    os.path.join(root, "tests", "cpp", "ic_readers.cpp"), "-L", libdir,
                    "-lvhlle_b200", "-Wl,-rpath," + libdir, "-o", exe], check=True)

    def run(*args):
        out = subprocess.run([exe, *args], capture_output=True, text=True, check=True).stdout
        res, lines, i = {}, out.split("\n"), 0
        while i < len(lines) and lines[i]:
            tag, n = lines[i].split()
            res[tag] = np.array([float(v) for v in lines[i + 1:i + 1 + int(n)]])
            i += 1 + int(n)
        return res
    return run


def test_cpp_readers_equal_the_python_readers(tmp_path):
    """vhb::IcGlissando / IcTrento / IC parse the files as the Python readers
    (and so as the reference's constructors, whose loops both follow),
    including a GLISSANDO file that ends without a newline, whose last event
    the reference does not count."""
    run = _cpp_readers(tmp_path)
    g = str(tmp_path / "g.txt")
    F.write_glissando(g, F.synthetic_glissando_events(3, seed=2))
    ev = F.read_glissando(g)
    got = run("glissando", g, "RHIC200")
    assert np.array_equal(got["npart"], ev.npart) and np.array_equal(got["c"], ev.c)
    assert np.array_equal(got["x"], ev.x) and np.array_equal(got["y"], ev.y)
    cut = str(tmp_path / "g2.txt")
    with open(g) as f:
        text = f.read()
    with open(cut, "w") as f:
        f.write(text.rstrip("\n"))
    assert len(F.read_glissando(cut).npart) == 2
    assert list(run("glissando", cut, "RHIC200")["npart"]) == list(ev.npart[:2])
    t = str(tmp_path / "t.dat")
    F.write_trento(t, F.synthetic_trento_events(2, seed=3, n=17))
    tev = F.read_trento(t)
    got = run("trento", t, "LHC276")
    assert np.array_equal(got["npart"], tev.npart) and list(got["ngrid"]) == [17, 17]
    assert np.array_equal(got["gmax"], tev.gmax)
    assert np.array_equal(got["grid"], np.concatenate([a.reshape(-1) for a in tev.grids]))
    u = str(tmp_path / "u.txt")
    F.write_urqmd(u, F.synthetic_urqmd_events(2, seed=4, nmean=50))
    uev = F.read_urqmd(u)
    assert list(run("urqmd", u)["npart"]) == list(uev.npart)
    s = str(tmp_path / "s.dat")
    F.synthetic_song_table(nx=9, ny=5).write(s)
    tab = F.read_song_table(s)
    got = run("table", s)
    assert np.array_equal(got["x"], tab.x) and np.array_equal(got["y"], tab.y)
    assert np.array_equal(got["val"], tab.val.reshape(-1))
