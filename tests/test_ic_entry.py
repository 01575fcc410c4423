"""The initial-state entry, Cell::setPrimVar (src/cll.cpp:222-241: primitive
e, n, v -> the tau-weighted Q an IC module stores in every cell), against
the reference's own function called through the compiled reference
(oracle/_ref, ref_set_prim_var), bit for bit:

  * workloads.conserved_from_primitive, the Python restatement every
    workload generator uses, with p from the oracle's EoS lookup (itself
    bit-equal to the reference's);
  * vhb::Fluid::setPrimVar of the C++ host layer (include/vhlle_b200.hpp)
    with its own EoS classes (vhb::EoS1f reading the same table file,
    vhb::EoSChiral the same two files, vhb::EoSConformal), compiled here
    from tests/cpp/host_setprimvar.cpp.

Points cover rest (v = 0), moderate and ultra-relativistic flow (|v| up to
0.999), e = 0 and e beyond the table, and nb across the table's axis."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import pyoracle as P
from vhlle_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
needs_ref = pytest.mark.skipif(not P.ref_available(), reason="compiled reference not present")


def _points(n=20000, seed=11, nbmax=0.8):
    rng = np.random.default_rng(seed)
    tau = rng.uniform(0.3, 3.0, n)
    e = 10 ** rng.uniform(-5, 3.3, n)
    e[::50] = 0.0
    nb = rng.uniform(0, nbmax, n) * (rng.uniform(0, 1, n) < 0.7)
    speed = np.concatenate([np.zeros(n // 5), rng.uniform(0, 0.999, n - n // 5)])
    rng.shuffle(speed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    v = d * speed[:, None]
    z = np.zeros(n)
    return np.stack([tau, e, nb, z, z, v[:, 0], v[:, 1], v[:, 2]], 1)


def _setups():
    return {
        "table_nb": W.glauber3d_nb_setup(9, 9, 5, eos=W.nb_table(200, 20)),
        "table_cs2": W.small_glauber3d(9, 5),
        "conformal": W.gubser_setup(nx=9, ny=9),
        "chiral": W.glauber3d_nb_setup(9, 9, 5, eos=W.chiral_eos()),
        "table3": W.glauber3d_nb_setup(9, 9, 5, eos=W.eos3f_table()),
    }


@needs_ref
@pytest.mark.parametrize("name", ["table_nb", "table_cs2", "conformal", "chiral", "table3"])
def test_conserved_from_primitive_equals_reference(name):
    setup = _setups()[name]
    pts = _points()
    ref = P.RefRun(setup).set_prim_var(pts)
    tau, e, nb, _, _, vx, vy, vz = pts.T
    p = P.OracleRun(setup).eos6(e, nb)[:, 4]  # EoS::p
    got = W.conserved_from_primitive(tau, e, p, nb, vx, vy, vz).T
    assert np.array_equal(got[:, :5], ref[:, :5]), np.argwhere(got[:, :5] != ref[:, :5])[:5]
    assert not ref[:, 5:].any()
    assert np.abs(ref[:, 1]).max() > 1.0 and np.abs(ref[:, 4]).max() > 0.1


@needs_ref
@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
@pytest.mark.parametrize("name", ["table_nb", "table_cs2", "conformal", "chiral", "table3"])
def test_host_layer_set_prim_var_equals_reference(name, tmp_path):
    exe = str(tmp_path / "host_setprimvar")
    src = os.path.join(ROOT, "tests", "cpp", "host_setprimvar.cpp")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                   check=True)
    setup = _setups()[name]
    pts = _points(seed=23)
    eos = setup.eos
    if eos.kind == 1:
        arg = str(tmp_path / "eos1f.dat")
        eos.write_eos1f(arg)
        kind = "table"
    elif eos.kind == 2:
        arg = str(tmp_path)
        eos.write_chiral(arg)
        kind = "chiral"
    elif eos.kind == 3:
        arg = str(tmp_path / "eos3f.dat")
        eos.write_eos3f(arg)
        kind = "table3"
    else:
        arg = repr(float(eos.conf_cnst))
        kind = "conformal"
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    pts.tofile(fin)
    subprocess.run([exe, kind, arg, fin, fout], check=True)
    got = np.fromfile(fout).reshape(-1, 7)
    ref = P.RefRun(setup).set_prim_var(pts)
    assert np.array_equal(got, ref), np.argwhere(got != ref)[:5]
