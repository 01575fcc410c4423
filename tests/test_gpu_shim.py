"""The reference-side binding (include/vhlle_b200_refshim.hpp: HydroB200
over the reference's own Fluid, Cell, EoS1f and TransportCoeff objects)
compiled with the reference's classes into oracle/_ref/shim_check
(`make -C oracle ref`).  One event runs through the reference's
Hydro::performStep and through HydroB200 from the same initial state; after
HydroB200::download every Cell holds the reference's bits, and the
reference's own Fluid::outputSurface writes the same freeze-out file from
either Fluid."""
import os
import subprocess

import numpy as np
import pytest

from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "shim_check")


def _write_ic(path, setup):
    g = setup.grid
    with open(path, "wb") as f:
        np.array([g.nx, g.ny, g.nz], dtype=np.int32).tofile(f)
        np.array(list(g.bounds()) + [setup.tau0, setup.dt, setup.ecrit, setup.tr["etaS0"]],
                 dtype=np.float64).tofile(f)
        np.ascontiguousarray(setup.Q, dtype=np.float64).tofile(f)
        np.ascontiguousarray(setup.m, dtype=np.float64).tofile(f)


@pytest.mark.skipif(not os.path.exists(EXE), reason="shim_check not built (needs the reference)")
@pytest.mark.parametrize("case", [("glauber_33x33x17", lambda: W.small_glauber3d(33, 17, b=6.0), 12),
                                  ("glauber_nb_25x25x13",
                                   lambda: W.glauber3d_nb_setup(25, 25, 13, eos=W.nb_table(200, 20)),
                                   8)],
                         ids=lambda c: c[0])
def test_reference_binding_steps_the_reference_event(case, tmp_path):
    _, fac, steps = case
    setup = fac()
    ic, eos = str(tmp_path / "ic.bin"), str(tmp_path / "eos1f.dat")
    _write_ic(ic, setup)
    setup.eos.write_eos1f(eos)
    a, b = tmp_path / "ref", tmp_path / "b200"
    a.mkdir()
    b.mkdir()
    r = subprocess.run([EXE, ic, eos, str(steps), str(a), str(b)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    words = r.stdout.split()
    assert words[words.index("values") + 1] == "0"
    n = int(words[-1])
    assert n > 100, r.stdout
    fa = (a / "freezeout.dat.unfinished").read_bytes()
    fb = (b / "freezeout.dat.unfinished").read_bytes()
    assert fa == fb
