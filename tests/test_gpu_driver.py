"""Device driver-loop pieces through the C ABI against the oracle: the
eta-CFL substeps (vh_advance, src/main.cpp:405-419) and the x2 transverse
resize (vh_resize2x, expandGrid2x src/main.cpp:246-271), bit-for-bit."""
import numpy as np
import pytest

import pyoracle as P
from helpers import compare_states, gpu_state_as_oracle
from vhlle_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _drive(run, setup, nloops, dtau, tau_resize):
    g = setup.grid
    counts, resized = [], False
    for _ in range(nloops):
        counts.append(run.advance(dtau, g.etamin, g.etamax, g.nz))
        if run_tau(run) >= tau_resize and not resized:
            assert run.resize2x() == 1
            resized = True
    return counts, resized


def run_tau(run):
    return run.tau_now if hasattr(run, "tau_now") else run.tau


@pytest.mark.parametrize("case", [
    ("glauber_17x17x9_tau005", lambda: W.small_glauber3d(17, 9, tau0=0.05, dt=0.1), 0.1, 8, 0.3),
    ("glauber_16x16x7_even", lambda: W.small_glauber3d(16, 7, tau0=0.04, dt=0.1, b=4.0), 0.1, 7,
     0.2),
    ("glauber_33x33x17", lambda: W.small_glauber3d(33, 17, tau0=0.1, dt=0.1), 0.1, 10, 0.5),
], ids=lambda c: c[0])
def test_gpu_substeps_and_resize_equal_oracle(case):
    from vhlle_b200.capi import GpuHydro
    name, fac, dtau, nloops, tres = case
    setup = fac()
    o = P.OracleRun(setup)
    d = GpuHydro(setup)
    co, ro = _drive(o, setup, nloops, dtau, tres)
    cd, rd = _drive(d, setup, nloops, dtau, tres)
    assert co == cd and ro and rd
    assert max(co) > 1
    assert o.tau_now == d.tau
    assert o.dt == d.dtau
    assert np.array_equal(o.grid_coords(), d.grid_coords())
    d.sync()
    assert d.error_bits() == 0
    bad = compare_states(gpu_state_as_oracle(d.get_state()), o.get_state())
    assert not bad, bad
    # totals on the resized grid (reduction order differs: 1e-10)
    to, td = o.totals(), d.totals()
    for k in P.TOTALS:
        a, b = to[k], td[k]
        assert abs(a - b) <= 1e-10 * max(abs(a), abs(b)) + 1e-300, (k, a, b)
    d.close()


def test_gpu_resize_2d_nan_eta_bounds():
    """nz = 1: the reference's getZ(0) = etamin + 0*inf is NaN, and the
    resized 2D grid carries it; evolution continues as in the oracle."""
    from vhlle_b200.capi import GpuHydro
    setup = W.gubser_setup(nx=21, ny=21)
    o, d = P.OracleRun(setup), GpuHydro(setup)
    o.step(2)
    d.step(2)
    assert o.resize2x() == 1 and d.resize2x() == 1
    go, gd = o.grid_coords(), d.grid_coords()
    assert ((go == gd) | (np.isnan(go) & np.isnan(gd))).all(), (go, gd)
    o.step(3)
    d.step(3)
    bad = compare_states(gpu_state_as_oracle(d.get_state()), o.get_state())
    assert not bad, bad
    d.close()


def test_gpu_resize_keeps_asymmetric_grid():
    from vhlle_b200.capi import GpuHydro
    setup = W.small_glauber3d(13, 5)
    g = setup.grid
    setup.grid = W.Grid(g.nx, g.ny, g.nz, g.xmin + 1.0, g.xmax + 1.0, g.ymin, g.ymax, g.etamin,
                        g.etamax)
    d = GpuHydro(setup)
    before = d.get_state()
    dt0 = d.dtau
    assert d.resize2x() == 0
    assert d.dtau == dt0
    assert not compare_states(d.get_state(), before)
    d.close()


def test_cpp_driver_loop_equals_oracle(tmp_path):
    """vhlle_run (C++ host layer over the C ABI) runs the reference driver
    loop -- substeps at small tau, outputSurface every iteration, the x2
    resize at tauGridResize, stop at tauMax or on an empty surface -- from a
    snapshot.  Its final grid equals the oracle driven through the same loop
    bit-for-bit; its printed element counts equal the oracle's and its
    freezeout.dat records (the corona at tau0, then every surface) match to
    1e-12 (15 printed digits)."""
    import subprocess
    from vhlle_b200 import build as B
    drv = B.build_driver()
    setup = W.small_glauber3d(17, 9, tau0=0.05, dt=0.1)
    ic = str(tmp_path / "ic.vhb")
    W.write_snapshot(ic, setup.grid, setup.tau0, setup.dt, W.initial_snapshot_state(setup))
    params = str(tmp_path / "params.txt")
    tau_max, tau_resize = 0.75, 0.3
    W.write_params(params, setup, tauMax=tau_max, tauGridResize=tau_resize, eos1fFile=str(
        tmp_path / "eos.dat"))
    setup.eos.write_eos1f(str(tmp_path / "eos.dat"))
    out = tmp_path / "out"
    run = subprocess.run([drv, "-params", params, "-ISinput", ic, "-outputDir", str(out)],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr
    proc_out = run.stdout
    assert "grid resize" in proc_out and "timestep reduced by 2" in proc_out

    o = P.OracleRun(setup)
    g = setup.grid
    resized = False
    # Fluid::outputCorona at tau0 opens the freeze-out file
    corona, _ = o.corona()
    assert "corona elements : %d" % len(corona) in proc_out
    recs, counts, nsusp = [corona], [], []
    while True:
        o.advance(setup.dt, g.etamin, g.etamax, g.nz)
        # Fluid::outputSurface; the Fluid's step is the full dtau (doubled
        # by the resize), which is what the oracle's step is between advances
        r, acc = o.surface(dtf=o.dt)
        recs.append(r)
        counts.append(len(r))
        nsusp.append(int(acc["nsusp"]))
        if o.tau_now >= tau_resize and not resized:
            assert o.resize2x() == 1
            resized = True
        if not (o.tau_now < tau_max + 0.0001 and len(r) > 0):
            break
    nx, ny, nz, b, tau, dt, st = W.read_snapshot(str(out / "final.vhb"))
    assert tau == o.tau_now and dt == o.dt
    og = o.grid
    assert np.array_equal(b, [og.xmin, og.xmax, og.ymin, og.ymax, og.zmin, og.zmax])
    exp = o.get_state()
    bad = compare_states(st, exp)
    assert not bad, bad
    # the printed surface lines and the freezeout.dat records
    printed = []
    for line in proc_out.splitlines():
        w = line.split()
        if len(w) == 9 and w[6].isdigit() and w[7].isdigit():
            printed.append((int(w[6]), int(w[7])))
    assert printed == list(zip(counts, nsusp)), (printed, counts, nsusp)
    assert sum(counts) > 0
    fz = P.read_freezeout(str(out / "freezeout.dat"))
    ref = np.concatenate(recs)[:, :27]
    assert fz.shape == ref.shape
    ok = np.abs(fz - ref) <= 1e-12 * np.maximum(np.abs(fz), np.abs(ref)) + 1e-300
    assert ok.all(), np.argwhere(~ok)[:5]


def test_cpp_driver_vorticity_equals_oracle(tmp_path):
    """vhlle_run with the params key `vorticity 1` (src/main.cpp:135,
    379-391): DIR/beta.dat holds Fluid::printDbetaHeader's lines after the
    corona, then every iteration's beta.dat lines, through the substeps and
    the x2 resize; they match the oracle's to 1e-12 (15 printed digits,
    plus a floor for the Jacobian's cosh/sinh cancellation)."""
    import subprocess
    from vhlle_b200 import build as B
    drv = B.build_driver()
    setup = W.small_glauber3d(17, 9, tau0=0.05, dt=0.1)
    ic = str(tmp_path / "ic.vhb")
    W.write_snapshot(ic, setup.grid, setup.tau0, setup.dt, W.initial_snapshot_state(setup))
    params = str(tmp_path / "params.txt")
    tau_max, tau_resize = 0.55, 0.3
    W.write_params(params, setup, tauMax=tau_max, tauGridResize=tau_resize, vorticity=1,
                   eos1fFile=str(tmp_path / "eos.dat"))
    setup.eos.write_eos1f(str(tmp_path / "eos.dat"))
    out = tmp_path / "out"
    run = subprocess.run([drv, "-params", params, "-ISinput", ic, "-outputDir", str(out)],
                         capture_output=True, text=True, timeout=300)
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr
    assert "grid resize" in run.stdout

    o = P.OracleRun(setup, vorticity=True)
    g = setup.grid
    corona, _ = o.corona()
    rows, resized = [], False
    while True:
        o.advance(setup.dt, g.etamin, g.etamax, g.nz)
        r, _, beta = o.surface_beta(dtf=o.dt)
        rows.append(np.concatenate([r[:, :16], beta, r[:, 27:28]], axis=1))
        if o.tau_now >= tau_resize and not resized:
            assert o.resize2x() == 1
            resized = True
        if not (o.tau_now < tau_max + 0.0001 and len(r) > 0):
            break
    with open(out / "beta.dat") as f:
        head = [f.readline() for _ in range(3)]
    assert head[0].startswith("# The derivatives of") and all(h.startswith("#") for h in head)
    assert head[1].strip() == "# Number of corona cells: %d" % len(corona)
    from make_golden import read_beta
    got = read_beta(str(out / "beta.dat"))
    exp = np.concatenate(rows)
    assert got.shape == exp.shape and len(exp) > 0
    scale = np.maximum(np.abs(got[:, 16:32]).max(axis=1), np.abs(exp[:, 16:32]).max(axis=1))[:, None]
    ok = np.abs(got - exp) <= 1e-12 * np.maximum(np.abs(got), np.abs(exp)) + 1e-13 * scale + 1e-300
    assert ok.all(), np.argwhere(~ok)[:5]


def test_cpp_driver_chiral_eos_equals_oracle(tmp_path):
    """vhlle_run with the reference's default eosType 1 and its EoSChiral
    tables under ./eos (src/main.cpp:291-292, src/eoChiral.cpp:153-156)
    ends on the oracle's grid, bit for bit."""
    import subprocess
    from vhlle_b200 import build as B
    drv = B.build_driver()
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=W.chiral_eos())
    setup.eos.write_chiral(str(tmp_path))
    ic = str(tmp_path / "ic.vhb")
    W.write_snapshot(ic, setup.grid, setup.tau0, setup.dt, W.initial_snapshot_state(setup))
    params = str(tmp_path / "params.txt")
    tau_max = setup.tau0 + 3.5 * setup.dt
    W.write_params(params, setup, tauMax=tau_max, tauGridResize=100.0, eosType=1)
    run = subprocess.run([drv, "-params", params, "-ISinput", ic, "-outputDir", "out"],
                         capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr
    assert "hydro EoS: EoSChiral" in run.stdout
    o = P.OracleRun(setup)
    g = setup.grid
    while True:
        o.advance(setup.dt, g.etamin, g.etamax, g.nz)
        r, _ = o.surface(dtf=o.dt)
        if not (o.tau_now < tau_max + 0.0001 and len(r) > 0):
            break
    nx, ny, nz, b, tau, dt, st = W.read_snapshot(str(tmp_path / "out" / "final.vhb"))
    assert tau == o.tau_now
    bad = compare_states(st, o.get_state())
    assert not bad, bad


@pytest.mark.parametrize("eos_type", [2, 4], ids=["EoSAZH", "EoSCMFe"])
def test_cpp_driver_table_eos_equals_oracle(tmp_path, eos_type):
    """vhlle_run with eosType 2 (EoSAZH, tables under ./eos/azhydro0p2,
    src/main.cpp:293-294, src/eoAZH.cpp:110-117) or 4 (EoSCMFe, ./eos/cmfe.dat
    and ./eos/cmfe_small.dat, src/main.cpp:297-298, src/eoCMFe.cpp:194-197)
    ends on the oracle's grid, bit for bit."""
    import subprocess
    from vhlle_b200 import build as B
    drv = B.build_driver()
    eos = W.azh_eos_table() if eos_type == 2 else W.cmfe_eos_table()
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=eos)
    (eos.write_azh if eos_type == 2 else eos.write_cmfe)(str(tmp_path))
    ic = str(tmp_path / "ic.vhb")
    W.write_snapshot(ic, setup.grid, setup.tau0, setup.dt, W.initial_snapshot_state(setup))
    params = str(tmp_path / "params.txt")
    tau_max = setup.tau0 + 3.5 * setup.dt
    W.write_params(params, setup, tauMax=tau_max, tauGridResize=100.0, eosType=eos_type)
    run = subprocess.run([drv, "-params", params, "-ISinput", ic, "-outputDir", "out"],
                         capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr
    assert ("hydro EoS: " + ("EoSAZH" if eos_type == 2 else "EoSCMFe")) in run.stdout
    o = P.OracleRun(setup)
    g = setup.grid
    while True:
        o.advance(setup.dt, g.etamin, g.etamax, g.nz)
        r, _ = o.surface(dtf=o.dt)
        if not (o.tau_now < tau_max + 0.0001 and len(r) > 0):
            break
    nx, ny, nz, b, tau, dt, st = W.read_snapshot(str(tmp_path / "out" / "final.vhb"))
    assert tau == o.tau_now
    bad = compare_states(st, o.get_state())
    assert not bad, bad


@pytest.mark.parametrize("kind", [0, 1], ids=["EoSHadron", "EoSSmash"])
def test_cpp_driver_freezeout_eos_equals_oracle(tmp_path, kind):
    """vhlle_run with eosTypeHadron 0 / 1 and the reference's table under
    ./eos (eos/eosHadronLog.dat, eos/hadgas_eos_SMASH.dat at 101 x 51 x 51,
    src/main.cpp:304-309): the corona and every surface of freezeout.dat
    are those of the oracle with that freeze-out EoS (1e-12, 15 printed
    digits), and the final grid, which the freeze-out EoS does not touch,
    is the oracle's bit for bit."""
    import os
    import subprocess
    from vhlle_b200 import build as B
    drv = B.build_driver()
    h = W.hadron_eos_table() if kind == 0 else W.smash_eos_table(101, 51, 51)
    os.makedirs(tmp_path / "eos")
    if kind == 0:
        h.write_hadron(str(tmp_path / "eos" / "eosHadronLog.dat"))
    else:
        h.write_smash(str(tmp_path / "eos" / "hadgas_eos_SMASH.dat"))
    setup = W.glauber3d_nb_setup(17, 17, 9, eos=W.nb_table(200, 20))
    setup.eos.write_eos1f(str(tmp_path / "eos.dat"))
    ic = str(tmp_path / "ic.vhb")
    W.write_snapshot(ic, setup.grid, setup.tau0, setup.dt, W.initial_snapshot_state(setup))
    params = str(tmp_path / "params.txt")
    tau_max = setup.tau0 + 4.5 * setup.dt
    W.write_params(params, setup, tauMax=tau_max, tauGridResize=100.0, eosTypeHadron=kind,
                   eos1fFile=str(tmp_path / "eos.dat"))
    run = subprocess.run([drv, "-params", params, "-ISinput", ic, "-outputDir", "out"],
                         capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert run.returncode == 0, run.stdout[-2000:] + run.stderr
    assert ("freeze-out EoS: " + ("EoSHadron" if kind == 0 else "EoSSmash")) in run.stdout
    o = P.OracleRun(setup, surface_eos=h)
    g = setup.grid
    corona, _ = o.corona()
    recs = [corona]
    while True:
        o.advance(setup.dt, g.etamin, g.etamax, g.nz)
        r, _ = o.surface(dtf=o.dt)
        recs.append(r)
        if not (o.tau_now < tau_max + 0.0001 and len(r) > 0):
            break
    fz = P.read_freezeout(str(tmp_path / "out" / "freezeout.dat"))
    ref = np.concatenate(recs)[:, :27]
    assert fz.shape == ref.shape and len(ref) > len(corona)
    ok = np.abs(fz - ref) <= 1e-12 * np.maximum(np.abs(fz), np.abs(ref)) + 1e-300
    assert ok.all(), np.argwhere(~ok)[:5]
    nx, ny, nz, b, tau, dt, st = W.read_snapshot(str(tmp_path / "out" / "final.vhb"))
    assert tau == o.tau_now
    bad = compare_states(st, o.get_state())
    assert not bad, bad
