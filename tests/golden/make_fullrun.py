"""Full-run digests of the benchmark's 3D events, from the reference itself.

The fixtures written here pin whole runs, not single steps: every field of
every cell is hashed every ``EVERY`` steps (a bit-for-bit pin of the full
state, small enough to commit), the interior totals are kept at the same
points, and every freeze-out call is summarised (element count, the printed
totals line, per-column sums of the records).  A sample of cells keeps the
final values, so that a digest mismatch can be reported as a relative error.

Arms (each a separate process; they run in parallel):

  ref  the reference compiled from its sources (oracle/_ref), Hydro::
       performStep + Fluid::outputSurface, exp/pow from the C library;
  cr   the oracle (vh_oracle.c) with exp and x^(1/4) correctly rounded, as
       the CUDA path evaluates them (only needed where the run evaluates an
       exp-based transport form: elsewhere both arms give the same bits).

For cases with a ``cr`` arm the merge step also compares the two arms'
full states at every checkpoint (saved under the scratch directory) and
stores the per-field maximum relative difference and the number of values
beyond 1e-12 and 1e-8: the reference's distance from correctly rounded math.

    python tests/golden/make_fullrun.py run  CASE ARM SCRATCH   # one arm
    python tests/golden/make_fullrun.py merge CASE SCRATCH      # -> fullrun_CASE.npz
    python tests/golden/make_fullrun.py all  SCRATCH            # every case, arms in parallel

The setups come from ``vhlle_b200.workloads`` (seeded), so the fixtures hold
no initial state, only its digest (checked by the test before it steps).
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from vhlle_b200 import workloads as W  # noqa: E402

FIELDS = ("Q", "Qh", "Qprev", "pi", "piH", "Pi", "PiH", "m", "vcc")
EVERY = 10          # steps between state digests
NSAMPLE = 4096      # cells whose final values are kept
SURF_COLS = 29      # extended freezeout.dat records (with e and nb)


def c5_zeta2():
    """The large event (201x201x101, shear + bulk + cross terms + nb, the
    (e, nb) table) with the reference's zeta/s form 2 in place of the bump,
    which the reference has no branch for."""
    s = W.large_event_setup(0)
    s.zetaSparam = 2
    s.name = "large_event_zeta2"
    return s


# name: (setup factory, steps, surface every n steps, arms)
CASES = {
    # the 101x101x51 viscous event: full 300 steps, surface every 2
    "c2_glauber3d": (lambda: W.glauber3d_setup(), 300, 2, ("ref",)),
    # the same event with baryon charge on the 2000 x 200 (e, nb) table
    "c4_glauber3d_nb": (lambda: W.glauber3d_nb_setup(), 300, 2, ("ref",)),
    # the first 100 of the large event's 1000 steps, surface every 5
    "c5_large_zeta2": (c5_zeta2, 100, 5, ("ref", "cr")),
}


def canonical(a):
    """float64 array with -0.0 as +0.0 and one NaN bit pattern, so that a
    digest compares values, not zero signs or NaN payloads."""
    a = np.ascontiguousarray(a, dtype=np.float64) + 0.0
    a[np.isnan(a)] = np.nan
    return a


def field_digest(a):
    return hashlib.sha256(canonical(a).tobytes()).hexdigest()[:32]


def state_digests(st):
    return [field_digest(st[k]) for k in FIELDS]


def sample_cells(setup, n=NSAMPLE, seed=7):
    """n cells, half among those with matter at the start, half anywhere."""
    N = setup.grid.ncells
    rng = np.random.default_rng(seed)
    matter = np.flatnonzero(setup.Q[0] > 0)
    a = rng.choice(matter, min(n // 2, len(matter)), replace=False)
    b = rng.choice(N, n - len(a), replace=False)
    return np.unique(np.concatenate([a, b]))


def surface_summary(rec):
    rec = np.asarray(rec, dtype=np.float64).reshape(-1, SURF_COLS)
    return rec.sum(0), np.abs(rec).sum(0)


def _read_new_records(path, pos):
    """Element lines appended to freezeout.dat since byte offset pos."""
    with open(path, "rb") as f:
        f.seek(pos)
        data = f.read()
        end = f.tell()
    if not data.strip():
        return np.zeros((0, SURF_COLS)), end
    v = np.array(data.split(), dtype=np.float64)
    return v.reshape(-1, SURF_COLS), end


def run_arm(case, arm, scratch):
    import pyoracle as P
    fac, nsteps, every_surf, arms = CASES[case]
    assert arm in arms, (case, arm)
    setup = fac()
    os.makedirs(scratch, exist_ok=True)
    keep_states = len(arms) > 1
    if arm == "ref":
        run = P.RefRun(setup)
    else:
        run = P.OracleRun(setup, crmath=True)
    idx = sample_cells(setup)
    out = dict(check_steps=[], digests=[], totals=[], tau=[], surf_steps=[], surf_n=[],
               surf_sum=[], surf_abs=[], surf_etot=[], surf_nsusp=[])
    t0 = time.time()
    with tempfile.TemporaryDirectory() as d:
        fo = os.path.join(d, "freezeout.dat.unfinished")
        pos = 0
        etot = 0.0  # Fluid::EtotSurf, summed over the calls as the reference prints it
        for step in range(1, nsteps + 1):
            run.step(1)
            if step % every_surf == 0:
                if arm == "ref":
                    n, line = run.output_surface(d, extend=True)
                    rec, pos = _read_new_records(fo, pos)
                    assert len(rec) == n, (len(rec), n)
                    words = line.split()
                    etot, nsusp = float(words[5]), int(words[7])
                else:
                    rec, info = run.surface(cap=4000000)
                    etot += info["EtotSurf"]
                    n, nsusp = len(rec), int(info["nsusp"])
                s, a = surface_summary(rec)
                out["surf_steps"].append(step)
                out["surf_n"].append(n)
                out["surf_sum"].append(s)
                out["surf_abs"].append(a)
                out["surf_etot"].append(etot)
                out["surf_nsusp"].append(nsusp)
            if step % EVERY == 0 or step == nsteps:
                st = run.get_state()
                tot = run.totals()
                out["check_steps"].append(step)
                out["digests"].append(state_digests(st))
                out["totals"].append([tot[k] for k in P.TOTALS])
                out["tau"].append(run.tau_now)
                if keep_states:
                    np.savez(os.path.join(scratch, "%s_%s_%04d.npz" % (case, arm, step)),
                             **{k: st[k] for k in FIELDS})
                print("%s/%s step %d  %.0f s" % (case, arm, step, time.time() - t0), flush=True)
        st = run.get_state()
    for k in FIELDS:
        v = np.asarray(st[k]).reshape(-1, setup.grid.ncells)
        out["sample_" + k] = v[:, idx]
    out["sample_idx"] = idx
    out["q0_digest"] = field_digest(setup.Q)
    out["seconds"] = time.time() - t0
    np.savez(os.path.join(scratch, "%s_%s.npz" % (case, arm)),
             **{k: np.array(v) for k, v in out.items()})


def _maxrel(a, b):
    a = canonical(a)
    b = canonical(b)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    d = np.where(same, 0.0, np.abs(a - b))
    scale = np.maximum(np.abs(a), np.abs(b))
    rel = np.where(same, 0.0, d / np.where(scale > 0, scale, 1.0))
    return float(rel.max()), int((rel > 1e-12).sum()), int((rel > 1e-8).sum()), int((~same).sum())


def merge(case, scratch):
    fac, nsteps, every_surf, arms = CASES[case]
    z = {arm: dict(np.load(os.path.join(scratch, "%s_%s.npz" % (case, arm)))) for arm in arms}
    ref = z["ref"]
    out = dict(nsteps=np.array(nsteps), every=np.array(EVERY), every_surf=np.array(every_surf),
               fields=np.array(FIELDS), ref_seconds=ref["seconds"])
    for k in ("check_steps", "digests", "totals", "tau", "surf_steps", "surf_n", "surf_sum",
              "surf_abs", "surf_etot", "surf_nsusp", "sample_idx", "q0_digest"):
        out[k] = ref[k]
    for k in FIELDS:
        out["sample_" + k] = ref["sample_" + k]
    if "cr" in z:
        cr = z["cr"]
        assert np.array_equal(cr["check_steps"], ref["check_steps"])
        for k in ("digests", "totals", "surf_n", "surf_sum", "surf_abs", "surf_etot",
                  "surf_nsusp"):
            out["cr_" + k] = cr[k]
        for k in FIELDS:
            out["cr_sample_" + k] = cr["sample_" + k]
        # the two arms' full states at every checkpoint
        rows = []
        for step in ref["check_steps"]:
            a = np.load(os.path.join(scratch, "%s_ref_%04d.npz" % (case, int(step))))
            b = np.load(os.path.join(scratch, "%s_cr_%04d.npz" % (case, int(step))))
            rows.append([_maxrel(a[k], b[k]) for k in FIELDS])
        rows = np.array(rows, dtype=np.float64)  # [checkpoint][field][4]
        out["cr_vs_ref_maxrel"] = rows[:, :, 0]
        out["cr_vs_ref_n1e12"] = rows[:, :, 1].astype(np.int64)
        out["cr_vs_ref_n1e8"] = rows[:, :, 2].astype(np.int64)
        out["cr_vs_ref_ndiff"] = rows[:, :, 3].astype(np.int64)
    np.savez_compressed(os.path.join(HERE, "fullrun_%s.npz" % case), **out)


def load(case):
    """The fixture as a dict, plus the setup rebuilt from workloads."""
    z = dict(np.load(os.path.join(HERE, "fullrun_%s.npz" % case)))
    return CASES[case][0](), z


if __name__ == "__main__":
    cmd = sys.argv[1] if len(sys.argv) > 1 else ""
    if cmd == "run":
        run_arm(sys.argv[2], sys.argv[3], sys.argv[4])
    elif cmd == "merge":
        merge(sys.argv[2], sys.argv[3])
    elif cmd == "all":
        scratch = sys.argv[2]
        os.makedirs(scratch, exist_ok=True)
        procs = []
        for case, (_, _, _, arms) in CASES.items():
            for arm in arms:
                log = open(os.path.join(scratch, "%s_%s.log" % (case, arm)), "w")
                procs.append(subprocess.Popen([sys.executable, __file__, "run", case, arm, scratch],
                                              stdout=log, stderr=subprocess.STDOUT))
        rc = [p.wait() for p in procs]
        if any(rc):
            sys.exit("an arm failed: %s" % rc)
        for case in CASES:
            merge(case, scratch)
            print("wrote fullrun_%s.npz" % case)
    else:
        sys.exit(__doc__)
