"""Benchmark: cell-updates/s of the hydro step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (one "step" = one Hydro::performStep over the whole grid): the 3D
viscous single event, 101x101x51 cells (x, y in [-15, 15] fm, eta_s in
[-7.5, 7.5]), tau0 = 0.5 fm/c, dtau = 0.05 fm/c, eta/s = 0.08, zeta/s = 0,
2000-point c_s^2(e) EoS table, seeded Monte-Carlo Glauber Pb+Pb event at
b = 7 fm (synthetic: the reference ships no input data), with the Cornelius
freeze-out surface at e_f = 0.5 GeV/fm^3 after every second step.  The timed
K steps are the first K steps of the event (warm-up runs on a throw-away
copy) and include those surface calls.

Multi-GPU (torchrun, N ranks): events are independent, so every rank runs
its own event (seed + rank) with no collective on the data path; the time is
the max over ranks (weak scaling).  The per-GPU legs below (batched_mlp,
batched_mlp_large, batch_2d, learned_guess, ic_build) run at N = 1 only.

The JSON line carries, besides the contract keys:
  roofline      the dominant kernel's algorithmic bytes per launch over its
                CUDA-event time, against the measured HBM copy bandwidth;
  step_roofline the whole step against the compulsory 288 B per
                cell-update (Q, pi, Pi read and written once);
  e2e           the same metric through the C ABI with host-resident state:
                every step uploads the state from pinned host memory, steps,
                and reads the updated state back (vh_step_host);
  cpu_baseline  the reference's own C++ step (compiled from its sources,
                single-threaded) timed on this host over a bounded sample;
  fp64_roofline the dominant kernel's and the step's FP64 operations (ncu
                counts, profiles/fp64.json) over their CUDA-event time,
                against a cuBLAS DGEMM measured in the same run;
  batched_mlp   the metric's numerator and denominator on the 256-event
                set: batched + table slope + learned start point against
                every event alone, at the tight tolerance, with errors and
                their noise floor;
  batched_mlp_large  the same on 8 large events (201x201x101);
  batch_2d      64 2+1D events batched (the tuner's form, the stage-batched
                form and a branch per event) against each alone;
  learned_guess the con2prim modes on one event with baryon charge;
  ic_build      the reference's IcGlissando initial state (10 seeded
                GLISSANDO events, setup RHIC62) built on the device
                (vh_init_glissando) on the benchmark grid, beside the
                reference's own module on one host thread (the reference
                time also sits in cpu_baseline.ic_build_reference_s).
`--ic-only` times the ic_build leg alone (for profiler captures).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from vhlle_b200.sharding import Ranks, dist_env  # noqa: E402

METRIC = "cell-updates/s per B200: batched+MLP-guess vs plain GPU at ≤1e-8 rel err"
UNIT = "cell-updates/s"
WORKLOAD = ("3D viscous single event %s (x,y in [-15,15] fm, eta_s in [-7.5,7.5]), "
            "tau0=0.5, dtau=0.05, eta/s=0.08, zeta/s=0, c_s^2(e) 2000-point EoS table, "
            "seeded MC-Glauber Pb+Pb b=7 fm, peak e=50 GeV/fm^3, Cornelius surface at "
            "e_f=0.5 GeV/fm^3 every 2 steps")
SURF_EVERY = 2
EVENT_SEED = 20260001  # the Glauber event of the timed run (rank r: EVENT_SEED + r)
COMPULSORY_B = 288  # bytes per cell-update: Q[7] + pi[10] + Pi, read + write

# Algorithmic bytes of each kernel: the fields a launch must read and write
# once (stencil neighbours come from cache), per grid cell, or for the
# relaxation and the advection per cell on the packed list of cells with
# matter (nactive, read from the device every step).
KERNEL_BYTES = {
    "k_update_m": 48,       # m[3] in, m[3] out
    "k_face_x": 120,        # Q or Qh [7] + m in, face flux [7] out
    "k_face_y": 120,
    "k_face_z": 120,
    "k_update": 336,        # 3 face fluxes [21] + Q/Qh [7] in, 2 x [7] out
    "k_ghost": 0,           # boundary planes only
    "k_visc_prims": 152,    # Qh [7] in, prims [8] + [4] out
    "k_visc_update": 288,   # prims [4], piH [10], PiH, m [3], flux [4], Q [7] in; Q [7] out
}
RELAX_ACTIVE_B = 528  # per listed cell: Q, Qprev [14], m [3], prims [12], pi, Pi [11] in;
                      # pi0, piH0, Pi0, PiH0 [22], flux [4] out
RELAX_VACUUM_B = 208  # per empty cell, by the list kernel: pi0, piH0, Pi0, PiH0, flux [26] out
RELAX_LIST_B = 12     # per cell: e of the half-step prims in, per listed cell its index out
ADVECT_ACTIVE_B = 496  # per listed cell: prims [5], pi0, piH0, Pi0, PiH0 [22], flux [4] in;
                       # pi, piH, Pi, PiH, vcc [23], flux [4] out
KERNEL_BYTES_RULE = {
    "k_is_relax": "%d B x listed cells + %d B x empty cells + %d B x cells (k_relax_list + k_is_relax)"
                  % (RELAX_ACTIVE_B, RELAX_VACUUM_B, RELAX_LIST_B),
    "k_is_advect": "%d B x listed cells" % ADVECT_ACTIVE_B,
}
for _k, _b in KERNEL_BYTES.items():
    KERNEL_BYTES_RULE[_k] = "%d B x cells" % _b


def kernel_alg_bytes(prof, cells, nactive):
    """Algorithmic bytes of every profiled kernel summed over its launches;
    nactive is the listed-cell count summed over the profiled steps."""
    out = {}
    for k, (n, _) in prof.items():
        if k in KERNEL_BYTES:
            out[k] = float(KERNEL_BYTES[k]) * cells * n
    if "k_is_relax" in prof:
        n = prof["k_is_relax"][0]
        out["k_is_relax"] = (RELAX_ACTIVE_B * nactive + RELAX_VACUUM_B * (n * cells - nactive)
                             + RELAX_LIST_B * n * cells)
    if "k_is_advect" in prof:
        out["k_is_advect"] = float(ADVECT_ACTIVE_B) * nactive
    return out


# the persistent per-cell state a step reads or leaves for the next one (the
# empty cells keep their piH, PiH and viscCorrCut, which the viscous fluxes
# and the surface read)
STATE_IO = ("Q", "pi", "piH", "Pi", "PiH", "m", "viscCorrCut")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def fp64_peak_tflops(device, n=8192, reps=6):
    """FP64 throughput of a cuBLAS DGEMM (n x n x n, through torch) on this
    GPU, measured now: the denominator of the FP64 co-roofline (the B200's
    FP64 rate is the same on its tensor and CUDA-core paths)."""
    import torch
    dev = "cuda:%d" % device
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    c = torch.mm(a, b)
    torch.cuda.synchronize(dev)
    s = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(reps):
        torch.mm(a, b, out=c)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (ms / 1e3) / 1e12


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.p = None
        # the raw samples go to $VH_CLOCKS_DIR (default: a temporary
        # directory); the JSON line carries their summary
        d = os.environ.get("VH_CLOCKS_DIR") or tempfile.mkdtemp(prefix="vh_clocks_")
        self.out = os.path.join(d, "clocks_rank%s.csv" % os.environ.get("RANK", "0"))
        try:
            os.makedirs(os.path.dirname(self.out), exist_ok=True)
            self.f = open(self.out, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.out):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def gpu_index_for(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return ids[local_rank]
    return str(local_rank)


# kernels whose work is the listed cells with matter (k_relax_list's list)
ACTIVE_KERNELS = ("k_is_relax", "k_is_advect")


def ncu_per_launch(fname, field, kernel, grid, launches, warmup, active_per_step):
    """A per-launch ncu figure of `kernel` from a committed summary of the
    same workload's timed steps (profiles/<fname>: per grid, per kernel,
    each launch's value in step order; "_capture" holds the capture's
    warm-up and step counts and its listed cells per step).  Returns
    (value, basis): the mean over this run's launches when the run starts
    where the capture did and the capture covers them; otherwise the
    capture's mean, per listed cell for the kernels that work on the list
    (times this run's listed cells per step) and per launch for the others;
    (None, None) without a capture of the grid."""
    p = os.path.join(ROOT, "profiles", fname)
    if not os.path.exists(p):
        return None, None
    d = json.load(open(p))
    key = "x".join(map(str, grid))
    v = d.get(key, {}).get(kernel)
    cap = d.get("_capture", {}).get(key)
    if not v or not v[field] or not cap:
        return None, None
    vals = v[field]
    if cap["warmup"] == warmup and len(vals) >= launches:
        return float(sum(vals[:launches]) / launches), "ncu, the same launches"
    m = float(sum(vals) / len(vals))
    what = "ncu of steps %d-%d" % (cap["warmup"] + 1, cap["warmup"] + cap["steps"])
    if kernel in ACTIVE_KERNELS:
        return m / cap["active_cells_per_step"] * active_per_step, what + ", per listed cell"
    return m, what + ", per launch"


def nvtx(name=None):
    """Marks the timed region for profiler captures (ncu --nvtx-include)."""
    try:
        import torch
        if name is None:
            torch.cuda.nvtx.range_pop()
        else:
            torch.cuda.nvtx.range_push(name)
    except Exception:
        pass


# the initial-state leg: IcGlissando (icModel 5) of IC_EVENTS seeded
# GLISSANDO events, collision setup IC_SETUP (baryon density on), on the
# benchmark grid
IC_EVENTS, IC_SEED, IC_SETUP = 10, 11, "RHIC62"


def ic_events(path):
    from vhlle_b200 import ic_files as F
    F.write_glissando(path, F.synthetic_glissando_events(IC_EVENTS, seed=IC_SEED))
    return F.read_glissando(path)


def ic_build_measure(capi, W, grid, device, reps=3):
    """vh_init_glissando on the device: the best of `reps` calls after one
    warm-up call, host wall clock around the call (it returns after its last
    copy), input file parsed beforehand."""
    import tempfile
    setup = W.glauber3d_setup(*grid, seed=EVENT_SEED)
    su = capi.ic_setup(capi.IC_GLISSANDO, IC_SETUP)
    with tempfile.TemporaryDirectory() as d:
        ev = ic_events(os.path.join(d, "sources.txt"))
    h = capi.GpuHydro(setup, device=device, upload=False)
    try:
        norms = h.init_glissando(ev, su)
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            h.init_glissando(ev, su)
            best = min(best, time.perf_counter() - t0)
    finally:
        h.close()
    return {"module": "IcGlissando (icModel 5)", "setup": IC_SETUP, "events": IC_EVENTS,
            "sources": int(len(ev.x)), "grid": "x".join(map(str, grid)), "device_s": best,
            "sNorm": norms[0], "nNorm": norms[1]}


def ic_reference_sample(grid):
    """The reference's IcGlissando constructor + setIC (oracle/_ref) on the
    same input, one thread; None where the reference is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    import tempfile
    from vhlle_b200 import workloads as W
    if not P.ref_available():
        return None
    setup = W.glauber3d_setup(*grid, seed=EVENT_SEED)
    run = P.RefRun(setup)
    try:
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "sources.txt")
            ic_events(path)
            t0 = time.perf_counter()
            run.ic(5, path, IC_SETUP)
            return time.perf_counter() - t0
    finally:
        run.close()


def cpu_baseline_sample(setup, steps=2):
    """The reference C++ step (oracle/_ref, single-threaded) on the same
    event; falls back to the C restatement if the reference is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as P
    import tempfile
    kind = "reference" if P.ref_available() else "port"
    run = P.RefRun(setup) if kind == "reference" else P.OracleRun(setup)
    run.step(1)  # warm-up step, as the reference timing plan asks
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        for k in range(1, steps + 1):
            run.step(1)
            if k % SURF_EVERY == 0:
                run.output_surface(d) if kind == "reference" else run.surface()
        dt = time.perf_counter() - t0
    if kind == "reference":
        run.close()
    cells = setup.grid.ncells
    return {"value": cells * steps / dt, "unit": UNIT, "cores": 1, "kind": kind,
            "cpu_model": cpu_model(),
            "sample": "%d performStep calls of the %dx%dx%d event with the freeze-out "
                      "surface after every %d, after 1 warm-up step, one thread, %.1f s"
                      % (steps, setup.grid.nx, setup.grid.ny, setup.grid.nz, SURF_EVERY, dt)}


def _ref_worker(args):
    seed, steps, budget, grid = args
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from vhlle_b200 import workloads as W
    import pyoracle as P
    import tempfile
    setup = W.glauber3d_setup(*grid, seed=seed)
    ref = P.ref_available()
    run = P.RefRun(setup) if ref else P.OracleRun(setup)
    done = 0
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        while done < steps:
            run.step(1)
            done += 1
            if done % SURF_EVERY == 0:
                run.output_surface(d) if ref else run.surface()
            if time.perf_counter() - t0 > budget:
                break
        dt = time.perf_counter() - t0
    return done * setup.grid.ncells, dt, ref


def run_reference_arm(args):
    """--impl reference: the reference's CPU step on all host cores, one
    independent copy of the event per process, time-boxed."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import multiprocessing as mp
    ncores = os.cpu_count() or 1
    nproc = max(1, min(ncores, 32))
    budget = float(os.environ.get("VH_REF_BUDGET_S", "60"))
    steps = max(1, args.steps)
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    # every process steps its own copy of the event the GPU arm times
    with ctx.Pool(nproc) as pool:
        res = pool.map(_ref_worker, [(EVENT_SEED, steps, budget, args.grid)] * nproc)
    wall = time.perf_counter() - t0
    total = sum(r[0] for r in res)
    slowest = max(r[1] for r in res)
    kind = "reference" if all(r[2] for r in res) else "port"
    value = total / slowest
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": WORKLOAD % ("x".join(map(str, args.grid))),
                   "path": "reference C++ Hydro::performStep + Fluid::outputSurface every %d steps"
                           % SURF_EVERY},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": kind,
                         "cpu_model": cpu_model(),
                         "sample": "%d processes, each stepping its own copy of the event (seed %d, "
                                   "surface every %d steps) for up to %d steps or %.0f s; %.1f s wall"
                                   % (nproc, EVENT_SEED, SURF_EVERY, steps, budget, wall)},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def _reset(h, setup):
    h.upload_initial()
    h.L.vh_set_tau(h.h, setup.tau0)
    h.set_dtau(setup.dt)


def batch_measure(capi, W, n_events, steps, device, nz=None):
    """Event-by-event batch (the 256-event configuration's generator, its
    first n_events): every event stepped alone through vh_advance, one after
    another on the default stream, against the same events advanced by one
    vh_batch graph per iteration after the online tuning.  Device time with
    CUDA events; the same states are reset between the two runs."""
    evs = W.batch_events(n_events, nz=nz)
    cells = sum(s.grid.ncells for s in evs)
    hs = [capi.GpuHydro(s, device=device) for s in evs]
    drv = [(s.dt, s.grid.etamin, s.grid.etamax, s.grid.nz) for s in evs]
    for h, d in zip(hs, drv):  # warm-up
        h.advance(*d)
    for h, s in zip(hs, evs):
        _reset(h, s)
    for h in hs:
        h.sync()
    hs[0].timer_start()
    for _ in range(steps):
        for h, d in zip(hs, drv):
            h.advance(*d)
    plain_ms = hs[0].timer_stop()
    for h in hs:
        h.sync()
    b = capi.Batch(hs)
    for k, d in enumerate(drv):
        b.set_driver(k, *d, 4.0)
    b.tune(True)
    b.advance(18)  # 9 configurations x 2 timed iterations, then the chosen one
    b.sync()
    tuned = b.info()

    def timed():
        for h, s in zip(hs, evs):
            _reset(h, s)
        for h in hs:
            h.sync()
        b.advance(2)  # graphs of the reset parity
        b.sync()
        for h, s in zip(hs, evs):
            _reset(h, s)
        for h in hs:
            h.sync()
        b.timer_start()
        b.advance(steps)
        ms = b.timer_stop()
        return ms, b.sync()

    tuned_ms, bits = timed()
    # each form on its own: stage-batched, and a branch per event (8 streams
    # when the tuner chose the stage-batched form)
    b.set_mode(True)
    stage_ms, bits_s = timed()
    b.set_mode(False)
    graph_ms, bits_g = timed()
    info = b.info()
    b.close()
    for h in hs:
        h.close()
    return {"events": n_events, "steps": steps, "cells": cells,
            "grids": "%d..%d cells (%s)" % (
                min(s.grid.ncells for s in evs), max(s.grid.ncells for s in evs),
                "61x61x1 .. 121x121x61 family" if nz is None else "nz = %d" % nz),
            "plain_per_event": cells * steps / (plain_ms / 1e3),
            "batched_tuned": cells * steps / (tuned_ms / 1e3),
            "batched_stage": cells * steps / (stage_ms / 1e3),
            "batched_graph": cells * steps / (graph_ms / 1e3),
            "speedup": plain_ms / tuned_ms, "speedup_stage": plain_ms / stage_ms,
            "speedup_graph": plain_ms / graph_ms, "unit": UNIT,
            "error_bits": bits | bits_s | bits_g,
            "tuned": {"form": "stage-batched" if tuned["nstreams"] == 0 else "branch per event",
                      "nstreams": tuned["nstreams"], "block": tuned["block"],
                      "captures": info["captures"]},
            "graph": {"nstreams": info["nstreams"], "block": info["block"]},
            "physics": "eta/s=0.12, zeta/s Gaussian bump 0.05 at T=0.175 GeV (width 0.02)"}


TIGHT = 1e-13  # con2prim stop at which the root does not depend on the path to it


def train_guess_network(capi, W, device, target=10_000_000):
    """The start-point network trained on about `target` (features, label)
    pairs that transformPV at the tight tolerance gives on the cells of
    runs of the 3D event, the event with baryon charge and eight events of
    the event-by-event set (every cell with matter, every 5th step)."""
    import torch
    t0 = time.perf_counter()
    sources = [W.glauber3d_setup(seed=EVENT_SEED), W.glauber3d_nb_setup(seed=EVENT_SEED)]
    sources += W.batch_events(8)
    per = target // len(sources)
    dev = "cuda:%d" % device
    X = torch.empty((target, 4), dtype=torch.float32, device=dev)
    Y = torch.empty((target, 3), dtype=torch.float32, device=dev)
    n = 0
    for s in sources:
        h = capi.GpuHydro(s, device=device)
        got = 0
        for _ in range(60):
            room = min(per - got, target - n)
            if room <= 0:
                break
            h.step(5)
            k = h.mlp_samples(X[n:n + room], Y[n:n + room])
            got += k
            n += k
        h.close()
    X, Y = X[:n].contiguous(), Y[:n].contiguous()
    m = capi.Mlp(device=device, seed=17)
    epochs = 6
    losses = m.train(X, Y, batch=16384, epochs=epochs, lr=3e-3, seed=5)
    torch.cuda.synchronize()
    info = {"samples": n, "epochs": epochs, "first_loss": float(losses[0]),
            "final_loss": float(losses[-1]), "seconds": time.perf_counter() - t0,
            "sources": "101x101x51 event, the same with nb, 8 events of the event-by-event set"}
    del X, Y
    torch.cuda.empty_cache()
    return m, info


def _c2p_mode(h, mode, mlp):
    """mode: 'reference' (tol 1e-5, constant slope), 'tight' (1e-13,
    constant slope), 'tight_mlp' (1e-13, constant slope, learned start),
    'tight_slope' (1e-13, the EoS's slope), 'tight_slope_mlp'."""
    h.set_con2prim_guess(None)
    h.set_con2prim_method(0)
    h.set_con2prim(1e-5 if mode == "reference" else (1e-14 if mode == "tight14" else TIGHT))
    if "slope" in mode:
        h.set_con2prim_method(1)
    if "mlp" in mode:
        h.set_con2prim_guess(mlp)


LG_MODES = ("reference", "tight", "tight_mlp", "tight_slope", "tight_slope_mlp")


def learned_guess_measure(capi, W, setup, steps, device, mlp):
    """The learned con2prim start point on one event: root-find iterations
    and device throughput for each con2prim mode (LG_MODES); what the trained
    network gains is tight_slope_mlp over tight_slope (same method) and over
    tight (the reference's method at the same tolerance)."""
    cells = setup.grid.ncells
    h = capi.GpuHydro(setup, device=device)
    out = {"tolerance": TIGHT}
    iters = {}
    for mode in LG_MODES:
        _c2p_mode(h, mode, mlp)
        _reset(h, setup)
        h.step(3)  # captures this mode's step graph
        h.sync()
        _reset(h, setup)
        h.timer_start()
        h.step(steps)
        ms = h.timer_stop()
        out[mode] = cells * steps / (ms / 1e3)
        _reset(h, setup)
        h.con2prim_stats(True)
        h.step(steps)
        c, it = h.con2prim_stats(False)
        iters[mode] = it / c
    _c2p_mode(h, "reference", None)
    out["iters_per_root_find"] = iters
    # the network with the reference's Newton, the table slope alone, both
    # together against the tight path, and what the network adds to the slope
    out["speedup_mlp_vs_tight"] = out["tight_mlp"] / out["tight"]
    out["speedup_slope_vs_tight"] = out["tight_slope"] / out["tight"]
    out["speedup_slope_mlp_vs_tight"] = out["tight_slope_mlp"] / out["tight"]
    out["speedup_mlp_vs_tight_slope"] = out["tight_slope_mlp"] / out["tight_slope"]
    out["unit"] = UNIT
    out["steps"] = steps
    out["workload"] = "%s %dx%dx%d" % (setup.name, setup.grid.nx, setup.grid.ny, setup.grid.nz)
    h.close()
    return out


def state_error(a, b, fields=("Q", "pi", "Pi")):
    """Per field: the largest relative difference and the fraction of
    values beyond 1e-8 relative (each difference less 1e-12 of the field's
    largest magnitude, for values near zero), and the relative 2-norm of the
    difference."""
    out = {}
    for k in fields:
        x, y = np.asarray(a[k]).reshape(-1), np.asarray(b[k]).reshape(-1)
        scale = float(np.abs(y).max()) if y.size else 0.0
        d = np.abs(x - y) - 1e-12 * scale
        r = np.where(d > 0, d / np.maximum(np.maximum(np.abs(x), np.abs(y)), 1e-300), 0.0)
        ny = float(np.linalg.norm(y))
        out[k] = {"max_rel": float(r.max()) if r.size else 0.0,
                  "frac_beyond_1e-8": float((r > 1e-8).mean()) if r.size else 0.0,
                  "norm_rel": float(np.linalg.norm(x - y)) / ny if ny > 0 else 0.0}
    return out


BUMP = "eta/s=0.12, zeta/s Gaussian bump 0.05 at T=0.175 GeV (width 0.02)"
LARGE = ("201x201x101 on [-20,20]^2 x [-10,10], tau0=0.4, dtau=0.02, eta/s=0.08 + the zeta/s "
         "bump, shear + bulk + cross terms, nb on the (e, nb) table")


def batched_mlp_measure(capi, W, evs, steps, device, mlp, tau_resize=4.0, nsample=8,
                        physics=BUMP):
    """The benchmark metric's numerator and denominator on a set of events
    `evs` (the event-by-event set's first seeded events: 61x61x1 ..
    121x121x61, eta/s = 0.12, the zeta/s bump, the one-shot x2 resize at
    tau_resize; or the large events): every event of the set stepped alone (one vh_advance per
    driver-loop iteration, event after event) at the reference tolerance and
    at the tight one, against the same events advanced together by one
    vh_batch graph per iteration at the tight tolerance, without and with
    the learned start point (with the EoS's own Newton slope).  Device time
    with CUDA events over `steps` iterations; every arm starts from fresh
    contexts with the initial states (a resize changes a context's grid).
    errors: the batched + learned path against the plain tight path
    (bit-identical to the tight oracle, tests/test_gpu_con2prim_tight.py)
    over nsample events (the smallest and the largest)."""
    n_events = len(evs)
    cells = sum(s.grid.ncells for s in evs)
    drv = [(s.dt, s.grid.etamin, s.grid.etamax, s.grid.nz) for s in evs]
    by_size = sorted(range(n_events), key=lambda k: evs[k].grid.ncells)
    sample = sorted(set(by_size[:nsample // 2] + by_size[-(nsample - nsample // 2):]))

    def fresh(mode):
        hs = [capi.GpuHydro(s, device=device) for s in evs]
        for h in hs:
            _c2p_mode(h, mode, mlp)
        return hs

    def plain(mode):
        hs = fresh(mode)
        for h, d in zip(hs, drv):  # captures each event's step graph for this mode
            h.advance(*d)
        for h, s in zip(hs, evs):
            _reset(h, s)
        for h in hs:
            h.sync()
        resized = [False] * n_events
        hs[0].timer_start()
        for _ in range(steps):
            for k, (h, d) in enumerate(zip(hs, drv)):
                h.advance(*d)
                if not resized[k] and h.tau >= tau_resize:  # src/main.cpp:423-427
                    h.resize2x()
                    resized[k] = True
        ms = hs[0].timer_stop()
        for h in hs:
            h.sync()
        return ms, hs

    def batched(mode):
        hs = fresh(mode)
        b = capi.Batch(hs)
        for k, d in enumerate(drv):
            b.set_driver(k, *d, tau_resize)
        b.tune(True)
        b.advance(18)  # the tuner's 9 configurations x 2 (18 iterations stay below tau_resize)
        b.sync()
        for h, s in zip(hs, evs):
            _reset(h, s)
        for h in hs:
            h.sync()
        b.advance(2)  # the graphs of the reset state's buffer parity
        b.sync()
        for h, s in zip(hs, evs):
            _reset(h, s)
        for h in hs:
            h.sync()
        b.timer_start()
        b.advance(steps)
        ms = b.timer_stop()
        bits = b.sync()
        info = b.info()
        b.close()
        return ms, hs, bits, info

    out = {"events": n_events, "steps": steps, "cells": cells, "unit": UNIT,
           "grids": "%d..%d cells" % (min(s.grid.ncells for s in evs), max(s.grid.ncells for s in evs)),
           "tau_resize": tau_resize, "tolerance": TIGHT, "physics": physics}
    ms = {}
    ms["plain_reference_tol"], hs = plain("reference")
    for h in hs:
        h.close()
    ms["plain_tight"], hs = plain("tight")
    ref_states = {k: hs[k].get_state(("Q", "pi", "Pi")) for k in sample}
    for h in hs:
        h.close()
    # the noise floor: the same sample events stepped alone with the stop
    # tightened to 1e-14 (the reference's method and start point).  Any
    # change of the root find's path (start point, slope, stop) moves each
    # root by ~1e-14 and the limiter and vacuum-edge branches amplify that
    # to O(1) in some cells within ~10-20 steps, the oracle included.
    floor = {}
    for k in sample:
        h = capi.GpuHydro(evs[k], device=device)
        _c2p_mode(h, "tight14", mlp)
        resized = False
        for _ in range(steps):
            h.advance(*drv[k])
            if not resized and h.tau >= tau_resize:
                h.resize2x()
                resized = True
        floor[k] = state_error(h.get_state(("Q", "pi", "Pi")), ref_states[k])
        h.close()
    out["errors_floor_tight_1e-14"] = {
        f: {"max_rel": max(e[f]["max_rel"] for e in floor.values()),
            "frac_beyond_1e-8": max(e[f]["frac_beyond_1e-8"] for e in floor.values()),
            "norm_rel": max(e[f]["norm_rel"] for e in floor.values())} for f in ("Q", "pi", "Pi")}
    for mode in ("tight", "tight_slope_mlp"):
        ms["batched_" + mode], hs, bits, info = batched(mode)
        out["error_bits_" + mode] = bits
        out["tuned_" + mode] = {"form": "stage-batched" if info["nstreams"] == 0 else
                                "branch per event", "nstreams": info["nstreams"],
                                "block": info["block"]}
        errs = {k: state_error(hs[k].get_state(("Q", "pi", "Pi")), ref_states[k]) for k in sample}
        out["errors_" + mode] = {
            f: {"max_rel": max(e[f]["max_rel"] for e in errs.values()),
                "frac_beyond_1e-8": max(e[f]["frac_beyond_1e-8"] for e in errs.values()),
                "norm_rel": max(e[f]["norm_rel"] for e in errs.values())} for f in ("Q", "pi", "Pi")}
        for h in hs:
            h.close()
    for k, v in ms.items():
        out[k] = cells * steps / (v / 1e3)
    out["error_max"] = max(v["max_rel"] for v in out["errors_tight_slope_mlp"].values())
    out["speedup"] = ms["plain_tight"] / ms["batched_tight_slope_mlp"]
    out["speedup_vs_plain_reference_tol"] = ms["plain_reference_tol"] / ms["batched_tight_slope_mlp"]
    out["speedup_batching_alone"] = ms["plain_tight"] / ms["batched_tight"]
    out["error_sample"] = "%d events (the smallest and the largest)" % len(sample)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--batch-events", type=int, default=256,
                    help="events of the batched + learned-guess measurement (0: skip)")
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--large-steps", type=int, default=10,
                    help="steps of the 8 large events' batched leg")
    ap.add_argument("--no-learned-guess", action="store_true")
    ap.add_argument("--vorticity", action="store_true",
                    help="the event with Hydro::enableVorticity (dbeta every step, beta.dat "
                         "values at every surface)")
    ap.add_argument("--no-ic", action="store_true",
                    help="skip the initial-state leg (IcGlissando on the device)")
    ap.add_argument("--ic-only", action="store_true",
                    help="time the initial-state leg alone and print it (profiler captures)")
    ap.add_argument("--grid", default="101,101,51",
                    help="nx,ny,nz of the event (smaller grids only for profiler captures)")
    args = ap.parse_args()
    args.grid = tuple(int(v) for v in args.grid.split(","))
    if args.impl == "reference":
        return run_reference_arm(args)

    from vhlle_b200 import capi
    from vhlle_b200 import workloads as W

    if args.ic_only:
        print(json.dumps({"ic_build": ic_build_measure(capi, W, args.grid, 0)}), flush=True)
        return 0

    ws, rank, local = dist_env()
    dist = Ranks(ws)
    nx, ny, nz = args.grid
    setup = W.glauber3d_setup(nx, ny, nz, seed=EVENT_SEED + rank)
    cells = setup.grid.ncells
    h = capi.GpuHydro(setup, device=local)
    if args.vorticity:
        h.enable_vorticity()
    lps = h.launches_per_step()

    # warm-up on the event itself (steps and pipelined surface calls, so
    # that the surface buffers and the step graphs exist before the timed
    # loop), then restart the event for the timed run
    for k in range(1, max(args.warmup, SURF_EVERY) + 1):
        h.step(1)
        if k % SURF_EVERY == 0:
            h.surface_begin()
            h.surface_end()
    h.sync()
    h.upload_initial()
    h.L.vh_set_tau(h.h, setup.tau0)

    sampler = ClockSampler(gpu_index_for(local))
    time.sleep(0.3)
    dist.barrier()
    nvtx("timed")
    h.timer_start()
    nel = 0
    pending = False
    for k in range(1, args.steps + 1):
        h.step(1)  # one captured graph per step (vh_step)
        # the surface call begun after the previous step is collected once
        # this step is queued behind it, so the GPU never waits for the host
        if pending:
            nel += h.surface_end()["nelements"]
            pending = False
        if k % SURF_EVERY == 0:
            h.surface_begin()
            pending = True
    if pending:
        nel += h.surface_end()["nelements"]
    ms = h.timer_stop()
    nvtx()
    dist.barrier()
    clocks = sampler.stop()
    h.sync()
    # the kernels' and the surface calls' own times: the same loop again,
    # the step's kernels launched one by one with CUDA events between them
    # (vh_profile) and a CUDA-event pair around every surface call
    # (vh_surface waits for its result, so the pair spans the call's kernels
    # and its host round trip)
    h.upload_initial()
    h.L.vh_set_tau(h.h, setup.tau0)
    h.profile(True)
    surf_ms_tot = 0.0
    nactive = 0  # cells the relaxation and the advection ran on, summed over the steps
    for k in range(1, args.steps + 1):
        h.step(1)
        nactive += h.active_cells()
        if k % SURF_EVERY == 0:
            h.timer_start()
            h.surface_only()
            surf_ms_tot += h.timer_stop()
    h.sync()
    prof = h.profile_read()
    h.profile(False)
    ms_max = dist.max(ms)
    value = ws * cells * args.steps / (ms_max / 1e3)

    # per-kernel algorithmic bytes over the timed steps and the dominant
    # kernel's roofline
    peak, peak_kind = measured_peaks()
    alg_total = kernel_alg_bytes(prof, cells, nactive)
    dom = max(prof.items(), key=lambda kv: kv[1][1])
    dname, (dn, dms) = dom
    avg_s = dms / dn / 1e3
    alg = alg_total.get(dname, 0.0) / dn
    achieved = alg / avg_s / 1e9
    roofline = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": None,
                "alg_bytes_per_launch": alg, "avg_launch_ms": avg_s * 1e3,
                "active_cells_per_step": nactive / args.steps,
                "alg_bytes_rule": KERNEL_BYTES_RULE.get(dname, "")}
    # FP64 co-roofline: the dominant kernel's and the whole step's FP64
    # operations (ncu counts of the same launches) over their CUDA-event
    # time, against a cuBLAS DGEMM measured now
    act = nactive / args.steps
    roofline["traffic"], roofline["traffic_basis"] = ncu_per_launch(
        "traffic.json", "bytes_per_launch", dname, args.grid, dn, args.warmup, act)
    fp64_peak = fp64_peak_tflops(local)
    fl, fl_basis = ncu_per_launch("fp64.json", "flops_per_launch", dname, args.grid, dn,
                                  args.warmup, act)
    step_fl = 0.0
    for k, (n, _) in prof.items():
        f, _ = ncu_per_launch("fp64.json", "flops_per_launch", k, args.grid, n, args.warmup, act)
        step_fl = None if (f is None or step_fl is None) else step_fl + f * n
    kern_s = sum(t for _, t in prof.values()) / 1e3
    fp64_roofline = {
        "kernel": dname, "unit": "TFLOP/s", "peak": fp64_peak,
        "peak_source": "measured now: cuBLAS DGEMM 8192^3 (torch.mm, float64)",
        "achieved": None if fl is None else fl / avg_s / 1e12,
        "flops_per_launch": fl,
        "step_achieved": None if step_fl is None else step_fl / kern_s / 1e12,
        "step_flops_per_cell_update": None if step_fl is None else step_fl / (cells * args.steps),
        "source": "profiles/fp64.json (ncu sm__sass_thread_inst_executed_op_d{add,mul,fma}_pred_on "
                  "of the same workload's timed launches; flops = add + mul + 2 fma)",
        "basis": fl_basis}
    if fl is not None:
        fp64_roofline["frac"] = fp64_roofline["achieved"] / fp64_peak
    if step_fl is not None:
        fp64_roofline["step_frac"] = fp64_roofline["step_achieved"] / fp64_peak
    step_bw = COMPULSORY_B * cells * args.steps / (ms / 1e3) / 1e9
    step_roofline = {"bound": "hbm", "achieved": step_bw, "peak": peak, "unit": "GB/s",
                     "frac": step_bw / peak, "bytes_per_cell_update": COMPULSORY_B}
    kernels = {}
    for k, (n, t) in prof.items():
        kernels[k] = {"launches": n, "total_ms": t, "share": t / ms}
        if k in alg_total and t > 0:
            kernels[k]["alg_gbs"] = alg_total[k] / (t / 1e3) / 1e9
    nsurf = args.steps // SURF_EVERY
    kernels["surface (vh_surface, 9 kernels)"] = {"launches": nsurf, "total_ms": surf_ms_tot,
                                                   "share": surf_ms_tot / ms, "elements": nel}

    # end to end through the C ABI with host-resident state
    e2e = None
    if not args.no_e2e:
        nE = args.e2e_steps or min(args.steps, 50)
        L = h.L
        bufs = {}
        view = capi.VhStateView()
        nbytes = 0
        for k in STATE_IO:
            n = capi.STATE_NCOMP[k] * cells * 8
            p = ctypes.c_void_p()
            h._check(L.vh_alloc_pinned(n, ctypes.byref(p)))
            bufs[k] = (p, n)
            setattr(view, k, p.value)
            nbytes += n
        # one untimed host step captures its graph (per buffer set); then
        # the event restarts from its initial state in the host buffers
        h.upload_initial()
        L.vh_set_tau(h.h, setup.tau0)
        h._check(L.vh_download_async(h.h, ctypes.byref(view)))
        h.sync()
        for _ in range(2):  # both fill-fraction buffer orders
            h._check(L.vh_step_host(h.h, ctypes.byref(view), ctypes.byref(view)))
        h.sync()
        h.upload_initial()
        L.vh_set_tau(h.h, setup.tau0)
        h._check(L.vh_download_async(h.h, ctypes.byref(view)))
        h.sync()
        dist.barrier()
        rec_cap = 400000
        rec_p = ctypes.c_void_p()
        h._check(L.vh_alloc_pinned(rec_cap * capi.SURF_REC * 8, ctypes.byref(rec_p)))
        rec_ptr = ctypes.cast(rec_p, ctypes.POINTER(ctypes.c_double))
        rec_bytes = 0
        h.timer_start()
        for k in range(1, nE + 1):
            # the state up, one step, the state back (vh_step_host: one graph
            # whose copies overlap the kernels where the step's data flow allows)
            h._check(L.vh_step_host(h.h, ctypes.byref(view), ctypes.byref(view)))
            if k % SURF_EVERY == 0:
                n = h.surface_only()["nelements"]
                got = ctypes.c_long()
                h._check(L.vh_surface_records(h.h, rec_ptr, rec_cap, ctypes.byref(got)))
                rec_bytes += min(n, rec_cap) * capi.SURF_REC * 8
        ems = h.timer_stop()
        h.sync()
        ems = dist.max(ems)
        for p, _ in bufs.values():
            L.vh_free_pinned(p)
        L.vh_free_pinned(rec_p)
        link = (2 * nbytes + rec_bytes / nE) * nE / (ems / 1e3) / 1e9
        e2e = {"value": ws * cells * nE / (ems / 1e3), "unit": UNIT, "h2d_bytes_per_step": nbytes,
               "d2h_bytes_per_step": nbytes + rec_bytes // nE, "steps": nE,
               "host_link_gbs": link,
               "note": "state uploaded and downloaded every step (vh_step_host), surface "
                       "records every %d; "
                       "host_link_gbs: both directions' bytes over the whole time (the "
                       "viscous fields' upload beside the ideal stages, m, piH, PiH back "
                       "before the end)" % SURF_EVERY}

    batch2d = learned = bmlp = large = None
    mlp = None
    # the per-GPU legs run on one GPU only (the multi-GPU line reports the
    # sharded step, which the legs do not change)
    legs = ws == 1
    if legs and not args.no_learned_guess:
        mlp, mlp_info = train_guess_network(capi, W, local)
        learned = learned_guess_measure(capi, W, W.glauber3d_nb_setup(nx, ny, nz, seed=EVENT_SEED + rank),
                                        30, local, mlp)
        learned["train"] = mlp_info
    if legs and args.batch_events > 0:
        if mlp is not None:
            bmlp = batched_mlp_measure(capi, W, W.batch_events(args.batch_events),
                                       args.batch_steps, local, mlp)
            # the large events (8 of them, 4.1 M cells each: 33 GB resident)
            large = batched_mlp_measure(capi, W, [W.large_event_setup(k) for k in range(8)],
                                        args.large_steps, local, mlp, nsample=2, physics=LARGE)
        batch2d = batch_measure(capi, W, 64, 2 * args.batch_steps, local, nz=1)
    if mlp is not None:
        mlp.close()

    ic = None
    if legs and not args.no_ic:
        ic = ic_build_measure(capi, W, args.grid, local)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(W.glauber3d_setup(nx, ny, nz, seed=EVENT_SEED))
        if ic is not None:
            ref_s = ic_reference_sample(args.grid)
            cpu["ic_build_reference_s"] = ref_s
            if ref_s is not None:
                ic["reference_s"] = ref_s
                ic["speedup"] = ref_s / ic["device_s"]

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD % ("x".join(map(str, args.grid))), "cells": cells,
                       "path": "plain FP64 step + device freeze-out surface every %d steps "
                               "(no MLP guess, single event per GPU)" % SURF_EVERY,
                       "parallelism": "events%d" % ws,
                       "vorticity": bool(args.vorticity),
                       "l2": "inputs larger than L2 (%.0f MB of resident fields)" % (
                           cells * 8 * 127 / 1e6)},
            "roofline": roofline, "step_roofline": step_roofline, "fp64_roofline": fp64_roofline,
            "kernels": kernels,
            "e2e": e2e, "cpu_baseline": cpu, "batched_mlp": bmlp, "batch_2d": batch2d,
            "batched_mlp_large": large,
            "learned_guess": learned, "ic_build": ic,
            # the step graph's kernels, and per pipelined surface call its
            # nine kernels
            "gpu_launches": lps * args.steps + 9 * (args.steps // SURF_EVERY), "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    h.close()
    dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
