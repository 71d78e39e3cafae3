#!/usr/bin/env python
"""Benchmark of the SW2D single-porosity MUSCL-EVR/HLLC step on B200.

Workload: the large SP forward solve: a 4M-cell jittered triangle mesh over 2 km x 2 km, bed
= 50 seeded Gaussian bumps + 1e-3 slope, h = max(0, 2 - z_b) (wet/dry fronts), porosity a
seeded smooth field in [0.3, 1], Manning n lognormal (median 0.03, sigma 0.3), walls, FP64,
MUSCL-EVR + the reference's slope limiter + HLLC.  A "step" is one explicit time step over all
cells (the body of the reference's time loop).  Synthetic data, seeded.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

For N > 1 (launched with torchrun, one rank per GPU) every rank runs its own replica of the
workload (the step does not shard across GPUs in this build): value = all ranks' cell updates
/ max-over-ranks device time, scaling "weak".

The reference arm (--impl reference) times the reference's own native solver, compiled from
its sources (oracle/_ref), on the host cores: one independent replica per core on a bounded
sample of the same workload (same construction at 250k cells).
"""
from __future__ import annotations

import argparse
import importlib
import json
import multiprocessing as mp
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "inria-internship-project-sw2d-enzyme_b200"

METRIC = "MUSCL-HLLC cell-updates/s"
UNIT = "cell-updates/s"
ALGO_BYTES_PER_CELL_UPDATE = 188   # FP64 MUSCL step: state r/w 48 + cell statics 56 + edge statics 72 + CSR 12
CPU_SAMPLE_CELLS = 250_000


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cells", type=int, default=4_000_000)
    ap.add_argument("--mesh", choices=["delaunay", "grid"], default="delaunay",
                    help="seeded jittered-Delaunay mesh in a random numbering (the configuration's), or the "
                         "jittered grid split into triangles")
    ap.add_argument("--wet-steps", type=int, default=100,
                    help="timed steps of the moving (dam-break) variant of the workload (0: skip)")
    ap.add_argument("--e2e-chunk", type=int, default=50, help="time steps per state upload/download in e2e")
    ap.add_argument("--cpu-steps", type=int, default=150, help="timed steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--phase-steps", type=int, default=20)
    ap.add_argument("--adjoint-cells", type=int, default=1_000_000, help="cells of the adjoint workload")
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--adjoint-every", type=int, default=100, help="checkpoint interval of the adjoint")
    ap.add_argument("--adjoint-store-states", type=int, default=1,
                    help="1: the segment recompute keeps each step's slopes and Riemann states for the reverse")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--dip-cells", type=int, default=4_000_000, help="cells of the DIP forward line (0: skip)")
    ap.add_argument("--ensemble-members", type=int, default=256, help="members of the ensemble line (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=500)
    ap.add_argument("--ensemble-every", type=int, default=50, help="checkpoint interval of the ensemble adjoints")
    ap.add_argument("--dip-steps", type=int, default=200)
    ap.add_argument("--ddp-cells", type=int, default=4_000_000, help="cells of the DDP forward line (0: skip)")
    ap.add_argument("--ddp-steps", type=int, default=200)
    ap.add_argument("--ddp-cpu-cells", type=int, default=50_000, help="cells of the DDP reference sample")
    ap.add_argument("--ddp-cpu-steps", type=int, default=30)
    ap.add_argument("--ddp-only", action="store_true", help="run only the DDP forward line")
    ap.add_argument("--closure-cells", type=int, default=4_000_000,
                    help="cells of the DIP run that times the learned closure")
    ap.add_argument("--no-closure", action="store_true", help="skip the learned-closure line")
    ap.add_argument("--closure-only", action="store_true", help="run only the learned-closure line")
    ap.add_argument("--result-cells", type=int, default=500_000,
                    help="cells of the ResultHydro.bin line (0: skip)")
    ap.add_argument("--result-only", action="store_true", help="run only the ResultHydro.bin line")
    ap.add_argument("--closure-no-pipeline", action="store_true",
                    help="time the closure inside the step only (no data generation, training or judging)")
    ap.add_argument("--assim-cells", type=int, default=1_000_000,
                    help="cells of the porosity-assimilation line (the reference's differentiated step; 0: skip)")
    ap.add_argument("--assim-steps", type=int, default=2000, help="approximate steps of its trajectory")
    ap.add_argument("--assim-only", action="store_true",
                    help="print only the porosity-assimilation measurement (one JSON line)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="print only the adjoint measurement (one JSON line), e.g. for profiling")
    ap.add_argument("--flux-variant", type=int, default=None,
                    help="launch variant of the fused step's k_flux instead of autotuning (profiling runs)")
    ap.add_argument("--launch-config", default=None,
                    help="'S,E': slope and edge kernel launch variants instead of autotuning (profiling runs)")
    return ap.parse_args()


def _config(args, world):
    return {"workload": f"SP gaussian-bumps forward solve, {args.cells} cells (2 km x 2 km), MUSCL-EVR + HLLC, "
                        "Manning, FP64", "cells": args.cells, "scheme": "muscl_evr", "friction": "manning",
            "mesh": args.mesh,
            "global_cells": args.cells * world, "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "inputs larger than L2 (state + mesh tables ~0.9 GB per replica)"}


# ------------------------------------------------------------------------------------------
# reference solver on the host (CPU baseline and reference arm)
# ------------------------------------------------------------------------------------------
def _ref_worker(folder, warmup, steps, barrier, out):
    from oracle.binding import RefSolver
    ref = RefSolver(folder)
    ref.step(warmup)
    barrier.wait()
    t0 = time.perf_counter()
    done = ref.step(steps)
    t1 = time.perf_counter()
    out.put((done, t1 - t0, ref.n))


def reference_timing(n_procs: int, warmup: int, steps: int, cells: int = CPU_SAMPLE_CELLS):
    """Runs n_procs independent replicas of the reference on the sample (spawned processes)."""
    pkg = importlib.import_module(PKG)
    case = pkg.workloads.gaussian_bumps(n_cells=cells)
    tmp = tempfile.mkdtemp(prefix="sw2d_ref_")
    try:
        folders = []
        for i in range(n_procs):
            f = os.path.join(tmp, f"r{i}")
            if i == 0:
                pkg.write_case(f, case)
            else:
                shutil.copytree(os.path.join(tmp, "r0", "input"), os.path.join(f, "input"))
            folders.append(f)
        ctx = mp.get_context("spawn")
        barrier = ctx.Barrier(n_procs)
        out = ctx.Queue()
        procs = [ctx.Process(target=_ref_worker, args=(f, warmup, steps, barrier, out)) for f in folders]
        for p in procs:
            p.start()
        res = [out.get() for _ in procs]
        for p in procs:
            p.join()
        done = min(r[0] for r in res)
        wall = max(r[1] for r in res)
        n = res[0][2]
        return {"value": n_procs * n * done / wall, "cells": n, "steps": done, "seconds": wall}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def _cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    from oracle.binding import reference_available
    base = {"impl": "reference", "metric": METRIC, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": _config(args, world)}
    if not reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference solver library oracle/_ref not built"}))
        return
    cores = os.cpu_count() or 1
    r = reference_timing(cores, args.warmup, args.steps)
    sample = (f"same construction at {r['cells']} cells, {r['steps']} MUSCL steps per replica, "
              f"{cores} independent single-threaded replicas (one per host core; the reference is serial), {_cpu_model()}")
    base.update({"value": r["value"], "ms_per_step": 1e3 * r["seconds"] / max(r["steps"], 1),
                 "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": cores, "kind": "reference",
                                  "sample": sample},
                 "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    print(json.dumps(base))


# ------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.proc = None
        self.dev = device_index

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=self.fh, stderr=subprocess.DEVNULL)
            # nvidia-smi's own start-up (NVML initialisation) must not fall inside the timed
            # region: wait for its first sample (at most 10 s), then a little more
            t0 = time.time()
            while time.time() - t0 < 10.0 and self.proc.poll() is None:
                self.fh.flush()
                if os.path.getsize(self.path) > 0:
                    break
                time.sleep(0.05)
            time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.fh.close()

    def summary(self):
        if not self.proc or not os.path.exists(self.path):
            return None
        rows = []
        for ln in open(self.path):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------
def _measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_per_step():
    p = os.path.join(ROOT, "profiles", "sp_step_traffic_gaussian_bumps_1M.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except ValueError:
            return None
    return None


def run_wet(pkg, args, local_rank):
    """The same bed, mesh and parameters under a dam break (free surface 5.0 m for x < 1 km,
    3.5 m beyond, at rest): a moving flow over most of the domain, with wet/dry fronts, timed like
    the headline (graph-launched steps, CUDA events on the library's stream) after 20 steps of
    motion."""
    import numpy as np
    import torch

    case = pkg.workloads.gaussian_bumps(n_cells=args.cells, mesh=args.mesh, initial="dam")
    model = pkg.SpModel(case, device=local_rank)
    tune = pkg.tuning.autotune_step(model, iters=3, device=local_rank, cache_path=None)
    stream = torch.cuda.ExternalStream(model.stream, device=local_rank)
    model.step(20)
    phases = model.phase_times(5)
    model.prepare()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = model.step(args.wet_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    n = case.mesh.cell_nb
    h = model.state()[0]
    step_ms = ms / max(done, 1)
    peak, peak_kind = _measured_peak()
    achieved = ALGO_BYTES_PER_CELL_UPDATE * n / (step_ms / 1e3) / 1e9
    return {"workload": f"gaussian-bumps bed under a dam break, {n} cells, MUSCL-EVR + HLLC, Manning, FP64",
            "metric": METRIC, "value": n * done / (ms / 1e3), "unit": UNIT, "steps": done, "ms_per_step": step_ms,
            "wet_fraction_initial": float(np.mean(case.h0 > float(case.opts["h_min"]))),
            "wet_fraction_after": float(np.mean(h > float(case.opts["h_min"]))),
            "roofline_frac": achieved / peak, "peak_kind": peak_kind, "phases_ms": phases,
            "launch_config": tune["report"]}


def run_adjoint(pkg, args, local_rank):
    """The adjoint 4D-Var gradient: the dam-break construction at `--adjoint-cells` cells,
    MUSCL-EVR + HLLC, Manning n = 0.03; 32 gauges at seeded cells observed every 10 steps;
    observations from a twin replay with n (1 +- 0.2 smooth field); `--adjoint-steps` steps with
    checkpoints every `--adjoint-every`.  Times the recording (the CFL-driven dry run), the
    replayed cost (func) and the gradient (grad: one checkpointed reverse sweep), with CUDA
    events on the library's stream."""
    import numpy as np
    import torch

    case = pkg.workloads.dam_break(n_cells=args.adjoint_cells, scheme="muscl_evr", friction="manning")
    free0, total = torch.cuda.mem_get_info(local_rank)
    model = pkg.SpModel(case, device=local_rank)
    pkg.tuning.autotune(model, iters=3, device=local_rank, cache_path=None)
    model.set_option("adjoint_store_states", args.adjoint_store_states)
    stream = torch.cuda.ExternalStream(model.stream, device=local_rank)
    n = case.mesh.cell_nb

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    done, ms_record = timed(lambda: model.record(args.adjoint_steps, args.adjoint_every))
    if done != args.adjoint_steps:
        raise RuntimeError(f"adjoint trajectory: {done} of {args.adjoint_steps} steps")
    x, y = case.mesh.cell_x, case.mesh.cell_y
    smooth = np.sin(2 * np.pi * x / 100.0) * np.cos(2 * np.pi * y / 40.0)
    n_b = model.get_param("friction_1")
    rng = np.random.default_rng(5)
    gauges = np.sort(rng.choice(n, size=32, replace=False))
    steps = np.arange(10, args.adjoint_steps + 1, 10)
    model.set_param("friction", n_b * (1.0 + 0.2 * smooth))
    h_obs = model.replay_sample(gauges, steps)
    model.set_param("friction", n_b)
    model.set_observations(gauges, steps, h_obs)
    J, ms_replay = timed(model.replay_cost)
    grads = []
    for _ in range(2):
        (Jg, g), ms = timed(model.adjoint)
        grads.append(ms)
    if Jg != J or not all(np.all(np.isfinite(v)) for v in g.values()):
        raise RuntimeError("adjoint: inconsistent cost or non-finite gradient")
    free1, _ = torch.cuda.mem_get_info(local_rank)
    ms_grad = min(grads)
    kinds = 10  # kernels per reverse step: 4 recompute + k_update_rev, k_slopes, k_edges_rev, k_cells_rev, k_nbr_rev, copy
    return {
        "workload": f"dam break construction at {n} cells, MUSCL-EVR + HLLC, Manning n = 0.03; 32 gauges every 10 "
                    f"steps, twin with n (1 +- 0.2 smooth); {done} steps, checkpoints every {args.adjoint_every}",
        "metric": "adjoint gradients/s", "value": 1e3 / ms_grad, "unit": "gradients/s",
        "ms_per_gradient": ms_grad, "ms_record": ms_record, "ms_replay_cost": ms_replay,
        "ratio_gradient_to_replay": ms_grad / ms_replay,
        "cell_updates_per_s_replay": n * done / (ms_replay / 1e3),
        "J": J, "controls": ["friction_1", "friction_2", "h0", "q0", "r0", "z_b"],
        "device_memory_gb": (free0 - free1) / 1e9,
        "gpu_launches_per_gradient": done * kinds,
        "check": "gradient vs central differences and bitwise checkpoint invariance: tests/test_gpu_adjoint.py",
        "nonfinite_entries_set_to_zero": int(sum(model.adjoint_nonfinite().values())),
    }


def run_assim(pkg, args, local_rank):
    """Porosity assimilation with the reference's differentiated step (sw2d_assim_*): the gradient
    dJ/dphi of get_spatial_gradient_checkpointed.
    * sp_toce, the reference's own case (tests/golden/sp_toce_assim.npz: 4,800 cells, 3,157 steps,
      41 full-field observations, 48 tiles): the GPU's dry run, replayed cost and gradient, and the
      reference's own dry run and replayed cost on this host's CPU (its library built from its
      sources, oracle/_ref), which a gradient costs at least.  The reference's gradient itself
      needs Enzyme, absent here.
    * the dam-break construction at `--assim-cells` cells (MUSCL-EVR + HLLC, phi ~ U[0.6, 1]),
      32 gauges observed every 10 steps' worth of time, about `--assim-steps` steps, checkpoints
      every 100: dry run, replayed cost and gradient, CUDA events on the library's stream."""
    import numpy as np
    import torch

    from tests.conftest import GOLDEN, sp_toce_case
    from tests.golden.make_assim_golden import decimals_to_float

    def timed(model, fn):
        stream = torch.cuda.ExternalStream(model.stream, device=local_rank)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    out = {}
    # sp_toce
    case, _ = sp_toce_case()
    ax = np.load(os.path.join(GOLDEN, "sp_toce_assim.npz"))
    cfg = json.loads(str(ax["config"]))
    frames = decimals_to_float(ax["obs_mant"], ax["obs_exp"])
    model = pkg.SpModel(case, device=local_rank)
    model.assim_configure(phi_transform="none", windowed=True, window_duration=cfg["window_duration"],
                          n_windows=int(cfg["n_windows"]), t_state_assimilation=cfg["t_state_assimilation"],
                          cost_normalize=True)
    model.assim_set_frames(ax["obs_times"], frames)
    m = ax["m"]
    stride = int(cfg["checkpoint_stride"])
    (ns, nk), ms_rec = timed(model, lambda: model.assim_record(m, stride))
    J, ms_rep = timed(model, lambda: model.assim_replay_cost(m))
    ms_grads = []
    for _ in range(3):
        (g, info), ms = timed(model, lambda: model.assim_gradient(m, stride))
        ms_grads.append(ms)
    toce = {"cells": case.mesh.cell_nb, "steps": ns, "segments": nk, "tiles": info["n_tiles"],
            "ms_record": ms_rec, "ms_replay_cost": ms_rep, "ms_per_gradient": min(ms_grads), "J": J,
            "J_reference_same_libm": float(ax["J_pm"])}
    out["sp_toce"] = toce
    del model
    # dam-break construction at scale
    n_req = args.assim_cells
    case = pkg.workloads.dam_break(n_cells=n_req, scheme="muscl_evr", friction="none")
    n = case.mesh.cell_nb
    probe = pkg.SpModel(case, device=local_rank)
    probe.step(3)
    dt = probe.dt
    del probe
    t_end = args.assim_steps * dt
    case.opts["t_max"] = t_end
    free0, _ = torch.cuda.mem_get_info(local_rank)
    model = pkg.SpModel(case, device=local_rank)
    model.assim_configure(phi_transform="none", cost_normalize=True)
    rng = np.random.default_rng(5)
    gauges = np.sort(rng.choice(n, size=32, replace=False))
    times = np.arange(1, args.assim_steps // 10 + 1) * (10 * dt)
    model.assim_set_gauges(times, gauges, np.ones(32), case.h0[gauges][None, :] * np.ones((len(times), 1)))
    m = case.phi.copy()
    (ns, nk), ms_rec = timed(model, lambda: model.assim_record(m, 100))
    J, ms_rep = timed(model, lambda: model.assim_replay_cost(m))
    grads = []
    for _ in range(2):
        (g, info), ms = timed(model, lambda: model.assim_gradient(m, 100))
        grads.append(ms)
    free1, _ = torch.cuda.mem_get_info(local_rank)
    ms_grad = min(grads)
    ref_cpu = _assim_reference_sample(pkg, args)
    out.update({
        "workload": f"dam break construction at {n} cells, MUSCL-EVR + HLLC with the reference's differentiated "
                    f"step, phi ~ U[0.6, 1]; 32 gauges every 10 steps' time; {ns} steps, checkpoints every 100",
        "metric": "porosity gradients/s", "value": 1e3 / ms_grad, "unit": "gradients/s",
        "ms_per_gradient": ms_grad, "ms_record": ms_rec, "ms_replay_cost": ms_rep,
        "ratio_gradient_to_replay": ms_grad / ms_rep, "cell_updates_per_s_replay": n * ns / (ms_rep / 1e3),
        "J": J, "nonfinite_entries_set_to_zero": int(info["n_nonfinite"]),
        "device_memory_gb": (free0 - free1) / 1e9,
        "check": "record and replay bit for bit against the reference's own layer, gradient against its central "
                 "differences: tests/test_gpu_assim.py",
        "cpu_baseline": ref_cpu,
    })
    if "cell_updates_per_s_replay" in ref_cpu:
        out["speedup_replay_vs_reference_cpu"] = out["cell_updates_per_s_replay"] / ref_cpu["cell_updates_per_s_replay"]
    return out


def _assim_reference_sample(pkg, args):
    """The reference's own dry run and replayed cost (its assimilation layer built from its
    sources, oracle/_ref, one host core) on a bounded sample of the same construction: 100,000
    cells, 200 steps.  Its gradient needs Enzyme (a clang-18 plugin), absent here; a reverse
    sweep costs at least a replay."""
    import numpy as np
    try:
        from oracle.binding import RefE, REF_E_SO
    except Exception as exc:
        return {"unavailable": f"oracle binding: {exc}"}
    if not os.path.exists(REF_E_SO):
        return {"unavailable": "reference library not built (oracle/_ref)"}
    case = pkg.workloads.dam_break(n_cells=100_000, scheme="muscl_evr", friction="none")
    n = case.mesh.cell_nb
    probe = pkg.SpModel(case)
    probe.step(3)
    dt = probe.dt
    del probe
    steps = 200
    case.opts["t_max"] = steps * dt
    rng = np.random.default_rng(5)
    gauges = np.sort(rng.choice(n, size=32, replace=False))
    times = np.arange(1, steps // 10 + 1) * (10 * dt)
    with tempfile.TemporaryDirectory() as tmp:
        pkg.write_case(tmp, case)
        ref = RefE(tmp)
        ref.set_gauges(times, gauges, np.ones(32), case.h0[gauges][None, :] * np.ones((len(times), 1)))
        ref.set_options(True, 0, 1.0)
        t0 = time.perf_counter()
        K = ref.record(case.phi, 100)
        t1 = time.perf_counter()
        ref.set_window()
        ref.replay_cost(case.phi)
        t2 = time.perf_counter()
        ns = sum(len(sg[1]) for sg in ref.segments())
        ref.close()
    return {"kind": "reference", "cores": 1, "sample": f"dam break construction at {n} cells, {ns} steps",
            "ms_record": 1e3 * (t1 - t0), "ms_replay_cost": 1e3 * (t2 - t1), "segments": K,
            "cell_updates_per_s_replay": n * ns / (t2 - t1), "unit": "cell-updates/s",
            "gradient": "unavailable: the reference differentiates with Enzyme (clang-18 plugin), absent here"}


def run_dip(pkg, args, local_rank):
    """The dual integral porosity forward step on the DIP feature channel at `--dip-cells`
    cells (MUSCL-EVR, HLLC, Manning, momentum dissipation, q inflow, fr outflow), graph-launched
    steps timed with CUDA events on the library's stream."""
    import torch

    case = pkg.workloads.dip_channel(n_cells=args.dip_cells, t_max=1.0e9)
    model = pkg.SpModel(case, device=local_rank)
    tune = pkg.tuning.autotune_step(model, iters=3, device=local_rank, cache_path=None)
    stream = torch.cuda.ExternalStream(model.stream, device=local_rank)
    model.step(5)
    model.prepare()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = model.step(args.dip_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    n = case.mesh.cell_nb
    return {"workload": f"DIP feature channel at {n} cells, MUSCL-EVR + DIP HLLC, Manning, momentum dissipation, "
                        f"q inflow, fr outflow", "metric": "DIP cell-updates/s", "value": n * done / (ms / 1e3),
            "unit": "cell-updates/s", "steps": done, "ms_per_step": ms / done, "launch_config": tune["report"]}


def ddp_algo_bytes(nc: int, ni: int, nb: int, ntab: int) -> int:
    """Compulsory HBM traffic of one DDP step with this library's layout: every input read once,
    every output written once.  Cells: state {theta, theta u, theta v, z} read and written (64),
    the derived {phiW, thetaW, Omega force} read and written (64), statics cst and dcs (64), CSR
    offsets (12), area (8), table levels {z, phi} (16 per level; theta is rebuilt from them).
    Internal edges: L/R, normal, length, coefficients, slots, statics (2 records), table offset
    (132), table levels (16 per level).  Boundary edges: cell, geometry, series index, slot (44).
    Balance slots: {a, b, c} + CFL share written by the edge kernel and read by the CFL and
    update kernels (2 x 40 per slot; 2 slots per internal edge, 1 per boundary edge)."""
    cells = nc * (64 + 64 + 64 + 12 + 8 + 16 * ntab)
    edges = ni * (132 + 16 * ntab) + nb * 44
    slots = (2 * ni + nb) * 2 * 40
    return cells + edges + slots


def _ddp_reference_sample(pkg, args):
    """The reference's own swDdp (built from its sources) on a bounded sample of the same
    construction: `--ddp-cpu-cells` cells, `--ddp-cpu-steps` steps, one host core."""
    from oracle.binding import RefSolver, reference_available
    if not reference_available():
        return {"unavailable": "reference solver library oracle/_ref not built"}
    case = pkg.workloads.ddp_channel(n_cells=args.ddp_cpu_cells, laws="linear", friction="manning", outflow="fr",
                                     t_max=1.0e9, seed=61)
    tmp = tempfile.mkdtemp(prefix="sw2d_ddp_ref_")
    try:
        pkg.write_case(tmp, case)
        ref = RefSolver(tmp)
        ref.step(2)
        t0 = time.perf_counter()
        done = ref.step(args.ddp_cpu_steps)
        t1 = time.perf_counter()
        n = ref.n
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return {"kind": "reference", "cores": 1, "value": n * done / (t1 - t0), "unit": "cell-updates/s",
            "sample": f"the same construction at {n} cells, {done} steps of swDdp's loop body, {_cpu_model()}"}


def run_ddp(pkg, args, local_rank):
    """The depth-dependent porosity (DDP) forward step on the DDP feature channel at
    `--ddp-cells` cells: porosity laws of types 3 (linear with an open top level), 2 and 1 on 5
    levels per cell and per edge, Godunov + DDP HLLC (the only path of the reference's DDP
    step), Manning, q inflow, fr outflow; graph-launched steps timed with CUDA events on the
    library's stream, the phase shares from sw2d_phase_times."""
    import numpy as np
    import torch

    case = pkg.workloads.ddp_channel(n_cells=args.ddp_cells, laws="linear", friction="manning", outflow="fr",
                                     t_max=1.0e9, seed=61)
    model = pkg.SpModel(case, device=local_rank)
    tune = pkg.tuning.autotune(model, iters=3, device=local_rank, cache_path=None)
    stream = torch.cuda.ExternalStream(model.stream, device=local_rank)
    model.step(5)
    model.prepare()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = model.step(args.ddp_steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    phases = model.phase_times(10)
    th = model.state()[0]
    if not np.all(np.isfinite(th)):
        raise RuntimeError("non-finite DDP state")
    m = case.mesh
    n = m.cell_nb
    step_ms = ms / done
    algo = ddp_algo_bytes(n, m.edge_int_nb, m.edge_bnd_nb, 5)
    achieved = algo / (step_ms / 1e3) / 1e9
    peak, peak_kind = _measured_peak()
    tot = sum(phases.values())
    line = {"workload": f"DDP feature channel at {n} cells, porosity laws 3/2/1 on 5 levels, Godunov + DDP HLLC, "
                        f"Manning, q inflow, fr outflow", "metric": "DDP cell-updates/s", "value": n * done / (ms / 1e3),
            "unit": "cell-updates/s", "steps": done, "ms_per_step": step_ms, "dtype": "f64",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": None,
                         "scope": f"whole step; algorithmic bytes {algo / n:.0f} B per cell-update x {n} cells "
                                  f"(bench.ddp_algo_bytes) / device time per step",
                         "kernels": {k: {"ms": v, "share": v / tot if tot > 0 else None} for k, v in phases.items()}},
            "gpu_launches": done * model.kernels_per_step, "launch_config": tune["report"]}
    if local_rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = _ddp_reference_sample(pkg, args)
    return line


def run_closure(pkg, args, local_rank):
    """The learned momentum-exchange closure.  (1) Cost inside the step: the DIP channel
    (Godunov, Manning, momentum dissipation) timed with the plain closure and with a network
    attached in its place (random weights, a hull that admits every cell: the network runs for
    every cell inside the cell-update kernel), CUDA events on the library's stream; the three
    layers' FLOPs per step over the added time.  (2) The pipeline on building layouts
    (400 m x 200 m, buildings 5-30 m at 30 % cover, fine 1 m triangles, coarse 8 m DIP cells):
    on-trajectory samples with nudging targets from three layouts, training on the tensor
    cores, and on two unseen layouts the coarse runs' errors against the fine run averaged onto
    them: without closure, with the plain closure (mu 0.1, 0.3), with the learned one."""
    import numpy as np
    import torch

    C = pkg.closure
    case = pkg.workloads.dip_channel(n_cells=args.closure_cells, scheme="godunov", t_max=1.0e9)
    model = pkg.SpModel(case, device=local_rank)
    stream = torch.cuda.ExternalStream(model.stream, device=local_rank)

    def timed(steps):
        model.step(40)  # warm-up, including the capture of the step graph
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        done = model.step(steps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / done

    base_ms = timed(100)
    norm = np.concatenate([np.zeros(10), np.ones(10), np.zeros(2), np.full(2, 1e-6)]).astype(np.float32)
    net = C.MLP(C.init_params(1), norm, device=local_rank)
    model.set_closure(net, np.full(10, -1e30, np.float32), np.full(10, 1e30, np.float32))
    clos_ms = timed(100)
    kps = model.kernels_per_step
    n = case.mesh.cell_nb
    flops = 2.0 * n * (16 * 64 + 64 * 64 + 64 * 16)
    model.close()
    net.close()
    peak = None
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        peak = float(json.load(open(p)).get("bf16_tflops", 0.0)) or None
    added = clos_ms - base_ms
    line = {"workload": f"DIP channel at {n} cells (Godunov, Manning, momentum dissipation); the network in place "
                        f"of the plain closure for every cell",
            "ms_per_step_plain_closure": base_ms, "ms_per_step_learned_closure": clos_ms,
            "added_ms_per_step": added, "kernels_per_step": kps,
            "network_flops_per_step": flops,
            "tensor_tflops_over_added_time": flops / (added * 1e-3) / 1e12 if added > 0 else None,
            "bf16_peak_tflops": peak}
    if args.closure_no_pipeline:
        return line
    t0 = time.perf_counter()
    lay = {s: C.urban_cases(lx=400.0, ly=200.0, dx_fine=1.0, coarse_factor=8, seed=s) for s in (1, 2, 3, 7, 8)}
    t1 = time.perf_counter()
    net, lo, hi, hist, n_samples = C.train_on_layouts([lay[1], lay[2], lay[3]], tau=16.0, epochs=12,
                                                      device=local_rank)
    t2 = time.perf_counter()
    ev = {f"layout{s}_{a:g}-{b:g}s": C.evaluate(*lay[s], a, b, net=net, hull=(lo, hi), device=local_rank)
          for s in (7, 8) for a, b in ((10.0, 30.0), (20.0, 45.0))}
    t3 = time.perf_counter()
    net.close()
    return {**line,
            "pipeline": {"layouts": "400 m x 200 m, buildings 5-30 m at 30 % cover, seeds 1-3 train, 7-8 judged",
                         "fine_cells": lay[1][0].mesh.cell_nb, "coarse_cells": lay[1][1].mesh.cell_nb,
                         "samples": n_samples, "tau_s": 16.0,
                         "s_layouts": t1 - t0, "s_collect_and_train": t2 - t1, "s_evaluate": t3 - t2,
                         "train_loss_first_last": [hist[0], hist[-1]],
                         "coarse_error_vs_fine_h_q": ev}}


def run_result(pkg, args, local_rank):
    """The binary map file written during a run: the Gaussian-bump construction at
    `--result-cells` cells, 200 graph-launched steps with a map every 20 steps' time (dt_map),
    without and with ResultHydro.bin attached (frames copied from the device on a side stream
    and written by the library's thread while the next steps run).  Host wall time around the
    steps and, with the file, until the last frame is on file."""
    import shutil
    import tempfile

    import torch

    folder = tempfile.mkdtemp(prefix="sw2d_result_")
    try:
        case = pkg.workloads.gaussian_bumps(n_cells=args.result_cells)
        probe = pkg.SpModel(case, device=local_rank)
        probe.step(5)
        dt = probe.dt
        probe.close()
        # a power of two near 20 steps' time: the snapped times are then multiples of it
        # exactly, which checkStore's test needs
        import math
        case.opts = dict(case.opts, dt_map=repr(2.0 ** round(math.log2(20 * dt))), t_max="1e9")
        pkg.write_case(folder, case)
        geo = os.path.join(folder, "input", "geometry.sw2d")

        def run(with_file):
            m = pkg.SpModel(case, device=local_rank)
            m.step(40)
            torch.cuda.synchronize()
            path = os.path.join(folder, "ResultHydro.bin")
            if with_file:
                m.result_open(path, geo, "default")
            t0 = time.perf_counter()
            done = m.step(200)
            if with_file:
                m.result_close()
            torch.cuda.synchronize()
            el = time.perf_counter() - t0
            size = os.path.getsize(path) if with_file else 0
            m.close()
            return el, done, size

        t_plain, n_plain, _ = run(False)
        t_file, n_file, size = run(True)
        with open(geo, "rb") as fh:
            geo_bytes = len(fh.read())
        n = case.mesh.cell_nb
        frame = 8 + 8 * 5 * n
        frames = (size - geo_bytes) // frame if size > geo_bytes else 0
        return {"workload": f"SP Gaussian bumps at {n} cells, 200 steps, a map every {case.opts['dt_map']} s "
                            f"(about 20 steps), store_flag default",
                "ms_per_step_without_file": 1e3 * t_plain / max(n_plain, 1),
                "ms_per_step_with_file": 1e3 * t_file / max(n_file, 1),
                "frames": int(frames), "frame_mb": frame / 1e6, "file_mb": size / 1e6,
                "frame_gb_per_s_over_run": frames * frame / t_file / 1e9,
                "overhead": (t_file / max(n_file, 1)) / (t_plain / max(n_plain, 1)) - 1.0,
                "timing": "host wall time; with the file, until every frame is on file"}
    finally:
        shutil.rmtree(folder, ignore_errors=True)


def run_result_only(args, local_rank):
    pkg = importlib.import_module(PKG)
    pkg.build.build()
    import torch
    torch.cuda.set_device(local_rank)
    print(json.dumps(run_result(pkg, args, local_rank)))


def run_closure_only(args, local_rank):
    pkg = importlib.import_module(PKG)
    pkg.build.build()
    import torch
    torch.cuda.set_device(local_rank)
    print(json.dumps(run_closure(pkg, args, local_rank)))


def run_ddp_only(args, local_rank):
    pkg = importlib.import_module(PKG)
    pkg.build.build()
    import torch
    torch.cuda.set_device(local_rank)
    line = run_ddp(pkg, args, local_rank)
    line["clocks"] = None
    print(json.dumps(line))


def run_ensemble(pkg, args, local_rank):
    """Batched ensemble: `--ensemble-members` independent SP solves, sizes log-uniform in
    [5k, 200k] cells (seeded), alternately the dam-break and the Gaussian-bump constructions,
    MUSCL-EVR + HLLC, Manning n perturbed by +-20 % (smooth field, per member).  Forward:
    `--ensemble-steps` steps of every member in three forms, each timed with CUDA events on the
    device: the work queue (one persistent kernel over (step, phase, member, tile) items, its
    launch variant and tile size autotuned first), the graph of per-member stream branches, and
    the members one after another (each with its own step graph; the sum of the members' device
    times).  Every form continues from the same states (saved and restored), and the queue's and
    the branches' results are checked bit for bit against the sequential ones.  Adjoint: each
    member records its trajectory and observes 16 gauges every 10 steps; the members' gradients
    run concurrently (batch, host threads) and one after another (host wall time)."""
    import numpy as np
    import torch

    rng = np.random.default_rng(17)
    M = args.ensemble_members
    sizes = np.exp(rng.uniform(np.log(5_000), np.log(200_000), M)).astype(int)
    models = []
    for i, nc in enumerate(sizes):
        if i % 2 == 0:
            case = pkg.workloads.dam_break(n_cells=int(nc), scheme="muscl_evr", seed_mesh=100 + i, seed_phi=300 + i)
        else:
            case = pkg.workloads.gaussian_bumps(n_cells=int(nc), seed_mesh=100 + i)
        m = pkg.SpModel(case, device=local_rank)
        x, y = case.mesh.cell_x, case.mesh.cell_y
        f = np.sin(2 * np.pi * (x - x.min()) / (np.ptp(x) or 1.0) + i) * np.cos(np.pi * (y - y.min()) / (np.ptp(y) or 1.0))
        n1 = m.get_param("friction_1")
        m.set_param("friction", n1 * (1.0 + 0.2 * f))
        models.append(m)
    cells = int(sum(m.n for m in models))
    K = args.ensemble_steps
    batch = pkg.Batch(models)
    batch.step(3)
    for m in models:
        m.save_point()

    def reset():
        for m in models:
            m.restore_point()

    bstream = torch.cuda.ExternalStream(batch.stream, device=local_rank)

    def timed_batch():
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(bstream)
        done = batch.step(K)
        e1.record(bstream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, done

    tune = batch.autotune(steps=4)
    reset()
    batch.step(32)       # warm-up (graph capture), then back to the start
    reset()
    t_queue, done_q = timed_batch()
    end_q = [m.state() for m in models]
    reset()
    batch.configure(pkg.Batch.BRANCHES)
    batch.step(32)
    reset()
    t_branch, done_b = timed_batch()
    end_b = [m.state() for m in models]
    # sequential: each member alone with its own step graph, device time per member summed
    reset()
    t_seq, done_seq = 0.0, []
    for m in models:
        m.prepare()
        s = torch.cuda.ExternalStream(m.stream, device=local_rank)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        done_seq.append(m.step(K))
        e1.record(s)
        e1.synchronize()
        t_seq += e0.elapsed_time(e1) / 1e3
    end_s = [m.state() for m in models]
    if int(np.sum(done_q)) != M * K or int(np.sum(done_b)) != M * K or sum(done_seq) != M * K:
        raise RuntimeError("ensemble: a member stopped early")
    same = lambda A, B: all(np.array_equal(x.view(np.int64), y.view(np.int64)) for a, b in zip(A, B) for x, y in zip(a, b))
    # adjoints: record, observe, then concurrent vs sequential gradients
    for m in models:
        m.record(K, args.ensemble_every)
        g = np.sort(rng.choice(m.n, size=16, replace=False))
        st = np.arange(10, K + 1, 10)
        m.set_observations(g, st, m.replay_sample(g, st) * 1.01)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = batch.adjoint(n_threads=16)
    t_adj_batch = time.perf_counter() - t0
    nonfinite = [int(sum(m.adjoint_nonfinite().values())) for m in models]
    t0 = time.perf_counter()
    res_seq = [m.adjoint() for m in models]
    t_adj_seq = time.perf_counter() - t0
    same_adj = all(a[0] == b[0] and all(np.array_equal(a[1][k], b[1][k]) for k in a[1]) for a, b in zip(res, res_seq))
    free, total = torch.cuda.mem_get_info(local_rank)
    batch.close()
    return {
        "workload": f"{M} SP members, {int(sizes.min())}-{int(sizes.max())} cells (log-uniform, {cells} in all), "
                    f"dam break / Gaussian bumps, MUSCL-EVR + HLLC, Manning n +-20 %, {K} steps each",
        "metric": "ensemble cell-updates/s", "unit": "cell-updates/s",
        "value": cells * K / t_queue,
        "arms_device_s": {"work_queue": t_queue, "stream_branches": t_branch, "sequential": t_seq},
        "arms_value": {"work_queue": cells * K / t_queue, "stream_branches": cells * K / t_branch,
                       "sequential": cells * K / t_seq},
        "speedup_queue_over_sequential": t_seq / t_queue, "speedup_queue_over_branches": t_branch / t_queue,
        "bitwise_same_as_sequential": {"work_queue": bool(same(end_q, end_s)), "stream_branches": bool(same(end_b, end_s))},
        "queue_tuning": tune,
        "adjoint": {"gradients_per_s": M / t_adj_batch, "sequential_gradients_per_s": M / t_adj_seq,
                    "speedup": t_adj_seq / t_adj_batch, "s_batched": t_adj_batch, "s_sequential": t_adj_seq,
                    "checkpoint_every": args.ensemble_every, "bitwise_same_as_sequential": bool(same_adj),
                    "timing": "host wall time (the adjoints run from host threads)",
                    "nonfinite_entries_set_to_zero": int(sum(nonfinite)),
                    "nonfinite_per_member": {str(i): c for i, c in enumerate(nonfinite) if c}},
        "device_memory_in_use_gb": (total - free) / 1e9,
        "timing": "forward: CUDA events on the device (queue and branches on the batch's stream; sequential: "
                  "sum of the members' own device times)",
    }


def run_assim_only(args, local_rank):
    import torch

    pkg = importlib.import_module(PKG)
    pkg.build.build()
    torch.cuda.set_device(local_rank)
    print(json.dumps(run_assim(pkg, args, local_rank)))


def run_adjoint_only(args, local_rank):
    import torch

    pkg = importlib.import_module(PKG)
    pkg.build.build()
    torch.cuda.set_device(local_rank)
    print(json.dumps(run_adjoint(pkg, args, local_rank)))


def run_ours(args, rank, world, local_rank):
    import numpy as np

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # before any GPU call; spawned processes
        from oracle.binding import reference_available
        if reference_available():
            r = reference_timing(1, 3, args.cpu_steps)
            cpu = {"value": r["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"reference native solver (oracle/_ref), same construction at {r['cells']} cells, "
                             f"{r['steps']} MUSCL steps, 1 thread ({_cpu_model()}); "
                             f"{r['seconds']:.1f} s of CPU time"}

    import torch

    pkg = importlib.import_module(PKG)
    pkg.build.build()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))

    case = pkg.workloads.gaussian_bumps(n_cells=args.cells, mesh=args.mesh)
    model = pkg.SpModel(case, device=local_rank)
    stream = torch.cuda.ExternalStream(model.stream, device=local_rank)
    n = case.mesh.cell_nb
    dry_fraction = float(np.mean(case.h0 <= float(case.opts["h_min"])))

    def barrier():
        if dist is not None:
            dist.barrier()

    # launch-configuration autotune on the live state (no step taken), then warm-up (also
    # builds the CUDA graph)
    if args.flux_variant is not None:
        model.set_option("flux_variant", args.flux_variant)
        tune = {"report": f"fixed k_flux variant {args.flux_variant}"}
    elif args.launch_config:
        sv, ev = (int(v) for v in args.launch_config.split(","))
        model._check(model.lib.sw2d_set_launch_config(model.handle, sv, ev))
        tune = {"report": f"fixed variants slopes={sv} edges={ev}"}
    else:
        tune = pkg.tuning.autotune_step(model, iters=5, device=local_rank, cache_path=None)
    model.step(args.warmup)
    phases = model.phase_times(args.phase_steps)
    model.prepare()  # the step graph is captured before the timed region

    # ---- timed region: K graph-captured steps with inputs resident in HBM
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        done = model.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if done != args.steps:
        raise RuntimeError(f"only {done} of {args.steps} steps ran (t_max reached?)")
    t_max_rank = torch.tensor([ms], dtype=torch.float64, device=f"cuda:{local_rank}")
    if dist is not None:
        dist.all_reduce(t_max_rank, op=dist.ReduceOp.MAX)
    ms = float(t_max_rank.item())

    # ---- e2e: the C ABI with host buffers, state uploaded and read back every chunk of steps
    chunk = max(1, min(args.e2e_chunk, args.steps))
    n_chunks = max(1, args.steps // chunk)
    hb = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    model.lib.sw2d_get_state(model.handle, *(t.data_ptr() for t in hb))
    lib = model.lib
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    import ctypes
    k = ctypes.c_int64(0)
    for _ in range(n_chunks):
        if lib.sw2d_set_state(model.handle, *(t.data_ptr() for t in hb)) != 0:
            raise RuntimeError(lib.sw2d_last_error(model.handle).decode())
        if lib.sw2d_step_n(model.handle, chunk, ctypes.byref(k)) != 0 or k.value != chunk:
            raise RuntimeError("e2e step failed")
        if lib.sw2d_get_state(model.handle, *(t.data_ptr() for t in hb)) != 0:
            raise RuntimeError(lib.sw2d_last_error(model.handle).decode())
    e1.record(stream)
    e1.synchronize()
    e2e_ms = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=f"cuda:{local_rank}")
    if dist is not None:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_ms = float(e2e_ms.item())
    h_final = hb[0].numpy()
    if not np.all(np.isfinite(h_final)):
        raise RuntimeError("non-finite depth")

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    kps = model.kernels_per_step
    del model
    wet = None if (args.wet_steps <= 0 or world > 1) else run_wet(pkg, args, local_rank)
    adjoint = None if (args.no_adjoint or world > 1) else run_adjoint(pkg, args, local_rank)
    dip = None if (args.dip_cells <= 0 or world > 1) else run_dip(pkg, args, local_rank)
    ddp = None if (args.ddp_cells <= 0 or world > 1) else run_ddp(pkg, args, local_rank)
    assim = None if (args.assim_cells <= 0 or world > 1) else run_assim(pkg, args, local_rank)
    ensemble = None if (args.ensemble_members <= 0 or world > 1) else run_ensemble(pkg, args, local_rank)
    closure = None if (args.no_closure or world > 1) else run_closure(pkg, args, local_rank)
    result = None if (args.result_cells <= 0 or world > 1) else run_result(pkg, args, local_rank)

    steps = args.steps
    value = n * steps * world / (ms / 1e3)
    e2e_steps = n_chunks * chunk
    e2e_value = n * e2e_steps * world / (e2e_ms / 1e3)
    peak, peak_kind = _measured_peak()
    step_ms = ms / steps
    algo_bytes = ALGO_BYTES_PER_CELL_UPDATE * n
    achieved = algo_bytes / (step_ms / 1e3) / 1e9
    traffic = _traffic_per_step()
    tot_phase = sum(phases.values())
    kernels = {k2: {"ms": v, "share": v / tot_phase if tot_phase > 0 else None} for k2, v in phases.items()}
    dominant = max(phases, key=phases.get)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": args.warmup,
        "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Gaussian-bump bed, smooth porosity field, lognormal Manning n)",
        "config": {**_config(args, world), "dry_fraction": dry_fraction,
                   "initial_state": "lake at rest h = max(0, 2 - z_b): dry cells and still water"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 3 * 8 * n / chunk,
                "d2h_bytes_per_step": (3 * 8 * n + 2 * 48) / chunk,
                "note": f"sw2d_set_state + sw2d_step_n({chunk}) + sw2d_get_state from pinned host buffers per chunk"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind,
                     "traffic": (traffic.get("bytes_per_cell_update") * n if traffic else None),
                     "scope": f"whole step ({kps} kernels); algorithmic bytes {ALGO_BYTES_PER_CELL_UPDATE} B per "
                              f"cell-update x {n} cells per step / device time per step in the timed region",
                     "dominant_kernel": dominant, "kernels": kernels},
        "gpu_launches": steps * kps,
        "launch_config": tune["report"],
        "clocks": clk.summary(),
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if wet is not None:
        line["wet"] = wet
    if adjoint is not None:
        line["adjoint"] = adjoint
    if dip is not None:
        line["dip"] = dip
    if ddp is not None:
        line["ddp"] = ddp
    if assim is not None:
        line["assim"] = assim
    if ensemble is not None:
        line["ensemble"] = ensemble
    if closure is not None:
        line["closure"] = closure
    if result is not None:
        line["result_file"] = result
    print(json.dumps(line))


def main():
    args = _args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
    elif args.adjoint_only:
        if rank == 0:
            run_adjoint_only(args, local_rank)
    elif args.assim_only:
        if rank == 0:
            run_assim_only(args, local_rank)
    elif args.ddp_only:
        if rank == 0:
            run_ddp_only(args, local_rank)
    elif args.closure_only:
        if rank == 0:
            run_closure_only(args, local_rank)
    elif args.result_only:
        if rank == 0:
            run_result_only(args, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
