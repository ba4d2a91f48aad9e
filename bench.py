#!/usr/bin/env python
"""Benchmark of the B200 MAC 3D smoke step.

Workload (synthetic, seeded): the Reflection + MacCormack plume of the
128^3 configuration, run at 256^3: box 1, dt 0.01, two profile sources
min(1, 3 exp(-3.5 (d/r)^2)) of radius .08 at (x, y, z) = (.3, .5, .15) and
(.7, .5, .15) (z up), buoyancy 1.5, smoke decay .995 per step, no kick or stir,
initial velocity a seeded swirl of 8 Gaussian vortices (amplitude .5). Every
projection solves to relative residual (= relative divergence) 1e-6, verified
in FP64. Two arms run on the same scene:
  learned (the headline value): flexible PCG whose preconditioner is red-black
    Gauss-Seidel smoothing around the learned U-Net coarse-grid correction
    (weights vapor_b200/weights/coarse_unet.npy);
  plain: the reference's red-black SOR (FP32 sweeps with FP64 residual and
    re-centring, since FP32 SOR alone stalls above 1e-6).
Metric: steps/s (higher is better), with the plain arm, the sweep ratio and
the kernels' roofline fractions beside it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N>1 runs under torchrun as independent replicas (one scene per GPU, no
collective on the data path); value = N*K / max over ranks of the timed
region. Prints one JSON line on rank 0.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from vapor_b200.plume import DT, omega_for, scene_params, swirl_fields  # noqa: E402
from vapor_b200.replicas import aggregate_steps_per_second, max_over_ranks, rank_info, scene_seed  # noqa: E402

METRIC = "256^3 steps/s: learned-warm-start vs plain GPU solve at rel div 1e-6; HBM %"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--rel", type=float, default=1e-6)
    ap.add_argument("--max-iterations", type=int, default=20000)
    ap.add_argument("--omega", type=float, default=None)
    ap.add_argument("--interval", type=int, default=8, help="residual check interval (sweeps)")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--reference-sweeps", type=float, default=None,
                    help="reference arm: SOR sweeps per step to charge (default: the plain GPU arm's, from "
                         "vapor_b200/tuning/plain_sweeps.json for the same warm-up and steps)")
    ap.add_argument("--cpu-sample", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--record-plain-sweeps", action="store_true",
                    help="write the plain arm's per-step sweep counts (vapor_b200/tuning/plain_sweeps.json)")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--weights", default=os.path.join(ROOT, "vapor_b200", "weights", "coarse_unet.npy"),
                    help="coarse-grid U-Net parameters of the learned arm")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.mark = 0

    def start(self):
        exe = shutil.which("nvidia-smi")
        if not exe:
            return
        self.proc = subprocess.Popen([exe, f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                      "--format=csv,noheader,nounits", "-lms", "50"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # the timed region starts once the sampler is live; earlier samples are dropped
        deadline = time.perf_counter() + 5.0
        while not self.lines and time.perf_counter() < deadline and self.proc.poll() is None:
            time.sleep(0.01)
        self.mark = len(self.lines)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.lines[self.mark:] or self.lines[-1:]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# Fixed SOR sweep counts of the two timed reference steps: the difference of
# their times is the cost of 64 sweeps at the full grid.
REFERENCE_SWEEPS_LOW, REFERENCE_SWEEPS_HIGH = 16, 80
PLAIN_SWEEPS_TABLE = os.path.join(ROOT, "vapor_b200", "tuning", "plain_sweeps.json")


def reference_step_costs(n, seed):
    """Times the reference's own compiled CPU MAC 3D step (oracle/_ref:
    MacGridFluidSolver3D::advance, MacGridFluidSolver3D.cpp:192-245) at the
    full n^3 grid on the benchmark plume's initial state: one untimed step
    (first touch of the solver's work arrays), then one complete step with
    REFERENCE_SWEEPS_HIGH and one with REFERENCE_SWEEPS_LOW fixed SOR sweeps.
    A step's time is linear in its sweep count by construction (each sweep is
    one pass of SOR.cpp:36-54 over the grid), so the two steps give the cost
    of one sweep and the rest of the step (advection, divergence, gradient,
    forcing). The reference has no profile emitter or second source; its
    step uses its own emitter at the first source position. Single-threaded:
    the reference's build enables no OpenMP and its sweep is serial."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_lib import RefSim, default_params, ref_available
    if not ref_available():
        return None
    sim = RefSim(n, 1.0, fields=swirl_fields(n, seed))
    p = default_params()
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = 1, 1, 1
    p.buoyancy, p.smoke_decay, p.emitter_radius, p.source_strength = 1.5, 0.5, 0.08, 1.0
    p.emitter_center_x, p.emitter_center_y, p.emitter_center_z = 0.3, 0.5, 0.15
    p.emitter_kick_multiplier, p.stir_strength = 0.0, 0.0
    p.sor_omega = omega_for(n)
    times = {}
    for sweeps, timed in ((REFERENCE_SWEEPS_LOW, False), (REFERENCE_SWEEPS_HIGH, True),
                          (REFERENCE_SWEEPS_LOW, True)):
        p.project_iterations = sweeps  # the Reflection step runs two projections of sweeps / 2
        sim.params = p
        t0 = time.perf_counter()
        if sim.advance(DT) != 0:
            raise RuntimeError("reference step failed")
        if timed:
            times[sweeps] = time.perf_counter() - t0
    per_sweep = (times[REFERENCE_SWEEPS_HIGH] - times[REFERENCE_SWEEPS_LOW]) / (REFERENCE_SWEEPS_HIGH -
                                                                               REFERENCE_SWEEPS_LOW)
    fixed = times[REFERENCE_SWEEPS_LOW] - REFERENCE_SWEEPS_LOW * per_sweep
    return {"n": n, "fixed_s": fixed, "per_sweep_s": per_sweep,
            "timed_steps": [{"sweeps": s, "seconds": t} for s, t in times.items()]}


def plain_sweeps_charged(warmup, steps):
    """Mean SOR sweeps per step of the plain GPU arm over the same window of
    steps (after `warmup` steps, `steps` steps) on the same seeded scene, from
    the per-step table that `bench.py --record-plain-sweeps` wrote (the plain
    arm is deterministic: fixed-order reductions, bit-identical replays).
    Steps past the table's end are charged its last entry."""
    with open(PLAIN_SWEEPS_TABLE) as f:
        table = json.load(f)
    per_step = table["per_step"]
    window = [per_step[min(i, len(per_step) - 1)] for i in range(warmup, warmup + max(1, steps))]
    return sum(window) / len(window), table


def reference_line(costs, sweeps, source):
    """cpu_baseline object: the reference step's measured costs charged
    `sweeps` sweeps per step."""
    step_s = costs["fixed_s"] + sweeps * costs["per_sweep_s"]
    timed = costs["timed_steps"]
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": 1, "kind": "reference",
            "extrapolated": True, "sweeps_charged": sweeps, "sweeps_source": source,
            "sample": (f"reference CPU MAC 3D step (oracle/_ref, single-threaded) at {costs['n']}^3, two complete "
                       f"steps after one untimed step: " +
                       ", ".join(f"{t['sweeps']} sweeps {t['seconds']:.2f} s" for t in timed) +
                       f" -> {costs['fixed_s']:.2f} s per step without the solve + "
                       f"{costs['per_sweep_s'] * 1e3:.1f} ms per sweep; value charges {sweeps:.1f} sweeps per step "
                       f"(linear along the sweep axis only)"),
            "measured_ms_per_step": 1e3 * sum(t["seconds"] for t in timed) / len(timed),
            "nproc": os.cpu_count()}


def run_reference(args):
    """--impl reference: the reference's CPU path on the host cores, at the
    benchmark grid, charged the plain GPU arm's sweeps for the same steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t_start = time.perf_counter()
    if args.reference_sweeps is not None:
        sweeps, source = float(args.reference_sweeps), "--reference-sweeps"
    else:
        sweeps, table = plain_sweeps_charged(args.warmup, args.steps)
        if table["n"] != args.n:
            raise SystemExit(f"{PLAIN_SWEEPS_TABLE} holds {table['n']}^3 counts; pass --reference-sweeps "
                             f"for {args.n}^3")
        source = (f"plain GPU arm's mean sweeps per step over steps {args.warmup}..{args.warmup + args.steps - 1} "
                  f"of the same scene ({os.path.relpath(PLAIN_SWEEPS_TABLE, ROOT)}: {table['command']})")
    costs = reference_step_costs(args.n, args.seed)
    if costs is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (reference CPU build) missing"}))
        return
    base = reference_line(costs, sweeps, source)
    value = base["value"]
    timed = costs["timed_steps"]
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": args.gpus,
            "steps": len(timed), "warmup": 1, "ms_per_step": base["measured_ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "extrapolated": True,
            "config": {"workload": f"mac3d_reflection_maccormack_{args.n}", "n": args.n,
                       "sweeps_per_step": sweeps,
                       "note": "steps, warmup and ms_per_step describe the reference steps that ran (fixed sweep "
                               "counts); value charges them the plain GPU arm's sweeps per step, because the "
                               "reference's FP32 SOR stagnates above relative residual 1e-6"},
            "cpu_baseline": base, "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0,
                                          "d2h_bytes_per_step": 0},
            "wall_s": time.perf_counter() - t_start}
    print(json.dumps(line))


def start_cpu_sample(args):
    """Starts the reference CPU timing in its own process, before any CUDA
    call, so that it runs beside the GPU arms on another host core."""
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-sample", "--n", str(args.n), "--seed", str(args.seed)]
    return subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)


def finish_cpu_sample(proc, sweeps, timeout=600):
    try:
        out, err = proc.communicate(timeout=timeout)
    except subprocess.TimeoutExpired:
        proc.kill()
        return {"value": None, "unavailable": f"reference CPU timing exceeded {timeout} s"}
    if proc.returncode != 0 or not out.strip():
        return {"value": None, "unavailable": f"reference CPU timing failed: {err.strip()[-200:]}"}
    costs = json.loads(out.strip().splitlines()[-1])
    if costs is None:
        return {"value": None, "unavailable": "oracle/_ref (reference CPU build) missing"}
    return reference_line(costs, sweeps, "plain GPU arm of this run")


def record_plain_sweeps(args):
    """Writes the plain arm's SOR sweeps for each of the first `steps` steps
    of the benchmark scene (the table the reference arm charges)."""
    import vapor_b200 as vb
    from vapor_b200.abi import SOLVER_MIXED_REFINEMENT
    n = args.n
    params = scene_params(vb.default_params(), n, args.rel, args.max_iterations, omega_for(n, args.omega),
                          interval=args.interval)
    params.solver_kind = SOLVER_MIXED_REFINEMENT
    sim = vb.MacSimulation3D(n, 1.0, params)
    sim.upload(*swirl_fields(n, scene_seed(args.seed, 0)))
    per_step = []
    for _ in range(args.steps):
        it0 = sim.total_iterations()
        sim.advance(DT)
        per_step.append(int(sim.total_iterations() - it0))
    sim.close()
    table = {"n": n, "seed": args.seed, "relative_tolerance": args.rel, "omega": omega_for(n, args.omega),
             "command": f"python bench.py --record-plain-sweeps --n {n} --steps {args.steps}",
             "per_step": per_step}
    with open(PLAIN_SWEEPS_TABLE, "w") as f:
        json.dump(table, f, indent=1)
    print(json.dumps(table))


# DRAM bytes (read 100.67 MB + written 8.95 MB) of one k_sor_rbz colour
# launch at 256^3, from an ncu --set full capture on the benchmark plume.
SOR_TRAFFIC_256 = 100.673792e6 + 8.947968e6


def network_flops(nc):
    """FLOPs of one U-Net forward on an nc^3 grid: the ten 3x3x3 convolutions
    (27 taps x cin x cout multiply-adds per voxel of their level)."""
    macs = 27 * nc ** 3 * (16 * 16 * 2 + 48 * 16 + 16 * 16 + (16 * 32 + 32 * 32 + 96 * 32 + 32 * 32) / 8.0 +
                           (32 * 64 + 64 * 64) / 64.0)
    return 2.0 * macs


# Algorithmic bytes per cell of one Reflection-MacCormack step by phase
# (compulsory FP32 traffic, counted per pass): forcing = emit + buoyancy +
# walls 12; advection = velocity with flow as source 24 + velocity with the
# reflected field as source 36 + smoke with decay 20; divergence 16 per
# projection; gradient 52 with the reflection + 28 without, plus the final
# FP64 residual 8 per projection.
PHASE_BYTES_PER_CELL = {"forcing": 12.0, "advect": 80.0, "rhs": 32.0, "gradient": 96.0}


def phase_rooflines(phases, steps, cells, peak, peak_kind):
    """HBM fraction of the memory-bound phases outside the solve: algorithmic
    bytes per step over the phase's event time per step (launch gaps
    included, so a lower bound on the kernels' own fractions)."""
    out = {}
    for name, per_cell in PHASE_BYTES_PER_CELL.items():
        ms = phases.get(name, {}).get("ms", 0.0) / max(1, steps)
        if ms <= 0:
            continue
        achieved = per_cell * cells / (ms * 1e-3) / 1e9
        out[name] = {"bytes_per_cell": per_cell, "ms_per_step": ms, "achieved": achieved, "unit": "GB/s",
                     "frac": achieved / peak, "peak": peak, "peak_kind": peak_kind}
    return out


def run_arm(vb, torch, args, n, fields, kind, net, dist, clocks=None):
    """Warm-up, then K timed steps (CUDA-graph replays) of one solver arm."""
    params = scene_params(vb.default_params(), n, args.rel, args.max_iterations, omega_for(n, args.omega),
                          interval=args.interval)
    params.solver_kind = kind
    sim = vb.MacSimulation3D(n, 1.0, params)
    sim.upload(*fields)
    if net is not None:
        sim.set_preconditioner(net)
    for _ in range(args.warmup):
        sim.advance(DT)
    sim.synchronize()
    stream = torch.cuda.ExternalStream(sim.stream())
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    it0 = sim.total_iterations()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    wall0 = time.perf_counter()
    start.record(stream)
    for _ in range(args.steps):
        sim.advance(DT)
    end.record(stream)
    end.synchronize()
    wall = time.perf_counter() - wall0
    clock_info = clocks.stop() if clocks else None
    torch.cuda.synchronize()
    ms = max_over_ranks(start.elapsed_time(end), dist, "cuda")
    r = sim.last_projection().linear_solve
    return sim, stream, {"ms": ms, "iterations": (sim.total_iterations() - it0) / args.steps,
                         "final_relative_residual": r.final_residual / max(r.initial_residual, 1e-300),
                         "converged": bool(r.converged), "wall_s": wall, "clocks": clock_info}


def eager_phases(vb, sim, steps):
    """The same step on the eager path with per-phase CUDA events on the
    simulation's stream; also counts this library's kernel launches."""
    sim.set_timing(True)
    launches0 = vb.kernel_launch_count()
    it0 = sim.total_iterations()
    for _ in range(steps):
        sim.advance(DT)
    sim.synchronize()
    launches = (vb.kernel_launch_count() - launches0) / steps
    phases = sim.timings()
    its = (sim.total_iterations() - it0) / steps
    sim.set_timing(False)
    return phases, launches, its


def main():
    args = parse()
    world, rank, local = rank_info()
    if args.cpu_sample:
        print(json.dumps(reference_step_costs(args.n, args.seed)))
        return
    if args.impl == "reference":
        run_reference(args)
        return
    if args.record_plain_sweeps:
        record_plain_sweeps(args)
        return
    cpu_proc = start_cpu_sample(args) if rank == 0 and world == 1 and not args.no_cpu_baseline else None

    import torch
    import vapor_b200 as vb
    from vapor_b200.abi import SOLVER_FPCG, SOLVER_MIXED_REFINEMENT
    from vapor_b200.learned import WarmStartNet

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    vb.set_device(local)
    torch.cuda.set_device(local)

    n = args.n
    fields = swirl_fields(n, scene_seed(args.seed, rank))
    if not os.path.exists(args.weights):
        raise SystemExit(f"learned coarse-grid weights not found: {args.weights}")
    net = WarmStartNet.load(args.weights)

    # Plain arm: the reference's red-black SOR (mixed precision to reach 1e-6).
    plain_sim, _, plain = run_arm(vb, torch, args, n, fields, SOLVER_MIXED_REFINEMENT, None, dist)
    plain_phases, _, plain_eager_sweeps = eager_phases(vb, plain_sim, 1)
    plain_sim.close()
    # Learned arm (headline): flexible PCG with the U-Net coarse-grid correction.
    clocks = ClockSampler(local)
    sim, stream, learned = run_arm(vb, torch, args, n, fields, SOLVER_FPCG, net, dist, clocks)
    roof_steps = max(1, min(args.steps, 2))
    phases, launches_per_step, eager_its = eager_phases(vb, sim, roof_steps)
    launches = int(round(launches_per_step * args.steps))

    # End to end through the public API: every step uploads the host state
    # from pinned memory and downloads the stepped state, with the streamed
    # transfers (upload_async / download_async): the copies of one step run
    # on copy streams under its neighbours' compute, and the timed region ends
    # after the last download reached the host.
    pinned = [torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy() for a in fields]
    for dst, src in zip(pinned, sim.download()):
        dst[...] = src
    out = [torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy() for a in fields]
    h2d = sum(a.nbytes for a in pinned)
    e2e_steps = max(1, args.e2e_steps)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        sim.upload_async(*pinned)
        sim.advance(DT)
        sim.download_async(out)
    sim.wait_transfers()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, dist, "cuda")

    peak, peak_kind = measured_peaks()
    cells = n ** 3

    def sor_roofline(ph, sweeps, dot_launches=0.0):
        """The red-black sweep phase of one eager step covering `sweeps`
        red+black iterations: per-launch algorithmic bytes over the average
        launch time. One red+black iteration reads x and b and writes x,
        12 B/cell, so a one-colour launch is charged half of that, 6 B/cell
        (the other colour's half of x, written by the previous launch, is
        mostly read back from L2); a temporally blocked launch of several
        iterations reads x and b and writes x once, 12 B/cell. In the FPCG
        preconditioner the last sweep of each CG step (`dot_launches` of
        them) also reads r of the other colour and q of both, 6 B/cell
        more."""
        sor = ph["sor"]
        launches = max(1, sor["launches"])
        launch_ms = sor["ms"] / launches
        per_launch = sweeps / launches
        blocked = per_launch >= 1.5
        nbytes = (12.0 if blocked else 6.0) * cells * (1.0 + dot_launches / launches)
        achieved = nbytes / (launch_ms * 1e-3) / 1e9
        line = {"bound": "hbm", "kernel": (f"k_sor_blocked ({per_launch:.0f} red+black iterations per launch)"
                                           if blocked else "k_sor_rbz (red-black colour sweep)"),
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": None if blocked else SOR_TRAFFIC_256 * cells / 256 ** 3,
                "traffic_note": ("see profiles/ for the blocked sweep's ncu traffic" if blocked else
                                 "dram bytes read + written per launch from an ncu --set full capture at 256^3, "
                                 "scaled by cells for other sizes"),
                "bytes_per_launch": nbytes, "avg_launch_us": launch_ms * 1e3,
                "sweeps_per_s": sweeps / (sor["ms"] * 1e-3) if sor["ms"] > 0 else None,
                "timing_note": "average launch time from CUDA events around the sweep phase of an eager replay of "
                               "the benchmarked step on the simulation's stream (the kernels inside the step's "
                               "CUDA graph cannot be bracketed one by one); launch gaps included"}
        return line

    # Network (tensor cores): FLOPs of the coarse U-Net per application over
    # the coarse phase's time per application (restriction, normalization,
    # Galerkin scale and prolongation included, so this is a lower bound).
    applications = eager_its + 2.0
    per_app = vb.fpcg_sweeps_per_application()
    sweeps_name, omega_now = vb.fpcg_smoothing()
    coarse_ms = phases["coarse"]["ms"] / roof_steps / max(1.0, applications)
    net_flops = network_flops(n // 4)
    tflops = net_flops / (coarse_ms * 1e-3) / 1e12 if coarse_ms > 0 else 0.0
    tpeak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("bf16_tflops_sustained", 1400.0)) \
        if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else 1400.0

    line = {
        "metric": METRIC, "value": aggregate_steps_per_second(world, args.steps, learned["ms"]), "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": learned["ms"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"mac3d_reflection_maccormack_{n}", "n": n, "dt": DT,
                   "solver": "flexible PCG, FP32 vectors + FP64 dots/residual/re-centring; preconditioner "
                             f"{sweeps_name}+{sweeps_name} red-black relaxation sweeps (omega {omega_now:g}) around "
                             f"the learned U-Net coarse-grid correction on {n // 4}^3 (BF16 tcgen05 convolutions)",
                   "weights": os.path.relpath(args.weights, ROOT), "relative_tolerance": args.rel,
                   "cg_iterations_per_step": learned["iterations"],
                   "sweeps_per_step": per_app * (learned["iterations"] + 2),
                   "final_relative_residual": learned["final_relative_residual"],
                   "converged": learned["converged"],
                   "l2": "state (4 x 67 MB fields) and solver vectors exceed the 126 MB L2",
                   "parallelism": f"replicas{world}"},
        "plain": {"solver": "red-black SOR (the reference's method), FP32 sweeps + FP64 residual/re-centring",
                  "value": aggregate_steps_per_second(world, args.steps, plain["ms"]), "unit": "steps/s",
                  "ms_per_step": plain["ms"] / args.steps, "sweeps_per_step": plain["iterations"],
                  "omega": omega_for(n, args.omega), "final_relative_residual": plain["final_relative_residual"],
                  "converged": plain["converged"], "roofline": sor_roofline(plain_phases, plain_eager_sweeps),
                  "phases_ms_per_step": {k: v["ms"] for k, v in plain_phases.items() if v["ms"] > 0}},
        "speedup_vs_plain": plain["ms"] / learned["ms"],
        "sweep_ratio_vs_plain": plain["iterations"] / max(1e-9, per_app * (learned["iterations"] + 2)),
        "gpu_launches": launches,
        "gpu_launches_note": "kernels per step counted on the eager replay of the same step, times steps",
        "roofline": sor_roofline(phases, per_app * (eager_its + 2.0) * roof_steps, eager_its * roof_steps),
        "roofline_tensor": {"bound": "tensor", "kernel": "coarse U-Net forward (k_conv3_zm and k_conv3_tc, 10 convolutions)",
                            "achieved": tflops, "peak": tpeak, "unit": "TFLOP/s", "frac": tflops / tpeak,
                            "peak_kind": "measured sustained", "flops_per_application": net_flops,
                            "ms_per_application": coarse_ms,
                            "note": "time includes restriction, normalization, Galerkin scale and prolongation"},
        "phases_ms_per_step": {k: v["ms"] / roof_steps for k, v in phases.items() if v["ms"] > 0},
        "phase_rooflines": phase_rooflines(phases, roof_steps, cells, peak, peak_kind),
        "e2e": {"value": world / (e2e_ms * 1e-3), "unit": "steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": h2d, "steps": e2e_steps,
                "transfers": "streamed: pinned upload_async before and download_async after every step"},
        "clocks": learned["clocks"], "wall_s": learned["wall_s"],
    }
    if cpu_proc is not None:
        line["cpu_baseline"] = finish_cpu_sample(cpu_proc, plain["iterations"])
    if rank == 0:
        print(json.dumps(line))
    sim.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
