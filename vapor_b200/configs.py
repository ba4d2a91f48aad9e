"""Measurement drivers for the configurations beside the headline benchmark.

  python -m vapor_b200.configs mixed-projection [--n 256 --seed 1 --rel 1e-8]
  python -m vapor_b200.configs batch [--scenes 48 --steps 100 --tuning tuning.json]

mixed-projection: one staged projection of a seeded random velocity field
(solenoidal plus gradient parts, energy spectrum ~ k^-5/3) in a closed box
with a seeded sphere obstacle (radius .1-.2), solved with FP32 red-black SOR
sweeps under FP64 residual checks and FP64 iterative refinement to relative
divergence 1e-8. Reports the device time, sweeps and the FP64-verified
residual. The error against the FP64 oracle is checked by the GPU tests
(tests/test_gpu_obstacles.py), which call mixed_projection with
return_fields=True.
"""
import argparse
import json
import numpy as np

from . import StageBackend
from .abi import SOLVER_MIXED_REFINEMENT, LinearSolveOptions, ProjectionOptions
from .plume import omega_for, spectral_fields


def sphere_mask(n, centre, radius):
    c = (np.arange(n) + 0.5) / n
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    d2 = (xx - centre[0]) ** 2 + (yy - centre[1]) ** 2 + (zz - centre[2]) ** 2
    return (d2 < radius * radius).astype(np.uint8)


def mixed_projection_scene(n, seed):
    rng = np.random.default_rng(seed)
    centre = tuple(float(c) for c in rng.uniform(0.3, 0.7, size=3))
    radius = float(rng.uniform(0.1, 0.2))
    u, v, w = spectral_fields(n, int(rng.integers(1 << 31)), slope=-5.0 / 3.0, gradient_fraction=0.5)
    return (u, v, w), sphere_mask(n, centre, radius), {"centre": centre, "radius": radius}


def mixed_projection(n=256, seed=1, rel=1e-8, dt=0.01, repeats=2, return_fields=False):
    """Returns the measurement; with return_fields also the scene's input
    velocity, mask and the projected (u, v, w, p) as numpy arrays."""
    import torch
    (u, v, w), mask, sphere = mixed_projection_scene(n, seed)
    stage = StageBackend(n, 1.0)
    stage.set_solver_kind(SOLVER_MIXED_REFINEMENT)
    stage.set_solid(mask)
    opts = ProjectionOptions(dt, omega_for(n), LinearSolveOptions.defaults(
        max_iterations=100000, relative_tolerance=rel, absolute_tolerance=0.0))
    dev = [torch.from_numpy(a.copy()).cuda() for a in (u, v, w)]
    p_dev = torch.zeros((n, n, n), dtype=torch.float32, device="cuda")
    times, result = [], None
    for _ in range(repeats):
        work = [d.clone() for d in dev]
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        result = stage.project_device(*[t.data_ptr() for t in work], opts, 6.0, p_dev.data_ptr())
        e1.record()
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ls = result.linear_solve
    out = {"config": "mixed_projection", "n": n, "seed": seed, "sphere": sphere,
           "solid_cells": int(mask.sum()), "relative_tolerance": rel, "sweeps": ls.iterations,
           "converged": bool(ls.converged), "fp64_relative_residual": ls.final_residual / ls.initial_residual,
           "ms": min(times), "sweeps_per_s": ls.iterations / (min(times) * 1e-3),
           "divergence_before": result.divergence_before, "divergence_after": result.divergence_after}
    if return_fields:
        got = [t.cpu().numpy() for t in work] + [p_dev.cpu().numpy()]
        return out, {"input": (u, v, w), "mask": mask, "dt": dt, "projected": got}
    return out


def batch_scenes(count=48, seed=11, steps=100, warmup=3, tuning=None, rel=1e-6):
    """Uneven-grid plume scenes stepped two ways from the same initial state:
    each scene's own step graph on its own stream, and all scenes in one
    batched graph (vapor_batch_advance). Sizes from {32,48,64,96,128}, per
    scene a seeded source position, radius .05-.12 and buoyancy .5-2;
    Reflection + MacCormack, mixed-precision red-black SOR to 1e-6."""
    import torch
    from . import Batch, MacSimulation3D, default_params
    from .autotune import apply
    from .plume import DT, scene_params
    omegas = apply(tuning) if tuning else {}
    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in rng.choice([32, 48, 64, 96, 128], size=count)]
    specs = []
    for n in sizes:
        src = (float(rng.uniform(0.3, 0.7)), float(rng.uniform(0.3, 0.7)), float(rng.uniform(0.1, 0.25)))
        specs.append((n, src, float(rng.uniform(0.05, 0.12)), float(rng.uniform(0.5, 2.0))))

    def make():
        sims = []
        for n, src, radius, buoy in specs:
            p = scene_params(default_params(), n, rel=rel, max_iterations=20000, omega=omegas.get(n),
                             sources=(src,), radius=radius, buoyancy=buoy)
            sims.append(MacSimulation3D(n, 1.0, p))
        return sims

    out = {"config": "batch", "scenes": count, "sizes": sizes, "cells": int(sum(n ** 3 for n in sizes)),
           "steps": steps, "tuned": bool(tuning)}
    for mode in ("separate", "batched"):
        sims = make()
        batch = Batch(sims) if mode == "batched" else None
        for _ in range(warmup):
            if batch:
                batch.advance(DT)
            else:
                for s in sims:
                    s.advance(DT)
        torch.cuda.synchronize()
        it0 = sum(s.total_iterations() for s in sims)
        start = torch.cuda.Event(enable_timing=True)
        if batch:
            stream = torch.cuda.ExternalStream(batch.stream())
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            for _ in range(steps):
                batch.advance(DT)
            end.record(stream)
            end.synchronize()
            ms = start.elapsed_time(end)
        else:
            streams = [torch.cuda.ExternalStream(s.stream()) for s in sims]
            start.record(streams[0])
            for st in streams[1:]:
                st.wait_event(start)
            for _ in range(steps):
                for s in sims:
                    s.advance(DT)
            ends = []
            for st in streams:
                e = torch.cuda.Event(enable_timing=True)
                e.record(st)
                ends.append(e)
            for e in ends:
                e.synchronize()
            ms = max(start.elapsed_time(e) for e in ends)
        sweeps = sum(s.total_iterations() for s in sims) - it0
        converged = all(s.last_projection().linear_solve.converged for s in sims)
        out[mode] = {"ms": ms, "scene_steps_per_s": count * steps / (ms * 1e-3),
                     "cell_steps_per_s": out["cells"] * steps / (ms * 1e-3), "sweeps": sweeps,
                     "all_converged": converged}
        if batch:
            batch.close()
        for s in sims:
            s.close()
    out["batched_vs_separate"] = out["separate"]["ms"] / out["batched"]["ms"]
    return out


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    m = sub.add_parser("mixed-projection")
    m.add_argument("--n", type=int, default=256)
    m.add_argument("--seed", type=int, default=1)
    m.add_argument("--rel", type=float, default=1e-8)
    b = sub.add_parser("batch")
    b.add_argument("--scenes", type=int, default=48)
    b.add_argument("--steps", type=int, default=100)
    b.add_argument("--warmup", type=int, default=3)
    b.add_argument("--seed", type=int, default=11)
    b.add_argument("--tuning", default=None, help="JSON table written by vapor_b200.autotune")
    args = ap.parse_args()
    if args.cmd == "mixed-projection":
        print(json.dumps(mixed_projection(n=args.n, seed=args.seed, rel=args.rel)))
    else:
        table = json.load(open(args.tuning)) if args.tuning else None
        print(json.dumps(batch_scenes(count=args.scenes, seed=args.seed, steps=args.steps, warmup=args.warmup,
                                      tuning=table)))


if __name__ == "__main__":
    main()
