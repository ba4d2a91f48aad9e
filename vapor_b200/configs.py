"""Measurement drivers for the configurations beside the headline benchmark.

  python -m vapor_b200.configs mixed-projection [--n 256 --seed 1 --rel 1e-8]

mixed-projection: one staged projection of a seeded random velocity field
(solenoidal plus gradient parts, energy spectrum ~ k^-5/3) in a closed box
with a seeded sphere obstacle (radius .1-.2), solved with FP32 red-black SOR
sweeps under FP64 residual checks and FP64 iterative refinement to relative
divergence 1e-8. Reports the device time, sweeps, the FP64-verified residual
and, with --fp64-check, the error of the projected velocity and pressure
against the FP64 oracle (CPU, so use it at small n; the oracle library is
test infrastructure and must have been built).
"""
import argparse
import json
import os
import sys

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


def mixed_projection(n=256, seed=1, rel=1e-8, dt=0.01, fp64_check=False, repeats=2):
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
    if fp64_check:
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        sys.path.insert(0, os.path.join(root, "tests"))
        from oracle_lib import oracle_project
        o64 = LinearSolveOptions.defaults(max_iterations=200000, relative_tolerance=rel, absolute_tolerance=0.0)
        st, r64, u64, v64, w64, p64 = oracle_project(n, 1.0, u, v, w, dt, omega_for(n), 6.0, o64, solver_kind=0,
                                                     dtype=np.float64, solid=mask)
        got = [t.cpu().numpy() for t in work] + [p_dev.cpu().numpy()]
        errs = {}
        for name, g, ref in zip(("u", "v", "w", "p"), got, (u64, v64, w64, p64)):
            errs[name] = float(np.abs(g.astype(np.float64) - ref).max() / max(1e-300, np.abs(ref).max()))
        out["fp64_oracle"] = {"status": st, "converged": bool(r64.linear_solve.converged),
                              "max_relative_error": errs}
    return out


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    m = sub.add_parser("mixed-projection")
    m.add_argument("--n", type=int, default=256)
    m.add_argument("--seed", type=int, default=1)
    m.add_argument("--rel", type=float, default=1e-8)
    m.add_argument("--fp64-check", action="store_true")
    args = ap.parse_args()
    print(json.dumps(mixed_projection(n=args.n, seed=args.seed, rel=args.rel, fp64_check=args.fp64_check)))


if __name__ == "__main__":
    main()
