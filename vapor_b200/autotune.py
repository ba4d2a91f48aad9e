"""Autotuner for the red-black solve: per grid size, the SOR relaxation factor
(which sets the sweep count to a tolerance) and the z-planes per thread of
the colour-sweep kernel (its tile shape), both measured on the GPU.

  python -m vapor_b200.autotune --sizes 32,48,64,96,128 --out tuning.json

omega: for each candidate, sweeps of the mixed-precision solve to relative
residual 1e-6 of a plume-like projection (a seeded k^-5/3 spectral velocity)
are counted; the candidate with the fewest sweeps wins (ties: the smaller).
planes: a fixed 64-sweep solve is timed with CUDA events for planes 1, 2, 4,
8; the fastest wins. Neither choice changes results beyond the sweep count:
every solve still stops on the same FP64 residual test.
"""
import argparse
import json

from . import StageBackend, tune_sor_planes
from .abi import SOLVER_MIXED_REFINEMENT, LinearSolveOptions, ProjectionOptions
from .plume import spectral_fields

OMEGAS = (1.90, 1.93, 1.95, 1.96, 1.97, 1.975, 1.98, 1.985)
PLANES = (1, 2, 4, 8)


def _fields(n, seed):
    return spectral_fields(n, seed, slope=-5.0 / 3.0, gradient_fraction=0.5)


def tune_omega(n, seed=3, rel=1e-6):
    u, v, w = _fields(n, seed)
    stage = StageBackend(n, 1.0)
    stage.set_solver_kind(SOLVER_MIXED_REFINEMENT)
    sweeps = {}
    for om in OMEGAS:
        opts = ProjectionOptions(0.01, om, LinearSolveOptions.defaults(
            max_iterations=50000, relative_tolerance=rel, absolute_tolerance=0.0))
        r, _ = stage.project(u.copy(), v.copy(), w.copy(), opts, 6.0)
        sweeps[om] = r.linear_solve.iterations if r.linear_solve.converged else 10 ** 9
    best = min(OMEGAS, key=lambda o: (sweeps[o], o))
    return best, sweeps


def tune_planes(n, seed=4, sweeps=64, repeats=3):
    import torch
    u, v, w = _fields(n, seed)
    dev = [torch.from_numpy(a.copy()).cuda() for a in (u, v, w)]
    opts = ProjectionOptions(0.01, 1.95, LinearSolveOptions.defaults(
        max_iterations=sweeps, fixed_iterations=1, relative_tolerance=0.0, absolute_tolerance=0.0))
    times = {}
    for planes in PLANES:
        if planes > n:
            continue
        tune_sor_planes(n, planes)
        stage = StageBackend(n, 1.0)
        stage.set_solver_kind(SOLVER_MIXED_REFINEMENT)
        best = None
        for _ in range(repeats):
            work = [d.clone() for d in dev]
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            stage.project_device(*[t.data_ptr() for t in work], opts, 6.0)
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        times[planes] = best
        stage.close()
    tune_sor_planes(n, 0)
    return min(times, key=times.get), times


def tune(sizes, log=None):
    table = {}
    for n in sizes:
        om, sweeps = tune_omega(n)
        planes, times = tune_planes(n)
        table[str(n)] = {"omega": om, "sor_planes": planes, "sweeps": {str(k): v for k, v in sweeps.items()},
                         "plane_ms": {str(k): v for k, v in times.items()}}
        if log:
            log(json.dumps({"n": n, **table[str(n)]}))
    return table


def apply(table):
    """Installs the tuned tile shapes; returns {n: omega}."""
    omegas = {}
    for key, entry in table.items():
        tune_sor_planes(int(key), int(entry["sor_planes"]))
        omegas[int(key)] = float(entry["omega"])
    return omegas


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="32,48,64,96,128")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    table = tune([int(x) for x in args.sizes.split(",")], log=print)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(table, f, indent=1)


if __name__ == "__main__":
    main()
