"""Learned pressure components: network handle, training drivers and the
comparisons against the plain solver.

The network is the library's 3-level 3D U-Net (16/32/64 channels, 3x3x3
convolutions on tcgen05 tensor cores, BF16 weights and activations, FP32
accumulation). It maps the RMS-normalized right-hand side of a projection to
the shape of the pressure; the projection scales the prediction by the
Galerkin condition and then runs its usual solver from it to the same
tolerance, so the plain solver remains both the fallback and the arbiter of
convergence.

  python -m vapor_b200.learned train --out weights.npy [--n 128 --rollouts 8 --steps 100]
  python -m vapor_b200.learned compare --weights weights.npy [--n 256 --steps 4]
  python -m vapor_b200.learned train-coarse --out coarse.npy [--n 64 --rollouts 8 --steps 60]
  python -m vapor_b200.learned compare-fpcg --weights coarse.npy [--n 256 --steps 3]
  python -m vapor_b200.learned train-random --out coarse.npy [--n 64 --pairs 3000]
  python -m vapor_b200.learned train-onpolicy --init coarse.npy --out coarse.npy [--n 256 --rounds 4]
  python -m vapor_b200.learned bench-net [--n 64]

The same network also serves as the coarse-grid correction of the flexible
PCG solver (VAPOR_SOLVER_FPCG): applied on the grid coarsened 4x per axis to
the restricted residual, scaled by the Galerkin condition, prolonged and
smoothed. For that role it is trained at the coarse resolution (64^3 for a
256^3 solve): first on projections of seeded random velocity fields
(train-random), then on the coarse right-hand sides the solver actually feeds
it, logged during FPCG solves and solved on the coarse grid by the plain
solver (train-onpolicy).
"""
import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import MacSimulation3D, StageBackend, check, default_params, fpcg_sweeps_per_application, library
from .abi import SOLVER_FPCG, SOLVER_MIXED_REFINEMENT, LinearSolveOptions, ProjectionOptions
from .plume import DT, omega_for, scene_params, spectral_fields, swirl_fields, training_scene

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warm_start_unet.npy")
COARSE_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "coarse_unet.npy")


class WarmStartNet:
    """Handle of one U-Net (its own stream, parameters, Adam state)."""

    def __init__(self, seed=0, parameters=None):
        lib = library()
        h = C.c_void_p()
        check(lib.vapor_unet_create(C.byref(h)))
        self._h = h
        self.count = int(lib.vapor_unet_parameter_count())
        check(lib.vapor_unet_init(h, int(seed) & 0xFFFFFFFF))
        if parameters is not None:
            self.set_parameters(parameters)

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS):
        return cls(parameters=np.load(path))

    def save(self, path):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.save(path, self.parameters())

    @property
    def handle(self):
        return self._h

    def parameters(self):
        p = np.zeros(self.count, np.float32)
        check(library().vapor_unet_get_parameters(self._h, p.ctypes.data, self.count))
        return p

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.count:
            raise ValueError(f"expected {self.count} parameters, got {p.size}")
        check(library().vapor_unet_set_parameters(self._h, p.ctypes.data, self.count))

    def close(self):
        if getattr(self, "_h", None):
            library().vapor_unet_destroy(self._h)
            self._h = None

    __del__ = close


def _lr(k, total, lr0, lr1):
    return lr1 + 0.5 * (lr0 - lr1) * (1.0 + math.cos(math.pi * min(1.0, k / max(1, total))))


def make_scene(n, seed, rel=1e-6, max_iterations=20000, scene=None):
    """A plume simulation of the training distribution (seeded)."""
    sc = scene or training_scene(seed)
    params = scene_params(default_params(), n, rel=rel, max_iterations=max_iterations, sources=sc["sources"],
                          radius=sc["radius"], buoyancy=sc["buoyancy"])
    sim = MacSimulation3D(n, 1.0, params)
    sim.upload(*swirl_fields(n, sc["swirl_seed"]))
    return sim


def train(net, n=128, rollouts=8, steps=100, updates=1, lr=1e-3, lr_final=1e-4, seed=0, skip=2, log=None):
    """Online training on plain-solver rollouts: each step's last projection
    (right-hand side, converged pressure) is one pair; `updates` Adam steps
    per pair. Returns the loss history."""
    total = rollouts * max(0, steps - skip) * updates
    history, k = [], 0
    t0 = time.perf_counter()
    for r in range(rollouts):
        sim = make_scene(n, seed * 7919 + r)
        for s in range(steps):
            sim.advance(DT)
            if s < skip:  # the first steps start from rest: atypical pairs
                continue
            for _ in range(updates):
                loss = sim.train_warm_start(net, _lr(k, total, lr, lr_final))
                history.append(loss)
                k += 1
            if log and (s % 10 == 0 or s == steps - 1):
                log(json.dumps({"rollout": r, "step": s, "loss": history[-1], "pairs": len(history),
                                "elapsed_s": round(time.perf_counter() - t0, 1)}))
        sim.close()
    return history


def compare(net, n=128, warmup=10, steps=4, seed=12345, scene=None, rel=1e-6):
    """Sweeps and device time per step with and without the warm start on the
    same plume (two simulations advanced side by side). Returns a dict."""
    import torch
    out = {}
    for name, use in (("plain", False), ("learned", True)):
        sim = make_scene(n, seed, rel=rel, scene=scene)
        for _ in range(warmup):
            sim.advance(DT)
        if use:
            sim.set_warm_start(net)
            sim.advance(DT)  # builds the step graph with the network in it
        sim.synchronize()
        stream = torch.cuda.ExternalStream(sim.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        it0 = sim.total_iterations()
        e0.record(stream)
        for _ in range(steps):
            sim.advance(DT)
        e1.record(stream)
        e1.synchronize()
        r = sim.last_projection().linear_solve
        out[name] = {"sweeps_per_step": (sim.total_iterations() - it0) / steps,
                     "ms_per_step": e0.elapsed_time(e1) / steps,
                     "final_relative_residual": r.final_residual / max(r.initial_residual, 1e-300),
                     "converged": bool(r.converged)}
        if use:
            out[name]["loss"] = sim.evaluate_warm_start(net)
        sim.close()
    out["sweep_ratio"] = out["plain"]["sweeps_per_step"] / max(1e-9, out["learned"]["sweeps_per_step"])
    out["speedup"] = out["plain"]["ms_per_step"] / max(1e-9, out["learned"]["ms_per_step"])
    return out


def train_coarse(net, n=64, rollouts=8, steps=60, random_pairs=1, lr=1e-3, lr_final=1e-4, seed=0, skip=2,
                 log=None):
    """Trains the coarse-grid network at resolution n: each plume step's last
    projection, plus `random_pairs` projections of seeded spectral velocity
    fields per step (a stage with the mixed solver to relative 1e-6)."""
    total = rollouts * max(0, steps - skip) * (1 + random_pairs)
    stage = StageBackend(n, 1.0)
    stage.set_solver_kind(SOLVER_MIXED_REFINEMENT)
    opts = ProjectionOptions(DT, omega_for(n), LinearSolveOptions.defaults(
        max_iterations=20000, relative_tolerance=1e-6, absolute_tolerance=0.0))
    history, k = [], 0
    t0 = time.perf_counter()
    rng = np.random.default_rng(seed + 99991)
    for r in range(rollouts):
        sim = make_scene(n, seed * 7919 + r)
        for s in range(steps):
            sim.advance(DT)
            if s < skip:
                continue
            history.append(sim.train_warm_start(net, _lr(k, total, lr, lr_final)))
            k += 1
            for _ in range(random_pairs):
                slope = float(rng.uniform(-3.0, -1.0))
                u, v, w = spectral_fields(n, int(rng.integers(1 << 31)), slope=slope,
                                          gradient_fraction=float(rng.uniform(0.2, 1.0)))
                stage.project(u, v, w, opts, 6.0)
                history.append(stage.train_network(net, _lr(k, total, lr, lr_final)))
                k += 1
            if log and (s % 10 == 0 or s == steps - 1):
                log(json.dumps({"rollout": r, "step": s, "loss": float(np.mean(history[-(1 + random_pairs):])),
                                "pairs": len(history), "elapsed_s": round(time.perf_counter() - t0, 1)}))
        sim.close()
    stage.close()
    return history


def train_random(net, n=64, pairs=2000, slopes=(-3.0, 0.0), lr=1e-3, lr_final=1e-4, seed=0, log=None):
    """Trains the coarse-grid network on projections of seeded random velocity
    fields only (spectral slope drawn from `slopes`, random solenoidal and
    gradient mix): a broad right-hand-side distribution, so the network learns
    the coarse Poisson inverse rather than the shapes of one flow."""
    stage = StageBackend(n, 1.0)
    stage.set_solver_kind(SOLVER_MIXED_REFINEMENT)
    opts = ProjectionOptions(DT, omega_for(n), LinearSolveOptions.defaults(
        max_iterations=20000, relative_tolerance=1e-6, absolute_tolerance=0.0))
    rng = np.random.default_rng(seed + 424242)
    history = []
    t0 = time.perf_counter()
    for k in range(pairs):
        u, v, w = spectral_fields(n, int(rng.integers(1 << 31)), slope=float(rng.uniform(*slopes)),
                                  gradient_fraction=float(rng.uniform(0.2, 1.0)))
        stage.project(u, v, w, opts, 6.0)
        history.append(stage.train_network(net, _lr(k, pairs, lr, lr_final)))
        if log and (k % 100 == 0 or k == pairs - 1):
            log(json.dumps({"pair": k, "loss": float(np.mean(history[-50:])),
                            "elapsed_s": round(time.perf_counter() - t0, 1)}))
    stage.close()
    return history


def train_onpolicy(net, n=256, rounds=4, warmup=3, steps=3, capacity=512, random_per_record=0.25, lr=3e-4,
                   lr_final=3e-5, seed=0, log=None):
    """Fine-tunes the coarse-grid network on the inputs it actually receives:
    each round runs seeded plume steps at n with the FPCG solver and the
    current network, logging every coarse right-hand side ((n/4)^3), then
    solves each logged right-hand side on the coarse grid with the plain
    mixed-precision solver and takes one Adam step on the pair; a fraction of
    random spectral pairs keeps the network general."""
    import torch
    nc = n // 4
    stage = StageBackend(nc, 1.0)
    stage.set_solver_kind(SOLVER_MIXED_REFINEMENT)
    opts = ProjectionOptions(DT, omega_for(nc), LinearSolveOptions.defaults(
        max_iterations=20000, relative_tolerance=1e-6, absolute_tolerance=0.0))
    buf = torch.zeros((capacity, nc ** 3), dtype=torch.float32, device="cuda")
    counter = torch.zeros(1, dtype=torch.int32, device="cuda")
    rng = np.random.default_rng(seed + 777)
    history, k = [], 0
    total = rounds * capacity * (1 + random_per_record)
    t0 = time.perf_counter()
    for rnd in range(rounds):
        sc = training_scene(seed * 7919 + 1000 + rnd)
        p = scene_params(default_params(), n, rel=1e-6, max_iterations=20000, sources=sc["sources"],
                         radius=sc["radius"], buoyancy=sc["buoyancy"])
        p.solver_kind = SOLVER_FPCG
        sim = MacSimulation3D(n, 1.0, p)
        sim.upload(*swirl_fields(n, sc["swirl_seed"]))
        sim.set_preconditioner(net)
        for _ in range(warmup):
            sim.advance(DT)
        counter.zero_()
        sim.synchronize()
        sim.set_coarse_log(buf.data_ptr(), capacity, counter.data_ptr())
        for _ in range(steps):
            sim.advance(DT)
        sim.synchronize()
        sim.set_coarse_log(None, 0, None)
        its = sim.last_projection().linear_solve.iterations
        sim.set_preconditioner(None)
        sim.close()
        count = min(int(counter.item()), capacity)
        for i in rng.permutation(count):
            stage.solve_rhs(buf[int(i)].data_ptr(), opts)
            history.append(stage.train_network(net, _lr(k, total, lr, lr_final)))
            k += 1
            if rng.random() < random_per_record:
                u, v, w = spectral_fields(nc, int(rng.integers(1 << 31)), slope=float(rng.uniform(-3.0, 0.0)),
                                          gradient_fraction=float(rng.uniform(0.2, 1.0)))
                stage.project(u, v, w, opts, 6.0)
                history.append(stage.train_network(net, _lr(k, total, lr, lr_final)))
                k += 1
        if log:
            log(json.dumps({"round": rnd, "records": count, "last_cg_iterations": its,
                            "loss": float(np.mean(history[-50:])) if history else None,
                            "elapsed_s": round(time.perf_counter() - t0, 1)}))
    stage.close()
    return history


def compare_fpcg(net, n=256, warmup=4, steps=3, seed=2024, rel=1e-6, phases=False,
                 arms=("sor", "fpcg", "fpcg_learned")):
    """Per-step sweeps/iterations and device time on the benchmark plume for
    the plain mixed-precision red-black SOR, FPCG with the smoothing-only
    preconditioner, and FPCG with the learned coarse-grid correction."""
    import torch
    out = {}
    for name, kind, use in (("sor", SOLVER_MIXED_REFINEMENT, False), ("fpcg", SOLVER_FPCG, False),
                            ("fpcg_learned", SOLVER_FPCG, True)):
        if name not in arms:
            continue
        p = scene_params(default_params(), n, rel=rel, max_iterations=20000)
        p.solver_kind = kind
        sim = MacSimulation3D(n, 1.0, p)
        sim.upload(*swirl_fields(n, seed))
        if use:
            sim.set_preconditioner(net)
        for _ in range(warmup):
            sim.advance(DT)
        sim.synchronize()
        stream = torch.cuda.ExternalStream(sim.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        it0 = sim.total_iterations()
        e0.record(stream)
        for _ in range(steps):
            sim.advance(DT)
        e1.record(stream)
        e1.synchronize()
        r = sim.last_projection().linear_solve
        its = (sim.total_iterations() - it0) / steps
        out[name] = {"iterations_per_step": its, "ms_per_step": e0.elapsed_time(e1) / steps,
                     "final_relative_residual": r.final_residual / max(r.initial_residual, 1e-300),
                     "converged": bool(r.converged)}
        if phases:
            sim.set_timing(True)
            sim.advance(DT)
            sim.synchronize()
            t = sim.timings()
            out[name]["phases_ms"] = {k: round(v["ms"], 3) for k, v in t.items() if v["ms"] > 0}
            out[name]["phase_launches"] = {k: v["launches"] for k, v in t.items() if v["launches"] > 0}
            sim.set_timing(False)
        if kind == SOLVER_FPCG:
            # each CG step applies the preconditioner once (2 x smoothing
            # red+black sweeps), plus one application per projection before
            # the loop (2 per step)
            out[name]["sweeps_per_step"] = fpcg_sweeps_per_application() * (its + 2)
        else:
            out[name]["sweeps_per_step"] = its
        sim.close()
    if "sor" in out:
        for name in ("fpcg", "fpcg_learned"):
            if name in out:
                out[name]["sweep_ratio_vs_sor"] = out["sor"]["sweeps_per_step"] / max(1e-9, out[name]["sweeps_per_step"])
                out[name]["speedup_vs_sor"] = out["sor"]["ms_per_step"] / max(1e-9, out[name]["ms_per_step"])
    if "fpcg" in out and "fpcg_learned" in out:
        out["learned_gain_vs_fpcg"] = out["fpcg"]["ms_per_step"] / max(1e-9, out["fpcg_learned"]["ms_per_step"])
    return out


def bench_net(n=64, reps=20, seed=0):
    """Times the raw network forward on an n^3 grid (16 BF16 input channels,
    FP32 output; each call synchronizes). Returns ms per call and TFLOP/s of
    the ten 3x3x3 convolutions."""
    import torch
    net = WarmStartNet(seed=seed)
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.zeros((n ** 3, 16), dtype=torch.bfloat16, device="cuda")
    x[:, 0] = torch.randn(n ** 3, generator=g, device="cuda").to(torch.bfloat16)
    out = torch.zeros(n ** 3, dtype=torch.float32, device="cuda")
    lib = library()
    for _ in range(3):
        check(lib.vapor_unet_forward_features(net.handle, n, x.data_ptr(), out.data_ptr()))
    t0 = time.perf_counter()
    for _ in range(reps):
        check(lib.vapor_unet_forward_features(net.handle, n, x.data_ptr(), out.data_ptr()))
    ms = (time.perf_counter() - t0) * 1e3 / reps
    macs = 27 * n ** 3 * (16 * 16 * 2 + 48 * 16 + 16 * 16 + (16 * 32 + 32 * 32 + 96 * 32 + 32 * 32) / 8.0 +
                          (32 * 64 + 64 * 64) / 64.0)
    return {"n": n, "ms_per_forward": ms, "conv_tflops": 2 * macs / (ms * 1e-3) / 1e12}


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train")
    t.add_argument("--out", default=DEFAULT_WEIGHTS)
    t.add_argument("--init", default=None, help="start from these weights")
    t.add_argument("--n", type=int, default=128)
    t.add_argument("--rollouts", type=int, default=8)
    t.add_argument("--steps", type=int, default=100)
    t.add_argument("--updates", type=int, default=1)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--lr-final", type=float, default=1e-4)
    t.add_argument("--seed", type=int, default=0)
    tc = sub.add_parser("train-coarse")
    tc.add_argument("--out", default=COARSE_WEIGHTS)
    tc.add_argument("--init", default=None)
    tc.add_argument("--n", type=int, default=64)
    tc.add_argument("--rollouts", type=int, default=8)
    tc.add_argument("--steps", type=int, default=60)
    tc.add_argument("--random-pairs", type=int, default=1)
    tc.add_argument("--lr", type=float, default=1e-3)
    tc.add_argument("--lr-final", type=float, default=1e-4)
    tc.add_argument("--seed", type=int, default=0)
    tr = sub.add_parser("train-random")
    tr.add_argument("--out", default=COARSE_WEIGHTS)
    tr.add_argument("--init", default=None)
    tr.add_argument("--n", type=int, default=64)
    tr.add_argument("--pairs", type=int, default=2000)
    tr.add_argument("--slope-min", type=float, default=-3.0)
    tr.add_argument("--slope-max", type=float, default=0.0)
    tr.add_argument("--lr", type=float, default=1e-3)
    tr.add_argument("--lr-final", type=float, default=1e-4)
    tr.add_argument("--seed", type=int, default=0)
    op = sub.add_parser("train-onpolicy")
    op.add_argument("--out", default=COARSE_WEIGHTS)
    op.add_argument("--init", default=COARSE_WEIGHTS)
    op.add_argument("--n", type=int, default=256)
    op.add_argument("--rounds", type=int, default=4)
    op.add_argument("--steps", type=int, default=3)
    op.add_argument("--capacity", type=int, default=512)
    op.add_argument("--lr", type=float, default=3e-4)
    op.add_argument("--lr-final", type=float, default=3e-5)
    op.add_argument("--seed", type=int, default=0)
    cf = sub.add_parser("compare-fpcg")
    cf.add_argument("--weights", default=COARSE_WEIGHTS)
    cf.add_argument("--n", type=int, default=256)
    cf.add_argument("--warmup", type=int, default=4)
    cf.add_argument("--steps", type=int, default=3)
    cf.add_argument("--phases", action="store_true", help="add a per-phase breakdown of one eager step")
    cf.add_argument("--arms", default="sor,fpcg,fpcg_learned")
    cf.add_argument("--seed", type=int, default=2024)
    bn = sub.add_parser("bench-net")
    bn.add_argument("--n", type=int, default=64)
    bn.add_argument("--reps", type=int, default=20)
    c = sub.add_parser("compare")
    c.add_argument("--weights", default=DEFAULT_WEIGHTS)
    c.add_argument("--n", type=int, default=128)
    c.add_argument("--warmup", type=int, default=10)
    c.add_argument("--steps", type=int, default=4)
    args = ap.parse_args()
    if args.cmd == "train":
        net = WarmStartNet.load(args.init) if args.init else WarmStartNet(seed=args.seed)
        hist = train(net, n=args.n, rollouts=args.rollouts, steps=args.steps, updates=args.updates, lr=args.lr,
                     lr_final=args.lr_final, seed=args.seed, log=print)
        net.save(args.out)
        tail = hist[-50:] if hist else [float("nan")]
        print(json.dumps({"saved": args.out, "pairs": len(hist), "final_loss_mean50": float(np.mean(tail))}))
    elif args.cmd == "train-coarse":
        net = WarmStartNet.load(args.init) if args.init else WarmStartNet(seed=args.seed)
        hist = train_coarse(net, n=args.n, rollouts=args.rollouts, steps=args.steps, random_pairs=args.random_pairs,
                            lr=args.lr, lr_final=args.lr_final, seed=args.seed, log=print)
        net.save(args.out)
        tail = hist[-50:] if hist else [float("nan")]
        print(json.dumps({"saved": args.out, "pairs": len(hist), "final_loss_mean50": float(np.mean(tail))}))
    elif args.cmd == "train-random":
        net = WarmStartNet.load(args.init) if args.init else WarmStartNet(seed=args.seed)
        hist = train_random(net, n=args.n, pairs=args.pairs, slopes=(args.slope_min, args.slope_max), lr=args.lr,
                            lr_final=args.lr_final, seed=args.seed, log=print)
        net.save(args.out)
        print(json.dumps({"saved": args.out, "pairs": len(hist), "final_loss_mean50": float(np.mean(hist[-50:]))}))
    elif args.cmd == "train-onpolicy":
        net = WarmStartNet.load(args.init)
        hist = train_onpolicy(net, n=args.n, rounds=args.rounds, steps=args.steps, capacity=args.capacity,
                              lr=args.lr, lr_final=args.lr_final, seed=args.seed, log=print)
        net.save(args.out)
        print(json.dumps({"saved": args.out, "pairs": len(hist),
                          "final_loss_mean50": float(np.mean(hist[-50:])) if hist else None}))
    elif args.cmd == "bench-net":
        print(json.dumps(bench_net(n=args.n, reps=args.reps)))
    elif args.cmd == "compare-fpcg":
        net = WarmStartNet.load(args.weights) if os.path.exists(args.weights) else WarmStartNet(seed=0)
        print(json.dumps(compare_fpcg(net, n=args.n, warmup=args.warmup, steps=args.steps, phases=args.phases,
                                      arms=tuple(args.arms.split(",")), seed=args.seed)))
    else:
        net = WarmStartNet.load(args.weights)
        print(json.dumps(compare(net, n=args.n, warmup=args.warmup, steps=args.steps)))


if __name__ == "__main__":
    main()
