"""Learned warm start for the pressure solve: network handle, training from
plain-solver plume rollouts, and the sweep-count comparison.

The network is the library's 3-level 3D U-Net (16/32/64 channels, 3x3x3
convolutions on tcgen05 tensor cores, BF16 weights and activations, FP32
accumulation). It maps the RMS-normalized right-hand side of a projection to
the shape of the pressure; the projection scales the prediction by the
Galerkin condition and then runs its usual solver from it to the same
tolerance, so the plain solver remains both the fallback and the judge.

  python -m vapor_b200.learned train --out weights.npy [--n 128 --rollouts 8 --steps 100]
  python -m vapor_b200.learned compare --weights weights.npy [--n 256 --steps 4]
"""
import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import MacSimulation3D, check, default_params, library
from .plume import DT, scene_params, swirl_fields, training_scene

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "warm_start_unet.npy")


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
    else:
        net = WarmStartNet.load(args.weights)
        print(json.dumps(compare(net, n=args.n, warmup=args.warmup, steps=args.steps)))


if __name__ == "__main__":
    main()
