"""Regenerates mac2d_steps.npz: fields and projection results of the
reference's own MacGridFluidSolver2D (src/solvers/mac2d/ of taehwann/vapor,
built from its sources into oracle/_ref/libvapor_ref2d.so by
`make -C oracle REF=<path/to/reference>`), so the GPU tests can pin the
device 2D solver when the reference build is not at hand.

Cases: the default-constructed solver's scene (simple and midpoint
reflection) from rest, 24 x 24 cells, box 1, 10 steps of 1/60 s; the fields
after steps 5 and 10 and every step's projection results.

Usage: python tests/golden/make_golden_2d.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle_lib import RefSim2D, ref2d_available  # noqa: E402
from vapor_b200.mac2d import plume_params_2d  # noqa: E402

N, BOX, STEPS, DT = 24, 1.0, 10, 1.0 / 60.0


def main():
    if not ref2d_available():
        raise SystemExit("oracle/_ref/libvapor_ref2d.so missing: make -C oracle REF=<path/to/reference>")
    out = {}
    for reflection in (0, 1):
        p = plume_params_2d()
        p.reflection = reflection
        ref = RefSim2D(N, BOX, p)
        proj = []
        for step in range(1, STEPS + 1):
            assert ref.advance(DT) == 0
            for r in (ref.last_projection(), ref.midpoint_projection()):
                ls = r.linear_solve
                proj.append([ls.iterations, ls.converged, ls.initial_residual, ls.final_residual,
                             r.divergence_before, r.divergence_after, r.removed_rhs_mean])
            if step in (5, 10):
                for name, a in zip(("density", "u", "v"), ref.fields()):
                    out[f"r{reflection}_s{step}_{name}"] = a
        out[f"r{reflection}_projections"] = np.array(proj, np.float64)
    np.savez_compressed(os.path.join(HERE, "mac2d_steps.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
