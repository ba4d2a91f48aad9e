"""Regenerates mac2d_steps.npz and mac2d_refl_steps.npz: fields and
projection results of the reference's own MacGridFluidSolver2D and
ReflectionMacFluidSolver2D (src/solvers/mac2d/ of taehwann/vapor, built from
its sources into oracle/_ref/libvapor_ref2d.so by
`make -C oracle REF=<path/to/reference>`), so the GPU tests can pin the
device 2D solvers when the reference build is not at hand.

Cases of mac2d_steps.npz: the default-constructed solver's scene (simple and
midpoint reflection) from rest, 24 x 24 cells, box 1, 10 steps of 1/60 s; the
fields after steps 5 and 10 and every step's projection results.

Cases of mac2d_refl_steps.npz: the reflection solver's defaults with
semi-Lagrangian or MacCormack smoke, random stirring off or at strength 2,
24 x 24 cells, 10 steps of 1/60 s; smoke, u, v and pressure after steps 5 and
10, and the diagnostics after step 10.

Usage: python tests/golden/make_golden_2d.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle_lib import RefReflection2D, RefSim2D, ref2d_available  # noqa: E402
from vapor_b200.mac2d import plume_params_2d, reflection_default_params  # noqa: E402

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
    out = {}
    for mc in (0, 1):
        for stir in (0.0, 2.0):
            key = f"mc{mc}_stir{int(stir)}"
            p = reflection_default_params()
            p.mac_cormack_smoke = mc
            p.stir_strength = stir
            ref = RefReflection2D(N, p)
            for step in range(1, STEPS + 1):
                assert ref.advance(DT) == 0
                if step in (5, 10):
                    for name, a in zip(("smoke", "u", "v", "pressure"), ref.fields()):
                        out[f"{key}_s{step}_{name}"] = a
            d = ref.diagnostics()
            out[f"{key}_diagnostics"] = np.array([d.kinetic_energy, d.max_velocity, d.max_divergence], np.float32)
    np.savez_compressed(os.path.join(HERE, "mac2d_refl_steps.npz"), **out)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
