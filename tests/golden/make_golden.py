"""Regenerates the golden fixtures in this folder (run in a checkout that has
the reference sources and the built oracle/_ref library; the fixtures are
committed so the GPU tests do not need the reference at run time).

  simulation_baselines.json
      The 16 diagnostics tuples of the reference's regression test
      (tests/SimulationTests.cpp:17-34 of taehwann/vapor), parsed from that file
      as text, with the run settings of tests/SimulationTests.cpp:105-136.
  reference_steps.npz
      Fields produced by the reference's own MacGridFluidSolver3D (built from its
      sources in oracle/_ref) for the resident-parity settings of
      tests/GraphicsSmokeTests.cpp:22-58 (9^3, box 1, r=.22, cz=.3, stir .5,
      20 iterations, 8 frames) over all 8 flag combinations, and for the
      baseline settings (8^3 and 12^3, 6 frames) over all 16 cases.

Usage: python tests/golden/make_golden.py <path/to/reference>
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle_lib import RefSim, default_params  # noqa: E402


def parse_baselines(path):
    text = open(path).read()
    block = text[text.index("const Baseline baselines[] = {"):]
    block = block[: block.index("};")]
    rows = re.findall(r"\{\s*(\d+),\s*(\d+),\s*(\d+),\s*([-\d.eE+]+),\s*([-\d.eE+]+),\s*([-\d.eE+]+),"
                      r"\s*([-\d.eE+]+),\s*([-\d.eE+]+)\s*\}", block)
    out = []
    for r in rows:
        out.append({"n": int(r[0]), "reflect": int(r[1]), "flags": int(r[2]),
                    "energy": float(r[3]), "max_velocity": float(r[4]), "divergence": float(r[5]),
                    "density_sum": float(r[6]), "weighted_density": float(r[7])})
    assert len(out) == 16, len(out)
    return out


def baseline_params(case):
    p = default_params()
    p.stir_strength = 0.0
    p.emitter_radius = 0.18
    p.emitter_center_z = 0.3
    p.mac_cormack_smoke = int(case["flags"] & 1 != 0)
    p.mac_cormack_vel = int(case["flags"] & 2 != 0)
    p.reflection = case["reflect"]
    p.project_iterations = 16
    return p


def resident_params(reflection, mc_vel, mc_smoke):
    p = default_params()
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = int(reflection), int(mc_vel), int(mc_smoke)
    p.emitter_radius, p.emitter_center_z, p.stir_strength, p.project_iterations = 0.22, 0.3, 0.5, 20
    return p


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_golden.py <reference checkout>")
    ref_root = sys.argv[1]
    baselines = parse_baselines(os.path.join(ref_root, "tests", "SimulationTests.cpp"))
    with open(os.path.join(HERE, "simulation_baselines.json"), "w") as f:
        json.dump({"source": "tests/SimulationTests.cpp:17-34 (taehwann/vapor)",
                   "settings": {"frames": 6, "dt": 1.0 / 60.0, "project_iterations": 16,
                                "emitter_radius": 0.18, "emitter_center_z": 0.3, "stir_strength": 0.0,
                                "box": 4.5, "relative_tolerance": 2e-5},
                   "cases": baselines}, f, indent=1)

    arrays = {}
    for reflection in (0, 1):
        for mc_vel in (0, 1):
            for mc_smoke in (0, 1):
                sim = RefSim(9, 1.0)
                sim.params = resident_params(reflection, mc_vel, mc_smoke)
                sim.reset()
                for _ in range(8):
                    assert sim.advance(1.0 / 60.0) == 0
                key = f"resident_r{reflection}_v{mc_vel}_s{mc_smoke}"
                for name, a in zip("duvw", sim.fields()):
                    arrays[f"{key}_{name}"] = a
    for case in baselines:
        sim = RefSim(case["n"])
        sim.params = baseline_params(case)
        for _ in range(6):
            assert sim.advance(1.0 / 60.0) == 0
        key = f"baseline_n{case['n']}_r{case['reflect']}_f{case['flags']}"
        for name, a in zip("duvw", sim.fields()):
            arrays[f"{key}_{name}"] = a
    np.savez_compressed(os.path.join(HERE, "reference_steps.npz"), **arrays)
    print("wrote", len(baselines), "baselines and", len(arrays), "arrays")


if __name__ == "__main__":
    main()
