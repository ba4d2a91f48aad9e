"""Headless diagnostics of the MAC 3D smoke step: the Reflection / MacCormack
comparison of the reference's diagnostic harness
(tests/ReflectionComparison.hpp:9-75), run on the device.

  python -m vapor_b200.diagnostics compare-reflection [--n 64 --frames 120 --iterations 40 --out DIR
                                                      --image 960]

For each of the four variants (Reflection with semi-Lagrangian or MacCormack
velocity and smoke) the scene of the harness is stepped at 60 frames per
second; every 60th frame and the last one print the harness's metric line
(mass, gradient and square per mass, rms and max divergence, smoke cells,
CFL and boundary fallbacks, max CFL; computed on the device by
vapor_mac3d_comparison_metrics) and write the raw density as
DIR/v<variant>_f<frame>.density: n^3 little-endian FP32 values, x fastest,
exactly the bytes the harness writes, and its image as
DIR/v<variant>_f<frame>.ppm: the headless CUDA ray-march of the density
(vapor_mac3d_render, the reference's volume shader and camera) in place of
the harness's OpenGL render.
"""
import argparse
import os

import numpy as np

from . import MacSimulation3D, default_params


def write_ppm(path, rgb):
    """The harness's image file: binary PPM, 8-bit RGB, top row first
    (rgb is (height, width, 3) in [0, 1] with row 0 at the bottom, as the
    renderer writes it)."""
    img = np.clip(np.rint(np.asarray(rgb, np.float32)[::-1] * 255.0), 0, 255).astype(np.uint8)
    h, w = img.shape[:2]
    with open(path, "wb") as f:
        f.write(f"P6\n{w} {h}\n255\n".encode())
        f.write(img.tobytes())


def write_density(path, density):
    """The harness's raw dump: the density array's FP32 bytes, x fastest."""
    np.ascontiguousarray(density, dtype="<f4").tofile(path)


def read_density(path, n):
    return np.fromfile(path, dtype="<f4").reshape(n, n, n)


def harness_params(variant, iterations):
    """The comparison scene (ReflectionComparison.hpp:11-21)."""
    p = default_params()
    p.reflection = 1
    p.mac_cormack_vel = int((variant & 1) != 0)
    p.mac_cormack_smoke = int((variant & 2) != 0)
    p.emitter_radius = 0.04
    p.source_strength = 1.0
    p.buoyancy = 0.8
    p.smoke_decay = 0.3007525
    p.project_iterations = iterations
    p.sor_omega = 1.9
    return p


def metric_line(variant, p, frame, m):
    return (f"compare variant={variant} mcV={p.mac_cormack_vel} mcD={p.mac_cormack_smoke} frame={frame} "
            f"mass={m['mass']:.6g} grad_per_mass={m['grad_per_mass']:.6g} "
            f"square_per_mass={m['square_per_mass']:.6g} rms_div={m['rms_div']:.6g} max_div={m['max_div']:.6g} "
            f"smoke_cells={m['smoke_cells']} smoke_cfl_fallback={m['cfl_fallback']} "
            f"smoke_boundary_fallback={m['boundary_fallback']} smoke_max_cfl={m['max_cfl']:.6g}")


def compare_reflection(n=64, frames=120, iterations=40, out=None, image_size=960):
    """Runs the four variants; returns their metric records. With `out`, every
    reported frame also writes the raw density and the harness's ray-marched
    image (image_size^2 pixels, 0: none) as .density and .ppm files."""
    from .abi import RenderParams
    records = []
    if out:
        os.makedirs(out, exist_ok=True)
    for variant in range(4):
        p = harness_params(variant, iterations)
        sim = MacSimulation3D(n, 1.0, p)
        for frame in range(1, frames + 1):
            sim.advance(1.0 / 60.0)
            if frame % 60 != 0 and frame != frames:
                continue
            m = sim.comparison_metrics(60.0)
            records.append({"variant": variant, "frame": frame, **m})
            print(metric_line(variant, p, frame, m), flush=True)
            if out:
                base = os.path.join(out, f"v{variant}_f{frame}")
                write_density(base + ".density", sim.download()[0])
                if image_size:
                    write_ppm(base + ".ppm", sim.render(RenderParams.harness(image_size, image_size)))
        sim.close()
    return records


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("compare-reflection")
    c.add_argument("--n", type=int, default=64)
    c.add_argument("--frames", type=int, default=120)
    c.add_argument("--iterations", type=int, default=40)
    c.add_argument("--out", default="reflection-comparison")
    c.add_argument("--image", type=int, default=960, help="image size in pixels (0: no images)")
    args = ap.parse_args()
    compare_reflection(args.n, args.frames, args.iterations, args.out, args.image)


if __name__ == "__main__":
    main()
