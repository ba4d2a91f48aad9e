"""Seeded synthetic plume scenes for the MAC 3D step.

The benchmark scene is the Reflection + MacCormack two-source plume: box 1,
dt 0.01, profile sources min(1, 3 exp(-3.5 (d/r)^2)) of radius .08 at
(x, y, z) = (.3, .5, .15) and (.7, .5, .15) (z up), buoyancy 1.5, smoke decay
.995 per step, no kick or stir, initial velocity a seeded swirl of 8 Gaussian
vortices (amplitude .5). Projections solve to a relative residual (relative
divergence) with the mixed-precision red-black SOR.

training_scene() draws the per-rollout variations used to generate the
learned warm start's (divergence, pressure) pairs: source positions, radius
and buoyancy from seeded ranges.
"""
import numpy as np

DT = 0.01
# SOR relaxation per grid size for the floor-6 red-black sweep (chosen by
# measured sweep counts to rel 1e-6 on this plume; larger grids want omega
# closer to 2).
OMEGA = {32: 1.95, 64: 1.95, 96: 1.96, 128: 1.97, 192: 1.975, 256: 1.98}


def omega_for(n, override=None):
    if override:
        return override
    keys = sorted(OMEGA)
    return OMEGA[min(keys, key=lambda k: abs(k - n))]


def solve_options(rel, max_iterations, interval=8):
    from .abi import LinearSolveOptions
    return LinearSolveOptions.defaults(max_iterations=max_iterations, residual_check_interval=interval,
                                       relative_tolerance=rel, absolute_tolerance=0.0, fixed_iterations=0)


def scene_params(p, n, rel=1e-6, max_iterations=20000, omega=None, sources=((0.3, 0.5, 0.15), (0.7, 0.5, 0.15)),
                 radius=0.08, buoyancy=1.5, interval=8):
    """Fill MacParams `p` with the plume scene (returns p)."""
    from .abi import SOLVER_MIXED_REFINEMENT
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = 1, 1, 1
    p.buoyancy, p.buoyancy_split, p.cfl_mc = buoyancy, 0.5, 3.0
    p.smoke_decay = 0.5  # factor clamp(1 - .5 * .01) = .995 per step
    p.emitter_radius, p.source_strength = radius, 1.0
    p.emitter_center_x, p.emitter_center_y, p.emitter_center_z = sources[0]
    p.emitter_count = len(sources)
    if len(sources) > 1:
        p.emitter2_center_x, p.emitter2_center_y, p.emitter2_center_z = sources[1]
    p.emitter_profile = 1
    p.emitter_kick_multiplier, p.stir_strength = 0.0, 0.0
    p.sor_omega = omega_for(n, omega)
    p.use_solve_options = 1
    p.solver_kind = SOLVER_MIXED_REFINEMENT
    p.solve = solve_options(rel, max_iterations, interval)
    return p


def training_scene(seed):
    """Per-rollout scene variation: two sources, radius .05-.12, buoyancy .5-2."""
    rng = np.random.default_rng(seed)
    x1, x2 = rng.uniform(0.2, 0.45), rng.uniform(0.55, 0.8)
    y1, y2 = rng.uniform(0.3, 0.7, size=2)
    z1, z2 = rng.uniform(0.1, 0.25, size=2)
    return {"sources": ((x1, y1, z1), (x2, y2, z2)), "radius": float(rng.uniform(0.05, 0.12)),
            "buoyancy": float(rng.uniform(0.5, 2.0)), "swirl_seed": int(rng.integers(1 << 31))}


def swirl_fields(n, seed, amplitude=0.5, vortices=8, sigma=0.08):
    """Seeded swirl: sum of Gaussian vortices (random centre and axis) on the
    MAC faces, normal velocity zero on the walls; density zero. Returns
    [density, u, v, w] in the MAC layout (z, y, x)."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.2, 0.8, size=(vortices, 3))
    axes = rng.normal(size=(vortices, 3))
    axes /= np.linalg.norm(axes, axis=1, keepdims=True)
    h = 1.0 / n

    def comp(c, shape):
        # separable coordinates broadcast over (z, y, x); each vortex adds
        # amplitude * (a x r)_c / sigma * exp(-|r|^2 / (2 sigma^2)) (the same
        # elementwise operations as a full-grid evaluation, plane by plane)
        axis = [(np.arange(s, dtype=np.float64) + (0.0 if c == d else 0.5)) * h
                for d, s in zip((2, 1, 0), shape)]  # z, y, x coordinates
        zs, ys, xs = axis
        out = np.zeros(shape)
        for k in range(vortices):
            a = axes[k]
            rx = (xs - centres[k, 0])[None, :]
            ry = (ys - centres[k, 1])[:, None]
            for iz in range(shape[0]):
                rz = zs[iz] - centres[k, 2]
                g = np.exp(-(rx ** 2 + ry ** 2 + rz ** 2) / (2 * sigma ** 2))
                if c == 0:
                    cr = a[1] * rz - a[2] * ry
                elif c == 1:
                    cr = a[2] * rx - a[0] * rz
                else:
                    cr = a[0] * ry - a[1] * rx
                out[iz] += amplitude * cr / sigma * g
        return out.astype(np.float32)

    u = comp(0, (n, n, n + 1))
    v = comp(1, (n, n + 1, n))
    w = comp(2, (n + 1, n, n))
    u[:, :, 0] = u[:, :, -1] = 0
    v[:, 0, :] = v[:, -1, :] = 0
    w[0] = w[-1] = 0
    return [np.zeros((n, n, n), np.float32), u, v, w]


def spectral_fields(n, seed, slope=-5.0 / 3.0, amplitude=1.0, gradient_fraction=0.5):
    """Seeded random velocity with energy spectrum ~ k^slope: a solenoidal
    part plus a gradient part (weight `gradient_fraction`), on the MAC faces,
    walls zeroed. Returns (u, v, w) in the MAC layout (z, y, x)."""
    rng = np.random.default_rng(seed)
    m = n + 1
    k = np.fft.fftfreq(m) * m
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    kk[0, 0, 0] = 1.0
    amp = kk ** ((slope - 2.0) / 2.0)
    amp[0, 0, 0] = 0.0
    comps = []
    for _ in range(3):
        noise = rng.standard_normal((m, m, m)) + 1j * rng.standard_normal((m, m, m))
        comps.append(noise * amp)
    # Helmholtz split in Fourier space: gradient part = k (k . a) / |k|^2
    dot = (kx * comps[0] + ky * comps[1] + kz * comps[2]) / kk ** 2
    grad = [kx * dot, ky * dot, kz * dot]
    sol = [c - g for c, g in zip(comps, grad)]
    fields = [np.real(np.fft.ifftn((1 - gradient_fraction) * s_ + gradient_fraction * g)) for s_, g in zip(sol, grad)]
    scale = amplitude / max(1e-30, max(float(np.abs(f).max()) for f in fields))
    u = (fields[0][:n, :n, :] * scale).astype(np.float32)
    v = (fields[1][:n, :, :n] * scale).astype(np.float32)
    w = (fields[2][:, :n, :n] * scale).astype(np.float32)
    u[:, :, 0] = u[:, :, -1] = 0
    v[:, 0, :] = v[:, -1, :] = 0
    w[0] = w[-1] = 0
    return u, v, w
