"""The benchmark's named scene configurations as parity cases.

Simple CPU configuration (64^3, h = 1/64, dt .01, semi-Lagrangian, profile
source at (.5, .5, .15) of radius .08, buoyancy 1 along +z, no decay, seeded
N(0, .01) initial velocity, red-black SOR omega 1.7 to relative residual
1e-5): the first steps bit for bit against the FP32 oracle (the reference's
CPU arithmetic, whose SOR is red-black too), then the full 100 steps on the
GPU (mixed-precision form of the sweep) against the properties the
configuration must keep.

Reflection + MacCormack plume (two profile sources, seeded swirl, buoyancy
1.5, decay .995 per step, mixed-precision red-black SOR to 1e-6): steps at 32^3
bit for bit against the oracle's mixed-precision solve; the 128^3 and 256^3
runs of this scene are the benchmark's.
"""
import numpy as np
import pytest

import vapor_b200 as vb
from oracle_lib import OracleSim
from vapor_b200.abi import SOLVER_MIXED_REFINEMENT, SOLVER_RED_BLACK_SOR, LinearSolveOptions, field_shapes
from vapor_b200.plume import DT, scene_params, swirl_fields

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def simple_cpu_params():
    p = vb.default_params()
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = 0, 0, 0
    p.buoyancy, p.buoyancy_split, p.smoke_decay = 1.0, 0.5, 0.0
    p.emitter_radius, p.source_strength = 0.08, 1.0
    p.emitter_center_x, p.emitter_center_y, p.emitter_center_z = 0.5, 0.5, 0.15
    p.emitter_count, p.emitter_profile = 1, 1
    p.emitter_kick_multiplier, p.stir_strength = 0.0, 0.0
    p.sor_omega = 1.7
    p.use_solve_options = 1
    p.solver_kind = SOLVER_RED_BLACK_SOR
    p.solve = LinearSolveOptions.defaults(max_iterations=4000, relative_tolerance=1e-5, absolute_tolerance=0.0)
    return p


def noise_velocity(n, seed, sigma=0.01):
    """density 0; u, v, w ~ N(0, sigma) with the wall-normal faces zeroed."""
    rng = np.random.default_rng(seed)
    d, u, v, w = [np.zeros(s, np.float32) for s in field_shapes(n)]
    u[...] = rng.normal(0.0, sigma, u.shape)
    v[...] = rng.normal(0.0, sigma, v.shape)
    w[...] = rng.normal(0.0, sigma, w.shape)
    u[:, :, 0] = u[:, :, n] = 0.0
    v[:, 0, :] = v[:, n, :] = 0.0
    w[0] = w[n] = 0.0
    return [d, u, v, w]


def test_simple_cpu_configuration_first_steps_match_oracle():
    n, p = 64, simple_cpu_params()
    fields = noise_velocity(n, seed=64)
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*fields)
    ref = OracleSim(n, 1.0)
    ref.params = p
    ref.set_fields(*fields)
    for _ in range(3):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        got, want = sim.last_projection().linear_solve, ref.last_projection().linear_solve
        assert got.iterations == want.iterations and got.converged and want.converged
    for x, y in zip(sim.download(), ref.fields()):
        assert bits_equal(x, y)


def test_simple_cpu_configuration_100_steps():
    """All 100 steps with the mixed-precision form of the same red-black SOR
    (FP32 sweeps, FP64 residual and re-centring): from the eighth step on, the
    plain FP32 sweep no longer reaches relative residual 1e-5 within 4000
    iterations on this grid (the GPU and the FP32 oracle agree bit for bit, so
    the reference's CPU sweep stops there too); the mixed solve reaches it
    every step."""
    n, p = 64, simple_cpu_params()
    p.solver_kind = SOLVER_MIXED_REFINEMENT
    p.solve = LinearSolveOptions.defaults(max_iterations=20000, relative_tolerance=1e-5, absolute_tolerance=0.0)
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*noise_velocity(n, seed=64))
    for step in range(100):
        sim.advance(DT)
        ls = sim.last_projection().linear_solve
        assert ls.converged and ls.final_residual <= 1e-5 * ls.initial_residual, step
    d, u, v, w = sim.download()
    # FP32 trilinear weights can overshoot 1 by an ulp or two (the reference's
    # own plume test allows 1.00001)
    assert np.isfinite(d).all() and d.min() >= 0.0 and d.max() <= 1.00001
    assert all(np.isfinite(a).all() for a in (u, v, w))
    assert d.sum() > 0.0 and w.max() > 0.0  # the source fills and buoyancy lifts
    diag = sim.diagnostics()
    assert np.isfinite(diag.kinetic_energy) and diag.max_divergence < 1.0


def test_reflection_plume_scene_matches_oracle_mixed_solve():
    n = 32
    p = scene_params(vb.default_params(), n, rel=1e-6, max_iterations=20000)
    fields = [np.asarray(a, np.float32) for a in swirl_fields(n, seed=5)]
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*fields)
    ref = OracleSim(n, 1.0)
    ref.params = p
    ref.set_fields(*fields)
    for _ in range(4):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        got, want = sim.last_projection().linear_solve, ref.last_projection().linear_solve
        assert got.iterations == want.iterations and got.converged
        assert got.final_residual <= 1e-6 * got.initial_residual
    for x, y in zip(sim.download(), ref.fields()):
        assert bits_equal(x, y)


def test_reflection_plume_128_matches_oracle_and_fp64_error():
    """The Reflection-MacCormack plume configuration at its own size, 128^3:
    three steps with the mixed-precision solve to relative divergence 1e-6,
    bit for bit against the FP32 oracle with equal iteration counts; then one
    step from the GPU's state against the FP64 oracle (the same step in
    double), both solved to relative divergence 1e-10 so that the difference
    is the FP32 arithmetic, not two stopping iterates.

    The MacCormack limiter clamps to the 8 source values around the cell that
    contains the back-traced point, so where a trace ends within rounding of
    a cell face the two precisions clamp to different bounds: a handful of
    velocity samples differ by up to 4.3e-5 relative (1, 5 and 4 samples of
    u, v, w above 1e-5 at this size; the FP32 oracle shows the same). The
    test bounds the rms relative error by 1e-6, the samples above 1e-5 by
    1e-5 of the grid, and the max by 1e-4; the semi-Lagrangian step, which
    has no such switch, is held to 1e-5 at every sample by the next test."""
    n = 128
    p = scene_params(vb.default_params(), n, rel=1e-6, max_iterations=20000)
    fields = [np.asarray(a, np.float32) for a in swirl_fields(n, seed=5)]
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*fields)
    ref = OracleSim(n, 1.0)
    ref.params = p
    ref.set_fields(*fields)
    for _ in range(3):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        got, want = sim.last_projection().linear_solve, ref.last_projection().linear_solve
        assert got.iterations == want.iterations and got.converged
        assert got.final_residual <= 1e-6 * got.initial_residual
    state = sim.download()
    for x, y in zip(state, ref.fields()):
        assert bits_equal(x, y)
    tight = scene_params(vb.default_params(), n, rel=1e-10, max_iterations=40000)
    sim.set_parameters(tight)
    f64 = OracleSim(n, 1.0, dtype=np.float64)
    f64.params = tight
    f64.set_fields(*[x.astype(np.float64) for x in state])
    sim.advance(DT)
    assert sim.last_projection().linear_solve.converged
    assert f64.advance(DT) == 0
    errs = fp64_errors(sim.download(), f64.fields())
    print("128^3 plume step vs FP64 oracle (max, rms, samples above 1e-5):", errs)
    for name, (mx, rms, above) in errs.items():
        assert mx <= 1e-4 and rms <= 1e-6 and above <= 1e-5 * n ** 3, (name, errs)


def fp64_errors(got, want):
    """Per field: max and rms of |got - want| relative to max |want|, and the
    count of samples whose error exceeds 1e-5 of it."""
    out = {}
    for name, x, y in zip(("density", "u", "v", "w"), got, want):
        d = np.abs(x.astype(np.float64) - y)
        m = max(1e-30, float(np.abs(y).max()))
        out[name] = (float(d.max() / m), float(np.sqrt((d * d).mean()) / m), int((d > 1e-5 * m).sum()))
    return out


def test_semi_lagrangian_plume_step_fp64_error():
    """The plume step with semi-Lagrangian velocity and smoke (every stage a
    continuous function of its inputs) at 64^3 from an evolved state, solved
    to 1e-10, against the FP64 oracle: every sample of every field within
    1e-5 relative of the double-precision step (measured: below 1e-6)."""
    n = 64
    p = scene_params(vb.default_params(), n, rel=1e-10, max_iterations=40000)
    p.mac_cormack_vel = 0
    p.mac_cormack_smoke = 0
    fields = [np.asarray(a, np.float32) for a in swirl_fields(n, seed=5)]
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*fields)
    for _ in range(3):
        sim.advance(DT)
    state = sim.download()
    f64 = OracleSim(n, 1.0, dtype=np.float64)
    f64.params = p
    f64.set_fields(*[x.astype(np.float64) for x in state])
    sim.advance(DT)
    assert sim.last_projection().linear_solve.converged
    assert f64.advance(DT) == 0
    errs = fp64_errors(sim.download(), f64.fields())
    print("64^3 semi-Lagrangian plume step vs FP64 oracle (max, rms, samples above 1e-5):", errs)
    for name, (mx, rms, above) in errs.items():
        assert mx <= 1e-5 and above == 0, (name, errs)


def test_plume_256_learned_arm_matches_plain_arm():
    """The benchmark's two arms at 256^3 from the same state: the learned
    solver (flexible PCG with the coarse network) and the plain red-black SOR,
    both to relative divergence 1e-6 (FP64-verified). After two steps the
    fields differ only by what two 1e-6 solves allow: the max difference of
    every field relative to its max is stated and bounded by 1e-4."""
    from vapor_b200.abi import SOLVER_FPCG
    from vapor_b200.learned import COARSE_WEIGHTS, WarmStartNet
    n = 256
    fields = [np.asarray(a, np.float32) for a in swirl_fields(n, seed=2024)]
    net = WarmStartNet.load(COARSE_WEIGHTS)
    outs = {}
    for kind in (SOLVER_MIXED_REFINEMENT, SOLVER_FPCG):
        p = scene_params(vb.default_params(), n, rel=1e-6, max_iterations=20000)
        p.solver_kind = kind
        sim = vb.MacSimulation3D(n, 1.0, p)
        sim.upload(*fields)
        if kind == SOLVER_FPCG:
            sim.set_preconditioner(net)
        for _ in range(2):
            sim.advance(DT)
            ls = sim.last_projection().linear_solve
            assert ls.converged and ls.final_residual <= 1e-6 * ls.initial_residual
        outs[kind] = sim.download()
        sim.close()
    diffs = {}
    for name, a, b in zip(("density", "u", "v", "w"), outs[SOLVER_MIXED_REFINEMENT], outs[SOLVER_FPCG]):
        diffs[name] = float(np.abs(a.astype(np.float64) - b).max() / max(1e-30, float(np.abs(a).max())))
    print("256^3 learned vs plain after 2 steps, max relative difference:", diffs)
    assert max(diffs.values()) <= 1e-4, diffs
