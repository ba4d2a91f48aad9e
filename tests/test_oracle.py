"""Pins the CPU oracle before anything is compared against it.

1. The float oracle reproduces the reference's golden diagnostics
   (tests/SimulationTests.cpp:17-34) at the reference's tolerance (2e-5 rel).
2. The float oracle is bit-identical to the reference's own CPU sources
   (oracle/_ref) on seeded inputs: sampling, advection, projection, full steps.
3. The reference's known-answer tests (AdvectionTests.cpp, NumericsTests.cpp)
   hold for the oracle.
4. The FP64 oracle agrees with the FP32 oracle to FP32 accuracy.
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle_lib import (OracleSim, RefSim, algorithm_params, default_params, oracle, oracle_advect,
                        oracle_project, random_fields, ref, ref_advect, ref_available, ref_project)
from vapor_b200.abi import LinearSolveOptions, field_shapes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
needs_ref = pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def load_baselines():
    with open(os.path.join(GOLDEN, "simulation_baselines.json")) as f:
        return json.load(f)


def baseline_params(case):
    p = default_params()
    p.stir_strength, p.emitter_radius, p.emitter_center_z = 0.0, 0.18, 0.3
    p.mac_cormack_smoke = int(case["flags"] & 1 != 0)
    p.mac_cormack_vel = int(case["flags"] & 2 != 0)
    p.reflection, p.project_iterations = case["reflect"], 16
    return p


def near(actual, expected, name):
    tol = 2e-5 * max(1.0, abs(expected))
    assert np.isfinite(actual) and abs(actual - expected) <= tol, f"{name}: {actual} vs {expected}"


@pytest.mark.parametrize("case", load_baselines()["cases"],
                         ids=lambda c: f"n{c['n']}-r{c['reflect']}-f{c['flags']}")
def test_oracle_reproduces_reference_baselines(case):
    sim = OracleSim(case["n"])
    sim.params = baseline_params(case)
    for _ in range(6):
        assert sim.advance(1.0 / 60.0) == 0
    d = sim.fields()[0].ravel().astype(np.float64)
    weights = 1 + (np.arange(d.size) % 31)
    diag = sim.diagnostics()
    near(diag.kinetic_energy, case["energy"], "kinetic energy")
    near(diag.max_velocity, case["max_velocity"], "max velocity")
    near(diag.max_divergence, case["divergence"], "divergence")
    near(d.sum(), case["density_sum"], "density sum")
    near((d * weights).sum(), case["weighted_density"], "weighted density")


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 4, 7])
@pytest.mark.parametrize("loc", [0, 1, 2, 3])
def test_sampling_bit_identical(n, loc):
    box = 3.7
    rng = np.random.default_rng(10 * n + loc)
    f = rng.standard_normal(n * n * (n + (loc > 0))).astype(np.float32)
    for _ in range(64):
        x, y, z = (rng.random(3) * 1.6 - 0.3) * box
        a = oracle().vo_sample_f32(n, box, loc, f, x, y, z)
        b = ref().ref_sample(n, box, loc, f, x, y, z)
        assert np.float32(a).view(np.uint32) == np.float32(b).view(np.uint32)


@needs_ref
@pytest.mark.parametrize("n", [1, 3, 6, 11])
@pytest.mark.parametrize("mc", [0, 1])
@pytest.mark.parametrize("dt,cfl", [(0.1, 3.0), (2.0, 3.0), (0.1, 0.001), (0.6, 1.5)])
def test_advection_bit_identical(n, mc, dt, cfl):
    box = 4.0
    d, u, v, w = random_fields(n, seed=n * 7 + mc, scale=0.8)
    for loc, src in enumerate((d, u, v, w)):
        a = oracle_advect(n, box, loc, dt, cfl, mc, src, u, v, w)
        b = ref_advect(n, box, loc, dt, cfl, mc, src, u, v, w)
        assert bits_equal(a, b), f"loc {loc}"


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 5, 10])
@pytest.mark.parametrize("floor", [0.0, 6.0])
@pytest.mark.parametrize("fixed,iters", [(1, 16), (0, 400)])
def test_projection_bit_identical(n, floor, fixed, iters):
    d, u, v, w = random_fields(n, seed=100 + n, scale=1.0)
    opts = LinearSolveOptions.defaults(max_iterations=iters, fixed_iterations=fixed,
                                       relative_tolerance=1e-6, absolute_tolerance=1e-7)
    sa, ra, ua, va, wa, pa = oracle_project(n, 4.5, u, v, w, 1 / 60, 1.7, floor, opts)
    sb, rb, ub, vb, wb, pb = ref_project(n, 4.5, u, v, w, 1 / 60, 1.7, floor, opts)
    assert sa == sb == 0
    for x, y in ((ua, ub), (va, vb), (wa, wb), (pa, pb)):
        assert bits_equal(x, y)
    assert ra.linear_solve.iterations == rb.linear_solve.iterations
    assert ra.linear_solve.final_residual == rb.linear_solve.final_residual
    assert ra.linear_solve.initial_residual == rb.linear_solve.initial_residual
    assert ra.removed_rhs_mean == rb.removed_rhs_mean
    assert ra.divergence_before == rb.divergence_before and ra.divergence_after == rb.divergence_after


@needs_ref
@pytest.mark.parametrize("alg", [0, 1, 2, 3])
@pytest.mark.parametrize("n,box", [(9, 1.0), (12, 4.5), (13, 2.0)])
def test_full_steps_bit_identical(alg, n, box):
    p = algorithm_params(alg)
    p.project_iterations, p.stir_strength, p.emitter_radius, p.emitter_center_z = 20, 0.5, 0.22, 0.3
    a, r = OracleSim(n, box), RefSim(n, box)
    a.params, r.params = p, p
    a.reset()
    r.reset()
    for _ in range(8):
        assert a.advance(1 / 60) == 0 and r.advance(1 / 60) == 0
    for x, y in zip(a.fields(), r.fields()):
        assert bits_equal(x, y)
    pa, pr = a.last_projection(), r.last_projection()
    assert pa.linear_solve.final_residual == pr.linear_solve.final_residual


@needs_ref
def test_tolerance_driven_steps_bit_identical():
    """Tolerance-driven projections through the reference's setPressureSolver hook."""
    p = algorithm_params(3)
    p.use_solve_options = 1
    p.solve = LinearSolveOptions.defaults(max_iterations=2000, relative_tolerance=1e-6, absolute_tolerance=0.0)
    a, r = OracleSim(12, 1.0), RefSim(12, 1.0)
    a.params, r.params = p, p
    a.reset()
    r.reset()
    for _ in range(4):
        assert a.advance(0.01) == 0 and r.advance(0.01) == 0
        assert a.last_projection().linear_solve.iterations == r.last_projection().linear_solve.iterations
    for x, y in zip(a.fields(), r.fields()):
        assert bits_equal(x, y)


def test_reference_step_fixtures_match_oracle():
    """The committed reference fixtures (made from oracle/_ref) equal the oracle."""
    data = np.load(os.path.join(GOLDEN, "reference_steps.npz"))
    for reflection in (0, 1):
        for mc_vel in (0, 1):
            for mc_smoke in (0, 1):
                p = default_params()
                p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = reflection, mc_vel, mc_smoke
                p.emitter_radius, p.emitter_center_z, p.stir_strength, p.project_iterations = 0.22, 0.3, 0.5, 20
                sim = OracleSim(9, 1.0)
                sim.params = p
                sim.reset()
                for _ in range(8):
                    assert sim.advance(1 / 60) == 0
                key = f"resident_r{reflection}_v{mc_vel}_s{mc_smoke}"
                for name, a in zip("duvw", sim.fields()):
                    assert bits_equal(a, data[f"{key}_{name}"]), key + name


# ---- the reference's own known-answer tests, run against the oracle ----

def test_sampling_known_answers():
    """AdvectionTests.cpp:29-56: linear fields are sampled exactly; clamping."""
    n, box = 4, 4.0
    value = lambda x, y, z: x + 2 * y + 3 * z
    sd, su, sv, sw = field_shapes(n)
    zz, yy, xx = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    d = value(xx[:n, :n, :n] + .5, yy[:n, :n, :n] + .5, zz[:n, :n, :n] + .5).astype(np.float32)
    u = value(xx[:n, :n, :], yy[:n, :n, :] + .5, zz[:n, :n, :] + .5).astype(np.float32)
    v = value(xx[:n, :, :n] + .5, yy[:n, :, :n], zz[:n, :, :n] + .5).astype(np.float32)
    w = value(xx[:, :n, :n] + .5, yy[:, :n, :n] + .5, zz[:, :n, :n]).astype(np.float32)
    o = oracle()
    p = (1.2, 1.6, 2.1)
    expected = value(*p)
    for loc, f in enumerate((d, u, v, w)):
        assert abs(o.vo_sample_f32(n, box, loc, f.ravel(), *p) - expected) <= 1e-5
    assert abs(o.vo_sample_f32(n, box, 0, d.ravel(), -1, -1, -1) - 3.0) <= 1e-5
    assert abs(o.vo_sample_f32(n, box, 1, u.ravel(), -1, -1, -1) - 2.5) <= 1e-5
    assert abs(o.vo_sample_f32(n, box, 0, d.ravel(), 9, 9, 9) - 21.0) <= 1e-5
    assert abs(o.vo_sample_f32(n, box, 1, u.ravel(), 9, 9, 9) - 21.5) <= 1e-5
    assert abs(o.vo_sample_f32(n, box, 2, v.ravel(), 9, 9, 9) - 22.0) <= 1e-5
    assert abs(o.vo_sample_f32(n, box, 3, w.ravel(), 9, 9, 9) - 22.5) <= 1e-5
    single = np.array([2.0], np.float32)
    assert abs(o.vo_sample_f32(1, 4.5, 0, single, 1, 1, 1) - 2.0) <= 1e-5


@pytest.mark.parametrize("mc", [0, 1])
def test_uniform_translation_known_answer(mc):
    """AdvectionTests.cpp:84-110: u=.5, dt=.5 translates a linear field by .25."""
    n, box = 6, 6.0
    d, u, v, w = [np.zeros(s, np.float32) for s in field_shapes(n)]
    u[:] = 0.5
    zz, yy, xx = np.meshgrid(np.arange(n + 1), np.arange(n + 1), np.arange(n + 1), indexing="ij")
    for loc, shape in enumerate(field_shapes(n)):
        src = (xx + 2 * yy + 3 * zz)[: shape[0], : shape[1], : shape[2]].astype(np.float32)
        out = oracle_advect(n, box, loc, 0.5, 3.0, mc, src, u, v, w)
        assert abs(out[2, 2, 2] - (12.0 - 0.25)) <= 1e-5


def test_projection_gradient_known_answer():
    """NumericsTests.cpp:255-278: a discrete gradient projects to zero and the
    pressure is recovered up to a constant."""
    n, box, dt = 8, 4.0, 0.1
    h = box / n
    x = np.arange(n, dtype=np.float32)
    zz, yy, xx = np.meshgrid(x, x, x, indexing="ij")
    pot = (np.sin(np.float32(0.3) * xx) * np.cos(np.float32(0.4) * yy) + np.float32(0.2) * zz * zz / (n * n)).astype(np.float32)
    f = np.float32(dt / h)
    _, u, v, w = [np.zeros(s, np.float32) for s in field_shapes(n)]
    u[:, :, 1:n] = f * (pot[:, :, 1:] - pot[:, :, :-1])
    v[:, 1:n, :] = f * (pot[:, 1:, :] - pot[:, :-1, :])
    w[1:n, :, :] = f * (pot[1:, :, :] - pot[:-1, :, :])
    opts = LinearSolveOptions.defaults(max_iterations=4000, absolute_tolerance=1e-5, relative_tolerance=1e-6)
    st, r, uo, vo, wo, p = oracle_project(n, box, u, v, w, dt, 1.5, 0.0, opts)
    assert st == 0 and r.linear_solve.converged
    for a in (uo, vo, wo):
        assert np.abs(a).max() <= 1e-5
    assert np.abs(p - (pot - pot.astype(np.float64).mean())).max() <= 1e-4


def test_projection_solenoidal_known_answer():
    """NumericsTests.cpp:311-325: a discrete curl is untouched (early exit)."""
    n = 4
    psi = lambda x, y: np.float32(x * (n - x) * y * (n - y))
    _, u, v, w = [np.zeros(s, np.float32) for s in field_shapes(n)]
    for z in range(n):
        for y in range(n):
            for x in range(n + 1):
                u[z, y, x] = psi(x, y + 1) - psi(x, y)
        for y in range(n + 1):
            for x in range(n):
                v[z, y, x] = -(psi(x + 1, y) - psi(x, y))
    opts = LinearSolveOptions.defaults(max_iterations=4000, absolute_tolerance=1e-5, relative_tolerance=1e-6)
    st, r, uo, vo, wo, _ = oracle_project(n, float(n), u, v, w, 0.02, 1.95, 0.0, opts)
    assert st == 0 and r.linear_solve.converged and r.linear_solve.iterations == 0
    assert np.array_equal(uo, u) and np.array_equal(vo, v) and np.array_equal(wo, w)


def _legacy_projection(n, box, u, v, w, dt, iterations, omega):
    """Independent restatement of the GLSL sor.comp loop (lagged Neumann ghost,
    denominator 6), as NumericsTests.cpp:343-373 states it."""
    o = oracle()
    u, v, w = u.copy(), v.copy(), w.copy()
    o.vo_enforce_walls_f32(n, u, v, w)
    h = np.float32(np.float32(box) / np.float32(n))
    div = np.zeros((n, n, n), np.float32)
    hinv = np.float32(1) / h
    for z in range(n):
        for y in range(n):
            for x in range(n):
                s = (np.float32(u[z, y, x + 1]) - u[z, y, x] + v[z, y + 1, x] - v[z, y, x] + w[z + 1, y, x] - w[z, y, x])
                div[z, y, x] = np.float32(s) * hinv
    p = np.zeros((n, n, n), np.float32)
    om = np.float32(omega)
    c = h * h / np.float32(dt)
    for _ in range(iterations):
        for parity in range(2):
            for z in range(n):
                for y in range(n):
                    for x in range((y + z + parity) & 1, n, 2):
                        cen = p[z, y, x]
                        s = np.float32(0)
                        s += p[z, y, x - 1] if x > 0 else cen
                        s += p[z, y, x + 1] if x + 1 < n else cen
                        s += p[z, y - 1, x] if y > 0 else cen
                        s += p[z, y + 1, x] if y + 1 < n else cen
                        s += p[z - 1, y, x] if z > 0 else cen
                        s += p[z + 1, y, x] if z + 1 < n else cen
                        p[z, y, x] = (np.float32(1) - om) * cen + om * (s - div[z, y, x] * c) / np.float32(6)
    o.vo_apply_gradient_f32(n, box, p, dt, u, v, w)
    o.vo_enforce_walls_f32(n, u, v, w)
    return u, v, w


@pytest.mark.parametrize("n", [2, 3, 6])
@pytest.mark.parametrize("iterations", [1, 8])
def test_projection_matches_legacy_shader_formula(n, iterations):
    """NumericsTests.cpp:375-384: floor-6 SOR equals the GLSL sor.comp formula."""
    _, u, v, w = random_fields(n, seed=7 + n)
    opts = LinearSolveOptions.defaults(max_iterations=iterations, fixed_iterations=1)
    st, r, uo, vo, wo, _ = oracle_project(n, 4.5, u, v, w, 1 / 60, 1.95, 6.0, opts)
    assert st == 0 and r.linear_solve.iterations == iterations
    lu, lv, lw = _legacy_projection(n, 4.5, u, v, w, 1 / 60, iterations, 1.95)
    for a, b in ((uo, lu), (vo, lv), (wo, lw)):
        assert np.abs(a - b).max() <= 2e-5


def test_seeded_replay():
    """SimulationTests.cpp:44-75: seeded streams are independent; reset replays."""
    def make(seed):
        s = OracleSim(8)
        p = s.params
        p.emitter_radius, p.emitter_center_z, p.project_iterations, p.random_seed = .18, .3, 16, seed
        s.params = p
        s.reset()
        return s
    first, second, other = make(12345), make(12345), make(54321)
    for _ in range(6):
        first.advance(1 / 60)
        other.advance(1 / 60)
        second.advance(1 / 60)
    assert all(bits_equal(a, b) for a, b in zip(first.fields(), second.fields()))
    assert not bits_equal(first.fields()[1], other.fields()[1])
    first.reset()
    for _ in range(6):
        first.advance(1 / 60)
    assert all(bits_equal(a, b) for a, b in zip(first.fields(), second.fields()))


@pytest.mark.parametrize("alg", [0, 3])
def test_fp64_oracle_tracks_fp32(alg):
    p = algorithm_params(alg)
    p.project_iterations, p.stir_strength = 40, 0.0
    a, b = OracleSim(10, 1.0), OracleSim(10, 1.0, dtype=np.float64)
    a.params, b.params = p, p
    a.reset()
    b.reset()
    for _ in range(4):
        assert a.advance(1 / 60) == 0 and b.advance(1 / 60) == 0
    for x, y in zip(a.fields(), b.fields()):
        scale = max(1.0, float(np.abs(y).max()))
        assert np.abs(x.astype(np.float64) - y).max() <= 1e-4 * scale


def test_solid_mask_without_solids_is_the_plain_projection():
    """The obstacle path with an empty mask reproduces the plain projection bit for bit."""
    from oracle_lib import oracle_project, random_fields
    from vapor_b200.abi import LinearSolveOptions
    n = 12
    _, u, v, w = random_fields(n, seed=41)
    opts = LinearSolveOptions.defaults(max_iterations=400, relative_tolerance=1e-6, absolute_tolerance=0.0)
    for kind in (0, 1):
        a = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=kind)
        b = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=kind,
                           solid=np.zeros((n, n, n), np.uint8))
        assert a[0] == b[0] == 0
        assert a[1].linear_solve.iterations == b[1].linear_solve.iterations
        for x, y in zip(a[2:], b[2:]):
            assert bits_equal(x, y)


def test_sphere_obstacle_projection_closes_its_faces():
    """Sphere obstacle: faces touching solid cells are zero, pressure is zero
    inside, the fluid divergence drops to the solve tolerance, and the FP32
    mixed-precision result tracks the FP64 oracle."""
    from oracle_lib import oracle_project, random_fields, sphere_mask
    from vapor_b200.abi import LinearSolveOptions
    n = 20
    solid = sphere_mask(n, (0.5, 0.45, 0.5), 0.2)
    assert 0 < solid.sum() < n ** 3
    _, u, v, w = random_fields(n, seed=43)
    opts = LinearSolveOptions.defaults(max_iterations=20000, relative_tolerance=1e-8, absolute_tolerance=0.0)
    st, r, uo, vo, wo, p = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=1, solid=solid)
    assert st == 0 and r.linear_solve.converged
    s = solid.astype(bool)
    assert np.all(p[s] == 0)
    # faces of solid cells
    assert np.all(uo[:, :, :-1][s] == 0) and np.all(uo[:, :, 1:][s] == 0)
    assert np.all(vo[:, :-1, :][s] == 0) and np.all(vo[:, 1:, :][s] == 0)
    assert np.all(wo[:-1][s] == 0) and np.all(wo[1:][s] == 0)
    assert r.divergence_after <= 1e-5 * r.divergence_before
    st64, r64, u64, v64, w64, p64 = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=0,
                                                   dtype=np.float64, solid=solid)
    assert st64 == 0 and r64.linear_solve.converged
    for a, b in ((uo, u64), (vo, v64), (wo, w64)):
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, np.abs(b).max())


def profile_emission(n, box, centres, radius, strength=1.0):
    """The profile sources restated with numpy in the oracle's FP32 operation
    order: min(1, s * 3 * exp(-3.5 q^2)) for cells with q^2 <= 1 (exp in
    double, rounded once), the larger value where sources overlap."""
    f = np.float32
    d = np.zeros((n, n, n), np.float32)
    dx = f(box) / f(n)
    erad = f(radius) * f(box)
    R = int(erad / dx + f(1))
    for cf in centres:
        ec = [f(c) * f(box) for c in cf]
        lo = [max(0, int(e / dx) - R) for e in ec]
        hi = [min(n, int(e / dx) + R) for e in ec]
        for z in range(lo[2], hi[2]):
            for y in range(lo[1], hi[1]):
                for x in range(lo[0], hi[0]):
                    q = [((f(i) + f(0.5)) * dx - e) / erad for i, e in zip((x, y, z), ec)]
                    q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2]
                    if q2 > f(1):
                        continue
                    prof = min(f(1), f(strength) * f(3) * f(np.exp(np.float64(f(-3.5) * q2))))
                    d[z, y, x] = max(d[z, y, x], prof)
    return d


def test_profile_sources_known_answer():
    """The profile emitter (no reference counterpart) against its formula: one
    step from rest with no buoyancy leaves exactly the emitted density (zero
    velocity: the advection samples every cell at its own centre, the
    projection has nothing to remove)."""
    n, box = 32, 1.0
    centres = ((0.3, 0.5, 0.15), (0.7, 0.5, 0.15))
    p = default_params()
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = 0, 0, 0
    p.buoyancy, p.smoke_decay, p.stir_strength, p.emitter_kick_multiplier = 0.0, 0.0, 0.0, 0.0
    p.emitter_radius, p.source_strength, p.emitter_profile, p.emitter_count = 0.08, 1.0, 1, 2
    p.emitter_center_x, p.emitter_center_y, p.emitter_center_z = centres[0]
    p.emitter2_center_x, p.emitter2_center_y, p.emitter2_center_z = centres[1]
    sim = OracleSim(n, box)
    sim.params = p
    sim.reset()
    assert sim.advance(0.01) == 0
    d, u, v, w = sim.fields()
    want = profile_emission(n, box, centres, 0.08)
    assert want.max() == 1.0 and np.count_nonzero(want) > 100
    assert bits_equal(d, want)
    assert not any(np.any(a) for a in (u, v, w))


def test_plume_step_error_against_fp64_oracle():
    """Per-step error statement for the benchmark plume scene (two profile
    sources, swirl, Reflection + MacCormack, mixed-precision solve to 1e-6) at
    32^3: from the same FP32 state, one FP32 step (bit-identical to the GPU
    step, test_gpu_configs.py) against one FP64 step; max relative error per
    field (density, u, v, w) within 1e-5 every step (measured 4e-7 to 8e-7)."""
    from vapor_b200 import default_params as vb_default_params
    from vapor_b200.plume import DT, scene_params, swirl_fields
    n = 32
    p = scene_params(vb_default_params(), n, rel=1e-6, max_iterations=20000)
    a, b = OracleSim(n, 1.0), OracleSim(n, 1.0, dtype=np.float64)
    a.params, b.params = p, p
    a.set_fields(*[np.asarray(x, np.float32) for x in swirl_fields(n, seed=5)])
    for _ in range(4):
        b.set_fields(*[x.astype(np.float64) for x in a.fields()])
        assert a.advance(DT) == 0 and b.advance(DT) == 0
        for x, y in zip(a.fields(), b.fields()):
            err = np.abs(x.astype(np.float64) - y).max() / max(1e-30, float(np.abs(y).max()))
            assert err <= 1e-5, err


def test_comparison_metrics_known_answers():
    """The harness metrics (tests/ReflectionComparison.hpp:32-75) on states
    whose values are known: one smoke cell at rest (grad counts its six
    faces, no fallbacks), then a uniform x-velocity of 6 cells per frame
    (CFL 6 > 3) whose traces leave the box from cells near the walls."""
    from oracle_lib import comparison_metrics
    n = 8
    d = np.zeros((n, n, n), np.float32)
    u = np.zeros((n, n, n + 1), np.float32)
    v = np.zeros((n, n + 1, n), np.float32)
    w = np.zeros((n + 1, n, n), np.float32)
    d[3, 3, 3] = 1.0
    m = comparison_metrics(n, 1.0, d, u, v, w)
    assert m["mass_sum"] == 1.0 and m["grad_per_mass"] == 6.0 and m["square_per_mass"] == 1.0
    assert m["smoke_cells"] == 1 and m["cfl_fallback"] == 0 and m["boundary_fallback"] == 0
    assert m["max_cfl"] == 0.0 and m["rms_div"] == 0.0 and m["max_div"] == 0.0
    d[...] = 0.5
    u[...] = 6.0 * 60.0 / n  # 6 cells per frame at 60 frames per second
    m = comparison_metrics(n, 1.0, d, u, v, w)
    assert m["smoke_cells"] == n ** 3 and m["cfl_fallback"] == n ** 3
    assert abs(m["max_cfl"] - 6.0) < 1e-6
    # traces of +-6 cells stay inside only for no cell of an 8-wide box
    assert m["boundary_fallback"] == n ** 3
    assert m["grad_per_mass"] == 0.0 and m["max_div"] == 0.0


def test_volume_render_restatement_known_answers(tmp_path):
    """The oracle's restatement of the volume shader (volume.frag:13-55): an
    empty volume leaves the clear colour everywhere; a box full of dense smoke
    saturates the pixels whose rays meet it (alpha reaches 0.99 in a few
    steps) and leaves the others at the clear colour; the PPM writer emits the
    harness's header and top row first."""
    from oracle_lib import render_volume
    from vapor_b200.abi import RenderParams
    from vapor_b200.diagnostics import write_ppm
    n = 16
    params = RenderParams.harness(48, 32)
    bg = np.array([0.03, 0.04, 0.07], np.float32)
    img = render_volume(n, 1.0, np.zeros((n, n, n), np.float32), params)
    assert np.array_equal(img, np.broadcast_to(bg, img.shape))
    full = render_volume(n, 1.0, np.full((n, n, n), 50.0, np.float32), params)
    centre = full[16, 24]
    assert not np.allclose(centre, bg) and 0.0 < centre.max() <= 1.0
    corner = full[0, 0]
    assert np.allclose(corner, bg)  # the box does not reach the image corner from this camera
    path = tmp_path / "img.ppm"
    write_ppm(path, full)
    data = path.read_bytes()
    assert data.startswith(b"P6\n48 32\n255\n") and len(data) == len(b"P6\n48 32\n255\n") + 48 * 32 * 3
