"""Parity of the CUDA path (through the C ABI) with the reference.

The kernels evaluate the reference's FP32 operations in the same order without
FMA contraction, so the bar here is bit equality with the reference's CPU code
(oracle/_ref, or the committed fixtures made from it) and with the FP32 oracle.
Where a case has no reference counterpart the FP32 oracle is the pin.
Mirrors tests/GraphicsSmokeTests.cpp (CPU/GPU advection parity, resident vs
staged parity, reset replay), tests/SimulationTests.cpp and
tests/NumericsTests.cpp of the reference.
"""
import json
import os

import numpy as np
import pytest

import vapor_b200 as vb
from oracle_lib import (OracleSim, RefSim, algorithm_params, oracle_advect, oracle_project, random_fields,
                        ref_advect, ref_available, ref_project)
from vapor_b200.abi import LinearSolveOptions, ProjectionOptions, field_shapes

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def bits_equal(a, b):
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


def values_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32), np.asarray(b, np.float32))


def cpu_advect(*args):
    return ref_advect(*args) if ref_available() else oracle_advect(*args)


def cpu_project(*args):
    return ref_project(*args) if ref_available() else oracle_project(*args)


def gpu_advect(n, box, loc, dt, cfl, mc, src, u, v, w):
    st = vb.StageBackend(n, box)
    method = vb.abi.MACCORMACK if mc else vb.abi.SEMI_LAGRANGIAN
    flow = [np.ascontiguousarray(a, np.float32) for a in (u, v, w)]
    if loc == 0:
        out = np.array(src, np.float32, copy=True)
        st.advect_scalar(dt, cfl, method, out, flow)
    else:
        out = np.zeros_like(src, np.float32)
        st.advect_face(loc - 1, dt, cfl, method, np.ascontiguousarray(src, np.float32), flow, out)
    return out


@pytest.mark.parametrize("n", [1, 3, 8, 17, 40])
@pytest.mark.parametrize("mc", [0, 1])
@pytest.mark.parametrize("dt,cfl", [(0.1, 3.0), (2.0, 3.0), (0.1, 0.001), (0.6, 1.5)])
def test_advection_bit_identical_to_reference(n, mc, dt, cfl):
    box = 4.0
    d, u, v, w = random_fields(n, seed=1000 + n, scale=0.8)
    for loc, src in enumerate((d, u, v, w)):
        expected = cpu_advect(n, box, loc, dt, cfl, mc, src, u, v, w)
        got = gpu_advect(n, box, loc, dt, cfl, mc, src, u, v, w)
        assert bits_equal(got, expected), f"loc {loc}: max |diff| {np.abs(got - expected).max()}"


def test_constant_field_advection_invariance():
    """GraphicsSmokeTests.cpp:150-165: constant fields stay constant."""
    n, box = 8, 4.0
    _, u, v, w = random_fields(n, seed=5, scale=0.3)
    for mc in (0, 1):
        d = np.full((n, n, n), 0.5, np.float32)
        out = gpu_advect(n, box, 0, 0.02, 3.0, mc, d, u, v, w)
        assert np.abs(out - 0.5).max() < 1e-5
        for loc, shape in enumerate(field_shapes(n)[1:], start=1):
            src = np.full(shape, 0.125, np.float32)
            out = gpu_advect(n, box, loc, 0.02, 3.0, mc, src, u, v, w)
            assert np.abs(out - 0.125).max() < 1e-5


@pytest.mark.parametrize("n", [1, 2, 5, 10, 24])
@pytest.mark.parametrize("floor", [0.0, 6.0])
@pytest.mark.parametrize("fixed,iters", [(1, 16), (0, 600)])
def test_projection_bit_identical_to_reference(n, floor, fixed, iters):
    _, u, v, w = random_fields(n, seed=200 + n, scale=1.0)
    opts = LinearSolveOptions.defaults(max_iterations=iters, fixed_iterations=fixed, relative_tolerance=1e-6,
                                       absolute_tolerance=1e-7)
    st, r, ue, ve, we, pe = cpu_project(n, 4.5, u, v, w, 1 / 60, 1.7, floor, opts)
    assert st == 0
    stage = vb.StageBackend(n, 4.5)
    ug, vg, wg = [np.array(a, np.float32, copy=True) for a in (u, v, w)]
    rg, pg = stage.project(ug, vg, wg, ProjectionOptions(1 / 60, 1.7, opts), floor, want_pressure=True)
    for a, b in ((ug, ue), (vg, ve), (wg, we), (pg, pe)):
        assert bits_equal(a, b)
    assert rg.linear_solve.iterations == r.linear_solve.iterations
    assert rg.linear_solve.initial_residual == r.linear_solve.initial_residual
    assert rg.linear_solve.final_residual == r.linear_solve.final_residual
    assert rg.linear_solve.converged == r.linear_solve.converged
    assert rg.divergence_before == r.divergence_before and rg.divergence_after == r.divergence_after
    assert rg.removed_rhs_mean == pytest.approx(r.removed_rhs_mean, rel=1e-12, abs=1e-300)
    assert rg.residual_available == 1


def test_projection_reduces_divergence():
    """GraphicsSmokeTests.cpp:136-148, with a real (FP64) residual reported."""
    n = 8
    _, u, v, w = [np.zeros(s, np.float32) for s in field_shapes(n)]
    u[4, 4, 4] = 1.0
    stage = vb.StageBackend(n, 4.0)
    before = np.float32(1.0) / np.float32(0.5)
    opts = ProjectionOptions(1 / 60, 1.5, LinearSolveOptions.defaults(max_iterations=200, fixed_iterations=1))
    r, _ = stage.project(u, v, w, opts)
    assert r.residual_available == 1 and r.divergence_before == pytest.approx(before)
    assert r.divergence_after < before * 0.01


def resident_params(reflection, mc_vel, mc_smoke):
    p = vb.default_params()
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = int(reflection), int(mc_vel), int(mc_smoke)
    p.emitter_radius, p.emitter_center_z, p.stir_strength, p.project_iterations = 0.22, 0.3, 0.5, 20
    return p


@pytest.mark.parametrize("reflection", [0, 1])
@pytest.mark.parametrize("mc_vel", [0, 1])
@pytest.mark.parametrize("mc_smoke", [0, 1])
def test_resident_matches_reference_fixtures(reflection, mc_vel, mc_smoke):
    """GraphicsSmokeTests.cpp:22-58: 8 steps at 9^3, stirred, all flag combinations;
    bit equality with the reference's fields, no downloads during advance,
    bounded uploads, reset replay."""
    data = np.load(os.path.join(GOLDEN, "reference_steps.npz"))
    key = f"resident_r{reflection}_v{mc_vel}_s{mc_smoke}"
    sim = vb.MacSimulation3D(9, 1.0, resident_params(reflection, mc_vel, mc_smoke))
    for _ in range(8):
        sim.advance(1 / 60)
    up, down = sim.byte_counters()
    assert down == 0 and up == 0
    snapshot = sim.download()
    for name, a in zip("duvw", snapshot):
        assert bits_equal(a, data[f"{key}_{name}"]), key + name
    sim.reset_state()
    for _ in range(8):
        sim.advance(1 / 60)
    replay = sim.download()
    assert all(bits_equal(a, b) for a, b in zip(snapshot, replay))
    # Disabling kick, buoyancy and stir leaves the velocity at rest while smoke is emitted.
    sim.reset_state()
    p = sim.parameters()
    p.emitter_kick_multiplier, p.buoyancy, p.stir_strength = 0.0, 0.0, 0.0
    sim.set_parameters(p)
    sim.advance(1 / 60)
    d, u, v, w = sim.download()
    assert np.abs(u).max() < 1e-5 and np.abs(v).max() < 1e-5 and np.abs(w).max() < 1e-5
    assert d.max() > 0
    sim.set_box_size(2.0)
    d, *_ = sim.download()
    assert np.abs(d).max() == 0
    p.source_strength = 0.0
    sim.set_parameters(p)
    sim.advance(1 / 60)
    _, u, v, w = sim.download()
    assert np.abs(u).max() < 1e-5 and np.abs(v).max() < 1e-5 and np.abs(w).max() < 1e-5


def load_baselines():
    with open(os.path.join(GOLDEN, "simulation_baselines.json")) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", load_baselines(), ids=lambda c: f"n{c['n']}-r{c['reflect']}-f{c['flags']}")
def test_resident_reproduces_reference_baselines(case):
    """SimulationTests.cpp:17-41,105-136 through the resident CUDA path."""
    p = vb.default_params()
    p.stir_strength, p.emitter_radius, p.emitter_center_z = 0.0, 0.18, 0.3
    p.mac_cormack_smoke = int(case["flags"] & 1 != 0)
    p.mac_cormack_vel = int(case["flags"] & 2 != 0)
    p.reflection, p.project_iterations = case["reflect"], 16
    sim = vb.MacSimulation3D(case["n"], 4.5, p)
    for _ in range(6):
        sim.advance(1 / 60)
    d = sim.download()[0].ravel().astype(np.float64)
    diag = sim.diagnostics()

    def near(actual, expected):
        assert abs(actual - expected) <= 2e-5 * max(1.0, abs(expected)), (actual, expected)
    near(diag.kinetic_energy, case["energy"])
    near(diag.max_velocity, case["max_velocity"])
    near(diag.max_divergence, case["divergence"])
    near(d.sum(), case["density_sum"])
    near((d * (1 + np.arange(d.size) % 31)).sum(), case["weighted_density"])
    assert sim.last_projection().residual_available == 1
    sim.reset_state()
    assert sim.diagnostics().kinetic_energy == 0.0
    assert np.abs(sim.download()[0]).max() == 0.0


@pytest.mark.parametrize("alg", [0, 1, 2, 3])
@pytest.mark.parametrize("n,box", [(16, 1.0), (33, 4.5)])
def test_resident_matches_oracle_steps(alg, n, box):
    """Whole resident steps against the FP32 oracle. Every kernel is
    bit-identical to the reference; the only order-dependent values are the
    FP64 means of the right-hand side and of the pressure (the reference sums
    sequentially, the GPU in a fixed tree). When such a sum nearly cancels, its
    FP32 cast can differ by an ulp (seen at 33^3, Reflection-MacCormack), so
    the bar here is the north star's per-step bound, max |diff| <= 1e-5 x the
    field's magnitude, with bit equality asserted whenever the means agree."""
    p = algorithm_params(alg)
    p.project_iterations, p.stir_strength = 24, 0.5
    a = OracleSim(n, box)
    a.params = p
    a.reset()
    sim = vb.MacSimulation3D(n, box, p)
    means_agree = True
    for _ in range(5):
        assert a.advance(1 / 60) == 0
        sim.advance(1 / 60)
        means_agree &= a.last_projection().removed_rhs_mean == sim.last_projection().removed_rhs_mean
    for x, y in zip(sim.download(), a.fields()):
        scale = max(1.0, float(np.abs(y).max()))
        assert np.abs(x - y).max() <= 1e-5 * scale
        if means_agree:
            assert bits_equal(x, y)
    ra, rg = a.last_projection(), sim.last_projection()
    assert rg.linear_solve.final_residual == pytest.approx(ra.linear_solve.final_residual, rel=1e-4)
    assert sim.total_iterations() == a.total_iterations()


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_tolerance_driven_resident_matches_reference():
    """Tolerance-driven projections (the reference's setPressureSolver hook):
    identical iteration counts and fields."""
    p = algorithm_params(3)
    p.use_solve_options = 1
    p.solve = LinearSolveOptions.defaults(max_iterations=3000, relative_tolerance=1e-6, absolute_tolerance=0.0)
    r = RefSim(20, 1.0)
    r.params = p
    r.reset()
    sim = vb.MacSimulation3D(20, 1.0, p)
    for _ in range(3):
        assert r.advance(0.01) == 0
        sim.advance(0.01)
        assert sim.last_projection().linear_solve.iterations == r.last_projection().linear_solve.iterations
    for x, y in zip(sim.download(), r.fields()):
        assert bits_equal(x, y)


def test_seeded_replay_and_independence():
    """SimulationTests.cpp:44-75 on the resident path."""
    def make(seed):
        p = vb.default_params()
        p.emitter_radius, p.emitter_center_z, p.project_iterations, p.random_seed = .18, .3, 16, seed
        return vb.MacSimulation3D(8, 4.5, p)
    first, second, other = make(12345), make(12345), make(54321)
    for _ in range(6):
        first.advance(1 / 60)
        other.advance(1 / 60)
        second.advance(1 / 60)
    a, b, c = first.download(), second.download(), other.download()
    assert all(bits_equal(x, y) for x, y in zip(a, b))
    assert not bits_equal(a[1], c[1])
    first.reset_state()
    for _ in range(6):
        first.advance(1 / 60)
    assert all(bits_equal(x, y) for x, y in zip(first.download(), b))


def test_plume_stays_bounded_and_incompressible():
    """SimulationTests.cpp:79-98 (24^3, 180 frames, 300 iterations, omega 1.8)."""
    for reflection in (0, 1):
        p = vb.default_params()
        p.reflection, p.project_iterations, p.emitter_radius, p.sor_omega = reflection, 300, .08, 1.8
        sim = vb.MacSimulation3D(24, 4.5, p)
        for frame in range(180):
            sim.advance(1 / 60)
            if frame % 20 == 19 or frame == 179:
                d = sim.diagnostics()
                assert np.isfinite(d.kinetic_energy) and d.max_divergence <= .005
                dens = sim.download()[0]
                assert np.isfinite(dens).all() and dens.min() >= 0 and dens.max() <= 1.00001


def test_upload_download_round_trip_and_counters():
    n = 12
    sim = vb.MacSimulation3D(n, 2.0, vb.default_params())
    fields = random_fields(n, seed=3)
    sim.upload(*fields)
    back = sim.download()
    assert all(bits_equal(a, b) for a, b in zip(fields, back))
    up, down = sim.byte_counters()
    expected = sum(a.nbytes for a in fields)
    assert up == expected and down == expected


def test_resident_from_uploaded_state_matches_reference():
    """upload() then advance equals the reference solver built from that state."""
    if not ref_available():
        pytest.skip("oracle/_ref not built")
    n = 14
    fields = random_fields(n, seed=11, scale=0.2)
    p = algorithm_params(1)
    p.project_iterations, p.stir_strength = 30, 0.0
    r = RefSim(n, 2.0, fields=fields)
    r.params = p
    sim = vb.MacSimulation3D(n, 2.0, p)
    sim.upload(*fields)
    for _ in range(3):
        assert r.advance(0.02) == 0
        sim.advance(0.02)
    for x, y in zip(sim.download(), r.fields()):
        assert bits_equal(x, y)


# ---- the reference's projection known answers on the GPU ----

def test_projection_gradient_field_is_removed():
    """NumericsTests.cpp:255-278."""
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
    opts = ProjectionOptions(dt, 1.5, LinearSolveOptions.defaults(max_iterations=4000, absolute_tolerance=1e-5,
                                                                   relative_tolerance=1e-6))
    r, p = vb.StageBackend(n, box).project(u, v, w, opts, 0.0, want_pressure=True)
    assert r.linear_solve.converged
    assert max(np.abs(a).max() for a in (u, v, w)) <= 1e-5
    assert np.abs(p - (pot - pot.astype(np.float64).mean())).max() <= 1e-4
    assert abs(p.astype(np.float64).mean()) <= 1e-5


def test_projection_solenoidal_early_exit():
    """NumericsTests.cpp:311-325."""
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
    u0, v0, w0 = u.copy(), v.copy(), w.copy()
    opts = ProjectionOptions(0.02, 1.95, LinearSolveOptions.defaults(max_iterations=4000, absolute_tolerance=1e-5,
                                                                      relative_tolerance=1e-6))
    r, _ = vb.StageBackend(n, float(n)).project(u, v, w, opts)
    assert r.linear_solve.converged and r.linear_solve.iterations == 0
    assert values_equal(u, u0) and values_equal(v, v0) and values_equal(w, w0)


def test_projection_rest_state():
    """NumericsTests.cpp:236-253: rest stays at rest; bad dt is rejected."""
    for n in (1, 5, 2):
        _, u, v, w = [np.zeros(s, np.float32) for s in field_shapes(n)]
        stage = vb.StageBackend(n, 4.5)
        opts = ProjectionOptions(0.02, 1.95, LinearSolveOptions.defaults(max_iterations=4000, absolute_tolerance=1e-5,
                                                                          relative_tolerance=1e-6))
        r, p = stage.project(u, v, w, opts, want_pressure=True)
        assert r.linear_solve.converged and r.linear_solve.iterations == 0 and r.divergence_after == 0
        assert p.size == n ** 3
        for bad in (0.0, float("nan"), np.finfo(np.float32).tiny * 1e-10):
            with pytest.raises(ValueError):
                stage.project(u, v, w, ProjectionOptions(bad, 1.95, LinearSolveOptions.defaults()))


# ---- failure detection, host-side injection only ----

def test_rejections():
    with pytest.raises(ValueError):
        vb.MacSimulation3D(0, 1.0, vb.default_params())
    with pytest.raises(OverflowError):
        vb.MacSimulation3D(2 ** 31 - 1, 1.0, vb.default_params())
    with pytest.raises(ValueError):
        vb.MacSimulation3D(4, float("inf"), vb.default_params())
    sim = vb.MacSimulation3D(6, 1.0, vb.default_params())
    for field, value in (("sor_omega", 2.0), ("emitter_kick_multiplier", -1.0), ("cfl_mc", 0.0),
                         ("smoke_decay", -1.0), ("emitter_radius", 1.5), ("project_iterations", -1)):
        p = vb.default_params()
        setattr(p, field, value)
        sim.set_parameters(p)
        with pytest.raises(ValueError):
            sim.advance(1 / 60)
    sim.set_parameters(vb.default_params())
    with pytest.raises(ValueError):
        sim.advance(0.0)
    with pytest.raises(ValueError):
        sim.set_box_size(-1.0)
    stage = vb.StageBackend(3, 4.5)
    f = np.zeros(3 * 3 * 4, np.float32)
    flow = [np.zeros_like(f) for _ in range(3)]
    with pytest.raises(ValueError):
        stage.advect_face(0, 0.1, 3.0, 0, f, flow, f)          # source aliases output
    with pytest.raises(ValueError):
        stage.advect_face(0, 0.1, 3.0, 0, f, flow, flow[0])    # output aliases the tracer
    with pytest.raises(ValueError):
        stage.advect_face(0, -1.0, 3.0, 0, f, flow, np.zeros_like(f))
    with pytest.raises(ValueError):
        stage.advect_face(0, float("nan"), 3.0, 0, f, flow, np.zeros_like(f))


def test_non_finite_input_is_reported():
    """A NaN planted on the host surfaces as a status, and the context stays usable."""
    n = 6
    fields = random_fields(n, seed=2)
    fields[1][2, 2, 3] = np.nan
    sim = vb.MacSimulation3D(n, 1.0, vb.default_params())
    sim.upload(*fields)
    sim.advance(1 / 60)
    with pytest.raises(vb.NonFinite):
        sim.last_projection()
    sim.reset_state()
    sim.advance(1 / 60)
    assert sim.last_projection().residual_available == 1
    stage = vb.StageBackend(n, 1.0)
    u, v, w = [a.copy() for a in fields[1:]]
    with pytest.raises(vb.NonFinite):
        stage.project(u, v, w, ProjectionOptions(0.02, 1.5, LinearSolveOptions.defaults()))


@pytest.mark.parametrize("n", [8, 20, 33])
def test_mixed_refinement_matches_oracle(n):
    """FP32 sweeps + FP64 re-centring: same sweep count as the oracle's
    definition, FP64-verified residual below tolerance, fields within FP32
    rounding of the oracle (the FP64 pressure mean is a tree sum on the GPU)."""
    _, u, v, w = random_fields(n, seed=300 + n, scale=1.0)
    opts = LinearSolveOptions.defaults(max_iterations=20000, relative_tolerance=1e-8, absolute_tolerance=0.0)
    st, r, ue, ve, we, pe = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=1)
    assert st == 0 and r.linear_solve.converged
    stage = vb.StageBackend(n, 1.0)
    stage.set_solver_kind(vb.abi.SOLVER_MIXED_REFINEMENT)
    ug, vg, wg = [np.array(a, np.float32, copy=True) for a in (u, v, w)]
    rg, pg = stage.project(ug, vg, wg, ProjectionOptions(0.01, 1.9, opts), 6.0, want_pressure=True)
    assert rg.linear_solve.iterations == r.linear_solve.iterations
    assert rg.linear_solve.converged
    assert rg.linear_solve.final_residual <= 1e-8 * rg.linear_solve.initial_residual
    assert rg.linear_solve.initial_residual == r.linear_solve.initial_residual
    for a, b in ((ug, ue), (vg, ve), (wg, we)):
        scale = max(1.0, float(np.abs(b).max()))
        assert np.abs(a - b).max() <= 4e-7 * scale
    assert np.abs(pg - pe).max() <= 1e-6 * max(1.0, float(np.abs(pe).max()))


def test_mixed_refinement_reaches_tolerance_plain_fp32_cannot():
    """Plain FP32 SOR stagnates above 1e-6 on a plume; the refinement gets there."""
    n = 32
    p = algorithm_params(3)
    p.project_iterations, p.stir_strength = 200, 0.5
    sim = OracleSim(n, 1.0)
    sim.params = p
    sim.reset()
    for _ in range(10):
        sim.advance(0.01)
    _, u, v, w = sim.fields()
    opts = LinearSolveOptions.defaults(max_iterations=3000, relative_tolerance=1e-6, absolute_tolerance=0.0)
    plain = vb.StageBackend(n, 1.0)
    r_plain, _ = plain.project(*[a.copy() for a in (u, v, w)], ProjectionOptions(0.005, 1.95, opts), 6.0)
    mixed = vb.StageBackend(n, 1.0)
    mixed.set_solver_kind(vb.abi.SOLVER_MIXED_REFINEMENT)
    r_mixed, _ = mixed.project(*[a.copy() for a in (u, v, w)], ProjectionOptions(0.005, 1.95, opts), 6.0)
    assert not r_plain.linear_solve.converged
    assert r_mixed.linear_solve.converged and r_mixed.linear_solve.iterations < 3000


@pytest.mark.parametrize("mode", ["fixed", "tolerance", "mixed"])
def test_graph_replay_equals_eager_steps(mode):
    """Whole-step CUDA graphs (solve loops as device-side while nodes) give the
    same bits and iteration counts as the host-driven eager path."""
    p = algorithm_params(3)
    p.project_iterations, p.stir_strength = 30, 0.5
    if mode != "fixed":
        p.use_solve_options = 1
        p.solve = LinearSolveOptions.defaults(max_iterations=3000, relative_tolerance=1e-5 if mode == "tolerance"
                                              else 1e-7, absolute_tolerance=0.0)
        p.solver_kind = vb.abi.SOLVER_MIXED_REFINEMENT if mode == "mixed" else vb.abi.SOLVER_RED_BLACK_SOR
    graph = vb.MacSimulation3D(24, 1.0, p)
    eager = vb.MacSimulation3D(24, 1.0, p)
    eager.set_timing(True)  # phase timing runs the eager path
    for _ in range(3):
        graph.advance(0.01)
        eager.advance(0.01)
        assert graph.last_projection().linear_solve.iterations == eager.last_projection().linear_solve.iterations
    for a, b in zip(graph.download(), eager.download()):
        assert bits_equal(a, b)
    assert graph.total_iterations() == eager.total_iterations()
    r = graph.last_projection()
    if mode == "mixed":
        assert r.linear_solve.converged and r.linear_solve.final_residual <= 1e-7 * r.linear_solve.initial_residual
