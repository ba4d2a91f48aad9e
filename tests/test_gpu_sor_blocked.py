"""Temporally blocked red-black SOR (several red+black iterations per launch)
against the one-colour-per-launch sweep: every solver path gives the same
bits, iteration counts and results with blocking on (1 or 2 iterations per
launch) and off, on unmasked and masked grids. The one-colour sweep is itself
pinned bit for bit to the reference's CPU SOR and to the oracle by the parity
tests, so equality here carries that pin over to the blocked kernel."""
import numpy as np
import pytest

import vapor_b200 as vb
from oracle_lib import oracle_project, random_fields, sphere_mask
from vapor_b200.abi import (SOLVER_FPCG, SOLVER_MIXED_REFINEMENT, SOLVER_RED_BLACK_SOR, LinearSolveOptions,
                            ProjectionOptions)

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _restore_blocking():
    yield
    vb.tune_sor_blocking(0)


def _project(n, fields, kind, blocking, opts, omega=1.9, floor=6.0, mask=None, net=None):
    vb.tune_sor_blocking(blocking)
    stage = vb.StageBackend(n, 1.0)
    stage.set_solver_kind(kind)
    if mask is not None:
        stage.set_solid(mask)
    if net is not None:
        stage.set_preconditioner(net)
    u, v, w = [np.array(a, np.float32, copy=True) for a in fields]
    r, p = stage.project(u, v, w, ProjectionOptions(0.01, omega, opts), floor, want_pressure=True)
    stage.close()
    return r, [u, v, w, p]


def _same(a, b):
    ra, fa = a
    rb, fb = b
    la, lb = ra.linear_solve, rb.linear_solve
    assert la.iterations == lb.iterations
    assert la.final_residual == lb.final_residual and la.converged == lb.converged
    assert ra.divergence_after == rb.divergence_after
    for x, y in zip(fa, fb):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


@pytest.mark.parametrize("n", [16, 40, 64])
def test_mixed_solver_blocked_equals_one_colour_sweeps(n):
    _, u, v, w = random_fields(n, seed=900 + n)
    opts = LinearSolveOptions.defaults(max_iterations=20000, relative_tolerance=1e-6, absolute_tolerance=0.0)
    runs = [_project(n, (u, v, w), SOLVER_MIXED_REFINEMENT, b, opts, omega=1.95) for b in (0, 1, 2)]
    assert runs[0][0].linear_solve.converged
    _same(runs[0], runs[1])
    _same(runs[0], runs[2])


@pytest.mark.parametrize("n", [24, 48])
def test_masked_blocked_equals_one_colour_sweeps(n):
    mask = sphere_mask(n, (0.45, 0.55, 0.5), 0.2)
    _, u, v, w = random_fields(n, seed=910 + n)
    opts = LinearSolveOptions.defaults(max_iterations=20000, relative_tolerance=1e-7, absolute_tolerance=0.0)
    runs = [_project(n, (u, v, w), SOLVER_MIXED_REFINEMENT, b, opts, mask=mask) for b in (0, 2)]
    assert runs[0][0].linear_solve.converged
    _same(runs[0], runs[1])


@pytest.mark.parametrize("iterations", [7, 13, 40])
def test_reference_sor_blocked_equals_one_colour_and_the_oracle(iterations):
    """The reference's own SOR (exact relaxation, fixed iteration budgets that
    are not a multiple of the blocking) bit for bit against the oracle."""
    n = 24
    _, u, v, w = random_fields(n, seed=920 + iterations)
    opts = LinearSolveOptions.defaults(max_iterations=iterations, residual_check_interval=8, fixed_iterations=1)
    runs = [_project(n, (u, v, w), SOLVER_RED_BLACK_SOR, b, opts, omega=1.7) for b in (0, 1, 2)]
    _same(runs[0], runs[1])
    _same(runs[0], runs[2])
    st, ro, ue, ve, we, pe = oracle_project(n, 1.0, u, v, w, 0.01, 1.7, 6.0, opts, solver_kind=0)
    assert st == 0 and ro.linear_solve.iterations == runs[2][0].linear_solve.iterations
    for got, want in zip(runs[2][1], (ue, ve, we, pe)):
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_iteration_cap_inside_a_blocked_launch():
    """A budget that ends in the middle of a two-iteration launch: the launch
    does only the sweeps left, as the guarded one-colour launches do."""
    n = 32
    _, u, v, w = random_fields(n, seed=930)
    opts = LinearSolveOptions.defaults(max_iterations=21, relative_tolerance=1e-12, absolute_tolerance=0.0)
    runs = [_project(n, (u, v, w), SOLVER_MIXED_REFINEMENT, b, opts) for b in (0, 2)]
    assert runs[0][0].linear_solve.iterations == 21 and not runs[0][0].linear_solve.converged
    _same(runs[0], runs[1])


@pytest.mark.parametrize("n", [32, 64])
def test_fpcg_smoothing_blocked_equals_one_colour_sweeps(n):
    """The FPCG preconditioner's smoothing runs one-colour sweeps whatever
    the blocking setting (its last sweep also forms the dot products of the
    direction update): the setting leaves the solve's bits unchanged."""
    from vapor_b200.learned import COARSE_WEIGHTS, WarmStartNet
    net = WarmStartNet.load(COARSE_WEIGHTS)
    _, u, v, w = random_fields(n, seed=940 + n)
    opts = LinearSolveOptions.defaults(max_iterations=2000, relative_tolerance=1e-6, absolute_tolerance=0.0)
    for coarse in (None, net):
        runs = [_project(n, (u, v, w), SOLVER_FPCG, b, opts, net=coarse) for b in (0, 2)]
        assert runs[0][0].linear_solve.converged
        _same(runs[0], runs[1])


def test_resident_plume_steps_blocked_equal_one_colour_sweeps():
    """Whole resident steps (CUDA graphs with device-side solve loops) of the
    benchmark plume scene at 64^3 with the plain and the learned solver."""
    from vapor_b200.learned import COARSE_WEIGHTS, WarmStartNet
    from vapor_b200.plume import scene_params, swirl_fields
    n = 64
    fields = swirl_fields(n, 5)
    net = WarmStartNet.load(COARSE_WEIGHTS)
    for kind in (SOLVER_MIXED_REFINEMENT, SOLVER_FPCG):
        outs = []
        for b in (0, 2):
            vb.tune_sor_blocking(b)
            p = scene_params(vb.default_params(), n, rel=1e-6, max_iterations=20000)
            p.solver_kind = kind
            sim = vb.MacSimulation3D(n, 1.0, p)
            sim.upload(*fields)
            if kind == SOLVER_FPCG:
                sim.set_preconditioner(net)
            for _ in range(3):
                sim.advance(0.01)
            outs.append((sim.total_iterations(), sim.download()))
            sim.close()
        assert outs[0][0] == outs[1][0]
        for x, y in zip(outs[0][1], outs[1][1]):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_batched_scenes_with_blocking_equal_one_colour_steps():
    """Blocked sweeps inside batched scene graphs (several scenes' solve loops
    running at once) against separate scenes stepped with the one-colour
    sweep: the out-of-place blocked update must see no half-written halo."""
    from oracle_lib import algorithm_params

    def scene(n, alg, k):
        p = algorithm_params(alg)
        p.stir_strength = 0.5
        p.emitter_center_x = 0.3 + 0.1 * k
        p.use_solve_options = 1
        p.solve = LinearSolveOptions.defaults(max_iterations=3000, relative_tolerance=1e-6, absolute_tolerance=0.0)
        p.solver_kind = SOLVER_MIXED_REFINEMENT
        return vb.MacSimulation3D(n, 1.0, p)

    sizes = [(16, 3), (24, 1), (32, 2), (40, 0)]
    vb.tune_sor_blocking(0)
    single = [scene(n, a, k) for k, (n, a) in enumerate(sizes)]
    for _ in range(4):
        for s in single:
            s.advance(0.01)
    vb.tune_sor_blocking(2)
    grouped = [scene(n, a, k) for k, (n, a) in enumerate(sizes)]
    batch = vb.Batch(grouped)
    for _ in range(4):
        batch.advance(0.01)
    batch.synchronize()
    for a, b in zip(single, grouped):
        assert a.total_iterations() == b.total_iterations()
        for x, y in zip(a.download(), b.download()):
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    batch.close()
