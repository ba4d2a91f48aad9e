"""Solid obstacles in the staged projection (extension, no reference
counterpart): GPU against the oracle's restatement of the same rules."""
import numpy as np
import pytest

import vapor_b200 as vb
from oracle_lib import oracle_project, random_fields, sphere_mask
from vapor_b200.abi import LinearSolveOptions, ProjectionOptions

pytestmark = pytest.mark.gpu


def _stage(n, mask):
    st = vb.StageBackend(n, 1.0)
    st.set_solver_kind(vb.abi.SOLVER_MIXED_REFINEMENT)
    st.set_solid(mask)
    return st


def _opts(rel):
    return LinearSolveOptions.defaults(max_iterations=20000, relative_tolerance=rel, absolute_tolerance=0.0)


def test_empty_mask_is_the_plain_projection():
    n = 24
    _, u, v, w = random_fields(n, seed=61)
    outs = []
    for mask in (None, np.zeros((n, n, n), np.uint8)):
        st = _stage(n, mask)
        fields = [a.copy() for a in (u, v, w)]
        r, p = st.project(*fields, ProjectionOptions(0.01, 1.9, _opts(1e-7)), 6.0, want_pressure=True)
        outs.append((r.linear_solve.iterations, fields, p))
    assert outs[0][0] == outs[1][0]
    for a, b in zip(outs[0][1] + [outs[0][2]], outs[1][1] + [outs[1][2]]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("n", [20, 33])
def test_sphere_obstacle_matches_the_oracle(n):
    """Same rules as the oracle (closed faces, fluid-only unknowns and means).
    The FP64 fluid means are sums in a different order, so the bar is the
    north star's 1e-5 relative; iteration counts agree within one check."""
    mask = sphere_mask(n, (0.5, 0.45, 0.55), 0.22)
    _, u, v, w = random_fields(n, seed=70 + n)
    opts = _opts(1e-8)
    st, ro, ue, ve, we, pe = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=1, solid=mask)
    assert st == 0 and ro.linear_solve.converged
    stage = _stage(n, mask)
    ug, vg, wg = [a.copy() for a in (u, v, w)]
    r, pg = stage.project(ug, vg, wg, ProjectionOptions(0.01, 1.9, opts), 6.0, want_pressure=True)
    ls = r.linear_solve
    assert ls.converged and ls.final_residual <= 1e-8 * ls.initial_residual
    assert abs(ls.iterations - ro.linear_solve.iterations) <= 8
    for a, b in ((ug, ue), (vg, ve), (wg, we), (pg, pe)):
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, float(np.abs(b).max()))
    s = mask.astype(bool)
    assert np.all(pg[s] == 0)
    assert np.all(ug[:, :, :-1][s] == 0) and np.all(ug[:, :, 1:][s] == 0)
    assert np.all(vg[:, :-1, :][s] == 0) and np.all(vg[:, 1:, :][s] == 0)
    assert np.all(wg[:-1][s] == 0) and np.all(wg[1:][s] == 0)


def test_obstacle_rejections():
    n = 16
    stage = vb.StageBackend(n, 1.0)
    with pytest.raises(vb.InvalidArgument):
        stage.set_solid(np.ones((n, n, n), np.uint8))  # no fluid left
    stage.set_solid(sphere_mask(n, (0.5, 0.5, 0.5), 0.2))
    _, u, v, w = random_fields(n, seed=5)
    with pytest.raises(vb.InvalidArgument):  # the reference's SOR kind has no obstacles
        stage.project(u.copy(), v.copy(), w.copy(), ProjectionOptions(0.01, 1.9, _opts(1e-6)), 6.0)


def test_mixed_projection_scene_error_against_the_fp64_oracle():
    """The 256^3 mixed-precision configuration's scene (k^-5/3 solenoidal +
    gradient velocity, seeded sphere obstacle) at 48^3: FP32 sweeps under FP64
    refinement to relative divergence 1e-8, against the FP64 oracle solved to
    the same tolerance. Measured max relative errors are about 1e-7 (u, v, w)
    and 2e-7 (p); the bound is 1e-6."""
    from oracle_lib import oracle_project
    from vapor_b200.configs import mixed_projection
    from vapor_b200.plume import omega_for
    n, rel = 48, 1e-8
    out, f = mixed_projection(n=n, seed=1, rel=rel, repeats=1, return_fields=True)
    assert out["converged"] and out["fp64_relative_residual"] <= rel
    u, v, w = f["input"]
    o64 = LinearSolveOptions.defaults(max_iterations=200000, relative_tolerance=rel, absolute_tolerance=0.0)
    st, r64, u64, v64, w64, p64 = oracle_project(n, 1.0, u, v, w, f["dt"], omega_for(n), 6.0, o64, solver_kind=0,
                                                 dtype=np.float64, solid=f["mask"])
    assert st == 0 and r64.linear_solve.converged
    errs = {}
    for name, g, ref in zip(("u", "v", "w", "p"), f["projected"], (u64, v64, w64, p64)):
        errs[name] = float(np.abs(g.astype(np.float64) - ref).max() / max(1e-300, np.abs(ref).max()))
    print("FP64 oracle max relative error:", errs)
    assert max(errs.values()) <= 1e-6, errs


def test_resident_steps_with_an_obstacle_match_the_oracle():
    """Whole resident steps (CUDA graphs) of the benchmark plume scene at 32^3
    with a sphere obstacle in every projection (vapor_mac3d_set_solid), the
    mixed-precision solve to 1e-7, against the oracle's steps with the same
    mask: the fluid means differ in summation order, so the fields agree to
    the projection test's 1e-5 relative per step (bounded here by 1e-4 after
    three steps), the faces touching the obstacle stay closed, and the
    iteration counts agree within one check interval per projection."""
    from oracle_lib import OracleSim
    from vapor_b200.plume import DT, scene_params, swirl_fields
    n = 32
    mask = sphere_mask(n, (0.5, 0.5, 0.55), 0.18)
    p = scene_params(vb.default_params(), n, rel=1e-7, max_iterations=20000)
    p.solver_kind = vb.abi.SOLVER_MIXED_REFINEMENT
    fields = [np.asarray(a, np.float32) for a in swirl_fields(n, seed=8)]
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*fields)
    sim.set_solid(mask)
    ref = OracleSim(n, 1.0)
    ref.params = p
    ref.set_fields(*fields)
    ref.set_solid(mask)
    s = mask.astype(bool)
    for _ in range(3):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        got, want = sim.last_projection().linear_solve, ref.last_projection().linear_solve
        assert got.converged and abs(got.iterations - want.iterations) <= 16
        d, u, v, w = sim.download()
        assert np.all(u[:, :, :-1][s] == 0) and np.all(u[:, :, 1:][s] == 0)
        assert np.all(v[:, :-1, :][s] == 0) and np.all(v[:, 1:, :][s] == 0)
        assert np.all(w[:-1][s] == 0) and np.all(w[1:][s] == 0)
    errs = {}
    for name, x, y in zip(("density", "u", "v", "w"), sim.download(), ref.fields()):
        errs[name] = float(np.abs(x - y).max() / max(1e-30, float(np.abs(y).max())))
    print("32^3 plume with obstacle, 3 steps vs oracle, max relative difference:", errs)
    assert max(errs.values()) <= 1e-4, errs
    # the plain red-black SOR has no obstacle form: a clear error, not a wrong answer
    p.solver_kind = vb.abi.SOLVER_RED_BLACK_SOR
    sim.set_parameters(p)
    with pytest.raises(vb.VaporError):
        sim.advance(DT)
        sim.synchronize()


def _fpcg_stage(n, mask, net=None):
    st = vb.StageBackend(n, 1.0)
    st.set_solver_kind(vb.abi.SOLVER_FPCG)
    st.set_solid(mask)
    if net is not None:
        st.set_preconditioner(net)
    return st


@pytest.mark.parametrize("n,learned", [(32, False), (64, True)])
def test_fpcg_with_an_obstacle_matches_the_oracle(n, learned):
    """The FPCG solver with a sphere obstacle (masked operator, smoothing and
    coarse correction; the coarse network where given, whose mask channel
    stays zero) solves the same masked system as the oracle's mixed-precision
    solver: fields and pressure to the projection test's 1e-5 relative, solid
    pressure zero, the faces touching the obstacle closed."""
    from vapor_b200.learned import WarmStartNet, COARSE_WEIGHTS
    mask = sphere_mask(n, (0.5, 0.45, 0.55), 0.22)
    _, u, v, w = random_fields(n, seed=90 + n)
    opts = _opts(1e-8)
    st, ro, ue, ve, we, pe = oracle_project(n, 1.0, u, v, w, 0.01, 1.9, 6.0, opts, solver_kind=1, solid=mask)
    assert st == 0 and ro.linear_solve.converged
    net = WarmStartNet.load(COARSE_WEIGHTS) if learned else None
    stage = _fpcg_stage(n, mask, net)
    ug, vg, wg = [a.copy() for a in (u, v, w)]
    r, pg = stage.project(ug, vg, wg, ProjectionOptions(0.01, 1.9, opts), 6.0, want_pressure=True)
    ls = r.linear_solve
    assert ls.converged and ls.final_residual <= 1e-8 * ls.initial_residual
    print(f"FPCG with obstacle at {n}^3 (learned={learned}): {ls.iterations} CG steps, "
          f"oracle mixed solver {ro.linear_solve.iterations} sweeps")
    for a, b in ((ug, ue), (vg, ve), (wg, we), (pg, pe)):
        assert np.abs(a - b).max() <= 1e-5 * max(1.0, float(np.abs(b).max()))
    s = mask.astype(bool)
    assert np.all(pg[s] == 0)
    assert np.all(ug[:, :, :-1][s] == 0) and np.all(ug[:, :, 1:][s] == 0)
    assert np.all(vg[:, :-1, :][s] == 0) and np.all(vg[:, 1:, :][s] == 0)
    assert np.all(wg[:-1][s] == 0) and np.all(wg[1:][s] == 0)
    stage.close()
    if net is not None:
        net.close()


def test_resident_fpcg_steps_with_an_obstacle_match_the_oracle():
    """Whole resident steps of the 64^3 plume with a sphere obstacle and the
    learned FPCG solver (to 1e-7) against the oracle's mixed-precision steps
    with the same mask: within the resident obstacle test's 1e-4 after two
    steps, faces touching the obstacle closed."""
    from oracle_lib import OracleSim
    from vapor_b200.learned import WarmStartNet, COARSE_WEIGHTS
    from vapor_b200.plume import DT, scene_params, swirl_fields
    n = 64
    mask = sphere_mask(n, (0.5, 0.5, 0.55), 0.18)
    p = scene_params(vb.default_params(), n, rel=1e-7, max_iterations=20000)
    fields = [np.asarray(a, np.float32) for a in swirl_fields(n, seed=9)]
    p.solver_kind = vb.abi.SOLVER_FPCG
    net = WarmStartNet.load(COARSE_WEIGHTS)
    sim = vb.MacSimulation3D(n, 1.0, p)
    sim.upload(*fields)
    sim.set_solid(mask)
    sim.set_preconditioner(net)
    p_ref = scene_params(vb.default_params(), n, rel=1e-7, max_iterations=20000)
    p_ref.solver_kind = vb.abi.SOLVER_MIXED_REFINEMENT
    ref = OracleSim(n, 1.0)
    ref.params = p_ref
    ref.set_fields(*fields)
    ref.set_solid(mask)
    s = mask.astype(bool)
    for _ in range(2):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        assert sim.last_projection().linear_solve.converged
        d, u, v, w = sim.download()
        assert np.all(u[:, :, :-1][s] == 0) and np.all(u[:, :, 1:][s] == 0)
        assert np.all(v[:, :-1, :][s] == 0) and np.all(v[:, 1:, :][s] == 0)
        assert np.all(w[:-1][s] == 0) and np.all(w[1:][s] == 0)
    errs = {}
    for name, x, y in zip(("density", "u", "v", "w"), sim.download(), ref.fields()):
        errs[name] = float(np.abs(x - y).max() / max(1e-30, float(np.abs(y).max())))
    print("64^3 plume with obstacle, learned FPCG, 2 steps vs oracle, max relative difference:", errs)
    assert max(errs.values()) <= 1e-4, errs
    sim.close()
    net.close()
    sim.close()
