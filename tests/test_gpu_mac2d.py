"""The MAC 2D solver on the device (vapor_mac2d_*) against the reference's own
MacGridFluidSolver2D compiled from its sources (oracle/_ref/libvapor_ref2d.so):
the same steps from the same state, compared bit for bit, with the
projection results (iteration counts, FP64 residuals, divergence before and
after, removed mean) and the diagnostics; plus the reference's argument
checks and reset semantics."""
import numpy as np
import pytest

import vapor_b200 as vb
from vapor_b200.mac2d import MacSimulation2D, default_params_2d, plume_params_2d
from oracle_lib import RefSim2D, ref2d_available

pytestmark = pytest.mark.gpu

needs_ref = pytest.mark.skipif(not ref2d_available(), reason="reference 2D build (oracle/_ref) missing")
DT = 1.0 / 60.0


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _same_projection(got, want):
    g, w = got.linear_solve, want.linear_solve
    assert g.iterations == w.iterations and g.converged == w.converged
    assert g.initial_residual == w.initial_residual and g.final_residual == w.final_residual
    assert got.residual_available == want.residual_available
    assert got.divergence_before == want.divergence_before and got.divergence_after == want.divergence_after
    assert got.removed_rhs_mean == want.removed_rhs_mean


def _seeded_state(n, seed):
    rng = np.random.default_rng(seed)
    d = rng.random((n, n)).astype(np.float32) * 0.5
    u = (rng.standard_normal((n, n + 1)) * 0.3).astype(np.float32)
    v = (rng.standard_normal((n + 1, n)) * 0.3).astype(np.float32)
    return d, u, v


def _run_pair(n, box, params, steps, state=None):
    sim = MacSimulation2D(n, box, params)
    ref = RefSim2D(n, box, params, *(state or (None, None, None)))
    if state is not None:
        sim.upload(*state)
    for k in range(steps):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        for got, want in zip(sim.download(), ref.fields()):
            assert _bits_equal(got, want), f"step {k + 1}"
        _same_projection(sim.last_projection(), ref.last_projection())
        _same_projection(sim.midpoint_projection(), ref.midpoint_projection())
    dg, dr = sim.diagnostics(), ref.diagnostics()
    assert (dg.kinetic_energy, dg.max_velocity, dg.max_divergence) == (dr.kinetic_energy, dr.max_velocity,
                                                                        dr.max_divergence)
    sim.close()


@needs_ref
@pytest.mark.parametrize("n,box", [(1, 1.0), (2, 4.0), (7, 1.0), (16, 4.0), (33, 1.0), (64, 1.0)])
def test_simple_plume_steps_equal_the_reference(n, box):
    """The default-constructed solver's scene (simple step) from rest."""
    _run_pair(n, box, plume_params_2d(), 12)


@needs_ref
@pytest.mark.parametrize("n,box", [(2, 1.0), (16, 1.0), (33, 4.0), (64, 1.0)])
def test_reflection_plume_steps_equal_the_reference(n, box):
    """Midpoint reflection: both projections of every step and the fields."""
    p = plume_params_2d()
    p.reflection = 1
    _run_pair(n, box, p, 12)


@needs_ref
@pytest.mark.parametrize("reflection", [0, 1])
def test_seeded_state_with_the_struct_defaults_equals_the_reference(reflection):
    """A random initial state (density and both velocity components) and the
    parameter struct's defaults (strong source and buoyancy, 600-iteration
    budget) on a 24 x 24 grid: six steps bit for bit."""
    n = 24
    p = default_params_2d()
    p.reflection = reflection
    _run_pair(n, 4.0, p, 6, state=_seeded_state(n, 5 + reflection))


def test_reset_replays_the_same_steps():
    n = 32
    p = plume_params_2d()
    p.reflection = 1
    sim = MacSimulation2D(n, 1.0, p)
    runs = []
    for _ in range(2):
        for _ in range(10):
            sim.advance(DT)
        runs.append(sim.download())
        sim.reset()
    for a, b in zip(*runs):
        assert _bits_equal(a, b)
    d, u, v = runs[0]
    assert np.all(u[:, 0] == 0) and np.all(u[:, n] == 0) and np.all(v[0, :] == 0) and np.all(v[n, :] == 0)
    assert float(d.max()) > 0 and np.all(d >= 0) and np.all(d <= 1)
    sim.close()


def test_argument_checks():
    with pytest.raises(vb.InvalidArgument):
        MacSimulation2D(0, 1.0)
    with pytest.raises(vb.InvalidArgument):
        MacSimulation2D(8, 0.0)
    sim = MacSimulation2D(8, 1.0, plume_params_2d())
    with pytest.raises(vb.InvalidArgument):
        sim.advance(0.0)
    for field, value in (("sor_omega", 2.0), ("emitter_radius", 0.0), ("emitter_center_x", 1.5),
                         ("smoke_decay", -1.0), ("emitter_kick_multiplier", -1.0)):
        p = plume_params_2d()
        setattr(p, field, value)
        sim.params = p
        with pytest.raises(vb.InvalidArgument):
            sim.advance(DT)
    sim.params = plume_params_2d()
    d, u, v = sim.download()
    u[3, 4] = np.nan
    sim.upload(u=u)
    with pytest.raises(vb.NonFinite):
        sim.advance(DT)
    sim.close()


@pytest.mark.parametrize("reflection", [0, 1])
def test_steps_equal_the_committed_reference_fixture(reflection):
    """The same comparison against fields and projection results the
    reference produced (tests/golden/mac2d_steps.npz, made by
    make_golden_2d.py), for a GPU box without the reference build."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "mac2d_steps.npz"))
    p = plume_params_2d()
    p.reflection = reflection
    sim = MacSimulation2D(24, 1.0, p)
    proj = g[f"r{reflection}_projections"]
    for step in range(1, 11):
        sim.advance(DT)
        for k, r in enumerate((sim.last_projection(), sim.midpoint_projection())):
            ls = r.linear_solve
            got = [ls.iterations, ls.converged, ls.initial_residual, ls.final_residual, r.divergence_before,
                   r.divergence_after, r.removed_rhs_mean]
            assert got == list(proj[2 * (step - 1) + k]), (step, k)
        if step in (5, 10):
            for name, a in zip(("density", "u", "v"), sim.download()):
                assert _bits_equal(a, g[f"r{reflection}_s{step}_{name}"]), (step, name)
    sim.close()
