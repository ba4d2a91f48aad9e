"""The simplicial 3D solver's compute stages (vapor_simplicial3d_*, installed
through the reference's setComputeBackend by vapor_b200/host/VaporSimplicial3D.hpp)
against the reference's own SimplicialFluidSolver3D compiled from its sources
(oracle/_ref/libvapor_ref_simplicial.so), on the reference's example meshes.

- The stages' arithmetic compiled for the host, with the reference's recovery
  copied in, keeps every field bit-identical to the reference's CPU path
  (box meshes by either nearest-site search, a resized box, a general domain).
- The CUDA advection stages do the same on the GPU.
- The full CUDA backend (advection and its Jacobi-CG recovery) passes the
  reference's own GPU backend test (SimplicialGpu3DTests.cpp): seeded
  circulation, 60 steps of flux and smoke against the CPU, boundary flux and
  divergence, resize, reset replay, and the smoke rising on the dense box.
"""
import numpy as np
import pytest

from oracle_lib import RefSimplicial, simplicial_available, sine_potential

needs_ref = pytest.mark.skipif(not simplicial_available(), reason="simplicial harness (oracle/_ref) missing")

# mesh file, box domain, size, nearest-site search
CASES = [
    ("box.tet", True, 1.0, 1),
    ("box.tet", True, 1.0, 2),
    ("box.tet", True, 2.5, 1),
    ("box-dense.tet", True, 1.0, 0),
    ("bunny-fluid.tet", False, 2.0, 0),
]
IDS = ["box-scan", "box-descent", "box2.5", "dense", "bunny"]


def _bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


def _lockstep(mode, mesh, box, size, search, steps, dt=1 / 60):
    """A solver on the CPU path and one with backend `mode` taking the first's
    recovery: every field equal bit for bit after every step. The recovery is
    handed over once per step, so the steps are short enough for one CFL
    substep each."""
    cpu = RefSimplicial(mesh, box, size)
    other = RefSimplicial(mesh, box, size)
    other.attach(mode, search, cpu)
    for k in range(steps):
        cpu.advance(dt)
        assert cpu.substeps() == 1, f"step {k + 1} took {cpu.substeps()} substeps"
        other.advance(dt)
        for name in ("vorticity", "flux", "vertex_density", "density", "potential"):
            assert _bits(getattr(cpu, name)(), getattr(other, name)()), f"step {k + 1} {name}"
    assert cpu.diagnostics()["smoke_mass"] > 0


@needs_ref
@pytest.mark.parametrize("mesh,box,size,search", CASES, ids=IDS)
def test_host_stages_equal_the_reference_cpu_path(mesh, box, size, search):
    _lockstep(RefSimplicial.HOST_ADVECTION, mesh, box, size, search, 12)


@needs_ref
@pytest.mark.parametrize("mesh,box,size", [("box.tet", True, 1.0), ("bunny-fluid.tet", False, 2.0)],
                         ids=["box", "bunny"])
def test_host_stages_with_stirring_and_a_moved_emitter_equal_the_reference(mesh, box, size):
    """The rotating stir force on, the emitter moved and stronger: a more
    varied velocity field through the same lockstep, bit for bit."""
    cpu = RefSimplicial(mesh, box, size)
    other = RefSimplicial(mesh, box, size)
    other.attach(RefSimplicial.HOST_ADVECTION, 0, cpu)
    for s in (cpu, other):
        s.set_stir(2.0, .25, 1.5)
        s.set_emitter(.4, .55, .25, strength=6.0, radius=.15, buoyancy=4.0)
    for k in range(12):
        cpu.advance(1 / 120)
        assert cpu.substeps() == 1
        other.advance(1 / 120)
        for name in ("vorticity", "flux", "vertex_density", "density"):
            assert _bits(getattr(cpu, name)(), getattr(other, name)()), f"step {k + 1} {name}"


@needs_ref
def test_host_stages_seeded_circulation_is_exact():
    cpu, host = RefSimplicial(), RefSimplicial()
    host.attach(RefSimplicial.HOST_ADVECTION, 1, cpu)
    phi = sine_potential(cpu)
    for s in (cpu, host):
        s.set_potential(phi)
        s.advect_vorticity(.017)
    assert _bits(cpu.vorticity(), host.vorticity())
    assert np.abs(cpu.vorticity()).max() > 1e-3


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("mesh,box,size,search", CASES, ids=IDS)
def test_device_advection_equals_the_reference_cpu_path(mesh, box, size, search):
    _lockstep(RefSimplicial.DEVICE_ADVECTION, mesh, box, size, search, 20)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("mesh,box,size,search", CASES, ids=IDS)
def test_device_backend_equals_the_reference_cpu_path(mesh, box, size, search):
    """The whole CUDA backend, recovery included (the CPU's preconditioner,
    the operator in its summation order, dot products in index order): every
    field and the recovery's report equal the CPU path's bit for bit, at the
    reference test's step of 1/30 s (CFL substeps included)."""
    cpu = RefSimplicial(mesh, box, size)
    gpu = RefSimplicial(mesh, box, size)
    gpu.attach(RefSimplicial.DEVICE, search, dots=1)
    for k in range(30):
        cpu.advance(1 / 30)
        gpu.advance(1 / 30)
        for name in ("vorticity", "flux", "vertex_density", "density", "potential"):
            assert _bits(getattr(cpu, name)(), getattr(gpu, name)()), f"step {k + 1} {name}"
        assert cpu.last_recovery() == gpu.last_recovery(), k + 1
    assert cpu.diagnostics() == gpu.diagnostics()


@pytest.mark.gpu
@needs_ref
def test_device_backend_tree_order_stays_within_rounding():
    """The parallel dot-product order: the recovery converges to the same
    tolerance, and the flux stays within 1e-9 of the CPU's over 10 steps."""
    cpu = RefSimplicial("bunny-fluid.tet", False, 2.0)
    gpu = RefSimplicial("bunny-fluid.tet", False, 2.0)
    gpu.attach(RefSimplicial.DEVICE, dots=2)
    for k in range(10):
        cpu.advance(1 / 30)
        gpu.advance(1 / 30)
        assert gpu.last_recovery()["converged"]
        assert _max_error(cpu.flux(), gpu.flux()) <= 1e-9, k + 1


@pytest.mark.gpu
@needs_ref
def test_device_backend_jacobi_option_within_the_reference_bound():
    """The Jacobi preconditioner on a general domain (the OpenGL backend's
    choice; not the CPU's iterates): the recovery converges and flux and
    smoke stay within the reference's GPU-backend bounds over 20 steps."""
    cpu = RefSimplicial("bunny-fluid.tet", False, 2.0)
    gpu = RefSimplicial("bunny-fluid.tet", False, 2.0)
    gpu.attach(RefSimplicial.DEVICE, dots=2, jacobi=True)
    for k in range(20):
        cpu.advance(1 / 30)
        gpu.advance(1 / 30)
        assert gpu.last_recovery()["converged"]
        assert _max_error(cpu.flux(), gpu.flux()) <= 1e-5, k + 1
        assert _max_error(cpu.vertex_density(), gpu.vertex_density()) <= 1e-3, k + 1


def _max_error(a, b):
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("mesh,box,size", [("box.tet", True, 1.0), ("box-dense.tet", True, 1.0),
                                           ("bunny-fluid.tet", False, 2.0)], ids=["box", "dense", "bunny"])
def test_device_backend_passes_the_reference_gpu_test(mesh, box, size):
    """SimplicialGpu3DTests.cpp with the CUDA backend in place of OpenGL."""
    cpu = RefSimplicial(mesh, box, size)
    gpu = RefSimplicial(mesh, box, size)
    gpu.attach(RefSimplicial.DEVICE)
    if box:
        phi = sine_potential(cpu)
        for s in (cpu, gpu):
            s.set_potential(phi)
            s.advect_vorticity(.017)
        # the reference allows 1e-8; the stages reproduce the CPU's arithmetic
        assert _max_error(cpu.vorticity(), gpu.vorticity()) == 0.0
        cpu.reset()
        gpu.reset()
    for i in range(60):
        cpu.advance(1 / 30)
        gpu.advance(1 / 30)
        d = gpu.diagnostics()
        assert np.isfinite(d["max_speed"])
        assert d["max_boundary_flux"] <= 1e-10 and d["max_divergence"] <= 1e-8, (i, d)
        assert _max_error(cpu.flux(), gpu.flux()) <= 1e-5, i
        assert _max_error(cpu.vertex_density(), gpu.vertex_density()) <= 1e-3, i
        assert gpu.last_recovery()["converged"]
    cpu.set_box_size(2.5)
    gpu.set_box_size(2.5)
    cpu.advance(.01)
    gpu.advance(.01)
    assert _max_error(cpu.flux(), gpu.flux()) <= 1e-5
    assert gpu.last_recovery()["converged"]
    replay = gpu.flux()
    gpu.reset()
    gpu.advance(.01)
    assert _bits(replay, gpu.flux())  # the reference allows 1e-10


@pytest.mark.gpu
@needs_ref
def test_device_backend_smoke_rises():
    """The motion case of SimplicialGpu3DTests.cpp: dense box, no decay, the
    emitter off after 30 of 90 frames; the smoke's centre rises by > 0.03."""
    s = RefSimplicial("box-dense.tet", True, 1.0)
    s.attach(RefSimplicial.DEVICE)
    s.set_parameters(emitter=True, decay=0.0)
    first = None
    for i in range(90):
        if i == 30:
            first = s.smoke_center()
            s.set_parameters(emitter=False, decay=0.0)
        s.advance(1 / 60)
    height, mass = s.smoke_center()
    assert height > first[0] + .03, (first, height)
    assert mass > 0


@pytest.mark.gpu
@needs_ref
def test_device_recovery_errors_follow_the_reference():
    """Invalid CG controls are rejected and an iteration budget too small to
    converge stops the step, on the CPU path and on the device alike."""
    for mode in (RefSimplicial.CPU, RefSimplicial.DEVICE):
        s = RefSimplicial()
        if mode:
            s.attach(mode)
        s.set_parameters(cg_iterations=-1)
        with pytest.raises(RuntimeError, match="CG parameters"):
            s.advance(1 / 30)
        s.set_parameters(cg_iterations=1)
        with pytest.raises(RuntimeError, match="did not converge"):
            s.advance(1 / 30)
