"""Drop-in at the reference's own plugin boundary.

The reference's unmodified MacGridFluidSolver3D (compiled from its sources in
oracle/_ref/libvapor_ref_plugins.so) runs with the product's CudaProjection3D /
CudaAdvection3D installed through setPressureSolver / setAdvection
(vapor_b200/host/VaporCudaStages.hpp). The result must equal the same
coordinator with its CPU stages bit for bit, and the stage call pattern must be
the reference's (tests/BackendTests.cpp:62-130). Also checks the C++ resident
wrapper vapor_b200::CudaMacSimulation3D against the committed reference fixtures.
"""
import ctypes as C
import os

import numpy as np
import pytest

import vapor_b200 as vb
from vapor_b200.abi import MacParams, field_shapes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(ROOT, "oracle", "_ref", "libvapor_ref_plugins.so")
GOLDEN = os.path.join(ROOT, "tests", "golden")
needs_harness = pytest.mark.skipif(not os.path.exists(HARNESS), reason="plugin harness not built")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def harness():
    vb.library()  # load the product library first (the harness links it)
    lib = C.CDLL(HARNESS)
    lib.harness_run.restype = C.c_int
    lib.harness_run.argtypes = [C.c_int, C.c_float, C.POINTER(MacParams), C.c_int, C.c_float, C.c_int, C.c_int,
                                _f32p, _f32p, _f32p, _f32p, C.POINTER(C.c_longlong)]
    lib.harness_resident_cpp.restype = C.c_int
    lib.harness_resident_cpp.argtypes = [C.c_int, C.c_float, C.POINTER(MacParams), C.c_int, C.c_float, _f32p,
                                         _f32p, _f32p, _f32p, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    return lib


def run(n, box, p, frames, dt, cuda_p, cuda_a):
    out = [np.zeros(s, np.float32) for s in field_shapes(n)]
    counts = (C.c_longlong * 3)()
    st = harness().harness_run(n, box, C.byref(p), frames, dt, cuda_p, cuda_a, *out, counts)
    assert st == 0
    return out, list(counts)


def bits_equal(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@needs_harness
@pytest.mark.parametrize("alg", [0, 1, 2, 3])
@pytest.mark.parametrize("n,box", [(9, 1.0), (12, 4.5)])
def test_reference_coordinator_with_cuda_stages_is_bit_identical(alg, n, box):
    p = vb.algorithm_params(alg)
    p.project_iterations, p.stir_strength, p.emitter_radius, p.emitter_center_z = 20, 0.5, 0.22, 0.3
    cpu, _ = run(n, box, p, 6, 1 / 60, 0, 0)
    gpu, counts = run(n, box, p, 6, 1 / 60, 1, 1)
    for a, b in zip(gpu, cpu):
        assert bits_equal(a, b)
    stages = 2 if p.reflection else 1
    assert counts == [6 * stages, 18 * stages, 6]


@needs_harness
def test_single_plugin_installations():
    p = vb.algorithm_params(3)
    p.project_iterations, p.stir_strength = 16, 0.5
    cpu, _ = run(10, 2.0, p, 4, 1 / 60, 0, 0)
    for cuda_p, cuda_a in ((1, 0), (0, 1)):
        mixed, _ = run(10, 2.0, p, 4, 1 / 60, cuda_p, cuda_a)
        for a, b in zip(mixed, cpu):
            assert bits_equal(a, b)


@needs_harness
def test_cpp_resident_wrapper_matches_reference_fixture():
    data = np.load(os.path.join(GOLDEN, "reference_steps.npz"))
    p = vb.default_params()
    p.reflection, p.mac_cormack_vel, p.mac_cormack_smoke = 1, 1, 1
    p.emitter_radius, p.emitter_center_z, p.stir_strength, p.project_iterations = 0.22, 0.3, 0.5, 20
    out = [np.zeros(s, np.float32) for s in field_shapes(9)]
    up, down = C.c_ulonglong(), C.c_ulonglong()
    st = harness().harness_resident_cpp(9, 1.0, C.byref(p), 8, 1 / 60, *out, C.byref(up), C.byref(down))
    assert st == 0
    for name, a in zip("duvw", out):
        assert bits_equal(a, data[f"resident_r1_v1_s1_{name}"])
    assert up.value == 0 and down.value == sum(a.nbytes for a in out)
