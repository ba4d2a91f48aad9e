"""CPU-side checks of the C ABI library (no compute calls, no GPU needed).

- the library loads and exports every function include/vapor_b200.h declares
- the parameter presets equal the reference's (MacGridParameters3D defaults and
  MacGridParameters3D(MacAlgorithm), via the reference build in oracle/_ref)
- grid validation happens before any device work and maps to the reference's
  exception types
- without a device the library fails loudly (no CPU fallback)
"""
import ctypes as C
import os
import re

import pytest

import vapor_b200 as vb
from oracle_lib import ref, ref_available
from vapor_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "vapor_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vapor_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = vb.library()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.vapor_abi_version() == abi.ABI_VERSION


def test_struct_sizes_match_header_layout():
    # Natural C layout on x86-64: checked field by field against the header.
    assert C.sizeof(abi.LinearSolveOptions) == 32
    assert C.sizeof(abi.LinearSolveResult) == 24
    assert C.sizeof(abi.ProjectionOptions) == 40
    assert C.sizeof(abi.ProjectionResult) == 48
    assert C.sizeof(abi.FluidDiagnostics) == 12
    assert abi.MacParams.solve.offset % 8 == 0


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_default_parameters_equal_reference():
    ours = vb.default_params()
    theirs = abi.MacParams()
    ref().vapor_mac3d_default_params(C.byref(theirs))
    for name, _ in abi.MacParams._fields_:
        assert getattr(ours, name) == getattr(theirs, name) or name.startswith("emitter2") or name == "solve", name
    for name, _ in abi.LinearSolveOptions._fields_:
        assert getattr(ours.solve, name) == getattr(theirs.solve, name), name


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("alg", [0, 1, 2, 3])
def test_algorithm_presets_equal_reference(alg):
    from oracle_lib import RefSim
    ours = vb.algorithm_params(alg)
    theirs = RefSim(algorithm=alg).params
    for name in ("emitter_radius", "source_strength", "buoyancy", "smoke_decay", "project_iterations",
                 "sor_omega", "reflection", "mac_cormack_smoke", "mac_cormack_vel", "stir_strength",
                 "random_seed", "cfl_mc", "buoyancy_split"):
        assert getattr(ours, name) == getattr(theirs, name), name


def test_algorithm_preset_rejects_unknown():
    with pytest.raises(ValueError):
        vb.algorithm_params(7)


def test_grid_validation_before_device_work():
    p = vb.default_params()
    for n, box, exc in ((0, 1.0, ValueError), (-2, 1.0, ValueError), (2 ** 31 - 1, 1.0, OverflowError),
                        (4, 0.0, ValueError), (4, float("inf"), ValueError), (4, float("nan"), ValueError)):
        with pytest.raises(exc):
            vb.MacSimulation3D(n, box, p)
        with pytest.raises(exc):
            vb.StageBackend(n, box)


def test_projection_option_defaults():
    o = vb.default_projection_options()
    assert o.dt == pytest.approx(1 / 60) and o.relaxation == pytest.approx(1.95)
    assert o.linear_solve.max_iterations == 200 and o.linear_solve.residual_check_interval == 8
    assert o.linear_solve.relative_tolerance == 1e-5 and o.linear_solve.absolute_tolerance == 1e-6


def _have_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_have_cuda(), reason="checks the no-device path")
def test_no_cpu_fallback_without_device():
    with pytest.raises(RuntimeError):
        vb.MacSimulation3D(8, 1.0, vb.default_params())
