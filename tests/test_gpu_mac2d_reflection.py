"""The reflection 2D solver on the device (vapor_mac2d_refl_*) against the
reference's own ReflectionMacFluidSolver2D compiled from its header
(oracle/_ref/libvapor_ref2d.so): the same frames from the same state,
compared bit for bit (smoke, u, v, pressure after every frame, and the
diagnostics), with semi-Lagrangian and MacCormack smoke, random stirring off
and on; plus the reference's own checks (Historical2DTests.cpp: smoke bounds,
wall leakage, reset replay, method selection) and its argument checks."""
import os

import numpy as np
import pytest

import vapor_b200 as vb
from vapor_b200.mac2d import (MACCORMACK, SEMI_LAGRANGIAN, ReflectionSimulation2D, reflection_app_params,
                              reflection_default_params)
from oracle_lib import RefHistorical2D, RefReflection2D, ref2d_available

needs_ref = pytest.mark.skipif(not ref2d_available(), reason="reference 2D build (oracle/_ref) missing")
DT = 1.0 / 60.0
FIELDS = ("smoke", "u", "v", "pressure")


def _bits_equal(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _params_tuple(p):
    return tuple(getattr(p, f) for f, _ in p._fields_)


def _diag_tuple(d):
    return d.kinetic_energy, d.max_velocity, d.max_divergence


def _params(mc, stir, **kw):
    p = reflection_default_params()
    p.mac_cormack_smoke = mc
    p.stir_strength = stir
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _compare(sim, ref, frames, where=""):
    for k in range(frames):
        assert ref.advance(DT) == 0
        sim.advance(DT)
        for name, got, want in zip(FIELDS, sim.download(), ref.fields()):
            assert _bits_equal(got, want), f"{where} frame {k + 1} {name}"
    assert _diag_tuple(sim.diagnostics()) == _diag_tuple(ref.diagnostics()), where


@needs_ref
def test_parameter_sets_equal_the_reference():
    """The member initialisers, and the solver built from an advection method
    (resolution 128, radius .04, 120 iterations)."""
    assert _params_tuple(reflection_default_params()) == _params_tuple(RefReflection2D(16).params)
    for method in (SEMI_LAGRANGIAN, MACCORMACK):
        ref = RefReflection2D(None, method=method)
        assert ref.n == 128
        assert _params_tuple(reflection_app_params(method)) == _params_tuple(ref.params)
    with pytest.raises(vb.InvalidArgument):
        reflection_app_params(2)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("n", [2, 16, 33, 64])
@pytest.mark.parametrize("mc", [0, 1])
@pytest.mark.parametrize("stir", [0.0, 2.0])
def test_frames_equal_the_reference(n, mc, stir):
    p = _params(mc, stir)
    sim = ReflectionSimulation2D(n, p)
    _compare(sim, RefReflection2D(n, p), 24, f"n={n} mc={mc} stir={stir}")
    sim.close()


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("method", [SEMI_LAGRANGIAN, MACCORMACK])
def test_application_scene_equals_the_reference(method):
    """The solver the 2D application builds: 128 x 128, 120 iterations."""
    ref = RefReflection2D(None, method=method)
    sim = ReflectionSimulation2D(ref.n, reflection_app_params(method))
    _compare(sim, ref, 8, f"method={method}")
    sim.close()


@pytest.mark.gpu
@needs_ref
def test_largest_grid_equals_the_reference():
    """n = 512, the largest resolution the reference accepts, with stirring."""
    p = _params(1, 1.5, project_iterations=20)
    sim = ReflectionSimulation2D(512, p)
    _compare(sim, RefReflection2D(512, p), 2, "n=512")
    sim.close()


@pytest.mark.gpu
@needs_ref
def test_seeded_state_and_changed_parameters_equal_the_reference():
    """A random initial state, another seed and emitter, and parameters
    changed between frames (the stirring stream continues across the change)."""
    n = 40
    rng = np.random.default_rng(11)
    smoke = rng.random((n, n)).astype(np.float32) * 0.6
    u = (rng.standard_normal((n, n + 1)) * 0.4).astype(np.float32)
    v = (rng.standard_normal((n + 1, n)) * 0.4).astype(np.float32)
    p = _params(1, 3.0, random_seed=12345, emitter_center_x=.3, emitter_center_y=.6, emitter_radius=.2,
                source_strength=.4, buoyancy=2.5, smoke_decay=.7, sor_omega=1.6, project_iterations=17,
                emitter_kick_multiplier=.5)
    sim = ReflectionSimulation2D(n, p)
    ref = RefReflection2D(n, p)
    sim.upload(smoke, u, v)
    ref.set_fields(smoke, u, v)
    _compare(sim, ref, 6, "seeded")
    p.mac_cormack_smoke = 0
    p.stir_strength = .5
    p.emitter_kick_multiplier = 0.0
    p.project_iterations = 0
    sim.params = p
    ref.params = p
    _compare(sim, ref, 6, "changed")
    sim.close()


@pytest.mark.gpu
@needs_ref
def test_reset_equals_the_reference_reset():
    """resetState(): zero fields and the stirring stream back to the seed,
    on both sides, then the same frames again."""
    n = 24
    p = _params(1, 2.0)
    sim = ReflectionSimulation2D(n, p)
    ref = RefReflection2D(n, p)
    _compare(sim, ref, 5, "before reset")
    sim.reset()
    ref.reset()
    _compare(sim, ref, 5, "after reset")
    sim.close()


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("n,frames", [(24, 24), (64, 60)])
def test_frames_equal_the_historical_plume(n, frames):
    """Historical2DTests.cpp's replay with the device in place of the
    reflection solver: the historical plume (closed walls, no stirring,
    step(1/60, .8, .995, 1, 60)) and the device solver with the member
    initialisers give the same smoke, u, v and pressure every frame."""
    old = RefHistorical2D(n)
    sim = ReflectionSimulation2D(n, reflection_default_params())
    for frame in range(1, frames + 1):
        old.step(DT, .8, .995, 1.0, 60)
        sim.advance(DT)
        for name, got, want in zip(FIELDS, sim.download(), old.fields()):
            assert np.all(np.isfinite(want))
            assert _bits_equal(got, want), f"frame {frame} {name}"
    sim.close()


@pytest.mark.gpu
def test_historical_bounds_walls_and_replay():
    """Historical2DTests.cpp's checks on the device: 120 semi-Lagrangian
    frames at 16 x 16 keep the smoke finite in [0, 1] and every wall face at
    zero; a reset replays them exactly and keeps the method; MacCormack smoke
    gives other fields."""
    n = 16
    sim = ReflectionSimulation2D(n, _params(0, 0.0))
    for _ in range(120):
        sim.advance(DT)
        s, u, v, _ = sim.download()
        assert np.all(np.isfinite(s)) and np.all(s >= 0) and np.all(s <= 1)
        assert np.all(u[:, 0] == 0) and np.all(u[:, n] == 0) and np.all(v[0, :] == 0) and np.all(v[n, :] == 0)
    first = sim.download()
    sim.reset()
    assert sim.params.mac_cormack_smoke == 0
    for _ in range(120):
        sim.advance(DT)
    for a, b in zip(first, sim.download()):
        assert _bits_equal(a, b)
    mc = ReflectionSimulation2D(n, _params(1, 0.0))
    for _ in range(120):
        mc.advance(DT)
    assert not _bits_equal(mc.download()[0], first[0])
    sim.close()
    mc.close()


@pytest.mark.gpu
def test_argument_checks():
    for n in (1, 513):
        with pytest.raises(vb.InvalidArgument):
            ReflectionSimulation2D(n)
    sim = ReflectionSimulation2D(8, reflection_default_params())
    for dt in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(vb.InvalidArgument):
            sim.advance(dt)
    bad = (("emitter_kick_multiplier", -1.0), ("emitter_kick_multiplier", float("nan")), ("buoyancy", float("inf")),
           ("smoke_decay", -.1), ("source_strength", -1.0), ("emitter_radius", 0.0), ("emitter_radius", 1.5),
           ("stir_strength", -1.0), ("sor_omega", 0.0), ("sor_omega", 2.0), ("project_iterations", -1))
    for field, value in bad:
        p = reflection_default_params()
        setattr(p, field, value)
        sim.params = p
        with pytest.raises(vb.InvalidArgument) as e:
            sim.advance(DT)
        want = "kick multiplier" if field == "emitter_kick_multiplier" else "step or parameters"
        assert want in str(e.value)
        if ref2d_available():
            ref = RefReflection2D(8, p)
            assert ref.advance(DT) == 1
    sim.params = reflection_default_params()
    sim.advance(DT)
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mc", [0, 1])
@pytest.mark.parametrize("stir", [0, 2])
def test_frames_equal_the_committed_reference_fixture(mc, stir):
    """The same comparison against fields the reference produced
    (tests/golden/mac2d_refl_steps.npz, made by make_golden_2d.py), for a GPU
    box without the reference build."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "mac2d_refl_steps.npz"))
    key = f"mc{mc}_stir{stir}"
    sim = ReflectionSimulation2D(24, _params(mc, float(stir)))
    for step in range(1, 11):
        sim.advance(DT)
        if step in (5, 10):
            for name, a in zip(FIELDS, sim.download()):
                assert _bits_equal(a, g[f"{key}_s{step}_{name}"]), (step, name)
    assert np.array_equal(np.array(_diag_tuple(sim.diagnostics()), np.float32), g[f"{key}_diagnostics"])
    sim.close()


def _quarter_exception_inputs(count, seed=3):
    """Floats in [2^-12, 1) whose C-library powf(x, .25f) is not the correctly
    rounded root: members of the periodic classes of powf_quarter_table.inc."""
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "vapor_b200", "csrc",
                        "powf_quarter_table.inc")
    text = open(path).read()
    body = text[text.index("kQuarterPeriodic["):text.index("kQuarterPeriodicCount")]
    entries = np.array([int(h, 16) for h in re.findall(r"0x[0-9a-f]+", body)], np.int64)
    rng = np.random.default_rng(seed)
    pick = rng.choice(entries, size=count, replace=False)
    cls, mant = (pick >> 1) >> 23, (pick >> 1) & 0x7FFFFF
    # unbiased exponent in [-12, -1] with exponent mod 4 == cls (-12 is 0 mod 4)
    e = -12 + cls + 4 * rng.integers(0, 3, size=count)
    bits = ((e + 127) << 23) | mant
    return bits.astype(np.uint32).view(np.float32)


def test_quarter_power_table_matches_the_c_library():
    """The table's classes really are where the C library's powf(x, .25f)
    leaves the correctly rounded root (a sample, through ctypes)."""
    import ctypes
    import ctypes.util
    libm = ctypes.CDLL(ctypes.util.find_library("m"))
    libm.powf.restype = ctypes.c_float
    libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]
    xs = _quarter_exception_inputs(200)
    for x in xs:
        lib = np.float32(libm.powf(float(x), 0.25))
        cr = np.float32(np.sqrt(np.sqrt(np.float64(x))))
        assert lib != cr, x


def test_quarter_power_function_matches_the_c_library_everywhere(tmp_path):
    """vb::powf_quarter (powf_quarter.cuh, compiled for the host) against the C
    library's powf(x, .25f) on every non-negative float."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "powf_quarter_check")
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-pthread", "-o", exe,
                    os.path.join(root, "tests", "powf_quarter_check.cpp")], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "differences 0," in r.stdout


@pytest.mark.gpu
@needs_ref
def test_buoyancy_power_equals_the_c_library_on_the_device():
    """Smoke made only of inputs where powf(x, .25f) is not the correctly
    rounded root, at rest on a 64 x 64 grid with no decay and no emitter (so
    the buoyancy sees exactly these values): one frame equals the reference."""
    n = 64
    smoke = _quarter_exception_inputs(n * n).reshape(n, n)
    p = _params(1, 0.0, source_strength=0.0, smoke_decay=0.0, buoyancy=3.0)
    sim = ReflectionSimulation2D(n, p)
    ref = RefReflection2D(n, p)
    sim.upload(smoke=smoke)
    ref.set_fields(smoke=smoke)
    _compare(sim, ref, 2, "exception smoke")
    sim.close()
