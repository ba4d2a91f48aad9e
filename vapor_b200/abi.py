"""ctypes mirror of include/vapor_b200.h (structs, enums, status codes).

Field order and types follow the C header exactly; the header documents which
reference struct each one mirrors (MacGridParameters3D, ProjectionOptions,
ProjectionResult, LinearSolveOptions, FluidDiagnostics).
"""
import ctypes as C

ABI_VERSION = 1

VAPOR_OK = 0
VAPOR_INVALID_ARGUMENT = 1
VAPOR_LENGTH_ERROR = 2
VAPOR_RUNTIME_ERROR = 3
VAPOR_NON_FINITE = 4
VAPOR_OUT_OF_MEMORY = 5

SIMPLE_SEMI_LAGRANGIAN = 0
SIMPLE_MACCORMACK = 1
REFLECTION_SEMI_LAGRANGIAN = 2
REFLECTION_MACCORMACK = 3

SEMI_LAGRANGIAN = 0
MACCORMACK = 1

FACE_X, FACE_Y, FACE_Z = 0, 1, 2

SOLVER_RED_BLACK_SOR = 0
SOLVER_MIXED_REFINEMENT = 1
SOLVER_FPCG = 2


class LinearSolveOptions(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int32),
        ("residual_check_interval", C.c_int32),
        ("absolute_tolerance", C.c_double),
        ("relative_tolerance", C.c_double),
        ("fixed_iterations", C.c_int32),
        ("reserved0", C.c_int32),
    ]

    @classmethod
    def defaults(cls, **kw):
        o = cls(200, 8, 1e-6, 1e-5, 0, 0)
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class LinearSolveResult(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("converged", C.c_int32),
        ("initial_residual", C.c_double),
        ("final_residual", C.c_double),
    ]


class ProjectionOptions(C.Structure):
    _fields_ = [("dt", C.c_float), ("relaxation", C.c_float), ("linear_solve", LinearSolveOptions)]

    @classmethod
    def defaults(cls, **kw):
        o = cls(1.0 / 60.0, 1.95, LinearSolveOptions.defaults())
        for k, v in kw.items():
            setattr(o, k, v)
        return o


class ProjectionResult(C.Structure):
    _fields_ = [
        ("linear_solve", LinearSolveResult),
        ("residual_available", C.c_int32),
        ("divergence_before", C.c_float),
        ("divergence_after", C.c_float),
        ("reserved0", C.c_int32),
        ("removed_rhs_mean", C.c_double),
    ]


class FluidDiagnostics(C.Structure):
    _fields_ = [("kinetic_energy", C.c_float), ("max_velocity", C.c_float), ("max_divergence", C.c_float)]


class ComparisonMetrics(C.Structure):
    """vapor_comparison_metrics: the reference harness's comparison metrics."""
    _fields_ = [("mass_sum", C.c_double), ("mass", C.c_double), ("grad_per_mass", C.c_double),
                ("square_per_mass", C.c_double), ("rms_div", C.c_double), ("max_div", C.c_double),
                ("smoke_cells", C.c_longlong), ("cfl_fallback", C.c_longlong),
                ("boundary_fallback", C.c_longlong), ("max_cfl", C.c_double), ("nonfinite", C.c_int32),
                ("reserved", C.c_int32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if name not in ("nonfinite", "reserved")}


class RenderParams(C.Structure):
    """vapor_render_params: camera, ray step, opacity and shadow of the
    headless ray-march. harness() gives the reference harness's image."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("azimuth", C.c_float), ("elevation", C.c_float),
                ("distance", C.c_float), ("step_scale", C.c_float), ("alpha_mul", C.c_float),
                ("light", C.c_float * 3), ("shadow_strength", C.c_float), ("shadow_step", C.c_float)]

    @classmethod
    def harness(cls, width=960, height=960):
        norm = 1.25 ** 0.5
        return cls(width, height, -1.2, 0.3, 2.5, 0.5, 30.0, (C.c_float * 3)(0.3 / norm, 0.4 / norm, 1.0 / norm),
                   0.3, 0.1)


class MacParams(C.Structure):
    _fields_ = [
        ("emitter_radius", C.c_float),
        ("emitter_center_x", C.c_float),
        ("emitter_center_y", C.c_float),
        ("emitter_center_z", C.c_float),
        ("emitter_kick_multiplier", C.c_float),
        ("emitter_kick_base", C.c_float),
        ("emitter_kick_scale", C.c_float),
        ("stir_strength", C.c_float),
        ("random_seed", C.c_uint32),
        ("sor_omega", C.c_float),
        ("buoyancy_split", C.c_float),
        ("cfl_mc", C.c_float),
        ("mac_cormack_smoke", C.c_int32),
        ("mac_cormack_vel", C.c_int32),
        ("smoke_decay", C.c_float),
        ("reflection", C.c_int32),
        ("buoyancy", C.c_float),
        ("source_strength", C.c_float),
        ("project_iterations", C.c_int32),
        ("use_solve_options", C.c_int32),
        ("solve", LinearSolveOptions),
        ("solver_kind", C.c_int32),
        ("emitter_profile", C.c_int32),
        ("emitter_count", C.c_int32),
        ("emitter2_center_x", C.c_float),
        ("emitter2_center_y", C.c_float),
        ("emitter2_center_z", C.c_float),
    ]

    def copy(self):
        other = MacParams()
        C.pointer(other)[0] = self
        return other

    def update(self, **kw):
        for k, v in kw.items():
            if k not in {f[0] for f in self._fields_}:
                raise AttributeError(k)
            setattr(self, k, v)
        return self


PHASES = ("forcing", "advect", "rhs", "sor", "residual", "gradient", "krylov", "coarse")


class PhaseTimings(C.Structure):
    _fields_ = [("milliseconds", C.c_double * 8), ("launches", C.c_int64 * 8), ("intervals", C.c_int64 * 8)]

    def as_dict(self):
        return {name: {"ms": self.milliseconds[i], "launches": self.launches[i], "intervals": self.intervals[i]}
                for i, name in enumerate(PHASES)}


def field_sizes(n):
    """Element counts of density, u, v, w for resolution n (MacGridState3D.cpp:12-15)."""
    c = n * n * n
    f = n * n * (n + 1)
    return c, f, f, f


def field_shapes(n):
    """numpy shapes (z, y, x) of density, u, v, w in the reference layout."""
    return (n, n, n), (n, n, n + 1), (n, n + 1, n), (n + 1, n, n)


class Mac2DParams(C.Structure):
    """vapor_mac2d_params (MacGridParameters2D, MacGridFluidSolver2D.hpp:5-15)."""
    _fields_ = [("reflection", C.c_int32), ("source_strength", C.c_float),
                ("emitter_kick_multiplier", C.c_float), ("emitter_radius", C.c_float),
                ("emitter_center_x", C.c_float), ("emitter_center_y", C.c_float), ("buoyancy", C.c_float),
                ("smoke_decay", C.c_float), ("sor_omega", C.c_float), ("project_iterations", C.c_int32)]


class Mac2DReflParams(C.Structure):
    """vapor_mac2d_refl_params (the public fields of ReflectionMacFluidSolver2D,
    ReflectionMacFluidSolver2D.hpp:19-22, 57-71)."""
    _fields_ = [("mac_cormack_smoke", C.c_int32), ("source_strength", C.c_float), ("buoyancy", C.c_float),
                ("smoke_decay", C.c_float), ("project_iterations", C.c_int32), ("emitter_radius", C.c_float),
                ("emitter_center_x", C.c_float), ("emitter_center_y", C.c_float),
                ("emitter_kick_multiplier", C.c_float), ("stir_strength", C.c_float), ("sor_omega", C.c_float),
                ("random_seed", C.c_uint32)]


def field_shapes_2d(n):
    """numpy shapes (y, x) of density, u, v of the MAC 2D state (MacGridState2D.hpp:7)."""
    return (n, n), (n, n + 1), (n + 1, n)
