"""Test-side loaders for the oracle libraries (checkers, never the product).

  Oracle     oracle/_build/libvapor_oracle.so   CPU restatement (float and double)
  Reference  oracle/_ref/libvapor_ref.so        the reference's own CPU sources

Both are built by `make -C oracle` (see oracle/Makefile); __graft_entry__.build()
runs it. Arrays are numpy, in the reference's MAC layout (z, y, x).
"""
import ctypes as C
import os

import numpy as np

from vapor_b200.abi import (FluidDiagnostics, LinearSolveOptions, LinearSolveResult, MacParams,
                            ProjectionResult, field_shapes)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libvapor_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libvapor_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


def _setup_oracle(lib):
    for suf, T, P in (("f32", C.c_float, _f32p), ("f64", C.c_double, _f64p)):
        def f(name, res, *args):
            fn = getattr(lib, f"{name}_{suf}")
            fn.restype = res
            fn.argtypes = list(args)
        f("vo_sample", C.c_double, C.c_int, T, C.c_int, P, T, T, T)
        f("vo_advect", None, C.c_int, T, C.c_int, T, T, C.c_int, P, P, P, P, P)
        f("vo_divergence", None, C.c_int, T, P, P, P, P)
        f("vo_max_divergence", C.c_double, C.c_int, T, P, P, P)
        f("vo_enforce_walls", None, C.c_int, P, P, P)
        f("vo_apply_gradient", None, C.c_int, T, P, T, P, P, P)
        f("vo_residual", C.c_double, C.c_int, P, P)
        f("vo_sor_solve", C.c_int, C.c_int, T, T, P, P, C.POINTER(LinearSolveOptions),
          C.POINTER(LinearSolveResult))
        f("vo_sor_iteration", None, C.c_int, T, T, P, P)
        f("vo_project", C.c_int, C.c_int, T, P, P, P, T, T, T, C.POINTER(LinearSolveOptions), C.c_int,
          C.POINTER(ProjectionResult), P)
        f("vo_project_masked", C.c_int, C.c_int, T, P, P, P, T, T, T, C.POINTER(LinearSolveOptions), C.c_int,
          _vp, C.POINTER(ProjectionResult), P)
        f("vo_sim_create", _vp, C.c_int, T)
        f("vo_sim_destroy", None, _vp)
        f("vo_sim_set_params", None, _vp, C.POINTER(MacParams))
        f("vo_sim_get_params", None, _vp, C.POINTER(MacParams))
        f("vo_sim_reset", None, _vp)
        f("vo_sim_set_solid", None, _vp, _vp)
        f("vo_sim_advance", C.c_int, _vp, T)
        f("vo_sim_get_fields", None, _vp, P, P, P, P)
        f("vo_sim_set_fields", None, _vp, P, P, P, P)
        f("vo_sim_rng", C.c_uint32, _vp)
        f("vo_sim_set_rng", None, _vp, C.c_uint32)
        f("vo_sim_diagnostics", None, _vp, C.POINTER(FluidDiagnostics))
        f("vo_sim_last_projection", None, _vp, C.POINTER(ProjectionResult))
        f("vo_sim_total_iterations", C.c_longlong, _vp)
    lib.vapor_mac3d_default_params.argtypes = [C.POINTER(MacParams)]
    lib.vapor_mac3d_algorithm_params.argtypes = [C.c_int32, C.POINTER(MacParams)]
    lib.vo_render_volume.restype = None
    lib.vo_render_volume.argtypes = [C.c_int, C.c_float, _f32p, C.c_void_p, _f32p]
    lib.vo_comparison_metrics.restype = None
    lib.vo_comparison_metrics.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, _f32p, _f32p, _f32p, _f32p,
                                          _f64p]
    return lib


def _setup_ref(lib):
    def f(name, res, *args):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)
    P = _f32p
    f("ref_sim_create", C.c_int, C.c_int, C.c_float, C.POINTER(_vp))
    f("ref_sim_create_algorithm", C.c_int, C.c_int, C.POINTER(_vp))
    f("ref_sim_create_from_fields", C.c_int, C.c_int, C.c_float, P, P, P, P, C.POINTER(_vp))
    f("ref_sim_destroy", None, _vp)
    f("ref_sim_set_params", C.c_int, _vp, C.POINTER(MacParams))
    f("ref_sim_get_params", None, _vp, C.POINTER(MacParams))
    f("ref_sim_reset", C.c_int, _vp)
    f("ref_sim_set_box", C.c_int, _vp, C.c_float)
    f("ref_sim_advance", C.c_int, _vp, C.c_float)
    f("ref_sim_get_fields", None, _vp, P, P, P, P)
    f("ref_sim_diagnostics", C.c_int, _vp, C.POINTER(FluidDiagnostics))
    f("ref_sim_last_projection", None, _vp, C.POINTER(ProjectionResult))
    f("ref_sim_resolution", C.c_int, _vp)
    f("ref_sim_box", C.c_float, _vp)
    f("ref_advect", C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float, C.c_int, P, P, P, P, P)
    f("ref_project", C.c_int, C.c_int, C.c_float, P, P, P, C.c_float, C.c_float, C.c_float,
      C.POINTER(LinearSolveOptions), C.POINTER(ProjectionResult), P)
    f("ref_sor_solve", C.c_int, C.c_int, C.c_float, C.c_float, P, P, P, P, P, P,
      C.POINTER(LinearSolveOptions), C.POINTER(LinearSolveResult))
    f("ref_sample", C.c_double, C.c_int, C.c_float, C.c_int, P, C.c_float, C.c_float, C.c_float)
    f("ref_max_divergence", C.c_int, C.c_int, C.c_float, P, P, P, C.POINTER(C.c_float))
    f("ref_divergence", C.c_int, C.c_int, C.c_float, P, P, P, P)
    lib.vapor_mac3d_default_params.argtypes = [C.POINTER(MacParams)]
    return lib


_oracle = None
_ref = None


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError(f"oracle library missing: {ORACLE_SO} (run make -C oracle)")
        _oracle = _setup_oracle(C.CDLL(ORACLE_SO))
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"reference library missing: {REF_SO}")
        _ref = _setup_ref(C.CDLL(REF_SO))
    return _ref


def default_params():
    p = MacParams()
    oracle().vapor_mac3d_default_params(C.byref(p))
    return p


def algorithm_params(alg):
    p = MacParams()
    assert oracle().vapor_mac3d_algorithm_params(alg, C.byref(p)) == 0
    return p


def zeros_fields(n, dtype=np.float32):
    return [np.zeros(s, dtype=dtype) for s in field_shapes(n)]


class OracleSim:
    """The oracle coordinator (float: reference-exact FP32; double: FP64 oracle)."""

    def __init__(self, n, box=4.5, dtype=np.float32):
        self.n, self.box, self.dtype = n, box, np.dtype(dtype)
        self.suf = "f32" if self.dtype == np.float32 else "f64"
        self.lib = oracle()
        self.h = self._fn("vo_sim_create")(n, box)

    def _fn(self, name):
        return getattr(self.lib, f"{name}_{self.suf}")

    def __del__(self):
        if getattr(self, "h", None):
            self._fn("vo_sim_destroy")(self.h)
            self.h = None

    @property
    def params(self):
        p = MacParams()
        self._fn("vo_sim_get_params")(self.h, C.byref(p))
        return p

    @params.setter
    def params(self, p):
        self._fn("vo_sim_set_params")(self.h, C.byref(p))

    def reset(self):
        self._fn("vo_sim_reset")(self.h)

    def set_solid(self, mask):
        """Obstacle mask (n^3, z, y, x order, nonzero = solid; None clears) for
        every later projection."""
        if mask is None:
            self._fn("vo_sim_set_solid")(self.h, None)
            return
        self._mask = np.ascontiguousarray(mask, dtype=np.uint8)
        self._fn("vo_sim_set_solid")(self.h, self._mask.ctypes.data)

    def advance(self, dt):
        return self._fn("vo_sim_advance")(self.h, dt)

    def fields(self):
        out = zeros_fields(self.n, self.dtype)
        self._fn("vo_sim_get_fields")(self.h, *out)
        return out

    def set_fields(self, d, u, v, w):
        arrs = [np.ascontiguousarray(a, dtype=self.dtype) for a in (d, u, v, w)]
        self._fn("vo_sim_set_fields")(self.h, *arrs)

    @property
    def rng(self):
        return self._fn("vo_sim_rng")(self.h)

    @rng.setter
    def rng(self, s):
        self._fn("vo_sim_set_rng")(self.h, s)

    def diagnostics(self):
        d = FluidDiagnostics()
        self._fn("vo_sim_diagnostics")(self.h, C.byref(d))
        return d

    def last_projection(self):
        r = ProjectionResult()
        self._fn("vo_sim_last_projection")(self.h, C.byref(r))
        return r

    def total_iterations(self):
        return self._fn("vo_sim_total_iterations")(self.h)


class RefSim:
    """The reference's MacGridFluidSolver3D, compiled from its own sources."""

    def __init__(self, n=None, box=4.5, algorithm=None, fields=None):
        self.lib = ref()
        h = _vp()
        if algorithm is not None:
            st = self.lib.ref_sim_create_algorithm(algorithm, C.byref(h))
        elif fields is not None:
            arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in fields]
            st = self.lib.ref_sim_create_from_fields(n, box, *arrs, C.byref(h))
        else:
            st = self.lib.ref_sim_create(n, box, C.byref(h))
        if st != 0:
            raise ValueError(f"reference construction failed with status {st}")
        self.h = h
        self.n = self.lib.ref_sim_resolution(h)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_sim_destroy(self.h)
            self.h = None

    @property
    def params(self):
        p = MacParams()
        self.lib.ref_sim_get_params(self.h, C.byref(p))
        return p

    @params.setter
    def params(self, p):
        st = self.lib.ref_sim_set_params(self.h, C.byref(p))
        if st != 0:
            raise ValueError(f"reference rejected parameters ({st})")

    def reset(self):
        return self.lib.ref_sim_reset(self.h)

    def set_box(self, b):
        return self.lib.ref_sim_set_box(self.h, b)

    def advance(self, dt):
        return self.lib.ref_sim_advance(self.h, dt)

    def fields(self):
        out = zeros_fields(self.n)
        self.lib.ref_sim_get_fields(self.h, *out)
        return out

    def diagnostics(self):
        d = FluidDiagnostics()
        st = self.lib.ref_sim_diagnostics(self.h, C.byref(d))
        return d if st == 0 else None

    def last_projection(self):
        r = ProjectionResult()
        self.lib.ref_sim_last_projection(self.h, C.byref(r))
        return r


def ref_advect(n, box, loc, dt, cfl, mc, src, u, v, w):
    out = np.zeros_like(src, dtype=np.float32)
    st = ref().ref_advect(n, box, loc, dt, cfl, int(mc), *[np.ascontiguousarray(a, np.float32) for a in (src, u, v, w)], out)
    if st != 0:
        raise ValueError(st)
    return out


def oracle_advect(n, box, loc, dt, cfl, mc, src, u, v, w, dtype=np.float32):
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    out = np.zeros(src.shape, dtype=dtype)
    getattr(oracle(), f"vo_advect_{suf}")(n, box, loc, dt, cfl, int(mc),
                                          *[np.ascontiguousarray(a, dtype) for a in (src, u, v, w)], out)
    return out


def ref_project(n, box, u, v, w, dt, omega, floor, opts):
    u, v, w = [np.array(a, dtype=np.float32, copy=True) for a in (u, v, w)]
    p = np.zeros((n, n, n), np.float32)
    r = ProjectionResult()
    st = ref().ref_project(n, box, u, v, w, dt, omega, floor, C.byref(opts), C.byref(r), p)
    return st, r, u, v, w, p


def oracle_project(n, box, u, v, w, dt, omega, floor, opts, solver_kind=0, dtype=np.float32, solid=None):
    """The oracle's projection; `solid` (n^3 uint8, x fastest, nonzero = solid)
    adds obstacles: closed faces, fluid-only unknowns and means."""
    suf = "f32" if np.dtype(dtype) == np.float32 else "f64"
    u, v, w = [np.array(a, dtype=dtype, copy=True) for a in (u, v, w)]
    p = np.zeros((n, n, n), dtype)
    r = ProjectionResult()
    if solid is None:
        st = getattr(oracle(), f"vo_project_{suf}")(n, box, u, v, w, dt, omega, floor, C.byref(opts), solver_kind,
                                                   C.byref(r), p)
    else:
        mask = np.ascontiguousarray(solid, dtype=np.uint8)
        assert mask.size == n ** 3
        st = getattr(oracle(), f"vo_project_masked_{suf}")(n, box, u, v, w, dt, omega, floor, C.byref(opts),
                                                          solver_kind, mask.ctypes.data, C.byref(r), p)
    return st, r, u, v, w, p


def sphere_mask(n, centre, radius):
    """Cells whose centres lie inside a sphere (box 1), as an n^3 uint8 mask."""
    c = (np.arange(n) + 0.5) / n
    zz, yy, xx = np.meshgrid(c, c, c, indexing="ij")
    d2 = (xx - centre[0]) ** 2 + (yy - centre[1]) ** 2 + (zz - centre[2]) ** 2
    return (d2 < radius * radius).astype(np.uint8)


def random_fields(n, seed, scale=1.0, density=True):
    """Seeded random MAC state (density in [0,1), velocities ~ N(0, scale))."""
    rng = np.random.default_rng(seed)
    sd, su, sv, sw = field_shapes(n)
    d = rng.random(sd, dtype=np.float32) if density else np.zeros(sd, np.float32)
    return [d] + [(rng.standard_normal(s) * scale).astype(np.float32) for s in (su, sv, sw)]


def comparison_metrics(n, box, d, u, v, w, fps=60.0, cfl_mc=3.0):
    """The reference harness's comparison metrics on the CPU (the oracle's
    restatement of tests/ReflectionComparison.hpp:32-75), as the device
    entry point reports them."""
    out = np.zeros(9, np.float64)
    arrs = [np.ascontiguousarray(a, np.float32) for a in (d, u, v, w)]
    oracle().vo_comparison_metrics(n, box, fps, cfl_mc, *arrs, out)
    mass_sum, grad, square, divsq, max_div, smoke, cfl_fb, bnd_fb, max_cfl = out
    return {"mass_sum": mass_sum, "mass": mass_sum / n ** 3, "grad_per_mass": grad / mass_sum,
            "square_per_mass": square / mass_sum, "rms_div": float(np.sqrt(divsq / n ** 3)), "max_div": max_div,
            "smoke_cells": int(smoke), "cfl_fallback": int(cfl_fb), "boundary_fallback": int(bnd_fb),
            "max_cfl": max_cfl}


def render_volume(n, box, density, params):
    """The oracle's restatement of the volume shader: (height, width, 3)."""
    rgb = np.zeros((params.height, params.width, 3), np.float32)
    oracle().vo_render_volume(n, box, np.ascontiguousarray(density, np.float32), C.addressof(params), rgb)
    return rgb


# ---- the reference's MAC 2D solver (oracle/_ref/libvapor_ref2d.so) ----

REF2D_SO = os.path.join(ROOT, "oracle", "_ref", "libvapor_ref2d.so")
_ref2d = None


def ref2d_available():
    return os.path.exists(REF2D_SO)


def _ref2d_lib():
    global _ref2d
    if _ref2d is None:
        from vapor_b200.abi import Mac2DParams
        lib = C.CDLL(REF2D_SO)

        def f(name, res, *args):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = list(args)
        f("ref2_create", _vp, C.c_int, C.c_float, _vp, _vp, _vp)
        f("ref2_destroy", None, _vp)
        f("ref2_set_params", None, _vp, C.POINTER(Mac2DParams))
        f("ref2_advance", C.c_int, _vp, C.c_float)
        f("ref2_get_fields", None, _vp, _vp, _vp, _vp)
        f("ref2_last_projection", None, _vp, C.POINTER(ProjectionResult))
        f("ref2_midpoint_projection", None, _vp, C.POINTER(ProjectionResult))
        f("ref2_diagnostics", None, _vp, C.POINTER(FluidDiagnostics))
        from vapor_b200.abi import Mac2DReflParams
        R = C.POINTER(Mac2DReflParams)
        f("ref2r_create", _vp, C.c_int, R)
        f("ref2r_create_app", _vp, C.c_int)
        f("ref2r_destroy", None, _vp)
        f("ref2r_resolution", C.c_int, _vp)
        f("ref2r_get_params", None, _vp, R)
        f("ref2r_set_params", None, _vp, R)
        f("ref2r_reset", None, _vp)
        f("ref2r_set_fields", None, _vp, _vp, _vp, _vp)
        f("ref2r_advance", C.c_int, _vp, C.c_float)
        f("ref2r_get_fields", None, _vp, _vp, _vp, _vp, _vp)
        f("ref2r_diagnostics", None, _vp, C.POINTER(FluidDiagnostics))
        f("ref2h_create", _vp, C.c_int)
        f("ref2h_destroy", None, _vp)
        f("ref2h_step", None, _vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int)
        f("ref2h_get_fields", None, _vp, _vp, _vp, _vp, _vp)
        _ref2d = lib
    return _ref2d


class RefSim2D:
    """The reference's MacGridFluidSolver2D on a given state (CPU)."""

    def __init__(self, n, box, params, density=None, u=None, v=None):
        from vapor_b200.abi import field_shapes_2d
        self.n = n
        self.lib = _ref2d_lib()
        keep = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (density, u, v)]
        self.h = self.lib.ref2_create(n, box, *[None if a is None else a.ctypes.data for a in keep])
        if not self.h:
            raise ValueError("the reference rejected the 2D grid")
        self.lib.ref2_set_params(self.h, C.byref(params))
        self.shapes = field_shapes_2d(n)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref2_destroy(self.h)
            self.h = None

    def advance(self, dt):
        return self.lib.ref2_advance(self.h, dt)

    def fields(self):
        out = [np.zeros(s, np.float32) for s in self.shapes]
        self.lib.ref2_get_fields(self.h, *[a.ctypes.data for a in out])
        return out

    def last_projection(self):
        r = ProjectionResult()
        self.lib.ref2_last_projection(self.h, C.byref(r))
        return r

    def midpoint_projection(self):
        r = ProjectionResult()
        self.lib.ref2_midpoint_projection(self.h, C.byref(r))
        return r

    def diagnostics(self):
        d = FluidDiagnostics()
        self.lib.ref2_diagnostics(self.h, C.byref(d))
        return d


class RefReflection2D:
    """The reference's ReflectionMacFluidSolver2D (CPU): resolution n with the
    given fields, or (n None) the solver built from an advection method."""

    def __init__(self, n, params=None, method=None):
        from vapor_b200.abi import field_shapes_2d
        self.lib = _ref2d_lib()
        if n is None:
            self.h = self.lib.ref2r_create_app(int(method))
        else:
            self.h = self.lib.ref2r_create(int(n), None if params is None else C.byref(params))
        if not self.h:
            raise ValueError("the reference rejected the reflection solver")
        self.n = self.lib.ref2r_resolution(self.h)
        self.shapes = field_shapes_2d(self.n) + ((self.n, self.n),)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref2r_destroy(self.h)
            self.h = None

    @property
    def params(self):
        from vapor_b200.abi import Mac2DReflParams
        p = Mac2DReflParams()
        self.lib.ref2r_get_params(self.h, C.byref(p))
        return p

    @params.setter
    def params(self, p):
        self.lib.ref2r_set_params(self.h, C.byref(p))

    def reset(self):
        self.lib.ref2r_reset(self.h)

    def set_fields(self, smoke=None, u=None, v=None):
        keep = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (smoke, u, v)]
        self.lib.ref2r_set_fields(self.h, *[None if a is None else a.ctypes.data for a in keep])

    def advance(self, dt):
        return self.lib.ref2r_advance(self.h, dt)

    def fields(self):
        """smoke, u, v, pressure."""
        out = [np.zeros(s, np.float32) for s in self.shapes]
        self.lib.ref2r_get_fields(self.h, *[a.ctypes.data for a in out])
        return out

    def diagnostics(self):
        d = FluidDiagnostics()
        self.lib.ref2r_diagnostics(self.h, C.byref(d))
        return d


class RefHistorical2D:
    """The reference's historical 2D plume (tests/fixtures/Ba20987Smoke2D.hpp)
    with closed walls and no stirring, as its Historical2DTests.cpp runs it."""

    def __init__(self, n):
        from vapor_b200.abi import field_shapes_2d
        self.lib = _ref2d_lib()
        self.n = int(n)
        self.h = self.lib.ref2h_create(self.n)
        self.shapes = field_shapes_2d(self.n) + ((self.n, self.n),)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref2h_destroy(self.h)
            self.h = None

    def step(self, dt, buoyancy, dissipation, strength, iterations):
        self.lib.ref2h_step(self.h, dt, buoyancy, dissipation, strength, iterations)

    def fields(self):
        """smoke, u, v, pressure."""
        out = [np.zeros(s, np.float32) for s in self.shapes]
        self.lib.ref2h_get_fields(self.h, *[a.ctypes.data for a in out])
        return out


# ---- the reference's simplicial 3D solver with the drop-in backend
#      (oracle/_ref/libvapor_ref_simplicial.so) ----

SIMPLICIAL_SO = os.path.join(ROOT, "oracle", "_ref", "libvapor_ref_simplicial.so")
SIMPLICIAL_MESHES = os.path.join(ROOT, "oracle", "_ref", "meshes")
_simplicial = None


def simplicial_available():
    return os.path.exists(SIMPLICIAL_SO) and os.path.isdir(SIMPLICIAL_MESHES)


def _simplicial_lib():
    global _simplicial
    if _simplicial is None:
        lib = C.CDLL(SIMPLICIAL_SO)

        def f(name, res, *args):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = list(args)
        f("rs_error", C.c_char_p)
        f("rs_create", _vp, C.c_char_p, C.c_int, C.c_double)
        f("rs_destroy", None, _vp)
        f("rs_attach", C.c_int, _vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp)
        f("rs_counts", None, _vp, _vp)
        f("rs_set_potential", C.c_int, _vp, _vp)
        f("rs_advect_vorticity", C.c_int, _vp, C.c_double)
        f("rs_advance", C.c_int, _vp, C.c_float)
        f("rs_set_box_size", C.c_int, _vp, C.c_float)
        f("rs_reset", C.c_int, _vp)
        f("rs_set_parameters", None, _vp, C.c_int, C.c_float, C.c_int, C.c_double, C.c_double)
        for name in ("rs_vorticity", "rs_potential", "rs_flux", "rs_vertex_density", "rs_density",
                     "rs_edge_midpoints", "rs_diagnostics"):
            f(name, None, _vp, _vp)
        f("rs_last_recovery", None, _vp, _vp, _vp, _vp, _vp)
        f("rs_smoke_center", None, _vp, _vp)
        f("rs_substeps", C.c_int, _vp)
        f("rs_set_stir", None, _vp, C.c_float, C.c_float, C.c_float)
        f("rs_set_emitter", None, _vp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float)
        _simplicial = lib
    return _simplicial


class RefSimplicial:
    """The reference's SimplicialFluidSolver3D on one of its example meshes,
    with a compute backend: 0 the CPU path, 1 the CUDA stages, 2 the stages'
    arithmetic on the host with `partner`'s recovery, 3 the CUDA advection
    with `partner`'s recovery. search: 0 automatic, 1 scan, 2 descent; dots:
    the recovery's dot order, 0 automatic, 1 index order, 2 tree."""

    CPU, DEVICE, HOST_ADVECTION, DEVICE_ADVECTION = 0, 1, 2, 3

    def __init__(self, mesh="box.tet", box=True, size=1.0):
        self.lib = _simplicial_lib()
        self.h = self.lib.rs_create(os.path.join(SIMPLICIAL_MESHES, mesh).encode(), 1 if box else 0, size)
        if not self.h:
            raise ValueError(self.lib.rs_error().decode())
        c = (C.c_int * 5)()
        self.lib.rs_counts(self.h, c)
        self.n_vertices, self.n_edges, self.n_faces, self.n_tets, self.n_dual = list(c)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.rs_destroy(self.h)
            self.h = None

    def _ok(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.rs_error().decode())

    def attach(self, mode, search=0, partner=None, dots=0, jacobi=False):
        self._ok(self.lib.rs_attach(self.h, mode, search, dots, 1 if jacobi else 0,
                                    partner.h if partner is not None else None))

    def set_parameters(self, emitter=True, decay=0.08, cg_iterations=600, abs_tol=1e-10, rel_tol=1e-9):
        self.lib.rs_set_parameters(self.h, 1 if emitter else 0, decay, cg_iterations, abs_tol, rel_tol)

    def set_stir(self, strength, radius=.18, frequency=1.0):
        self.lib.rs_set_stir(self.h, strength, radius, frequency)

    def set_emitter(self, x, y, z, strength=4.0, radius=.12, buoyancy=3.0):
        self.lib.rs_set_emitter(self.h, x, y, z, strength, radius, buoyancy)

    def set_potential(self, phi):
        phi = np.ascontiguousarray(phi, np.float64)
        self._ok(self.lib.rs_set_potential(self.h, phi.ctypes.data))

    def advect_vorticity(self, dt):
        self._ok(self.lib.rs_advect_vorticity(self.h, dt))

    def advance(self, dt):
        self._ok(self.lib.rs_advance(self.h, dt))

    def set_box_size(self, size):
        self._ok(self.lib.rs_set_box_size(self.h, size))

    def reset(self):
        self._ok(self.lib.rs_reset(self.h))

    def _get(self, name, count, dtype):
        out = np.zeros(count, dtype)
        getattr(self.lib, name)(self.h, out.ctypes.data)
        return out

    def vorticity(self):
        return self._get("rs_vorticity", self.n_edges, np.float64)

    def potential(self):
        return self._get("rs_potential", self.n_edges, np.float64)

    def flux(self):
        return self._get("rs_flux", self.n_faces, np.float64)

    def vertex_density(self):
        return self._get("rs_vertex_density", self.n_vertices, np.float32)

    def density(self):
        return self._get("rs_density", self.n_tets, np.float32)

    def edge_ends(self):
        return self._get("rs_edge_midpoints", 6 * self.n_edges, np.float64).reshape(-1, 2, 3)

    def diagnostics(self):
        names = ("max_divergence", "max_boundary_flux", "kinetic_energy", "max_speed", "recovery_curl_error",
                 "smoke_mass")
        return dict(zip(names, self._get("rs_diagnostics", 6, np.float64)))

    def substeps(self):
        """CFL substeps of the last advance."""
        return self.lib.rs_substeps(self.h)

    def smoke_center(self):
        """(centre height, mass) of the tet smoke."""
        out = self._get("rs_smoke_center", 2, np.float64)
        return float(out[0]), float(out[1])

    def last_recovery(self):
        it, cv = C.c_int(), C.c_int()
        a, b = C.c_double(), C.c_double()
        self.lib.rs_last_recovery(self.h, C.byref(it), C.byref(cv), C.byref(a), C.byref(b))
        return {"iterations": it.value, "converged": bool(cv.value), "initial": a.value, "final": b.value}


def sine_potential(ref):
    """The seeded potential of the reference's GPU simplicial test
    (SimplicialGpu3DTests.cpp): sin(pi x/L) sin(pi y/L) sin(pi z/L) (b_z - a_z)
    at each edge's midpoint."""
    ends = ref.edge_ends()
    a, b = ends[:, 0], ends[:, 1]
    p = (a + b) * .5
    size = max(float(ends.max()), 1e-30)
    s = np.sin(np.pi * p / size)
    return s[:, 0] * s[:, 1] * s[:, 2] * (b[:, 2] - a[:, 2])
