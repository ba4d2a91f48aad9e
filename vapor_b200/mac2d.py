"""MAC 2D smoke solvers on the device, through the C ABI: the reference's
MacGridFluidSolver2D (src/solvers/mac2d/MacGridFluidSolver2D.cpp,
vapor_mac2d_*) and its compatibility ReflectionMacFluidSolver2D
(src/solvers/mac2d/ReflectionMacFluidSolver2D.hpp, vapor_mac2d_refl_*).
Fields are numpy arrays in the reference layout: density or smoke (n, n), u
(n, n + 1), v (n + 1, n), pressure (n, n), indexed [y, x]."""
import ctypes as C

import numpy as np

from . import check, library
from .abi import FluidDiagnostics, Mac2DParams, Mac2DReflParams, ProjectionResult, field_shapes_2d

_vp = C.c_void_p
_declared = False


def _lib():
    global _declared
    lib = library()
    if not _declared:
        def f(name, *args):
            fn = getattr(lib, name)
            fn.restype = C.c_int
            fn.argtypes = list(args)
        f("vapor_mac2d_default_params", C.POINTER(Mac2DParams))
        f("vapor_mac2d_plume_params", C.POINTER(Mac2DParams))
        f("vapor_mac2d_create", C.c_int32, C.c_float, C.POINTER(Mac2DParams), C.POINTER(_vp))
        f("vapor_mac2d_destroy", _vp)
        f("vapor_mac2d_get_params", _vp, C.POINTER(Mac2DParams))
        f("vapor_mac2d_set_params", _vp, C.POINTER(Mac2DParams))
        f("vapor_mac2d_advance", _vp, C.c_float)
        f("vapor_mac2d_reset", _vp)
        f("vapor_mac2d_set_box", _vp, C.c_float)
        f("vapor_mac2d_upload", _vp, _vp, _vp, _vp)
        f("vapor_mac2d_download", _vp, _vp, _vp, _vp)
        f("vapor_mac2d_last_projection", _vp, C.POINTER(ProjectionResult))
        f("vapor_mac2d_midpoint_projection", _vp, C.POINTER(ProjectionResult))
        f("vapor_mac2d_diagnostics", _vp, C.POINTER(FluidDiagnostics))
        R = C.POINTER(Mac2DReflParams)
        f("vapor_mac2d_refl_default_params", R)
        f("vapor_mac2d_refl_app_params", C.c_int32, R)
        f("vapor_mac2d_refl_create", C.c_int32, R, C.POINTER(_vp))
        f("vapor_mac2d_refl_destroy", _vp)
        f("vapor_mac2d_refl_get_params", _vp, R)
        f("vapor_mac2d_refl_set_params", _vp, R)
        f("vapor_mac2d_refl_advance", _vp, C.c_float)
        f("vapor_mac2d_refl_reset", _vp)
        f("vapor_mac2d_refl_upload", _vp, _vp, _vp, _vp)
        f("vapor_mac2d_refl_download", _vp, _vp, _vp, _vp, _vp)
        f("vapor_mac2d_refl_diagnostics", _vp, C.POINTER(FluidDiagnostics))
        _declared = True
    return lib


def default_params_2d():
    """MacGridParameters2D's defaults."""
    p = Mac2DParams()
    check(_lib().vapor_mac2d_default_params(C.byref(p)))
    return p


def plume_params_2d():
    """The scene of the reference's default-constructed 2D solver."""
    p = Mac2DParams()
    check(_lib().vapor_mac2d_plume_params(C.byref(p)))
    return p


class MacSimulation2D:
    def __init__(self, n, box=4.0, params=None):
        self.n = int(n)
        h = _vp()
        p = params if params is not None else default_params_2d()
        check(_lib().vapor_mac2d_create(self.n, float(box), C.byref(p), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().vapor_mac2d_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def params(self):
        p = Mac2DParams()
        check(_lib().vapor_mac2d_get_params(self._h, C.byref(p)))
        return p

    @params.setter
    def params(self, p):
        check(_lib().vapor_mac2d_set_params(self._h, C.byref(p)))

    def advance(self, dt):
        check(_lib().vapor_mac2d_advance(self._h, float(dt)))

    def reset(self):
        check(_lib().vapor_mac2d_reset(self._h))

    def set_box(self, box):
        check(_lib().vapor_mac2d_set_box(self._h, float(box)))

    def upload(self, density=None, u=None, v=None):
        arrays = []
        ptrs = []
        for a, shape in zip((density, u, v), field_shapes_2d(self.n)):
            if a is None:
                ptrs.append(None)
                continue
            a = np.ascontiguousarray(a, dtype=np.float32)
            if a.size != int(np.prod(shape)):
                raise ValueError(f"field needs shape {shape}")
            arrays.append(a)
            ptrs.append(a.ctypes.data)
        check(_lib().vapor_mac2d_upload(self._h, *ptrs))

    def download(self):
        out = [np.zeros(s, np.float32) for s in field_shapes_2d(self.n)]
        check(_lib().vapor_mac2d_download(self._h, *[a.ctypes.data for a in out]))
        return out

    def last_projection(self):
        r = ProjectionResult()
        check(_lib().vapor_mac2d_last_projection(self._h, C.byref(r)))
        return r

    def midpoint_projection(self):
        r = ProjectionResult()
        check(_lib().vapor_mac2d_midpoint_projection(self._h, C.byref(r)))
        return r

    def diagnostics(self):
        d = FluidDiagnostics()
        check(_lib().vapor_mac2d_diagnostics(self._h, C.byref(d)))
        return d


# ---- ReflectionMacFluidSolver2D ----

SEMI_LAGRANGIAN, MACCORMACK = 0, 1


def reflection_default_params():
    """The reflection solver's member initialisers (MacCormack smoke, 60
    iterations, emitter radius .08)."""
    p = Mac2DReflParams()
    check(_lib().vapor_mac2d_refl_default_params(C.byref(p)))
    return p


def reflection_app_params(method=SEMI_LAGRANGIAN):
    """The solver built from an advection method: resolution 128, emitter
    radius .04, 120 iterations (ReflectionMacFluidSolver2D.hpp:77-85)."""
    p = Mac2DReflParams()
    check(_lib().vapor_mac2d_refl_app_params(int(method), C.byref(p)))
    return p


class ReflectionSimulation2D:
    """The historical 2D plume on the unit box with a midpoint reflection every
    step; n in 2..512."""

    def __init__(self, n=128, params=None):
        self.n = int(n)
        h = _vp()
        p = params if params is not None else reflection_default_params()
        check(_lib().vapor_mac2d_refl_create(self.n, C.byref(p), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            _lib().vapor_mac2d_refl_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def params(self):
        p = Mac2DReflParams()
        check(_lib().vapor_mac2d_refl_get_params(self._h, C.byref(p)))
        return p

    @params.setter
    def params(self, p):
        check(_lib().vapor_mac2d_refl_set_params(self._h, C.byref(p)))

    def advance(self, dt):
        check(_lib().vapor_mac2d_refl_advance(self._h, float(dt)))

    def reset(self):
        """resetState(): zero fields, stirring stream back to the seed."""
        check(_lib().vapor_mac2d_refl_reset(self._h))

    def upload(self, smoke=None, u=None, v=None):
        arrays = []
        ptrs = []
        for a, shape in zip((smoke, u, v), field_shapes_2d(self.n)):
            if a is None:
                ptrs.append(None)
                continue
            a = np.ascontiguousarray(a, dtype=np.float32)
            if a.size != int(np.prod(shape)):
                raise ValueError(f"field needs shape {shape}")
            arrays.append(a)
            ptrs.append(a.ctypes.data)
        check(_lib().vapor_mac2d_refl_upload(self._h, *ptrs))

    def download(self):
        """smoke, u, v, pressure."""
        out = [np.zeros(s, np.float32) for s in field_shapes_2d(self.n) + ((self.n, self.n),)]
        check(_lib().vapor_mac2d_refl_download(self._h, *[a.ctypes.data for a in out]))
        return out

    def diagnostics(self):
        d = FluidDiagnostics()
        check(_lib().vapor_mac2d_refl_diagnostics(self._h, C.byref(d)))
        return d
