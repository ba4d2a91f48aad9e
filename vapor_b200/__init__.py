"""vapor_b200: B200-native MAC 3D smoke step (Simple and Reflection variants).

Python mirror of the reference's solver interface over the C ABI in
include/vapor_b200.h (the shared library vapor_b200/_lib/libvapor_b200.so,
built by vapor_b200._build). Names follow the reference:

  MacSimulation3D   GpuMacSimulation3D (src/solvers/mac3d/gpu/GpuMacSimulation3D.hpp:9-46):
                    advance / reset_state / set_box_size / parameters /
                    last_projection / upload / download / byte counters,
                    plus diagnostics() (MacGridFluidSolver3D.cpp:332-334)
  StageBackend      the staged Projection3D / Advection3D plugins
                    (Projection3D.hpp:6-11, Advection3D.hpp:6-14)

Errors raise the reference's exception types: ValueError for
std::invalid_argument (VAPOR_INVALID_ARGUMENT / VAPOR_NON_FINITE),
OverflowError for std::length_error, RuntimeError for backend failures.
There is no CPU fallback: without the built library or a B200 device every
call fails.
"""
import ctypes as C
import os

import numpy as np

from . import abi
from .abi import (FluidDiagnostics, LinearSolveOptions, MacParams, ProjectionOptions, ProjectionResult,
                  field_shapes, field_sizes)

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "_lib", "libvapor_b200.so")

_lib = None


class VaporError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"[{status}] {message}")
        self.status = status


class InvalidArgument(VaporError, ValueError):
    pass


class LengthError(VaporError, OverflowError):
    pass


class NonFinite(InvalidArgument):
    pass


class OutOfMemory(VaporError, MemoryError):
    pass


_ERRORS = {abi.VAPOR_INVALID_ARGUMENT: InvalidArgument, abi.VAPOR_LENGTH_ERROR: LengthError,
           abi.VAPOR_NON_FINITE: NonFinite, abi.VAPOR_OUT_OF_MEMORY: OutOfMemory}

_vp = C.c_void_p
_fp = C.POINTER(C.c_float)


def _declare(lib):
    def f(name, *args, res=C.c_int):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)
    f("vapor_last_error", res=C.c_char_p)
    f("vapor_abi_version", res=C.c_int32)
    f("vapor_kernel_launch_count", res=C.c_int64)
    f("vapor_set_device", C.c_int32)
    f("vapor_mac3d_default_params", C.POINTER(MacParams))
    f("vapor_mac3d_algorithm_params", C.c_int32, C.POINTER(MacParams))
    f("vapor_default_projection_options", C.POINTER(ProjectionOptions))
    f("vapor_mac3d_create", C.c_int32, C.c_float, C.POINTER(MacParams), C.POINTER(_vp))
    f("vapor_mac3d_destroy", _vp)
    f("vapor_mac3d_reset", _vp)
    f("vapor_mac3d_set_box", _vp, C.c_float)
    f("vapor_mac3d_get_params", _vp, C.POINTER(MacParams))
    f("vapor_mac3d_set_params", _vp, C.POINTER(MacParams))
    f("vapor_mac3d_advance", _vp, C.c_float)
    f("vapor_mac3d_advance_n", _vp, C.c_float, C.c_int32)
    f("vapor_mac3d_synchronize", _vp)
    f("vapor_mac3d_last_projection", _vp, C.POINTER(ProjectionResult))
    f("vapor_mac3d_total_iterations", _vp, C.POINTER(C.c_int64))
    f("vapor_mac3d_diagnostics", _vp, C.POINTER(FluidDiagnostics))
    f("vapor_mac3d_comparison_metrics", _vp, C.c_float, C.POINTER(abi.ComparisonMetrics))
    f("vapor_mac3d_render", _vp, C.POINTER(abi.RenderParams), _vp)
    f("vapor_render_volume", _vp, C.c_int32, C.c_float, C.POINTER(abi.RenderParams), _vp, _vp)
    f("vapor_mac3d_upload", _vp, _vp, _vp, _vp, _vp)
    f("vapor_mac3d_download", _vp, _vp, _vp, _vp, _vp)
    f("vapor_mac3d_upload_async", _vp, _vp, _vp, _vp, _vp)
    f("vapor_mac3d_download_async", _vp, _vp, _vp, _vp, _vp)
    f("vapor_mac3d_wait_transfers", _vp)
    f("vapor_mac3d_byte_counters", _vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64))
    f("vapor_mac3d_device_fields", _vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp))
    f("vapor_mac3d_stream", _vp, C.POINTER(_vp))
    f("vapor_mac3d_resolution", _vp, C.POINTER(C.c_int32), C.POINTER(C.c_float))
    f("vapor_mac3d_set_timing", _vp, C.c_int32)
    f("vapor_mac3d_timings", _vp, C.POINTER(abi.PhaseTimings))
    f("vapor_stage_create", C.c_int32, C.c_float, C.POINTER(_vp))
    f("vapor_stage_destroy", _vp)
    f("vapor_stage_reset", _vp)
    f("vapor_stage_project", _vp, _vp, _vp, _vp, C.POINTER(ProjectionOptions), C.c_float,
      C.POINTER(ProjectionResult), _vp)
    f("vapor_stage_project_device", _vp, _vp, _vp, _vp, C.POINTER(ProjectionOptions), C.c_float,
      C.POINTER(ProjectionResult), _vp)
    f("vapor_stage_advect_face", _vp, C.c_int32, C.c_float, C.c_float, C.c_int32, _vp, _vp, _vp, _vp, _vp)
    f("vapor_stage_advect_face_device", _vp, C.c_int32, C.c_float, C.c_float, C.c_int32, _vp, _vp, _vp, _vp, _vp)
    f("vapor_stage_advect_scalar", _vp, C.c_float, C.c_float, C.c_int32, _vp, _vp, _vp, _vp)
    f("vapor_stage_advect_scalar_device", _vp, C.c_float, C.c_float, C.c_int32, _vp, _vp, _vp, _vp)
    f("vapor_stage_set_solver_kind", _vp, C.c_int32)
    f("vapor_stage_stream", _vp, C.POINTER(_vp))
    f("vapor_stage_set_solid", _vp, _vp)
    f("vapor_stage_solve_rhs", _vp, _vp, C.POINTER(ProjectionOptions), C.c_float, C.POINTER(ProjectionResult), _vp)
    f("vapor_mac3d_set_coarse_log", _vp, _vp, C.c_int32, _vp)
    f("vapor_tune_sor_planes", C.c_int32, C.c_int32)
    f("vapor_tune_sor_blocking", C.c_int32)
    f("vapor_tune_sor_blocked_chunks", C.c_int32, C.c_int32)
    f("vapor_tune_conv_kernel", C.c_int32)
    f("vapor_tune_fpcg_smoothing", C.c_int32, C.c_float)
    f("vapor_tune_wgrad_kernel", C.c_int32)
    f("vapor_fpcg_smoothing", C.POINTER(C.c_int32), C.POINTER(C.c_float))
    f("vapor_batch_create", C.c_int32, C.POINTER(_vp), C.POINTER(_vp))
    f("vapor_batch_destroy", _vp)
    f("vapor_batch_advance", _vp, C.c_float)
    f("vapor_batch_synchronize", _vp)
    f("vapor_batch_stream", _vp, C.POINTER(_vp))
    f("vapor_advect_noalloc", C.c_int32, C.c_float, C.c_int32, C.c_float, C.c_float, C.c_int32,
      _vp, _vp, _vp, _vp, _vp, _vp)
    f("vapor_unet_parameter_count", res=C.c_int64)
    f("vapor_unet_create", C.POINTER(_vp))
    f("vapor_unet_destroy", _vp)
    f("vapor_unet_init", _vp, C.c_uint32)
    f("vapor_unet_set_parameters", _vp, _vp, C.c_int64)
    f("vapor_unet_get_parameters", _vp, _vp, C.c_int64)
    f("vapor_unet_forward_features", _vp, C.c_int32, _vp, _vp)
    f("vapor_unet_backward", _vp, C.c_int32, _vp, _vp)
    f("vapor_unet_set_wait_probe", _vp, C.c_int32)
    f("vapor_mac3d_set_warm_start", _vp, _vp)
    f("vapor_mac3d_train_warm_start", _vp, _vp, C.c_float, C.POINTER(C.c_double))
    f("vapor_mac3d_evaluate_warm_start", _vp, _vp, C.POINTER(C.c_double))
    f("vapor_mac3d_set_preconditioner", _vp, _vp)
    f("vapor_mac3d_set_solid", _vp, _vp)
    f("vapor_stage_set_preconditioner", _vp, _vp)
    f("vapor_stage_train_network", _vp, _vp, C.c_float, C.POINTER(C.c_double))
    return lib


def library():
    """The loaded C library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBRARY_PATH):
            raise RuntimeError(f"vapor_b200 CUDA library not built: {LIBRARY_PATH} "
                               "(run vapor_b200._build.build())")
        _lib = _declare(C.CDLL(LIBRARY_PATH))
        if _lib.vapor_abi_version() != abi.ABI_VERSION:
            raise RuntimeError("vapor_b200 library ABI version mismatch")
    return _lib


def check(status):
    if status != abi.VAPOR_OK:
        msg = library().vapor_last_error().decode(errors="replace")
        raise _ERRORS.get(status, VaporError)(status, msg)


def set_device(device):
    """Select the CUDA device for handles created afterwards on this thread."""
    check(library().vapor_set_device(int(device)))


def kernel_launch_count():
    """Kernels launched by the library so far (exact counter)."""
    return library().vapor_kernel_launch_count()


def default_params():
    p = MacParams()
    check(library().vapor_mac3d_default_params(C.byref(p)))
    return p


def algorithm_params(algorithm):
    p = MacParams()
    check(library().vapor_mac3d_algorithm_params(algorithm, C.byref(p)))
    return p


def default_projection_options():
    o = ProjectionOptions()
    check(library().vapor_default_projection_options(C.byref(o)))
    return o


def _host(a, n_expected, writable=False):
    if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous:
        raise TypeError("fields must be C-contiguous float32 numpy arrays")
    if a.size != n_expected:
        raise InvalidArgument(abi.VAPOR_INVALID_ARGUMENT, "field size does not match the grid layout")
    if writable and not a.flags.writeable:
        raise TypeError("output array is read-only")
    return a.ctypes.data


class MacSimulation3D:
    """Resident MAC 3D simulation on one B200 (GpuMacSimulation3D's interface).

    MacSimulation3D(algorithm) builds the reference's 32^3, box 4.5 preset;
    MacSimulation3D(n, box, params) takes an explicit grid and parameters.
    """

    def __init__(self, n_or_algorithm, box=None, params=None):
        lib = library()
        if box is None and params is None:
            params = algorithm_params(n_or_algorithm)
            n, box = 32, 4.5
        else:
            n = n_or_algorithm
            params = params if params is not None else default_params()
        self.n = int(n)
        self._in_flight = []  # host arrays of streamed transfers not yet waited for
        h = _vp()
        check(lib.vapor_mac3d_create(self.n, float(box), C.byref(params), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            library().vapor_mac3d_destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # parameters() -> mutable copy; assign back with set_parameters
    def parameters(self):
        p = MacParams()
        check(library().vapor_mac3d_get_params(self._h, C.byref(p)))
        return p

    def set_parameters(self, p):
        check(library().vapor_mac3d_set_params(self._h, C.byref(p)))

    def advance(self, dt, steps=1):
        if steps == 1:
            check(library().vapor_mac3d_advance(self._h, float(dt)))
        else:
            check(library().vapor_mac3d_advance_n(self._h, float(dt), int(steps)))

    def synchronize(self):
        check(library().vapor_mac3d_synchronize(self._h))

    def reset_state(self):
        check(library().vapor_mac3d_reset(self._h))

    def set_box_size(self, box):
        check(library().vapor_mac3d_set_box(self._h, float(box)))

    @property
    def box_size(self):
        n, b = C.c_int32(), C.c_float()
        check(library().vapor_mac3d_resolution(self._h, C.byref(n), C.byref(b)))
        return b.value

    def last_projection(self):
        r = ProjectionResult()
        check(library().vapor_mac3d_last_projection(self._h, C.byref(r)))
        return r

    def total_iterations(self):
        v = C.c_int64()
        check(library().vapor_mac3d_total_iterations(self._h, C.byref(v)))
        return v.value

    def diagnostics(self):
        d = FluidDiagnostics()
        check(library().vapor_mac3d_diagnostics(self._h, C.byref(d)))
        return d

    def render(self, params=None):
        """Headless ray-marched image of the current density (the reference's
        volume shader): a (height, width, 3) float32 array, row 0 at the
        bottom. params: abi.RenderParams (default: the harness's 960 x 960)."""
        params = params or abi.RenderParams.harness()
        rgb = np.empty((params.height, params.width, 3), np.float32)
        check(library().vapor_mac3d_render(self._h, C.byref(params), rgb.ctypes.data))
        return rgb

    def comparison_metrics(self, frames_per_second=60.0):
        """The reference harness's comparison metrics of the current state
        (mass, gradient and square per mass, rms and max divergence, smoke
        cells and their CFL / boundary fallbacks, max CFL), on the device."""
        m = abi.ComparisonMetrics()
        check(library().vapor_mac3d_comparison_metrics(self._h, float(frames_per_second), C.byref(m)))
        return m.as_dict()

    def upload(self, density, u, v, w):
        sizes = field_sizes(self.n)
        ptrs = [_host(a, s) for a, s in zip((density, u, v, w), sizes)]
        check(library().vapor_mac3d_upload(self._h, *ptrs))

    def download(self, out=None):
        if out is None:
            out = [np.empty(s, np.float32) for s in field_shapes(self.n)]
        sizes = field_sizes(self.n)
        ptrs = [_host(a, s, writable=True) for a, s in zip(out, sizes)]
        check(library().vapor_mac3d_download(self._h, *ptrs))
        return out

    def upload_async(self, density, u, v, w):
        """Stage a host snapshot on a copy stream; the next advance takes it
        in. The arrays (pinned for full overlap) are kept referenced and must
        stay unchanged until wait_transfers()."""
        sizes = field_sizes(self.n)
        arrays = (density, u, v, w)
        ptrs = [_host(a, s) for a, s in zip(arrays, sizes)]
        check(library().vapor_mac3d_upload_async(self._h, *ptrs))
        self._in_flight.extend(arrays)

    def download_async(self, out):
        """Snapshot the state after the steps issued so far and copy it into
        `out` (four float32 arrays, pinned for full overlap) on a copy stream;
        read `out` only after wait_transfers()."""
        sizes = field_sizes(self.n)
        ptrs = [_host(a, s, writable=True) for a, s in zip(out, sizes)]
        check(library().vapor_mac3d_download_async(self._h, *ptrs))
        self._in_flight.extend(out)
        return out

    def wait_transfers(self):
        """Block until every staged upload and download has finished."""
        check(library().vapor_mac3d_wait_transfers(self._h))
        self._in_flight = []

    def byte_counters(self):
        up, down = C.c_uint64(), C.c_uint64()
        check(library().vapor_mac3d_byte_counters(self._h, C.byref(up), C.byref(down)))
        return up.value, down.value

    def device_fields(self):
        ptrs = [_vp() for _ in range(4)]
        check(library().vapor_mac3d_device_fields(self._h, *[C.byref(p) for p in ptrs]))
        return [p.value for p in ptrs]

    def stream(self):
        s = _vp()
        check(library().vapor_mac3d_stream(self._h, C.byref(s)))
        return s.value

    def set_timing(self, enabled):
        check(library().vapor_mac3d_set_timing(self._h, int(bool(enabled))))

    def timings(self):
        t = abi.PhaseTimings()
        check(library().vapor_mac3d_timings(self._h, C.byref(t)))
        return t.as_dict()

    # ---- learned warm start (vapor_b200.learned.WarmStartNet) ----
    def set_warm_start(self, net):
        """Initial guess of every later projection from `net` (None: zero)."""
        check(library().vapor_mac3d_set_warm_start(self._h, net.handle if net is not None else None))
        self._warm = net  # the network must outlive its use here

    def train_warm_start(self, net, learning_rate):
        """One Adam step of `net` on the last projection; returns the loss
        (relative squared error of the mean-free prediction) before it."""
        loss = C.c_double()
        check(library().vapor_mac3d_train_warm_start(self._h, net.handle, float(learning_rate), C.byref(loss)))
        return loss.value

    def evaluate_warm_start(self, net):
        loss = C.c_double()
        check(library().vapor_mac3d_evaluate_warm_start(self._h, net.handle, C.byref(loss)))
        return loss.value

    def set_coarse_log(self, log_ptr, capacity, counter_ptr):
        """Copies every FPCG coarse right-hand side into a device ring (0/None disables)."""
        check(library().vapor_mac3d_set_coarse_log(self._h, log_ptr or None, int(capacity), counter_ptr or None))

    def set_preconditioner(self, net):
        """Learned coarse-grid correction of the FPCG solver (None: smoothing only)."""
        check(library().vapor_mac3d_set_preconditioner(self._h, net.handle if net is not None else None))
        self._coarse = net

    def set_solid(self, mask):
        """Obstacles for every later projection of the steps: n^3 uint8 mask
        (z, y, x order, nonzero = solid) or None. Needs the mixed-precision
        solver."""
        if mask is None:
            check(library().vapor_mac3d_set_solid(self._h, None))
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.size != self.n ** 3:
            raise ValueError(f"mask needs {self.n ** 3} cells")
        check(library().vapor_mac3d_set_solid(self._h, m.ctypes.data))


def tune_sor_planes(n, planes):
    """z-planes per thread of the colour sweep for grids of size n (0: automatic)."""
    check(library().vapor_tune_sor_planes(int(n), int(planes)))


def tune_sor_blocking(iterations_per_launch):
    """Red+black iterations per temporally blocked sweep launch (1 or 2; 0,
    the default: one launch per colour). Same results either way."""
    check(library().vapor_tune_sor_blocking(int(iterations_per_launch)))


# Convolution kernel and FPCG smoothing the library starts with (the measured
# fastest on the 256^3 benchmark plume).
DEFAULT_CONV_KERNEL = 3
DEFAULT_FPCG_SMOOTHING = (2, 1.2)


def tune_conv_kernel(kind):
    """tcgen05 convolution kernel: 0 block-synchronous z-march, 1 its
    warp-specialised form, 2 the plane-window form (three output planes per
    MMA), 3 (default) the plane-window form fed by TMA (same results as 2;
    grids under 10 x 18 voxels run 0)."""
    check(library().vapor_tune_conv_kernel(int(kind)))


def tune_fpcg_smoothing(sweeps=DEFAULT_FPCG_SMOOTHING[0], omega=DEFAULT_FPCG_SMOOTHING[1]):
    """Relaxation sweeps before and after the FPCG preconditioner's coarse
    correction (default 2) and their weight (default 1.2). Set it before
    creating the simulations whose steps are recorded."""
    check(library().vapor_tune_fpcg_smoothing(int(sweeps), float(omega)))


def tune_wgrad_kernel(kind):
    """Weight-gradient kernel of the network's training: 1 (default) tcgen05,
    0 the CUDA-core form (equal to FP32 rounding)."""
    check(library().vapor_tune_wgrad_kernel(int(kind)))


def fpcg_smoothing():
    """(sweeps, omega) of the FPCG preconditioner's smoothing."""
    sw, om = C.c_int32(), C.c_float()
    check(library().vapor_fpcg_smoothing(C.byref(sw), C.byref(om)))
    return sw.value, om.value


def fpcg_sweeps_per_application():
    """Red+black sweeps in one application of the FPCG preconditioner."""
    return 2 * fpcg_smoothing()[0]


def tune_sor_blocked_chunks(n, chunks):
    """z chunks per blocked sweep launch for grids of size n (0: automatic)."""
    check(library().vapor_tune_sor_blocked_chunks(int(n), int(chunks)))


class Batch:
    """Steps several MacSimulation3D scenes with one CUDA-graph launch."""

    def __init__(self, sims):
        self.sims = list(sims)  # keeps the scenes alive while batched
        arr = (_vp * len(self.sims))(*[s.handle for s in self.sims])
        h = _vp()
        check(library().vapor_batch_create(len(self.sims), arr, C.byref(h)))
        self._h = h

    def advance(self, dt):
        check(library().vapor_batch_advance(self._h, float(dt)))

    def synchronize(self):
        check(library().vapor_batch_synchronize(self._h))

    def stream(self):
        s = _vp()
        check(library().vapor_batch_stream(self._h, C.byref(s)))
        return s.value

    def close(self):
        if getattr(self, "_h", None):
            library().vapor_batch_destroy(self._h)
            self._h = None

    __del__ = close


class StageBackend:
    """Staged Projection3D / Advection3D plugins over host (numpy) spans."""

    def __init__(self, n, box):
        self.n = int(n)
        h = _vp()
        check(library().vapor_stage_create(self.n, float(box), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            library().vapor_stage_destroy(self._h)
            self._h = None

    __del__ = close

    def reset(self):
        check(library().vapor_stage_reset(self._h))

    def set_solver_kind(self, kind):
        check(library().vapor_stage_set_solver_kind(self._h, int(kind)))

    def set_solid(self, mask):
        """Solid obstacles: n^3 uint8 mask (z, y, x order, nonzero = solid) or None."""
        if mask is None:
            check(library().vapor_stage_set_solid(self._h, None))
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.size != self.n ** 3:
            raise ValueError(f"mask needs {self.n ** 3} cells")
        check(library().vapor_stage_set_solid(self._h, m.ctypes.data))

    def set_preconditioner(self, net):
        """Coarse-grid network of the FPCG solver (None: smoothing only)."""
        check(library().vapor_stage_set_preconditioner(self._h, net.handle if net is not None else None))
        self._coarse = net

    def train_network(self, net, learning_rate):
        """One Adam step of `net` on this stage's last projection; returns the loss."""
        loss = C.c_double()
        check(library().vapor_stage_train_network(self._h, net.handle, float(learning_rate), C.byref(loss)))
        return loss.value

    def project(self, u, v, w, options, diagonal_floor=0.0, want_pressure=False):
        """Projection3D::project in place on (u, v, w); returns (result, pressure)."""
        f = field_sizes(self.n)[1]
        ptrs = [_host(a, f, writable=True) for a in (u, v, w)]
        r = ProjectionResult()
        p = np.empty((self.n,) * 3, np.float32) if want_pressure else None
        check(library().vapor_stage_project(self._h, *ptrs, C.byref(options), float(diagonal_floor), C.byref(r),
                                            p.ctypes.data if p is not None else None))
        return r, p

    def solve_rhs(self, rhs_ptr, options, diagonal_floor=6.0, pressure_ptr=None):
        """Mixed-precision solve of A x = rhs (device pointer, n^3 floats); returns the result."""
        r = ProjectionResult()
        check(library().vapor_stage_solve_rhs(self._h, rhs_ptr, C.byref(options), float(diagonal_floor), C.byref(r),
                                              pressure_ptr))
        return r

    def project_device(self, u_ptr, v_ptr, w_ptr, options, diagonal_floor=0.0, pressure_ptr=None):
        """The same projection on device pointers (in place); returns the result."""
        r = ProjectionResult()
        check(library().vapor_stage_project_device(self._h, u_ptr, v_ptr, w_ptr, C.byref(options),
                                                   float(diagonal_floor), C.byref(r), pressure_ptr))
        return r

    def advect_face(self, axis, dt, cfl, method, source, flow, output):
        f = field_sizes(self.n)[1]
        ptrs = [_host(a, f) for a in (source,) + tuple(flow)]
        out = _host(output, f, writable=True)
        check(library().vapor_stage_advect_face(self._h, int(axis), float(dt), float(cfl), int(method), ptrs[0],
                                                ptrs[1], ptrs[2], ptrs[3], out))

    def advect_scalar(self, dt, cfl, method, field, flow):
        c, f = field_sizes(self.n)[:2]
        fp = _host(field, c, writable=True)
        ptrs = [_host(a, f) for a in flow]
        check(library().vapor_stage_advect_scalar(self._h, float(dt), float(cfl), int(method), fp, *ptrs))


__all__ = ["MacSimulation3D", "StageBackend", "MacParams", "ProjectionOptions", "LinearSolveOptions",
           "ProjectionResult", "FluidDiagnostics", "default_params", "algorithm_params",
           "default_projection_options", "library", "check", "VaporError", "InvalidArgument", "LengthError",
           "NonFinite", "OutOfMemory", "field_shapes", "field_sizes", "LIBRARY_PATH"]
