/*
 * vapor_b200 — C ABI of the B200-native MAC 3D smoke step.
 *
 * This is the drop-in boundary for Vapor's MAC 3D hot path. It replaces the
 * OpenGL compute coordinator and the two stage plugins of the reference:
 *
 *   reference interface (taehwann/vapor)                      replaced by
 *   ------------------------------------------------------    ---------------------------
 *   GpuMacSimulation3D ctor/advance/resetState/setBoxSize/     vapor_mac3d_*      (resident)
 *     parameters/lastProjection/upload/download/byte counters
 *     src/solvers/mac3d/gpu/GpuMacSimulation3D.hpp:9-46
 *   MacGridFluidSolver3D::diagnostics                          vapor_mac3d_diagnostics
 *     src/solvers/mac3d/MacGridFluidSolver3D.cpp:332-334
 *   Projection3D::project / reset                              vapor_stage_project
 *     src/solvers/mac3d/Projection3D.hpp:6-11                  vapor_stage_reset
 *   Advection3D::advectScalar / advectFace                     vapor_stage_advect_scalar
 *     src/solvers/mac3d/Advection3D.hpp:6-14                   vapor_stage_advect_face
 *
 * Conventions
 *   - Every entry point returns a vapor_status; VAPOR_OK is 0. No C++
 *     exception crosses this boundary. vapor_last_error() returns the message
 *     of the last failure on the calling thread.
 *   - The reference throws std::invalid_argument for contract violations,
 *     std::length_error for index overflow and std::runtime_error for backend
 *     failures; these map to VAPOR_INVALID_ARGUMENT, VAPOR_LENGTH_ERROR and
 *     VAPOR_RUNTIME_ERROR.
 *   - Fields use the reference's MAC layout (MacGridDomain3D.hpp:22-31), FP32,
 *     x fastest: density n^3 at x+n(y+nz); u (n+1)n^2 at x+(n+1)(y+nz);
 *     v n(n+1)n at x+n(y+(n+1)z); w n^2(n+1) at x+n(y+nz), z in [0,n].
 *   - Axis convention is the reference's: z is up (buoyancy acts on w).
 *   - A handle owns one CUDA stream and all of its device buffers. A handle is
 *     not thread-safe; distinct handles may be used concurrently.
 *   - Host pointers passed to upload/download/stage calls may be pageable or
 *     pinned; pinned memory makes the copies asynchronous-capable and faster.
 */
#ifndef VAPOR_B200_H
#define VAPOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VAPOR_B200_ABI_VERSION 1

typedef enum vapor_status {
    VAPOR_OK = 0,
    VAPOR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
    VAPOR_LENGTH_ERROR = 2,     /* std::length_error (index range overflow) */
    VAPOR_RUNTIME_ERROR = 3,    /* std::runtime_error (CUDA failure, no device) */
    VAPOR_NON_FINITE = 4,       /* non-finite divergence or velocity found on the device;
                                   the reference throws std::invalid_argument here */
    VAPOR_OUT_OF_MEMORY = 5
} vapor_status;

/* MacAlgorithm (src/common/MacAlgorithm.hpp:3-9). */
typedef enum vapor_mac_algorithm {
    VAPOR_SIMPLE_SEMI_LAGRANGIAN = 0,
    VAPOR_SIMPLE_MACCORMACK = 1,
    VAPOR_REFLECTION_SEMI_LAGRANGIAN = 2,
    VAPOR_REFLECTION_MACCORMACK = 3
} vapor_mac_algorithm;

/* AdvectionMethod (src/common/MacAlgorithm.hpp:10). */
typedef enum vapor_advection_method {
    VAPOR_SEMI_LAGRANGIAN = 0,
    VAPOR_MACCORMACK = 1
} vapor_advection_method;

/* FaceAxis (src/solvers/mac3d/AdvectionContext.hpp:9). */
typedef enum vapor_face_axis { VAPOR_FACE_X = 0, VAPOR_FACE_Y = 1, VAPOR_FACE_Z = 2 } vapor_face_axis;

/* Pressure solver kinds. RED_BLACK_SOR is the reference's SOR (SOR.cpp:22-64)
 * with its red-black colour order, so iterates match it exactly. The other
 * kinds are extensions that always finish with the same residual test. */
typedef enum vapor_solver_kind {
    VAPOR_SOLVER_RED_BLACK_SOR = 0,
    VAPOR_SOLVER_MIXED_REFINEMENT = 1, /* FP32 SOR inner sweeps, FP64 residual and correction */
    /* Flexible PCG: FP32 vectors, FP64 dot products, FP64 residual and
     * re-centring. Preconditioner: 2 red-black Gauss-Seidel sweeps, the
     * learned coarse-grid correction when a network is attached
     * (vapor_mac3d_set_preconditioner / vapor_stage_set_preconditioner), then
     * 2 sweeps in reverse colour order. Iterations count CG steps. */
    VAPOR_SOLVER_FPCG = 2
} vapor_solver_kind;

/* LinearSolveOptions / LinearSolveResult (src/common/LinearSolveOptions.hpp:4-24). */
typedef struct vapor_linear_solve_options {
    int32_t max_iterations;          /* default 200 */
    int32_t residual_check_interval; /* default 8 */
    double absolute_tolerance;       /* default 1e-6 */
    double relative_tolerance;       /* default 1e-5 */
    int32_t fixed_iterations;        /* default 0 (stop at tolerance) */
    int32_t reserved0;
} vapor_linear_solve_options;

typedef struct vapor_linear_solve_result {
    int32_t iterations;
    int32_t converged;
    double initial_residual; /* FP64 infinity norm of b - A x0 */
    double final_residual;   /* FP64 infinity norm of b - A x after the mean gauge */
} vapor_linear_solve_result;

/* ProjectionOptions / ProjectionResult (src/common/ProjectionOptions.hpp:5-18). */
typedef struct vapor_projection_options {
    float dt;         /* default 1/60 */
    float relaxation; /* SOR omega, default 1.95 */
    vapor_linear_solve_options linear_solve;
} vapor_projection_options;

typedef struct vapor_projection_result {
    vapor_linear_solve_result linear_solve;
    int32_t residual_available; /* always 1: the residual is measured in FP64 */
    float divergence_before;    /* max |div u| before projection */
    float divergence_after;     /* max |div u| after projection */
    int32_t reserved0;
    double removed_rhs_mean;
} vapor_projection_result;

/* FluidDiagnostics (src/common/FluidDiagnostics.hpp:3-7). */
typedef struct vapor_fluid_diagnostics {
    float kinetic_energy;
    float max_velocity;
    float max_divergence;
} vapor_fluid_diagnostics;

/*
 * MacGridParameters3D (src/solvers/mac3d/MacGridFluidSolver3D.hpp:14-36), field
 * for field, followed by extensions the reference does not have. With the
 * extensions at their defaults the step is the reference's step.
 */
typedef struct vapor_mac3d_params {
    float emitter_radius;            /* .035 (fraction of box) */
    float emitter_center_x;          /* .5 */
    float emitter_center_y;          /* .5 */
    float emitter_center_z;          /* .1 (z is up) */
    float emitter_kick_multiplier;   /* 1 */
    float emitter_kick_base;         /* .8 */
    float emitter_kick_scale;        /* .8 */
    float stir_strength;             /* .5 */
    uint32_t random_seed;            /* 0x9E3779B9, applied at construction and reset */
    float sor_omega;                 /* 1.95 */
    float buoyancy_split;            /* .5 */
    float cfl_mc;                    /* 3 */
    int32_t mac_cormack_smoke;       /* 1 */
    int32_t mac_cormack_vel;         /* 1 */
    float smoke_decay;               /* .06 */
    int32_t reflection;              /* 1 */
    float buoyancy;                  /* 2.5 */
    float source_strength;           /* 1 */
    int32_t project_iterations;      /* 64 */

    /* ---- extensions (no reference counterpart) ---- */
    /* 0: projections run project_iterations fixed sweeps (reference semantics,
     *    MacGridFluidSolver3D.cpp:131-138). 1: projections use `solve`. */
    int32_t use_solve_options;
    vapor_linear_solve_options solve;
    int32_t solver_kind;             /* vapor_solver_kind */
    /* 0: reference emitter (density = 1 inside the sphere, kick, stir).
     * 1: smooth profile density = max(density, min(1, 3 s exp(-3.5 (d/r)^2))). */
    int32_t emitter_profile;
    int32_t emitter_count;           /* 1 or 2 */
    float emitter2_center_x, emitter2_center_y, emitter2_center_z;
} vapor_mac3d_params;

/* Per-phase device timings of a handle, accumulated between enabling timing
 * and reading it (CUDA events on the handle's stream; the analogue of the
 * reference's TimedAdvection/TimedPressure wrappers, tests/GpuPerformance.cpp:14-44).
 * Index the arrays with vapor_phase. `launches` counts kernel launches and
 * `cells` the grid cells each launch covers (for bytes-per-cell rooflines). */
typedef enum vapor_phase {
    VAPOR_PHASE_FORCING = 0,   /* emit, buoyancy, walls */
    VAPOR_PHASE_ADVECT = 1,    /* velocity and smoke transport */
    VAPOR_PHASE_RHS = 2,       /* divergence, right-hand side, mean */
    VAPOR_PHASE_SOR = 3,       /* red-black colour sweeps */
    VAPOR_PHASE_RESIDUAL = 4,  /* FP64 residual checks and re-centring */
    VAPOR_PHASE_GRADIENT = 5,  /* pressure gauge, final residual, gradient, divergence after */
    VAPOR_PHASE_KRYLOV = 6,    /* FPCG: A p, dot products, vector updates */
    VAPOR_PHASE_COARSE = 7,    /* FPCG: restriction, network, Galerkin scale, prolongation */
    VAPOR_PHASE_COUNT = 8
} vapor_phase;

typedef struct vapor_phase_timings {
    double milliseconds[VAPOR_PHASE_COUNT];
    int64_t launches[VAPOR_PHASE_COUNT];
    int64_t intervals[VAPOR_PHASE_COUNT]; /* timed event pairs */
} vapor_phase_timings;

/* Error message of the last failing call on this thread ("" if none). */
const char *vapor_last_error(void);
/* VAPOR_B200_ABI_VERSION of the loaded library. */
int32_t vapor_abi_version(void);
/* Kernels launched by this library so far (all handles, all threads). */
int64_t vapor_kernel_launch_count(void);
/* Select the CUDA device for handles created afterwards on this thread
 * (one process per GPU: pass the local rank). */
vapor_status vapor_set_device(int32_t device);

/* Defaults of MacGridParameters3D() and of MacGridParameters3D(MacAlgorithm)
 * (MacGridFluidSolver3D.cpp:11-26). */
vapor_status vapor_mac3d_default_params(vapor_mac3d_params *out);
vapor_status vapor_mac3d_algorithm_params(int32_t algorithm, vapor_mac3d_params *out);
vapor_status vapor_default_projection_options(vapor_projection_options *out);

/* ------------------------------------------------------------------------ */
/* Resident coordinator: GpuMacSimulation3D (gpu/GpuMacSimulation3D.hpp:9-46) */
/* ------------------------------------------------------------------------ */
typedef struct vapor_mac3d vapor_mac3d;

/* GpuMacSimulation3D(int, float, MacGridParameters3D) (GpuMacSimulation3D.cpp:49-63).
 * Validates the grid like MacGridDomain3D (MacGridDomain3D.cpp:7-22), allocates
 * every buffer on the current device and resets the state. */
vapor_status vapor_mac3d_create(int32_t n, float box, const vapor_mac3d_params *params,
                                vapor_mac3d **out);
vapor_status vapor_mac3d_destroy(vapor_mac3d *sim);
/* resetState (GpuMacSimulation3D.cpp:89-98): zero all fields, reseed the RNG. */
vapor_status vapor_mac3d_reset(vapor_mac3d *sim);
/* setBoxSize (GpuMacSimulation3D.cpp:99-106): reset when the size changes. */
vapor_status vapor_mac3d_set_box(vapor_mac3d *sim, float box);
vapor_status vapor_mac3d_get_params(const vapor_mac3d *sim, vapor_mac3d_params *out);
/* parameters() returns a mutable struct read on every advance. */
vapor_status vapor_mac3d_set_params(vapor_mac3d *sim, const vapor_mac3d_params *params);
/* advance(dt) (GpuMacSimulation3D.cpp:224-264): one step, enqueued on the
 * handle's stream; it does not wait for the device. Parameter validation
 * happens here (VAPOR_INVALID_ARGUMENT). Device-side failures (non-finite
 * divergence) surface from vapor_mac3d_synchronize / last_projection. */
vapor_status vapor_mac3d_advance(vapor_mac3d *sim, float dt);
/* Advance `steps` times with the same dt (one graph launch per step). */
vapor_status vapor_mac3d_advance_n(vapor_mac3d *sim, float dt, int32_t steps);
/* Wait for the handle's stream; report a deferred device-side error. */
vapor_status vapor_mac3d_synchronize(vapor_mac3d *sim);
/* lastProjection(): result of the last projection of the last step (waits). */
vapor_status vapor_mac3d_last_projection(vapor_mac3d *sim, vapor_projection_result *out);
/* Sum of SOR iterations over all projections since reset (waits). */
vapor_status vapor_mac3d_total_iterations(vapor_mac3d *sim, int64_t *out);
/* diagnostics(): kinetic energy, max |velocity|, max |divergence| (waits). */
vapor_status vapor_mac3d_diagnostics(vapor_mac3d *sim, vapor_fluid_diagnostics *out);

/* Comparison metrics of the current state (extension): the quantities the
 * reference's diagnostic harness prints for its Reflection / MacCormack
 * comparison (tests/ReflectionComparison.hpp:32-75), computed on the device.
 * frames_per_second sets the frame time 1 / fps of the CFL and trace tests
 * (the harness uses 60). Sums are FP64 (a fixed tree; the harness sums
 * sequentially, so they agree to FP64 rounding); counts and maxima are exact.
 * VAPOR_NON_FINITE when a divergence is not finite. */
typedef struct vapor_comparison_metrics {
    double mass_sum;          /* sum of density */
    double mass;              /* mass_sum / n^3 */
    double grad_per_mass;     /* sum of |d - d(+x)|, |d - d(+y)|, |d - d(+z)| over mass_sum */
    double square_per_mass;   /* sum of d^2 over mass_sum */
    double rms_div;           /* sqrt(mean divergence^2) */
    double max_div;           /* max |divergence| */
    long long smoke_cells;    /* cells with density > 0.001 */
    long long cfl_fallback;   /* smoke cells with |v| / (h fps) > cfl_mc */
    long long boundary_fallback; /* smoke cells whose trace -v/fps or +v/fps leaves the box */
    double max_cfl;           /* max |v| / (h fps) over smoke cells */
    int32_t nonfinite;
    int32_t reserved;
} vapor_comparison_metrics;
vapor_status vapor_mac3d_comparison_metrics(vapor_mac3d *sim, float frames_per_second,
                                            vapor_comparison_metrics *out);

/* Headless volume ray-march of the smoke density (extension): the reference's
 * volume shader (src/renderer/shaders/volume.frag:13-55) seen from its orbit
 * camera (src/renderer/OrbitCamera.cpp:5-28), one CUDA thread per pixel and
 * no graphics API. The image is width x height RGB floats in [0, 1], pixel
 * (i, j) at rgb[3 (j width + i)] with row j = 0 at the bottom (OpenGL's
 * order); pixels without smoke hold the clear colour (.03, .04, .07). The
 * harness's image: azimuth -1.2, elevation .3, distance 2.5, step_scale .5,
 * alpha_mul 30, light (.3, .4, 1) / sqrt(1.25), shadow_strength .3,
 * shadow_step .1. */
typedef struct vapor_render_params {
    int32_t width, height;
    float azimuth, elevation, distance;  /* orbit camera around the box centre */
    float step_scale;                    /* ray step = step_scale / n (world units for box 1) */
    float alpha_mul;                     /* opacity per unit density and length */
    float light[3];                      /* unit direction towards the light */
    float shadow_strength;               /* 0: no shadow march */
    float shadow_step;
} vapor_render_params;
/* density_device: n^3 FP32 on the current device; rgb_device: 3 * width *
 * height floats on the device. Allocates nothing. */
vapor_status vapor_render_volume(const float *density_device, int32_t n, float box,
                                 const vapor_render_params *params, float *rgb_device, void *stream);
/* The simulation's current density into host memory (3 * width * height
 * floats); waits. */
vapor_status vapor_mac3d_render(vapor_mac3d *sim, const vapor_render_params *params, float *rgb_host);
/* upload/download (GpuMacSimulation3D.cpp:110-141): host snapshot <-> device.
 * Array sizes are implied by n (see layout above). */
vapor_status vapor_mac3d_upload(vapor_mac3d *sim, const float *density, const float *u,
                                const float *v, const float *w);
vapor_status vapor_mac3d_download(vapor_mac3d *sim, float *density, float *u, float *v,
                                  float *w);
/* Streamed transfers, for hosts that exchange the state every step.
 * vapor_mac3d_upload_async stages a host snapshot on a copy stream and
 * returns; the next vapor_mac3d_advance takes it in at the start of its step
 * (a device-to-device copy), so the copy overlaps whatever runs before.
 * vapor_mac3d_download_async snapshots the fields after the steps issued so
 * far (on the step stream) and copies the snapshot to the host on another
 * stream, overlapping the steps issued after it. Host arrays (pinned memory
 * for full overlap) must stay valid and unchanged, and downloaded arrays
 * unread, until vapor_mac3d_wait_transfers returns. A synchronous upload
 * replaces a staged upload that no step took in yet. The byte counters count
 * both forms. */
vapor_status vapor_mac3d_upload_async(vapor_mac3d *sim, const float *density, const float *u,
                                      const float *v, const float *w);
vapor_status vapor_mac3d_download_async(vapor_mac3d *sim, float *density, float *u, float *v,
                                        float *w);
vapor_status vapor_mac3d_wait_transfers(vapor_mac3d *sim);
/* uploadedBytes/downloadedBytes (GpuMacSimulation3D.hpp:25-26). */
vapor_status vapor_mac3d_byte_counters(const vapor_mac3d *sim, uint64_t *uploaded,
                                       uint64_t *downloaded);
/* renderData() analogue: borrowed device pointers of the resident fields.
 * They stay valid until the next advance/reset/destroy on this handle. */
vapor_status vapor_mac3d_device_fields(vapor_mac3d *sim, float **density, float **u, float **v,
                                       float **w);
/* The handle's CUDA stream (a cudaStream_t), for callers that order their own
 * work or record CUDA events against the step. */
vapor_status vapor_mac3d_stream(vapor_mac3d *sim, void **stream);
vapor_status vapor_mac3d_resolution(const vapor_mac3d *sim, int32_t *n, float *box);
/* Enable (1) or disable (0) phase timing; enabling clears the accumulators. */
vapor_status vapor_mac3d_set_timing(vapor_mac3d *sim, int32_t enabled);
/* Waits for the stream, folds recorded intervals into the totals and returns them. */
vapor_status vapor_mac3d_timings(vapor_mac3d *sim, vapor_phase_timings *out);

/* ------------------------------------------------------------------------ */
/* Staged stage plugins: Projection3D / Advection3D with host spans           */
/* (the GpuPressureSolver/GpuAdvection pattern, GpuMacBackend.cpp:91-109)     */
/* ------------------------------------------------------------------------ */
typedef struct vapor_stage vapor_stage;

/* One workspace per concurrent operation (AdvectionContext.hpp:18-19). */
vapor_status vapor_stage_create(int32_t n, float box, vapor_stage **out);
vapor_status vapor_stage_destroy(vapor_stage *stage);
/* Projection3D::reset: clear the pressure and divergence workspace. */
vapor_status vapor_stage_reset(vapor_stage *stage);
/* Projection3D::project (CpuPressureSolver3D.cpp:25-60) on host velocity
 * spans, in place. diagonal_floor is the SOR relaxation floor (6 reproduces
 * MacGridFluidSolver3D's solver, MacGridFluidSolver3D.hpp:118). pressure_out
 * (may be NULL) receives the zero-mean pressure, n^3 floats. */
vapor_status vapor_stage_project(vapor_stage *stage, float *u, float *v, float *w,
                                 const vapor_projection_options *options, float diagonal_floor,
                                 vapor_projection_result *result, float *pressure_out);
/* Advection3D::advectFace (CpuAdvectionKernels.cpp:82-269): source and output
 * are face arrays of `axis`; flow_u/v/w are the tracer velocity. The output
 * must not alias the source or the flow (AdvectionContext.cpp:53-67). */
vapor_status vapor_stage_advect_face(vapor_stage *stage, int32_t axis, float dt, float cfl_limit,
                                     int32_t method, const float *source, const float *flow_u,
                                     const float *flow_v, const float *flow_w, float *output);
/* Advection3D::advectScalar (CpuAdvectionKernels.cpp:18-80), in place. */
vapor_status vapor_stage_advect_scalar(vapor_stage *stage, float dt, float cfl_limit,
                                       int32_t method, float *field, const float *flow_u,
                                       const float *flow_v, const float *flow_w);
/* Device-pointer variants: every pointer is device memory of the right size. */
vapor_status vapor_stage_project_device(vapor_stage *stage, float *u, float *v, float *w,
                                        const vapor_projection_options *options,
                                        float diagonal_floor, vapor_projection_result *result,
                                        float *pressure_out);
vapor_status vapor_stage_advect_face_device(vapor_stage *stage, int32_t axis, float dt,
                                            float cfl_limit, int32_t method, const float *source,
                                            const float *flow_u, const float *flow_v,
                                            const float *flow_w, float *output);
vapor_status vapor_stage_advect_scalar_device(vapor_stage *stage, float dt, float cfl_limit,
                                              int32_t method, float *field, const float *flow_u,
                                              const float *flow_v, const float *flow_w);
/* Pressure solver used by vapor_stage_project (vapor_solver_kind); the default
 * is VAPOR_SOLVER_RED_BLACK_SOR, the reference's SOR. */
vapor_status vapor_stage_set_solver_kind(vapor_stage *stage, int32_t kind);
/* Solid obstacles for vapor_stage_project (extension, no reference
 * counterpart; Vapor's solvers have walls only). `mask` is n^3 host bytes,
 * x fastest, nonzero = solid; NULL removes the obstacles. Faces touching a
 * solid cell are closed (velocity 0 before and after the projection), solid
 * cells are not unknowns (pressure 0, excluded from the residual), the
 * diagonal of a fluid cell counts its fluid neighbours, and the right-hand-side
 * and pressure means run over fluid cells. Needs VAPOR_SOLVER_MIXED_REFINEMENT
 * or VAPOR_SOLVER_FPCG (masked operator, smoothing and coarse correction; the
 * coarse network's mask channel stays zero); a mask without fluid cells is
 * VAPOR_INVALID_ARGUMENT. */
vapor_status vapor_stage_set_solid(vapor_stage *stage, const uint8_t *mask);
/* The same obstacle mask (extension) for every later projection of a
 * resident simulation's steps: solid cells carry no pressure and the faces
 * touching them are closed; advection, forcing and smoke are unchanged.
 * Needs solver_kind VAPOR_SOLVER_MIXED_REFINEMENT or VAPOR_SOLVER_FPCG (the
 * step fails otherwise); mask NULL removes it. Waits for the simulation's
 * stream. */
vapor_status vapor_mac3d_set_solid(vapor_mac3d *sim, const uint8_t *mask);
vapor_status vapor_stage_stream(vapor_stage *stage, void **stream);

/* Advection of one staggered field that allocates no device memory. No
 * counterpart in the reference: it is for callers that may not allocate at
 * the call site (a frame loop that cannot absorb cudaFree's device-wide
 * synchronization, a host that owns all device memory and hands plugins only
 * their buffers). Same
 * arithmetic as vapor_stage_advect_face_device / _scalar_device (results are
 * bit-identical), with the MacCormack forward pass kept in a fixed 4 MiB
 * array inside this library's device image instead of an allocated buffer.
 *   loc: 0 cell (smoke), 1/2/3 faces of x/y/z; every pointer is device memory
 *   on the current device, of the reference's MAC sizes for n; output must not
 *   alias source or the flow; stream may be NULL (the default stream).
 * Limit: the field may have at most 1048576 values (faces: n <= 101); larger
 * fields return VAPOR_LENGTH_ERROR. The 4 MiB are committed when the driver
 * loads the array's module into a context, which under lazy module loading
 * (CUDA_MODULE_LOADING=LAZY) is the first call in that context; that call also
 * looks up and caches the array's address for the context. Make the first
 * call during set-up, before any stream capture begins. Contexts other than
 * the primary one are supported (the cache is per context); a device reset
 * ends the context, so do not call this after cudaDeviceReset in the same
 * process.
 * All calls share the array, so calls that can overlap on the GPU (different
 * streams, unordered threads) race and must be serialized by the caller.
 * Nothing needs to start at zero. */
vapor_status vapor_advect_noalloc(int32_t n, float box, int32_t loc, float dt, float cfl_limit,
                                  int32_t method, const float *source, const float *flow_u,
                                  const float *flow_v, const float *flow_w, float *output,
                                  void *stream);

/* Tuning (extension): z-planes per thread of the red-black colour sweep for
 * grids of size n (0 = automatic: at least four waves of blocks). Results do
 * not depend on it; set it before creating the simulations whose steps are
 * recorded into graphs. vapor_b200/autotune.py measures and chooses it. */
vapor_status vapor_tune_sor_planes(int32_t n, int32_t planes);
/* Tuning (extension): red+black iterations per launch of the temporally
 * blocked sweep (1 or 2), or 0 (default) for one launch per colour (the
 * z-marching sweep, faster on B200 at the benchmark's sizes). Applies to
 * grids with n divisible by 8; results are bit for bit the same either way.
 * Process-wide; set it before recording steps. */
vapor_status vapor_tune_sor_blocking(int32_t iterations_per_launch);
/* Tuning (extension): z chunks per blocked launch for grids of size n (0 =
 * automatic: one wave of resident CTAs). Results do not depend on it. */
vapor_status vapor_tune_sor_blocked_chunks(int32_t n, int32_t chunks);
/* Tuning (extension): the tcgen05 kernel of the learned network's 3x3x3
 * convolutions whose weights fit in shared memory. 0: the
 * block-synchronous z-march (27 MMAs of width cout per output plane); 1: its
 * warp-specialised form (producer, MMA and epilogue warps on mbarriers; same
 * results); 2: the plane-window form (9 MMAs of width 3 cout per input
 * plane, three output planes per MMA; same results for 16 input channels,
 * FP32-rounding differences for more); 3 (default): the plane-window form
 * fed by the TMA unit (weights in one bulk copy, input planes as tensor-map
 * boxes; the same results as 2; grids narrower than 10 x 18 voxels run 0). */
vapor_status vapor_tune_conv_kernel(int32_t kind);
/* Tuning (extension): the FPCG preconditioner's relaxation sweeps before and
 * after the coarse correction (1..8, default 2) and their weight (0 < omega
 * < 2, default 1.2; 1 is symmetric Gauss-Seidel). Changes the iteration count, not
 * the accepted answer (the stopping test is the FP64 residual). Process-wide;
 * set it before recording steps. */
vapor_status vapor_tune_fpcg_smoothing(int32_t sweeps, float omega);
/* Tuning (extension): the kernel of the network's weight gradients in
 * training: 1 (default) tcgen05 implicit GEMM (M = 8 taps x 16 output
 * channels, N = input channels, K = voxels), 0 the CUDA-core form. Both add
 * FP32 products of the same BF16 values with atomics: equal to FP32
 * rounding. */
vapor_status vapor_tune_wgrad_kernel(int32_t kind);
vapor_status vapor_fpcg_smoothing(int32_t *sweeps, float *omega);

/* ---- Batched scenes (extension, no reference counterpart) ----
 * Steps many resident simulations (uneven grid sizes allowed, each with its
 * own parameters) with one CUDA-graph launch: every scene's whole step,
 * tolerance-driven solve loops included, is a parallel branch of one graph,
 * so small grids fill the GPU together. The batch orders itself after each
 * scene's earlier work and each scene's later work after the batch; the
 * scenes stay usable one by one (upload, download, diagnostics). The batch
 * does not own the simulations: destroy it before them. */
typedef struct vapor_batch vapor_batch;
vapor_status vapor_batch_create(int32_t count, vapor_mac3d *const *sims, vapor_batch **out);
vapor_status vapor_batch_destroy(vapor_batch *batch);
vapor_status vapor_batch_advance(vapor_batch *batch, float dt);
vapor_status vapor_batch_synchronize(vapor_batch *batch);
vapor_status vapor_batch_stream(vapor_batch *batch, void **stream);

/* ---- Learned warm start for the pressure solve ----
 * No counterpart in the reference, whose projection starts every solve from
 * zero pressure (CpuPressureSolver3D.cpp:46). The model is a fixed 3-level 3D
 * U-Net (16/32/64 channels, about 0.35 M parameters, BF16 weights and
 * activations, FP32 accumulation on tcgen05 tensor cores) that maps the normalized right-hand side to the normalized
 * zero-mean pressure; the projection then runs its usual solver from that
 * guess, so convergence criteria and results keep their meaning. Parameters
 * are one FP32 vector: for each of the 10 convolutions its weights
 * [27][cout][cin] then its bias [cout], then the 1x1 head's 16 weights and
 * its bias. Grids must have n divisible by 4. */
typedef struct vapor_unet vapor_unet;
int64_t vapor_unet_parameter_count(void);
vapor_status vapor_unet_create(vapor_unet **out);
vapor_status vapor_unet_destroy(vapor_unet *net);
/* He-uniform weights from `seed`, zero biases, Adam state cleared. */
vapor_status vapor_unet_init(vapor_unet *net, uint32_t seed);
vapor_status vapor_unet_set_parameters(vapor_unet *net, const float *host, int64_t count);
vapor_status vapor_unet_get_parameters(vapor_unet *net, float *host, int64_t count);
/* Raw network on device buffers: input is n^3 voxels x 16 BF16 channels
 * (channels-last; channel 0 the normalized RHS, channel 1 the solid mask,
 * the rest zero), output n^3 FP32. Synchronizes. */
vapor_status vapor_unet_forward_features(vapor_unet *net, int32_t n, const void *input_bf16,
                                         float *output);
/* Gradient of sum(output * grad_output) with respect to the parameters after
 * vapor_unet_forward_features on the same n; grad_output is device memory,
 * grad_params host memory of vapor_unet_parameter_count() floats. */
vapor_status vapor_unet_backward(vapor_unet *net, int32_t n, const float *grad_output,
                                 float *grad_params);
/* Test hook for the tensor-core convolutions' bounded waits (no reference
 * counterpart): with iterations > 0, the first completion wait of every CTA
 * of the next convolutions polls an mbarrier that nothing completes that many
 * times, runs out, and the call returns VAPOR_RUNTIME_ERROR ("timed out")
 * after the CTA has drained its in-flight MMAs and freed its TMEM; 0 restores
 * normal waits. The error flag is cleared when it is reported, so the next
 * call starts clean. */
vapor_status vapor_unet_set_wait_probe(vapor_unet *net, int32_t iterations);
/* Use `net` (NULL: none) for the initial guess of every later projection of
 * `sim`. The network must outlive the simulation or be detached first. */
vapor_status vapor_mac3d_set_warm_start(vapor_mac3d *sim, vapor_unet *net);
/* One Adam step on the simulation's last projection (its right-hand side and
 * converged pressure); *loss (may be NULL) receives the loss before the step:
 * the relative squared error of the mean-free prediction after its best
 * scaling, 1 - cos^2 against the converged pressure. The warm start applies
 * that scaling itself: x0 = alpha q with q the mean-free prediction and
 * alpha = (q.b)/(q.Aq), the Galerkin condition on span{q}, so the guess is
 * never worse than zero in the A-norm. */
vapor_status vapor_mac3d_train_warm_start(vapor_mac3d *sim, vapor_unet *net, float learning_rate,
                                          double *loss);
/* The same loss without an update. */
vapor_status vapor_mac3d_evaluate_warm_start(vapor_mac3d *sim, vapor_unet *net, double *loss);
/* Coarse-grid correction of the VAPOR_SOLVER_FPCG preconditioner (NULL: the
 * smoothing-only preconditioner). The network runs on the grid coarsened 4x
 * per axis (right-hand side: 4^3 block sums of the smoothed residual), its
 * output is scaled by the Galerkin condition of the coarse operator 16 L and
 * prolonged piecewise constant. Needs n divisible by 16 (n >= 32). The
 * network must outlive the simulation or be detached first, and serves one
 * simulation or stage at a time (its activation buffers are shared state). */
vapor_status vapor_mac3d_set_preconditioner(vapor_mac3d *sim, vapor_unet *net);
vapor_status vapor_stage_set_preconditioner(vapor_stage *stage, vapor_unet *net);
/* Training data for the coarse-grid network: every FPCG coarse right-hand
 * side ((n/4)^3 floats, natural layout) of later steps of `sim` is copied to
 * record (*counter % capacity) of the device ring `log`, then *counter is
 * incremented on the device. NULL log and counter disable it. */
vapor_status vapor_mac3d_set_coarse_log(vapor_mac3d *sim, float *log, int32_t capacity, int32_t *counter);
/* Mixed-precision solve of A x = rhs on the stage's grid for a given
 * right-hand side (device memory, n^3 floats, x fastest; its mean is removed
 * as for a projection); the zero-mean solution into `pressure` (device, may
 * be NULL). The stage keeps (rhs, x) for vapor_stage_train_network. */
vapor_status vapor_stage_solve_rhs(vapor_stage *stage, const float *rhs,
                                   const vapor_projection_options *options, float diagonal_floor,
                                   vapor_projection_result *result, float *pressure);
/* One Adam step of `net` on the stage's last projection (its right-hand side
 * and converged pressure, on the stage's own n^3 grid); the loss as for
 * vapor_mac3d_train_warm_start. Used to train the coarse-grid network on
 * solves at the coarse resolution. */
vapor_status vapor_stage_train_network(vapor_stage *stage, vapor_unet *net, float learning_rate,
                                       double *loss);

/* ---- MAC 2D smoke solver (src/solvers/mac2d/MacGridFluidSolver2D.cpp) ----
 * The reference's 2D solver on the device: closed square box, semi-Lagrangian
 * advection with clamped bilinear sampling (SemiLagrangian2D.cpp:13-50),
 * buoyancy (d^1/4 averaged onto the v faces), replenished Gaussian emitter,
 * FP64 red-black SOR projection (CpuPressureSolver2D.cpp:8-82), density
 * decay exp(-dt decay), and the midpoint-reflection variant
 * (MacGridFluidSolver2D.cpp:104-128). Layout as MacGridState2D: density
 * n^2 (x fastest), u (n+1) x n (idX = x + (n+1) y), v n x (n+1)
 * (idY = x + n y). Each call waits for its work. */
typedef struct vapor_mac2d vapor_mac2d;
/* MacGridParameters2D (MacGridFluidSolver2D.hpp:5-15). */
typedef struct vapor_mac2d_params {
    int32_t reflection;            /* 0: simple step, 1: midpoint reflection */
    float source_strength;
    float emitter_kick_multiplier;
    float emitter_radius;          /* fraction of the box */
    float emitter_center_x, emitter_center_y;
    float buoyancy;
    float smoke_decay;
    float sor_omega;
    int32_t project_iterations;    /* SOR iteration budget of each projection */
} vapor_mac2d_params;
/* The struct's defaults (MacGridFluidSolver2D.hpp:5-15). */
vapor_status vapor_mac2d_default_params(vapor_mac2d_params *out);
/* The scene of the default-constructed solver (MacGridFluidSolver2D.cpp:8-14:
 * radius .04, strength 1, buoyancy .8, decay .3007525, 120 iterations). */
vapor_status vapor_mac2d_plume_params(vapor_mac2d_params *out);
/* MacGridFluidSolver2D(resolution, boxSize) + its parameters; zero state. */
vapor_status vapor_mac2d_create(int32_t n, float box, const vapor_mac2d_params *params, vapor_mac2d **out);
vapor_status vapor_mac2d_destroy(vapor_mac2d *sim);
vapor_status vapor_mac2d_get_params(const vapor_mac2d *sim, vapor_mac2d_params *out);
vapor_status vapor_mac2d_set_params(vapor_mac2d *sim, const vapor_mac2d_params *params);
/* advance(dt) (MacGridFluidSolver2D.cpp:22-44), with the reference's
 * argument checks; non-finite fields give VAPOR_NON_FINITE. */
vapor_status vapor_mac2d_advance(vapor_mac2d *sim, float dt);
/* resetState() and setBoxSize() (MacGridFluidSolver2D.cpp:130-141). */
vapor_status vapor_mac2d_reset(vapor_mac2d *sim);
vapor_status vapor_mac2d_set_box(vapor_mac2d *sim, float box);
/* Host arrays in the layout above; any pointer may be NULL to skip it. */
vapor_status vapor_mac2d_upload(vapor_mac2d *sim, const float *density, const float *u, const float *v);
vapor_status vapor_mac2d_download(vapor_mac2d *sim, float *density, float *u, float *v);
/* lastProjection() / midpointProjection(): the step's final projection and,
 * with reflection, the midpoint one (zero otherwise). */
vapor_status vapor_mac2d_last_projection(vapor_mac2d *sim, vapor_projection_result *out);
vapor_status vapor_mac2d_midpoint_projection(vapor_mac2d *sim, vapor_projection_result *out);
/* diagnostics() (MacGridFluidSolver2D.cpp:142-153): FP64 kinetic energy
 * summed in the reference's order, max |velocity|, max |div|. */
vapor_status vapor_mac2d_diagnostics(vapor_mac2d *sim, vapor_fluid_diagnostics *out);

/* ---- MAC 2D reflection solver (src/solvers/mac2d/ReflectionMacFluidSolver2D.hpp) ----
 * The reference's compatibility solver for the historical 2D plume (unit
 * box, n in 2..512): semi-Lagrangian velocity, semi-Lagrangian or MacCormack
 * smoke with its in-place 3x3 limiter, FP32 red-black SOR with a fixed
 * iteration count, buoyancy d^1/4 split onto both faces of a cell, emitter
 * with optional random stirring, midpoint reflection every step
 * (ReflectionMacFluidSolver2D.hpp:32-45, 309-425). Layout as vapor_mac2d;
 * the pressure is n^2 FP32. Each call waits for its work. */
typedef struct vapor_mac2d_refl vapor_mac2d_refl;
/* The solver's public fields (ReflectionMacFluidSolver2D.hpp:19-22, 57-71). */
typedef struct vapor_mac2d_refl_params {
    int32_t mac_cormack_smoke;     /* 1: MacCormack smoke, 0: semi-Lagrangian */
    float source_strength;
    float buoyancy;
    float smoke_decay;             /* per second; the step uses exp(-decay / 60) per frame */
    int32_t project_iterations;    /* red-black SOR iterations, half of them per projection */
    float emitter_radius;          /* fraction of the box */
    float emitter_center_x, emitter_center_y;
    float emitter_kick_multiplier;
    float stir_strength;           /* random inlet stirring; 0 keeps the historical replay */
    float sor_omega;
    uint32_t random_seed;          /* stirring stream, applied at creation and reset */
} vapor_mac2d_refl_params;
/* The struct's defaults (MC smoke, 60 iterations, radius .08). */
vapor_status vapor_mac2d_refl_default_params(vapor_mac2d_refl_params *out);
/* The solver built from an advection method (ReflectionMacFluidSolver2D.hpp:77-85:
 * radius .04, 120 iterations; method VAPOR_SEMI_LAGRANGIAN or
 * VAPOR_MACCORMACK); its resolution is 128. */
vapor_status vapor_mac2d_refl_app_params(int32_t method, vapor_mac2d_refl_params *out);
vapor_status vapor_mac2d_refl_create(int32_t n, const vapor_mac2d_refl_params *params, vapor_mac2d_refl **out);
vapor_status vapor_mac2d_refl_destroy(vapor_mac2d_refl *sim);
vapor_status vapor_mac2d_refl_get_params(const vapor_mac2d_refl *sim, vapor_mac2d_refl_params *out);
vapor_status vapor_mac2d_refl_set_params(vapor_mac2d_refl *sim, const vapor_mac2d_refl_params *params);
vapor_status vapor_mac2d_refl_advance(vapor_mac2d_refl *sim, float dt);
/* resetState(): zero fields, stirring stream back to the seed. */
vapor_status vapor_mac2d_refl_reset(vapor_mac2d_refl *sim);
/* Host arrays; any pointer may be NULL to skip it (pressure: download only). */
vapor_status vapor_mac2d_refl_upload(vapor_mac2d_refl *sim, const float *smoke, const float *u, const float *v);
vapor_status vapor_mac2d_refl_download(vapor_mac2d_refl *sim, float *smoke, float *u, float *v, float *pressure);
vapor_status vapor_mac2d_refl_diagnostics(vapor_mac2d_refl *sim, vapor_fluid_diagnostics *out);

/* ---- Simplicial 3D compute stages (src/solvers/simplicial3d/SimplicialCompute3D.hpp:7-13) ----
 * The reference's optional compute backend of SimplicialFluidSolver3D
 * (its OpenGL GpuSimplicial3D, gpu/GpuSimplicial3D.cpp) on the device, FP64:
 * the circulation advection (trace every dual vertex by the midpoint rule,
 * integrate the dual edges, sum each primal edge's dual face), the smoke
 * advection with decay (trace every primal vertex, interpolate the vertex
 * smoke) and the flux recovery (CG on the Dirichlet potential operator of
 * SimplicialFluidSolver3D::laplacian, preconditioned as the CPU solver
 * preconditions it: its IC(0) factor or its diagonal). The sampling
 * keeps the CPU solver's operation order: traces, velocities, circulations
 * and smoke equal the CPU's bit for bit (box nearest-site search by a scan;
 * the descent search and general domains follow the same arithmetic).
 * vapor_b200/host/VaporSimplicial3D.hpp flattens a solver into this struct
 * and implements SimplicialCompute3D on these calls. Each call waits for
 * its work. */
typedef struct vapor_simplicial3d vapor_simplicial3d;
typedef struct vapor_simplicial3d_mesh {
    int32_t box_domain;              /* Mesh::boxDomain: Voronoi-cell interpolation; 0: subdivision */
    int32_t bins;                    /* spatial bins per axis (0: none, one list of all items) */
    double size;                     /* Mesh::size */
    int32_t n_primal, n_dual, n_nodes, n_edges, n_dual_edges, n_tets, n_faces;
    int32_t n_planes, n_corners, n_cones, n_subtets;
    const double *dual_position;     /* 3 n_dual: dual vertices */
    const double *node_position;     /* 3 n_nodes: box: the primal vertices; domain: subdivision nodes */
    const double *tet_geometry;      /* 12 n_tets: vertex 0, barycentric gradients 1..3 */
    const int32_t *tet_vertices;     /* 4 n_tets */
    const int32_t *dual_hint;        /* n_dual: a tet near each dual vertex, or -1 */
    const int32_t *primal_hint;      /* n_primal: a tet of each primal vertex */
    const int32_t *bin_offsets;      /* max(1, bins^3) + 1 */
    const int32_t *bin_items;        /* tets per bin */
    const int32_t *wall_offsets;     /* max(1, bins^3) + 1 */
    const int32_t *wall_items;       /* boundary faces per bin */
    const double *wall_geometry;     /* 6 n_faces: outward area normal, first vertex */
    const int32_t *wall_owner;       /* n_faces: the tet on the inner side */
    const double *box_planes;        /* 4 n_planes: Voronoi cell planes (normal, offset) */
    const int32_t *cell_corners;     /* n_primal + 1 */
    const int32_t *corner_vertices;  /* n_corners: dual vertex of each cell corner */
    const int32_t *corner_cones;     /* n_corners + 1 */
    const int32_t *cone_planes;      /* 3 n_cones */
    const int32_t *neighbor_offsets; /* n_primal + 1: Delaunay neighbours */
    const int32_t *neighbors;
    const int32_t *sub_offsets;      /* n_tets + 1: circumcentric subtets (domain) */
    const int32_t *sub_nodes;        /* 4 n_subtets */
    const double *sub_gradients;     /* 9 n_subtets */
    const int32_t *loop_offsets;     /* n_edges + 1: each primal edge's dual face */
    const int32_t *loop_items;       /* sign * (dual edge + 1) */
    const int32_t *dual_edges;       /* 2 n_dual_edges */
    /* the Dirichlet potential operator */
    const int32_t *face_edges;       /* 3 n_faces */
    const int32_t *face_signs;       /* 3 n_faces */
    const int32_t *edge_vertices;    /* 2 n_edges */
    const uint8_t *edge_boundary;    /* n_edges */
    const uint8_t *vertex_boundary;  /* n_primal */
    const double *star0;             /* n_primal */
    const double *star1;             /* n_edges */
    const double *star2;             /* n_faces */
    /* the preconditioner of SimplicialFluidSolver3D::solve: its IC(0) factor
     * when it has one (general domains), else its diagonal (Jacobi) */
    const double *jacobi_diagonal;   /* n_edges; NULL: the assembled operator's diagonal */
    const int32_t *ic_offsets;       /* n_edges + 1, or NULL: no factor */
    const int32_t *ic_columns;       /* strictly lower entries, ascending per row */
    const double *ic_values;
    const double *ic_diagonal;       /* n_edges */
} vapor_simplicial3d_mesh;
/* Uploads the mesh. site_search: 0 automatic (a scan of all sites up to
 * 4096 primal vertices, else the descent), 1 scan, 2 descent over Delaunay
 * neighbours from the sample's tet. dot_order: 0 automatic (index order up
 * to 262144 edges), 1 index order on one thread (std::inner_product's: the
 * recovery's iterates equal the CPU solver's bit for bit), 2 a parallel
 * tree (faster on large meshes; equal to rounding). preconditioner: 0 the
 * CPU solver's (its IC(0) factor where it has one, else its diagonal), 1
 * always the diagonal (Jacobi, the OpenGL backend's choice: no sequential
 * triangular solves, more iterations, not the CPU's iterates). */
vapor_status vapor_simplicial3d_create(const vapor_simplicial3d_mesh *mesh, int32_t site_search,
                                       int32_t dot_order, int32_t preconditioner, vapor_simplicial3d **out);
vapor_status vapor_simplicial3d_destroy(vapor_simplicial3d *stages);
/* advectCirculation: omega (n_edges) from the dual velocities (3 n_dual) and,
 * on general domains, the node samples (3 n_nodes; NULL on boxes). */
vapor_status vapor_simplicial3d_advect_circulation(vapor_simplicial3d *stages, double dt,
                                                   const double *dual_velocity, const double *node_samples,
                                                   double *omega);
/* advectDensity: the vertex smoke (n_primal) traced back by dt, times decay
 * (the caller's exp(-smokeDecay dt)). */
vapor_status vapor_simplicial3d_advect_density(vapor_simplicial3d *stages, double dt, double decay,
                                               const double *dual_velocity, const double *node_samples,
                                               const float *vertex_density, float *density_out);
/* recover: x (n_edges) with A x = rhs from x0 (the CPU solver starts from
 * zero on boxes and from the current potential on general domains),
 * boundary edges held at zero; stops when the infinity norm of the
 * residual is at most max(absolute, relative * |rhs|_inf) or after
 * `iterations`; the final residual is recomputed from x. Invalid controls:
 * VAPOR_INVALID_ARGUMENT; a non-finite rhs or a lost positive definiteness:
 * VAPOR_RUNTIME_ERROR (the reference's messages). */
vapor_status vapor_simplicial3d_recover(vapor_simplicial3d *stages, const double *rhs, const double *x0,
                                        int32_t iterations, double absolute_tolerance, double relative_tolerance,
                                        double *x, vapor_linear_solve_result *result);

#ifdef __cplusplus
}
#endif

#endif /* VAPOR_B200_H */
