// Host-side launch wrappers of the MAC 3D kernels (kernels_*.cu). All
// launches are asynchronous on the given stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/vapor_b200.h"
#include "mac3d_common.cuh"

namespace vb {

// Per-projection device state: reduction accumulators, loop control and the
// assembled ProjectionResult. Lives in device memory, one per workspace.
struct ProjControl {
    // accumulators, cleared at the start of a projection
    unsigned int div_before_bits;   // max |div| before, float bits
    unsigned int div_after_bits;    // max |div| after, float bits
    int rhs_max_key, rhs_min_key;   // order keys of max/min of b = -div*h^2/dt
    unsigned long long res_bits;    // max |b - Ax| of the last residual pass, double bits
    unsigned int nonfinite;         // bit 0: divergence before, bit 1: after, bit 2: solve
    unsigned int reserved0;
    // derived values
    float rhs_mean_f;               // (float)(sum b / C), subtracted from b on the fly
    float p_mean_f;                 // (float)(sum x / C), subtracted from x on the fly
    double p_mean64;                // sum x64 / C (mixed-precision solver)
    double removed_mean;
    double target;                  // max(abs tol, rel tol * initial residual)
    // loop control
    int iterations;
    int done;                       // 1 once the solve loop must stop
    int max_iterations;
    int check_interval;
    int fixed;
    int continue_flag;              // mirror of the graph while-condition
    int x64_cur;                    // mixed precision: index of the current FP64 pressure
    int recentre;                   // mixed precision: 1 when this check re-centres in FP64
    double* x64[2];                 // mixed precision: FP64 pressure ping-pong buffers
    double r0;                      // mixed precision: FP64 residual at the last re-centring
    unsigned int res32_bits;        // mixed precision: FP32 error-equation residual, float bits
    int since;                      // mixed precision: sweeps since the last re-centring
    vapor_projection_result result;
    // persistent across projections (cleared only by a workspace reset)
    unsigned int sticky_nonfinite;  // OR of `nonfinite` over finished projections
    unsigned int reserved1;
    long long total_iterations;     // SOR iterations over finished projections
};

// Scalars of the flexible PCG solve (device).
struct CgControl {
    double rho;      // z.r of the current search direction
    double alpha;    // step length rho / (p.Ap)
    double beta;     // flexible (Polak-Ribiere) direction update
    double pq;       // p.Ap
    double gamma;    // scale of the coarse-grid correction (Galerkin)
    double zc_mean;  // mean of the coarse correction, removed before use
    // fused step (n % 8 == 0): the direction lives in two buffers, p_cur the
    // current one; alpha_pending * p_cur is the error update not yet added
    // to e (added by the next direction kernel, or folded before a
    // re-centring). flags: bit 0 a direction exists, bit 1 an update is pending.
    double alpha_pending;
    int p_cur;
    int flags;
};

// Simulation-wide reduction outputs (diagnostics).
struct DiagControl {
    unsigned int max_velocity_bits;
    unsigned int max_divergence_bits;
    unsigned int nonfinite;
    unsigned int reserved0;
    double kinetic_sum;
};

// ---- forcing: emit, buoyancy, walls, decay ----
struct EmitterBox {
    int lo[3];
    int size[3];
    float ec[3];       // centre in world units
    float erad;        // radius in world units
    float kick;        // emitterKickMultiplier * (base + scale * strength)
    int apply_kick;    // emitterKickMultiplier > 0
    float stir_scale;  // stirStrength * dt * 60, applied as (r - .5) * stir * dtScale
    float stir;        // stirStrength
    float dt_scale;    // dt * 60
    int profile;       // 0: density = 1, 1: smooth profile
    float strength;    // sourceStrength
};
// Emitter patch [lo, lo+size) per axis, as MacGridFluidSolver3D::emit bounds it.
void launch_emit(const Grid& g, const EmitterBox& e, uint32_t* rng_state, float* noise, float* density,
                 float* u, float* v, float* w, cudaStream_t s);
// w += split * (buoyancy * d_below * dt); w += split * (buoyancy * d_above * dt)
// on interior z-faces, then zero every wall face.
void launch_buoyancy_walls(const Grid& g, float buoyancy, float dt, float split, const float* density, float* u,
                           float* v, float* w, cudaStream_t s);
void launch_walls(const Grid& g, float* u, float* v, float* w, cudaStream_t s);

// ---- advection ----
// Semi-Lagrangian (fwd only) or MacCormack (fwd into `fwd`, then the limiter)
// transport of the field at `loc`; `post_scale` multiplies every output value
// (the smoke dissipation factor; 1 for velocity).
void launch_advect(const Grid& g, int loc, float dt, float cfl_limit, bool maccormack, const float* src,
                   const float* u, const float* v, const float* w, float* fwd, float* out, float post_scale,
                   cudaStream_t s);
// The three velocity components src[c] (faces of axis c) through the flow
// (u, v, w) into out[c], in one forward launch (into fwd[c]) and one
// MacCormack launch; same results as three launch_advect calls. With
// `vel_cache` (9 face arrays) the forward pass stores each point's traced
// velocity and the MacCormack pass reads it back instead of sampling again.
void launch_advect_velocity(const Grid& g, float dt, float cfl_limit, bool maccormack, const float* const src[3],
                            const float* u, const float* v, const float* w, float* const fwd[3],
                            float* const out[3], float* vel_cache, cudaStream_t s);
// The smoke (cell centres) the same way, with `vel_cache` of 3 cell arrays.
void launch_advect_smoke(const Grid& g, float dt, float cfl_limit, bool maccormack, const float* src,
                         const float* u, const float* v, const float* w, float* fwd, float* out, float post_scale,
                         float* vel_cache, cudaStream_t s);

// ---- projection ----
struct ProjectionArgs {
    Grid g;
    float dt;
    float omega;
    float diagonal_floor;
    vapor_linear_solve_options options;
    // Solid obstacles (extension; all null/zero without a mask): `diag` is
    // the split-layout diagonal (fluid-neighbour count, 0 = solid cell),
    // `solid` the natural-layout mask, `fluid` the number of fluid cells.
    const uint8_t* diag = nullptr;
    const uint8_t* solid = nullptr;
    double fluid = 0.0;
};
// Graph while-loop control: when `active`, kernels that decide whether the
// solve continues also set this conditional handle.
struct LoopCond {
    int active = 0;
    unsigned long long handle = 0;
};
// Clear accumulators, compute b = -div(walls(u_in)) h^2/dt with its sum,
// max/min and max |div|; then derive mean, initial residual and target.
// x64a/x64b are the mixed-precision buffers (may be null).
void launch_rhs(const ProjectionArgs& a, const float* u, const float* v, const float* w, float* b,
                double* partials, int partial_capacity, ProjControl* ctrl, double* x64a, double* x64b,
                LoopCond cond, cudaStream_t s,
                const float* field = nullptr);
// One red-black colour sweep over x (parity 0 updates i+j+k even). With
// `subtract_mean` the right-hand side is b - ctrl->rhs_mean_f, else b. A
// guarded sweep returns at once when the solve is done or when
// ctrl->iterations + sweep_index reaches the iteration budget.
// `exact` = false selects the mixed solver's divide-free relaxation
// x += (b - off - diag x) * (omega / max(diag, floor)).
// `measure` (colour 1 only) also records max |b' - off - diag x| of the updated
// cells into ctrl->res32_bits when sor_fuses_measure(n); otherwise
// launch_error_check measures the same value in a separate pass.
// `from_zero` (fast relaxation without measuring, z-marching kernel only):
// the sweep starts from x = 0 and also writes the other colour as 0, so x
// needs no clearing first. Callers check sor_fuses_measure(n).
void launch_sor_color(const ProjectionArgs& a, int parity, float* x, const float* b, ProjControl* ctrl,
                      bool guarded, int sweep_index, bool subtract_mean, cudaStream_t s, bool exact = true,
                      bool measure = false, bool from_zero = false);
bool sor_fuses_measure(int n);
// The fast relaxation sweep (no mask, unguarded) of colour `parity` that
// also writes FP64 block partials of x.b and x.q (x after the sweep, both
// colours) to partials[2 * block]; returns the number of blocks, or 0 when
// the grid has no such form (then nothing ran).
int launch_sor_color_dot(const ProjectionArgs& a, int parity, float* x, const float* b, const float* q,
                         double* partials, int partial_capacity, ProjControl* ctrl, cudaStream_t s);
// Temporally blocked form of the same sweeps (kernels_sor_blocked.cu):
// `iterations` (1 or 2) red+black iterations in one launch, starting with
// colour `first_colour`, bit-identical to 2 * iterations one-colour launches
// with the same flags (for first_colour 1: the plain relaxation only). The
// update is out of place, xin -> xout (they may coincide only with
// `from_zero`, which reads no iterate). A guarded launch covers sweep indices
// sweep_index .. + iterations - 1 and stops at the iteration budget (copying
// xin to xout when no sweep is left); `measure` records the residual of its
// last half-sweep (colour 1) when it ran all iterations. Needs
// sor_blocked_applies(n).
bool sor_blocked_applies(int n);
void launch_sor_blocked(const ProjectionArgs& a, int iterations, int first_colour, const float* xin, float* xout,
                        const float* b, ProjControl* ctrl, bool guarded, int sweep_index, bool subtract_mean,
                        cudaStream_t s, bool exact, bool measure = false, bool from_zero = false);
// Autotuner hook: z chunks per blocked launch for grid size n (<= 0: one
// wave of CTAs).
void set_sor_blocked_chunks(int n, int chunks);
// Iterations per blocked launch that the solvers use (0: one launch per
// colour); sor_block_iterations(n) is 0 where the blocked form does not apply.
void set_sor_block_iterations(int iterations);
int sor_block_iterations(int n);
// Autotuner hook: planes per thread of the z-marching colour sweep for grid
// size n (planes <= 0 restores the automatic choice).
void set_sor_planes(int n, int planes);
// Mixed precision: x64[1-cur] = x64[cur] + e (FP64), r32 = float(b' - A x)
// with the FP64 residual norm into ctrl->res_bits.
void launch_refine_residual(const ProjectionArgs& a, const float* b, const float* e, float* r32,
                            ProjControl* ctrl, cudaStream_t s);
// Mixed precision check between re-centrings: the FP32 residual of the error
// equation over the colour-1 cells, max |r32 - A e| (measured here unless the
// last sweep already did, `measured`), then the decision (ctrl->recentre) to
// re-centre in FP64: when that residual reaches the target, drops below
// kRecentreDrop * r0, after kRecentreSweeps sweeps, or at the iteration budget.
// Adds `sweeps` to the iteration count. Without a re-centring it sets the
// loop condition to continue; `recentre_cond` (a graph if-condition) receives
// the decision.
constexpr float kRecentreDrop = 1e-2f;
constexpr int kRecentreSweeps = 1024;
void launch_error_check(const ProjectionArgs& a, const float* e, const float* r32, ProjControl* ctrl, int sweeps,
                        bool measured, LoopCond cond, LoopCond recentre_cond, cudaStream_t s);
// Gated forms (they do nothing unless ctrl->recentre): the re-centring pass,
// its check, and e = 0 afterwards.
void launch_refine_residual_gated(const ProjectionArgs& a, const float* b, const float* e, float* r32,
                                  ProjControl* ctrl, cudaStream_t s);
void launch_check_gated(ProjControl* ctrl, LoopCond cond, cudaStream_t s);
// Sets the graph loop condition to !ctrl->done.
void launch_loop_condition(const ProjControl* ctrl, LoopCond cond, cudaStream_t s);
void launch_zero_error_gated(const ProjectionArgs& a, float* e, const ProjControl* ctrl, cudaStream_t s);
// Mixed precision epilogue: FP64 pressure mean, final FP64 residual, float
// pressure copy (x64 - mean) into p32 with ctrl->p_mean_f = 0, then (u_in
// given) the gradient step with the FP64 pressure (x64 - mean): the
// difference, scaling and subtraction in FP64, rounded to FP32; walls,
// reflection hat (u_hat given) and divergence after. Unmasked grids with n %
// 4 == 0 run the residual and the gradient as one pass. Returns the number
// of kernels launched.
int launch_finish_projection64(const ProjectionArgs& a, const float* b, float* p32, double* partials,
                               int partial_capacity, ProjControl* ctrl, const float* u_in, const float* v_in,
                               const float* w_in, float* u_out, float* v_out, float* w_out, float* u_hat,
                               float* v_hat, float* w_hat, cudaStream_t s);
// FP64 infinity norm of (b - mean_b) - A (x - mean_x) into ctrl->res_bits;
// `final_pass` subtracts the pressure mean.
void launch_residual(const ProjectionArgs& a, const float* x, const float* b, ProjControl* ctrl, bool final_pass,
                     cudaStream_t s);
// Record a residual check: iterations/final residual/converged/done. With
// `accumulate` the iteration count grows by min(iterations, budget left),
// else it is set to `iterations`. `flip_x64` swaps the mixed-precision
// buffers (after a re-centring pass).
void launch_check(ProjControl* ctrl, int iterations, bool accumulate, bool flip_x64, LoopCond cond,
                  cudaStream_t s);
// Pressure mean (deterministic FP64 sum) into ctrl->p_mean_f.
void launch_pressure_mean(const ProjectionArgs& a, const float* x, double* partials, int partial_capacity,
                          ProjControl* ctrl, cudaStream_t s);
// u_out = walls(u_in - dt grad(x - mean)) and max |div u_out|; when hat
// pointers are given also hat = 2 u_out - u_in (the reflection step).
void launch_gradient(const ProjectionArgs& a, const float* x, const float* u_in, const float* v_in,
                     const float* w_in, float* u_out, float* v_out, float* w_out, float* u_hat, float* v_hat,
                     float* w_hat, ProjControl* ctrl, cudaStream_t s);
// Natural-order zero-mean pressure (x - ctrl->p_mean_f) from the split iterate.
void launch_unsplit_pressure(const Grid& g, const float* p, const ProjControl* ctrl, float* out, cudaStream_t s);
// Assemble ctrl->result from the accumulators.
void launch_finish_projection(ProjControl* ctrl, cudaStream_t s);

// ---- flexible PCG (kernels_fpcg.cu) ----
// Vectors are FP32 in the split layout (count = rb_count(n) slots, padding
// zero). Partials need cg_partial_capacity(n) doubles.
int cg_partial_capacity(int n);
// q = A p.
void launch_apply_A(int n, const float* p, float* q, cudaStream_t s);
// cg->rho = z.r (FP64).
void launch_cg_rho(size_t count, const float* z, const float* r, double* partials, CgControl* cg, cudaStream_t s);
// cg->alpha = rho / p.q.
void launch_cg_alpha(size_t count, const float* p, const float* q, double* partials, CgControl* cg,
                     cudaStream_t s);
// q = A p and cg->alpha = rho / p.q in one pass over p (two launches).
// diag: the solid-obstacle mask (split-layout fluid-neighbour counts), or null.
void launch_apply_A_alpha(int n, const float* p, float* q, double* partials, CgControl* cg, cudaStream_t s,
                          const uint8_t* diag = nullptr);
// e += alpha p; r -= alpha q; then count the iteration and decide the FP64
// re-centring (ctrl->recentre, and the graph if-condition when active).
void launch_cg_update(size_t count, float* e, float* r, const float* p, const float* q, const CgControl* cg,
                      ProjControl* ctrl, LoopCond recentre_cond, cudaStream_t s);
// beta = -alpha z.q / rho; rho = z.r.
void launch_cg_beta(size_t count, const float* z, const float* r, const float* q, double* partials, CgControl* cg,
                    cudaStream_t s);
// beta and rho from `blocks` pairs of partials of z.r and z.q already written.
void launch_cg_beta_finish(const double* partials, int blocks, CgControl* cg, cudaStream_t s);
// p = z + beta p.
void launch_cg_direction(size_t count, float* p, const float* z, const CgControl* cg, cudaStream_t s);
// The fused form of one CG step's direction and update passes (n % 8 == 0),
// with the direction in two buffers p[2] (cg->p_cur the current):
// launch_cg_direction_apply: e += alpha_pending p_cur (the previous step's
// deferred update), p_new = z + beta p_cur (z when beta == 0) into the other
// buffer, q = A p_new, alpha = rho / (p_new.q), p_cur = new, alpha_pending =
// alpha. launch_cg_update_r: r -= alpha q with max |r|, then the decision.
// launch_cg_fold (gated, before a re-centring): e += alpha_pending p_cur,
// alpha_pending = 0. Same values as the unfused sequence, bit for bit.
void launch_cg_direction_apply(int n, const float* z, float* const* p, float* e, float* q, double* partials,
                               CgControl* cg, cudaStream_t s);
void launch_cg_update_r(size_t count, float* r, const float* q, const CgControl* cg, ProjControl* ctrl,
                        LoopCond recentre_cond, cudaStream_t s);
void launch_cg_fold(size_t count, float* e, float* const* p, CgControl* cg, const ProjControl* ctrl, cudaStream_t s);
// rc = 4^3 block sums of r - A z on the (n/4)^3 grid (natural layout); n % 4 == 0.
// `rows` holds n^3 / 4 floats of scratch.
void launch_restrict_residual(int n, const float* r, const float* z, float* rows, float* rc, cudaStream_t s,
                              const uint8_t* diag = nullptr);
// Appends the coarse right-hand side (cells floats) to a device ring of
// `capacity` records: record *counter % capacity, then ++*counter.
void launch_log_coarse(const float* rc, size_t cells, float* log, int capacity, int* counter, cudaStream_t s);
// z += gamma (P zc - mean zc), gamma by the Galerkin condition on the coarse grid.
void launch_coarse_correction(int n, float* z, const float* zc, const float* rc, double* partials, CgControl* cg,
                              cudaStream_t s, const uint8_t* diag = nullptr);

// ---- headless rendering (kernels_render.cu) ----
void render_volume(const float* density, int n, float box, const vapor_render_params& p, float* rgb, cudaStream_t s);

// ---- diagnostics ----
// Comparison metrics of (d, u, v, w) (kernels_metrics.cu); waits for the
// stream; VAPOR_NON_FINITE on a non-finite divergence.
void comparison_metrics(const Grid& g, float fps, float cfl_limit, const float* d, const float* u, const float* v,
                        const float* w, vapor_comparison_metrics* out, cudaStream_t s);
void launch_diagnostics(const Grid& g, const float* u, const float* v, const float* w, double* partials,
                        int partial_capacity, DiagControl* diag, cudaStream_t s);

int reduction_blocks(size_t count);

// Number of kernels this library has launched (all handles, all threads).
void count_launch();
long long launch_count();

}  // namespace vb
