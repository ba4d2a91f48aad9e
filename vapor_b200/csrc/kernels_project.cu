// Closed-box pressure projection (reference: src/solvers/mac3d/
// CpuPressureSolver3D.cpp:25-60, SOR.cpp:22-64, StencilLinearSystem.cpp:53-70,
// MacGridOperators3D.cpp:8-67).
//
// The Neumann system A = -h^2 Laplacian is never stored: the diagonal is the
// number of existing neighbours and every coupling is -1, computed on the fly.
// b and x are FP32 as in the reference; the right-hand-side mean and the
// pressure mean are kept as scalars and subtracted on the fly, which yields the
// same FP32 values as the reference's in-place subtraction. Sums use fixed-order
// (deterministic) FP64 reductions; maxima use exact atomics on bit patterns.
#include "kernels.hpp"

#include <algorithm>
#include <atomic>
#include <climits>

namespace vb {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxReductionBlocks = 148 * 8;

__device__ __forceinline__ void decode_cell(size_t c, int n, int& x, int& y, int& z) {
    const size_t nn = size_t(n) * n;
    z = int(c / nn);
    const size_t r = c - size_t(z) * nn;
    y = int(r / n);
    x = int(r - size_t(y) * n);
}

__device__ __forceinline__ int neighbours(int n, int x, int y, int z) {
    return (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
}

__device__ __forceinline__ int block_min_int(int v, int* scratch) {
    return -block_max(v == INT_MIN ? INT_MAX : -v, scratch);
}

__global__ void k_begin_projection(ProjControl* ctrl, vapor_linear_solve_options o) {
    ctrl->div_before_bits = 0u;
    ctrl->div_after_bits = 0u;
    ctrl->rhs_max_key = INT_MIN;
    ctrl->rhs_min_key = INT_MAX;
    ctrl->res_bits = 0ull;
    ctrl->nonfinite = 0u;
    ctrl->rhs_mean_f = 0.f;
    ctrl->p_mean_f = 0.f;
    ctrl->p_mean64 = 0.0;
    ctrl->removed_mean = 0.0;
    ctrl->target = 0.0;
    ctrl->iterations = 0;
    ctrl->done = 0;
    ctrl->max_iterations = o.max_iterations;
    ctrl->check_interval = o.residual_check_interval;
    ctrl->fixed = o.fixed_iterations;
    ctrl->continue_flag = 0;
    vapor_projection_result r = {};
    ctrl->result = r;
}

// b = -div(walls(u)) * h^2/dt; walls read as zero, which equals enforcing the
// closed boundaries before computing the divergence.
__global__ void __launch_bounds__(kThreads) k_rhs(Grid g, float scale, const float* __restrict__ u,
                                                  const float* __restrict__ v, const float* __restrict__ w,
                                                  float* __restrict__ b, double* __restrict__ partials,
                                                  ProjControl* ctrl) {
    __shared__ double s_sum[32];
    __shared__ float s_max[32];
    __shared__ int s_key[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    double sum = 0.0;
    float div_max = 0.f;
    int kmax = INT_MIN, kmin = INT_MAX;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        const float u0 = x == 0 ? 0.f : u[index_of(n, FACE_X, x, y, z)];
        const float u1 = x + 1 == n ? 0.f : u[index_of(n, FACE_X, x + 1, y, z)];
        const float v0 = y == 0 ? 0.f : v[index_of(n, FACE_Y, x, y, z)];
        const float v1 = y + 1 == n ? 0.f : v[index_of(n, FACE_Y, x, y + 1, z)];
        const float w0 = z == 0 ? 0.f : w[index_of(n, FACE_Z, x, y, z)];
        const float w1 = z + 1 == n ? 0.f : w[index_of(n, FACE_Z, x, y, z + 1)];
        const float div = (u1 - u0 + v1 - v0 + w1 - w0) / g.h;
        if (!isfinite(div)) bad = 1u;
        div_max = maxf_ref(div_max, fabsf(div));
        const float rhs = -div * scale;
        b[c] = rhs;
        sum += double(rhs);
        const int key = float_order_key(rhs);
        kmax = max(kmax, key);
        kmin = min(kmin, key);
    }
    const double bs = block_sum(sum, s_sum);
    const float bm = block_max(div_max, s_max);
    const int bkmax = block_max(kmax, s_key);
    __syncthreads();
    const int bkmin = block_min_int(kmin, s_key);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = bs;
        atomic_max_nonneg(&ctrl->div_before_bits, bm);
        atomicMax(&ctrl->rhs_max_key, bkmax);
        atomicMin(&ctrl->rhs_min_key, bkmin);
        if (any_bad) atomicOr(&ctrl->nonfinite, 1u);
    }
}

// Deterministic sum of the block partials, then the mean, the initial
// residual and the stopping target (SOR.cpp:28-33).
__global__ void k_rhs_finish(ProjControl* ctrl, const double* __restrict__ partials, int blocks, double cells,
                             double abs_tol, double rel_tol) {
    __shared__ double s_sum[32];
    double sum = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) sum += partials[i];
    const double total = block_sum(sum, s_sum);
    if (threadIdx.x != 0) return;
    const double mean = total / cells;
    const float mf = float(mean);
    ctrl->removed_mean = mean;
    ctrl->rhs_mean_f = mf;
    // With x0 = 0 the residual is max |fl(b - mean)|; FP32 rounding is monotone,
    // so the maximum is attained at the largest or the smallest b.
    const float bmax = key_to_float(ctrl->rhs_max_key), bmin = key_to_float(ctrl->rhs_min_key);
    const double r0 = fmax(fabs(double(bmax - mf)), fabs(double(bmin - mf)));
    const double target = fmax(abs_tol, rel_tol * r0);
    ctrl->target = target;
    const int converged = r0 <= target;
    ctrl->result.linear_solve.initial_residual = r0;
    ctrl->result.linear_solve.final_residual = r0;
    ctrl->result.linear_solve.converged = converged;
    ctrl->result.linear_solve.iterations = 0;
    ctrl->done = (converged && !ctrl->fixed) || ctrl->max_iterations == 0 || ctrl->nonfinite != 0u;
}

// One colour of red-black SOR (SOR.cpp:36-54) in the reference's operation
// order: off = sum(-1 * x_nb) over existing neighbours in x-,x+,y-,y+,z-,z+
// order; x += omega * (b - off - diag * x) / max(diag, floor).
__global__ void __launch_bounds__(kThreads) k_sor_color(Grid g, int parity, float omega, float floor_diag,
                                                        float* __restrict__ x, const float* __restrict__ b,
                                                        const ProjControl* __restrict__ ctrl, int guarded,
                                                        int subtract_mean) {
    if (guarded && ctrl->done) return;
    const int n = g.n;
    const int half = (n + 1) >> 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    const int y = t / half;
    if (y >= n) return;
    const int i = 2 * (t - y * half) + ((y + z + parity) & 1);
    if (i >= n) return;
    const size_t nn = size_t(n) * n;
    const size_t id = size_t(i) + size_t(n) * (size_t(y) + size_t(n) * z);
    const float diag = float(neighbours(n, i, y, z));
    if (diag == 0.f) return;
    float off = 0.f;
    if (i > 0) off += -1.f * x[id - 1];
    if (i + 1 < n) off += -1.f * x[id + 1];
    if (y > 0) off += -1.f * x[id - n];
    if (y + 1 < n) off += -1.f * x[id + n];
    if (z > 0) off += -1.f * x[id - nn];
    if (z + 1 < n) off += -1.f * x[id + nn];
    const float relax = maxf_ref(diag, floor_diag);
    const float bi = subtract_mean ? b[id] - ctrl->rhs_mean_f : b[id];
    const float xi = x[id];
    x[id] = xi + omega * (bi - off - diag * xi) / relax;
}

// Mixed precision re-centring: x_out = x_in + e and r32 = float(b' - A x_out),
// both in FP64, with the neighbour order of the reference residual.
__global__ void __launch_bounds__(kThreads) k_refine_residual(Grid g, const float* __restrict__ b,
                                                              const double* __restrict__ xin,
                                                              const float* __restrict__ e,
                                                              double* __restrict__ xout, float* __restrict__ r32,
                                                              ProjControl* ctrl) {
    __shared__ double s_max[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const size_t nn = size_t(n) * n;
    const float bm = ctrl->rhs_mean_f;
    double r = 0.0;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        auto xv = [&](size_t id) { return xin[id] + double(e[id]); };
        const double xc = xv(c);
        double ax = double(neighbours(n, i, j, k)) * xc;
        if (i > 0) ax -= xv(c - 1);
        if (i + 1 < n) ax -= xv(c + 1);
        if (j > 0) ax -= xv(c - n);
        if (j + 1 < n) ax -= xv(c + n);
        if (k > 0) ax -= xv(c - nn);
        if (k + 1 < n) ax -= xv(c + nn);
        const float bi = b[c] - bm;
        const double res = double(bi) - ax;
        if (!isfinite(res)) bad = 1u;
        xout[c] = xc;
        r32[c] = float(res);
        const double a = fabs(res);
        r = r < a ? a : r;
    }
    const double br = block_max(r, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->res_bits, br);
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

__global__ void __launch_bounds__(kThreads) k_psum64(Grid g, const double* __restrict__ x,
                                                     double* __restrict__ partials) {
    __shared__ double s_sum[32];
    const size_t cells = size_t(g.n) * g.n * g.n;
    double sum = 0.0;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x)
        sum += x[c];
    const double bs = block_sum(sum, s_sum);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

__global__ void k_psum64_finish(ProjControl* ctrl, const double* __restrict__ partials, int blocks, double cells) {
    __shared__ double s_sum[32];
    double sum = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) sum += partials[i];
    const double total = block_sum(sum, s_sum);
    if (threadIdx.x == 0) {
        ctrl->p_mean64 = total / cells;
        ctrl->p_mean_f = 0.f;
    }
}

// Final FP64 residual of x64 - mean (StencilLinearSystem.cpp:53-70 order) and
// the float pressure copy.
__global__ void __launch_bounds__(kThreads) k_residual64(Grid g, const double* __restrict__ x,
                                                         const float* __restrict__ b, float* __restrict__ p32,
                                                         ProjControl* ctrl) {
    __shared__ double s_max[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const size_t nn = size_t(n) * n;
    const float bm = ctrl->rhs_mean_f;
    const double pm = ctrl->p_mean64;
    double r = 0.0;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        auto xv = [&](size_t id) { return x[id] - pm; };
        const double xc = xv(c);
        double ax = double(float(neighbours(n, i, j, k))) * xc;
        if (i > 0) ax += -1.0 * xv(c - 1);
        if (i + 1 < n) ax += -1.0 * xv(c + 1);
        if (j > 0) ax += -1.0 * xv(c - n);
        if (j + 1 < n) ax += -1.0 * xv(c + n);
        if (k > 0) ax += -1.0 * xv(c - nn);
        if (k + 1 < n) ax += -1.0 * xv(c + nn);
        const float bi = b[c] - bm;
        if (!isfinite(xc)) bad = 1u;
        p32[c] = float(xc);
        const double a = fabs(double(bi) - ax);
        r = r < a ? a : r;
    }
    const double br = block_max(r, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->res_bits, br);
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

// Gradient with an FP64 pressure: u_out = float(u - dt (p1 - p0) / h) in FP64.
__global__ void __launch_bounds__(kThreads) k_gradient64(Grid g, float dt, const double* __restrict__ p,
                                                         const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, float* __restrict__ uo,
                                                         float* __restrict__ vo, float* __restrict__ wo,
                                                         float* __restrict__ uh, float* __restrict__ vh,
                                                         float* __restrict__ wh, ProjControl* ctrl) {
    __shared__ float s_max[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const size_t nn = size_t(n) * n;
    const double hInv = 1.0 / double(g.h), dtd = double(dt);
    const double pm = ctrl->p_mean64;
    float div_max = 0.f;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        const double pc = p[c] - pm;
        const size_t ix0 = index_of(n, FACE_X, x, y, z), ix1 = ix0 + 1;
        const size_t iy0 = index_of(n, FACE_Y, x, y, z), iy1 = iy0 + n;
        const size_t iz0 = c, iz1 = c + nn;
        const float ux0 = x == 0 ? 0.f : float(double(u[ix0]) - dtd * (pc - (p[c - 1] - pm)) * hInv);
        const float ux1 = x + 1 == n ? 0.f : float(double(u[ix1]) - dtd * ((p[c + 1] - pm) - pc) * hInv);
        const float vy0 = y == 0 ? 0.f : float(double(v[iy0]) - dtd * (pc - (p[c - n] - pm)) * hInv);
        const float vy1 = y + 1 == n ? 0.f : float(double(v[iy1]) - dtd * ((p[c + n] - pm) - pc) * hInv);
        const float wz0 = z == 0 ? 0.f : float(double(w[iz0]) - dtd * (pc - (p[c - nn] - pm)) * hInv);
        const float wz1 = z + 1 == n ? 0.f : float(double(w[iz1]) - dtd * ((p[c + nn] - pm) - pc) * hInv);
        uo[ix0] = ux0;
        vo[iy0] = vy0;
        wo[iz0] = wz0;
        if (x + 1 == n) uo[ix1] = ux1;
        if (y + 1 == n) vo[iy1] = vy1;
        if (z + 1 == n) wo[iz1] = wz1;
        if (uh) {
            uh[ix0] = 2.f * ux0 - u[ix0];
            vh[iy0] = 2.f * vy0 - v[iy0];
            wh[iz0] = 2.f * wz0 - w[iz0];
            if (x + 1 == n) uh[ix1] = 2.f * ux1 - u[ix1];
            if (y + 1 == n) vh[iy1] = 2.f * vy1 - v[iy1];
            if (z + 1 == n) wh[iz1] = 2.f * wz1 - w[iz1];
        }
        const float div = (ux1 - ux0 + vy1 - vy0 + wz1 - wz0) / g.h;
        if (!isfinite(div)) bad = 1u;
        div_max = maxf_ref(div_max, fabsf(div));
    }
    const float bm = block_max(div_max, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->div_after_bits, bm);
        if (any_bad) atomicOr(&ctrl->nonfinite, 2u);
    }
}

// FP64 infinity norm of b' - A x' (StencilLinearSystem.cpp:53-70) with
// b' = b - rhs mean and, on the final pass, x' = x - pressure mean.
__global__ void __launch_bounds__(kThreads) k_residual(Grid g, const float* __restrict__ x,
                                                       const float* __restrict__ b, ProjControl* ctrl,
                                                       int final_pass) {
    __shared__ double s_max[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const size_t nn = size_t(n) * n;
    const float bm = ctrl->rhs_mean_f;
    const float pm = final_pass ? ctrl->p_mean_f : 0.f;
    double r = 0.0;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        auto xv = [&](size_t id) { return final_pass ? x[id] - pm : x[id]; };
        const float xc = xv(c);
        double ax = double(float(neighbours(n, i, j, k))) * double(xc);
        if (i > 0) ax += -1.0 * double(xv(c - 1));
        if (i + 1 < n) ax += -1.0 * double(xv(c + 1));
        if (j > 0) ax += -1.0 * double(xv(c - n));
        if (j + 1 < n) ax += -1.0 * double(xv(c + n));
        if (k > 0) ax += -1.0 * double(xv(c - nn));
        if (k + 1 < n) ax += -1.0 * double(xv(c + nn));
        const float bi = b[c] - bm;
        if (!isfinite(xc) || !isfinite(bi)) bad = 1u;
        const double e = fabs(double(bi) - ax);
        r = r < e ? e : r;
    }
    const double br = block_max(r, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->res_bits, br);
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

// Records one residual check (SOR.cpp:56-61): iterations, final residual,
// converged, and whether the loop stops. Optionally sets the CUDA graph
// while-condition so the loop can run on the device without the host.
__global__ void k_check(ProjControl* ctrl, int iterations_done, int use_conditional,
                        cudaGraphConditionalHandle handle, int add_to_iterations) {
    if (add_to_iterations) ctrl->iterations += iterations_done;
    else ctrl->iterations = iterations_done;
    const double res = __longlong_as_double((long long)ctrl->res_bits);
    ctrl->res_bits = 0ull;
    const int converged = res <= ctrl->target;
    ctrl->result.linear_solve.iterations = ctrl->iterations;
    ctrl->result.linear_solve.final_residual = res;
    ctrl->result.linear_solve.converged = converged;
    const int stop = (converged && !ctrl->fixed) || ctrl->iterations >= ctrl->max_iterations ||
                     (ctrl->nonfinite & 4u) != 0u;
    ctrl->done = stop;
    ctrl->continue_flag = !stop;
    if (use_conditional) cudaGraphSetConditional(handle, stop ? 0u : 1u);
}

__global__ void __launch_bounds__(kThreads) k_psum(Grid g, const float* __restrict__ x,
                                                   double* __restrict__ partials) {
    __shared__ double s_sum[32];
    const size_t cells = size_t(g.n) * g.n * g.n;
    double sum = 0.0;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x)
        sum += double(x[c]);
    const double bs = block_sum(sum, s_sum);
    if (threadIdx.x == 0) partials[blockIdx.x] = bs;
}

__global__ void k_psum_finish(ProjControl* ctrl, const double* __restrict__ partials, int blocks, double cells) {
    __shared__ double s_sum[32];
    double sum = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) sum += partials[i];
    const double total = block_sum(sum, s_sum);
    if (threadIdx.x == 0) ctrl->p_mean_f = float(total / cells);
}

// Final residual after the pressure gauge (CpuPressureSolver3D.cpp:50-56).
__global__ void k_final_check(ProjControl* ctrl) {
    const double res = __longlong_as_double((long long)ctrl->res_bits);
    ctrl->res_bits = 0ull;
    ctrl->result.linear_solve.final_residual = res;
    ctrl->result.linear_solve.converged = res <= ctrl->target;
    ctrl->result.linear_solve.iterations = ctrl->iterations;
}

// Gradient step on interior faces, zero walls, divergence after, and the
// reflected velocity hat = 2 u_out - u_in (MacGridFluidSolver3D.cpp:213-218).
// One thread per cell owns the cell's low faces and, on the last layer, the
// high wall faces.
__global__ void __launch_bounds__(kThreads) k_gradient(Grid g, float dt, const float* __restrict__ p,
                                                       const float* __restrict__ u, const float* __restrict__ v,
                                                       const float* __restrict__ w, float* __restrict__ uo,
                                                       float* __restrict__ vo, float* __restrict__ wo,
                                                       float* __restrict__ uh, float* __restrict__ vh,
                                                       float* __restrict__ wh, ProjControl* ctrl) {
    __shared__ float s_max[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const size_t nn = size_t(n) * n;
    const float hInv = 1.f / g.h;
    const float pm = ctrl->p_mean_f;
    float div_max = 0.f;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        const float pc = p[c] - pm;
        const size_t ix0 = index_of(n, FACE_X, x, y, z), ix1 = ix0 + 1;
        const size_t iy0 = index_of(n, FACE_Y, x, y, z), iy1 = iy0 + n;
        const size_t iz0 = c, iz1 = c + nn;
        const float ux0 = x == 0 ? 0.f : u[ix0] - dt * (pc - (p[c - 1] - pm)) * hInv;
        const float ux1 = x + 1 == n ? 0.f : u[ix1] - dt * ((p[c + 1] - pm) - pc) * hInv;
        const float vy0 = y == 0 ? 0.f : v[iy0] - dt * (pc - (p[c - n] - pm)) * hInv;
        const float vy1 = y + 1 == n ? 0.f : v[iy1] - dt * ((p[c + n] - pm) - pc) * hInv;
        const float wz0 = z == 0 ? 0.f : w[iz0] - dt * (pc - (p[c - nn] - pm)) * hInv;
        const float wz1 = z + 1 == n ? 0.f : w[iz1] - dt * ((p[c + nn] - pm) - pc) * hInv;
        uo[ix0] = ux0;
        vo[iy0] = vy0;
        wo[iz0] = wz0;
        if (x + 1 == n) uo[ix1] = ux1;
        if (y + 1 == n) vo[iy1] = vy1;
        if (z + 1 == n) wo[iz1] = wz1;
        if (uh) {
            uh[ix0] = 2.f * ux0 - u[ix0];
            vh[iy0] = 2.f * vy0 - v[iy0];
            wh[iz0] = 2.f * wz0 - w[iz0];
            if (x + 1 == n) uh[ix1] = 2.f * ux1 - u[ix1];
            if (y + 1 == n) vh[iy1] = 2.f * vy1 - v[iy1];
            if (z + 1 == n) wh[iz1] = 2.f * wz1 - w[iz1];
        }
        const float div = (ux1 - ux0 + vy1 - vy0 + wz1 - wz0) / g.h;
        if (!isfinite(div)) bad = 1u;
        div_max = maxf_ref(div_max, fabsf(div));
    }
    const float bm = block_max(div_max, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->div_after_bits, bm);
        if (any_bad) atomicOr(&ctrl->nonfinite, 2u);
    }
}

__global__ void k_finish_projection(ProjControl* ctrl) {
    ctrl->sticky_nonfinite |= ctrl->nonfinite;
    ctrl->total_iterations += ctrl->iterations;
    ctrl->result.residual_available = 1;
    ctrl->result.divergence_before = __uint_as_float(ctrl->div_before_bits);
    ctrl->result.divergence_after = __uint_as_float(ctrl->div_after_bits);
    ctrl->result.removed_rhs_mean = ctrl->removed_mean;
    ctrl->result.linear_solve.iterations = ctrl->iterations;
}

__global__ void __launch_bounds__(kThreads) k_diagnostics(Grid g, const float* __restrict__ u,
                                                          const float* __restrict__ v,
                                                          const float* __restrict__ w,
                                                          double* __restrict__ partials, DiagControl* diag) {
    __shared__ double s_sum[32];
    __shared__ float s_max[32];
    const int n = g.n;
    const size_t faces = size_t(n) * n * (n + 1);
    const size_t cells = size_t(n) * n * n;
    double ke = 0.0;
    float vmax = 0.f, dmax = 0.f;
    unsigned int bad = 0u;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < faces; i += size_t(gridDim.x) * blockDim.x) {
        const float a = u[i], b = v[i], c = w[i];
        ke += double(a) * double(a) + double(b) * double(b) + double(c) * double(c);
        vmax = maxf_ref(vmax, fabsf(a));
        vmax = maxf_ref(vmax, fabsf(b));
        vmax = maxf_ref(vmax, fabsf(c));
        if (i < cells) {
            int x, y, z;
            decode_cell(i, n, x, y, z);
            const float d = (u[index_of(n, FACE_X, x + 1, y, z)] - u[index_of(n, FACE_X, x, y, z)] +
                             v[index_of(n, FACE_Y, x, y + 1, z)] - v[index_of(n, FACE_Y, x, y, z)] +
                             w[index_of(n, FACE_Z, x, y, z + 1)] - w[index_of(n, FACE_Z, x, y, z)]) /
                            g.h;
            if (!isfinite(d)) bad = 1u;
            dmax = maxf_ref(dmax, fabsf(d));
        }
    }
    const double bs = block_sum(ke, s_sum);
    const float bv = block_max(vmax, s_max);
    __syncthreads();
    const float bd = block_max(dmax, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = bs;
        atomic_max_nonneg(&diag->max_velocity_bits, bv);
        atomic_max_nonneg(&diag->max_divergence_bits, bd);
        if (any_bad) atomicOr(&diag->nonfinite, 1u);
    }
}

__global__ void k_diag_begin(DiagControl* diag) {
    diag->max_velocity_bits = 0u;
    diag->max_divergence_bits = 0u;
    diag->nonfinite = 0u;
    diag->kinetic_sum = 0.0;
}

__global__ void k_diag_finish(DiagControl* diag, const double* __restrict__ partials, int blocks) {
    __shared__ double s_sum[32];
    double sum = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) sum += partials[i];
    const double total = block_sum(sum, s_sum);
    if (threadIdx.x == 0) diag->kinetic_sum = total;
}

}  // namespace

namespace {
std::atomic<long long> g_launches{0};
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

int reduction_blocks(size_t count) {
    const size_t b = (count + size_t(kThreads) * 8 - 1) / (size_t(kThreads) * 8);
    return int(std::max<size_t>(1, std::min<size_t>(b, kMaxReductionBlocks)));
}

void launch_rhs(const ProjectionArgs& a, const float* u, const float* v, const float* w, float* b,
                double* partials, int partial_capacity, ProjControl* ctrl, cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    const int blocks = std::min(reduction_blocks(cells), partial_capacity);
    const float scale = a.g.h * a.g.h / a.dt;
    count_launch();
    k_begin_projection<<<1, 1, 0, s>>>(ctrl, a.options);
    count_launch();
    k_rhs<<<blocks, kThreads, 0, s>>>(a.g, scale, u, v, w, b, partials, ctrl);
    count_launch();
    k_rhs_finish<<<1, 1024, 0, s>>>(ctrl, partials, blocks, double(cells), a.options.absolute_tolerance,
                                    a.options.relative_tolerance);
}

void launch_sor_color(const ProjectionArgs& a, int parity, float* x, const float* b, const ProjControl* ctrl,
                      bool guarded, cudaStream_t s, bool subtract_mean) {
    const int n = a.g.n;
    const int half = (n + 1) / 2;
    const dim3 grid((half * n + kThreads - 1) / kThreads, n);
    count_launch();
    k_sor_color<<<grid, kThreads, 0, s>>>(a.g, parity, a.omega, a.diagonal_floor, x, b, ctrl, guarded ? 1 : 0,
                                          subtract_mean ? 1 : 0);
}

void launch_refine_residual(const ProjectionArgs& a, const float* b, const double* x_in, const float* e,
                            double* x_out, float* r32, ProjControl* ctrl, cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    count_launch();
    k_refine_residual<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, b, x_in, e, x_out, r32, ctrl);
}

void launch_pressure_mean64(const ProjectionArgs& a, const double* x64, const float* b, float* p32,
                            double* partials, int partial_capacity, ProjControl* ctrl, cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    const int blocks = std::min(reduction_blocks(cells), partial_capacity);
    count_launch();
    k_psum64<<<blocks, kThreads, 0, s>>>(a.g, x64, partials);
    count_launch();
    k_psum64_finish<<<1, 1024, 0, s>>>(ctrl, partials, blocks, double(cells));
    count_launch();
    k_residual64<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, x64, b, p32, ctrl);
    count_launch();
    k_final_check<<<1, 1, 0, s>>>(ctrl);
}

void launch_gradient64(const ProjectionArgs& a, const double* x64, const float* u_in, const float* v_in,
                       const float* w_in, float* u_out, float* v_out, float* w_out, float* u_hat, float* v_hat,
                       float* w_hat, ProjControl* ctrl, cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    count_launch();
    k_gradient64<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, a.dt, x64, u_in, v_in, w_in, u_out, v_out,
                                                              w_out, u_hat, v_hat, w_hat, ctrl);
}

void launch_residual(const ProjectionArgs& a, const float* x, const float* b, ProjControl* ctrl, bool final_pass,
                     cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    count_launch();
    k_residual<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, x, b, ctrl, final_pass ? 1 : 0);
    if (final_pass) {
        count_launch();
        k_final_check<<<1, 1, 0, s>>>(ctrl);
    }
}

void launch_check(ProjControl* ctrl, int iterations_done, bool graph_conditional, unsigned long long cond_handle,
                  cudaStream_t s) {
    count_launch();
    k_check<<<1, 1, 0, s>>>(ctrl, iterations_done, graph_conditional ? 1 : 0,
                            (cudaGraphConditionalHandle)cond_handle, graph_conditional ? 1 : 0);
}

void launch_pressure_mean(const ProjectionArgs& a, const float* x, double* partials, int partial_capacity,
                          ProjControl* ctrl, cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    const int blocks = std::min(reduction_blocks(cells), partial_capacity);
    count_launch();
    k_psum<<<blocks, kThreads, 0, s>>>(a.g, x, partials);
    count_launch();
    k_psum_finish<<<1, 1024, 0, s>>>(ctrl, partials, blocks, double(cells));
}

void launch_gradient(const ProjectionArgs& a, const float* x, const float* u_in, const float* v_in,
                     const float* w_in, float* u_out, float* v_out, float* w_out, float* u_hat, float* v_hat,
                     float* w_hat, ProjControl* ctrl, cudaStream_t s) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    count_launch();
    k_gradient<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, a.dt, x, u_in, v_in, w_in, u_out, v_out, w_out,
                                                            u_hat, v_hat, w_hat, ctrl);
}

void launch_finish_projection(ProjControl* ctrl, cudaStream_t s) {
    count_launch();
    k_finish_projection<<<1, 1, 0, s>>>(ctrl);
}

void launch_diagnostics(const Grid& g, const float* u, const float* v, const float* w, double* partials,
                        int partial_capacity, DiagControl* diag, cudaStream_t s) {
    const size_t faces = size_t(g.n) * g.n * (g.n + 1);
    const int blocks = std::min(reduction_blocks(faces), partial_capacity);
    count_launch();
    k_diag_begin<<<1, 1, 0, s>>>(diag);
    count_launch();
    k_diagnostics<<<blocks, kThreads, 0, s>>>(g, u, v, w, partials, diag);
    count_launch();
    k_diag_finish<<<1, 1024, 0, s>>>(diag, partials, blocks);
}

}  // namespace vb
