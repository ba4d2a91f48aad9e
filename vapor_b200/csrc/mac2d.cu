// MAC 2D smoke solver on the device: the step of the reference's
// MacGridFluidSolver2D (src/solvers/mac2d/MacGridFluidSolver2D.cpp:22-128)
// with its semi-Lagrangian advection (SemiLagrangian2D.cpp:13-50), FP64
// red-black SOR projection (CpuPressureSolver2D.cpp:8-82) and wall/gradient
// operators (MacGridOperators2D.cpp:13-41).
//
// Parity with the reference's CPU arithmetic:
//   - one thread per sample point or cell, the reference's expressions in its
//     order (the library builds with --fmad=false, so nothing is contracted);
//   - std::lerp is restated as the C++ standard library defines it (the
//     published P0811 algorithm: the exact form when the end points straddle
//     zero, b at t == 1, else a + t (b - a) clamped to stay monotonic);
//   - the red-black sweep is the reference's: within one parity no cell is a
//     neighbour of another, so the cells of a parity update in any order;
//   - the FP64 means of the right-hand side and of the pressure are
//     sequential sums (std::accumulate's order) on one thread, and the
//     kinetic energy likewise;
//   - the emitter's Gaussian weights exp(-3.5 q) and the decay exp(-dt k)
//     are evaluated on the host with the C library, as the reference does;
//   - buoyancy's d^(1/4) is the C library's powf(d, .25f) bit for bit
//     (powf_quarter.cuh: the correctly rounded root corrected by a table of
//     the library's one-ulp differences).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "engine.hpp"
#include "powf_quarter.cuh"

namespace vb {
namespace {

constexpr int kThreads2 = 256;

int blocks2(long count) { return int(std::max<long>(1, (count + kThreads2 - 1) / kThreads2)); }

// Device flags of a step (bits) and FP64 scalars.
struct Mac2DControl {
    unsigned int flags;            // 1 non-finite advection input, 2 non-finite backtrace, 4 non-finite
                                   // divergence, 8 RHS overflow, 16 non-finite pressure, 32 non-finite
                                   // velocity before a projection
    unsigned int div_bits;         // max |div| (float bits)
    unsigned long long res_bits;   // max |residual| (double bits)
    double sum;                    // sequential sum
};

// std::lerp (C++20), the standard library's algorithm.
__device__ __forceinline__ float lerp_std(float a, float b, float t) {
    if ((a <= 0.f && b >= 0.f) || (a >= 0.f && b <= 0.f)) return t * b + (1.f - t) * a;
    if (t == 1.f) return b;
    const float x = a + t * (b - a);
    return (t > 1.f) == (b > a) ? (b < x ? x : b) : (b > x ? x : b);
}

__device__ __forceinline__ float clamp_std(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }

// Bilinear sample in index coordinates clamped to the boundary samples
// (SemiLagrangian2D.cpp:13-22); a non-finite coordinate sets flag 2.
__device__ __forceinline__ float sample2(const float* __restrict__ f, int w, int h, float x, float y,
                                         unsigned int& flags) {
    if (!isfinite(x) || !isfinite(y)) {
        flags |= 2u;
        return 0.f;
    }
    x = clamp_std(x, 0.f, float(w - 1));
    y = clamp_std(y, 0.f, float(h - 1));
    const int i = int(floorf(x)), j = int(floorf(y));
    const int ip = min(i + 1, w - 1), jp = min(j + 1, h - 1);
    const float tx = x - float(i), ty = y - float(j);
    return lerp_std(lerp_std(f[i + w * j], f[ip + w * j], tx), lerp_std(f[i + w * jp], f[ip + w * jp], tx), ty);
}

// Closed walls: the normal velocity on the box faces is zero
// (MacGridOperators2D.cpp:13-19).
__global__ void k2_walls(int n, float* __restrict__ u, float* __restrict__ v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u[size_t(n + 1) * i] = 0.f;
    u[size_t(n + 1) * i + n] = 0.f;
    v[i] = 0.f;
    v[size_t(n) * n + i] = 0.f;
}

// One field of SemiLagrangian2D::advect (loc 0 density, 1 u faces, 2 v
// faces). The launch covers max(w h, n (n + 1)) threads so that, as the
// reference does before advecting, every value of the source and of both
// velocity arrays is checked for finiteness.
__global__ void k2_advect(int n, int loc, float dt_over_h, const float* __restrict__ src,
                          const float* __restrict__ vx, const float* __restrict__ vy, float* __restrict__ out,
                          Mac2DControl* ctrl) {
    const int w = n + (loc == 1), h = n + (loc == 2);
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const long faces = long(n) * (n + 1), points = long(w) * h;
    unsigned int flags = 0u;
    if (i < points && !isfinite(src[i])) flags |= 1u;
    if (i < faces && (!isfinite(vx[i]) || !isfinite(vy[i]))) flags |= 1u;
    if (i < points) {
        const int y = int(i / w), x = int(i - long(y) * w);
        const float ox = loc == 1 ? 0.f : .5f, oy = loc == 2 ? 0.f : .5f;
        const float px = float(x) + ox, py = float(y) + oy;
        const float uu = sample2(vx, n + 1, n, px, py - .5f, flags);
        const float vv = sample2(vy, n, n + 1, px - .5f, py, flags);
        out[i] = sample2(src, w, h, px - dt_over_h * uu - ox, py - dt_over_h * vv - oy, flags);
    }
    if (flags) atomicOr(&ctrl->flags, flags);
}

// uNext/vNext committed to the state, density scaled by the decay.
__global__ void k2_copy(long count, const float* __restrict__ a, float* __restrict__ b) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) b[i] = a[i];
}
__global__ void k2_decay(long count, float decay, const float* __restrict__ next, float* __restrict__ d) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) d[i] = decay * next[i];
}

// Buoyancy on the interior v faces (MacGridFluidSolver2D.cpp:75-86):
// v += (dt buoyancy) (.5 (d_below^1/4 + d_above^1/4)).
__global__ void k2_buoyancy(int n, float dt_buoyancy, const float* __restrict__ d, float* __restrict__ v) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * (n - 1)) return;
    const int y = int(i / n) + 1, x = int(i - long(y - 1) * n);
    const float smoke = .5f * (powf_quarter(d[x + size_t(n) * (y - 1)]) + powf_quarter(d[x + size_t(n) * y]));
    v[x + size_t(n) * y] += dt_buoyancy * smoke;
}

// Emitter (MacGridFluidSolver2D.cpp:46-65) over the precomputed patch of
// cells with q <= 1 and their weights.
__global__ void k2_emit(int count, const int* __restrict__ cells, const float* __restrict__ weights,
                        float strength3, float kick, int kick_on, float* __restrict__ d, float* __restrict__ v) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int i = cells[k];
    const float wgt = weights[k];
    const float s = strength3 * wgt;
    const float add = s < 1.f ? s : 1.f;  // std::min(1.f, s)
    d[i] = d[i] < add ? add : d[i];       // std::max(d, add)
    if (kick_on) {
        const float kv = kick * wgt;
        v[i] = v[i] < kv ? kv : v[i];
    }
}

// ---- projection (CpuPressureSolver2D.cpp:8-82) ----

__device__ __forceinline__ float divergence2(int n, float h, const float* __restrict__ u, const float* __restrict__ v,
                                             int x, int y) {
    return (u[x + 1 + size_t(n + 1) * y] - u[x + size_t(n + 1) * y] + v[x + size_t(n) * (y + 1)] -
            v[x + size_t(n) * y]) /
           h;
}

// rhs = -scale div (the divergence before the solve, its max |.| and the
// finiteness checks of MacGridOperators2D.cpp:7-11 and the RHS overflow check).
__global__ void k2_rhs(int n, float h, float neg_scale, const float* __restrict__ u, const float* __restrict__ v,
                       float* __restrict__ rhs, Mac2DControl* ctrl) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * n) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    const float div = divergence2(n, h, u, v, x, y);
    unsigned int flags = 0u;
    if (!isfinite(div)) flags |= 4u;
    else atomicMax(&ctrl->div_bits, __float_as_uint(fabsf(div)));
    const float value = div * neg_scale;
    if (!isfinite(value)) flags |= 8u;
    rhs[i] = value;
    if (flags) atomicOr(&ctrl->flags, flags);
}

// Sequential FP64 sum in index order, as std::accumulate(begin, end, 0.0):
// one thread, so the rounding of every partial sum is the reference's.
template <class T>
__global__ void k2_serial_sum(long count, const T* __restrict__ a, Mac2DControl* ctrl) {
    double s = 0.0;
    for (long i = 0; i < count; ++i) s += double(a[i]);
    ctrl->sum = s;
}

// The reference's check that every velocity value is finite before a
// projection (flag 32).
__global__ void k2_check_finite(long count, const float* __restrict__ u, const float* __restrict__ v,
                                Mac2DControl* ctrl) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count && (!isfinite(u[i]) || !isfinite(v[i]))) atomicOr(&ctrl->flags, 32u);
}

__global__ void k2_sub_rhs_mean(long count, float mean, float* __restrict__ rhs) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) rhs[i] -= mean;
}

__device__ __forceinline__ int diagonal2(int n, int x, int y) { return (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n); }

// neighbors(x, y): FP64 sum in the order x-1, x+1, y-1, y+1.
__device__ __forceinline__ double neighbours2(int n, const double* __restrict__ p, int x, int y) {
    double s = 0.0;
    const size_t i = x + size_t(n) * y;
    if (x > 0) s += p[i - 1];
    if (x + 1 < n) s += p[i + 1];
    if (y > 0) s += p[i - n];
    if (y + 1 < n) s += p[i + n];
    return s;
}

// max |rhs + neighbors - diagonal p| (FP64), exact by atomic max on the bits.
__global__ void k2_residual(int n, const float* __restrict__ rhs, const double* __restrict__ p, Mac2DControl* ctrl) {
    __shared__ double s_max[32];
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    double r = 0.0;
    if (i < long(n) * n) {
        const int y = int(i / n), x = int(i - long(y) * n);
        r = fabs(double(rhs[i]) + neighbours2(n, p, x, y) - double(diagonal2(n, x, y)) * p[i]);
    }
    const double br = block_max(r, s_max);
    if (threadIdx.x == 0) atomic_max_nonneg(&ctrl->res_bits, br);
}

// One parity of the red-black sweep: the cells with (x + y + parity) even.
__global__ void k2_sor(int n, int parity, float omega, const float* __restrict__ rhs, double* __restrict__ p) {
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;  // k-th cell of this parity in row-major order
    const int half = (n + 1) / 2;
    const int y = int(k / half);
    if (y >= n) return;
    const int x = 2 * int(k - long(y) * half) + ((y + parity) & 1);
    if (x >= n) return;
    const int d = diagonal2(n, x, y);
    if (d == 0) return;
    const size_t i = x + size_t(n) * y;
    p[i] += omega * ((rhs[i] + neighbours2(n, p, x, y)) / d - p[i]);
}

__global__ void k2_sub_pressure_mean(long count, double mean, double* __restrict__ p, Mac2DControl* ctrl) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const double value = p[i] - mean;
    p[i] = value;
    if (!isfinite(value)) atomicOr(&ctrl->flags, 16u);
}

// applyPressureGradient on the interior faces (MacGridOperators2D.cpp:32-41).
__global__ void k2_gradient(int n, double scale, const double* __restrict__ p, float* __restrict__ u,
                            float* __restrict__ v) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * n) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    if (x > 0) {
        float& f = u[x + size_t(n + 1) * y];
        f = float(f - scale * (p[i] - p[i - 1]));
    }
    if (y > 0) {
        float& f = v[x + size_t(n) * y];
        f = float(f - scale * (p[i] - p[i - n]));
    }
}

// maxDivergence (MacGridOperators2D.cpp:26-30) into div_bits; flag 4 if a
// divergence is not finite.
__global__ void k2_max_div(int n, float h, const float* __restrict__ u, const float* __restrict__ v,
                           Mac2DControl* ctrl) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * n) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    const float div = divergence2(n, h, u, v, x, y);
    if (!isfinite(div)) atomicOr(&ctrl->flags, 4u);
    else atomicMax(&ctrl->div_bits, __float_as_uint(fabsf(div)));
}

// Reflection: hat = 2 state - advected, with the wall faces zero.
__global__ void k2_hat(long count, const float* __restrict__ s, const float* __restrict__ next, float* __restrict__ hat) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) hat[i] = 2.f * s[i] - next[i];
}

// diagnostics(): sequential FP64 sum of u^2 then v^2 and max |value|.
__global__ void k2_energy(long count_u, const float* __restrict__ u, long count_v, const float* __restrict__ v,
                          Mac2DControl* ctrl) {
    double s = 0.0;
    float m = 0.f;
    for (long i = 0; i < count_u; ++i) {
        s += double(u[i]) * u[i];
        const float a = fabsf(u[i]);
        m = m < a ? a : m;
    }
    for (long i = 0; i < count_v; ++i) {
        s += double(v[i]) * v[i];
        const float a = fabsf(v[i]);
        m = m < a ? a : m;
    }
    ctrl->sum = s;
    ctrl->div_bits = __float_as_uint(m);
}

}  // namespace

// ---- host side ----

class Mac2D {
public:
    Mac2D(int n, float box, const vapor_mac2d_params& p) : n_(n) {
        if (n <= 0) fail(VAPOR_INVALID_ARGUMENT, "2D MAC resolution must be positive");
        const size_t nn = size_t(n);
        if (nn > size_t(std::numeric_limits<int>::max()) / (nn + 1))
            fail(VAPOR_LENGTH_ERROR, "2D MAC grid exceeds the supported index range");
        check_box(box);
        box_ = box;
        p_ = p;
        const size_t cells = nn * nn, faces = nn * (nn + 1);
        d_.allocate(cells);
        dn_.allocate(cells);
        rhs_.allocate(cells);
        pr_.allocate(cells);
        for (DevArray<float>* a : {&u_, &v_, &un_, &vn_, &uh_, &vh_}) a->allocate(faces);
        VB_CUDA(cudaMalloc(&ctrl_, sizeof(Mac2DControl)));
        zero_all();
    }
    ~Mac2D() {
        cudaStreamSynchronize(st_.s);
        cudaFree(ctrl_);
    }

    const vapor_mac2d_params& params() const { return p_; }
    void set_params(const vapor_mac2d_params& p) { p_ = p; }
    int n() const { return n_; }
    const vapor_projection_result& last() const { return last_; }
    const vapor_projection_result& midpoint() const { return mid_; }

    // MacGridFluidSolver2D::advance (MacGridFluidSolver2D.cpp:22-44).
    void advance(float dt) {
        const auto& p = p_;
        if (!std::isfinite(p.emitter_kick_multiplier) || p.emitter_kick_multiplier < 0.f)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid emitter kick multiplier");
        if (!std::isfinite(dt) || dt <= 0.f || !std::isfinite(p.source_strength) || p.source_strength < 0.f ||
            !std::isfinite(p.emitter_radius) || p.emitter_radius <= 0.f || p.emitter_radius > 1.f ||
            !std::isfinite(p.emitter_center_x) || p.emitter_center_x < 0.f || p.emitter_center_x > 1.f ||
            !std::isfinite(p.emitter_center_y) || p.emitter_center_y < 0.f || p.emitter_center_y > 1.f ||
            !std::isfinite(p.buoyancy) || !std::isfinite(p.smoke_decay) || p.smoke_decay < 0.f ||
            !std::isfinite(p.sor_omega) || p.sor_omega <= 0.f || p.sor_omega >= 2.f || p.project_iterations < 0)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid 2D simulation time step or parameters");
        walls(u_.p, v_.p);
        mid_ = vapor_projection_result{};
        if (p.reflection) {
            const float half = .5f * dt;
            advect_density(half);
            advect_velocity(u_.p, v_.p, half);  // un_, vn_ keep the advected, pre-force velocity
            add_buoyancy(half);
            emit();
            mid_ = project(half);
            const long faces = long(n_) * (n_ + 1);
            k2_hat<<<blocks2(faces), kThreads2, 0, st_.s>>>(faces, u_.p, un_.p, uh_.p);
            k2_hat<<<blocks2(faces), kThreads2, 0, st_.s>>>(faces, v_.p, vn_.p, vh_.p);
            walls(uh_.p, vh_.p);
            advect_density(half);
            advect_velocity(uh_.p, vh_.p, half);  // the hats trace through the projected midpoint
            last_ = project(half);
            return;
        }
        advect_velocity(u_.p, v_.p, dt);
        add_buoyancy(dt);
        emit();
        last_ = project(dt);
        advect_density(dt);
    }

    void reset() {
        VB_CUDA(cudaStreamSynchronize(st_.s));
        zero_all();
        last_ = vapor_projection_result{};
        mid_ = vapor_projection_result{};
    }

    void set_box(float box) {
        check_box(box);
        const float previous = box_;
        box_ = box;
        if (box != previous) reset();
    }

    void upload(const float* d, const float* u, const float* v) {
        VB_CUDA(cudaStreamSynchronize(st_.s));
        if (d) VB_CUDA(cudaMemcpy(d_.p, d, d_.bytes(), cudaMemcpyHostToDevice));
        if (u) VB_CUDA(cudaMemcpy(u_.p, u, u_.bytes(), cudaMemcpyHostToDevice));
        if (v) VB_CUDA(cudaMemcpy(v_.p, v, v_.bytes(), cudaMemcpyHostToDevice));
    }
    void download(float* d, float* u, float* v) {
        VB_CUDA(cudaStreamSynchronize(st_.s));
        if (d) VB_CUDA(cudaMemcpy(d, d_.p, d_.bytes(), cudaMemcpyDeviceToHost));
        if (u) VB_CUDA(cudaMemcpy(u, u_.p, u_.bytes(), cudaMemcpyDeviceToHost));
        if (v) VB_CUDA(cudaMemcpy(v, v_.p, v_.bytes(), cudaMemcpyDeviceToHost));
    }

    // diagnostics() (MacGridFluidSolver2D.cpp:142-153).
    vapor_fluid_diagnostics diagnostics() {
        const long faces = long(n_) * (n_ + 1);
        reset_ctrl();
        k2_energy<<<1, 1, 0, st_.s>>>(faces, u_.p, faces, v_.p, ctrl_);
        const Mac2DControl c = read_ctrl();
        vapor_fluid_diagnostics out{};
        const float h = cell();
        out.kinetic_energy = float(.5 * double(h) * double(h) * c.sum);
        out.max_velocity = uint_as_float(c.div_bits);
        out.max_divergence = max_divergence();
        return out;
    }

private:
    static float uint_as_float(unsigned int b) {
        float f;
        std::memcpy(&f, &b, sizeof f);
        return f;
    }
    static double bits_as_double(unsigned long long b) {
        double f;
        std::memcpy(&f, &b, sizeof f);
        return f;
    }
    // MacGridDomain2D::setBoxSize's checks (MacGridDomain2D.cpp:15-20).
    void check_box(float size) const {
        if (!std::isfinite(size) || size <= 0.f || size / float(n_) <= 0.f || !std::isfinite(1.f / (size / float(n_))))
            fail(VAPOR_INVALID_ARGUMENT, "2D MAC requires finite positive size and spacing");
    }
    float cell() const { return box_ / float(n_); }

    void zero_all() {
        for (DevArray<float>* a : {&d_, &dn_, &rhs_, &u_, &v_, &un_, &vn_, &uh_, &vh_}) a->zero(st_.s);
        pr_.zero(st_.s);
        VB_CUDA(cudaStreamSynchronize(st_.s));
    }
    void reset_ctrl() { VB_CUDA(cudaMemsetAsync(ctrl_, 0, sizeof(Mac2DControl), st_.s)); }
    Mac2DControl read_ctrl() {
        Mac2DControl c;
        VB_CUDA(cudaMemcpyAsync(&c, ctrl_, sizeof c, cudaMemcpyDeviceToHost, st_.s));
        VB_CUDA(cudaStreamSynchronize(st_.s));
        return c;
    }
    void walls(float* u, float* v) { k2_walls<<<blocks2(n_), kThreads2, 0, st_.s>>>(n_, u, v); }

    // One SemiLagrangian2D::advect call; reports the reference's errors.
    void advect(int loc, const float* src, float* out, float dt) {
        if (!std::isfinite(dt) || dt < 0.f)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid 2D advection timestep, extent, or overlapping output");
        const int w = n_ + (loc == 1), h = n_ + (loc == 2);
        const long threads = std::max(long(w) * h, long(n_) * (n_ + 1));
        reset_ctrl();
        k2_advect<<<blocks2(threads), kThreads2, 0, st_.s>>>(n_, loc, dt / cell(), src, u_.p, v_.p, out, ctrl_);
        const Mac2DControl c = read_ctrl();
        if (c.flags & 1u) fail(VAPOR_NON_FINITE, "Non-finite 2D advection input");
        if (c.flags & 2u) fail(VAPOR_NON_FINITE, "Non-finite 2D backtrace");
    }
    // advectVelocity (MacGridFluidSolver2D.cpp:67-73): both components trace
    // through the state's velocity; committed after both passes.
    void advect_velocity(const float* us, const float* vs, float dt) {
        advect(1, us, un_.p, dt);
        advect(2, vs, vn_.p, dt);
        const long faces = long(n_) * (n_ + 1);
        k2_copy<<<blocks2(faces), kThreads2, 0, st_.s>>>(faces, un_.p, u_.p);
        k2_copy<<<blocks2(faces), kThreads2, 0, st_.s>>>(faces, vn_.p, v_.p);
    }
    // advectDensity (MacGridFluidSolver2D.cpp:97-102).
    void advect_density(float dt) {
        advect(0, d_.p, dn_.p, dt);
        const float decay = std::exp(-dt * p_.smoke_decay);
        const long cells = long(n_) * n_;
        k2_decay<<<blocks2(cells), kThreads2, 0, st_.s>>>(cells, decay, dn_.p, d_.p);
    }
    void add_buoyancy(float dt) {
        if (n_ < 2) return;
        const long faces = long(n_) * (n_ - 1);
        k2_buoyancy<<<blocks2(faces), kThreads2, 0, st_.s>>>(n_, dt * p_.buoyancy, d_.p, v_.p);
    }
    // emit(): the cells inside the emitter and their weights depend only on
    // n and the emitter's geometry, so they are computed on the host (with the
    // C library's expf, as the reference evaluates them) and kept.
    void emit() {
        const auto& p = p_;
        if (p.source_strength <= 0.f) return;
        if (!patch_valid_ || patch_r_ != p.emitter_radius || patch_cx_ != p.emitter_center_x ||
            patch_cy_ != p.emitter_center_y) {
            std::vector<uint32_t> cells;
            std::vector<float> weights;
            const float r2 = p.emitter_radius * p.emitter_radius;
            for (int y = 0; y < n_; ++y)
                for (int x = 0; x < n_; ++x) {
                    const float dx = (float(x) + .5f) / float(n_) - p.emitter_center_x;
                    const float dy = (float(y) + .5f) / float(n_) - p.emitter_center_y;
                    const float q = (dx * dx + dy * dy) / r2;
                    if (q > 1.f) continue;
                    cells.push_back(uint32_t(x + size_t(n_) * y));
                    weights.push_back(std::exp(-3.5f * q));
                }
            VB_CUDA(cudaStreamSynchronize(st_.s));
            patch_count_ = int(cells.size());
            if (patch_count_ > 0) {
                patch_cells_.allocate(cells.size());
                patch_weights_.allocate(weights.size());
                VB_CUDA(cudaMemcpy(patch_cells_.p, cells.data(), cells.size() * 4, cudaMemcpyHostToDevice));
                VB_CUDA(cudaMemcpy(patch_weights_.p, weights.data(), weights.size() * 4, cudaMemcpyHostToDevice));
            }
            patch_valid_ = true;
            patch_r_ = p.emitter_radius;
            patch_cx_ = p.emitter_center_x;
            patch_cy_ = p.emitter_center_y;
        }
        if (patch_count_ == 0) return;
        k2_emit<<<blocks2(patch_count_), kThreads2, 0, st_.s>>>(
            patch_count_, reinterpret_cast<const int*>(patch_cells_.p), patch_weights_.p, p.source_strength * 3.f,
            p.emitter_kick_multiplier * (.6f + p.source_strength), p.emitter_kick_multiplier > 0.f ? 1 : 0, d_.p,
            v_.p);
    }

    float max_divergence() {
        const long cells = long(n_) * n_;
        reset_ctrl();
        k2_max_div<<<blocks2(cells), kThreads2, 0, st_.s>>>(n_, cell(), u_.p, v_.p, ctrl_);
        const Mac2DControl c = read_ctrl();
        if (c.flags & 4u) fail(VAPOR_NON_FINITE, "Non-finite 2D MAC divergence");
        return uint_as_float(c.div_bits);
    }

    double residual() {
        const long cells = long(n_) * n_;
        VB_CUDA(cudaMemsetAsync(&ctrl_->res_bits, 0, sizeof(unsigned long long), st_.s));
        k2_residual<<<blocks2(cells), kThreads2, 0, st_.s>>>(n_, rhs_.p, pr_.p, ctrl_);
        return bits_as_double(read_ctrl().res_bits);
    }

    // CpuPressureSolver2D::project (CpuPressureSolver2D.cpp:8-82) with the
    // solver's options (MacGridFluidSolver2D.cpp:88-95): iteration budget
    // project_iterations, residual every 8 iterations, tolerances 1e-6
    // absolute / 1e-5 relative, stop at tolerance.
    vapor_projection_result project(float dt) {
        const int max_iterations = p_.project_iterations, interval = 8;
        const double abs_tol = 1e-6, rel_tol = 1e-5;
        const float h = cell();
        const float scale = h * h / dt;
        if (!std::isfinite(dt) || dt <= 0.f || !std::isfinite(scale) || scale <= 0.f || !std::isfinite(p_.sor_omega) ||
            p_.sor_omega <= 0.f || p_.sor_omega >= 2.f || max_iterations < 0)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid 2D SOR projection options");
        const long cells = long(n_) * n_, faces = long(n_) * (n_ + 1);
        reset_ctrl();
        k2_check_finite<<<blocks2(faces), kThreads2, 0, st_.s>>>(faces, u_.p, v_.p, ctrl_);
        pr_.zero(st_.s);
        walls(u_.p, v_.p);
        k2_rhs<<<blocks2(cells), kThreads2, 0, st_.s>>>(n_, h, -scale, u_.p, v_.p, rhs_.p, ctrl_);
        k2_serial_sum<float><<<1, 1, 0, st_.s>>>(cells, rhs_.p, ctrl_);
        Mac2DControl c = read_ctrl();
        if (c.flags & 32u) fail(VAPOR_NON_FINITE, "Non-finite 2D velocity");
        if (c.flags & 4u) fail(VAPOR_NON_FINITE, "Non-finite 2D MAC divergence");
        if (c.flags & 8u) fail(VAPOR_INVALID_ARGUMENT, "2D pressure RHS overflow");
        vapor_projection_result r{};
        r.divergence_before = uint_as_float(c.div_bits);
        r.removed_rhs_mean = c.sum / double(cells);
        k2_sub_rhs_mean<<<blocks2(cells), kThreads2, 0, st_.s>>>(cells, float(r.removed_rhs_mean), rhs_.p);
        auto& ls = r.linear_solve;
        ls.initial_residual = ls.final_residual = residual();
        const double target = std::max(abs_tol, rel_tol * ls.initial_residual);
        ls.converged = ls.final_residual <= target;
        const int half = (n_ + 1) / 2;
        const long per_parity = long(half) * n_;
        for (int it = 0; it < max_iterations && !ls.converged; ++it) {
            for (int parity = 0; parity < 2; ++parity)
                k2_sor<<<blocks2(per_parity), kThreads2, 0, st_.s>>>(n_, parity, p_.sor_omega, rhs_.p, pr_.p);
            ls.iterations = it + 1;
            if (ls.iterations % interval == 0 || ls.iterations == max_iterations) {
                ls.final_residual = residual();
                ls.converged = ls.final_residual <= target;
            }
        }
        reset_ctrl();
        k2_serial_sum<double><<<1, 1, 0, st_.s>>>(cells, pr_.p, ctrl_);
        const double mean = read_ctrl().sum / double(cells);
        k2_sub_pressure_mean<<<blocks2(cells), kThreads2, 0, st_.s>>>(cells, mean, pr_.p, ctrl_);
        if (read_ctrl().flags & 16u) fail(VAPOR_RUNTIME_ERROR, "2D SOR produced non-finite pressure");
        ls.final_residual = residual();
        ls.converged = ls.final_residual <= target;
        r.residual_available = 1;
        k2_gradient<<<blocks2(cells), kThreads2, 0, st_.s>>>(n_, double(dt) / double(h), pr_.p, u_.p, v_.p);
        walls(u_.p, v_.p);
        r.divergence_after = max_divergence();
        return r;
    }

    int n_;
    float box_ = 1.f;
    vapor_mac2d_params p_{};
    Stream st_;
    DevArray<float> d_, dn_, rhs_, u_, v_, un_, vn_, uh_, vh_;
    DevArray<double> pr_;
    DevArray<uint32_t> patch_cells_;
    DevArray<float> patch_weights_;
    int patch_count_ = 0;
    bool patch_valid_ = false;
    float patch_r_ = 0.f, patch_cx_ = 0.f, patch_cy_ = 0.f;
    Mac2DControl* ctrl_ = nullptr;
    vapor_projection_result last_{}, mid_{};
};

}  // namespace vb

// ---- C ABI ----

struct vapor_mac2d {
    vb::Mac2D sim;
    vapor_mac2d(int n, float box, const vapor_mac2d_params& p) : sim(n, box, p) {}
};

#define VB_API2 extern "C" __attribute__((visibility("default")))

namespace {
void require2(bool ok, const char* message) {
    if (!ok) vb::fail(VAPOR_INVALID_ARGUMENT, message);
}
vapor_mac2d_params struct_defaults() {
    vapor_mac2d_params p{};
    p.reflection = 0;
    p.source_strength = 4.f;
    p.emitter_kick_multiplier = 1.f;
    p.emitter_radius = .08f;
    p.emitter_center_x = .5f;
    p.emitter_center_y = .2f;
    p.buoyancy = 3.f;
    p.smoke_decay = .08f;
    p.sor_omega = 1.9f;
    p.project_iterations = 600;
    return p;
}
}  // namespace

VB_API2 vapor_status vapor_mac2d_default_params(vapor_mac2d_params* out) {
    return vb::guard([&] {
        require2(out != nullptr, "null output");
        *out = struct_defaults();
    });
}
VB_API2 vapor_status vapor_mac2d_plume_params(vapor_mac2d_params* out) {
    return vb::guard([&] {
        require2(out != nullptr, "null output");
        vapor_mac2d_params p = struct_defaults();
        p.emitter_radius = .04f;
        p.source_strength = 1.f;
        p.buoyancy = .8f;
        p.smoke_decay = .3007525f;
        p.project_iterations = 120;
        *out = p;
    });
}
VB_API2 vapor_status vapor_mac2d_create(int32_t n, float box, const vapor_mac2d_params* params, vapor_mac2d** out) {
    return vb::guard([&] {
        require2(out != nullptr, "null output");
        *out = nullptr;
        const vapor_mac2d_params p = params ? *params : struct_defaults();
        *out = new vapor_mac2d(n, box, p);
    });
}
VB_API2 vapor_status vapor_mac2d_destroy(vapor_mac2d* sim) {
    return vb::guard([&] { delete sim; });
}
VB_API2 vapor_status vapor_mac2d_get_params(const vapor_mac2d* sim, vapor_mac2d_params* out) {
    return vb::guard([&] {
        require2(sim && out, "null handle or output");
        *out = sim->sim.params();
    });
}
VB_API2 vapor_status vapor_mac2d_set_params(vapor_mac2d* sim, const vapor_mac2d_params* params) {
    return vb::guard([&] {
        require2(sim && params, "null handle or parameters");
        sim->sim.set_params(*params);
    });
}
VB_API2 vapor_status vapor_mac2d_advance(vapor_mac2d* sim, float dt) {
    return vb::guard([&] {
        require2(sim != nullptr, "null handle");
        sim->sim.advance(dt);
    });
}
VB_API2 vapor_status vapor_mac2d_reset(vapor_mac2d* sim) {
    return vb::guard([&] {
        require2(sim != nullptr, "null handle");
        sim->sim.reset();
    });
}
VB_API2 vapor_status vapor_mac2d_set_box(vapor_mac2d* sim, float box) {
    return vb::guard([&] {
        require2(sim != nullptr, "null handle");
        sim->sim.set_box(box);
    });
}
VB_API2 vapor_status vapor_mac2d_upload(vapor_mac2d* sim, const float* density, const float* u, const float* v) {
    return vb::guard([&] {
        require2(sim != nullptr, "null handle");
        sim->sim.upload(density, u, v);
    });
}
VB_API2 vapor_status vapor_mac2d_download(vapor_mac2d* sim, float* density, float* u, float* v) {
    return vb::guard([&] {
        require2(sim != nullptr, "null handle");
        sim->sim.download(density, u, v);
    });
}
VB_API2 vapor_status vapor_mac2d_last_projection(vapor_mac2d* sim, vapor_projection_result* out) {
    return vb::guard([&] {
        require2(sim && out, "null handle or output");
        *out = sim->sim.last();
    });
}
VB_API2 vapor_status vapor_mac2d_midpoint_projection(vapor_mac2d* sim, vapor_projection_result* out) {
    return vb::guard([&] {
        require2(sim && out, "null handle or output");
        *out = sim->sim.midpoint();
    });
}
VB_API2 vapor_status vapor_mac2d_diagnostics(vapor_mac2d* sim, vapor_fluid_diagnostics* out) {
    return vb::guard([&] {
        require2(sim && out, "null handle or output");
        *out = sim->sim.diagnostics();
    });
}
