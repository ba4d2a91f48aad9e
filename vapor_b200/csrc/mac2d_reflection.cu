// The reference's compatibility 2D solver on the device:
// ReflectionMacFluidSolver2D (src/solvers/mac2d/ReflectionMacFluidSolver2D.hpp),
// the historical plume on the unit box with a midpoint reflection every step.
//
// Parity with the reference's CPU arithmetic (FP32 throughout, FP64 only in
// the kinetic energy):
//   - samplers, traces, the FP32 red-black SOR (the two parities have no
//     internal neighbours), buoyancy and the gradient run one thread per cell
//     or face with the reference's expressions in its order; a face's two
//     buoyancy contributions are added in the reference's loop order;
//   - the MacCormack limiter updates the smoke in place in raster order, so a
//     cell's 3x3 bounds see the new values of the four cells before it
//     ((x-1, y-1), (x, y-1), (x+1, y-1), (x-1, y)) and the old values of the
//     rest. Cell (x, y) therefore runs at wavefront step x + 2y (every earlier
//     neighbour has a smaller step, every later one a larger), in one block;
//   - the emitter, whose random stirring draws the reference's LCG stream in
//     patch order, runs on one device thread over the patch the host lists
//     with the C library's expf, as the reference evaluates its weights;
//   - the per-frame dissipation exp(-k / 60) and its half-step power are
//     host values; d^(1/4) is the C library's powf(d, .25f) bit for bit
//     (powf_quarter.cuh).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.hpp"
#include "powf_quarter.cuh"

namespace vb {
namespace {

constexpr int kT = 256;
int blocks_r(long count) { return int(std::max<long>(1, (count + kT - 1) / kT)); }

__device__ __forceinline__ float clampf_std(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }
__device__ __forceinline__ float mix_r(float a, float b, float t) { return a + (b - a) * t; }

// sampleCell / sampleVxField / sampleVyField (ReflectionMacFluidSolver2D.hpp:107-137).
__device__ __forceinline__ float sample_cell(const float* __restrict__ f, int n, float h, float px, float py) {
    const float gx = clampf_std(px / h - 0.5f, 0.f, float(n - 1));
    const float gy = clampf_std(py / h - 0.5f, 0.f, float(n - 1));
    const int x0 = int(gx), y0 = int(gy);
    const int x1 = min(x0 + 1, n - 1), y1 = min(y0 + 1, n - 1);
    const float tx = gx - float(x0), ty = gy - float(y0);
    return mix_r(mix_r(f[x0 + n * y0], f[x1 + n * y0], tx), mix_r(f[x0 + n * y1], f[x1 + n * y1], tx), ty);
}
__device__ __forceinline__ float sample_vx(const float* __restrict__ f, int n, float h, float px, float py) {
    const float gx = clampf_std(px / h, 0.f, float(n));
    const float gy = clampf_std(py / h - 0.5f, 0.f, float(n - 1));
    const int x0 = min(int(gx), n - 1), y0 = int(gy);
    const int x1 = x0 + 1, y1 = min(y0 + 1, n - 1);
    const float tx = gx - float(x0), ty = gy - float(y0);
    const int w = n + 1;
    return mix_r(mix_r(f[x0 + w * y0], f[x1 + w * y0], tx), mix_r(f[x0 + w * y1], f[x1 + w * y1], tx), ty);
}
__device__ __forceinline__ float sample_vy(const float* __restrict__ f, int n, float h, float px, float py) {
    const float gx = clampf_std(px / h - 0.5f, 0.f, float(n - 1));
    const float gy = clampf_std(py / h, 0.f, float(n));
    const int x0 = int(gx), y0 = min(int(gy), n - 1);
    const int x1 = min(x0 + 1, n - 1), y1 = y0 + 1;
    const float tx = gx - float(x0), ty = gy - float(y0);
    return mix_r(mix_r(f[x0 + n * y0], f[x1 + n * y0], tx), mix_r(f[x0 + n * y1], f[x1 + n * y1], tx), ty);
}

// Semi-Lagrangian smoke (dir -1) or the MacCormack back trace (dir +1) of
// advectScalar (ReflectionMacFluidSolver2D.hpp:146-176): q = p -/+ v(p) dt,
// clamped half a cell inside the box, sampled from `src`.
__global__ void kr_trace_cell(int n, float h, float dt, float dir, const float* __restrict__ vx,
                              const float* __restrict__ vy, const float* __restrict__ src, float* __restrict__ out) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * n) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    const float px = (float(x) + .5f) * h, py = (float(y) + .5f) * h;
    const float vxv = sample_vx(vx, n, h, px, py), vyv = sample_vy(vy, n, h, px, py);
    float qx = dir < 0.f ? px - vxv * dt : px + vxv * dt;
    float qy = dir < 0.f ? py - vyv * dt : py + vyv * dt;
    const float pad = 0.5f * h;
    qx = clampf_std(qx, pad, 1.0f - pad);
    qy = clampf_std(qy, pad, 1.0f - pad);
    out[i] = sample_cell(src, n, h, qx, qy);
}

// The MacCormack correction and in-place limiter
// (ReflectionMacFluidSolver2D.hpp:178-194) as a wavefront: one block, step t
// holds the cells with x + 2 y == t.
__global__ void kr_limit(int n, float* __restrict__ field, const float* __restrict__ fwd,
                         const float* __restrict__ back) {
    const int steps = 3 * n - 2;
    for (int t = 0; t < steps; ++t) {
        const int y_lo = max(0, (t - (n - 1) + 1) / 2), y_hi = min(n - 1, t / 2);
        for (int y = y_lo + int(threadIdx.x); y <= y_hi; y += blockDim.x) {
            const int x = t - 2 * y;
            const int i = x + n * y;
            const float corrected = fwd[i] + 0.5f * (field[i] - back[i]);
            float lo = fwd[i] < field[i] ? fwd[i] : field[i];  // std::min(field, fwd)
            float hi = field[i] < fwd[i] ? fwd[i] : field[i];  // std::max(field, fwd)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int a = x + dx, b = y + dy;
                    if (a < 0 || b < 0 || a >= n || b >= n) continue;
                    const float fw = fwd[a + n * b], fd = field[a + n * b];
                    // std::min / std::max over {bound, fwd, field}: the first extreme wins
                    if (fw < lo) lo = fw;
                    if (fd < lo) lo = fd;
                    if (hi < fw) hi = fw;
                    if (hi < fd) hi = fd;
                }
            field[i] = clampf_std(corrected, lo, hi);
        }
        __syncthreads();
    }
}

// advectVx / advectVy (ReflectionMacFluidSolver2D.hpp:196-220) with the flow
// and source of the caller (the stage-4 passes trace through the midpoint
// velocity and sample the reflected one, :394-419).
__global__ void kr_advect_vx(int n, float h, float dt, const float* __restrict__ fx, const float* __restrict__ fy,
                             const float* __restrict__ src, float* __restrict__ out) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const int w = n + 1;
    if (i >= long(w) * n) return;
    const int y = int(i / w), x = int(i - long(y) * w);
    const float px = float(x) * h, py = (float(y) + .5f) * h;
    float qx = px - sample_vx(fx, n, h, px, py) * dt, qy = py - sample_vy(fy, n, h, px, py) * dt;
    qx = clampf_std(qx, 0.f, 1.0f);
    qy = clampf_std(qy, 0.5f * h, 1.0f - 0.5f * h);
    out[i] = sample_vx(src, n, h, qx, qy);
}
__global__ void kr_advect_vy(int n, float h, float dt, const float* __restrict__ fx, const float* __restrict__ fy,
                             const float* __restrict__ src, float* __restrict__ out) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * (n + 1)) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    const float px = (float(x) + .5f) * h, py = float(y) * h;
    float qx = px - sample_vx(fx, n, h, px, py) * dt, qy = py - sample_vy(fy, n, h, px, py) * dt;
    qx = clampf_std(qx, 0.5f * h, 1.0f - 0.5f * h);
    qy = clampf_std(qy, 0.f, 1.0f);
    out[i] = sample_vy(src, n, h, qx, qy);
}

// Closed free-slip walls: zero normal face velocity (:222-232).
__global__ void kr_walls(int n, float* __restrict__ vx, float* __restrict__ vy) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    vx[size_t(n + 1) * i] = 0.f;
    vx[size_t(n + 1) * i + n] = 0.f;
    vy[i] = 0.f;
    vy[size_t(n) * n + i] = 0.f;
}

// project(dt, iterations) (ReflectionMacFluidSolver2D.hpp:235-285).
__global__ void kr_divergence(int n, float h_inv, const float* __restrict__ vx, const float* __restrict__ vy,
                              float* __restrict__ div) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * n) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    div[i] = (vx[x + 1 + size_t(n + 1) * y] - vx[x + size_t(n + 1) * y] + vy[x + size_t(n) * (y + 1)] -
              vy[x + size_t(n) * y]) *
             h_inv;
}

// One parity of the FP32 SOR: the cells with (x + y) & 1 == parity.
__global__ void kr_sor(int n, int parity, float omega, float h2, float dt, const float* __restrict__ div,
                       float* __restrict__ p) {
    const long k = long(blockIdx.x) * blockDim.x + threadIdx.x;
    const int half = (n + 1) / 2;
    const int y = int(k / half);
    if (y >= n) return;
    const int x = 2 * int(k - long(y) * half) + ((y + parity) & 1);
    if (x >= n) return;
    const int i = x + n * y;
    float sum = 0.f;
    int terms = 0;
    if (x > 0) { ++terms; sum += p[i - 1]; }
    if (x + 1 < n) { ++terms; sum += p[i + 1]; }
    if (y > 0) { ++terms; sum += p[i - n]; }
    if (y + 1 < n) { ++terms; sum += p[i + n]; }
    p[i] = (1.f - omega) * p[i] + omega * (sum - div[i] * h2 / dt) / float(max(terms, 1));
}

__global__ void kr_gradient(int n, float dt, float h_inv, const float* __restrict__ p, float* __restrict__ vx,
                            float* __restrict__ vy) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * n) return;
    const int y = int(i / n), x = int(i - long(y) * n);
    if (x > 0) {
        float& f = vx[x + size_t(n + 1) * y];
        f -= dt * (p[i] - p[i - 1]) * h_inv;
    }
    if (y > 0) {
        float& f = vy[x + size_t(n) * y];
        f -= dt * (p[i] - p[i - n]) * h_inv;
    }
}

// Buoyancy (:339-344): cell (x, y) adds split * f to its lower and upper v
// face, f = buoyancy d^1/4 dt/2. Face (x, j) takes the contribution of cell
// j - 1 first, then that of cell j, as the reference's loop does.
__global__ void kr_buoyancy(int n, float buoyancy, float half_dt, float split, const float* __restrict__ smoke,
                            float* __restrict__ vy) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= long(n) * (n + 1)) return;
    const int j = int(i / n), x = int(i - long(j) * n);
    float v = vy[i];
    if (j > 0) v += split * (buoyancy * powf_quarter(smoke[x + size_t(n) * (j - 1)]) * half_dt);
    if (j < n) v += split * (buoyancy * powf_quarter(smoke[x + size_t(n) * j]) * half_dt);
    vy[i] = v;
}

// emit(strength) (:287-307) over the host's patch list, on one thread: the
// stirring draws the LCG stream cell by cell in the reference's order.
__global__ void kr_emit(int count, const int2* __restrict__ cells, const float* __restrict__ weights, int n,
                        float strength3, float kick, int kick_on, float stir, unsigned int* state,
                        float* __restrict__ smoke, float* __restrict__ vx, float* __restrict__ vy) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    unsigned int r = *state;
    auto unit = [&]() {
        r = r * 1664525u + 1013904223u;
        return float(r >> 8) * (1.0f / 16777216.0f);
    };
    for (int k = 0; k < count; ++k) {
        const int x = cells[k].x, y = cells[k].y;
        const float w = weights[k];
        const int i = x + n * y;
        const float s = strength3 * w;
        const float add = s < 1.0f ? s : 1.0f;
        smoke[i] = smoke[i] < add ? add : smoke[i];
        if (kick_on) {
            const float kv = kick * w;
            vy[i] = vy[i] < kv ? kv : vy[i];
        }
        if (stir > 0.f) {
            vx[x + (n + 1) * y] += (unit() - 0.5f) * stir * w;
            vx[x + 1 + (n + 1) * y] += (unit() - 0.5f) * stir * w;
        }
    }
    *state = r;
}

__global__ void kr_scale(long count, float factor, float* __restrict__ a) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) a[i] *= factor;
}
__global__ void kr_copy(long count, const float* __restrict__ a, float* __restrict__ b) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) b[i] = a[i];
}
__global__ void kr_hat(long count, const float* __restrict__ mid, const float* __restrict__ tilde,
                       float* __restrict__ hat) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) hat[i] = 2.f * mid[i] - tilde[i];
}

// diagnostics() (:48-56): sequential FP64 energy and max |velocity|, max |div|.
__global__ void kr_diagnostics(int n, float h, const float* __restrict__ vx, const float* __restrict__ vy,
                               double* __restrict__ energy, float* __restrict__ maxima) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const long faces = long(n) * (n + 1);
    double e = 0.0;
    float mv = 0.f, md = 0.f;
    for (const float* f : {vx, vy})
        for (long i = 0; i < faces; ++i) {
            e += double(f[i]) * f[i];
            const float a = fabsf(f[i]);
            mv = mv < a ? a : mv;
        }
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const float d = fabsf((vx[x + 1 + (n + 1) * y] - vx[x + (n + 1) * y] + vy[x + n * (y + 1)] -
                                   vy[x + n * y]) /
                                  h);
            md = md < d ? d : md;
        }
    *energy = e;
    maxima[0] = mv;
    maxima[1] = md;
}

}  // namespace

// ---- host side ----

class Mac2DReflection {
public:
    Mac2DReflection(int n, const vapor_mac2d_refl_params& p) : n_(n), p_(p) {
        if (n < 2 || n > 512) fail(VAPOR_INVALID_ARGUMENT, "2D reflection resolution must be 2..512");
        const size_t cells = size_t(n) * n, faces = size_t(n) * (n + 1);
        for (DevArray<float>* a : {&smoke_, &fwd_, &back_, &pressure_, &div_}) a->allocate(cells);
        for (DevArray<float>* a : {&vx_, &vy_, &vxt_, &vyt_, &vxm_, &vym_, &vxh_, &vyh_}) a->allocate(faces);
        state_.allocate(1);
        energy_.allocate(1);
        maxima_.allocate(2);
        reset();
    }
    ~Mac2DReflection() { cudaStreamSynchronize(st_.s); }

    const vapor_mac2d_refl_params& params() const { return p_; }
    void set_params(const vapor_mac2d_refl_params& p) {
        p_ = p;
        patch_valid_ = false;
    }

    void reset() {
        VB_CUDA(cudaStreamSynchronize(st_.s));
        for (DevArray<float>* a : {&smoke_, &fwd_, &back_, &pressure_, &div_, &vx_, &vy_, &vxt_, &vyt_, &vxm_, &vym_,
                                   &vxh_, &vyh_})
            a->zero(st_.s);
        const uint32_t seed = p_.random_seed;
        VB_CUDA(cudaMemcpyAsync(state_.p, &seed, 4, cudaMemcpyHostToDevice, st_.s));
        VB_CUDA(cudaStreamSynchronize(st_.s));
    }

    // advance(dt) (ReflectionMacFluidSolver2D.hpp:32-45).
    void advance(float dt) {
        const auto& p = p_;
        if (!std::isfinite(p.emitter_kick_multiplier) || p.emitter_kick_multiplier < 0.f)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid emitter kick multiplier");
        if (!std::isfinite(dt) || dt <= 0.f || !std::isfinite(p.buoyancy) || !std::isfinite(p.smoke_decay) ||
            p.smoke_decay < 0.f || !std::isfinite(p.source_strength) || p.source_strength < 0.f ||
            !std::isfinite(p.emitter_radius) || p.emitter_radius <= 0.f || p.emitter_radius > 1.f ||
            !std::isfinite(p.stir_strength) || p.stir_strength < 0.f || !std::isfinite(p.sor_omega) ||
            p.sor_omega <= 0.f || p.sor_omega >= 2.f || p.project_iterations < 0)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid 2D reflection step or parameters");
        walls(vx_.p, vy_.p);
        step(dt, p.buoyancy, std::exp(-p.smoke_decay / 60.f), p.source_strength, p.project_iterations);
        VB_CUDA(cudaStreamSynchronize(st_.s));
    }

    void upload(const float* s, const float* u, const float* v) {
        VB_CUDA(cudaStreamSynchronize(st_.s));
        if (s) VB_CUDA(cudaMemcpy(smoke_.p, s, smoke_.bytes(), cudaMemcpyHostToDevice));
        if (u) VB_CUDA(cudaMemcpy(vx_.p, u, vx_.bytes(), cudaMemcpyHostToDevice));
        if (v) VB_CUDA(cudaMemcpy(vy_.p, v, vy_.bytes(), cudaMemcpyHostToDevice));
    }
    void download(float* s, float* u, float* v, float* pr) {
        VB_CUDA(cudaStreamSynchronize(st_.s));
        if (s) VB_CUDA(cudaMemcpy(s, smoke_.p, smoke_.bytes(), cudaMemcpyDeviceToHost));
        if (u) VB_CUDA(cudaMemcpy(u, vx_.p, vx_.bytes(), cudaMemcpyDeviceToHost));
        if (v) VB_CUDA(cudaMemcpy(v, vy_.p, vy_.bytes(), cudaMemcpyDeviceToHost));
        if (pr) VB_CUDA(cudaMemcpy(pr, pressure_.p, pressure_.bytes(), cudaMemcpyDeviceToHost));
    }

    vapor_fluid_diagnostics diagnostics() {
        kr_diagnostics<<<1, 1, 0, st_.s>>>(n_, h(), vx_.p, vy_.p, energy_.p, maxima_.p);
        double e = 0.0;
        float m[2] = {0.f, 0.f};
        VB_CUDA(cudaMemcpyAsync(&e, energy_.p, sizeof e, cudaMemcpyDeviceToHost, st_.s));
        VB_CUDA(cudaMemcpyAsync(m, maxima_.p, sizeof m, cudaMemcpyDeviceToHost, st_.s));
        VB_CUDA(cudaStreamSynchronize(st_.s));
        vapor_fluid_diagnostics out{};
        const float hh = h();
        out.kinetic_energy = float(.5 * e * hh * hh);
        out.max_velocity = m[0];
        out.max_divergence = m[1];
        return out;
    }

private:
    float h() const { return 1.0f / float(n_); }
    long cells() const { return long(n_) * n_; }
    long faces() const { return long(n_) * (n_ + 1); }
    void walls(float* u, float* v) { kr_walls<<<blocks_r(n_), kT, 0, st_.s>>>(n_, u, v); }

    // advectScalar(smoke, dt) through the current velocity.
    void advect_smoke(float dt) {
        kr_trace_cell<<<blocks_r(cells()), kT, 0, st_.s>>>(n_, h(), dt, -1.f, vx_.p, vy_.p, smoke_.p, fwd_.p);
        if (!p_.mac_cormack_smoke) {
            kr_copy<<<blocks_r(cells()), kT, 0, st_.s>>>(cells(), fwd_.p, smoke_.p);
            return;
        }
        kr_trace_cell<<<blocks_r(cells()), kT, 0, st_.s>>>(n_, h(), dt, 1.f, vx_.p, vy_.p, fwd_.p, back_.p);
        kr_limit<<<1, 512, 0, st_.s>>>(n_, smoke_.p, fwd_.p, back_.p);
    }

    // emit(strength, dt): the patch of cells and weights, listed in the
    // reference's loop order with its bounds (:287-300).
    void emit(float strength) {
        if (strength <= 0.f) return;
        const auto& p = p_;
        if (!patch_valid_) {
            std::vector<int2> cells;
            std::vector<float> weights;
            const float r2 = p.emitter_radius * p.emitter_radius, dx = h();
            const int n = n_;
            const int emit_h = std::min(int(p.emitter_center_y * float(n) + p.emitter_radius * float(n) + 2.f), n);
            for (int y = std::max(0, int(p.emitter_center_y * float(n) - p.emitter_radius * float(n) - 1.f));
                 y < emit_h; ++y)
                for (int x = 0; x < n; ++x) {
                    const float px = (float(x) + .5f) * dx, py = (float(y) + .5f) * dx;
                    const float dx2 = (px - p.emitter_center_x) * (px - p.emitter_center_x);
                    const float dy2 = (py - p.emitter_center_y) * (py - p.emitter_center_y);
                    const float q = (dx2 + dy2) / r2;
                    if (q > 1.0f) continue;
                    cells.push_back(make_int2(x, y));
                    weights.push_back(std::exp(-3.5f * q));
                }
            VB_CUDA(cudaStreamSynchronize(st_.s));
            patch_count_ = int(cells.size());
            if (patch_count_ > 0) {
                patch_cells_.allocate(2 * cells.size());
                patch_weights_.allocate(weights.size());
                VB_CUDA(cudaMemcpy(patch_cells_.p, cells.data(), cells.size() * sizeof(int2), cudaMemcpyHostToDevice));
                VB_CUDA(cudaMemcpy(patch_weights_.p, weights.data(), weights.size() * 4, cudaMemcpyHostToDevice));
            }
            patch_valid_ = true;
        }
        if (patch_count_ == 0) return;
        kr_emit<<<1, 1, 0, st_.s>>>(patch_count_, reinterpret_cast<const int2*>(patch_cells_.p), patch_weights_.p, n_,
                                    strength * 3.0f, p.emitter_kick_multiplier * (0.6f + 1.0f * strength),
                                    p.emitter_kick_multiplier > 0.f ? 1 : 0, p.stir_strength, state_.p, smoke_.p,
                                    vx_.p, vy_.p);
    }

    // project(dt, iterations) (:235-285).
    void project(float dt, int iterations) {
        const float h_inv = 1.0f / h(), h2 = h() * h();
        walls(vx_.p, vy_.p);
        kr_divergence<<<blocks_r(cells()), kT, 0, st_.s>>>(n_, h_inv, vx_.p, vy_.p, div_.p);
        pressure_.zero(st_.s);
        const long per_parity = long((n_ + 1) / 2) * n_;
        for (int it = 0; it < iterations; ++it)
            for (int parity = 0; parity < 2; ++parity)
                kr_sor<<<blocks_r(per_parity), kT, 0, st_.s>>>(n_, parity, p_.sor_omega, h2, dt, div_.p, pressure_.p);
        kr_gradient<<<blocks_r(cells()), kT, 0, st_.s>>>(n_, dt, h_inv, pressure_.p, vx_.p, vy_.p);
        walls(vx_.p, vy_.p);
    }

    // step (:309-425).
    void step(float dt, float buoyancy, float dissipation, float strength, int iterations) {
        const float half = 0.5f * dt;
        const int half_iters = std::max(1, iterations / 2);
        const float half_decay = std::pow(dissipation, half * 60.0f);
        // stage 1: smoke half step through u0
        advect_smoke(half);
        kr_scale<<<blocks_r(cells()), kT, 0, st_.s>>>(cells(), half_decay, smoke_.p);
        // stage 2: both components advected from u0, forces, projection
        kr_advect_vx<<<blocks_r(faces()), kT, 0, st_.s>>>(n_, h(), half, vx_.p, vy_.p, vx_.p, vxt_.p);
        kr_advect_vy<<<blocks_r(faces()), kT, 0, st_.s>>>(n_, h(), half, vx_.p, vy_.p, vy_.p, vyt_.p);
        kr_copy<<<blocks_r(faces()), kT, 0, st_.s>>>(faces(), vxt_.p, vx_.p);
        kr_copy<<<blocks_r(faces()), kT, 0, st_.s>>>(faces(), vyt_.p, vy_.p);
        kr_buoyancy<<<blocks_r(faces()), kT, 0, st_.s>>>(n_, buoyancy, half, 0.5f, smoke_.p, vy_.p);
        emit(strength);
        project(half, half_iters);
        // stage 3: reflection about the projected midpoint
        kr_copy<<<blocks_r(faces()), kT, 0, st_.s>>>(faces(), vx_.p, vxm_.p);
        kr_copy<<<blocks_r(faces()), kT, 0, st_.s>>>(faces(), vy_.p, vym_.p);
        kr_hat<<<blocks_r(faces()), kT, 0, st_.s>>>(faces(), vxm_.p, vxt_.p, vxh_.p);
        kr_hat<<<blocks_r(faces()), kT, 0, st_.s>>>(faces(), vym_.p, vyt_.p, vyh_.p);
        // stage 4: smoke through the midpoint, reflected velocity traced
        // through it, final projection
        advect_smoke(half);
        kr_scale<<<blocks_r(cells()), kT, 0, st_.s>>>(cells(), half_decay, smoke_.p);
        kr_advect_vx<<<blocks_r(faces()), kT, 0, st_.s>>>(n_, h(), half, vxm_.p, vym_.p, vxh_.p, vx_.p);
        kr_advect_vy<<<blocks_r(faces()), kT, 0, st_.s>>>(n_, h(), half, vxm_.p, vym_.p, vyh_.p, vy_.p);
        project(half, half_iters);
    }

    int n_;
    vapor_mac2d_refl_params p_;
    Stream st_;
    DevArray<float> smoke_, fwd_, back_, pressure_, div_, vx_, vy_, vxt_, vyt_, vxm_, vym_, vxh_, vyh_;
    DevArray<uint32_t> state_;
    DevArray<double> energy_;
    DevArray<float> maxima_;
    DevArray<uint32_t> patch_cells_;
    DevArray<float> patch_weights_;
    int patch_count_ = 0;
    bool patch_valid_ = false;
};

}  // namespace vb

// ---- C ABI ----

struct vapor_mac2d_refl {
    vb::Mac2DReflection sim;
    vapor_mac2d_refl(int n, const vapor_mac2d_refl_params& p) : sim(n, p) {}
};

#define VB_APIR extern "C" __attribute__((visibility("default")))

namespace {
void require_r(bool ok, const char* message) {
    if (!ok) vb::fail(VAPOR_INVALID_ARGUMENT, message);
}
// The struct's member initialisers (ReflectionMacFluidSolver2D.hpp:19-22, 57-71).
vapor_mac2d_refl_params refl_defaults() {
    vapor_mac2d_refl_params p{};
    p.mac_cormack_smoke = 1;
    p.source_strength = 1.f;
    p.buoyancy = .8f;
    p.smoke_decay = .3007525f;
    p.project_iterations = 60;
    p.emitter_radius = .08f;
    p.emitter_center_x = .5f;
    p.emitter_center_y = .2f;
    p.emitter_kick_multiplier = 1.f;
    p.stir_strength = 0.f;
    p.sor_omega = 1.9f;
    p.random_seed = 0x9E3779B9u;
    return p;
}
}  // namespace

VB_APIR vapor_status vapor_mac2d_refl_default_params(vapor_mac2d_refl_params* out) {
    return vb::guard([&] {
        require_r(out != nullptr, "null output");
        *out = refl_defaults();
    });
}
VB_APIR vapor_status vapor_mac2d_refl_app_params(int32_t method, vapor_mac2d_refl_params* out) {
    return vb::guard([&] {
        require_r(out != nullptr, "null output");
        if (method != VAPOR_SEMI_LAGRANGIAN && method != VAPOR_MACCORMACK)
            vb::fail(VAPOR_INVALID_ARGUMENT, "Unknown smoke advection method");
        vapor_mac2d_refl_params p = refl_defaults();
        p.mac_cormack_smoke = method == VAPOR_MACCORMACK ? 1 : 0;
        p.emitter_radius = .04f;
        p.project_iterations = 120;
        *out = p;
    });
}
VB_APIR vapor_status vapor_mac2d_refl_create(int32_t n, const vapor_mac2d_refl_params* params,
                                             vapor_mac2d_refl** out) {
    return vb::guard([&] {
        require_r(out != nullptr, "null output");
        *out = nullptr;
        *out = new vapor_mac2d_refl(n, params ? *params : refl_defaults());
    });
}
VB_APIR vapor_status vapor_mac2d_refl_destroy(vapor_mac2d_refl* sim) {
    return vb::guard([&] { delete sim; });
}
VB_APIR vapor_status vapor_mac2d_refl_get_params(const vapor_mac2d_refl* sim, vapor_mac2d_refl_params* out) {
    return vb::guard([&] {
        require_r(sim && out, "null handle or output");
        *out = sim->sim.params();
    });
}
VB_APIR vapor_status vapor_mac2d_refl_set_params(vapor_mac2d_refl* sim, const vapor_mac2d_refl_params* params) {
    return vb::guard([&] {
        require_r(sim && params, "null handle or parameters");
        sim->sim.set_params(*params);
    });
}
VB_APIR vapor_status vapor_mac2d_refl_advance(vapor_mac2d_refl* sim, float dt) {
    return vb::guard([&] {
        require_r(sim != nullptr, "null handle");
        sim->sim.advance(dt);
    });
}
VB_APIR vapor_status vapor_mac2d_refl_reset(vapor_mac2d_refl* sim) {
    return vb::guard([&] {
        require_r(sim != nullptr, "null handle");
        sim->sim.reset();
    });
}
VB_APIR vapor_status vapor_mac2d_refl_upload(vapor_mac2d_refl* sim, const float* smoke, const float* u,
                                             const float* v) {
    return vb::guard([&] {
        require_r(sim != nullptr, "null handle");
        sim->sim.upload(smoke, u, v);
    });
}
VB_APIR vapor_status vapor_mac2d_refl_download(vapor_mac2d_refl* sim, float* smoke, float* u, float* v,
                                               float* pressure) {
    return vb::guard([&] {
        require_r(sim != nullptr, "null handle");
        sim->sim.download(smoke, u, v, pressure);
    });
}
VB_APIR vapor_status vapor_mac2d_refl_diagnostics(vapor_mac2d_refl* sim, vapor_fluid_diagnostics* out) {
    return vb::guard([&] {
        require_r(sim && out, "null handle or output");
        *out = sim->sim.diagnostics();
    });
}
