// Staggered-grid semi-Lagrangian and MacCormack advection
// (reference: src/solvers/mac3d/CpuAdvectionKernels.cpp:18-269, GLSL
// semi_lagrangian.comp:100-110 and maccormack.comp:151-204).
//
// One thread per sample point of the advected location. The forward pass
// writes fwd; the MacCormack pass re-traces forward through fwd, applies the
// 8-donor clamping limiter on the immutable source and falls back to fwd when
// either trace leaves [0, box] or |v| dt / h exceeds the CFL limit.
//
// A launch covers a set of fields: the smoke (cell centres) alone, or the
// three velocity components together (grid rows are the planes of u, then v,
// then w), so a velocity advection is one forward launch and one MacCormack
// launch. When the cell size is a power of two the divisions by h run as
// multiplications by the exact 1/h (same bits, see div_h).
#include "kernels.hpp"

#include <cmath>

namespace vb {
namespace {

constexpr int kThreads = 256;

struct FieldSet {
    const float* src[3];
    float* fwd[3];
    float* out[3];
    // Traced velocity of every sample point, written by the forward pass and
    // read back by the MacCormack pass instead of sampling the flow again
    // (null: the MacCormack pass samples it itself). [field][component].
    float* vel[3][3];
};

// Sample point of location LOC: staggered axis at i*h, the others at (i+.5)h
// (`Vec3 face{ x * dx, (y + .5f) * dx, (z + .5f) * dx }`).
template <int LOC>
__device__ __forceinline__ void position(int x, int y, int z, float h, float& px, float& py, float& pz) {
    px = LOC == FACE_X ? float(x) * h : (float(x) + 0.5f) * h;
    py = LOC == FACE_Y ? float(y) * h : (float(y) + 0.5f) * h;
    pz = LOC == FACE_Z ? float(z) * h : (float(z) + 0.5f) * h;
}

// Base donor index of the limiter: int(pos/h) on the staggered axis, else
// int(pos/h - .5), clamped to the location's index range.
template <bool STAGGERED, bool POW2>
__device__ __forceinline__ int donor(float coord, float h, float ih, int n) {
    return STAGGERED ? clampi_ref(int(div_h<POW2>(coord, h, ih)), 0, n)
                     : clampi_ref(int(div_h<POW2>(coord, h, ih) - 0.5f), 0, n - 1);
}

template <int LOC, bool POW2>
__device__ __forceinline__ void forward_point(const Grid& g, float ih, float dt, int x, int y, int z,
                                              const float* __restrict__ src, const float* __restrict__ u,
                                              const float* __restrict__ v, const float* __restrict__ w,
                                              float* __restrict__ out, float post_scale,
                                              float* const* vel_out = nullptr) {
    float px, py, pz;
    position<LOC>(x, y, z, g.h, px, py, pz);
    const Vel vel = POW2 ? velocity_at_node<LOC>(u, v, w, g.n, x, y, z)
                         : velocity_at<POW2>(u, v, w, g.n, g.h, px, py, pz, ih);
    const int i = int(index_of(g.n, LOC, x, y, z));
    if (vel_out) {
        vel_out[0][i] = vel.x;
        vel_out[1][i] = vel.y;
        vel_out[2][i] = vel.z;
    }
    const float qx = px - vel.x * dt, qy = py - vel.y * dt, qz = pz - vel.z * dt;
    const float value = sample<LOC, POW2>(src, g.n, g.h, qx, qy, qz, ih);
    out[i] = value * post_scale;
}

template <int LOC, bool POW2>
__device__ __forceinline__ void maccormack_point(const Grid& g, float ih, float dt, float cfl_limit, int x, int y,
                                                 int z, const float* __restrict__ src,
                                                 const float* __restrict__ fwd, const float* __restrict__ u,
                                                 const float* __restrict__ v, const float* __restrict__ w,
                                                 float* __restrict__ out, float post_scale,
                                                 float* const* vel_in = nullptr) {
    const int n = g.n;
    const float h = g.h, box = g.box;
    const int i = int(index_of(n, LOC, x, y, z));
    float px, py, pz;
    position<LOC>(x, y, z, h, px, py, pz);
    Vel vel;
    if (vel_in) {  // the forward pass's values for this point (the same bits)
        vel.x = __ldg(vel_in[0] + i);
        vel.y = __ldg(vel_in[1] + i);
        vel.z = __ldg(vel_in[2] + i);
    } else {
        vel = POW2 ? velocity_at_node<LOC>(u, v, w, n, x, y, z) : velocity_at<POW2>(u, v, w, n, h, px, py, pz, ih);
    }
    const float fx = px - vel.x * dt, fy = py - vel.y * dt, fz = pz - vel.z * dt;
    const float bx = px + vel.x * dt, by = py + vel.y * dt, bz = pz + vel.z * dt;
    const float cfl = div_h<POW2>(sqrtf(vel.x * vel.x + vel.y * vel.y + vel.z * vel.z) * dt, h, ih);
    const float f0 = fwd[i];
    const bool leaves = fx < 0.f || fx > box || fy < 0.f || fy > box || fz < 0.f || fz > box || bx < 0.f ||
                        bx > box || by < 0.f || by > box || bz < 0.f || bz > box;
    float result;
    if (leaves || cfl > cfl_limit) {
        result = f0;
    } else {
        const float back = sample<LOC, POW2>(fwd, n, h, bx, by, bz, ih);
        const float corrected = f0 + 0.5f * (__ldg(src + i) - back);
        const int ex = n + (LOC == FACE_X), ey = n + (LOC == FACE_Y), ez = n + (LOC == FACE_Z);
        const int gx = donor<LOC == FACE_X, POW2>(fx, h, ih, n);
        const int gy = donor<LOC == FACE_Y, POW2>(fy, h, ih, n);
        const int gz = donor<LOC == FACE_Z, POW2>(fz, h, ih, n);
        const int x1 = min(gx + 1, ex - 1), y1 = min(gy + 1, ey - 1), z1 = min(gz + 1, ez - 1);
        // row offsets of the donor cube (32-bit: fields hold < 2^31 values)
        const int r00 = ex * (gy + ey * gz), r10 = ex * (y1 + ey * gz);
        const int r01 = ex * (gy + ey * z1), r11 = ex * (y1 + ey * z1);
        const float s000 = __ldg(src + (r00 + gx));
        float lo = s000, hi = s000;
        const float s[7] = {__ldg(src + (r00 + x1)), __ldg(src + (r10 + gx)), __ldg(src + (r10 + x1)),
                            __ldg(src + (r01 + gx)), __ldg(src + (r01 + x1)), __ldg(src + (r11 + gx)),
                            __ldg(src + (r11 + x1))};
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            lo = minf_ref(lo, s[k]);
            hi = maxf_ref(hi, s[k]);
        }
        result = clampf_ref(corrected, lo, hi);
    }
    out[i] = result * post_scale;
}

// Grid row blockIdx.y -> (field of the set, z plane); blockIdx.x * blockDim.x
// + threadIdx.x -> (x, y) within that field's plane. FACES: the set is u, v,
// w (planes n, n and n + 1); otherwise the smoke (n planes).
template <bool FACES, bool MC, bool POW2>
__global__ void __launch_bounds__(kThreads) k_advect_set(Grid g, float dt, float cfl_limit, FieldSet f,
                                                         const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, float post_scale) {
    const int n = g.n;
    const float ih = POW2 ? 1.f / g.h : 0.f;
    int field = 0, z = int(blockIdx.y);
    if (FACES) {
        field = z < n ? 0 : (z < 2 * n ? 1 : 2);
        z -= field * n;
    }
    const int xy = int(blockIdx.x) * blockDim.x + threadIdx.x;
    const int ex = n + (FACES && field == 0), ey = n + (FACES && field == 1);
    if (xy >= ex * ey) return;
    const int y = xy / ex, x = xy - y * ex;
    const float* src = f.src[field];
    float* out = MC ? f.out[field] : f.fwd[field];
    float* const* vc = f.vel[field][0] ? f.vel[field] : nullptr;
    if (!FACES) {
        if (MC) maccormack_point<CELL, POW2>(g, ih, dt, cfl_limit, x, y, z, src, f.fwd[0], u, v, w, out, post_scale, vc);
        else forward_point<CELL, POW2>(g, ih, dt, x, y, z, src, u, v, w, out, post_scale, vc);
    } else if (field == 0) {
        if (MC) maccormack_point<FACE_X, POW2>(g, ih, dt, cfl_limit, x, y, z, src, f.fwd[0], u, v, w, out, 1.f, vc);
        else forward_point<FACE_X, POW2>(g, ih, dt, x, y, z, src, u, v, w, out, 1.f, vc);
    } else if (field == 1) {
        if (MC) maccormack_point<FACE_Y, POW2>(g, ih, dt, cfl_limit, x, y, z, src, f.fwd[1], u, v, w, out, 1.f, vc);
        else forward_point<FACE_Y, POW2>(g, ih, dt, x, y, z, src, u, v, w, out, 1.f, vc);
    } else {
        if (MC) maccormack_point<FACE_Z, POW2>(g, ih, dt, cfl_limit, x, y, z, src, f.fwd[2], u, v, w, out, 1.f, vc);
        else forward_point<FACE_Z, POW2>(g, ih, dt, x, y, z, src, u, v, w, out, 1.f, vc);
    }
}

// One location at a time (staged calls): the same device code, one field.
template <int LOC, bool MC, bool POW2>
__global__ void __launch_bounds__(kThreads) k_advect_one(Grid g, float dt, float cfl_limit,
                                                         const float* __restrict__ src,
                                                         const float* __restrict__ fwd,
                                                         const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, float* __restrict__ out,
                                                         float post_scale) {
    const int n = g.n;
    const float ih = POW2 ? 1.f / g.h : 0.f;
    const int ex = n + (LOC == FACE_X), ey = n + (LOC == FACE_Y);
    const int xy = int(blockIdx.x) * blockDim.x + threadIdx.x;
    if (xy >= ex * ey) return;
    const int z = int(blockIdx.y), y = xy / ex, x = xy - y * ex;
    if (MC) maccormack_point<LOC, POW2>(g, ih, dt, cfl_limit, x, y, z, src, fwd, u, v, w, out, post_scale);
    else forward_point<LOC, POW2>(g, ih, dt, x, y, z, src, u, v, w, out, post_scale);
}

bool power_of_two(float h) {
    int e = 0;
    return std::isfinite(h) && h > 0.f && std::frexp(h, &e) == 0.5f;
}

template <bool FACES, bool POW2>
void advect_set(const Grid& g, float dt, float cfl_limit, bool maccormack, const FieldSet& f, const float* u,
                const float* v, const float* w, float post_scale, cudaStream_t s) {
    const int n = g.n;
    const int plane = FACES ? (n + 1) * n : n * n;
    const dim3 grid((plane + kThreads - 1) / kThreads, FACES ? 3 * n + 1 : n);
    count_launch();
    k_advect_set<FACES, false, POW2><<<grid, kThreads, 0, s>>>(g, dt, cfl_limit, f, u, v, w,
                                                               maccormack ? 1.f : post_scale);
    if (!maccormack) return;
    count_launch();
    k_advect_set<FACES, true, POW2><<<grid, kThreads, 0, s>>>(g, dt, cfl_limit, f, u, v, w, post_scale);
}

template <int LOC, bool POW2>
void advect_loc(const Grid& g, float dt, float cfl_limit, bool maccormack, const float* src, const float* u,
                const float* v, const float* w, float* fwd, float* out, float post_scale, cudaStream_t s) {
    const int ex = extent(g.n, LOC, 0), ey = extent(g.n, LOC, 1), ez = extent(g.n, LOC, 2);
    const dim3 grid((ex * ey + kThreads - 1) / kThreads, ez);
    if (!maccormack) {
        count_launch();
        k_advect_one<LOC, false, POW2><<<grid, kThreads, 0, s>>>(g, dt, cfl_limit, src, nullptr, u, v, w, out,
                                                                 post_scale);
        return;
    }
    count_launch();
    k_advect_one<LOC, false, POW2><<<grid, kThreads, 0, s>>>(g, dt, cfl_limit, src, nullptr, u, v, w, fwd, 1.f);
    count_launch();
    k_advect_one<LOC, true, POW2><<<grid, kThreads, 0, s>>>(g, dt, cfl_limit, src, fwd, u, v, w, out, post_scale);
}

template <bool POW2>
void advect_any(const Grid& g, int loc, float dt, float cfl_limit, bool maccormack, const float* src,
                const float* u, const float* v, const float* w, float* fwd, float* out, float post_scale,
                cudaStream_t s) {
    switch (loc) {
        case CELL: advect_loc<CELL, POW2>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
        case FACE_X: advect_loc<FACE_X, POW2>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
        case FACE_Y: advect_loc<FACE_Y, POW2>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
        default: advect_loc<FACE_Z, POW2>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
    }
}

}  // namespace

void launch_advect(const Grid& g, int loc, float dt, float cfl_limit, bool maccormack, const float* src,
                   const float* u, const float* v, const float* w, float* fwd, float* out, float post_scale,
                   cudaStream_t s) {
    if (power_of_two(g.h)) advect_any<true>(g, loc, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s);
    else advect_any<false>(g, loc, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s);
}

void launch_advect_velocity(const Grid& g, float dt, float cfl_limit, bool maccormack, const float* const src[3],
                            const float* u, const float* v, const float* w, float* const fwd[3],
                            float* const out[3], float* vel_cache, cudaStream_t s) {
    FieldSet f{};
    const size_t faces = size_t(g.n) * g.n * (g.n + 1);
    for (int c = 0; c < 3; ++c) {
        f.src[c] = src[c];
        // without MacCormack the forward pass is the result
        f.fwd[c] = maccormack ? fwd[c] : out[c];
        f.out[c] = out[c];
        for (int k = 0; k < 3; ++k) f.vel[c][k] = (maccormack && vel_cache) ? vel_cache + (3 * c + k) * faces : nullptr;
    }
    if (power_of_two(g.h)) advect_set<true, true>(g, dt, cfl_limit, maccormack, f, u, v, w, 1.f, s);
    else advect_set<true, false>(g, dt, cfl_limit, maccormack, f, u, v, w, 1.f, s);
}

void launch_advect_smoke(const Grid& g, float dt, float cfl_limit, bool maccormack, const float* src,
                         const float* u, const float* v, const float* w, float* fwd, float* out, float post_scale,
                         float* vel_cache, cudaStream_t s) {
    FieldSet f{};
    const size_t cells = size_t(g.n) * g.n * g.n;
    f.src[0] = src;
    f.fwd[0] = maccormack ? fwd : out;
    f.out[0] = out;
    for (int k = 0; k < 3; ++k) f.vel[0][k] = (maccormack && vel_cache) ? vel_cache + k * cells : nullptr;
    if (power_of_two(g.h)) advect_set<false, true>(g, dt, cfl_limit, maccormack, f, u, v, w, post_scale, s);
    else advect_set<false, false>(g, dt, cfl_limit, maccormack, f, u, v, w, post_scale, s);
}

}  // namespace vb
