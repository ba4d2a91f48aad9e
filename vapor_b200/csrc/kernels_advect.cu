// Staggered-grid semi-Lagrangian and MacCormack advection
// (reference: src/solvers/mac3d/CpuAdvectionKernels.cpp:18-269, GLSL
// semi_lagrangian.comp:100-110 and maccormack.comp:151-204).
//
// One thread per sample point of the advected location. The forward pass
// writes fwd; the MacCormack pass re-traces forward through fwd, applies the
// 8-donor clamping limiter on the immutable source and falls back to fwd when
// either trace leaves [0, box] or |v| dt / h exceeds the CFL limit.
#include "kernels.hpp"

namespace vb {
namespace {

constexpr int kThreads = 256;

template <int LOC>
__device__ __forceinline__ void decode(int n, int& x, int& y, int& z, bool& valid) {
    const int ex = n + (LOC == FACE_X), ey = n + (LOC == FACE_Y), ez = n + (LOC == FACE_Z);
    const int xy = blockIdx.x * blockDim.x + threadIdx.x;
    z = blockIdx.y;
    y = xy / ex;
    x = xy - y * ex;
    valid = xy < ex * ey && z < ez;
}

// Sample point of location LOC: staggered axis at i*h, the others at (i+.5)h
// (`Vec3 face{ x * dx, (y + .5f) * dx, (z + .5f) * dx }`).
template <int LOC>
__device__ __forceinline__ void position(int x, int y, int z, float h, float& px, float& py, float& pz) {
    px = LOC == FACE_X ? float(x) * h : (float(x) + 0.5f) * h;
    py = LOC == FACE_Y ? float(y) * h : (float(y) + 0.5f) * h;
    pz = LOC == FACE_Z ? float(z) * h : (float(z) + 0.5f) * h;
}

template <int LOC>
__global__ void __launch_bounds__(kThreads) k_advect_forward(Grid g, float dt, const float* __restrict__ src,
                                                             const float* __restrict__ u,
                                                             const float* __restrict__ v,
                                                             const float* __restrict__ w,
                                                             float* __restrict__ out, float post_scale) {
    int x, y, z;
    bool valid;
    decode<LOC>(g.n, x, y, z, valid);
    if (!valid) return;
    float px, py, pz;
    position<LOC>(x, y, z, g.h, px, py, pz);
    const Vel vel = velocity_at(u, v, w, g.n, g.h, px, py, pz);
    const float qx = px - vel.x * dt, qy = py - vel.y * dt, qz = pz - vel.z * dt;
    const float value = sample<LOC>(src, g.n, g.h, qx, qy, qz);
    out[index_of(g.n, LOC, x, y, z)] = value * post_scale;
}

// Base donor index of the limiter: int(pos/h) on the staggered axis, else
// int(pos/h - .5), clamped to the location's index range.
template <bool STAGGERED>
__device__ __forceinline__ int donor(float coord, float h, int n) {
    return STAGGERED ? clampi_ref(int(coord / h), 0, n) : clampi_ref(int(coord / h - 0.5f), 0, n - 1);
}

template <int LOC>
__global__ void __launch_bounds__(kThreads) k_advect_maccormack(Grid g, float dt, float cfl_limit,
                                                                const float* __restrict__ src,
                                                                const float* __restrict__ fwd,
                                                                const float* __restrict__ u,
                                                                const float* __restrict__ v,
                                                                const float* __restrict__ w,
                                                                float* __restrict__ out, float post_scale) {
    int x, y, z;
    bool valid;
    decode<LOC>(g.n, x, y, z, valid);
    if (!valid) return;
    const int n = g.n;
    const float h = g.h, box = g.box;
    const size_t i = index_of(n, LOC, x, y, z);
    float px, py, pz;
    position<LOC>(x, y, z, h, px, py, pz);
    const Vel vel = velocity_at(u, v, w, n, h, px, py, pz);
    const float fx = px - vel.x * dt, fy = py - vel.y * dt, fz = pz - vel.z * dt;
    const float bx = px + vel.x * dt, by = py + vel.y * dt, bz = pz + vel.z * dt;
    const float cfl = sqrtf(vel.x * vel.x + vel.y * vel.y + vel.z * vel.z) * dt / h;
    const float f0 = fwd[i];
    const bool leaves = fx < 0.f || fx > box || fy < 0.f || fy > box || fz < 0.f || fz > box || bx < 0.f ||
                        bx > box || by < 0.f || by > box || bz < 0.f || bz > box;
    float result;
    if (leaves || cfl > cfl_limit) {
        result = f0;
    } else {
        const float back = sample<LOC>(fwd, n, h, bx, by, bz);
        const float corrected = f0 + 0.5f * (__ldg(src + i) - back);
        const int ex = n + (LOC == FACE_X), ey = n + (LOC == FACE_Y), ez = n + (LOC == FACE_Z);
        const int gx = donor<LOC == FACE_X>(fx, h, n);
        const int gy = donor<LOC == FACE_Y>(fy, h, n);
        const int gz = donor<LOC == FACE_Z>(fz, h, n);
        const int x1 = min(gx + 1, ex - 1), y1 = min(gy + 1, ey - 1), z1 = min(gz + 1, ez - 1);
        const float s000 = __ldg(src + index_of(n, LOC, gx, gy, gz));
        float lo = s000, hi = s000;
        const float s[7] = {__ldg(src + index_of(n, LOC, x1, gy, gz)), __ldg(src + index_of(n, LOC, gx, y1, gz)),
                            __ldg(src + index_of(n, LOC, x1, y1, gz)), __ldg(src + index_of(n, LOC, gx, gy, z1)),
                            __ldg(src + index_of(n, LOC, x1, gy, z1)), __ldg(src + index_of(n, LOC, gx, y1, z1)),
                            __ldg(src + index_of(n, LOC, x1, y1, z1))};
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            lo = minf_ref(lo, s[k]);
            hi = maxf_ref(hi, s[k]);
        }
        result = clampf_ref(corrected, lo, hi);
    }
    out[i] = result * post_scale;
}

template <int LOC>
void advect_loc(const Grid& g, float dt, float cfl_limit, bool maccormack, const float* src, const float* u,
                const float* v, const float* w, float* fwd, float* out, float post_scale, cudaStream_t s) {
    const int ex = extent(g.n, LOC, 0), ey = extent(g.n, LOC, 1), ez = extent(g.n, LOC, 2);
    const dim3 grid((ex * ey + kThreads - 1) / kThreads, ez);
    if (!maccormack) {
        count_launch();
        k_advect_forward<LOC><<<grid, kThreads, 0, s>>>(g, dt, src, u, v, w, out, post_scale);
        return;
    }
    count_launch();
    k_advect_forward<LOC><<<grid, kThreads, 0, s>>>(g, dt, src, u, v, w, fwd, 1.f);
    count_launch();
    k_advect_maccormack<LOC><<<grid, kThreads, 0, s>>>(g, dt, cfl_limit, src, fwd, u, v, w, out, post_scale);
}

}  // namespace

void launch_advect(const Grid& g, int loc, float dt, float cfl_limit, bool maccormack, const float* src,
                   const float* u, const float* v, const float* w, float* fwd, float* out, float post_scale,
                   cudaStream_t s) {
    switch (loc) {
        case CELL: advect_loc<CELL>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
        case FACE_X: advect_loc<FACE_X>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
        case FACE_Y: advect_loc<FACE_Y>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
        default: advect_loc<FACE_Z>(g, dt, cfl_limit, maccormack, src, u, v, w, fwd, out, post_scale, s); break;
    }
}

}  // namespace vb
