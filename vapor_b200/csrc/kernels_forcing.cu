// Source injection, buoyancy and closed walls (reference:
// src/solvers/mac3d/MacGridFluidSolver3D.cpp:140-181, MacGridOperators3D.cpp:16-28,
// GLSL resident_ops.comp:18-39).
//
// The reference draws one LCG number per in-sphere cell in z, y, x order
// (MacGridFluidSolver3D.cpp:33-36, 161). The device reproduces that stream
// exactly: each patch row counts its in-sphere cells, a block scan gives every
// row its rank, and the affine LCG map is jumped ahead to that rank in
// O(log rank). The generator state lives in device memory, so a captured step
// replays without host work.
#include "kernels.hpp"

namespace vb {
namespace {

constexpr uint32_t kLcgA = 1664525u, kLcgC = 1013904223u;

__device__ __forceinline__ uint32_t lcg_jump(uint32_t s, uint32_t k) {
    uint32_t A = 1u, C = 0u, a = kLcgA, c = kLcgC;
    while (k) {
        if (k & 1u) {
            A = a * A;
            C = a * C + c;
        }
        c = a * c + c;
        a = a * a;
        k >>= 1;
    }
    return A * s + C;
}

// In-sphere test of MacGridFluidSolver3D.cpp:149-153.
__device__ __forceinline__ bool inside(const EmitterBox& e, float h, int x, int y, int z, float* q2out) {
    const float px = (float(x) + 0.5f) * h, py = (float(y) + 0.5f) * h, pz = (float(z) + 0.5f) * h;
    const float qx = (px - e.ec[0]) / e.erad, qy = (py - e.ec[1]) / e.erad, qz = (pz - e.ec[2]) / e.erad;
    const float q2 = qx * qx + qy * qy + qz * qz;
    if (q2out) *q2out = q2;
    return !(q2 > 1.0f);
}

// One block: stir noise for every in-sphere cell of the patch (NaN outside).
__global__ void __launch_bounds__(1024) k_emit_noise(Grid g, EmitterBox e, uint32_t* rng_state, float* noise) {
    __shared__ int s_scan[1024];
    __shared__ uint32_t s_state0;
    __shared__ int s_base;
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_state0 = *rng_state;
        s_base = 0;
    }
    __syncthreads();
    const uint32_t s0 = s_state0;
    const int sx = e.size[0], sy = e.size[1];
    const int rows = e.size[1] * e.size[2];
    for (int chunk = 0; chunk < rows; chunk += blockDim.x) {
        const int r = chunk + tid;
        const int y = e.lo[1] + (r % sy), z = e.lo[2] + (r / sy);
        int count = 0;
        if (r < rows)
            for (int i = 0; i < sx; ++i) count += inside(e, g.h, e.lo[0] + i, y, z, nullptr) ? 1 : 0;
        // Inclusive Hillis-Steele scan over the chunk.
        s_scan[tid] = count;
        __syncthreads();
        for (int off = 1; off < blockDim.x; off <<= 1) {
            const int add = tid >= off ? s_scan[tid - off] : 0;
            __syncthreads();
            s_scan[tid] += add;
            __syncthreads();
        }
        const int exclusive = s_scan[tid] - count;
        const int base = s_base;
        if (r < rows) {
            uint32_t s = lcg_jump(s0, uint32_t(base + exclusive));
            for (int i = 0; i < sx; ++i) {
                const size_t idx = size_t(i) + size_t(sx) * size_t(r);
                if (inside(e, g.h, e.lo[0] + i, y, z, nullptr)) {
                    s = s * kLcgA + kLcgC;
                    const float unit = float(s >> 8) * (1.0f / 16777216.0f);
                    noise[idx] = (unit - 0.5f) * e.stir * e.dt_scale;
                } else {
                    noise[idx] = __int_as_float(0x7fc00000);
                }
            }
        }
        __syncthreads();
        if (tid == blockDim.x - 1) s_base = base + s_scan[tid];
        __syncthreads();
    }
    __syncthreads();
    if (tid == 0) *rng_state = lcg_jump(s0, uint32_t(s_base));
}

__device__ __forceinline__ bool emitted(const EmitterBox& e, const float* noise, int x, int y, int z, float* j) {
    const int ix = x - e.lo[0], iy = y - e.lo[1], iz = z - e.lo[2];
    if (ix < 0 || iy < 0 || iz < 0 || ix >= e.size[0] || iy >= e.size[1] || iz >= e.size[2]) return false;
    const float v = noise[size_t(ix) + size_t(e.size[0]) * (size_t(iy) + size_t(e.size[1]) * size_t(iz))];
    if (isnan(v)) return false;
    *j = v;
    return true;
}

// Applies the emitter: density, kick on the z-faces below/above, stir on the
// x- and y-faces. A face touched by two cells receives the lower cell's
// noise first, as in the reference's traversal.
__global__ void k_emit_apply(Grid g, EmitterBox e, const float* __restrict__ noise, float* d, float* u, float* v,
                             float* w) {
    const int ex = e.size[0] + 1, ey = e.size[1] + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int tz = blockIdx.y;
    const int ty = t / ex, tx = t - ty * ex;
    if (ty >= ey || tz > e.size[2]) return;
    const int n = g.n;
    const int x = e.lo[0] + tx, y = e.lo[1] + ty, z = e.lo[2] + tz;
    const bool inX = tx < e.size[0], inY = ty < e.size[1], inZ = tz < e.size[2];
    float jc = 0.f, jm = 0.f;
    const bool here = emitted(e, noise, x, y, z, &jc);
    if (inX && inY && inZ && here) {
        float& cell = d[index_of(n, CELL, x, y, z)];
        if (e.profile) {
            float q2;
            inside(e, g.h, x, y, z, &q2);
            // exp in double, rounded once to float: the oracle's CPU
            // evaluation gives the same float
            const float weight = float(exp(double(-3.5f * q2)));
            const float prof = minf_ref(1.f, e.strength * 3.f * weight);
            cell = maxf_ref(cell, prof);
        } else {
            cell = 1.0f;
        }
    }
    if (inY && inZ) {
        const bool below = emitted(e, noise, x - 1, y, z, &jm);
        if (below || here) {
            float& f = u[index_of(n, FACE_X, x, y, z)];
            float val = f;
            if (below) val = val + jm;
            if (here) val = val + jc;
            f = val;
        }
    }
    if (inX && inZ) {
        const bool below = emitted(e, noise, x, y - 1, z, &jm);
        if (below || here) {
            float& f = v[index_of(n, FACE_Y, x, y, z)];
            float val = f;
            if (below) val = val + jm;
            if (here) val = val + jc;
            f = val;
        }
    }
    if (inX && inY && e.apply_kick) {
        const bool below = emitted(e, noise, x, y, z - 1, &jm);
        if (below || here) {
            float& f = w[index_of(n, FACE_Z, x, y, z)];
            f = maxf_ref(f, e.kick);
        }
    }
}

// applyBuoyancy + enforceClosedBoundaries (MacGridFluidSolver3D.cpp:167-181,
// MacGridOperators3D.cpp:16-28): interior z-faces get two separate adds,
// lower cell first; every wall face is zeroed.
__global__ void k_buoyancy_walls(Grid g, float buoyancy, float dt, float split, int apply_buoyancy,
                                 const float* __restrict__ d, float* u, float* v, float* w) {
    const int n = g.n, m = n + 1;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    const int y = t / m, x = t - y * m;
    if (y > n) return;
    if (x < n && y < n) {
        const size_t i = index_of(n, FACE_Z, x, y, z);
        if (z == 0 || z == n) {
            w[i] = 0.f;
        } else if (apply_buoyancy) {
            const float lower = buoyancy * d[index_of(n, CELL, x, y, z - 1)] * dt;
            const float upper = buoyancy * d[index_of(n, CELL, x, y, z)] * dt;
            float f = w[i];
            f = f + split * lower;
            f = f + split * upper;
            w[i] = f;
        }
    }
    if (y < n && z < n && (x == 0 || x == n)) u[index_of(n, FACE_X, x, y, z)] = 0.f;
    if (x < n && z < n && (y == 0 || y == n)) v[index_of(n, FACE_Y, x, y, z)] = 0.f;
}

}  // namespace

void launch_emit(const Grid& g, const EmitterBox& e, uint32_t* rng_state, float* noise, float* density, float* u,
                 float* v, float* w, cudaStream_t s) {
    if (e.size[0] <= 0 || e.size[1] <= 0 || e.size[2] <= 0) return;
    count_launch();
    k_emit_noise<<<1, 1024, 0, s>>>(g, e, rng_state, noise);
    const int ex = e.size[0] + 1, ey = e.size[1] + 1;
    const dim3 grid((ex * ey + 255) / 256, e.size[2] + 1);
    count_launch();
    k_emit_apply<<<grid, 256, 0, s>>>(g, e, noise, density, u, v, w);
}

void launch_buoyancy_walls(const Grid& g, float buoyancy, float dt, float split, const float* density, float* u,
                           float* v, float* w, cudaStream_t s) {
    const int m = g.n + 1;
    const dim3 grid((m * m + 255) / 256, m);
    count_launch();
    k_buoyancy_walls<<<grid, 256, 0, s>>>(g, buoyancy, dt, split, 1, density, u, v, w);
}

void launch_walls(const Grid& g, float* u, float* v, float* w, cudaStream_t s) {
    const int m = g.n + 1;
    const dim3 grid((m * m + 255) / 256, m);
    count_launch();
    k_buoyancy_walls<<<grid, 256, 0, s>>>(g, 0.f, 0.f, 0.f, 0, nullptr, u, v, w);
}

}  // namespace vb
