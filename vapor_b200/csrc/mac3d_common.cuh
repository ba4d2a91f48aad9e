// Device-side building blocks of the MAC 3D step: grid indexing, the clamped
// trilinear sampler and reduction helpers.
//
// Exactness contract: every FP32 expression here evaluates the same IEEE
// operations in the same order as the reference CPU code it cites, and the
// library is compiled with --fmad=false (no FMA contraction) and IEEE division
// and square root. With that, results are bit-identical to the reference's CPU
// path, which is itself compiled without FMA.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vb {

// Staggered locations of a MAC grid.
enum Loc : int { CELL = 0, FACE_X = 1, FACE_Y = 2, FACE_Z = 3 };

// Cubic grid: n cells per side, box size and cell size h = box / n
// (MacGridDomain3D::cellSize, MacGridDomain3D.hpp:20).
struct Grid {
    int n;
    float box;
    float h;
};

__host__ __device__ inline int extent(int n, int loc, int dim) { return n + (loc == dim + 1 ? 1 : 0); }

// idC/idX/idY/idZ (MacGridDomain3D.hpp:22-31): x fastest.
__host__ __device__ inline size_t index_of(int n, int loc, int x, int y, int z) {
    return size_t(x) + size_t(extent(n, loc, 0)) * (size_t(y) + size_t(extent(n, loc, 1)) * size_t(z));
}

__host__ __device__ inline size_t count_of(int n, int loc) {
    return size_t(extent(n, loc, 0)) * size_t(extent(n, loc, 1)) * size_t(extent(n, loc, 2));
}

__device__ __forceinline__ float clampf_ref(float v, float lo, float hi) {
    // std::clamp(v, lo, hi) == v < lo ? lo : (hi < v ? hi : v)
    return v < lo ? lo : (hi < v ? hi : v);
}
__device__ __forceinline__ int clampi_ref(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }
__device__ __forceinline__ float minf_ref(float a, float b) { return b < a ? b : a; }  // std::min
__device__ __forceinline__ float maxf_ref(float a, float b) { return a < b ? b : a; }  // std::max

// Division by the cell size as the reference writes it, coord / h, or, when h
// is a power of two, coord * (1 / h): 1 / h is then exact, so both forms round
// the same real quotient to the same float (also for subnormal results) and
// the multiplication saves the IEEE division's instruction sequence.
template <bool POW2>
__device__ __forceinline__ float div_h(float coord, float h, float ih) {
    return POW2 ? coord * ih : coord / h;
}

// One axis of the clamped trilinear lookup (MacGridSampler3D.cpp:6-11 and the
// staggered variants :23-28, :42-47, :61-66).
struct Bracket {
    int i0, i1;
    float t;
};

template <bool STAGGERED, bool POW2 = false>
__device__ __forceinline__ Bracket bracket(float coord, float h, int n, float ih = 0.f) {
    Bracket b;
    if (STAGGERED) {
        const float g = clampf_ref(div_h<POW2>(coord, h, ih), 0.f, float(n));
        b.i0 = min(int(g), n - 1);
        b.i1 = b.i0 + 1;
        b.t = g - float(b.i0);
    } else {
        const float g = clampf_ref(div_h<POW2>(coord, h, ih) - 0.5f, 0.f, float(n - 1));
        b.i0 = int(g);
        b.i1 = min(b.i0 + 1, n - 1);
        b.t = g - float(b.i0);
    }
    return b;
}

// The reference's fixed 8-term trilinear sum with left-to-right products.
__device__ __forceinline__ float trilinear(float f000, float f100, float f010, float f110, float f001, float f101,
                                           float f011, float f111, float tx, float ty, float tz) {
    const float ux = 1.f - tx, uy = 1.f - ty, uz = 1.f - tz;
    float s = f000 * ux * uy * uz;
    s = s + f100 * tx * uy * uz;
    s = s + f010 * ux * ty * uz;
    s = s + f110 * tx * ty * uz;
    s = s + f001 * ux * uy * tz;
    s = s + f101 * tx * uy * tz;
    s = s + f011 * ux * ty * tz;
    s = s + f111 * tx * ty * tz;
    return s;
}

// Trilinear lookup of a field at location LOC from the three axes' brackets,
// with the reference's fixed 8-term order and left-to-right products. Offsets
// are 32-bit: every field of a valid grid has fewer than 2^31 values.
template <int LOC>
__device__ __forceinline__ float sample_at(const float* __restrict__ f, int n, const Bracket& bx, const Bracket& by,
                                           const Bracket& bz) {
    const int ex = n + (LOC == FACE_X), ey = n + (LOC == FACE_Y);
    const int r00 = ex * (by.i0 + ey * bz.i0);
    const int r10 = ex * (by.i1 + ey * bz.i0);
    const int r01 = ex * (by.i0 + ey * bz.i1);
    const int r11 = ex * (by.i1 + ey * bz.i1);
    return trilinear(__ldg(f + (r00 + bx.i0)), __ldg(f + (r00 + bx.i1)), __ldg(f + (r10 + bx.i0)),
                     __ldg(f + (r10 + bx.i1)), __ldg(f + (r01 + bx.i0)), __ldg(f + (r01 + bx.i1)),
                     __ldg(f + (r11 + bx.i0)), __ldg(f + (r11 + bx.i1)), bx.t, by.t, bz.t);
}

// Trilinear sample of a field at location LOC, world position (px,py,pz), with
// the reference's fixed 8-term order and left-to-right products.
template <int LOC, bool POW2 = false>
__device__ __forceinline__ float sample(const float* __restrict__ f, int n, float h, float px, float py,
                                        float pz, float ih = 0.f) {
    const Bracket bx = bracket<LOC == FACE_X, POW2>(px, h, n, ih);
    const Bracket by = bracket<LOC == FACE_Y, POW2>(py, h, n, ih);
    const Bracket bz = bracket<LOC == FACE_Z, POW2>(pz, h, n, ih);
    return sample_at<LOC>(f, n, bx, by, bz);
}

// Red-black split storage of the projection's cell arrays (b, p, e, r32,
// x64): the cells of colour c = (x+y+z)&1 in row (y,z) lie contiguously at
// c*stride + (z*n + y)*hw + (x>>1), with hw = (n+1)/2 slots per row. A colour
// sweep then reads and writes only dense, coalesced runs: its own half of the
// iterate and of b, and the other colour's half for the neighbours.
struct RBLayout {
    int n, hw;
    size_t stride;  // elements per colour
};
__host__ __device__ inline RBLayout rb_layout(int n) {
    RBLayout L;
    L.n = n;
    L.hw = (n + 1) / 2;
    L.stride = size_t(n) * n * L.hw;
    return L;
}
__host__ __device__ inline size_t rb_count(int n) { return 2 * rb_layout(n).stride; }
__host__ __device__ inline size_t rb_index(const RBLayout& L, int x, int y, int z) {
    return size_t((x + y + z) & 1) * L.stride + (size_t(z) * L.n + y) * L.hw + size_t(x >> 1);
}

struct Vel {
    float x, y, z;
};

// MacGridSampler3D::velocity (MacGridSampler3D.cpp:73-75). The three
// components share their brackets: per axis one staggered (the component
// along it) and one centred (the other two).
template <bool POW2 = false>
__device__ __forceinline__ Vel velocity_at(const float* __restrict__ u, const float* __restrict__ v,
                                           const float* __restrict__ w, int n, float h, float px, float py,
                                           float pz, float ih = 0.f) {
    const Bracket sx = bracket<true, POW2>(px, h, n, ih), cx = bracket<false, POW2>(px, h, n, ih);
    const Bracket sy = bracket<true, POW2>(py, h, n, ih), cy = bracket<false, POW2>(py, h, n, ih);
    const Bracket sz = bracket<true, POW2>(pz, h, n, ih), cz = bracket<false, POW2>(pz, h, n, ih);
    Vel r;
    r.x = sample_at<FACE_X>(u, n, sx, cy, cz);
    r.y = sample_at<FACE_Y>(v, n, cx, sy, cz);
    r.z = sample_at<FACE_Z>(w, n, cx, cy, sz);
    return r;
}

// The brackets of a grid coordinate g = k / 2 (k = 2 i at a staggered
// position i h, 2 i + 1 at a centred one) when h is a power of two: the
// position, its product with 1 / h and the 0.5 shift are then exact, so the
// float brackets above reduce to this integer arithmetic, bit for bit.
__device__ __forceinline__ Bracket bracket_half(int k, int n, bool staggered) {
    Bracket b;
    if (staggered) {
        const int c = min(max(k, 0), 2 * n);  // clamp(g, 0, n)
        b.i0 = min(c >> 1, n - 1);
        b.i1 = b.i0 + 1;
        b.t = 0.5f * float(c - 2 * b.i0);
    } else {
        const int c = min(max(k - 1, 0), 2 * (n - 1));  // clamp(g - .5, 0, n - 1)
        b.i0 = c >> 1;
        b.i1 = min(b.i0 + 1, n - 1);
        b.t = 0.5f * float(c & 1);
    }
    return b;
}

// velocity_at at the sample point of location LOC's node (x, y, z), for a
// power-of-two cell size: the same values from integer brackets.
template <int LOC>
__device__ __forceinline__ Vel velocity_at_node(const float* __restrict__ u, const float* __restrict__ v,
                                                const float* __restrict__ w, int n, int x, int y, int z) {
    const int kx = 2 * x + (LOC == FACE_X ? 0 : 1);
    const int ky = 2 * y + (LOC == FACE_Y ? 0 : 1);
    const int kz = 2 * z + (LOC == FACE_Z ? 0 : 1);
    const Bracket sx = bracket_half(kx, n, true), cx = bracket_half(kx, n, false);
    const Bracket sy = bracket_half(ky, n, true), cy = bracket_half(ky, n, false);
    const Bracket sz = bracket_half(kz, n, true), cz = bracket_half(kz, n, false);
    Vel r;
    r.x = sample_at<FACE_X>(u, n, sx, cy, cz);
    r.y = sample_at<FACE_Y>(v, n, cx, sy, cz);
    r.z = sample_at<FACE_Z>(w, n, cx, cy, sz);
    return r;
}

// ---- reductions -------------------------------------------------------------

// Non-negative floats/doubles order like their bit patterns as unsigned ints,
// so atomicMax on the bits is an exact, order-independent max.
__device__ __forceinline__ void atomic_max_nonneg(unsigned int* addr, float value) {
    atomicMax(addr, __float_as_uint(value));
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* addr, double value) {
    atomicMax(addr, (unsigned long long)__double_as_longlong(value));
}

// Total order key for signed floats (for max and min of signed values).
__device__ __forceinline__ int float_order_key(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : (i ^ 0x7fffffff);
}
__host__ __device__ inline float key_to_float(int k) {
    const int i = k >= 0 ? k : (k ^ 0x7fffffff);
#ifdef __CUDA_ARCH__
    return __int_as_float(i);
#else
    float f;
    __builtin_memcpy(&f, &i, sizeof f);
    return f;
#endif
}

template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T other = __shfl_xor_sync(0xffffffffu, v, o);
        v = v < other ? other : v;
    }
    return v;
}

// Deterministic block sum (fixed tree: warp shuffles, then warp 0).
// `scratch` holds at least 32 T. Result valid in thread 0.
template <class T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T r = T(0);
    if (warp == 0) {
        r = lane < warps ? scratch[lane] : T(0);
        r = warp_sum(r);
    }
    return r;
}
template <class T>
__device__ __forceinline__ T block_max(T v, T* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    T r = T(0);
    if (warp == 0) {
        r = lane < warps ? scratch[lane] : scratch[0];  // pad with a real entry, not 0
        r = warp_max(r);
    }
    return r;
}

}  // namespace vb
