// Flexible preconditioned conjugate gradients for the pressure solve, with a
// two-level preconditioner: red-black SOR smoothing on the fine grid and a
// coarse-grid correction on the grid coarsened 4x per axis. The coarse
// correction is the learned part (the U-Net maps the coarse residual to the
// coarse pressure); without a network the preconditioner is the smoothing
// alone. No counterpart in the reference, whose only solver is SOR
// (SOR.cpp:22-64); convergence is decided by the same FP64 residual test.
//
// Vectors are FP32 in the solver's red-black split layout (padding slots stay
// zero); dot products are FP64 per-block partials summed in a fixed order by
// one block, so every scalar is deterministic.
#include "kernels.hpp"

#include <algorithm>

namespace vb {
namespace {

constexpr int kThreads = 256;
constexpr int kDotBlocks = 148 * 8;

__device__ __forceinline__ int neighbours(int n, int x, int y, int z) {
    return (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
}

// q = A p (A: Neumann 7-point operator, neighbour-count diagonal). One thread
// per VEC slots of one row of one colour; padding slots get 0.
template <int VEC>
__global__ void __launch_bounds__(kThreads) k_apply_A(int n, const float* __restrict__ ps, float* __restrict__ qs) {
    const RBLayout L = rb_layout(n);
    const int hw = L.hw, groups = hw / VEC;
    const int colour = blockIdx.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    const int y = t / groups;
    if (y >= n) return;
    const int i0 = (t - y * groups) * VEC;
    const int s = (y + z + colour) & 1;
    const size_t row = (size_t(z) * n + y) * hw;
    const size_t own = size_t(colour) * L.stride + row, oth = size_t(1 - colour) * L.stride + row;
    const size_t yo = size_t(hw), zo = size_t(n) * hw;
    const int ny = (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
#pragma unroll
    for (int k = 0; k < VEC; ++k) {
        const int slot = i0 + k;
        const int xc = 2 * slot + s;
        float out = 0.f;
        if (xc < n) {
            const float xo = ps[own + slot];
            float ax = float((xc > 0) + (xc + 1 < n) + ny) * xo;
            const int lo = slot - 1 + s;
            if (xc > 0) ax -= ps[oth + lo];
            if (xc + 1 < n) ax -= ps[oth + lo + 1];
            if (y > 0) ax -= ps[oth + slot - yo];
            if (y + 1 < n) ax -= ps[oth + slot + yo];
            if (z > 0) ax -= ps[oth + slot - zo];
            if (z + 1 < n) ax -= ps[oth + slot + zo];
            out = ax;
        }
        qs[own + slot] = out;
    }
}

// Solid obstacles: `diag` holds each slot's fluid-neighbour count, 0 for a
// solid cell (the mixed solver's split-layout mask). The solver keeps every
// vector at 0 on solid cells, so a solid neighbour adds nothing to a sum;
// the operator's diagonal is the fluid-neighbour count and its row is 0 on a
// solid cell (the rules of the mixed solver's masked sweep and residual).
__global__ void __launch_bounds__(kThreads) k_apply_A_masked(int n, const float* __restrict__ ps,
                                                             const uint8_t* __restrict__ diag,
                                                             float* __restrict__ qs) {
    const RBLayout L = rb_layout(n);
    const size_t count = 2 * L.stride;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        const int colour = int(i / L.stride);
        const size_t rem = i - size_t(colour) * L.stride;
        const int slot = int(rem % L.hw);
        const size_t row = rem / L.hw;
        const int y = int(row % n), z = int(row / n);
        const int x = 2 * slot + ((y + z + colour) & 1);
        float out = 0.f;
        const int d = diag[i];
        if (x < n && d > 0) {
            float ax = float(d) * ps[i];
            if (x > 0) ax -= ps[rb_index(L, x - 1, y, z)];
            if (x + 1 < n) ax -= ps[rb_index(L, x + 1, y, z)];
            if (y > 0) ax -= ps[rb_index(L, x, y - 1, z)];
            if (y + 1 < n) ax -= ps[rb_index(L, x, y + 1, z)];
            if (z > 0) ax -= ps[rb_index(L, x, y, z - 1)];
            if (z + 1 < n) ax -= ps[rb_index(L, x, y, z + 1)];
            out = ax;
        }
        qs[i] = out;
    }
}

// Row-pair access (n % 8 == 0): thread t owns slots 4j..4j+3 of both colours
// in row (y, z), i.e. the 8 cells x = 8j .. 8j+7. In that row the cells with
// even x have colour (y + z) & 1, those with odd x the other colour, so the
// two colour rows are read as E (even x: cell 8j + 2k) and O (odd x: cell
// 8j + 2k + 1) by swapping row pointers: every register index is static.
// Loads are float4 per colour and row, index arithmetic is 32-bit.
struct RowEO {
    float e[4], o[4];
};
__device__ __forceinline__ RowEO load_eo(const float* __restrict__ a, int stride, int off, int sy) {
    const float* even = a + (sy ? stride : 0) + off;  // colour (y + z) & 1 holds the even x
    const float* odd = a + (sy ? 0 : stride) + off;
    const float4 ev = *reinterpret_cast<const float4*>(even);
    const float4 od = *reinterpret_cast<const float4*>(odd);
    RowEO r;
    r.e[0] = ev.x; r.e[1] = ev.y; r.e[2] = ev.z; r.e[3] = ev.w;
    r.o[0] = od.x; r.o[1] = od.y; r.o[2] = od.z; r.o[3] = od.w;
    return r;
}
__device__ __forceinline__ RowEO zero_eo() {
    RowEO r;
#pragma unroll
    for (int k = 0; k < 4; ++k) r.e[k] = r.o[k] = 0.f;
    return r;
}

// (A a) at the 8 cells of a row pair (out[m] for x = 8j + m), in the
// residual's operation order: count * a, minus x-, x+, y-, y+, z-, z+
// (missing neighbours skipped). The x-parity split is the same in every row,
// so the y and z neighbours of an even cell are the neighbour rows' even cells.
__device__ __forceinline__ void apply_pair(const float* __restrict__ a, int n, int hw, int j, int y, int z,
                                           float out[8]) {
    const int plane = n * hw, stride = n * plane;
    const int off = z * plane + y * hw + 4 * j;
    const RowEO me = load_eo(a, stride, off, (y + z) & 1);
    const RowEO ym = y > 0 ? load_eo(a, stride, off - hw, (y + z - 1) & 1) : zero_eo();
    const RowEO yp = y + 1 < n ? load_eo(a, stride, off + hw, (y + z + 1) & 1) : zero_eo();
    const RowEO zm = z > 0 ? load_eo(a, stride, off - plane, (y + z - 1) & 1) : zero_eo();
    const RowEO zp = z + 1 < n ? load_eo(a, stride, off + plane, (y + z + 1) & 1) : zero_eo();
    const int x0 = 8 * j;
    // x-neighbours outside the run: cell x0 - 1 (odd, slot 4j - 1) and x0 + 8 (even, slot 4j + 4)
    const int sy = (y + z) & 1;
    const float left = x0 > 0 ? a[(sy ? 0 : stride) + off - 1] : 0.f;
    const float right = x0 + 8 < n ? a[(sy ? stride : 0) + off + 4] : 0.f;
    const int nyz = (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
        const int x = x0 + m, k = m >> 1;
        const bool even = (m & 1) == 0;
        const float v = even ? me.e[k] : me.o[k];
        float ax = float((x > 0) + (x + 1 < n) + nyz) * v;
        if (x > 0) ax -= even ? (m > 0 ? me.o[k - 1 < 0 ? 0 : k - 1] : left) : me.e[k];
        if (x + 1 < n) ax -= even ? me.o[k] : (m < 7 ? me.e[k + 1 > 3 ? 3 : k + 1] : right);
        if (y > 0) ax -= even ? ym.e[k] : ym.o[k];
        if (y + 1 < n) ax -= even ? yp.e[k] : yp.o[k];
        if (z > 0) ax -= even ? zm.e[k] : zm.o[k];
        if (z + 1 < n) ax -= even ? zp.e[k] : zp.o[k];
        out[m] = ax;
    }
}

// q = A p with FP64 block partials of p.q (n % 8 == 0). Grid (row-pair
// groups of one plane / 256, n planes): no index division beyond one per thread.
__global__ void __launch_bounds__(kThreads) k_apply_A_dot(int n, const float* __restrict__ ps, float* __restrict__ qs,
                                                          double* __restrict__ partials) {
    __shared__ double s_sum[32];
    const int hw = n >> 1, groups = hw >> 2;
    const int plane = n * hw, stride = n * plane;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y, y = t / groups, j = t - y * groups;
    double acc = 0.0;
    if (y < n) {
        float q[8];
        apply_pair(ps, n, hw, j, y, z, q);
        const int off = z * plane + y * hw + 4 * j;
        const int sy = (y + z) & 1;
        float* qe = qs + (sy ? stride : 0) + off;  // even-x cells of this row
        float* qo = qs + (sy ? 0 : stride) + off;
        const RowEO pp = load_eo(ps, stride, off, sy);
        *reinterpret_cast<float4*>(qe) = make_float4(q[0], q[2], q[4], q[6]);
        *reinterpret_cast<float4*>(qo) = make_float4(q[1], q[3], q[5], q[7]);
#pragma unroll
        for (int k = 0; k < 4; ++k) acc += double(pp.e[k]) * q[2 * k] + double(pp.o[k]) * q[2 * k + 1];
    }
    const double b = block_sum(acc, s_sum);
    if (threadIdx.x == 0) {
        const int blk = blockIdx.y * gridDim.x + blockIdx.x;
        partials[2 * blk] = b;
        partials[2 * blk + 1] = 0.0;
    }
}

// Fused direction step on row pairs (n % 8 == 0), grid as k_apply_A_dot.
// Capped at 64 registers (4 resident blocks per SM instead of 3; a few
// bytes spill): the pass is bound by the latency of its neighbour-row
// loads, and the higher occupancy measured 0.3 ms per 256^3 step faster.
// with po = p[p_cur] and pn the other buffer, e += alpha_pending po (when an
// update is pending), pn = z + beta po (a copy of z for the first direction),
// q = A pn and FP64 block partials of pn.q. The stencil reads pn at the
// neighbours as z + beta po, the value the neighbour's thread stores, so q
// equals A applied to the stored pn.
__device__ __forceinline__ float dir_value(float zv, float pv, float beta, bool first) {
    return first ? zv : zv + beta * pv;
}
__device__ __forceinline__ RowEO dir_eo(const float* __restrict__ z, const float* __restrict__ po, int stride,
                                        int off, int sy, float beta, bool first) {
    const RowEO a = load_eo(z, stride, off, sy);
    if (first) return a;
    const RowEO b = load_eo(po, stride, off, sy);
    RowEO r;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        r.e[k] = a.e[k] + beta * b.e[k];
        r.o[k] = a.o[k] + beta * b.o[k];
    }
    return r;
}

__global__ void __launch_bounds__(kThreads, 4) k_direction_apply(int n, const float* __restrict__ zs, float* P0, float* P1,
                                                              float* __restrict__ es, float* __restrict__ qs,
                                                              const CgControl* __restrict__ cg,
                                                              double* __restrict__ partials) {
    __shared__ double s_sum[32];
    const float* __restrict__ po = cg->p_cur ? P1 : P0;
    float* __restrict__ pn = cg->p_cur ? P0 : P1;
    const float beta = float(cg->beta), ap = float(cg->alpha_pending);
    const bool first = (cg->flags & 1) == 0, pending = (cg->flags & 2) != 0;
    const int hw = n >> 1, groups = hw >> 2;
    const int plane = n * hw, stride = n * plane;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y, y = t / groups, j = t - y * groups;
    double acc = 0.0;
    if (y < n) {
        const int off = z * plane + y * hw + 4 * j;
        const int sy = (y + z) & 1;
        const RowEO me = dir_eo(zs, po, stride, off, sy, beta, first);
        const RowEO ym = y > 0 ? dir_eo(zs, po, stride, off - hw, (y + z - 1) & 1, beta, first) : zero_eo();
        const RowEO yp = y + 1 < n ? dir_eo(zs, po, stride, off + hw, (y + z + 1) & 1, beta, first) : zero_eo();
        const RowEO zm = z > 0 ? dir_eo(zs, po, stride, off - plane, (y + z - 1) & 1, beta, first) : zero_eo();
        const RowEO zp = z + 1 < n ? dir_eo(zs, po, stride, off + plane, (y + z + 1) & 1, beta, first) : zero_eo();
        const int x0 = 8 * j;
        const int lo = (sy ? 0 : stride) + off - 1, ro = (sy ? stride : 0) + off + 4;
        const float left = x0 > 0 ? dir_value(zs[lo], po[lo], beta, first) : 0.f;
        const float right = x0 + 8 < n ? dir_value(zs[ro], po[ro], beta, first) : 0.f;
        const int nyz = (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
        float q[8];
#pragma unroll
        for (int m = 0; m < 8; ++m) {  // apply_pair's operation order
            const int x = x0 + m, k = m >> 1;
            const bool even = (m & 1) == 0;
            const float v = even ? me.e[k] : me.o[k];
            float ax = float((x > 0) + (x + 1 < n) + nyz) * v;
            if (x > 0) ax -= even ? (m > 0 ? me.o[k - 1 < 0 ? 0 : k - 1] : left) : me.e[k];
            if (x + 1 < n) ax -= even ? me.o[k] : (m < 7 ? me.e[k + 1 > 3 ? 3 : k + 1] : right);
            if (y > 0) ax -= even ? ym.e[k] : ym.o[k];
            if (y + 1 < n) ax -= even ? yp.e[k] : yp.o[k];
            if (z > 0) ax -= even ? zm.e[k] : zm.o[k];
            if (z + 1 < n) ax -= even ? zp.e[k] : zp.o[k];
            q[m] = ax;
        }
        const int ev = (sy ? stride : 0) + off, od = (sy ? 0 : stride) + off;
        *reinterpret_cast<float4*>(qs + ev) = make_float4(q[0], q[2], q[4], q[6]);
        *reinterpret_cast<float4*>(qs + od) = make_float4(q[1], q[3], q[5], q[7]);
        *reinterpret_cast<float4*>(pn + ev) = make_float4(me.e[0], me.e[1], me.e[2], me.e[3]);
        *reinterpret_cast<float4*>(pn + od) = make_float4(me.o[0], me.o[1], me.o[2], me.o[3]);
        if (pending) {
            const RowEO pe = load_eo(po, stride, off, sy);
            const RowEO ee = load_eo(es, stride, off, sy);
            *reinterpret_cast<float4*>(es + ev) = make_float4(ee.e[0] + ap * pe.e[0], ee.e[1] + ap * pe.e[1],
                                                              ee.e[2] + ap * pe.e[2], ee.e[3] + ap * pe.e[3]);
            *reinterpret_cast<float4*>(es + od) = make_float4(ee.o[0] + ap * pe.o[0], ee.o[1] + ap * pe.o[1],
                                                              ee.o[2] + ap * pe.o[2], ee.o[3] + ap * pe.o[3]);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc += double(me.e[k]) * q[2 * k] + double(me.o[k]) * q[2 * k + 1];
    }
    const double b = block_sum(acc, s_sum);
    if (threadIdx.x == 0) {
        const int blk = blockIdx.y * gridDim.x + blockIdx.x;
        partials[2 * blk] = b;
        partials[2 * blk + 1] = 0.0;
    }
}

// r -= alpha q and max |r| (FP32) into ctrl->res32_bits (count % 4 == 0).
__global__ void __launch_bounds__(kThreads) k_update_r4(size_t count4, float4* __restrict__ r,
                                                        const float4* __restrict__ q,
                                                        const CgControl* __restrict__ cg, ProjControl* ctrl) {
    __shared__ float s_max[32];
    const float alpha = float(cg->alpha);
    float m = 0.f;
    unsigned int bad = 0u;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count4; i += size_t(gridDim.x) * blockDim.x) {
        const float4 qv = q[i];
        float4 rv = r[i];
        rv.x = rv.x - alpha * qv.x;
        rv.y = rv.y - alpha * qv.y;
        rv.z = rv.z - alpha * qv.z;
        rv.w = rv.w - alpha * qv.w;
        r[i] = rv;
        if (!isfinite(rv.x) || !isfinite(rv.y) || !isfinite(rv.z) || !isfinite(rv.w)) bad = 1u;
        m = fmaxf(m, fmaxf(fmaxf(fabsf(rv.x), fabsf(rv.y)), fmaxf(fabsf(rv.z), fabsf(rv.w))));
    }
    const float bm = block_max(m, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomicMax(&ctrl->res32_bits, __float_as_uint(bm));
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

// Before a re-centring (gated on ctrl->recentre): e += alpha_pending p_cur.
__global__ void __launch_bounds__(kThreads) k_fold_pending(size_t count4, float4* __restrict__ e,
                                                           const float4* __restrict__ P0, const float4* __restrict__ P1,
                                                           const CgControl* __restrict__ cg,
                                                           const ProjControl* __restrict__ ctrl) {
    if (!ctrl->recentre || (cg->flags & 2) == 0) return;
    const float ap = float(cg->alpha_pending);
    const float4* __restrict__ p = cg->p_cur ? P1 : P0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count4; i += size_t(gridDim.x) * blockDim.x) {
        const float4 pv = p[i];
        float4 ev = e[i];
        ev.x = ev.x + ap * pv.x;
        ev.y = ev.y + ap * pv.y;
        ev.z = ev.z + ap * pv.z;
        ev.w = ev.w + ap * pv.w;
        e[i] = ev;
    }
}

__global__ void k_fold_clear(CgControl* cg, const ProjControl* __restrict__ ctrl) {
    if (ctrl->recentre) cg->flags &= ~2;
}

// Restriction pass 1 on row pairs (n % 16 == 0): the residuals r - A z of the
// 8 cells, summed per coarse block in x order, into rows[(z n + y) nc + cx].
// Grid as k_apply_A_dot.
__global__ void __launch_bounds__(kThreads) k_restrict_pairs(int n, const float* __restrict__ r,
                                                             const float* __restrict__ zs, float* __restrict__ rows) {
    const int hw = n >> 1, groups = hw >> 2, nc = n >> 2;
    const int plane = n * hw, stride = n * plane;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y, y = t / groups, j = t - y * groups;
    if (y >= n) return;
    float az[8];
    apply_pair(zs, n, hw, j, y, z, az);
    const RowEO rr = load_eo(r, stride, z * plane + y * hw + 4 * j, (y + z) & 1);
    float sum[2] = {0.f, 0.f};
#pragma unroll
    for (int m = 0; m < 8; ++m) sum[m >> 2] += ((m & 1) ? rr.o[m >> 1] : rr.e[m >> 1]) - az[m];
    const int base = (z * n + y) * nc + 2 * j;
    rows[base] = sum[0];
    rows[base + 1] = sum[1];
}

// z += gamma (zc[C] - mean) on row pairs (n % 16 == 0); grid as k_apply_A_dot.
__global__ void __launch_bounds__(kThreads) k_prolong_pairs(int n, float* __restrict__ zs,
                                                            const float* __restrict__ zc,
                                                            const CgControl* __restrict__ cg) {
    const int hw = n >> 1, groups = hw >> 2, nc = n >> 2;
    const int plane = n * hw, stride = n * plane;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y, y = t / groups, j = t - y * groups;
    if (y >= n) return;
    const float g = float(cg->gamma), mean = float(cg->zc_mean);
    const int cbase = ((z >> 2) * nc + (y >> 2)) * nc + 2 * j;
    const float a = g * (zc[cbase] - mean), b = g * (zc[cbase + 1] - mean);
    const int off = z * plane + y * hw + 4 * j;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
        float4* p = reinterpret_cast<float4*>(zs + c * stride + off);
        float4 v = *p;
        // slots 4j, 4j+1 hold x in [8j, 8j+3] (coarse 2j); 4j+2, 4j+3 hold [8j+4, 8j+7]
        v.x = v.x + a;
        v.y = v.y + a;
        v.z = v.z + b;
        v.w = v.w + b;
        *p = v;
    }
}

// Per-block FP64 partials of sum a.b (and of c.d when c is given).
__global__ void __launch_bounds__(kThreads) k_dot2(size_t count, const float* __restrict__ a,
                                                   const float* __restrict__ b, const float* __restrict__ c,
                                                   const float* __restrict__ d, double* __restrict__ partials) {
    __shared__ double s_sum[32];
    double ab = 0.0, cd = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        ab += double(a[i]) * double(b[i]);
        if (c) cd += double(c[i]) * double(d[i]);
    }
    const double sab = block_sum(ab, s_sum);
    const double scd = block_sum(cd, s_sum);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = sab;
        partials[2 * blockIdx.x + 1] = scd;
    }
}

__device__ void sum2(const double* __restrict__ partials, int blocks, double* s_sum, double& a, double& b) {
    double x = 0.0, y = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
        x += partials[2 * i];
        y += partials[2 * i + 1];
    }
    a = block_sum(x, s_sum);
    b = block_sum(y, s_sum);
}

// rho = z.r for the first direction (which the fused step forms as z: beta
// 0, nothing pending, buffer 0 current).
__global__ void k_rho_finish(const double* __restrict__ partials, int blocks, CgControl* cg) {
    __shared__ double s_sum[32];
    double zr, unused;
    sum2(partials, blocks, s_sum, zr, unused);
    if (threadIdx.x == 0) {
        cg->rho = zr;
        cg->beta = 0.0;
        cg->alpha_pending = 0.0;
        cg->p_cur = 0;
        cg->flags = 0;
    }
}

// The fused step's alpha: as k_alpha_finish, then the new direction becomes
// current and its update pending.
__global__ void k_alpha_finish_pp(const double* __restrict__ partials, int blocks, CgControl* cg) {
    __shared__ double s_sum[32];
    double pq, unused;
    sum2(partials, blocks, s_sum, pq, unused);
    if (threadIdx.x == 0) {
        cg->pq = pq;
        cg->alpha = (pq > 0.0 && isfinite(cg->rho / pq)) ? cg->rho / pq : 0.0;
        cg->alpha_pending = cg->alpha;
        cg->p_cur ^= 1;
        cg->flags = 3;
    }
}

// alpha = rho / (p.q).
__global__ void k_alpha_finish(const double* __restrict__ partials, int blocks, CgControl* cg) {
    __shared__ double s_sum[32];
    double pq, unused;
    sum2(partials, blocks, s_sum, pq, unused);
    if (threadIdx.x == 0) {
        cg->pq = pq;
        cg->alpha = (pq > 0.0 && isfinite(cg->rho / pq)) ? cg->rho / pq : 0.0;
    }
}

// Flexible (Polak-Ribiere) beta = z_new.(r_new - r_old) / rho_old with
// r_new - r_old = -alpha q, then rho = z_new.r_new.
__global__ void k_beta_finish(const double* __restrict__ partials, int blocks, CgControl* cg) {
    __shared__ double s_sum[32];
    double zr, zq;
    sum2(partials, blocks, s_sum, zr, zq);
    if (threadIdx.x == 0) {
        const double beta = -cg->alpha * zq / cg->rho;
        cg->beta = (cg->rho != 0.0 && isfinite(beta)) ? beta : 0.0;
        cg->rho = zr;
    }
}

// e += alpha p, r -= alpha q, and max |r| (FP32) into ctrl->res32_bits.
__global__ void __launch_bounds__(kThreads) k_cg_update(size_t count, float* __restrict__ e, float* __restrict__ r,
                                                        const float* __restrict__ p, const float* __restrict__ q,
                                                        const CgControl* __restrict__ cg, ProjControl* ctrl) {
    __shared__ float s_max[32];
    const float alpha = float(cg->alpha);
    float m = 0.f;
    unsigned int bad = 0u;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        e[i] = e[i] + alpha * p[i];
        const float rn = r[i] - alpha * q[i];
        r[i] = rn;
        if (!isfinite(rn)) bad = 1u;
        m = fmaxf(m, fabsf(rn));
    }
    const float bm = block_max(m, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomicMax(&ctrl->res32_bits, __float_as_uint(bm));
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

// The same update four elements at a time (count % 4 == 0, 16-byte aligned).
__global__ void __launch_bounds__(kThreads) k_cg_update4(size_t count4, float4* __restrict__ e,
                                                         float4* __restrict__ r, const float4* __restrict__ p,
                                                         const float4* __restrict__ q,
                                                         const CgControl* __restrict__ cg, ProjControl* ctrl) {
    __shared__ float s_max[32];
    const float alpha = float(cg->alpha);
    float m = 0.f;
    unsigned int bad = 0u;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count4; i += size_t(gridDim.x) * blockDim.x) {
        const float4 pv = p[i], qv = q[i];
        float4 ev = e[i], rv = r[i];
        ev.x = ev.x + alpha * pv.x;
        ev.y = ev.y + alpha * pv.y;
        ev.z = ev.z + alpha * pv.z;
        ev.w = ev.w + alpha * pv.w;
        rv.x = rv.x - alpha * qv.x;
        rv.y = rv.y - alpha * qv.y;
        rv.z = rv.z - alpha * qv.z;
        rv.w = rv.w - alpha * qv.w;
        e[i] = ev;
        r[i] = rv;
        if (!isfinite(rv.x) || !isfinite(rv.y) || !isfinite(rv.z) || !isfinite(rv.w)) bad = 1u;
        m = fmaxf(m, fmaxf(fmaxf(fabsf(rv.x), fabsf(rv.y)), fmaxf(fabsf(rv.z), fabsf(rv.w))));
    }
    const float bm = block_max(m, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomicMax(&ctrl->res32_bits, __float_as_uint(bm));
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

// p = z + beta p.
__global__ void __launch_bounds__(kThreads) k_p_update(size_t count, float* __restrict__ p,
                                                       const float* __restrict__ z, const CgControl* __restrict__ cg) {
    const float beta = float(cg->beta);
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
        p[i] = z[i] + beta * p[i];
}

// One iteration done: count it, and decide whether to re-centre in FP64 (the
// recurrence residual reached the target or dropped by kRecentreDrop since
// the last re-centring, the budget is spent, or kRecentreSweeps iterations
// passed). Sets the if-condition of the re-centring group.
__global__ void k_cg_decide(ProjControl* ctrl, int use_if, cudaGraphConditionalHandle if_handle) {
    ctrl->iterations = min(ctrl->iterations + 1, ctrl->max_iterations);
    ctrl->since += 1;
    const float rho = __uint_as_float(ctrl->res32_bits);
    ctrl->res32_bits = 0u;
    const int recentre = double(rho) <= ctrl->target || double(rho) <= double(kRecentreDrop) * ctrl->r0 ||
                         ctrl->since >= kRecentreSweeps || ctrl->iterations >= ctrl->max_iterations ||
                         (ctrl->nonfinite & 4u) != 0u;
    ctrl->recentre = recentre;
    ctrl->result.linear_solve.iterations = ctrl->iterations;
    if (!recentre) ctrl->done = 0;
    if (use_if) cudaGraphSetConditional(if_handle, recentre ? 1u : 0u);
}

// Coarse right-hand side rc[C] = sum over the 4^3 fine cells of C of
// r - A z, in two deterministic passes. Pass 1: one thread per run of 4
// fine cells along x (row y, plane z) sums their residuals (FP32, x order)
// into rows[(z * n + y) * nc + cx].
__global__ void __launch_bounds__(kThreads) k_restrict_rows(int n, const float* __restrict__ r,
                                                            const float* __restrict__ zs, float* __restrict__ rows) {
    const RBLayout L = rb_layout(n);
    const int nc = n >> 2;
    const long total = long(n) * n * nc;
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int cx = int(t % nc);
        const long yz = t / nc;
        const int y = int(yz % n), z = int(yz / n);
        float acc = 0.f;
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
            const int x = 4 * cx + dx;
            const size_t me = rb_index(L, x, y, z);
            float ax = float(neighbours(n, x, y, z)) * zs[me];
            if (x > 0) ax -= zs[rb_index(L, x - 1, y, z)];
            if (x + 1 < n) ax -= zs[rb_index(L, x + 1, y, z)];
            if (y > 0) ax -= zs[rb_index(L, x, y - 1, z)];
            if (y + 1 < n) ax -= zs[rb_index(L, x, y + 1, z)];
            if (z > 0) ax -= zs[rb_index(L, x, y, z - 1)];
            if (z + 1 < n) ax -= zs[rb_index(L, x, y, z + 1)];
            acc += r[me] - ax;
        }
        rows[t] = acc;
    }
}

// k_restrict_rows with obstacles: solid cells contribute nothing (their r
// and z are 0), fluid cells r - A z with the masked operator.
__global__ void __launch_bounds__(kThreads) k_restrict_rows_masked(int n, const float* __restrict__ r,
                                                                   const float* __restrict__ zs,
                                                                   const uint8_t* __restrict__ diag,
                                                                   float* __restrict__ rows) {
    const RBLayout L = rb_layout(n);
    const int nc = n >> 2;
    const long total = long(n) * n * nc;
    for (long t = long(blockIdx.x) * blockDim.x + threadIdx.x; t < total; t += long(gridDim.x) * blockDim.x) {
        const int cx = int(t % nc);
        const long yz = t / nc;
        const int y = int(yz % n), z = int(yz / n);
        float acc = 0.f;
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
            const int x = 4 * cx + dx;
            const size_t me = rb_index(L, x, y, z);
            const int d = diag[me];
            if (d == 0) continue;
            float ax = float(d) * zs[me];
            if (x > 0) ax -= zs[rb_index(L, x - 1, y, z)];
            if (x + 1 < n) ax -= zs[rb_index(L, x + 1, y, z)];
            if (y > 0) ax -= zs[rb_index(L, x, y - 1, z)];
            if (y + 1 < n) ax -= zs[rb_index(L, x, y + 1, z)];
            if (z > 0) ax -= zs[rb_index(L, x, y, z - 1)];
            if (z + 1 < n) ax -= zs[rb_index(L, x, y, z + 1)];
            acc += r[me] - ax;
        }
        rows[t] = acc;
    }
}

// Pass 2: rc[C] = sum of the 4 x 4 (y, z) row sums of C, fixed order.
__global__ void __launch_bounds__(kThreads) k_restrict_blocks(int n, const float* __restrict__ rows,
                                                              float* __restrict__ rc) {
    const int nc = n >> 2;
    const long cells = long(nc) * nc * nc;
    for (long c = long(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += long(gridDim.x) * blockDim.x) {
        const int cx = int(c % nc), cy = int((c / nc) % nc), cz = int(c / (long(nc) * nc));
        float acc = 0.f;
        for (int dz = 0; dz < 4; ++dz)
            for (int dy = 0; dy < 4; ++dy)
                acc += rows[(long(4 * cz + dz) * n + (4 * cy + dy)) * nc + cx];
        rc[c] = acc;
    }
}

// Coarse Galerkin sums for the correction q = zc - mean(zc): partials of
// zc.rc, zc.(L zc), sum zc, sum rc (L: coarse Neumann 7-point operator).
__global__ void __launch_bounds__(kThreads) k_coarse_sums(int nc, const float* __restrict__ zc,
                                                          const float* __restrict__ rc,
                                                          double* __restrict__ partials) {
    __shared__ double s_sum[32];
    const long cells = long(nc) * nc * nc;
    const long plane = long(nc) * nc;
    double zr = 0.0, zlz = 0.0, sz = 0.0, sr = 0.0;
    for (long c = long(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += long(gridDim.x) * blockDim.x) {
        const int x = int(c % nc), y = int((c / nc) % nc), z = int(c / plane);
        const double v = double(zc[c]);
        double lz = double(neighbours(nc, x, y, z)) * v;
        if (x > 0) lz -= double(zc[c - 1]);
        if (x + 1 < nc) lz -= double(zc[c + 1]);
        if (y > 0) lz -= double(zc[c - nc]);
        if (y + 1 < nc) lz -= double(zc[c + nc]);
        if (z > 0) lz -= double(zc[c - plane]);
        if (z + 1 < nc) lz -= double(zc[c + plane]);
        zr += v * double(rc[c]);
        zlz += v * lz;
        sz += v;
        sr += double(rc[c]);
    }
    const double a = block_sum(zr, s_sum);
    const double b = block_sum(zlz, s_sum);
    const double c2 = block_sum(sz, s_sum);
    const double d = block_sum(sr, s_sum);
    if (threadIdx.x == 0) {
        partials[4 * blockIdx.x] = a;
        partials[4 * blockIdx.x + 1] = b;
        partials[4 * blockIdx.x + 2] = c2;
        partials[4 * blockIdx.x + 3] = d;
    }
}

// gamma = (q.rc) / (q.(A_c q)) with A_c = 16 L (the Galerkin operator P^T A P
// of piecewise-constant prolongation by 4 per axis), q = zc - mean(zc).
__global__ void k_coarse_finish(const double* __restrict__ partials, int blocks, double cells, CgControl* cg) {
    __shared__ double s_sum[32];
    double zr = 0.0, zlz = 0.0, sz = 0.0, sr = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
        zr += partials[4 * i];
        zlz += partials[4 * i + 1];
        sz += partials[4 * i + 2];
        sr += partials[4 * i + 3];
    }
    zr = block_sum(zr, s_sum);
    zlz = block_sum(zlz, s_sum);
    sz = block_sum(sz, s_sum);
    sr = block_sum(sr, s_sum);
    if (threadIdx.x == 0) {
        const double mean = sz / cells;
        const double num = zr - mean * sr;
        const double den = 16.0 * zlz;
        const double g = num / den;
        cg->zc_mean = mean;
        cg->gamma = (den > 0.0 && isfinite(g)) ? g : 0.0;
    }
}

// z += gamma (zc[C(cell)] - mean) over every fine cell, walking the split
// layout in storage order (coalesced); padding slots are left alone.
__global__ void __launch_bounds__(kThreads) k_prolong_add(int n, float* __restrict__ zs, const float* __restrict__ zc,
                                                          const CgControl* __restrict__ cg) {
    const RBLayout L = rb_layout(n);
    const int nc = n >> 2;
    const float g = float(cg->gamma), m = float(cg->zc_mean);
    const size_t count = 2 * L.stride;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        const int colour = int(i / L.stride);
        const size_t rem = i - size_t(colour) * L.stride;
        const int slot = int(rem % L.hw);
        const size_t row = rem / L.hw;
        const int y = int(row % n), z = int(row / n);
        const int x = 2 * slot + ((y + z + colour) & 1);
        if (x >= n) continue;
        const size_t coarse = (size_t(z >> 2) * nc + (y >> 2)) * nc + (x >> 2);
        zs[i] = zs[i] + g * (zc[coarse] - m);
    }
}

// k_prolong_add on fluid cells only (solid cells keep z = 0).
__global__ void __launch_bounds__(kThreads) k_prolong_add_masked(int n, float* __restrict__ zs,
                                                                 const float* __restrict__ zc,
                                                                 const uint8_t* __restrict__ diag,
                                                                 const CgControl* __restrict__ cg) {
    const RBLayout L = rb_layout(n);
    const int nc = n >> 2;
    const float g = float(cg->gamma), m = float(cg->zc_mean);
    const size_t count = 2 * L.stride;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x) {
        if (diag[i] == 0) continue;
        const int colour = int(i / L.stride);
        const size_t rem = i - size_t(colour) * L.stride;
        const int slot = int(rem % L.hw);
        const size_t row = rem / L.hw;
        const int y = int(row % n), z = int(row / n);
        const int x = 2 * slot + ((y + z + colour) & 1);
        if (x >= n) continue;
        const size_t coarse = (size_t(z >> 2) * nc + (y >> 2)) * nc + (x >> 2);
        zs[i] = zs[i] + g * (zc[coarse] - m);
    }
}

__global__ void __launch_bounds__(kThreads) k_log_coarse(const float* __restrict__ rc, size_t cells,
                                                         float* __restrict__ log, int capacity,
                                                         const int* __restrict__ counter) {
    const size_t slot = size_t(*counter % capacity);
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < cells; i += size_t(gridDim.x) * blockDim.x)
        log[slot * cells + i] = rc[i];
}
__global__ void k_log_advance(int* counter) { *counter += 1; }

int blocks_for(size_t count) {
    return int(std::min<size_t>((count + kThreads - 1) / kThreads, size_t(kDotBlocks)));
}

}  // namespace

static dim3 pair_grid(int n) {
    const int groups = n / 8;
    return dim3(unsigned((groups * n + kThreads - 1) / kThreads), unsigned(n));
}

int cg_partial_capacity(int n) {
    const dim3 g = pair_grid(n);
    return std::max(4 * kDotBlocks, int(2 * g.x * g.y));
}

void launch_apply_A(int n, const float* p, float* q, cudaStream_t s) {
    const RBLayout L = rb_layout(n);
    count_launch();
    if (L.hw % 4 == 0) {
        const dim3 grid((L.hw / 4 * n + kThreads - 1) / kThreads, n, 2);
        k_apply_A<4><<<grid, kThreads, 0, s>>>(n, p, q);
    } else {
        const dim3 grid((L.hw * n + kThreads - 1) / kThreads, n, 2);
        k_apply_A<1><<<grid, kThreads, 0, s>>>(n, p, q);
    }
}

void launch_cg_rho(size_t count, const float* z, const float* r, double* partials, CgControl* cg, cudaStream_t s) {
    const int blocks = blocks_for(count);
    count_launch();
    k_dot2<<<blocks, kThreads, 0, s>>>(count, z, r, nullptr, nullptr, partials);
    count_launch();
    k_rho_finish<<<1, 1024, 0, s>>>(partials, blocks, cg);
}

void launch_cg_alpha(size_t count, const float* p, const float* q, double* partials, CgControl* cg,
                     cudaStream_t s) {
    const int blocks = blocks_for(count);
    count_launch();
    k_dot2<<<blocks, kThreads, 0, s>>>(count, p, q, nullptr, nullptr, partials);
    count_launch();
    k_alpha_finish<<<1, 1024, 0, s>>>(partials, blocks, cg);
}

void launch_apply_A_alpha(int n, const float* p, float* q, double* partials, CgControl* cg, cudaStream_t s,
                          const uint8_t* diag) {
    if (diag) {
        count_launch();
        k_apply_A_masked<<<blocks_for(rb_count(n)), kThreads, 0, s>>>(n, p, diag, q);
        launch_cg_alpha(rb_count(n), p, q, partials, cg, s);
        return;
    }
    if (n % 8 != 0) {
        launch_apply_A(n, p, q, s);
        launch_cg_alpha(rb_count(n), p, q, partials, cg, s);
        return;
    }
    const dim3 grid = pair_grid(n);
    count_launch();
    k_apply_A_dot<<<grid, kThreads, 0, s>>>(n, p, q, partials);
    count_launch();
    k_alpha_finish<<<1, 1024, 0, s>>>(partials, int(grid.x * grid.y), cg);
}

void launch_cg_update(size_t count, float* e, float* r, const float* p, const float* q, const CgControl* cg,
                      ProjControl* ctrl, LoopCond recentre_cond, cudaStream_t s) {
    count_launch();
    const bool aligned = ((uintptr_t(e) | uintptr_t(r) | uintptr_t(p) | uintptr_t(q)) & 15u) == 0;
    if (count % 4 == 0 && aligned)
        k_cg_update4<<<blocks_for(count / 4), kThreads, 0, s>>>(count / 4, reinterpret_cast<float4*>(e),
                                                                 reinterpret_cast<float4*>(r),
                                                                 reinterpret_cast<const float4*>(p),
                                                                 reinterpret_cast<const float4*>(q), cg, ctrl);
    else
        k_cg_update<<<blocks_for(count), kThreads, 0, s>>>(count, e, r, p, q, cg, ctrl);
    count_launch();
    k_cg_decide<<<1, 1, 0, s>>>(ctrl, recentre_cond.active, (cudaGraphConditionalHandle)recentre_cond.handle);
}

void launch_cg_beta(size_t count, const float* z, const float* r, const float* q, double* partials, CgControl* cg,
                    cudaStream_t s) {
    const int blocks = blocks_for(count);
    count_launch();
    k_dot2<<<blocks, kThreads, 0, s>>>(count, z, r, z, q, partials);
    count_launch();
    k_beta_finish<<<1, 1024, 0, s>>>(partials, blocks, cg);
}

void launch_cg_beta_finish(const double* partials, int blocks, CgControl* cg, cudaStream_t s) {
    count_launch();
    k_beta_finish<<<1, 1024, 0, s>>>(partials, blocks, cg);
}

void launch_cg_direction(size_t count, float* p, const float* z, const CgControl* cg, cudaStream_t s) {
    count_launch();
    k_p_update<<<blocks_for(count), kThreads, 0, s>>>(count, p, z, cg);
}

void launch_cg_direction_apply(int n, const float* z, float* const* p, float* e, float* q, double* partials,
                               CgControl* cg, cudaStream_t s) {
    const dim3 grid = pair_grid(n);
    count_launch();
    k_direction_apply<<<grid, kThreads, 0, s>>>(n, z, p[0], p[1], e, q, cg, partials);
    count_launch();
    k_alpha_finish_pp<<<1, 1024, 0, s>>>(partials, int(grid.x * grid.y), cg);
}

void launch_cg_update_r(size_t count, float* r, const float* q, const CgControl* cg, ProjControl* ctrl,
                        LoopCond recentre_cond, cudaStream_t s) {
    count_launch();
    k_update_r4<<<blocks_for(count / 4), kThreads, 0, s>>>(count / 4, reinterpret_cast<float4*>(r),
                                                          reinterpret_cast<const float4*>(q), cg, ctrl);
    count_launch();
    k_cg_decide<<<1, 1, 0, s>>>(ctrl, recentre_cond.active, (cudaGraphConditionalHandle)recentre_cond.handle);
}

void launch_cg_fold(size_t count, float* e, float* const* p, CgControl* cg, const ProjControl* ctrl, cudaStream_t s) {
    count_launch();
    k_fold_pending<<<blocks_for(count / 4), kThreads, 0, s>>>(count / 4, reinterpret_cast<float4*>(e),
                                                             reinterpret_cast<const float4*>(p[0]),
                                                             reinterpret_cast<const float4*>(p[1]), cg, ctrl);
    count_launch();
    k_fold_clear<<<1, 1, 0, s>>>(cg, ctrl);
}

void launch_restrict_residual(int n, const float* r, const float* z, float* rows, float* rc, cudaStream_t s,
                              const uint8_t* diag) {
    const int nc = n / 4;
    count_launch();
    if (diag) k_restrict_rows_masked<<<blocks_for(size_t(n) * n * nc), kThreads, 0, s>>>(n, r, z, diag, rows);
    else if (n % 16 == 0) k_restrict_pairs<<<pair_grid(n), kThreads, 0, s>>>(n, r, z, rows);
    else k_restrict_rows<<<blocks_for(size_t(n) * n * nc), kThreads, 0, s>>>(n, r, z, rows);
    count_launch();
    k_restrict_blocks<<<blocks_for(size_t(nc) * nc * nc), kThreads, 0, s>>>(n, rows, rc);
}

void launch_log_coarse(const float* rc, size_t cells, float* log, int capacity, int* counter, cudaStream_t s) {
    count_launch();
    k_log_coarse<<<blocks_for(cells), kThreads, 0, s>>>(rc, cells, log, capacity, counter);
    count_launch();
    k_log_advance<<<1, 1, 0, s>>>(counter);
}

void launch_coarse_correction(int n, float* z, const float* zc, const float* rc, double* partials, CgControl* cg,
                              cudaStream_t s, const uint8_t* diag) {
    const int nc = n / 4;
    const size_t cells = size_t(nc) * nc * nc;
    const int blocks = blocks_for(cells);
    count_launch();
    k_coarse_sums<<<blocks, kThreads, 0, s>>>(nc, zc, rc, partials);
    count_launch();
    k_coarse_finish<<<1, 1024, 0, s>>>(partials, blocks, double(cells), cg);
    count_launch();
    if (diag) k_prolong_add_masked<<<blocks_for(rb_count(n)), kThreads, 0, s>>>(n, z, zc, diag, cg);
    else if (n % 16 == 0) k_prolong_pairs<<<pair_grid(n), kThreads, 0, s>>>(n, z, zc, cg);
    else k_prolong_add<<<blocks_for(rb_count(n)), kThreads, 0, s>>>(n, z, zc, cg);
}

}  // namespace vb
