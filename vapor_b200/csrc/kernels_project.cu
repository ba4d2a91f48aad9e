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
#include <map>
#include <mutex>

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

__global__ void k_begin_projection(ProjControl* ctrl, vapor_linear_solve_options o, double* x64a, double* x64b) {
    ctrl->x64[0] = x64a;
    ctrl->x64[1] = x64b;
    ctrl->x64_cur = 0;
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
    ctrl->recentre = 1;
    ctrl->r0 = 0.0;
    ctrl->res32_bits = 0u;
    ctrl->since = 0;
    vapor_projection_result r = {};
    ctrl->result = r;
}

// b = -div(walls(u)) * h^2/dt; walls read as zero, which equals enforcing the
// closed boundaries before computing the divergence.
__global__ void __launch_bounds__(kThreads) k_rhs(Grid g, float scale, const float* __restrict__ u,
                                                  const float* __restrict__ v, const float* __restrict__ w,
                                                  float* __restrict__ b, double* __restrict__ partials,
                                                  ProjControl* ctrl, const uint8_t* __restrict__ solid,
                                                  const float* __restrict__ field) {
    __shared__ double s_sum[32];
    __shared__ float s_max[32];
    __shared__ int s_key[32];
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const size_t cells = size_t(n) * n * n;
    double sum = 0.0;
    float div_max = 0.f;
    int kmax = INT_MIN, kmin = INT_MAX;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        if (solid && solid[c]) {  // not an unknown: b = 0, outside every reduction
            b[rb_index(L, x, y, z)] = 0.f;
            continue;
        }
        if (field) {  // a given right-hand side (natural layout) instead of a divergence
            const float rhs = field[c];
            if (!isfinite(rhs)) bad = 1u;
            b[rb_index(L, x, y, z)] = rhs;
            sum += double(rhs);
            const int key = float_order_key(rhs);
            kmax = max(kmax, key);
            kmin = min(kmin, key);
            continue;
        }
        // faces on walls or touching a solid are closed (read as zero)
        auto open = [&](int xx, int yy, int zz) { return !solid || !solid[(size_t(zz) * n + yy) * n + xx]; };
        const float u0 = (x == 0 || !open(x - 1, y, z)) ? 0.f : u[index_of(n, FACE_X, x, y, z)];
        const float u1 = (x + 1 == n || !open(x + 1, y, z)) ? 0.f : u[index_of(n, FACE_X, x + 1, y, z)];
        const float v0 = (y == 0 || !open(x, y - 1, z)) ? 0.f : v[index_of(n, FACE_Y, x, y, z)];
        const float v1 = (y + 1 == n || !open(x, y + 1, z)) ? 0.f : v[index_of(n, FACE_Y, x, y + 1, z)];
        const float w0 = (z == 0 || !open(x, y, z - 1)) ? 0.f : w[index_of(n, FACE_Z, x, y, z)];
        const float w1 = (z + 1 == n || !open(x, y, z + 1)) ? 0.f : w[index_of(n, FACE_Z, x, y, z + 1)];
        const float div = (u1 - u0 + v1 - v0 + w1 - w0) / g.h;
        if (!isfinite(div)) bad = 1u;
        div_max = maxf_ref(div_max, fabsf(div));
        const float rhs = -div * scale;
        b[rb_index(L, x, y, z)] = rhs;
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
                             double abs_tol, double rel_tol, int use_conditional,
                             cudaGraphConditionalHandle handle) {
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
    ctrl->continue_flag = !ctrl->done;
    if (use_conditional) cudaGraphSetConditional(handle, ctrl->done ? 0u : 1u);
}

// One colour of red-black SOR (SOR.cpp:36-54) on the split layout, in the
// reference's operation order: off = sum(-1 * x_nb) over existing neighbours in
// x-,x+,y-,y+,z-,z+ order; x += omega * (b - off - diag * x) / max(diag, floor).
// Each thread updates VEC consecutive slots of one row (VEC = 4 uses vector
// loads and needs hw % 4 == 0). The x-neighbours of slot i are the other
// colour's slots i-1+s and i+s (s = (y+z+colour)&1, x = 2i+s); the y- and
// z-neighbours are slot i of the adjacent rows of the other colour.
// EXACT = false is the mixed solver's inner sweep: the relaxation is a
// multiplication by wr[diag] = omega / max(diag, floor) (FP32, from the host)
// instead of omega * t / max(diag, floor); the oracle's refinement uses the
// same formula.
struct RelaxTable {
    float w[7];
};
template <int VEC, bool EXACT>
__global__ void __launch_bounds__(kThreads) k_sor_rb(Grid g, int colour, float omega, float floor_diag,
                                                     RelaxTable wr, float* __restrict__ xs,
                                                     const float* __restrict__ bs,
                                                     const ProjControl* __restrict__ ctrl, int guarded,
                                                     int sweep_index, int subtract_mean,
                                                     const uint8_t* __restrict__ diag_arr) {
    if (guarded && (ctrl->done || ctrl->iterations + sweep_index >= ctrl->max_iterations)) return;
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const int hw = L.hw;
    const int groups = hw / VEC;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    const int y = t / groups;
    if (y >= n) return;
    const int i0 = (t - y * groups) * VEC;
    const int s = (y + z + colour) & 1;
    const size_t row = (size_t(z) * n + y) * hw;
    float* __restrict__ own = xs + size_t(colour) * L.stride + row;
    const float* __restrict__ oth = xs + size_t(1 - colour) * L.stride + row;
    const float* __restrict__ rhs = bs + size_t(colour) * L.stride + row;
    const float bm = subtract_mean ? ctrl->rhs_mean_f : 0.f;

    float xo[VEC], bv[VEC], xl[VEC + 1], ym[VEC], yp[VEC], zm[VEC], zp[VEC];
    const size_t yo = size_t(hw), zo = size_t(n) * hw;
    if (VEC == 4) {
        const float4 a4 = *reinterpret_cast<const float4*>(own + i0);
        const float4 b4 = __ldg(reinterpret_cast<const float4*>(rhs + i0));
        const float4 c4 = *reinterpret_cast<const float4*>(oth + i0);
        xo[0] = a4.x; xo[1] = a4.y; xo[2] = a4.z; xo[3] = a4.w;
        bv[0] = b4.x; bv[1] = b4.y; bv[2] = b4.z; bv[3] = b4.w;
        // xl[k] = other-colour slot i0 - 1 + s + k, k = 0..VEC
        if (s == 0) {
            xl[0] = i0 > 0 ? oth[i0 - 1] : 0.f;
            xl[1] = c4.x; xl[2] = c4.y; xl[3] = c4.z; xl[4] = c4.w;
        } else {
            xl[0] = c4.x; xl[1] = c4.y; xl[2] = c4.z; xl[3] = c4.w;
            xl[4] = i0 + VEC < hw ? oth[i0 + VEC] : 0.f;
        }
        const float4 z0 = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 m4 = y > 0 ? *reinterpret_cast<const float4*>(oth - yo + i0) : z0;
        const float4 p4 = y + 1 < n ? *reinterpret_cast<const float4*>(oth + yo + i0) : z0;
        const float4 q4 = z > 0 ? *reinterpret_cast<const float4*>(oth - zo + i0) : z0;
        const float4 r4 = z + 1 < n ? *reinterpret_cast<const float4*>(oth + zo + i0) : z0;
        ym[0] = m4.x; ym[1] = m4.y; ym[2] = m4.z; ym[3] = m4.w;
        yp[0] = p4.x; yp[1] = p4.y; yp[2] = p4.z; yp[3] = p4.w;
        zm[0] = q4.x; zm[1] = q4.y; zm[2] = q4.z; zm[3] = q4.w;
        zp[0] = r4.x; zp[1] = r4.y; zp[2] = r4.z; zp[3] = r4.w;
    } else {
        xo[0] = own[i0];
        bv[0] = __ldg(rhs + i0);
        const int lo = i0 - 1 + s;
        xl[0] = lo >= 0 ? oth[lo] : 0.f;
        xl[1] = lo + 1 < hw ? oth[lo + 1] : 0.f;
        ym[0] = y > 0 ? oth[i0 - yo] : 0.f;
        yp[0] = y + 1 < n ? oth[i0 + yo] : 0.f;
        zm[0] = z > 0 ? oth[i0 - zo] : 0.f;
        zp[0] = z + 1 < n ? oth[i0 + zo] : 0.f;
    }
    const int ny = (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
    float res[VEC];
#pragma unroll
    for (int k = 0; k < VEC; ++k) {
        const int xc = 2 * (i0 + k) + s;
        res[k] = xo[k];
        if (xc >= n) continue;
        const float diag = diag_arr ? float(diag_arr[size_t(colour) * L.stride + row + i0 + k])
                                    : float((xc > 0) + (xc + 1 < n) + ny);
        if (diag == 0.f) continue;
        float off = 0.f;
        if (xc > 0) off += -1.f * xl[k];
        if (xc + 1 < n) off += -1.f * xl[k + 1];
        if (y > 0) off += -1.f * ym[k];
        if (y + 1 < n) off += -1.f * yp[k];
        if (z > 0) off += -1.f * zm[k];
        if (z + 1 < n) off += -1.f * zp[k];
        const float bi = subtract_mean ? bv[k] - bm : bv[k];
        if (EXACT) {
            const float relax = maxf_ref(diag, floor_diag);
            res[k] = xo[k] + omega * (bi - off - diag * xo[k]) / relax;
        } else {
            res[k] = xo[k] + (bi - off - diag * xo[k]) * wr.w[int(diag)];
        }
    }
    if (VEC == 4) {
        *reinterpret_cast<float4*>(own + i0) = make_float4(res[0], res[1], res[2], res[3]);
    } else {
        if (2 * i0 + s < n) own[i0] = res[0];
    }
}

// The same colour sweep marching in z: each thread owns 4 consecutive slots
// of one row (y) for zb consecutive planes and keeps the other colour's rows
// of planes z-1, z, z+1 in registers, so a plane costs 5 vector loads (own,
// rhs, other colour at z+1, y-1, y+1) instead of 7, and the index arithmetic
// is 32-bit and amortised over the column. Missing neighbours read as zero,
// which leaves the reference's sum unchanged (x + (-1 * 0) == x bitwise for
// every x, including signed zeros), so results equal k_sor_rb's bit for bit.
// Needs hw % 4 == 0 and 2 * n^2 * hw < 2^31.
// FROM_ZERO: the sweep starts from x = 0 (both colours): the other colour is
// not read but written as 0, and the own colour is not read (0 + (b - 0 -
// d * 0) * w == 0 + b * w). Replaces clearing x and the first colour sweep.
// PLAIN: no solid mask and n even (selected by the launcher), which allows
// the interior-x form of the update below.
// DOT (with PLAIN; the FPCG preconditioner's last sweep): also FP64 block
// partials of z.r and z.q over both colours, where z is the iterate after
// this sweep, r = b and q a further vector (2 values per block at
// partials[2 * block]); the other colour's z is the row this thread already
// holds, so the dot products cost three more vector loads per plane.
template <bool EXACT, bool RESID, bool FROM_ZERO = false, bool PLAIN = false, bool DOT = false>
__global__ void __launch_bounds__(kThreads, (RESID || DOT) ? 4 : 5) k_sor_rbz(Grid g, int colour, float omega, float floor_diag,
                                                      RelaxTable wr, float* __restrict__ xs,
                                                      const float* __restrict__ bs, ProjControl* ctrl,
                                                      int guarded, int sweep_index, int subtract_mean, int zb,
                                                      const uint8_t* __restrict__ diag,
                                                      const float* __restrict__ qs = nullptr,
                                                      double* __restrict__ partials = nullptr) {
    if (guarded && (ctrl->done || ctrl->iterations + sweep_index >= ctrl->max_iterations)) return;
    const int n = g.n;
    const int hw = (n + 1) >> 1;
    const int groups = hw >> 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = t / groups;
    float rmax = 0.f;
    double dzr = 0.0, dzq = 0.0;
    if (y < n) {
        const int i0 = (t - y * groups) << 2;
        const int plane = n * hw;
        const int stride = n * plane;
        float* __restrict__ own = xs + colour * stride + y * hw + i0;
        const float* __restrict__ oth = xs + (1 - colour) * stride + y * hw + i0;
        const float* __restrict__ rhs = bs + colour * stride + y * hw + i0;
        const float* __restrict__ rhs_o = bs + (1 - colour) * stride + y * hw + i0;
        const float* __restrict__ q_own = DOT ? qs + colour * stride + y * hw + i0 : nullptr;
        const float* __restrict__ q_oth = DOT ? qs + (1 - colour) * stride + y * hw + i0 : nullptr;
        const uint8_t* __restrict__ dg = diag ? diag + colour * stride + y * hw + i0 : nullptr;
        const float bm = subtract_mean ? ctrl->rhs_mean_f : 0.f;
        const int z0 = blockIdx.y * zb;
        const int z1 = min(n, z0 + zb);
        const bool has_ym = y > 0, has_yp = y + 1 < n;
        const int nyz = int(has_ym) + int(has_yp);
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        auto ld4 = [](const float* p) { return *reinterpret_cast<const float4*>(p); };
        float4 cm = (!FROM_ZERO && z0 > 0) ? ld4(oth + (z0 - 1) * plane) : zero4;
        float4 cc = FROM_ZERO ? zero4 : ld4(oth + z0 * plane);
        const float w3 = wr.w[3], w4 = wr.w[4], w5 = wr.w[5], w6 = wr.w[6];
        for (int z = z0; z < z1; ++z) {
            const int zoff = z * plane;
            const float4 cp = (!FROM_ZERO && z + 1 < n) ? ld4(oth + zoff + plane) : zero4;
            const float4 m4 = (!FROM_ZERO && has_ym) ? ld4(oth + zoff - hw) : zero4;
            const float4 p4 = (!FROM_ZERO && has_yp) ? ld4(oth + zoff + hw) : zero4;
            const float4 a4 = FROM_ZERO ? zero4 : ld4(own + zoff);
            if (FROM_ZERO) *reinterpret_cast<float4*>(const_cast<float*>(oth) + zoff) = zero4;
            const float4 b4 = __ldg(reinterpret_cast<const float4*>(rhs + zoff));
            const int sh = (y + z + colour) & 1;
            float xl[5];
            if (FROM_ZERO) {
#pragma unroll
                for (int k = 0; k < 5; ++k) xl[k] = 0.f;
            } else if (sh == 0) {
                xl[0] = i0 > 0 ? oth[zoff - 1] : 0.f;
                xl[1] = cc.x; xl[2] = cc.y; xl[3] = cc.z; xl[4] = cc.w;
            } else {
                xl[0] = cc.x; xl[1] = cc.y; xl[2] = cc.z; xl[3] = cc.w;
                xl[4] = i0 + 4 < hw ? oth[zoff + 4] : 0.f;
            }
            const float xo[4] = {a4.x, a4.y, a4.z, a4.w};
            const float bv[4] = {b4.x, b4.y, b4.z, b4.w};
            const float ym[4] = {m4.x, m4.y, m4.z, m4.w};
            const float yp[4] = {p4.x, p4.y, p4.z, p4.w};
            const float zm[4] = {cm.x, cm.y, cm.z, cm.w};
            const float zp[4] = {cp.x, cp.y, cp.z, cp.w};
            const int ny = nyz + int(z > 0) + int(z + 1 < n);
            float res[4];
            if (PLAIN) {
                // No mask, n even: every slot is a cell, the neighbours outside
                // the box were loaded as 0 (adding -1 * 0 leaves the sum's bits
                // unchanged), and only cell 0 at x = 0 and cell 3 at x = n - 1
                // have one x-neighbour less. Same operations as the general path.
                // ny is 2, 3 or 4 (n >= 8): diagonals and weights by selection,
                // no int-to-float conversion and no indexed parameter access
                const float diag0 = ny == 4 ? 6.f : (ny == 3 ? 5.f : 4.f), diag1 = diag0 - 1.f;
                const float w0 = EXACT ? maxf_ref(diag0, floor_diag) : (ny == 4 ? w6 : (ny == 3 ? w5 : w4));
                const float w1 = EXACT ? maxf_ref(diag1, floor_diag) : (ny == 4 ? w5 : (ny == 3 ? w4 : w3));
                const bool ledge = i0 == 0 && sh == 0, redge = i0 + 4 >= hw && sh == 1;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const bool edge = (k == 0 && ledge) || (k == 3 && redge);
                    const float diag = edge ? diag1 : diag0;
                    float off = 0.f;
                    off += -1.f * xl[k];
                    off += -1.f * xl[k + 1];
                    off += -1.f * ym[k];
                    off += -1.f * yp[k];
                    off += -1.f * zm[k];
                    off += -1.f * zp[k];
                    const float bi = subtract_mean ? bv[k] - bm : bv[k];
                    float r;
                    if (EXACT) r = xo[k] + omega * (bi - off - diag * xo[k]) / (edge ? w1 : w0);
                    else r = xo[k] + (bi - off - diag * xo[k]) * (edge ? w1 : w0);
                    res[k] = r;
                    if (RESID) {
                        const float rr = bi - off - diag * r;
                        rmax = fmaxf(rmax, fabsf(rr));
                    }
                }
                if (DOT) {
                    const float4 ro = __ldg(reinterpret_cast<const float4*>(rhs_o + zoff));
                    const float4 qa = __ldg(reinterpret_cast<const float4*>(q_own + zoff));
                    const float4 qb = __ldg(reinterpret_cast<const float4*>(q_oth + zoff));
                    const float zo[4] = {cc.x, cc.y, cc.z, cc.w}, rv[4] = {ro.x, ro.y, ro.z, ro.w};
                    const float qv[4] = {qa.x, qa.y, qa.z, qa.w}, qw[4] = {qb.x, qb.y, qb.z, qb.w};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        dzr += double(res[k]) * double(bv[k]) + double(zo[k]) * double(rv[k]);
                        dzq += double(res[k]) * double(qv[k]) + double(zo[k]) * double(qw[k]);
                    }
                }
            } else {  // general form: any n, optional solid mask
                uchar4 dm = make_uchar4(0, 0, 0, 0);
                if (dg) dm = *reinterpret_cast<const uchar4*>(dg + zoff);
                const int dmask[4] = {dm.x, dm.y, dm.z, dm.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int xc = 2 * (i0 + k) + sh;
                    const bool left = xc > 0, right = xc + 1 < n;
                    // solid neighbours hold 0, so summing them changes nothing
                    const int d = dg ? dmask[k] : int(left) + int(right) + ny;
                    const float diag = float(d);
                    float off = 0.f;
                    off += -1.f * (left ? xl[k] : 0.f);
                    off += -1.f * (right ? xl[k + 1] : 0.f);
                    off += -1.f * ym[k];
                    off += -1.f * yp[k];
                    off += -1.f * zm[k];
                    off += -1.f * zp[k];
                    const float bi = subtract_mean ? bv[k] - bm : bv[k];
                    float r;
                    if (EXACT) {
                        const float relax = maxf_ref(diag, floor_diag);
                        r = xo[k] + omega * (bi - off - diag * xo[k]) / relax;
                    } else {
                        const float w = d == 6 ? w6 : (d == 5 ? w5 : (d == 4 ? w4 : w3));
                        r = xo[k] + (bi - off - diag * xo[k]) * w;
                    }
                    const bool valid = xc < n && d > 0;
                    res[k] = valid ? r : xo[k];
                    if (RESID && valid) {
                        // residual of this cell after its update: the other
                        // colour (all its neighbours) does not change in this sweep
                        const float rr = bi - off - diag * r;
                        rmax = fmaxf(rmax, fabsf(rr));
                    }
                }
            }
            *reinterpret_cast<float4*>(own + zoff) = make_float4(res[0], res[1], res[2], res[3]);
            cm = cc;
            cc = cp;
        }
    }
    if (RESID) {
        __shared__ float s_max[32];
        const float br = block_max(rmax, s_max);
        if (threadIdx.x == 0 && br > 0.f) atomicMax(&ctrl->res32_bits, __float_as_uint(br));
    }
    if (DOT) {
        __shared__ double s_sum[32];
        const double a = block_sum(dzr, s_sum);
        const double b = block_sum(dzq, s_sum);
        if (threadIdx.x == 0) {
            const int blk = blockIdx.y * gridDim.x + blockIdx.x;
            partials[2 * blk] = a;
            partials[2 * blk + 1] = b;
        }
    }
}

// Mixed precision re-centring on the split layout: x_out = x_in + e and
// r32 = float(b' - A x_out), both in FP64 with the neighbour order of the
// reference residual. One thread per VEC consecutive slots of one row of one
// colour (blockIdx.z); neighbours are the other colour's x_in + e.
template <int VEC>
__global__ void __launch_bounds__(kThreads) k_refine_rb(Grid g, const float* __restrict__ bs,
                                                        const float* __restrict__ es, float* __restrict__ r32,
                                                        ProjControl* ctrl, int gated,
                                                        const uint8_t* __restrict__ diag) {
    __shared__ double s_max[32];
    if (gated && !ctrl->recentre) return;
    const double* __restrict__ xin = ctrl->x64[ctrl->x64_cur];
    double* __restrict__ xout = ctrl->x64[1 - ctrl->x64_cur];
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const int hw = L.hw, groups = hw / VEC;
    const int colour = blockIdx.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    const int y = t / groups;
    const bool active = y < n;
    const float bm = ctrl->rhs_mean_f;
    double rmax = 0.0;
    unsigned int bad = 0u;
    if (active) {
        const int i0 = (t - y * groups) * VEC;
        const int s = (y + z + colour) & 1;
        const size_t row = (size_t(z) * n + y) * hw;
        const size_t own = size_t(colour) * L.stride + row, oth = size_t(1 - colour) * L.stride + row;
        const size_t yo = size_t(hw), zo = size_t(n) * hw;
        auto nb = [&](size_t idx) { return xin[oth + idx] + double(es[oth + idx]); };
        double xo[VEC], xl[VEC + 1], ym[VEC], yp[VEC], zm[VEC], zp[VEC];
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
            xo[k] = xin[own + i0 + k] + double(es[own + i0 + k]);
            ym[k] = y > 0 ? nb(i0 + k - yo) : 0.0;
            yp[k] = y + 1 < n ? nb(i0 + k + yo) : 0.0;
            zm[k] = z > 0 ? nb(i0 + k - zo) : 0.0;
            zp[k] = z + 1 < n ? nb(i0 + k + zo) : 0.0;
        }
#pragma unroll
        for (int k = 0; k <= VEC; ++k) {
            const int slot = i0 - 1 + s + k;
            xl[k] = (slot >= 0 && slot < hw) ? nb(size_t(slot)) : 0.0;
        }
        const int ny = (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
            const int xc = 2 * (i0 + k) + s;
            if (xc >= n) continue;
            const int dcell = diag ? int(diag[own + i0 + k]) : (xc > 0) + (xc + 1 < n) + ny;
            if (diag && dcell == 0) {  // solid cell: not an unknown
                xout[own + i0 + k] = xo[k];
                r32[own + i0 + k] = 0.f;
                continue;
            }
            double ax = double(dcell) * xo[k];
            if (xc > 0) ax -= xl[k];
            if (xc + 1 < n) ax -= xl[k + 1];
            if (y > 0) ax -= ym[k];
            if (y + 1 < n) ax -= yp[k];
            if (z > 0) ax -= zm[k];
            if (z + 1 < n) ax -= zp[k];
            const float bi = bs[own + i0 + k] - bm;
            const double res = double(bi) - ax;
            if (!isfinite(res)) bad = 1u;
            xout[own + i0 + k] = xo[k];
            r32[own + i0 + k] = float(res);
            const double aa = fabs(res);
            rmax = rmax < aa ? aa : rmax;
        }
    }
    const double br = block_max(rmax, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->res_bits, br);
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

// FP32 residual of the mixed solver's error equation, max |r32 - A e| over
// the colour-1 cells (the colour a sweep updates last), with A the Neumann
// operator (neighbour-count diagonal) and the operations in the sweep's order:
// (r32 - off) - count * e with off = sum of -1 * e_nb in x-, x+, y-, y+, z-,
// z+ order. Same value as the fused measurement of k_sor_rbz<*, true>; used
// when that kernel does not apply (hw % 4 != 0).
template <int VEC>
__global__ void __launch_bounds__(kThreads) k_error_residual(Grid g, const float* __restrict__ es,
                                                             const float* __restrict__ r32, ProjControl* ctrl,
                                                             int first_colour, const uint8_t* __restrict__ diag) {
    __shared__ float s_max[32];
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const int hw = L.hw, groups = hw / VEC;
    const int colour = first_colour + blockIdx.z;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.y;
    const int y = t / groups;
    float rmax = 0.f;
    unsigned int bad = 0u;
    if (y < n) {
        const int i0 = (t - y * groups) * VEC;
        const int s = (y + z + colour) & 1;
        const size_t row = (size_t(z) * n + y) * hw;
        const size_t own = size_t(colour) * L.stride + row, oth = size_t(1 - colour) * L.stride + row;
        const size_t yo = size_t(hw), zo = size_t(n) * hw;
        float xo[VEC], xl[VEC + 1], ym[VEC], yp[VEC], zm[VEC], zp[VEC];
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
            xo[k] = es[own + i0 + k];
            ym[k] = y > 0 ? es[oth + i0 + k - yo] : 0.f;
            yp[k] = y + 1 < n ? es[oth + i0 + k + yo] : 0.f;
            zm[k] = z > 0 ? es[oth + i0 + k - zo] : 0.f;
            zp[k] = z + 1 < n ? es[oth + i0 + k + zo] : 0.f;
        }
#pragma unroll
        for (int k = 0; k <= VEC; ++k) {
            const int slot = i0 - 1 + s + k;
            xl[k] = (slot >= 0 && slot < hw) ? es[oth + slot] : 0.f;
        }
        const int ny = (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
#pragma unroll
        for (int k = 0; k < VEC; ++k) {
            const int xc = 2 * (i0 + k) + s;
            if (xc >= n) continue;
            const int dcell = diag ? int(diag[own + i0 + k]) : (xc > 0) + (xc + 1 < n) + ny;
            if (dcell == 0) continue;
            const float dg = float(dcell);
            float off = 0.f;
            if (xc > 0) off += -1.f * xl[k];
            if (xc + 1 < n) off += -1.f * xl[k + 1];
            if (y > 0) off += -1.f * ym[k];
            if (y + 1 < n) off += -1.f * yp[k];
            if (z > 0) off += -1.f * zm[k];
            if (z + 1 < n) off += -1.f * zp[k];
            const float res = r32[own + i0 + k] - off - dg * xo[k];
            if (!isfinite(res)) bad = 1u;
            const float aa = fabsf(res);
            rmax = rmax < aa ? aa : rmax;
        }
    }
    const float br = block_max(rmax, s_max);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        atomicMax(&ctrl->res32_bits, __float_as_uint(br));
        if (any_bad) atomicOr(&ctrl->nonfinite, 4u);
    }
}

__global__ void k_error_decide(ProjControl* ctrl, int sweeps, int use_conditional,
                               cudaGraphConditionalHandle handle, int use_if, cudaGraphConditionalHandle if_handle) {
    ctrl->iterations = min(ctrl->iterations + sweeps, ctrl->max_iterations);
    ctrl->since += sweeps;
    const float rho = __uint_as_float(ctrl->res32_bits);
    ctrl->res32_bits = 0u;
    const int recentre = double(rho) <= ctrl->target || double(rho) <= double(kRecentreDrop) * ctrl->r0 ||
                         ctrl->since >= kRecentreSweeps || ctrl->iterations >= ctrl->max_iterations ||
                         (ctrl->nonfinite & 4u) != 0u;
    ctrl->recentre = recentre;
    if (use_if) cudaGraphSetConditional(if_handle, recentre ? 1u : 0u);
    ctrl->result.linear_solve.iterations = ctrl->iterations;
    if (!recentre) {
        ctrl->done = 0;
        ctrl->continue_flag = 1;
        if (use_conditional) cudaGraphSetConditional(handle, 1u);
    }
}

// e = 0 over both colours after a re-centring (e is the next correction).
__global__ void k_zero_error_gated(float* __restrict__ e, size_t count, const ProjControl* __restrict__ ctrl) {
    if (!ctrl->recentre) return;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += size_t(gridDim.x) * blockDim.x)
        e[i] = 0.f;
}

__global__ void __launch_bounds__(kThreads) k_psum64(Grid g, const ProjControl* __restrict__ ctrl,
                                                     double* __restrict__ partials) {
    __shared__ double s_sum[32];
    const double* __restrict__ x = ctrl->x64[ctrl->x64_cur];
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const size_t cells = size_t(n) * n * n;
    double sum = 0.0;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        sum += x[rb_index(L, i, j, k)];
    }
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
// the float pressure copy (split layout).
__global__ void __launch_bounds__(kThreads) k_residual64(Grid g, const float* __restrict__ b,
                                                         float* __restrict__ p32, ProjControl* ctrl,
                                                         const uint8_t* __restrict__ diag) {
    __shared__ double s_max[32];
    const double* __restrict__ x = ctrl->x64[ctrl->x64_cur];
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const size_t cells = size_t(n) * n * n;
    const float bm = ctrl->rhs_mean_f;
    const double pm = ctrl->p_mean64;
    double r = 0.0;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        const size_t me = rb_index(L, i, j, k);
        if (diag && diag[me] == 0) {  // solid cell: pressure 0, no residual
            p32[me] = 0.f;
            continue;
        }
        // solid neighbours enter as 0 (their x64 is 0 and is not shifted)
        auto xv = [&](int a, int bb, int cc) {
            const size_t id = rb_index(L, a, bb, cc);
            return (diag && diag[id] == 0) ? 0.0 : x[id] - pm;
        };
        const double xc = x[me] - pm;
        const int dcell = diag ? int(diag[me]) : neighbours(n, i, j, k);
        double ax = double(float(dcell)) * xc;
        if (i > 0) ax += -1.0 * xv(i - 1, j, k);
        if (i + 1 < n) ax += -1.0 * xv(i + 1, j, k);
        if (j > 0) ax += -1.0 * xv(i, j - 1, k);
        if (j + 1 < n) ax += -1.0 * xv(i, j + 1, k);
        if (k > 0) ax += -1.0 * xv(i, j, k - 1);
        if (k + 1 < n) ax += -1.0 * xv(i, j, k + 1);
        const float bi = b[me] - bm;
        if (!isfinite(xc)) bad = 1u;
        p32[me] = float(xc);
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
__global__ void __launch_bounds__(kThreads) k_gradient64(Grid g, float dt,
                                                         const float* __restrict__ u, const float* __restrict__ v,
                                                         const float* __restrict__ w, float* __restrict__ uo,
                                                         float* __restrict__ vo, float* __restrict__ wo,
                                                         float* __restrict__ uh, float* __restrict__ vh,
                                                         float* __restrict__ wh, ProjControl* ctrl,
                                                         const uint8_t* __restrict__ solid) {
    __shared__ float s_max[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const size_t nn = size_t(n) * n;
    const double hInv = 1.0 / double(g.h), dtd = double(dt);
    const double pm = ctrl->p_mean64;
    const double* __restrict__ p = ctrl->x64[ctrl->x64_cur];
    const RBLayout L = rb_layout(n);
    float div_max = 0.f;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        auto pv = [&](int a, int bb, int cc) { return p[rb_index(L, a, bb, cc)] - pm; };
        const double pc = pv(x, y, z);
        const size_t ix0 = index_of(n, FACE_X, x, y, z), ix1 = ix0 + 1;
        const size_t iy0 = index_of(n, FACE_Y, x, y, z), iy1 = iy0 + n;
        const size_t iz0 = c, iz1 = c + nn;
        // faces on walls or touching a solid cell are closed
        const bool me_solid = solid && solid[c];
        auto shut = [&](int xx, int yy, int zz) { return me_solid || (solid && solid[(size_t(zz) * n + yy) * n + xx]); };
        const float ux0 = (x == 0 || shut(x - 1, y, z)) ? 0.f : float(double(u[ix0]) - dtd * (pc - pv(x - 1, y, z)) * hInv);
        const float ux1 = (x + 1 == n || shut(x + 1, y, z)) ? 0.f : float(double(u[ix1]) - dtd * (pv(x + 1, y, z) - pc) * hInv);
        const float vy0 = (y == 0 || shut(x, y - 1, z)) ? 0.f : float(double(v[iy0]) - dtd * (pc - pv(x, y - 1, z)) * hInv);
        const float vy1 = (y + 1 == n || shut(x, y + 1, z)) ? 0.f : float(double(v[iy1]) - dtd * (pv(x, y + 1, z) - pc) * hInv);
        const float wz0 = (z == 0 || shut(x, y, z - 1)) ? 0.f : float(double(w[iz0]) - dtd * (pc - pv(x, y, z - 1)) * hInv);
        const float wz1 = (z + 1 == n || shut(x, y, z + 1)) ? 0.f : float(double(w[iz1]) - dtd * (pv(x, y, z + 1) - pc) * hInv);
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

// The two FP64 passes that end a mixed-precision or FPCG projection, fused
// for unmasked grids with n % 4 == 0: the final residual of x64 - mean
// (k_residual64: same neighbour order, missing neighbours contribute -1 * 0,
// which leaves the FP64 sum's bits unchanged), the float pressure copy, and
// the gradient step with walls, reflection hat and divergence after
// (k_gradient64: same expressions). One thread owns 4 consecutive cells of a
// row (2 slots of each colour of the split layout) for zb consecutive planes
// and marches up z keeping the pressure rows of planes z - 1, z, z + 1 in
// registers, so x64 is read once from DRAM and every access is a 16-byte
// vector load except the row-end neighbours and the x faces.
__global__ void __launch_bounds__(kThreads) k_finish64(Grid g, float dt, const float* __restrict__ b,
                                                       float* __restrict__ p32, ProjControl* ctrl,
                                                       const float* __restrict__ u, const float* __restrict__ v,
                                                       const float* __restrict__ w, float* __restrict__ uo,
                                                       float* __restrict__ vo, float* __restrict__ wo,
                                                       float* __restrict__ uh, float* __restrict__ vh,
                                                       float* __restrict__ wh, int zb) {
    __shared__ double s_res[32];
    __shared__ float s_div[32];
    const int n = g.n;
    const int hw = n >> 1, groups = n >> 2;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = t / groups;
    double rmax = 0.0;
    float dmax = 0.f;
    unsigned int bad_solve = 0u, bad_div = 0u;
    if (y < n) {
        const int j = t - y * groups;
        const int x0 = 4 * j;
        const double* __restrict__ X = ctrl->x64[ctrl->x64_cur];
        const double pm = ctrl->p_mean64;
        const float bm = ctrl->rhs_mean_f;
        const double hInv = 1.0 / double(g.h), dtd = double(dt);
        const size_t stride = size_t(n) * n * hw;  // values per colour
        // natural-order cells x0 .. x0 + 3 of row (yy, zz) minus the mean:
        // slots 2j, 2j + 1 of colour (yy + zz) & 1 hold x0, x0 + 2, those of
        // the other colour x0 + 1, x0 + 3
        auto row = [&](int yy, int zz, double (&o)[4]) {
            const size_t base = (size_t(zz) * n + yy) * hw + 2 * j;
            const int c0 = (yy + zz) & 1;
            const double2 A = *reinterpret_cast<const double2*>(X + size_t(c0) * stride + base);
            const double2 B = *reinterpret_cast<const double2*>(X + size_t(1 - c0) * stride + base);
            o[0] = A.x - pm;
            o[1] = B.x - pm;
            o[2] = A.y - pm;
            o[3] = B.y - pm;
        };
        const int z0 = blockIdx.y * zb, z1 = min(n, z0 + zb);
        double zm[4] = {0.0, 0.0, 0.0, 0.0}, zc[4], zp[4];
        if (z0 > 0) row(y, z0 - 1, zm);
        row(y, z0, zc);
        const size_t nn = size_t(n) * n;
        for (int z = z0; z < z1; ++z) {
            if (z + 1 < n) row(y, z + 1, zp);
            double ym[4] = {0.0, 0.0, 0.0, 0.0}, yp[4] = {0.0, 0.0, 0.0, 0.0};
            if (y > 0) row(y - 1, z, ym);
            if (y + 1 < n) row(y + 1, z, yp);
            const size_t rb = (size_t(z) * n + y) * hw + 2 * j;
            const int c0 = (y + z) & 1;
            // row-end neighbours: x0 - 1 (odd, the colour of x0 + 1) and
            // x0 + 4 (even, the colour of x0)
            const double left = x0 > 0 ? X[size_t(1 - c0) * stride + rb - 1] - pm : 0.0;
            const double right = x0 + 4 < n ? X[size_t(c0) * stride + rb + 2] - pm : 0.0;
            const float2 bA = *reinterpret_cast<const float2*>(b + size_t(c0) * stride + rb);
            const float2 bB = *reinterpret_cast<const float2*>(b + size_t(1 - c0) * stride + rb);
            const float bv[4] = {bA.x, bB.x, bA.y, bB.y};
            const double xl[6] = {left, zc[0], zc[1], zc[2], zc[3], right};  // cells x0 - 1 .. x0 + 4
            const size_t ix0 = size_t(n + 1) * (size_t(y) + size_t(n) * z) + x0;
            const size_t iy0 = size_t(n) * (size_t(y) + size_t(n + 1) * z) + x0;
            const size_t iz0 = nn * z + size_t(y) * n + x0;
            float uin[5];
#pragma unroll
            for (int k = 0; k < 5; ++k) uin[k] = u[ix0 + k];
            const float4 v0 = *reinterpret_cast<const float4*>(v + iy0);
            const float4 v1 = *reinterpret_cast<const float4*>(v + iy0 + n);
            const float4 w0 = *reinterpret_cast<const float4*>(w + iz0);
            const float4 w1 = *reinterpret_cast<const float4*>(w + iz0 + nn);
            const float vin0[4] = {v0.x, v0.y, v0.z, v0.w}, vin1[4] = {v1.x, v1.y, v1.z, v1.w};
            const float win0[4] = {w0.x, w0.y, w0.z, w0.w}, win1[4] = {w1.x, w1.y, w1.z, w1.w};
            float p32v[4], ux0[4], ux1[4], vy0[4], vy1[4], wz0[4], wz1[4];
            const int nyz = int(y > 0) + int(y + 1 < n) + int(z > 0) + int(z + 1 < n);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int x = x0 + k;
                const double pc = zc[k];
                // residual, neighbour order x-1, x+1, y-1, y+1, z-1, z+1
                const int dcell = int(x > 0) + int(x + 1 < n) + nyz;
                double ax = double(float(dcell)) * pc;
                if (x > 0) ax += -1.0 * xl[k];
                if (x + 1 < n) ax += -1.0 * xl[k + 2];
                if (y > 0) ax += -1.0 * ym[k];
                if (y + 1 < n) ax += -1.0 * yp[k];
                if (z > 0) ax += -1.0 * zm[k];
                if (z + 1 < n) ax += -1.0 * zp[k];
                const float bi = bv[k] - bm;
                if (!isfinite(pc)) bad_solve = 1u;
                p32v[k] = float(pc);
                const double a = fabs(double(bi) - ax);
                rmax = rmax < a ? a : rmax;
                // gradient, walls closed
                ux0[k] = x == 0 ? 0.f : float(double(uin[k]) - dtd * (pc - xl[k]) * hInv);
                ux1[k] = x + 1 == n ? 0.f : float(double(uin[k + 1]) - dtd * (xl[k + 2] - pc) * hInv);
                vy0[k] = y == 0 ? 0.f : float(double(vin0[k]) - dtd * (pc - ym[k]) * hInv);
                vy1[k] = y + 1 == n ? 0.f : float(double(vin1[k]) - dtd * (yp[k] - pc) * hInv);
                wz0[k] = z == 0 ? 0.f : float(double(win0[k]) - dtd * (pc - zm[k]) * hInv);
                wz1[k] = z + 1 == n ? 0.f : float(double(win1[k]) - dtd * (zp[k] - pc) * hInv);
                const float div = (ux1[k] - ux0[k] + vy1[k] - vy0[k] + wz1[k] - wz0[k]) / g.h;
                if (!isfinite(div)) bad_div = 1u;
                dmax = maxf_ref(dmax, fabsf(div));
            }
            *reinterpret_cast<float2*>(p32 + size_t(c0) * stride + rb) = make_float2(p32v[0], p32v[2]);
            *reinterpret_cast<float2*>(p32 + size_t(1 - c0) * stride + rb) = make_float2(p32v[1], p32v[3]);
#pragma unroll
            for (int k = 0; k < 4; ++k) uo[ix0 + k] = ux0[k];
            *reinterpret_cast<float4*>(vo + iy0) = make_float4(vy0[0], vy0[1], vy0[2], vy0[3]);
            *reinterpret_cast<float4*>(wo + iz0) = make_float4(wz0[0], wz0[1], wz0[2], wz0[3]);
            const bool xwall = x0 + 4 == n, ywall = y + 1 == n, zwall = z + 1 == n;
            if (xwall) uo[ix0 + 4] = ux1[3];
            if (ywall) *reinterpret_cast<float4*>(vo + iy0 + n) = make_float4(vy1[0], vy1[1], vy1[2], vy1[3]);
            if (zwall) *reinterpret_cast<float4*>(wo + iz0 + nn) = make_float4(wz1[0], wz1[1], wz1[2], wz1[3]);
            if (uh) {
#pragma unroll
                for (int k = 0; k < 4; ++k) uh[ix0 + k] = 2.f * ux0[k] - uin[k];
                *reinterpret_cast<float4*>(vh + iy0) =
                    make_float4(2.f * vy0[0] - vin0[0], 2.f * vy0[1] - vin0[1], 2.f * vy0[2] - vin0[2],
                                2.f * vy0[3] - vin0[3]);
                *reinterpret_cast<float4*>(wh + iz0) =
                    make_float4(2.f * wz0[0] - win0[0], 2.f * wz0[1] - win0[1], 2.f * wz0[2] - win0[2],
                                2.f * wz0[3] - win0[3]);
                if (xwall) uh[ix0 + 4] = 2.f * ux1[3] - uin[4];
                if (ywall)
                    *reinterpret_cast<float4*>(vh + iy0 + n) =
                        make_float4(2.f * vy1[0] - vin1[0], 2.f * vy1[1] - vin1[1], 2.f * vy1[2] - vin1[2],
                                    2.f * vy1[3] - vin1[3]);
                if (zwall)
                    *reinterpret_cast<float4*>(wh + iz0 + nn) =
                        make_float4(2.f * wz1[0] - win1[0], 2.f * wz1[1] - win1[1], 2.f * wz1[2] - win1[2],
                                    2.f * wz1[3] - win1[3]);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                zm[k] = zc[k];
                zc[k] = zp[k];
            }
        }
    }
    const double br = block_max(rmax, s_res);
    const float bd = block_max(dmax, s_div);
    const int any_solve = __syncthreads_or(int(bad_solve));
    const int any_div = __syncthreads_or(int(bad_div));
    if (threadIdx.x == 0) {
        atomic_max_nonneg(&ctrl->res_bits, br);
        atomic_max_nonneg(&ctrl->div_after_bits, bd);
        if (any_solve) atomicOr(&ctrl->nonfinite, 4u);
        if (any_div) atomicOr(&ctrl->nonfinite, 2u);
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
    const float bm = ctrl->rhs_mean_f;
    const float pm = final_pass ? ctrl->p_mean_f : 0.f;
    const RBLayout L = rb_layout(n);
    double r = 0.0;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        auto xv = [&](int a, int bb, int cc) {
            const float v = x[rb_index(L, a, bb, cc)];
            return final_pass ? v - pm : v;
        };
        const float xc = xv(i, j, k);
        double ax = double(float(neighbours(n, i, j, k))) * double(xc);
        if (i > 0) ax += -1.0 * double(xv(i - 1, j, k));
        if (i + 1 < n) ax += -1.0 * double(xv(i + 1, j, k));
        if (j > 0) ax += -1.0 * double(xv(i, j - 1, k));
        if (j + 1 < n) ax += -1.0 * double(xv(i, j + 1, k));
        if (k > 0) ax += -1.0 * double(xv(i, j, k - 1));
        if (k + 1 < n) ax += -1.0 * double(xv(i, j, k + 1));
        const float bi = b[rb_index(L, i, j, k)] - bm;
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
__global__ void k_check(ProjControl* ctrl, int iterations, int accumulate, int flip_x64, int use_conditional,
                        cudaGraphConditionalHandle handle, int gated) {
    if (gated && !ctrl->recentre) return;
    if (accumulate) ctrl->iterations = min(ctrl->iterations + iterations, ctrl->max_iterations);
    else ctrl->iterations = iterations;
    if (flip_x64) ctrl->x64_cur = 1 - ctrl->x64_cur;
    const double res = __longlong_as_double((long long)ctrl->res_bits);
    ctrl->res_bits = 0ull;
    ctrl->r0 = res;
    ctrl->since = 0;
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
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const size_t cells = size_t(n) * n * n;
    double sum = 0.0;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int i, j, k;
        decode_cell(c, n, i, j, k);
        sum += double(x[rb_index(L, i, j, k)]);
    }
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
    const RBLayout L = rb_layout(n);
    float div_max = 0.f;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        auto pv = [&](int a, int bb, int cc) { return p[rb_index(L, a, bb, cc)] - pm; };
        const float pc = pv(x, y, z);
        const size_t ix0 = index_of(n, FACE_X, x, y, z), ix1 = ix0 + 1;
        const size_t iy0 = index_of(n, FACE_Y, x, y, z), iy1 = iy0 + n;
        const size_t iz0 = c, iz1 = c + nn;
        const float ux0 = x == 0 ? 0.f : u[ix0] - dt * (pc - pv(x - 1, y, z)) * hInv;
        const float ux1 = x + 1 == n ? 0.f : u[ix1] - dt * (pv(x + 1, y, z) - pc) * hInv;
        const float vy0 = y == 0 ? 0.f : v[iy0] - dt * (pc - pv(x, y - 1, z)) * hInv;
        const float vy1 = y + 1 == n ? 0.f : v[iy1] - dt * (pv(x, y + 1, z) - pc) * hInv;
        const float wz0 = z == 0 ? 0.f : w[iz0] - dt * (pc - pv(x, y, z - 1)) * hInv;
        const float wz1 = z + 1 == n ? 0.f : w[iz1] - dt * (pv(x, y, z + 1) - pc) * hInv;
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

// Natural-order copy of the zero-mean pressure (x - pressure mean) for callers.
__global__ void __launch_bounds__(kThreads) k_unsplit_pressure(Grid g, const float* __restrict__ p,
                                                               const ProjControl* __restrict__ ctrl,
                                                               float* __restrict__ out) {
    const int n = g.n;
    const RBLayout L = rb_layout(n);
    const size_t cells = size_t(n) * n * n;
    const float pm = ctrl->p_mean_f;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode_cell(c, n, x, y, z);
        out[c] = p[rb_index(L, x, y, z)] - pm;
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
                double* partials, int partial_capacity, ProjControl* ctrl, double* x64a, double* x64b,
                LoopCond cond, cudaStream_t s, const float* field) {
    const size_t cells = size_t(a.g.n) * a.g.n * a.g.n;
    const int blocks = std::min(reduction_blocks(cells), partial_capacity);
    const float scale = a.g.h * a.g.h / a.dt;
    count_launch();
    k_begin_projection<<<1, 1, 0, s>>>(ctrl, a.options, x64a, x64b);
    count_launch();
    k_rhs<<<blocks, kThreads, 0, s>>>(a.g, scale, u, v, w, b, partials, ctrl, a.solid, field);
    count_launch();
    k_rhs_finish<<<1, 1024, 0, s>>>(ctrl, partials, blocks, a.solid ? a.fluid : double(cells),
                                    a.options.absolute_tolerance,
                                    a.options.relative_tolerance, cond.active,
                                    (cudaGraphConditionalHandle)cond.handle);
}

bool sor_fuses_measure(int n) {
    const RBLayout L = rb_layout(n);
    return L.hw % 4 == 0 && 2 * L.stride < (size_t(1) << 31);
}

// Planes per thread of the z-marching sweep chosen by the autotuner for a
// grid size (0: automatic). Read when a sweep is launched or recorded.
std::mutex g_tuning_mutex;
std::map<int, int> g_sor_planes;

void set_sor_planes(int n, int planes) {
    std::lock_guard<std::mutex> lock(g_tuning_mutex);
    if (planes <= 0) g_sor_planes.erase(n);
    else g_sor_planes[n] = planes;
}

// Planes per thread of the z-marching sweep: the tuned value; else, when
// it is at least 2 and at most 16, the largest count whose full-length
// chunks still fit one wave of resident blocks (148 SMs x 5, or x 4 for the
// variants that also reduce a residual or dot products), so that only
// the short last chunk runs after the wave; else about 2.5 waves. At 256^3
// this gives 11 planes (768 blocks: 23.4 us per colour launch, against
// 25.2 us at 4 planes / 2048 blocks and 25.0 us at 12 planes / 704 blocks).
static int sor_planes(int n, int blocks_x, int blocks_per_sm = 5) {
    {
        std::lock_guard<std::mutex> lock(g_tuning_mutex);
        const auto it = g_sor_planes.find(n);
        if (it != g_sor_planes.end()) return std::max(1, std::min(it->second, n));
    }
    const long slots = 148L * blocks_per_sm;
    const long per_plane = long(blocks_x);
    const long one_wave = (per_plane * n) / slots;
    if (one_wave >= 2 && one_wave <= 16) return int(one_wave);
    const long target_blocks = slots * 5 / 2;
    int zb = int(std::max(1L, (per_plane * n) / target_blocks));
    return std::min(zb, 8);
}

int launch_sor_color_dot(const ProjectionArgs& a, int parity, float* x, const float* b, const float* q,
                         double* partials, int partial_capacity, ProjControl* ctrl, cudaStream_t s) {
    const int n = a.g.n;
    const RBLayout L = rb_layout(n);
    if (!sor_fuses_measure(n) || a.diag != nullptr || n % 2 != 0) return 0;
    const int bx = (L.hw / 4 * n + kThreads - 1) / kThreads;
    const int zb = sor_planes(n, bx, 4);
    const dim3 grid(bx, (n + zb - 1) / zb);
    const int blocks = int(grid.x * grid.y);
    if (2 * blocks > partial_capacity) return 0;
    RelaxTable wr;
    for (int d = 0; d < 7; ++d) wr.w[d] = a.omega / std::max(float(d), a.diagonal_floor);
    count_launch();
    k_sor_rbz<false, false, false, true, true><<<grid, kThreads, 0, s>>>(
        a.g, parity, a.omega, a.diagonal_floor, wr, x, b, ctrl, 0, 0, 0, zb, nullptr, q, partials);
    return blocks;
}

void launch_sor_color(const ProjectionArgs& a, int parity, float* x, const float* b, ProjControl* ctrl,
                      bool guarded, int sweep_index, bool subtract_mean, cudaStream_t s, bool exact, bool measure,
                      bool from_zero) {
    const int n = a.g.n;
    const RBLayout L = rb_layout(n);
    RelaxTable wr;
    for (int d = 0; d < 7; ++d) wr.w[d] = a.omega / std::max(float(d), a.diagonal_floor);
    const int g = guarded ? 1 : 0, m = subtract_mean ? 1 : 0;
    count_launch();
    if (sor_fuses_measure(n)) {
        const int bx = (L.hw / 4 * n + kThreads - 1) / kThreads;
        const int zb = sor_planes(n, bx, measure ? 4 : 5);
        const dim3 grid(bx, (n + zb - 1) / zb);
        const bool plain = a.diag == nullptr && n % 2 == 0;
#define VB_SOR_RBZ(E, R, Z, P)                                                                                \
    k_sor_rbz<E, R, Z, P><<<grid, kThreads, 0, s>>>(a.g, parity, a.omega, a.diagonal_floor, wr, x, b, ctrl, g, \
                                                    sweep_index, m, zb, a.diag)
        if (from_zero && !exact && !measure) {
            if (plain) VB_SOR_RBZ(false, false, true, true);
            else VB_SOR_RBZ(false, false, true, false);
        } else if (exact && measure) {
            if (plain) VB_SOR_RBZ(true, true, false, true);
            else VB_SOR_RBZ(true, true, false, false);
        } else if (exact) {
            if (plain) VB_SOR_RBZ(true, false, false, true);
            else VB_SOR_RBZ(true, false, false, false);
        } else if (measure) {
            if (plain) VB_SOR_RBZ(false, true, false, true);
            else VB_SOR_RBZ(false, true, false, false);
        } else {
            if (plain) VB_SOR_RBZ(false, false, false, true);
            else VB_SOR_RBZ(false, false, false, false);
        }
#undef VB_SOR_RBZ
    } else if (L.hw % 4 == 0) {
        const dim3 grid((L.hw / 4 * n + kThreads - 1) / kThreads, n);
        if (exact) k_sor_rb<4, true><<<grid, kThreads, 0, s>>>(a.g, parity, a.omega, a.diagonal_floor, wr, x, b, ctrl, g, sweep_index, m, a.diag);
        else k_sor_rb<4, false><<<grid, kThreads, 0, s>>>(a.g, parity, a.omega, a.diagonal_floor, wr, x, b, ctrl, g, sweep_index, m, a.diag);
    } else {
        const dim3 grid((L.hw * n + kThreads - 1) / kThreads, n);
        if (exact) k_sor_rb<1, true><<<grid, kThreads, 0, s>>>(a.g, parity, a.omega, a.diagonal_floor, wr, x, b, ctrl, g, sweep_index, m, a.diag);
        else k_sor_rb<1, false><<<grid, kThreads, 0, s>>>(a.g, parity, a.omega, a.diagonal_floor, wr, x, b, ctrl, g, sweep_index, m, a.diag);
    }
}

void launch_unsplit_pressure(const Grid& g, const float* p, const ProjControl* ctrl, float* out, cudaStream_t s) {
    const size_t cells = size_t(g.n) * g.n * g.n;
    count_launch();
    k_unsplit_pressure<<<reduction_blocks(cells), kThreads, 0, s>>>(g, p, ctrl, out);
}

static void refine_launch(const ProjectionArgs& a, const float* b, const float* e, float* r32, ProjControl* ctrl,
                          int gated, cudaStream_t s) {
    const int n = a.g.n;
    const RBLayout L = rb_layout(n);
    count_launch();
    if (L.hw % 4 == 0) {
        const dim3 grid((L.hw / 4 * n + kThreads - 1) / kThreads, n, 2);
        k_refine_rb<4><<<grid, kThreads, 0, s>>>(a.g, b, e, r32, ctrl, gated, a.diag);
    } else {
        const dim3 grid((L.hw * n + kThreads - 1) / kThreads, n, 2);
        k_refine_rb<1><<<grid, kThreads, 0, s>>>(a.g, b, e, r32, ctrl, gated, a.diag);
    }
}

void launch_refine_residual(const ProjectionArgs& a, const float* b, const float* e, float* r32,
                            ProjControl* ctrl, cudaStream_t s) {
    refine_launch(a, b, e, r32, ctrl, 0, s);
}

void launch_refine_residual_gated(const ProjectionArgs& a, const float* b, const float* e, float* r32,
                                  ProjControl* ctrl, cudaStream_t s) {
    refine_launch(a, b, e, r32, ctrl, 1, s);
}

void launch_error_check(const ProjectionArgs& a, const float* e, const float* r32, ProjControl* ctrl, int sweeps,
                        bool measured, LoopCond cond, LoopCond recentre_cond, cudaStream_t s) {
    const int n = a.g.n;
    const RBLayout L = rb_layout(n);
    if (!measured) {
        count_launch();
        if (L.hw % 4 == 0) {
            const dim3 grid((L.hw / 4 * n + kThreads - 1) / kThreads, n, 1);
            k_error_residual<4><<<grid, kThreads, 0, s>>>(a.g, e, r32, ctrl, 1, a.diag);
        } else {
            const dim3 grid((L.hw * n + kThreads - 1) / kThreads, n, 1);
            k_error_residual<1><<<grid, kThreads, 0, s>>>(a.g, e, r32, ctrl, 1, a.diag);
        }
    }
    count_launch();
    k_error_decide<<<1, 1, 0, s>>>(ctrl, sweeps, cond.active, (cudaGraphConditionalHandle)cond.handle,
                                   recentre_cond.active, (cudaGraphConditionalHandle)recentre_cond.handle);
}

__global__ void k_loop_condition(const ProjControl* ctrl, cudaGraphConditionalHandle handle) {
    cudaGraphSetConditional(handle, ctrl->done ? 0u : 1u);
}

void launch_loop_condition(const ProjControl* ctrl, LoopCond cond, cudaStream_t s) {
    if (!cond.active) return;
    count_launch();
    k_loop_condition<<<1, 1, 0, s>>>(ctrl, (cudaGraphConditionalHandle)cond.handle);
}

void launch_check_gated(ProjControl* ctrl, LoopCond cond, cudaStream_t s) {
    count_launch();
    k_check<<<1, 1, 0, s>>>(ctrl, 0, 1, 1, cond.active, (cudaGraphConditionalHandle)cond.handle, 1);
}

void launch_zero_error_gated(const ProjectionArgs& a, float* e, const ProjControl* ctrl, cudaStream_t s) {
    const RBLayout L = rb_layout(a.g.n);
    const size_t count = 2 * L.stride;
    count_launch();
    k_zero_error_gated<<<kMaxReductionBlocks, kThreads, 0, s>>>(e, count, ctrl);
}

int launch_finish_projection64(const ProjectionArgs& a, const float* b, float* p32, double* partials,
                               int partial_capacity, ProjControl* ctrl, const float* u_in, const float* v_in,
                               const float* w_in, float* u_out, float* v_out, float* w_out, float* u_hat,
                               float* v_hat, float* w_hat, cudaStream_t s) {
    const int n = a.g.n;
    const size_t cells = size_t(n) * n * n;
    const int blocks = std::min(reduction_blocks(cells), partial_capacity);
    count_launch();
    k_psum64<<<blocks, kThreads, 0, s>>>(a.g, ctrl, partials);
    count_launch();
    k_psum64_finish<<<1, 1024, 0, s>>>(ctrl, partials, blocks, a.solid ? a.fluid : double(cells));
    if (u_in && !a.solid && !a.diag && n % 4 == 0) {
        // residual, pressure copy and gradient in one z-marching pass
        constexpr int zb = 8;
        const dim3 grid(unsigned((size_t(n) * (n / 4) + kThreads - 1) / kThreads), unsigned((n + zb - 1) / zb));
        count_launch();
        k_finish64<<<grid, kThreads, 0, s>>>(a.g, a.dt, b, p32, ctrl, u_in, v_in, w_in, u_out, v_out, w_out,
                                             u_hat, v_hat, w_hat, zb);
        count_launch();
        k_final_check<<<1, 1, 0, s>>>(ctrl);
        return 4;
    }
    count_launch();
    k_residual64<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, b, p32, ctrl, a.diag);
    count_launch();
    k_final_check<<<1, 1, 0, s>>>(ctrl);
    if (!u_in) return 4;
    count_launch();
    k_gradient64<<<reduction_blocks(cells), kThreads, 0, s>>>(a.g, a.dt, u_in, v_in, w_in, u_out, v_out, w_out,
                                                              u_hat, v_hat, w_hat, ctrl, a.solid);
    return 5;
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

void launch_check(ProjControl* ctrl, int iterations, bool accumulate, bool flip_x64, LoopCond cond,
                  cudaStream_t s) {
    count_launch();
    k_check<<<1, 1, 0, s>>>(ctrl, iterations, accumulate ? 1 : 0, flip_x64 ? 1 : 0, cond.active,
                            (cudaGraphConditionalHandle)cond.handle, 0);
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
