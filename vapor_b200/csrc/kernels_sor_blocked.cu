// Temporally blocked red-black SOR: K full red+black iterations per launch
// (SOR.cpp:36-54 and sor.comp:7-23 for one colour; colour = (x+y+z+parity)&1,
// parity 0 first), bit-identical to 2K launches of the one-colour sweep.
//
// A CTA owns a tile of 8 float4 groups (32 slots = 64 cells) in x by TY rows in
// y and a chunk of zc planes in z, and marches up the chunk as a wavefront:
// at step tau, half-sweep t (t = 1..2K) updates its colour in plane
// tau - t + 1. Every value a half-sweep reads in its own (row, slot) column
// (the cell itself and its z-neighbours) was produced by the same thread, so
// it stays in registers; only the in-plane neighbours (rows y-1, y+1 and the
// x-neighbour slot) come from shared memory, where they were written in the
// previous step. One barrier per plane therefore orders everything.
//
// Shared memory holds rings of 2K + 3 planes (both colours) of the iterate
// and of the right-hand side over the tile and its halo: one float4 group on
// each side in x and 2K rows on each side in y (every half-sweep invalidates
// one more ring of cells at the tile edge). The z-chunk loads 2K extra planes
// on each side for the same reason. Planes are loaded two steps ahead with
// cp.async (16 bytes per thread, colour and field; zero fill outside the
// grid, where missing neighbours read as zero exactly as in the one-colour
// sweep), so no global load sits on a step's critical path.
//
// The update is out of place: the launch reads x_in and writes x_out, because
// neighbouring CTAs read each other's cells as halo while they run. A guarded
// launch past the iteration budget copies x_in to x_out.
//
// DRAM traffic per launch is the tile's halo-inflated read of x and b plus one
// write of x: at 256^3 with TY = 16 about 2x (4 + 4) + 4 B per cell for K = 2
// iterations, against 16 B per iteration for the one-colour sweep.
#include "engine.hpp"
#include "kernels.hpp"

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>

namespace vb {
namespace {

constexpr int kGroups = 8;        // interior float4 groups per tile row
constexpr int kGX = kGroups + 2;  // plus one halo group on each side

template <int K, int TY>
struct Blocked {
    static constexpr int S = 2 * K;        // colour half-sweeps per launch
    static constexpr int HY = S;           // halo rows on each side
    static constexpr int R = TY + 2 * HY;  // rows held
    static constexpr int RING = S + 3;     // planes held (two loading ahead)
    static constexpr int POS = R * kGX;    // (row, group) positions, one per thread
    static constexpr int THREADS = (POS + 31) / 32 * 32;
    static constexpr int PLANE = R * kGX;  // float4 per plane and colour
    static constexpr int SMEM = 2 * RING * 2 * PLANE * 16;  // iterate and right-hand side
};

struct RelaxW {
    float w[7];
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ float comp(const float4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}

// One half-sweep of colour C on the thread's 4 slots: the one-colour sweep's
// arithmetic in its operation order (k_sor_rbz), PLAIN (no mask, n even:
// diagonals from the neighbour counts) or with the solid-mask diagonal.
template <bool EXACT, bool MASK>
__device__ __forceinline__ float4 relax4(const float4 xo, const float (&xl)[5], const float4 ym, const float4 yp,
                                         const float4 zm, const float4 zp, const float4 b4, float bm, int ny,
                                         bool ledge, bool redge, int xc0, int n, uchar4 dm, float omega,
                                         float floor_diag, const RelaxW& wr, bool resid, float& rmax) {
    float res[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float x0 = comp(xo, k), bi = comp(b4, k) - bm;
        if (!MASK) {
            const float diag0 = ny == 4 ? 6.f : (ny == 3 ? 5.f : 4.f), diag1 = diag0 - 1.f;
            const float w0 = EXACT ? maxf_ref(diag0, floor_diag) : (ny == 4 ? wr.w[6] : (ny == 3 ? wr.w[5] : wr.w[4]));
            const float w1 = EXACT ? maxf_ref(diag1, floor_diag) : (ny == 4 ? wr.w[5] : (ny == 3 ? wr.w[4] : wr.w[3]));
            const bool edge = (k == 0 && ledge) || (k == 3 && redge);
            const float diag = edge ? diag1 : diag0;
            float off = 0.f;
            off += -1.f * xl[k];
            off += -1.f * xl[k + 1];
            off += -1.f * comp(ym, k);
            off += -1.f * comp(yp, k);
            off += -1.f * comp(zm, k);
            off += -1.f * comp(zp, k);
            float r;
            if (EXACT) r = x0 + omega * (bi - off - diag * x0) / (edge ? w1 : w0);
            else r = x0 + (bi - off - diag * x0) * (edge ? w1 : w0);
            res[k] = r;
            if (resid) rmax = fmaxf(rmax, fabsf(bi - off - diag * r));
        } else {
            const int xc = xc0 + 2 * k;
            const bool left = xc > 0, right = xc + 1 < n;
            const int d = k == 0 ? dm.x : (k == 1 ? dm.y : (k == 2 ? dm.z : dm.w));
            const float diag = float(d);
            float off = 0.f;
            off += -1.f * (left ? xl[k] : 0.f);
            off += -1.f * (right ? xl[k + 1] : 0.f);
            off += -1.f * comp(ym, k);
            off += -1.f * comp(yp, k);
            off += -1.f * comp(zm, k);
            off += -1.f * comp(zp, k);
            float r;
            if (EXACT) {
                r = x0 + omega * (bi - off - diag * x0) / maxf_ref(diag, floor_diag);
            } else {
                const float w = d == 6 ? wr.w[6] : (d == 5 ? wr.w[5] : (d == 4 ? wr.w[4] : wr.w[3]));
                r = x0 + (bi - off - diag * x0) * w;
            }
            const bool valid = xc < n && d > 0;
            res[k] = valid ? r : x0;
            if (resid && valid) rmax = fmaxf(rmax, fabsf(bi - off - diag * r));
        }
    }
    return make_float4(res[0], res[1], res[2], res[3]);
}

// FIRST: colour of the first half-sweep (the reference order is 0 then 1;
// the FPCG post-smoother runs 1 then 0). FROM_ZERO: the sweep starts from
// x = 0 (x_in is not read; both colours are written). RESID: the last
// half-sweep also records max |b' - off - diag x| over its updated cells into
// ctrl->res32_bits, as the one-colour sweep's measuring form does.
// A guarded launch covers sweeps sweep_index .. sweep_index + K - 1 of the
// current chunk and does only those the iteration budget still allows (the
// remaining half-sweeps pass values through unchanged); it measures only when
// it ran all K.
template <int K, int TY, int FIRST, bool EXACT, bool RESID, bool FROM_ZERO, bool MASK>
__global__ void __launch_bounds__(Blocked<K, TY>::THREADS, 2) k_sor_blocked(
    Grid g, float omega, float floor_diag, RelaxW wr, const float* __restrict__ xin, float* __restrict__ xout,
    const float* __restrict__ bs, ProjControl* ctrl, int guarded, int sweep_index, int subtract_mean, int zc,
    const uint8_t* __restrict__ dg) {
    using B = Blocked<K, TY>;
    constexpr int S = B::S, RING = B::RING, R = B::R, PL = B::PLANE;
    extern __shared__ float4 ring[];  // x: [RING][2][R][kGX], then b: the same
    __shared__ float s_max[32];

    const int n = g.n, hw = n >> 1, hg = hw >> 2;
    const int plane = n * hw, cstride = n * plane;
    const int tid = threadIdx.x;
    const bool thread_live = tid < B::POS;
    const int r = thread_live ? tid / kGX : 0, gl = thread_live ? tid - r * kGX : 0;
    const int y = int(blockIdx.y) * TY - B::HY + r;
    const int gg = int(blockIdx.x) * kGroups - 1 + gl;
    const bool in_dom = thread_live && y >= 0 && y < n && gg >= 0 && gg < hg;
    const bool interior = in_dom && r >= B::HY && r < B::HY + TY && gl >= 1 && gl <= kGroups;
    const int z0 = int(blockIdx.z) * zc, z1 = min(n, z0 + zc);
    const int col = y * hw + gg * 4;  // offset of the thread's group in a plane of one colour

    int live = S;  // half-sweeps that update (the rest pass through)
    if (guarded) {
        const int left = ctrl->max_iterations - ctrl->iterations - sweep_index;
        live = ctrl->done ? 0 : 2 * max(0, min(K, left));
    }
    if (live == 0) {  // nothing to do: x_out = x_in over the CTA's own cells
        if (interior)
            for (int zz = z0; zz < z1; ++zz)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int o = c * cstride + zz * plane + col;
                    *reinterpret_cast<float4*>(xout + o) = *reinterpret_cast<const float4*>(xin + o);
                }
        return;
    }
    const bool measure = RESID && live == S;
    const float bm = subtract_mean ? ctrl->rhs_mean_f : 0.f;
    const int tau0 = max(0, z0 - (S - 1)), tau_end = z1 + S - 1;
    const int me = r * kGX + gl;
    const int ny_yz = int(y > 0) + int(y + 1 < n);
    const bool left_group = gg == 0, right_group = gg == hg - 1;
    const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
    float4* bring = ring + RING * 2 * PL;
    float rmax = 0.f;

    auto slot_of = [&](int p) { return (p - tau0 + 1 + RING) % RING; };
    auto at = [&](int slot, int c) { return ring + (slot * 2 + c) * PL; };
    auto bat = [&](int slot, int c) { return bring + (slot * 2 + c) * PL; };
    // plane p (both colours, iterate and right-hand side) of the thread's
    // position into its ring slot
    auto load_plane = [&](int p) {
        if (!thread_live) return;
        const int slot = slot_of(p);
        const bool ok = in_dom && p >= 0 && p < n;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int o = c * cstride + p * plane + col;
            if (FROM_ZERO) at(slot, c)[me] = zero4;
            else cp_async16(at(slot, c) + me, ok ? xin + o : xin, ok);
            cp_async16(bat(slot, c) + me, ok ? bs + o : bs, ok);
        }
    };

    // V[c][k]: the thread's values of colour c in plane tau + 1 - k
    float4 V[2][S + 2];
#pragma unroll
    for (int c = 0; c < 2; ++c)
#pragma unroll
        for (int k = 0; k < S + 2; ++k) V[c][k] = zero4;

    load_plane(tau0 - 1);
    load_plane(tau0);
    load_plane(tau0 + 1);
    cp_async_commit();
    load_plane(tau0 + 2);
    cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
    if (thread_live) {
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            V[c][2] = at(slot_of(tau0 - 1), c)[me];
            V[c][1] = at(slot_of(tau0), c)[me];
        }
    }

    for (int tau = tau0; tau < tau_end; ++tau) {
        const int s1 = slot_of(tau + 1);
        if (thread_live) {
#pragma unroll
            for (int c = 0; c < 2; ++c) V[c][0] = at(s1, c)[me];
        }
        load_plane(tau + 3);  // into the slot of plane tau - S, last read in the previous step
        cp_async_commit();
#pragma unroll
        for (int t = 1; t <= S; ++t) {
            const int C = (FIRST + t - 1) & 1, OC = 1 - C;
            const int zt = tau - t + 1;
            const int lo = max(0, z0 - (S - t)), hi = min(n, z1 + (S - t));
            if (t <= live && in_dom && zt >= lo && zt < hi) {
                const int st = (s1 - t + RING) % RING;
                const float4* oth = at(st, OC);
                const float4 xc = V[OC][t];
                const float4 ym = r > 0 ? oth[me - kGX] : zero4;
                const float4 yp = r < R - 1 ? oth[me + kGX] : zero4;
                const int sh = (y + zt + C) & 1;
                float xl[5];
                if (sh == 0) {
                    xl[0] = gl > 0 ? reinterpret_cast<const float*>(oth + me - 1)[3] : 0.f;
                    xl[1] = xc.x; xl[2] = xc.y; xl[3] = xc.z; xl[4] = xc.w;
                } else {
                    xl[0] = xc.x; xl[1] = xc.y; xl[2] = xc.z; xl[3] = xc.w;
                    xl[4] = gl < kGX - 1 ? reinterpret_cast<const float*>(oth + me + 1)[0] : 0.f;
                }
                const float4 b4 = bat(st, C)[me];
                uchar4 dm = make_uchar4(0, 0, 0, 0);
                if (MASK) dm = __ldg(reinterpret_cast<const uchar4*>(dg + C * cstride + zt * plane + col));
                const int ny = ny_yz + int(zt > 0) + int(zt + 1 < n);
                const bool resid = measure && t == S && interior;
                const float4 res = relax4<EXACT, MASK>(V[C][t], xl, ym, yp, V[OC][t + 1], V[OC][t - 1], b4, bm, ny,
                                                       left_group && sh == 0, right_group && sh == 1,
                                                       2 * gg * 4 + sh, n, dm, omega, floor_diag, wr, resid, rmax);
                V[C][t] = res;
                at(st, C)[me] = res;
            }
        }
        // plane tau - S + 1 is final for both colours
        const int zf = tau - S + 1;
        if (interior && zf >= z0 && zf < z1) {
            constexpr int CL = (FIRST + S - 1) & 1;
            *reinterpret_cast<float4*>(xout + CL * cstride + zf * plane + col) = V[CL][S];
            *reinterpret_cast<float4*>(xout + (1 - CL) * cstride + zf * plane + col) = V[1 - CL][S];
        }
#pragma unroll
        for (int c = 0; c < 2; ++c)
#pragma unroll
            for (int k = S + 1; k > 0; --k) V[c][k] = V[c][k - 1];
        cp_async_wait_one();  // plane tau + 2 has landed (tau + 3 may still be in flight)
        __syncthreads();
    }
    cp_async_wait_all();
    if (RESID) {
        const float br = block_max(rmax, s_max);
        if (threadIdx.x == 0 && measure && br > 0.f) atomicMax(&ctrl->res32_bits, __float_as_uint(br));
    }
}

std::mutex g_blocked_mutex;
std::map<int, int> g_blocked_chunks;  // grid size -> z chunks per launch (tuning)
// Off by default: on B200 at 256^3 the blocked launch costs more per
// iteration than two one-colour launches (see set_sor_block_iterations).
std::atomic<int> g_block_iterations{0};

template <int K, int TY, int FIRST, bool EXACT, bool RESID, bool FROM_ZERO, bool MASK>
void launch_blocked(const ProjectionArgs& a, const float* xin, float* xout, const float* b, ProjControl* ctrl,
                    bool guarded, int sweep_index, bool subtract_mean, cudaStream_t s) {
    using B = Blocked<K, TY>;
    auto kern = k_sor_blocked<K, TY, FIRST, EXACT, RESID, FROM_ZERO, MASK>;
    static const int resident = [&] {
        VB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, B::SMEM));
        // all of the unified L1 / shared storage as shared memory, so that
        // two CTAs fit on an SM
        VB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     int(cudaSharedmemCarveoutMaxShared)));
        int blocks = 0;
        VB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kern, B::THREADS, B::SMEM));
        int dev = 0, sms = 0;
        VB_CUDA(cudaGetDevice(&dev));
        VB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        return std::max(1, blocks) * sms;
    }();
    const int n = a.g.n;
    const int hg = n / 8;
    const dim3 xy((hg + kGroups - 1) / kGroups, (n + TY - 1) / TY);
    int chunks = 0;
    {
        std::lock_guard<std::mutex> lock(g_blocked_mutex);
        const auto it = g_blocked_chunks.find(n);
        if (it != g_blocked_chunks.end()) chunks = it->second;
    }
    if (chunks <= 0) chunks = std::max(1, resident / int(xy.x * xy.y));  // one wave of CTAs
    // at least 2K planes per chunk, so that the chunk's halo planes stay a
    // fraction of its work
    const int zc = std::max((n + chunks - 1) / chunks, std::min(n, B::S));
    const dim3 grid(xy.x, xy.y, (n + zc - 1) / zc);
    RelaxW wr;
    for (int d = 0; d < 7; ++d) wr.w[d] = a.omega / std::max(float(d), a.diagonal_floor);
    count_launch();
    kern<<<grid, B::THREADS, B::SMEM, s>>>(a.g, a.omega, a.diagonal_floor, wr, xin, xout, b, ctrl, guarded ? 1 : 0,
                                          sweep_index, subtract_mean ? 1 : 0, zc, a.diag);
}

}  // namespace

bool sor_blocked_applies(int n) {
    // whole float4 groups per row (n % 8 == 0) and 32-bit offsets
    return n >= 8 && n % 8 == 0 && size_t(n) * n * n < (size_t(1) << 31);
}

void set_sor_block_iterations(int iterations) {
    if (iterations < 0 || iterations > 2) fail(VAPOR_INVALID_ARGUMENT, "blocked sweep: 0, 1 or 2 iterations per launch");
    g_block_iterations.store(iterations);
}

int sor_block_iterations(int n) { return sor_blocked_applies(n) ? g_block_iterations.load() : 0; }

void set_sor_blocked_chunks(int n, int chunks) {
    std::lock_guard<std::mutex> lock(g_blocked_mutex);
    if (chunks <= 0) g_blocked_chunks.erase(n);
    else g_blocked_chunks[n] = chunks;
}

void launch_sor_blocked(const ProjectionArgs& a, int iterations, int first_colour, const float* xin, float* xout,
                        const float* b, ProjControl* ctrl, bool guarded, int sweep_index, bool subtract_mean,
                        cudaStream_t s, bool exact, bool measure, bool from_zero) {
    if (xin == xout && !from_zero) fail(VAPOR_RUNTIME_ERROR, "blocked sweep: the update is out of place");
    const bool mask = a.diag != nullptr;
    if (iterations != 1 && iterations != 2) fail(VAPOR_RUNTIME_ERROR, "blocked sweep: 1 or 2 iterations per launch");
    if (first_colour == 1 && (exact || measure || from_zero || mask))
        fail(VAPOR_RUNTIME_ERROR, "blocked sweep: colour-1-first form is the plain relaxation only");
    if (from_zero && (exact || measure || mask))
        fail(VAPOR_RUNTIME_ERROR, "blocked sweep: start-from-zero form is the plain relaxation only");
    if (exact && measure) fail(VAPOR_RUNTIME_ERROR, "blocked sweep: the exact form does not measure");
    constexpr int TY = 16;
#define VB_BLK(KK, F, E, R, Z, M) \
    launch_blocked<KK, TY, F, E, R, Z, M>(a, xin, xout, b, ctrl, guarded, sweep_index, subtract_mean, s)
#define VB_BLK_K(F, E, R, Z, M)                    \
    if (iterations == 2) VB_BLK(2, F, E, R, Z, M); \
    else VB_BLK(1, F, E, R, Z, M)
    if (first_colour == 1) {
        VB_BLK_K(1, false, false, false, false);
    } else if (from_zero) {
        VB_BLK_K(0, false, false, true, false);
    } else if (exact) {
        if (mask) { VB_BLK_K(0, true, false, false, true); }
        else { VB_BLK_K(0, true, false, false, false); }
    } else if (measure) {
        if (mask) { VB_BLK_K(0, false, true, false, true); }
        else { VB_BLK_K(0, false, true, false, false); }
    } else {
        if (mask) { VB_BLK_K(0, false, false, false, true); }
        else { VB_BLK_K(0, false, false, false, false); }
    }
#undef VB_BLK_K
#undef VB_BLK
}

}  // namespace vb
