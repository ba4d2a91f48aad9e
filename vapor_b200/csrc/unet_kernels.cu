// Kernels of the learned pressure components: a 3-level 3D U-Net (16/32/64
// channels, 3x3x3 convolutions, BF16 weights and activations, FP32
// accumulation), its inference as warm start or FPCG coarse-grid correction,
// and its training (backward + Adam).
//
// The 3x3x3 convolutions - forward, and backward with respect to the input
// (a convolution with the spatially flipped, channel-transposed weights) - run
// on the tensor cores: k_conv3_zm (z-marching, weights resident) when the
// layer's weights and halo ring fit in shared memory, else k_conv3_tc (one
// plane per CTA, channel chunks streamed); PTX helpers in tc_conv.cuh. Weight
// gradients, pooling, upsampling, the 1x1 output head, the loss and Adam are
// memory-bound or small and run on CUDA cores.
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>

#include "kernels.hpp"
#include "tc_conv.cuh"
#include "unet.hpp"

namespace vb {
namespace unet {
namespace {

constexpr int kWaitLimit = 1 << 22;

// Kernel for the convolutions whose weights fit in shared memory: 0 the
// block-synchronous z-march, 1 its warp-specialised form, 2 the plane-window
// form (three output planes per MMA), 3 (default) the plane-window form fed
// by TMA.
std::atomic<int> g_conv_kind{3};

__device__ __forceinline__ void decode(long v, int H, int W, int& x, int& y, int& z) {
    x = int(v % W);
    const long r = v / W;
    y = int(r % H);
    z = int(r / H);
}

template <int N>
struct TmemColumns {
    static constexpr int value = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));
};

// The 27 MMAs (M = 128, N, K = 16) of one 16-channel chunk into the
// accumulator at TMEM address d. a_desc addresses the chunk's halo rows of
// plane z-1; the planes z and z+1 sit dz_bytes[1], dz_bytes[2] further; rows
// (next y) are 320 bytes apart and the 10 voxels of a row 16 bytes apart. b_desc
// addresses tap 0 of the chunk's weights, taps N * 32 bytes apart. Descriptor
// addresses are in 16-byte units in the low bits, so an offset is a plain add.
template <int N>
__device__ __forceinline__ void issue_taps(uint32_t d, uint64_t a_desc, const uint32_t (&dz_bytes)[3],
                                           uint64_t b_desc, uint32_t idesc, bool accumulate) {
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int t = dz * 9 + dy * 3 + dx;
                const uint64_t ad = a_desc + ((dz_bytes[dz] + uint32_t(dy * 320 + dx * 16)) >> 4);
                const uint64_t bd = b_desc + uint32_t(t * N * 2);  // t * N * 32 bytes
                tc::mma_bf16(d, ad, bd, idesc, accumulate || t > 0);
            }
}

// Epilogue of one tile of 128 voxels (8 x by 16 y in plane z): accumulator
// columns [0, N) at TMEM address acc, plus bias, optional ReLU, into the
// output (BF16 or FP32, out_stride channels per voxel from out_offset). Warp w
// reads TMEM lanes 32 (w & 3) .. + 31 (voxel m = lane index, x = m & 7,
// y = m >> 3) and the column half w >> 2, 8 columns (16 or 32 bytes) a store.
template <int N>
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, uint32_t acc, const float* s_bias, int x0, int y0,
                                              int z, int warp, int lane) {
    constexpr int kHalf = N / 2;
    const int q = warp & 3, h = warp >> 2;
    const int m = q * 32 + lane;
    const int x = x0 + (m & 7), y = y0 + (m >> 3);
    const bool vin = x < a.W && y < a.H;
    const long v = (long(z) * a.H + y) * a.W + x;
    const uint32_t lane_base = uint32_t(q * 32) << 16;
#pragma unroll
    for (int j = 0; j < kHalf / 8; ++j) {
        const int c0 = h * kHalf + j * 8;
        float val[8];
        tc::tmem_ld8(acc + lane_base + uint32_t(c0), val);
        if (vin) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                val[i] += s_bias[c0 + i];
                if (a.relu) val[i] = fmaxf(val[i], 0.f);
            }
            const long o = v * a.out_stride + a.out_offset + c0;
            if (a.out_fp32) {
                float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.out) + o);
                dst[0] = make_float4(val[0], val[1], val[2], val[3]);
                dst[1] = make_float4(val[4], val[5], val[6], val[7]);
            } else {
                __align__(16) __nv_bfloat16 hv[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) hv[i] = __float2bfloat16_rn(val[i]);
                *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.out) + o) =
                    *reinterpret_cast<const uint4*>(hv);
            }
        }
    }
}

// Implicit-GEMM 3x3x3 convolution on tcgen05 with a halo tile in shared
// memory. A CTA computes M = 128 voxels: 8 consecutive x by 16 consecutive y
// in one z plane (row m = 8 * yi + xi, TMEM lane m). For each 16-channel
// chunk of the input it stages
//   A: the halo x0-1 .. x0+8, y0-1 .. y0+16, z-1 .. z+1 once, as 54 rows
//      (dz, y) of 320 bytes: the 10 voxels' channels 0-7 (16 bytes each),
//      then their channels 8-15;
//   B: the chunk's weights of all 27 taps, [tap][N/8][2][8][16 B];
// then one thread issues the 27 MMAs (M=128, N, K=16) back to back. The A
// operand of tap (dz, dy, dx) is a view of the halo in the canonical K-major
// layout without swizzle: its 8-row core matrices are the 8 voxels from
// x0-1+dx (16-byte rows), the second K half sits 160 bytes further (LBO) and
// the next 8 rows (next y) 320 bytes further (SBO); so no data moves per tap.
// Chunks are double-buffered when there are several and two stages fit.
// Out-of-range neighbours are zero-filled (zero padding). Every wait is
// bounded; a timeout sets the error flag and skips the epilogue.
template <int N>
struct ConvTile {
    static constexpr int kRows = 3 * 18;                   // (dz, y) halo rows
    static constexpr int kRowBytes = 320;                  // 10 voxels x 2 K halves x 16 B
    static constexpr int kA = kRows * kRowBytes;           // bytes
    static constexpr int kB = 27 * N * 32;                 // bytes
    static constexpr int kStage = kA + kB;
    static constexpr bool kTwoStages = 2 * kStage <= 200 * 1024;
    static constexpr int kSmemMax = (kTwoStages ? 2 : 1) * kStage + 1024;  // + alignment slack
    static constexpr uint32_t kCols = TmemColumns<N>::value;
    static int smem(int chunks) { return ((kTwoStages && chunks > 1) ? 2 : 1) * kStage + 1024; }
};

template <int N>
__global__ void __launch_bounds__(256) k_conv3_tc(ConvArgs a) {
    using T = ConvTile<N>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[3];
    __shared__ uint32_t tmem_slot;
    __shared__ float s_bias[N];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16, z = blockIdx.z;
    const int chunks = a.cin / 16;
    const int stages = (T::kTwoStages && chunks > 1) ? 2 : 1;

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), T::kCols);
    const uint32_t bar0 = tc::smem_addr(&bars[0]);  // stage st's barrier at bar0 + 8 st
    const uint32_t probe = bar0 + 16;               // never arrived on (timeout test hook)
    if (tid == 0) {
        tc::mbar_init(bar0, 1);
        tc::mbar_init(bar0 + 8, 1);
        tc::mbar_init(probe, 1);
        tc::fence_mbarrier_init();
    }
    for (int i = tid; i < N; i += blockDim.x) s_bias[i] = a.bias ? a.bias[i] : 0.f;
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = tc::instr_desc_bf16(128, N);
    const uint32_t sbase = tc::smem_addr(smem);
    bool ok = true;
    int issued0 = 0, issued1 = 0;  // commits per stage (phase tracking)

    for (int cc = 0; cc < chunks; ++cc) {
        const int st = stages == 2 ? (cc & 1) : 0;
        const uint32_t abase = sbase + uint32_t(st * T::kStage);
        const uint32_t bbase = abase + T::kA;
        // the stage's previous MMAs must be done before it is overwritten
        const int before = st ? issued1 : issued0;
        if (before > 0) {
            const bool mine = a.wait_probe ? tc::mbar_wait(probe, 0u, a.wait_probe)
                                           : tc::mbar_wait(bar0 + uint32_t(8 * st), uint32_t(before - 1) & 1u,
                                                           kWaitLimit);
            if (!__syncthreads_and(mine)) {
                ok = false;
                break;
            }
        }
        for (int i = tid; i < T::kRows * 20; i += blockDim.x) {
            const int half = i & 1, v = (i >> 1) % 10, row = (i >> 1) / 10;  // row = dz * 18 + ry
            const int ry = row % 18, dz = row / 18;
            const int x = x0 - 1 + v, y = y0 + ry - 1, zz = z + dz - 1;
            const bool valid = x >= 0 && x < a.W && y >= 0 && y < a.H && zz >= 0 && zz < a.D;
            const __nv_bfloat16* src =
                valid ? a.in + ((long(zz) * a.H + y) * a.W + x) * a.in_stride + cc * 16 + half * 8 : a.in;
            tc::cp_async16(abase + uint32_t(row * T::kRowBytes + half * 160 + v * 16), src, valid);
        }
        for (int i = tid; i < 27 * N * 2; i += blockDim.x) {
            const int half = i & 1, co = (i >> 1) % N, t = (i >> 1) / N;
            const __nv_bfloat16* wsrc = a.w + (long(t) * N + co) * a.cin + cc * 16 + half * 8;
            tc::cp_async16(bbase + uint32_t(t * N * 32 + (co >> 3) * 256 + half * 128 + (co & 7) * 16), wsrc, true);
        }
        tc::cp_async_wait_all();
        tc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            constexpr uint32_t kDz[3] = {0u, 18u * T::kRowBytes, 36u * T::kRowBytes};
            issue_taps<N>(tmem, tc::smem_desc(abase, 160, T::kRowBytes), kDz, tc::smem_desc(bbase, 128, 256), idesc,
                          cc > 0);
            tc::mma_commit(bar0 + uint32_t(8 * st));
        }
        if (st) ++issued1;
        else ++issued0;
    }
    if (ok) {
        // the last commit covers every earlier MMA of this thread
        const int st = stages == 2 ? ((chunks - 1) & 1) : 0;
        const int commits = st ? issued1 : issued0;
        const bool mine = a.wait_probe ? tc::mbar_wait(probe, 0u, a.wait_probe)
                                       : tc::mbar_wait(bar0 + uint32_t(8 * st), uint32_t(commits - 1) & 1u,
                                                       kWaitLimit);
        ok = __syncthreads_and(mine);
    }
    tc::tc_fence_after();
    if (ok) {
        conv_epilogue<N>(a, tmem, s_bias, x0, y0, z, warp, lane);
    } else {
        if (tid == 0) atomicOr(a.error, 1u);
        // drain: wait (bounded) for every commit still in flight; if that
        // also runs out, MMAs may still write the columns freed below
        bool drained = true;
        if (issued0 > 0) drained &= tc::mbar_wait(bar0, uint32_t(issued0 - 1) & 1u, kWaitLimit);
        if (issued1 > 0) drained &= tc::mbar_wait(bar0 + 8, uint32_t(issued1 - 1) & 1u, kWaitLimit);
        if (!drained) atomicOr(a.error, 2u);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, T::kCols);
}

// The same convolution marching in z: a CTA computes zt consecutive planes of
// its 8 x 16 tile. All of the layer's weights stay in shared memory
// ([chunk][tap][N/8][2][8][16 B]) and the input halo is a ring of planes
// (each [chunk][18 rows][320 B] as above), so every input plane is loaded
// once per CTA. Two TMEM accumulators alternate between planes: the MMAs of
// plane z + 1 are issued before the epilogue of plane z drains the other
// accumulator. The ring has `ring` = 4 or 6 planes: the MMAs of planes z and
// z + 1 read 4 of them and the others load ahead (plane z + ring - 2 is
// requested at plane z; with 6 planes the loads run two planes ahead of
// their use). Used when the weights and the ring fit in shared memory
// (ConvMarch<N>::fits).
template <int N>
struct ConvMarch {
    static constexpr int kPlane = 18 * 320;                       // one chunk of one halo plane
    static constexpr uint32_t kCols = TmemColumns<2 * N>::value;  // two accumulators
    static constexpr uint32_t kAcc1 = kCols / 2;                  // column of the second
    static int smem(int cin, int ring) { return 27 * N * cin * 2 + ring * (cin / 16) * kPlane + 1024; }
    static bool fits(int cin, int ring) { return smem(cin, ring) <= 200 * 1024; }
};

template <int N>
__global__ void __launch_bounds__(256) k_conv3_zm(ConvArgs a, int zt, int ring) {
    using Z = ConvMarch<N>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[3];
    __shared__ uint32_t tmem_slot;
    __shared__ float s_bias[N];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16;
    const int z0 = blockIdx.z * zt, z1 = min(a.D, z0 + zt);
    const int chunks = a.cin / 16;
    const uint32_t sbase = tc::smem_addr(smem);
    const uint32_t wbase = sbase;
    const uint32_t rbase = sbase + uint32_t(27 * N * a.cin * 2);
    const uint32_t bar0 = tc::smem_addr(&bars[0]);  // accumulator k's barrier at bar0 + 8 k
    const uint32_t probe = bar0 + 16;               // never arrived on (timeout test hook)

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), Z::kCols);
    if (tid == 0) {
        tc::mbar_init(bar0, 1);
        tc::mbar_init(bar0 + 8, 1);
        tc::mbar_init(probe, 1);
        tc::fence_mbarrier_init();
    }
    for (int i = tid; i < N; i += blockDim.x) s_bias[i] = a.bias ? a.bias[i] : 0.f;
    // all weights: (chunk, tap, co, half) segments of 16 bytes
    for (int i = tid; i < chunks * 27 * N * 2; i += blockDim.x) {
        const int half = i & 1, co = (i >> 1) % N, ct = (i >> 1) / N;  // ct = chunk * 27 + tap
        const int t = ct % 27, cc = ct / 27;
        const __nv_bfloat16* wsrc = a.w + (long(t) * N + co) * a.cin + cc * 16 + half * 8;
        tc::cp_async16(wbase + uint32_t(ct * N * 32 + (co >> 3) * 256 + half * 128 + (co & 7) * 16), wsrc, true);
    }
    // halo plane zz >= -1 (all chunks) into ring slot (zz mod ring); rows
    // outside the grid read as zero
    const uint32_t plane_bytes = uint32_t(chunks * Z::kPlane);
    auto slot_of = [&](int zz) { return uint32_t((zz + ring) % ring) * plane_bytes; };
    auto load_plane = [&](int zz) {
        const uint32_t slot = rbase + slot_of(zz);
        for (int i = tid; i < chunks * 18 * 20; i += blockDim.x) {
            const int half = i & 1, v = (i >> 1) % 10, rc = (i >> 1) / 10;  // rc = chunk * 18 + ry
            const int ry = rc % 18, cc = rc / 18;
            const int x = x0 - 1 + v, y = y0 + ry - 1;
            const bool valid = x >= 0 && x < a.W && y >= 0 && y < a.H && zz >= 0 && zz < a.D;
            const __nv_bfloat16* src =
                valid ? a.in + ((long(zz) * a.H + y) * a.W + x) * a.in_stride + cc * 16 + half * 8 : a.in;
            tc::cp_async16(slot + uint32_t(rc * 320 + half * 160 + v * 16), src, valid);
        }
    };
    // one cp.async group: the weights and planes z0 - 1 .. z0 + 1; then one
    // group per plane ahead (z0 + 2 .. z0 + ring - 3; empty past z1)
    auto wait_ahead = [&]() {  // all but the ring - 4 newest groups have landed
        if (ring == 6) tc::cp_async_wait_group<2>();
        else tc::cp_async_wait_group<0>();
    };
    load_plane(z0 - 1);
    load_plane(z0);
    load_plane(z0 + 1);
    tc::cp_async_commit();
    for (int zz = z0 + 2; zz <= z0 + ring - 3; ++zz) {
        if (zz <= z1) load_plane(zz);
        tc::cp_async_commit();
    }
    wait_ahead();
    tc::fence_proxy_async();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t idesc = tc::instr_desc_bf16(128, N);
    const uint64_t a_desc = tc::smem_desc(rbase, 160, 320);
    const uint64_t b_desc = tc::smem_desc(wbase, 128, 256);
    // one thread: the MMAs of plane z into accumulator k, committed to barrier k
    auto issue = [&](int z, int k) {
        tc::tc_fence_after();
        const uint32_t dz_bytes[3] = {slot_of(z - 1), slot_of(z), slot_of(z + 1)};
#pragma unroll 1
        for (int cc = 0; cc < chunks; ++cc)
            issue_taps<N>(tmem + uint32_t(k) * Z::kAcc1, a_desc + uint32_t(cc * (Z::kPlane >> 4)), dz_bytes,
                          b_desc + uint32_t(cc * 27 * N * 2), idesc, cc > 0);
        tc::mma_commit(bar0 + uint32_t(8 * k));
    };
    bool ok = true;
    int issued0 = 1, issued1 = 0;  // commits per barrier, counted by every thread
    if (tid == 0) issue(z0, 0);
    for (int z = z0; z < z1; ++z) {
        const int k = (z - z0) & 1;
        const bool next = z + 1 < z1;
        if (next) {
            // into the ring slot of plane z - 2, last read by the MMAs of
            // plane z - 1 (complete)
            const int zz = z + ring - 2;
            if (zz <= z1) load_plane(zz);
            tc::cp_async_commit();
            wait_ahead();  // plane z + 2 has landed
            tc::fence_proxy_async();
        }
        // plane z + 2 is visible to the tensor core and the epilogue of plane
        // z - 1 has read accumulator k ^ 1
        tc::tc_fence_before();
        __syncthreads();
        if (next) {
            if (tid == 0) issue(z + 1, k ^ 1);
            if (k) ++issued0;
            else ++issued1;
        }
        const int commits = k ? issued1 : issued0;
        const bool mine = a.wait_probe ? tc::mbar_wait(probe, 0u, a.wait_probe)
                                       : tc::mbar_wait(bar0 + uint32_t(8 * k), uint32_t(commits - 1) & 1u,
                                                       kWaitLimit);
        if (!__syncthreads_and(mine)) {
            ok = false;
            break;
        }
        tc::tc_fence_after();
        conv_epilogue<N>(a, tmem + uint32_t(k) * Z::kAcc1, s_bias, x0, y0, z, warp, lane);
    }
    if (!ok) {
        if (tid == 0) atomicOr(a.error, 1u);
        // drain every commit still in flight, bounded; if that also runs out,
        // MMAs may still write the columns freed below
        bool drained = tc::mbar_wait(bar0, uint32_t(issued0 - 1) & 1u, kWaitLimit);
        if (issued1 > 0) drained &= tc::mbar_wait(bar0 + 8, uint32_t(issued1 - 1) & 1u, kWaitLimit);
        if (!drained) atomicOr(a.error, 2u);
        tc::cp_async_wait_all();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, Z::kCols);
}

// Warp-specialised form of the z-marching convolution. The CTA's roles run
// as a pipeline on mbarriers, with no block-wide barrier inside the march:
//   warp 0 (producer): loads halo plane q (all chunks, cp.async with zero
//     fill) into ring slot q % ring once the MMAs that read the slot's previous
//     plane are complete (`empty`), and signals `full` when its copies land;
//   warp 1 (MMA, one lane): for plane z waits for planes z - 1 .. z + 1 and
//     for accumulator k = plane & 1 to be drained (`acc_empty`), issues the
//     27 x chunks MMAs into it, then commits to `acc_full[k]` and to the
//     `empty` barrier of plane z - 1's slot (its last reader);
//   warps 2-5 (epilogue): wait for `acc_full[k]`, read their 32 TMEM lanes
//     (all N columns), add bias, ReLU, store, and arrive on `acc_empty[k]`.
// The weights stay resident as in k_conv3_zm; the A and B operands and the
// accumulator layout are the same, so results equal k_conv3_zm's. Every wait
// is bounded; a role that runs out sets the error flag and an abort flag that
// ends the other roles' waits, after which the MMA lane drains its in-flight
// MMAs (commit + bounded wait) before TMEM is freed.
template <int N>
struct ConvWS {
    static constexpr int kThreads = 192;
    static constexpr int kMaxRing = 6;
    static constexpr int kPlane = 18 * 320;
    static constexpr uint32_t kCols = TmemColumns<2 * N>::value;
    static constexpr uint32_t kAcc1 = kCols / 2;
    static int smem(int cin, int ring) { return 27 * N * cin * 2 + ring * (cin / 16) * kPlane + 1024; }
    static bool fits(int cin, int ring) { return smem(cin, ring) <= 200 * 1024; }
};

// Epilogue of one plane for one warp: TMEM lanes 32 quarter .. + 31 (voxel
// m = lane index within the 8 x 16 tile), all N accumulator columns.
template <int N>
__device__ __forceinline__ void ws_epilogue(const ConvArgs& a, uint32_t acc, const float* s_bias, int x0, int y0,
                                            int z, int quarter, int lane) {
    const int m = quarter * 32 + lane;
    const int x = x0 + (m & 7), y = y0 + (m >> 3);
    const bool vin = x < a.W && y < a.H;
    const long v = (long(z) * a.H + y) * a.W + x;
    const uint32_t lane_base = uint32_t(quarter * 32) << 16;
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 8) {
        float val[8];
        tc::tmem_ld8(acc + lane_base + uint32_t(c0), val);
        if (vin) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                val[i] += s_bias[c0 + i];
                if (a.relu) val[i] = fmaxf(val[i], 0.f);
            }
            const long o = v * a.out_stride + a.out_offset + c0;
            if (a.out_fp32) {
                float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.out) + o);
                dst[0] = make_float4(val[0], val[1], val[2], val[3]);
                dst[1] = make_float4(val[4], val[5], val[6], val[7]);
            } else {
                __align__(16) __nv_bfloat16 hv[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) hv[i] = __float2bfloat16_rn(val[i]);
                *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.out) + o) =
                    *reinterpret_cast<const uint4*>(hv);
            }
        }
    }
}

template <int N>
__global__ void __launch_bounds__(ConvWS<N>::kThreads) k_conv3_ws(ConvArgs a, int zt, int ring) {
    using W = ConvWS<N>;
    extern __shared__ uint8_t smem_raw[];
    // full[6], empty[6], acc_full[2], acc_empty[2], drain, probe
    __shared__ __align__(8) uint64_t bars[2 * W::kMaxRing + 6];
    __shared__ uint32_t tmem_slot;
    __shared__ int abort_flag;
    __shared__ float s_bias[N];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16;
    const int z0 = blockIdx.z * zt, z1 = min(a.D, z0 + zt);
    const int planes = z1 - z0;    // MMA / epilogue steps
    const int loads = planes + 2;  // halo planes z0 - 1 .. z1
    const int chunks = a.cin / 16;
    const uint32_t sbase = tc::smem_addr(smem);
    const uint32_t wbase = sbase;
    const uint32_t rbase = sbase + uint32_t(27 * N * a.cin * 2);
    const uint32_t plane_bytes = uint32_t(chunks * W::kPlane);
    const uint32_t b0 = tc::smem_addr(&bars[0]);
    auto full = [&](int s) { return b0 + uint32_t(8 * s); };
    auto empty = [&](int s) { return b0 + uint32_t(8 * (W::kMaxRing + s)); };
    auto acc_full = [&](int k) { return b0 + uint32_t(8 * (2 * W::kMaxRing + k)); };
    auto acc_empty = [&](int k) { return b0 + uint32_t(8 * (2 * W::kMaxRing + 2 + k)); };
    const uint32_t drain = b0 + uint32_t(8 * (2 * W::kMaxRing + 4));
    const uint32_t probe = b0 + uint32_t(8 * (2 * W::kMaxRing + 5));
    volatile int* abort_v = &abort_flag;

    if (tid == 0) {
        for (int s = 0; s < ring; ++s) {
            tc::mbar_init(full(s), 32);  // one cp.async arrival per producer lane
            tc::mbar_init(empty(s), 1);
        }
        tc::mbar_init(acc_full(0), 1);
        tc::mbar_init(acc_full(1), 1);
        tc::mbar_init(acc_empty(0), 4);  // one arrival per epilogue warp
        tc::mbar_init(acc_empty(1), 4);
        tc::mbar_init(drain, 1);
        tc::mbar_init(probe, 1);
        tc::fence_mbarrier_init();
        abort_flag = 0;
    }
    if (warp == 1) tc::tmem_alloc(tc::smem_addr(&tmem_slot), W::kCols);
    for (int i = tid; i < N; i += blockDim.x) s_bias[i] = a.bias ? a.bias[i] : 0.f;
    // all weights: (chunk, tap, co, half) segments of 16 bytes
    for (int i = tid; i < chunks * 27 * N * 2; i += blockDim.x) {
        const int half = i & 1, co = (i >> 1) % N, ct = (i >> 1) / N;  // ct = chunk * 27 + tap
        const int t = ct % 27, cc = ct / 27;
        const __nv_bfloat16* wsrc = a.w + (long(t) * N + co) * a.cin + cc * 16 + half * 8;
        tc::cp_async16(wbase + uint32_t(ct * N * 32 + (co >> 3) * 256 + half * 128 + (co & 7) * 16), wsrc, true);
    }
    tc::cp_async_commit();
    tc::cp_async_wait_all();
    tc::fence_proxy_async();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;
    bool ok = true;

    if (warp == 0) {
        // producer: halo plane zz = z0 - 1 + q into slot q % ring
        for (int q = 0; q < loads; ++q) {
            const int slot = q % ring;
            if (q >= ring) {  // the slot's previous plane q - ring is last read by the MMAs of step q - ring
                const bool got =
                    tc::mbar_wait_or_abort(empty(slot), uint32_t((q / ring - 1) & 1), kWaitLimit, abort_v);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
            }
            const int zz = z0 - 1 + q;
            const uint32_t dst = rbase + uint32_t(slot) * plane_bytes;
            for (int i = lane; i < chunks * 18 * 20; i += 32) {
                const int half = i & 1, v = (i >> 1) % 10, rc = (i >> 1) / 10;  // rc = chunk * 18 + ry
                const int ry = rc % 18, cc = rc / 18;
                const int x = x0 - 1 + v, y = y0 + ry - 1;
                const bool valid = x >= 0 && x < a.W && y >= 0 && y < a.H && zz >= 0 && zz < a.D;
                const __nv_bfloat16* src =
                    valid ? a.in + ((long(zz) * a.H + y) * a.W + x) * a.in_stride + cc * 16 + half * 8 : a.in;
                tc::cp_async16(dst + uint32_t(rc * 320 + half * 160 + v * 16), src, valid);
            }
            tc::cp_async_arrive(full(slot));
        }
        tc::cp_async_wait_all();
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = tc::instr_desc_bf16(128, N);
            const uint64_t a_desc = tc::smem_desc(rbase, 160, 320);
            const uint64_t b_desc = tc::smem_desc(wbase, 128, 256);
            for (int j = 0; j < planes && ok; ++j) {
                // planes j .. j + 2 (z - 1 .. z + 1) have landed; the first
                // two were waited for in earlier steps
                for (int q = (j == 0 ? 0 : j + 2); q <= j + 2 && ok; ++q) {
                    ok = a.wait_probe ? tc::mbar_wait_or_abort(probe, 0u, a.wait_probe, abort_v)
                                      : tc::mbar_wait_or_abort(full(q % ring), uint32_t((q / ring) & 1), kWaitLimit,
                                                               abort_v);
                }
                const int k = j & 1;
                if (ok && j >= 2)
                    ok = tc::mbar_wait_or_abort(acc_empty(k), uint32_t(((j - 2) >> 1) & 1), kWaitLimit, abort_v);
                if (!ok) break;
                tc::fence_proxy_async();  // cp.async data -> tensor core (async proxy)
                tc::tc_fence_after();
                const uint32_t dz_bytes[3] = {uint32_t(j % ring) * plane_bytes, uint32_t((j + 1) % ring) * plane_bytes,
                                              uint32_t((j + 2) % ring) * plane_bytes};
#pragma unroll 1
                for (int cc = 0; cc < chunks; ++cc)
                    issue_taps<N>(tmem + uint32_t(k) * W::kAcc1, a_desc + uint32_t(cc * (W::kPlane >> 4)), dz_bytes,
                                  b_desc + uint32_t(cc * 27 * N * 2), idesc, cc > 0);
                tc::mma_commit(acc_full(k));
                tc::mma_commit(empty(j % ring));  // plane j (z - 1) has no later reader
            }
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
    } else {
        // epilogue warps 2..5 -> TMEM lane quarters 2, 3, 0, 1
        const int quarter = warp & 3;
        for (int j = 0; j < planes; ++j) {
            const int k = j & 1;
            const bool got = tc::mbar_wait_or_abort(acc_full(k), uint32_t((j >> 1) & 1), kWaitLimit, abort_v);
            if (!__all_sync(0xffffffffu, got)) {
                ok = false;
                break;
            }
            tc::tc_fence_after();
            ws_epilogue<N>(a, tmem + uint32_t(k) * W::kAcc1, s_bias, x0, y0, z0 + j, quarter, lane);
            tc::tc_fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(acc_empty(k));
        }
    }
    if (!ok) {
        *abort_v = 1;
        if (lane == 0) atomicOr(a.error, 1u);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (tid == 32) {
        // every MMA this thread issued is complete before TMEM is freed
        tc::mma_commit(drain);
        if (!tc::mbar_wait(drain, 0u, kWaitLimit)) atomicOr(a.error, 2u);
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    if (warp == 1) tc::tmem_dealloc(tmem, W::kCols);
}

// Plane-window form of the z-marching convolution. The MMA's N dimension
// holds the output channels of three consecutive output planes: for input
// plane zi and in-plane tap (dy, dx), one MMA (M = 128 voxels, N = 3 cout,
// K = 16 channels) multiplies the input voxels shifted by (dy, dx) with the
// weights of taps (dz = -1, 0, +1; dy, dx) and accumulates into the TMEM
// columns of output planes zi + 1, zi and zi - 1, which lie next to each
// other: output plane z owns columns N (z1 + 1 - z) .. + N. So a CTA issues
// 9 MMAs of width 3N per input plane and chunk instead of 27 of width N per
// output plane, with every input plane staged once. An output plane is
// complete once the MMAs of the input plane above it have finished; its
// epilogue then runs while the next input plane's MMAs execute. The TMEM
// window is cleared first, so every MMA accumulates. With one 16-channel
// chunk the sum over the 27 taps runs in the same order as in k_conv3_zm
// (dz, dy, dx), and the results are the same; with several chunks the order
// is (dz, chunk, dy, dx) in place of (chunk, dz, dy, dx).
template <int N>
struct ConvWindow {
    static constexpr int kPlane = 18 * 320;
    static constexpr bool kSupported = 3 * N <= 256;
    __host__ __device__ static uint32_t cols(int zt) {
        const uint32_t need = uint32_t(N) * uint32_t(zt + 4);
        uint32_t c = 32;
        while (c < need) c <<= 1;
        return c;
    }
    static int smem(int cin, int ring) { return 27 * N * cin * 2 + ring * (cin / 16) * kPlane + 1024; }
    static bool fits(int cin, int ring, int zt) {
        return kSupported && smem(cin, ring) <= 200 * 1024 && cols(zt) <= 512;
    }
};

template <int N>
__global__ void __launch_bounds__(256) k_conv3_zn(ConvArgs a, int zt, int ring) {
    using Wd = ConvWindow<N>;
    constexpr int NW = 3 * N;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[3];
    __shared__ uint32_t tmem_slot;
    __shared__ float s_bias[N];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16;
    const int z0 = blockIdx.z * zt, z1 = min(a.D, z0 + zt);
    const int inputs = z1 - z0 + 2;  // input planes z0 - 1 .. z1
    const int chunks = a.cin / 16;
    const uint32_t ncols = Wd::cols(zt);
    const uint32_t sbase = tc::smem_addr(smem);
    const uint32_t wbase = sbase;
    const uint32_t rbase = sbase + uint32_t(27 * N * a.cin * 2);
    const uint32_t plane_bytes = uint32_t(chunks * Wd::kPlane);
    const uint32_t bar0 = tc::smem_addr(&bars[0]);  // commits of input planes alternate bar0, bar0 + 8
    const uint32_t probe = bar0 + 16;               // never arrived on (timeout test hook)

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), ncols);
    if (tid == 0) {
        tc::mbar_init(bar0, 1);
        tc::mbar_init(bar0 + 8, 1);
        tc::mbar_init(probe, 1);
        tc::fence_mbarrier_init();
    }
    for (int i = tid; i < N; i += blockDim.x) s_bias[i] = a.bias ? a.bias[i] : 0.f;
    // weights as B rows (j, co) = tap (j * 9 + s), co: [chunk][s][3N rows / 8][2][8][16 B]
    for (int i = tid; i < chunks * 9 * NW * 2; i += blockDim.x) {
        const int half = i & 1, row = (i >> 1) % NW, cs = (i >> 1) / NW;  // cs = chunk * 9 + s
        const int j = row / N, co = row - j * N, s = cs % 9, cc = cs / 9;
        const int t = j * 9 + s;
        const __nv_bfloat16* wsrc = a.w + (long(t) * N + co) * a.cin + cc * 16 + half * 8;
        tc::cp_async16(wbase + uint32_t(cs * NW * 32 + (row >> 3) * 256 + half * 128 + (row & 7) * 16), wsrc, true);
    }
    auto slot_of = [&](int q) { return uint32_t(q % ring) * plane_bytes; };
    // input plane q (zz = z0 - 1 + q, all chunks) into its ring slot; rows
    // outside the grid read as zero
    auto load_plane = [&](int q) {
        const int zz = z0 - 1 + q;
        const uint32_t slot = rbase + slot_of(q);
        for (int i = tid; i < chunks * 18 * 20; i += blockDim.x) {
            const int half = i & 1, v = (i >> 1) % 10, rc = (i >> 1) / 10;  // rc = chunk * 18 + ry
            const int ry = rc % 18, cc = rc / 18;
            const int x = x0 - 1 + v, y = y0 + ry - 1;
            const bool valid = x >= 0 && x < a.W && y >= 0 && y < a.H && zz >= 0 && zz < a.D;
            const __nv_bfloat16* src =
                valid ? a.in + ((long(zz) * a.H + y) * a.W + x) * a.in_stride + cc * 16 + half * 8 : a.in;
            tc::cp_async16(slot + uint32_t(rc * 320 + half * 160 + v * 16), src, valid);
        }
    };
    // group 0: the weights and input planes 0, 1; then one group per plane
    // until every slot is filled (planes 2 .. ring - 1)
    load_plane(0);
    load_plane(1);
    tc::cp_async_commit();
    for (int q = 2; q <= ring - 1; ++q) {
        if (q < inputs) load_plane(q);
        tc::cp_async_commit();
    }
    tc::tc_fence_before();
    __syncthreads();  // the TMEM allocation is visible
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;
    {
        // clear the accumulator window (warp w: the lanes of quarter w & 3,
        // the columns of half w >> 2)
        const uint32_t zero[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        const uint32_t half_cols = ncols / 2;
        for (uint32_t c = 0; c < half_cols; c += 8)
            tc::tmem_st8(tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(warp >> 2) * half_cols + c, zero);
    }
    tc::cp_async_wait_group<0>();  // the weights and the first ring planes have landed
    tc::fence_proxy_async();
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    constexpr uint32_t idesc = tc::instr_desc_bf16(128, NW);
    const uint64_t a_desc = tc::smem_desc(rbase, 160, 320);
    const uint64_t b_desc = tc::smem_desc(wbase, 128, 256);
    auto col_of = [&](int z) { return uint32_t(N * (z1 + 1 - z)); };  // output plane z's first column
    // one thread: the 9 x chunks MMAs of input plane q, committed to bar0 + 8 (q & 1)
    auto issue = [&](int q) {
        tc::tc_fence_after();
        const int zi = z0 - 1 + q;
        if (zi >= 0 && zi < a.D) {  // planes outside the grid are zero and add nothing
            const uint32_t d = tmem + col_of(zi + 1);
            const uint64_t ad = a_desc + (slot_of(q) >> 4);
#pragma unroll 1
            for (int cc = 0; cc < chunks; ++cc)
#pragma unroll
                for (int s = 0; s < 9; ++s) {
                    const int dy = s / 3, dx = s - 3 * dy;
                    tc::mma_bf16(d, ad + uint32_t(cc * (Wd::kPlane >> 4)) + uint32_t((dy * 320 + dx * 16) >> 4),
                                 b_desc + uint32_t((cc * 9 + s) * NW * 2), idesc, true);
                }
        }
        tc::mma_commit(bar0 + uint32_t(8 * (q & 1)));
    };
    bool ok = true;
    int commits[2] = {0, 0};  // per barrier, counted by every thread
    auto wait_commit = [&](int q) {
        const int k = q & 1;
        const bool mine = a.wait_probe ? tc::mbar_wait(probe, 0u, a.wait_probe)
                                       : tc::mbar_wait(bar0 + uint32_t(8 * k), uint32_t(commits[k] - 1) & 1u,
                                                       kWaitLimit);
        return __syncthreads_and(mine) != 0;
    };
    for (int q = 0; q < inputs; ++q) {
        // input plane q has landed (its group and all earlier ones)
        if (q >= 2) {
            // plane q + ring - 2 goes into the slot of plane q - 2, whose MMAs
            // completed (waited for in step q - 1); plane q >= ring was
            // requested in step q - ring + 2 (planes below ring were all in
            // the first groups), so all but the ring - 2 newest groups must land
            if (q + ring - 2 < inputs) load_plane(q + ring - 2);
            tc::cp_async_commit();
            if (ring == 6) tc::cp_async_wait_group<4>();
            else tc::cp_async_wait_group<2>();
            tc::fence_proxy_async();
            tc::tc_fence_before();
            __syncthreads();
        }
        if (tid == 0) issue(q);
        ++commits[q & 1];
        if (q >= 1) {
            // MMAs of input plane q - 1 complete: output plane z0 + q - 3 + 1
            // = zi(q) - 2 has all its contributions
            if (!wait_commit(q - 1)) {
                ok = false;
                break;
            }
            tc::tc_fence_after();
            const int zo = z0 - 1 + q - 2;
            if (zo >= z0 && zo < z1) conv_epilogue<N>(a, tmem + col_of(zo), s_bias, x0, y0, zo, warp, lane);
        }
    }
    if (ok) {
        // the last input plane's MMAs: output plane z1 - 1
        if (!wait_commit(inputs - 1)) {
            ok = false;
        } else {
            tc::tc_fence_after();
            const int zo = z1 - 1;
            if (zo >= z0) conv_epilogue<N>(a, tmem + col_of(zo), s_bias, x0, y0, zo, warp, lane);
        }
    }
    if (!ok) {
        if (tid == 0) atomicOr(a.error, 1u);
        // drain every commit still in flight, bounded
        bool drained = true;
        for (int k = 0; k < 2; ++k)
            if (commits[k] > 0) drained &= tc::mbar_wait(bar0 + uint32_t(8 * k), uint32_t(commits[k] - 1) & 1u, kWaitLimit);
        if (!drained) atomicOr(a.error, 2u);
        tc::cp_async_wait_all();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// The plane-window convolution fed by the TMA unit. The MMAs, their operands'
// values and their order are those of k_conv3_zn; what changes is how the
// operands reach shared memory and how the CTA synchronises:
//   - the layer's weights arrive in one bulk copy from their packed image
//     (launch_pack_window: the shared-memory layout of k_conv3_zn), and each
//     input plane as 2 x chunks tensor-map boxes of 8 channels x 10 x 18
//     voxels (zero outside the grid), each completing on the plane slot's
//     `full` mbarrier. The A operand of chunk c sits at [half][y][x][16 B]:
//     K halves 2944 bytes apart (LBO), 8-voxel rows 160 bytes apart (SBO);
//   - thread 0 issues plane q's MMAs once its slot is full and commits them
//     to cbar[q & 1]; every thread waits for the MMAs of plane q - 1, thread 0
//     refills their slot with plane q - 1 + ring, and the epilogue of the
//     output plane they completed runs. No block-wide barrier sits in the
//     march, so warps 1-7 drain plane q - 2 while thread 0 issues plane q.
// Every wait is bounded; a timeout sets the error flag and an abort flag that
// ends the other threads' waits, and thread 0 drains its MMAs and copies
// (bounded) before TMEM is freed and the CTA exits.
template <int N>
struct ConvTma {
    static constexpr int kHalf = 2944;           // one K half of a chunk's plane: 18 x 10 x 16 B, 128-byte padded
    static constexpr int kChunk = 2 * kHalf;     // one chunk of one plane
    static constexpr uint32_t kBox = 8 * 10 * 18 * 2;  // bytes of one box
    static constexpr int kMaxRing = 6;
    static int smem(int cin, int ring) { return 27 * N * cin * 2 + ring * (cin / 16) * kChunk + 1024; }
    static bool fits(int cin, int ring, int zt) {
        return ConvWindow<N>::kSupported && smem(cin, ring) <= 200 * 1024 && ConvWindow<N>::cols(zt) <= 512;
    }
};

template <int N>
__global__ void __launch_bounds__(256) k_conv3_zt(const __grid_constant__ CUtensorMap in_map, ConvArgs a, int zt,
                                                  int ring) {
    using Wd = ConvWindow<N>;
    using Tm = ConvTma<N>;
    constexpr int NW = 3 * N;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[Tm::kMaxRing + 4];  // full[ring], weights, cbar[2], probe
    __shared__ uint32_t tmem_slot;
    __shared__ float s_bias[N];
    __shared__ volatile int s_abort;
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16;
    const int z0 = blockIdx.z * zt, z1 = min(a.D, z0 + zt);
    const int inputs = z1 - z0 + 2;  // input planes z0 - 1 .. z1
    const int chunks = a.cin / 16;
    const uint32_t ncols = Wd::cols(zt);
    const uint32_t wbytes = uint32_t(27 * N * a.cin * 2);
    const uint32_t wbase = tc::smem_addr(smem);
    const uint32_t rbase = wbase + wbytes;
    const uint32_t plane_bytes = uint32_t(chunks * Tm::kChunk);
    const uint32_t full0 = tc::smem_addr(&bars[0]);  // slot r's barrier at full0 + 8 r
    const uint32_t wbar = tc::smem_addr(&bars[Tm::kMaxRing]);
    const uint32_t cbar0 = wbar + 8;                 // commits of input planes alternate cbar0, cbar0 + 8
    const uint32_t probe = wbar + 24;                // never arrived on (timeout test hook)
    const uint32_t tx_plane = uint32_t(chunks * 2) * Tm::kBox;

    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), ncols);
    if (tid == 0) {
        for (int r = 0; r < ring; ++r) tc::mbar_init(full0 + 8u * r, 1);
        tc::mbar_init(wbar, 1);
        tc::mbar_init(cbar0, 1);
        tc::mbar_init(cbar0 + 8, 1);
        tc::mbar_init(probe, 1);
        tc::fence_mbarrier_init();
        s_abort = 0;
    }
    for (int i = tid; i < N; i += blockDim.x) s_bias[i] = a.bias ? a.bias[i] : 0.f;
    tc::tc_fence_before();
    __syncthreads();  // barriers initialised, TMEM allocation visible
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;
    // input plane q (zz = z0 - 1 + q, all chunks, both K halves) into its
    // slot (thread 0; fills counted per slot for the drain)
    int filled[Tm::kMaxRing] = {0, 0, 0, 0, 0, 0};
    auto load_plane = [&](int q) {
        const uint32_t slot = rbase + uint32_t(q % ring) * plane_bytes;
        const uint32_t bar = full0 + 8u * uint32_t(q % ring);
        ++filled[q % ring];
        tc::mbar_expect_tx(bar, tx_plane);
        for (int cc = 0; cc < chunks; ++cc)
            for (int h = 0; h < 2; ++h)
                tc::tma_load_4d(slot + uint32_t(cc * Tm::kChunk + h * Tm::kHalf), &in_map, cc * 16 + h * 8, x0 - 1,
                                y0 - 1, z0 - 1 + q, bar);
    };
    if (tid == 0) {
        tc::mbar_expect_tx(wbar, wbytes);
        tc::bulk_load(wbase, a.w_window, wbytes, wbar);
        for (int q = 0; q < min(ring, inputs); ++q) load_plane(q);
    }
    {
        // clear the accumulator window (warp w: the lanes of quarter w & 3,
        // the columns of half w >> 2)
        const uint32_t zero[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        const uint32_t half_cols = ncols / 2;
        for (uint32_t c = 0; c < half_cols; c += 8)
            tc::tmem_st8(tmem + (uint32_t((warp & 3) * 32) << 16) + uint32_t(warp >> 2) * half_cols + c, zero);
    }
    tc::tc_fence_before();
    __syncthreads();  // the cleared window precedes every MMA
    tc::tc_fence_after();
    constexpr uint32_t idesc = tc::instr_desc_bf16(128, NW);
    const uint64_t a_desc = tc::smem_desc(rbase, Tm::kHalf, 160);
    const uint64_t b_desc = tc::smem_desc(wbase, 128, 256);
    auto col_of = [&](int z) { return uint32_t(N * (z1 + 1 - z)); };  // output plane z's first column
    int commits = 0;     // MMA commits issued (thread 0)
    bool ok = true;
    auto fail_wait = [&]() {
        s_abort = 1;
        atomicOr(a.error, 1u);
        ok = false;
    };
    for (int q = 0; q < inputs && ok; ++q) {
        if (tid == 0) {
            bool ready = q > 0 || tc::mbar_wait_or_abort(wbar, 0u, kWaitLimit, &s_abort);
            ready = ready && tc::mbar_wait_or_abort(full0 + 8u * uint32_t(q % ring), uint32_t(q / ring) & 1u,
                                                    kWaitLimit, &s_abort);
            if (!ready) {
                fail_wait();
            } else {
                tc::tc_fence_after();
                const int zi = z0 - 1 + q;
                if (zi >= 0 && zi < a.D) {  // planes outside the grid are zero and add nothing
                    const uint32_t d = tmem + col_of(zi + 1);
                    const uint64_t ad = a_desc + (uint32_t(q % ring) * plane_bytes >> 4);
#pragma unroll 1
                    for (int cc = 0; cc < chunks; ++cc)
#pragma unroll
                        for (int s = 0; s < 9; ++s) {
                            const int dy = s / 3, dx = s - 3 * dy;
                            tc::mma_bf16(d, ad + uint32_t(cc * (Tm::kChunk >> 4)) + uint32_t((dy * 160 + dx * 16) >> 4),
                                         b_desc + uint32_t((cc * 9 + s) * NW * 2), idesc, true);
                        }
                }
                tc::mma_commit(cbar0 + uint32_t(8 * (q & 1)));
                ++commits;
            }
        }
        if (q >= 1 && ok && !s_abort) {
            // MMAs of input plane q - 1 complete: output plane zi(q) - 2 has
            // all its contributions and slot (q - 1) % ring is free
            const int p = q - 1;
            const bool done = a.wait_probe
                                  ? tc::mbar_wait_or_abort(probe, 0u, a.wait_probe, &s_abort)
                                  : tc::mbar_wait_or_abort(cbar0 + uint32_t(8 * (p & 1)), uint32_t(p >> 1) & 1u,
                                                           kWaitLimit, &s_abort);
            if (!done) {
                fail_wait();
            } else {
                tc::tc_fence_after();
                if (tid == 0 && p + ring < inputs) load_plane(p + ring);
                const int zo = z0 - 1 + q - 2;
                if (zo >= z0 && zo < z1) conv_epilogue<N>(a, tmem + col_of(zo), s_bias, x0, y0, zo, warp, lane);
            }
        }
        if (s_abort) ok = false;
    }
    if (ok) {
        // the last input plane's MMAs: output plane z1 - 1
        const int p = inputs - 1;
        if (!tc::mbar_wait_or_abort(cbar0 + uint32_t(8 * (p & 1)), uint32_t(p >> 1) & 1u, kWaitLimit, &s_abort)) {
            fail_wait();
        } else {
            tc::tc_fence_after();
            const int zo = z1 - 1;
            if (zo >= z0) conv_epilogue<N>(a, tmem + col_of(zo), s_bias, x0, y0, zo, warp, lane);
        }
    }
    __syncthreads();
    if (s_abort && tid == 0) {
        // drain (bounded): the last commit covers every MMA issued before it,
        // and every slot's latest fill must land before the CTA exits
        bool drained = true;
        if (commits > 0)
            drained &= tc::mbar_wait(cbar0 + uint32_t(8 * ((commits - 1) & 1)), uint32_t((commits - 1) >> 1) & 1u,
                                     kWaitLimit);
        drained &= tc::mbar_wait(wbar, 0u, kWaitLimit);
        for (int r = 0; r < ring; ++r)  // the f-th fill of a slot completes its phase f - 1
            if (filled[r] > 0)
                drained &= tc::mbar_wait(full0 + 8u * uint32_t(r), uint32_t(filled[r] - 1) & 1u, kWaitLimit);
        if (!drained) atomicOr(a.error, 2u);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// Packs [27][cout][cin] weights into k_conv3_zn's shared-memory image: B rows
// (j, co) = tap j * 9 + s, co, as [chunk][s][3 cout / 8][2][8][16 B].
__global__ void k_pack_window(int cout, int cin, const __nv_bfloat16* __restrict__ w, __nv_bfloat16* __restrict__ out) {
    const int NW = 3 * cout;
    const long pieces = 27L * cout * cin / 8;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < pieces; i += long(gridDim.x) * blockDim.x) {
        const int half = int(i & 1), row = int((i >> 1) % NW);
        const long cs = (i >> 1) / NW;  // chunk * 9 + s
        const int j = row / cout, co = row - j * cout, sidx = int(cs % 9), cc = int(cs / 9);
        const int t = j * 9 + sidx;
        const uint4 v = *reinterpret_cast<const uint4*>(w + (long(t) * cout + co) * cin + cc * 16 + half * 8);
        const long byte = cs * NW * 32 + (row >> 3) * 256 + half * 128 + (row & 7) * 16;
        *reinterpret_cast<uint4*>(reinterpret_cast<uint8_t*>(out) + byte) = v;
    }
}

// ---- CUDA-core kernels -------------------------------------------------------

// Input features: channel 0 = b / scale (from the solver's red-black split RHS,
// minus the RHS mean), channel 1 = solid mask (0: fluid), channels 2..15 = 0.
__global__ void k_prep_input(int n, const float* __restrict__ b_split, const ProjControl* __restrict__ ctrl,
                             const float* __restrict__ scale, __nv_bfloat16* __restrict__ out) {
    const RBLayout L = rb_layout(n);
    const long V = long(n) * n * n;
    const float inv = 1.f / fmaxf(*scale, 1e-30f);
    const float bm = ctrl ? ctrl->rhs_mean_f : 0.f;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(v, n, n, x, y, z);
        const float bv = (b_split[rb_index(L, x, y, z)] - bm) * inv;
        __nv_bfloat16* o = out + v * 16;
        o[0] = __float2bfloat16_rn(bv);
#pragma unroll
        for (int c = 1; c < 16; ++c) o[c] = __float2bfloat16_rn(0.f);
    }
}

// Input features from a natural-layout FP32 field a (a coarse residual):
// channel 0 = (a - mean a) / scale, channels 1..15 = 0.
__global__ void k_prep_natural(long V, const float* __restrict__ a, const double* __restrict__ mean,
                               const float* __restrict__ scale, __nv_bfloat16* __restrict__ out) {
    const float inv = 1.f / fmaxf(*scale, 1e-30f);
    const float m = float(*mean);
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        __align__(16) __nv_bfloat16 h[8];
        h[0] = __float2bfloat16_rn((a[v] - m) * inv);
#pragma unroll
        for (int c = 1; c < 8; ++c) h[c] = __float2bfloat16_rn(0.f);
        uint4* o = reinterpret_cast<uint4*>(out + v * 16);
        o[0] = *reinterpret_cast<const uint4*>(h);
        o[1] = make_uint4(0u, 0u, 0u, 0u);
    }
}
__global__ void k_rms_natural(long V, const float* __restrict__ a, const double* __restrict__ mean,
                              double* __restrict__ partial) {
    __shared__ double s_sum[32];
    const double m = *mean;
    double acc = 0.0;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        const double d = double(a[v]) - m;
        acc += d * d;
    }
    const double s = block_sum(acc, s_sum);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// Root-mean-square of the mean-free RHS (FP64), the normalization scale.
__global__ void k_rms(int n, const float* __restrict__ b_split, const ProjControl* __restrict__ ctrl,
                      double* __restrict__ partial) {
    __shared__ double s_sum[32];
    const RBLayout L = rb_layout(n);
    const long V = long(n) * n * n;
    const float bm = ctrl ? ctrl->rhs_mean_f : 0.f;
    double acc = 0.0;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(v, n, n, x, y, z);
        const double bv = double(b_split[rb_index(L, x, y, z)] - bm);
        acc += bv * bv;
    }
    const double s = block_sum(acc, s_sum);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}
__global__ void k_rms_finish(const double* __restrict__ partial, int blocks, double count, float* scale) {
    __shared__ double s_sum[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) acc += partial[i];
    const double s = block_sum(acc, s_sum);
    if (threadIdx.x == 0) *scale = float(sqrt(s / count));
}

// 2x average pooling, channels-last BF16 (input dims even).
__global__ void k_avgpool2(int D, int H, int W, int C, const __nv_bfloat16* __restrict__ in, int in_stride,
                           __nv_bfloat16* __restrict__ out) {
    const int d = D / 2, h = H / 2, w = W / 2;
    const long total = long(d) * h * w * C;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long v = i / C;
        int x, y, z;
        decode(v, h, w, x, y, z);
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int xx = 2 * x + (k & 1), yy = 2 * y + ((k >> 1) & 1), zz = 2 * z + (k >> 2);
            s += __bfloat162float(in[((long(zz) * H + yy) * W + xx) * in_stride + c]);
        }
        out[v * C + c] = __float2bfloat16_rn(s * 0.125f);
    }
}

// Nearest 2x upsampling of a coarse tensor into channels [0, C) of a fine
// buffer with channel stride out_stride.
// Nearest 2x upsampling into the first C channels of a concatenation buffer,
// 8 channels (16 bytes) per thread (C, out_stride multiples of 8).
__global__ void k_upsample2(int d, int h, int w, int C, const __nv_bfloat16* __restrict__ in,
                            __nv_bfloat16* __restrict__ out, int out_stride) {
    const int D = 2 * d, H = 2 * h, W = 2 * w;
    const int C8 = C / 8;
    const long total = long(D) * H * W * C8;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C8) * 8;
        const long v = i / C8;
        int x, y, z;
        decode(v, H, W, x, y, z);
        *reinterpret_cast<uint4*>(out + v * out_stride + c) =
            *reinterpret_cast<const uint4*>(in + ((long(z / 2) * h + y / 2) * w + x / 2) * C + c);
    }
}

// 1x1 output head: p[v] = bias + sum_c w[c] * act[v, c] (FP32 out).
__global__ void k_head(long V, int C, const __nv_bfloat16* __restrict__ act, const float* __restrict__ w,
                       const float* __restrict__ bias, float* __restrict__ out) {
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        float s = bias[0];
        for (int c = 0; c < C; ++c) s += w[c] * __bfloat162float(act[v * C + c]);
        out[v] = s;
    }
}

// Warm start scale by the Galerkin condition on span{q}, q = p - mean p:
// alpha = (q . b) / (q . A q) minimises the A-norm error of alpha q against the
// exact pressure (A: the Neumann 7-point operator of the residual, b: the
// mean-free right-hand side). The network then only has to predict the shape
// of the pressure, and the guess is never worse than zero in the A-norm.
__global__ void k_galerkin_sums(int n, const float* __restrict__ p, const double* __restrict__ mean,
                                const float* __restrict__ b_split, const ProjControl* __restrict__ ctrl,
                                double* __restrict__ partial) {
    __shared__ double s_sum[32];
    const RBLayout L = rb_layout(n);
    const long V = long(n) * n * n;
    const double m = *mean;
    const float bm = ctrl->rhs_mean_f;
    double num = 0.0, den = 0.0;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(v, n, n, x, y, z);
        const double q = double(p[v]) - m;
        double aq = 0.0;
        int nb = 0;
        auto add = [&](long u) {
            aq -= double(p[u]) - m;
            ++nb;
        };
        if (x > 0) add(v - 1);
        if (x + 1 < n) add(v + 1);
        if (y > 0) add(v - n);
        if (y + 1 < n) add(v + n);
        if (z > 0) add(v - long(n) * n);
        if (z + 1 < n) add(v + long(n) * n);
        aq += double(nb) * q;
        num += q * double(b_split[rb_index(L, x, y, z)] - bm);
        den += q * aq;
    }
    const double sn = block_sum(num, s_sum);
    const double sd = block_sum(den, s_sum);
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = sn;
        partial[2 * blockIdx.x + 1] = sd;
    }
}
__global__ void k_galerkin_finish(const double* __restrict__ partial, int blocks, double* __restrict__ alpha) {
    __shared__ double s_sum[32];
    double num = 0.0, den = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
        num += partial[2 * i];
        den += partial[2 * i + 1];
    }
    const double sn = block_sum(num, s_sum);
    const double sd = block_sum(den, s_sum);
    if (threadIdx.x == 0) *alpha = (sd > 0.0 && isfinite(sn / sd)) ? sn / sd : 0.0;
}

// Warm start into the solver's split iterate: x = alpha * (p - mean p).
__global__ void k_store_warm_start(int n, const float* __restrict__ p, const double* __restrict__ alpha,
                                   const double* __restrict__ mean, float* __restrict__ x_split) {
    const RBLayout L = rb_layout(n);
    const long V = long(n) * n * n;
    const double a = *alpha, m = *mean;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(v, n, n, x, y, z);
        x_split[rb_index(L, x, y, z)] = float(a * (double(p[v]) - m));
    }
}
__global__ void k_store_warm_start64(int n, const float* __restrict__ p, const double* __restrict__ alpha,
                                     const double* __restrict__ mean, double* __restrict__ x_split) {
    const RBLayout L = rb_layout(n);
    const long V = long(n) * n * n;
    const double a = *alpha, m = *mean;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(v, n, n, x, y, z);
        x_split[rb_index(L, x, y, z)] = a * (double(p[v]) - m);
    }
}

// Deterministic FP64 mean of an FP32 array (partials then one block).
__global__ void k_sum(long V, const float* __restrict__ a, double* __restrict__ partial) {
    __shared__ double s_sum[32];
    double acc = 0.0;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x)
        acc += double(a[v]);
    const double s = block_sum(acc, s_sum);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}
__global__ void k_mean_finish(const double* __restrict__ partial, int blocks, double count, double* mean) {
    __shared__ double s_sum[32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) acc += partial[i];
    const double s = block_sum(acc, s_sum);
    if (threadIdx.x == 0) *mean = s / count;
}

// Training target: zero-mean pressure / scale from the solver's split iterate.
__global__ void k_target(int n, const float* __restrict__ p_split, const ProjControl* __restrict__ ctrl,
                         const float* __restrict__ scale, float* __restrict__ target) {
    const RBLayout L = rb_layout(n);
    const long V = long(n) * n * n;
    const float pm = ctrl->p_mean_f;
    const float inv = 1.f / fmaxf(*scale, 1e-30f);
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        int x, y, z;
        decode(v, n, n, x, y, z);
        target[v] = (p_split[rb_index(L, x, y, z)] - pm) * inv;
    }
}

// Scale-invariant loss: with q = p - mean p and r = t - mean t,
//   L = min_c |c q - r|^2 / |r|^2 = 1 - (q.r)^2 / (|q|^2 |r|^2),
// the relative squared error left after the best scaling of the prediction
// (the warm start applies its own scale). Per-block sums of q.r, q.q, r.r.
__global__ void k_loss_sums(long V, const float* __restrict__ p, const float* __restrict__ t,
                            const double* __restrict__ means, double* __restrict__ partial) {
    __shared__ double s_sum[32];
    const double mp = means[0], mt = means[1];
    double qr = 0.0, qq = 0.0, rr = 0.0;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        const double q = double(p[v]) - mp, r = double(t[v]) - mt;
        qr += q * r;
        qq += q * q;
        rr += r * r;
    }
    const double a = block_sum(qr, s_sum);
    const double b = block_sum(qq, s_sum);
    const double c = block_sum(rr, s_sum);
    if (threadIdx.x == 0) {
        partial[3 * blockIdx.x] = a;
        partial[3 * blockIdx.x + 1] = b;
        partial[3 * blockIdx.x + 2] = c;
    }
}
// scalars: [0] mean p, [1] mean t, [2] loss, [3] coefficient of r, [4] of q.
__global__ void k_loss_finish(const double* __restrict__ partial, int blocks, double* __restrict__ scalars) {
    __shared__ double s_sum[32];
    double qr = 0.0, qq = 0.0, rr = 0.0;
    for (int i = threadIdx.x; i < blocks; i += blockDim.x) {
        qr += partial[3 * i];
        qq += partial[3 * i + 1];
        rr += partial[3 * i + 2];
    }
    const double a = block_sum(qr, s_sum);
    const double b = block_sum(qq, s_sum);
    const double c = block_sum(rr, s_sum);
    if (threadIdx.x == 0) {
        const bool ok = b > 0.0 && c > 0.0;
        scalars[2] = ok ? 1.0 - a * a / (b * c) : 1.0;
        // dL/dq = -2 (q.r)/(|q|^2 |r|^2) r + 2 (q.r)^2/(|q|^4 |r|^2) q; it has
        // zero mean, so it is also dL/dp.
        scalars[3] = ok ? -2.0 * a / (b * c) : 0.0;
        scalars[4] = ok ? 2.0 * a * a / (b * b * c) : 0.0;
    }
}
__global__ void k_loss_grad(long V, const float* __restrict__ p, const float* __restrict__ t,
                            const double* __restrict__ scalars, float* __restrict__ grad) {
    const double mp = scalars[0], mt = scalars[1], cr = scalars[3], cq = scalars[4];
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x)
        grad[v] = float(cr * (double(t[v]) - mt) + cq * (double(p[v]) - mp));
}

__global__ void k_head_backward(long V, int C, const __nv_bfloat16* __restrict__ act, const float* __restrict__ w,
                                const float* __restrict__ g, __nv_bfloat16* __restrict__ dact,
                                float* __restrict__ dw, float* __restrict__ db) {
    float lw[64], lb = 0.f;
    for (int c = 0; c < C; ++c) lw[c] = 0.f;
    for (long v = long(blockIdx.x) * blockDim.x + threadIdx.x; v < V; v += long(gridDim.x) * blockDim.x) {
        const float gv = g[v];
        lb += gv;
        for (int c = 0; c < C; ++c) {
            const float a = __bfloat162float(act[v * C + c]);
            lw[c] += gv * a;
            dact[v * C + c] = __float2bfloat16_rn(a > 0.f ? gv * w[c] : 0.f);
        }
    }
    for (int c = 0; c < C; ++c) atomicAdd(&dw[c], lw[c]);
    atomicAdd(db, lb);
}

// ReLU backward in place on a gradient with channel stride: g *= (act > 0).
__global__ void k_relu_mask(long V, int C, const __nv_bfloat16* __restrict__ act, int act_stride, int act_offset,
                            __nv_bfloat16* __restrict__ g, int g_stride, int g_offset) {
    const long total = V * C;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long v = i / C;
        if (!(__bfloat162float(act[v * act_stride + act_offset + c]) > 0.f))
            g[v * g_stride + g_offset + c] = __float2bfloat16_rn(0.f);
    }
}

// Bias gradient: db[co] += sum_v g[v, co].
__global__ void k_bias_grad(long V, int C, const __nv_bfloat16* __restrict__ g, int g_stride, int g_offset,
                            float* __restrict__ db) {
    __shared__ float s_acc[128];
    if (threadIdx.x < C) s_acc[threadIdx.x] = 0.f;
    __syncthreads();
    const int c = threadIdx.x % C;
    const int lanes = blockDim.x / C;
    const int l = threadIdx.x / C;
    float acc = 0.f;
    if (l < lanes)
        for (long v = long(blockIdx.x) * lanes + l; v < V; v += long(gridDim.x) * lanes)
            acc += __bfloat162float(g[v * g_stride + g_offset + c]);
    if (l < lanes) atomicAdd(&s_acc[c], acc);
    __syncthreads();
    if (threadIdx.x < C) atomicAdd(&db[threadIdx.x], s_acc[threadIdx.x]);
}

// Weight gradient of a 3x3x3 convolution on CUDA cores:
// dw[tap][co][ci] += sum_v g[v, co] * x[v + tap, ci]. One block per
// (tap, 16-co block, 16-ci block, voxel chunk); thread (co, ci) accumulates.
__global__ void __launch_bounds__(256) k_conv3_wgrad(WGradArgs a) {
    __shared__ float sg[64][17];
    __shared__ float sx[64][17];
    const int tap = blockIdx.y;
    const int cob = blockIdx.z % (a.cout / 16), cib = blockIdx.z / (a.cout / 16);
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    const long V = long(a.D) * a.H * a.W;
    const long chunk = (V + gridDim.x - 1) / gridDim.x;
    const long v_begin = long(blockIdx.x) * chunk, v_end = min(V, v_begin + chunk);
    const int tco = threadIdx.x >> 4, tci = threadIdx.x & 15;
    float acc = 0.f;
    for (long v0 = v_begin; v0 < v_end; v0 += 64) {
        // stage 64 voxels x 16 channels of g and of the shifted input
        for (int i = threadIdx.x; i < 64 * 16; i += 256) {
            const int r = i >> 4, c = i & 15;
            const long v = v0 + r;
            float gv = 0.f, xv = 0.f;
            if (v < v_end) {
                gv = __bfloat162float(a.g[v * a.g_stride + a.g_offset + cob * 16 + c]);
                int x, y, z;
                decode(v, a.H, a.W, x, y, z);
                const int xs = x + dx, ys = y + dy, zs = z + dz;
                if (xs >= 0 && xs < a.W && ys >= 0 && ys < a.H && zs >= 0 && zs < a.D)
                    xv = __bfloat162float(a.x[((long(zs) * a.H + ys) * a.W + xs) * a.x_stride + cib * 16 + c]);
            }
            sg[r][c] = gv;
            sx[r][c] = xv;
        }
        __syncthreads();
#pragma unroll 8
        for (int r = 0; r < 64; ++r) acc += sg[r][tco] * sx[r][tci];
        __syncthreads();
    }
    atomicAdd(&a.dw[(long(tap) * a.cout + cob * 16 + tco) * a.cin + cib * 16 + tci], acc);
}

// Weight gradient on the tensor cores. dW[t][co][ci] = sum over voxels v of
// g[v][co] x[v + t][ci], written as sum over v' of g[v' - t][co] x[v'][ci], is
// a GEMM per CTA: M = 128 rows (8 taps x 16 output channels of one chunk), N
// = cin, K = the voxels of the CTA's range. Shared memory holds, per stage
// of 64 voxels, A[(tap, co)][v'] = g[v' - t][co] (zero where v' - t leaves
// the grid) and B[ci][v'] = x[v'][ci], both in the canonical K-major layout
// without swizzle ([8-row group][8-voxel chunk][8 rows][16 B]: LBO 128 B, SBO
// 1024 B), staged by all threads (each voxel's channels scattered down one K
// column); one thread issues the 4 MMAs (K = 16) of a stage into the FP32
// TMEM accumulator, two stages alternate on commit barriers. The epilogue
// adds the accumulator to dW with FP32 atomics, as the CUDA-core form does.
struct WGradTc {
    static constexpr int kK = 64;                 // voxels per stage
    static constexpr int kA = 128 * kK * 2;       // 16 KB
    __host__ __device__ static int b_bytes(int cin) { return cin * kK * 2; }
    __host__ __device__ static int stage(int cin) { return kA + b_bytes(cin); }
    static int smem(int cin) { return 2 * stage(cin) + 1024; }
};

__device__ __forceinline__ uint32_t kmajor_offset(int row, int k) {
    return uint32_t((row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__global__ void __launch_bounds__(256) k_conv3_wgrad_tc(WGradArgs a, long chunk) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t bars[2];
    __shared__ uint32_t tmem_slot;
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int group = blockIdx.y;                     // taps 8 group .. 8 group + 7
    const int cob = blockIdx.z;                       // output channels 16 cob .. + 15
    const long V = long(a.D) * a.H * a.W;
    const long v_begin = long(blockIdx.x) * chunk, v_end = min(V, v_begin + chunk);
    const int cin = a.cin;
    const uint32_t ncols = cin <= 32 ? 32u : (cin <= 64 ? 64u : 128u);
    const uint32_t sbase = tc::smem_addr(smem);
    const uint32_t bar0 = tc::smem_addr(&bars[0]);
    if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tmem_slot), ncols);
    if (tid == 0) {
        tc::mbar_init(bar0, 1);
        tc::mbar_init(bar0 + 8, 1);
        tc::fence_mbarrier_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = tmem_slot;
    const uint32_t idesc = tc::instr_desc_bf16(128, cin);
    int issued[2] = {0, 0};
    bool ok = true;
    int s_idx = 0;
    for (long k0 = v_begin; k0 < v_end; k0 += WGradTc::kK, s_idx ^= 1) {
        uint8_t* st = smem + s_idx * WGradTc::stage(cin);
        const uint32_t sa = sbase + uint32_t(s_idx * WGradTc::stage(cin));
        // the MMAs that last read this stage must be done
        if (issued[s_idx] > 0) {
            const bool mine = tc::mbar_wait(bar0 + 8u * s_idx, uint32_t(issued[s_idx] - 1) & 1u, kWaitLimit);
            if (!__syncthreads_and(mine)) {
                ok = false;
                break;
            }
        }
        // A: (tap j, voxel k) -> 16 channels of g at v' - t
        for (int i = tid; i < 8 * WGradTc::kK; i += blockDim.x) {
            const int j = i / WGradTc::kK, k = i - j * WGradTc::kK;
            const int t = group * 8 + j;
            const long v = k0 + k;
            uint4 lo = make_uint4(0, 0, 0, 0), hi = lo;
            if (t < 27 && v < v_end) {
                int x, y, z;
                decode(v, a.H, a.W, x, y, z);
                const int xs = x - (t % 3 - 1), ys = y - ((t / 3) % 3 - 1), zs = z - (t / 9 - 1);
                if (xs >= 0 && xs < a.W && ys >= 0 && ys < a.H && zs >= 0 && zs < a.D) {
                    const uint4* src = reinterpret_cast<const uint4*>(
                        a.g + ((long(zs) * a.H + ys) * a.W + xs) * a.g_stride + a.g_offset + cob * 16);
                    lo = src[0];
                    hi = src[1];
                }
            }
            const uint16_t* e0 = reinterpret_cast<const uint16_t*>(&lo);
            const uint16_t* e1 = reinterpret_cast<const uint16_t*>(&hi);
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                *reinterpret_cast<uint16_t*>(st + kmajor_offset(j * 16 + c, k)) = e0[c];
                *reinterpret_cast<uint16_t*>(st + kmajor_offset(j * 16 + 8 + c, k)) = e1[c];
            }
        }
        // B: (8-channel group, voxel k) -> x at v'
        uint8_t* sb = st + WGradTc::kA;
        for (int i = tid; i < (cin / 8) * WGradTc::kK; i += blockDim.x) {
            const int cg = i / WGradTc::kK, k = i - cg * WGradTc::kK;
            const long v = k0 + k;
            uint4 val = make_uint4(0, 0, 0, 0);
            if (v < v_end) val = *reinterpret_cast<const uint4*>(a.x + v * a.x_stride + cg * 8);
            const uint16_t* e = reinterpret_cast<const uint16_t*>(&val);
#pragma unroll
            for (int c = 0; c < 8; ++c) *reinterpret_cast<uint16_t*>(sb + kmajor_offset(cg * 8 + c, k)) = e[c];
        }
        tc::fence_proxy_async();  // generic-proxy stores visible to the tensor core
        tc::tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc::tc_fence_after();
            const uint64_t ad = tc::smem_desc(sa, 128, 1024);
            const uint64_t bd = tc::smem_desc(sa + WGradTc::kA, 128, 1024);
#pragma unroll
            for (int kk = 0; kk < WGradTc::kK / 16; ++kk)
                tc::mma_bf16(tmem, ad + uint32_t(kk * 16), bd + uint32_t(kk * 16), idesc, k0 > v_begin || kk > 0);
            tc::mma_commit(bar0 + 8u * s_idx);
        }
        ++issued[s_idx];
    }
    // the last commit of each stage covers every earlier MMA
    bool drained = true;
    for (int k = 0; k < 2; ++k)
        if (issued[k] > 0) drained &= tc::mbar_wait(bar0 + 8u * k, uint32_t(issued[k] - 1) & 1u, kWaitLimit);
    ok = __syncthreads_and(ok && drained) != 0;
    tc::tc_fence_after();
    if (ok && v_begin < v_end) {
        // rows (tap j, co) on TMEM lanes; columns ci, half of them per warp pair
        const int q = warp & 3, hlf = warp >> 2;
        const int row = q * 32 + lane;
        const int t = group * 8 + row / 16, co = cob * 16 + (row & 15);
        const int half = cin / 2;
        for (int c0 = hlf * half; c0 < (hlf + 1) * half; c0 += 8) {
            float val[8];
            tc::tmem_ld8(tmem + (uint32_t(q * 32) << 16) + uint32_t(c0), val);
            if (t < 27) {
#pragma unroll
                for (int c = 0; c < 8; ++c) atomicAdd(&a.dw[(long(t) * a.cout + co) * cin + c0 + c], val[c]);
            }
        }
    } else if (!ok && tid == 0 && a.error) {
        atomicOr(a.error, drained ? 1u : 3u);
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// Flip and transpose 3x3x3 weights for the input-gradient convolution:
// wt[26 - tap][ci][co] = w[tap][co][ci] (BF16).
__global__ void k_flip_weights(int cout, int cin, const __nv_bfloat16* __restrict__ w,
                               __nv_bfloat16* __restrict__ wt) {
    const long total = 27L * cout * cin;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int ci = int(i % cin);
        const long r = i / cin;
        const int co = int(r % cout);
        const int tap = int(r / cout);
        wt[(long(26 - tap) * cin + ci) * cout + co] = w[i];
    }
}

// avgpool backward: d_in[fine] = d_out[coarse] / 8 (into channels with stride).
__global__ void k_avgpool2_backward(int D, int H, int W, int C, const __nv_bfloat16* __restrict__ dout,
                                    __nv_bfloat16* __restrict__ din, int din_stride, int din_offset, int add) {
    const long total = long(D) * H * W * C;
    const int h = H / 2, w = W / 2;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long v = i / C;
        int x, y, z;
        decode(v, H, W, x, y, z);
        float g = __bfloat162float(dout[((long(z / 2) * h + y / 2) * w + x / 2) * C + c]) * 0.125f;
        __nv_bfloat16& o = din[v * din_stride + din_offset + c];
        if (add) g += __bfloat162float(o);
        o = __float2bfloat16_rn(g);
    }
}

// upsample backward: d_coarse[c] = sum of the 8 fine gradients of channel c.
__global__ void k_upsample2_backward(int d, int h, int w, int C, const __nv_bfloat16* __restrict__ dfine,
                                     int fine_stride, __nv_bfloat16* __restrict__ dcoarse) {
    const long total = long(d) * h * w * C;
    const int H = 2 * h, W = 2 * w;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += long(gridDim.x) * blockDim.x) {
        const int c = int(i % C);
        const long v = i / C;
        int x, y, z;
        decode(v, h, w, x, y, z);
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int xx = 2 * x + (k & 1), yy = 2 * y + ((k >> 1) & 1), zz = 2 * z + (k >> 2);
            s += __bfloat162float(dfine[((long(zz) * H + yy) * W + xx) * fine_stride + c]);
        }
        dcoarse[v * C + c] = __float2bfloat16_rn(s);
    }
}

// Adam (decoupled weight decay off), FP32 master weights, BF16 copy.
__global__ void k_adam(long count, float* __restrict__ w, float* __restrict__ m, float* __restrict__ vv,
                       const float* __restrict__ g, __nv_bfloat16* __restrict__ wb, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += long(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * vv[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        vv[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void k_to_bf16(long count, const float* __restrict__ a, __nv_bfloat16* __restrict__ b) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += long(gridDim.x) * blockDim.x)
        b[i] = __float2bfloat16_rn(a[i]);
}

int blocks_for(long count) { return int(std::max<long>(1, std::min<long>((count + 255) / 256, 148L * 16))); }

// Streaming multiprocessors of the current device.
int device_sm_count() {
    int dev = 0, sms = 0;
    VB_CUDA(cudaGetDevice(&dev));
    VB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    return sms;
}

// CTAs of 256 threads that one SM holds at once with `smem` bytes of dynamic
// shared memory: 228 KB per SM, 1 KB reserved per CTA plus its static shared
// memory (barriers, bias; under 512 bytes), 64 K registers at up to 40 per
// thread, 8 CTAs of 256 threads.
int resident_ctas(int smem) {
    constexpr int kSmemPerSm = 228 * 1024, kPerCta = 1024 + 512;
    return std::max(1, std::min({8, 65536 / (256 * 40), kSmemPerSm / (smem + kPerCta)}));
}

// Shared memory bounds the blocks per SM, so the tensor memory the blocks of
// one launch allocate fits in 512 columns: k_conv3_tc at most 7 x 32, 5 x 32,
// 3 x 64 or 2 x 128 (N = 16, 32, 64, 96); k_conv3_zm, with two accumulators,
// at most 6 x 32, 4 x 64, 3 x 128, 2 x 128 or 2 x 256 (N = 16, 32, 48, 64, 96).
template <int N>
void configure_n() {
    VB_CUDA(cudaFuncSetAttribute(k_conv3_tc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 ConvTile<N>::kSmemMax));
    VB_CUDA(cudaFuncSetAttribute(k_conv3_zm<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    VB_CUDA(cudaFuncSetAttribute(k_conv3_ws<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    if constexpr (ConvWindow<N>::kSupported) {
        VB_CUDA(cudaFuncSetAttribute(k_conv3_zn<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        VB_CUDA(cudaFuncSetAttribute(k_conv3_zt<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    }
}

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q);
        return (e == cudaSuccess && q == cudaDriverEntryPointSuccess)
                   ? reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f)
                   : nullptr;
    }();
    if (!fn) fail(VAPOR_RUNTIME_ERROR, "cuTensorMapEncodeTiled is not available from the CUDA driver");
    return fn;
}

// 4D map (channel, x, y, z) over a channels-last BF16 activation with
// in_stride channels per voxel; box = 8 channels x 10 x 18 x 1 (one K half of
// one 16-channel chunk of a halo plane).
CUtensorMap activation_map(const ConvArgs& a) {
    CUtensorMap map;
    const cuuint64_t dims[4] = {cuuint64_t(a.in_stride), cuuint64_t(a.W), cuuint64_t(a.H), cuuint64_t(a.D)};
    const cuuint64_t row = cuuint64_t(a.in_stride) * 2;
    const cuuint64_t strides[3] = {row, row * cuuint64_t(a.W), row * cuuint64_t(a.W) * cuuint64_t(a.H)};
    const cuuint32_t box[4] = {8, 10, 18, 1};
    const cuuint32_t elem[4] = {1, 1, 1, 1};
    const CUresult r = tensor_map_encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(a.in),
                                            dims, strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) fail(VAPOR_RUNTIME_ERROR, "cuTensorMapEncodeTiled failed for a convolution input");
    return map;
}

// Resident CTAs per SM of the warp-specialised convolution: shared memory,
// threads, and the 512 TMEM columns (two accumulators per CTA).
template <int N>
int resident_ws(int smem) {
    constexpr int kSmemPerSm = 228 * 1024, kPerCta = 1024 + 512;
    return std::max(1, std::min({2048 / ConvWS<N>::kThreads, 512 / int(ConvWS<N>::kCols),
                                 kSmemPerSm / (smem + kPerCta)}));
}

template <int N>
void launch_conv_n(const ConvArgs& a, cudaStream_t s) {
    if (a.cin % 16 != 0 || a.in_stride % 8 != 0 || a.out_stride % 8 != 0 || a.out_offset % 8 != 0)
        fail(VAPOR_INVALID_ARGUMENT, "convolution channel counts and strides must be multiples of 16 / 8");
    const unsigned gx = unsigned((a.W + 7) / 8), gy = unsigned((a.H + 15) / 16);
    count_launch();
    const int kind = g_conv_kind.load();
    bool done = false;
    if constexpr (ConvWindow<N>::kSupported) {
        // the TMA-fed form: packed weights, a 16-byte aligned input, and a
        // grid at least as wide as the 10 x 18 box
        const bool tma = kind == 3 && a.w_window != nullptr && ConvTma<N>::fits(a.cin, 3, 2) && a.W >= 10 &&
                         a.H >= 18 && (reinterpret_cast<uintptr_t>(a.in) & 15) == 0;
        if (tma) {
            // planes per CTA and ring depth: the pair that minimises waves x
            // (planes + 2), the input planes a CTA multiplies; resident CTAs
            // by shared memory and by TMEM columns (512 per SM); on ties the
            // deeper ring
            const int sms = device_sm_count();
            int best = 2, best_ring = 3;
            long best_cost = -1;
            for (int ring : {6, 4, 3})
                for (int zt : {2, 4, 6, 8, 12, 16}) {
                    if (!ConvTma<N>::fits(a.cin, ring, zt)) continue;
                    const int by_smem = std::max(1, (228 * 1024) / (ConvTma<N>::smem(a.cin, ring) + 1536));
                    const int by_tmem = int(512 / ConvWindow<N>::cols(zt));
                    const long slots = long(std::max(1, std::min({by_smem, by_tmem, 8}))) * sms;
                    const long ctas = long(gx) * gy * ((a.D + zt - 1) / zt);
                    const long cost = ((ctas + slots - 1) / slots) * (std::min(zt, a.D) + 2);
                    if (best_cost < 0 || cost < best_cost) {
                        best_cost = cost;
                        best = zt;
                        best_ring = ring;
                    }
                }
            const CUtensorMap map = activation_map(a);
            const dim3 grid(gx, gy, unsigned((a.D + best - 1) / best));
            k_conv3_zt<N><<<grid, 256, ConvTma<N>::smem(a.cin, best_ring), s>>>(map, a, best, best_ring);
            done = true;
        } else if (kind == 2 && ConvWindow<N>::fits(a.cin, 4, 2)) {
        // planes per CTA: the count that minimises waves x (planes + 2), the
        // input planes a CTA multiplies; resident CTAs by shared memory and
        // by TMEM columns (512 per SM)
        const int ring = ConvWindow<N>::fits(a.cin, 6, 2) ? 6 : 4;
        const int sms = device_sm_count();
        int best = 2;
        long best_cost = -1;
        for (int zt : {2, 4, 6, 8, 12, 16}) {
            if (!ConvWindow<N>::fits(a.cin, ring, zt)) continue;
            const int by_smem = std::max(1, (228 * 1024) / (ConvWindow<N>::smem(a.cin, ring) + 1536));
            const int by_tmem = int(512 / ConvWindow<N>::cols(zt));
            const long slots = long(std::max(1, std::min({by_smem, by_tmem, 8}))) * sms;
            const long ctas = long(gx) * gy * ((a.D + zt - 1) / zt);
            const long cost = ((ctas + slots - 1) / slots) * (std::min(zt, a.D) + 2);
            if (best_cost < 0 || cost < best_cost) {
                best_cost = cost;
                best = zt;
            }
        }
        const dim3 grid(gx, gy, unsigned((a.D + best - 1) / best));
        k_conv3_zn<N><<<grid, 256, ConvWindow<N>::smem(a.cin, ring), s>>>(a, best, ring);
        done = true;
        }
    }
    if (done) {
    } else if (kind == 1 && ConvWS<N>::fits(a.cin, 4)) {
        // planes per CTA: the smallest power of two (at least 2, up to 16)
        // whose grid runs in one wave of resident CTAs; the 6-plane ring when
        // it fits without lowering the resident count
        const int ring = (ConvWS<N>::fits(a.cin, 6) &&
                          resident_ws<N>(ConvWS<N>::smem(a.cin, 6)) == resident_ws<N>(ConvWS<N>::smem(a.cin, 4)))
                             ? 6 : 4;
        const long slots = long(resident_ws<N>(ConvWS<N>::smem(a.cin, ring))) * device_sm_count();
        int zt = 2;
        while (zt < 16 && long(gx) * gy * ((a.D + zt - 1) / zt) > slots) zt <<= 1;
        const dim3 grid(gx, gy, unsigned((a.D + zt - 1) / zt));
        k_conv3_ws<N><<<grid, ConvWS<N>::kThreads, ConvWS<N>::smem(a.cin, ring), s>>>(a, zt, ring);
    } else if (ConvMarch<N>::fits(a.cin, 4)) {
        // planes per CTA: the smallest power of two (up to 16) whose grid runs
        // in one wave of resident CTAs; the 6-plane ring when it fits, keeps
        // that plane count and the CTAs march at least 4 planes
        auto planes_for = [&](int ring) {
            const long slots = long(resident_ctas(ConvMarch<N>::smem(a.cin, ring))) * device_sm_count();
            int zt = 1;
            while (zt < 16 && long(gx) * gy * ((a.D + zt - 1) / zt) > slots) zt <<= 1;
            return zt;
        };
        const int zt = planes_for(4);
        const int ring = (zt >= 4 && ConvMarch<N>::fits(a.cin, 6) && planes_for(6) == zt) ? 6 : 4;
        const dim3 grid(gx, gy, unsigned((a.D + zt - 1) / zt));
        k_conv3_zm<N><<<grid, 256, ConvMarch<N>::smem(a.cin, ring), s>>>(a, zt, ring);
    } else {
        const dim3 grid(gx, gy, unsigned(a.D));
        k_conv3_tc<N><<<grid, 256, ConvTile<N>::smem(a.cin / 16), s>>>(a);
    }
}

}  // namespace

void set_conv_kernel(int kind) {
    if (kind < 0 || kind > 3) fail(VAPOR_INVALID_ARGUMENT, "convolution kernel: 0, 1, 2 or 3");
    g_conv_kind.store(kind);
}

void configure_conv_kernels() {
    VB_CUDA(cudaFuncSetAttribute(k_conv3_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, WGradTc::smem(96)));
    configure_n<16>();
    configure_n<32>();
    configure_n<48>();
    configure_n<64>();
    configure_n<96>();
}

void launch_pack_window(int cout, int cin, const __nv_bfloat16* w, __nv_bfloat16* packed, cudaStream_t s) {
    count_launch();
    k_pack_window<<<blocks_for(27L * cout * cin / 8), 256, 0, s>>>(cout, cin, w, packed);
}

void launch_conv3(const ConvArgs& a, int cout, cudaStream_t s) {
    switch (cout) {
        case 16: launch_conv_n<16>(a, s); break;
        case 32: launch_conv_n<32>(a, s); break;
        case 48: launch_conv_n<48>(a, s); break;
        case 64: launch_conv_n<64>(a, s); break;
        case 96: launch_conv_n<96>(a, s); break;
        default: fail(VAPOR_INVALID_ARGUMENT, "unsupported convolution output width");
    }
}

std::atomic<int> g_wgrad_kind{1};

void set_wgrad_kernel(int kind) {
    if (kind < 0 || kind > 1) fail(VAPOR_INVALID_ARGUMENT, "weight-gradient kernel: 0 or 1");
    g_wgrad_kind.store(kind);
}

void launch_conv3_wgrad(const WGradArgs& a, cudaStream_t s) {
    const long V = long(a.D) * a.H * a.W;
    if (g_wgrad_kind.load() == 1 && a.cin <= 96 && a.cout % 16 == 0 && a.cin % 16 == 0 &&
        a.g_stride % 8 == 0 && a.g_offset % 8 == 0 && a.x_stride % 8 == 0) {
        // voxel ranges: about two waves of CTAs over the tap groups and
        // output-channel chunks, at least one stage of voxels each
        const int others = 4 * (a.cout / 16);
        const long target = std::max<long>(1, (2L * device_sm_count() + others - 1) / others);
        const long chunk = std::max<long>(WGradTc::kK, ((V + target - 1) / target + WGradTc::kK - 1) /
                                                           WGradTc::kK * WGradTc::kK);
        const dim3 grid(unsigned((V + chunk - 1) / chunk), 4, unsigned(a.cout / 16));
        count_launch();
        k_conv3_wgrad_tc<<<grid, 256, WGradTc::smem(a.cin), s>>>(a, chunk);
        return;
    }
    const int chunks = int(std::max<long>(1, std::min<long>(V / 4096, 256)));
    const dim3 grid(chunks, 27, (a.cout / 16) * (a.cin / 16));
    count_launch();
    k_conv3_wgrad<<<grid, 256, 0, s>>>(a);
}

void launch_prep_input(int n, const float* b_split, const ProjControl* ctrl, double* partial, float* scale,
                       __nv_bfloat16* out, cudaStream_t s) {
    const long V = long(n) * n * n;
    const int blocks = std::min(blocks_for(V), 1184);
    count_launch();
    k_rms<<<blocks, 256, 0, s>>>(n, b_split, ctrl, partial);
    count_launch();
    k_rms_finish<<<1, 1024, 0, s>>>(partial, blocks, double(V), scale);
    count_launch();
    k_prep_input<<<blocks_for(V), 256, 0, s>>>(n, b_split, ctrl, scale, out);
}

void launch_prep_natural(long V, const float* a, double* partial, double* scalars, float* scale,
                         __nv_bfloat16* out, cudaStream_t s) {
    launch_mean(V, a, partial, scalars, s);
    const int blocks = std::min(blocks_for(V), 1184);
    count_launch();
    k_rms_natural<<<blocks, 256, 0, s>>>(V, a, scalars, partial);
    count_launch();
    k_rms_finish<<<1, 1024, 0, s>>>(partial, blocks, double(V), scale);
    count_launch();
    k_prep_natural<<<blocks_for(V), 256, 0, s>>>(V, a, scalars, scale, out);
}

void launch_avgpool2(int D, int H, int W, int C, const __nv_bfloat16* in, int in_stride, __nv_bfloat16* out,
                     cudaStream_t s) {
    count_launch();
    k_avgpool2<<<blocks_for(long(D) * H * W * C / 8), 256, 0, s>>>(D, H, W, C, in, in_stride, out);
}

void launch_upsample2(int d, int h, int w, int C, const __nv_bfloat16* in, __nv_bfloat16* out, int out_stride,
                      cudaStream_t s) {
    count_launch();
    if (C % 8 != 0 || out_stride % 8 != 0) fail(VAPOR_INVALID_ARGUMENT, "upsampling needs channels in multiples of 8");
    k_upsample2<<<blocks_for(long(d) * h * w * C), 256, 0, s>>>(d, h, w, C, in, out, out_stride);
}

void launch_head(long V, int C, const __nv_bfloat16* act, const float* w, const float* bias, float* out,
                 cudaStream_t s) {
    count_launch();
    k_head<<<blocks_for(V), 256, 0, s>>>(V, C, act, w, bias, out);
}

void launch_mean(long V, const float* a, double* partial, double* mean, cudaStream_t s) {
    const int blocks = std::min(blocks_for(V), 1184);
    count_launch();
    k_sum<<<blocks, 256, 0, s>>>(V, a, partial);
    count_launch();
    k_mean_finish<<<1, 1024, 0, s>>>(partial, blocks, double(V), mean);
}

void launch_store_warm_start(int n, const float* p, const float* b_split, const ProjControl* ctrl,
                             double* partial, double* scalars, float* x_split, double* x64_split, cudaStream_t s) {
    const long V = long(n) * n * n;
    launch_mean(V, p, partial, scalars, s);
    const int blocks = std::min(blocks_for(V), 592);
    count_launch();
    k_galerkin_sums<<<blocks, 256, 0, s>>>(n, p, scalars, b_split, ctrl, partial);
    count_launch();
    k_galerkin_finish<<<1, 1024, 0, s>>>(partial, blocks, scalars + 1);
    count_launch();
    if (x64_split) k_store_warm_start64<<<blocks_for(V), 256, 0, s>>>(n, p, scalars + 1, scalars, x64_split);
    else k_store_warm_start<<<blocks_for(V), 256, 0, s>>>(n, p, scalars + 1, scalars, x_split);
}

void launch_target(int n, const float* p_split, const ProjControl* ctrl, const float* scale, float* target,
                   cudaStream_t s) {
    count_launch();
    k_target<<<blocks_for(long(n) * n * n), 256, 0, s>>>(n, p_split, ctrl, scale, target);
}

void launch_loss_grad(long V, const float* p, const float* t, double* partial, double* scalars, float* grad,
                      cudaStream_t s) {
    launch_mean(V, p, partial, scalars, s);
    launch_mean(V, t, partial, scalars + 1, s);
    const int blocks = std::min(blocks_for(V), 392);
    count_launch();
    k_loss_sums<<<blocks, 256, 0, s>>>(V, p, t, scalars, partial);
    count_launch();
    k_loss_finish<<<1, 1024, 0, s>>>(partial, blocks, scalars);
    if (grad) {
        count_launch();
        k_loss_grad<<<blocks_for(V), 256, 0, s>>>(V, p, t, scalars, grad);
    }
}

void launch_head_backward(long V, int C, const __nv_bfloat16* act, const float* w, const float* g,
                          __nv_bfloat16* dact, float* dw, float* db, cudaStream_t s) {
    count_launch();
    k_head_backward<<<std::min(blocks_for(V), 592), 256, 0, s>>>(V, C, act, w, g, dact, dw, db);
}

void launch_relu_mask(long V, int C, const __nv_bfloat16* act, int act_stride, int act_offset, __nv_bfloat16* g,
                      int g_stride, int g_offset, cudaStream_t s) {
    count_launch();
    k_relu_mask<<<blocks_for(V * C), 256, 0, s>>>(V, C, act, act_stride, act_offset, g, g_stride, g_offset);
}

void launch_bias_grad(long V, int C, const __nv_bfloat16* g, int g_stride, int g_offset, float* db, cudaStream_t s) {
    count_launch();
    k_bias_grad<<<std::min(blocks_for(V), 1184), 256, 0, s>>>(V, C, g, g_stride, g_offset, db);
}

void launch_flip_weights(int cout, int cin, const __nv_bfloat16* w, __nv_bfloat16* wt, cudaStream_t s) {
    count_launch();
    k_flip_weights<<<blocks_for(27L * cout * cin), 256, 0, s>>>(cout, cin, w, wt);
}

void launch_avgpool2_backward(int D, int H, int W, int C, const __nv_bfloat16* dout, __nv_bfloat16* din,
                              int din_stride, int din_offset, bool add, cudaStream_t s) {
    count_launch();
    k_avgpool2_backward<<<blocks_for(long(D) * H * W * C), 256, 0, s>>>(D, H, W, C, dout, din, din_stride,
                                                                         din_offset, add ? 1 : 0);
}

void launch_upsample2_backward(int d, int h, int w, int C, const __nv_bfloat16* dfine, int fine_stride,
                               __nv_bfloat16* dcoarse, cudaStream_t s) {
    count_launch();
    k_upsample2_backward<<<blocks_for(long(d) * h * w * C), 256, 0, s>>>(d, h, w, C, dfine, fine_stride, dcoarse);
}

void launch_adam(long count, float* w, float* m, float* v, const float* g, __nv_bfloat16* wb, float lr, int step,
                 cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    count_launch();
    k_adam<<<blocks_for(count), 256, 0, s>>>(count, w, m, v, g, wb, lr, b1, b2, eps, c1, c2);
}

void launch_to_bf16(long count, const float* a, __nv_bfloat16* b, cudaStream_t s) {
    count_launch();
    k_to_bf16<<<blocks_for(count), 256, 0, s>>>(count, a, b);
}

}  // namespace unet
}  // namespace vb
