// The simplicial 3D solver's compute stages on the device
// (SimplicialCompute3D, src/solvers/simplicial3d/SimplicialCompute3D.hpp:7-13):
// the reference's OpenGL backend (gpu/GpuSimplicial3D.cpp, shaders
// advection.comp and recovery.comp) as CUDA, FP64 throughout.
//
//   advect_circulation  one thread per dual vertex traces it by the midpoint
//                       rule and samples the velocity at its foot; one thread
//                       per dual edge forms .5 (v_a + v_b).(x_b - x_a); one
//                       thread per primal edge sums its dual face's signed
//                       edge integrals in loop order
//   advect_density      one thread per primal vertex: trace, interpolate the
//                       vertex smoke at the foot, decay, round to float
//   recover             CG on the CSR Dirichlet potential operator with the
//                       CPU solver's preconditioner (its IC(0) factor by two
//                       level-scheduled triangular solves in one block, the
//                       vector in shared memory when it fits, each row in
//                       the CPU's operation order, or its diagonal);
//                       the operator applied matrix-free by gather kernels
//                       in the CPU's summation order and the dot products
//                       summed in index order (std::inner_product's), so the
//                       iterates equal the CPU's bit for bit; for large
//                       meshes a block-partial tree order instead; the state of
//                       the iteration (rz, alpha, beta, residuals, counts) in
//                       device memory so that a batch of iterations runs
//                       without host round trips; the host reads it every 8
//                       iterations, as the reference's backend does
//
// The per-sample arithmetic is simplicial_math.cuh, in the CPU solver's
// operation order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine.hpp"
#include "simplicial_math.cuh"

namespace vb {
namespace {

using simplicial::View;
constexpr int kT = 256;
int blocks_s(long count) { return int(std::max<long>(1, (count + kT - 1) / kT)); }

__global__ void ks_trace_dual(View v, double dt, const double* __restrict__ dual_velocity,
                              const double* __restrict__ samples, double* __restrict__ traced,
                              double* __restrict__ velocity, int* error) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.n_dual) return;
    int e = 0;
    simplicial::P3 t, u;
    simplicial::trace_dual(v, i, dt, dual_velocity, samples, &t, &u, &e);
    traced[3 * i] = t.x;
    traced[3 * i + 1] = t.y;
    traced[3 * i + 2] = t.z;
    velocity[3 * i] = u.x;
    velocity[3 * i + 1] = u.y;
    velocity[3 * i + 2] = u.z;
    if (e) atomicOr(error, e);
}

__global__ void ks_edge_integral(View v, const double* __restrict__ traced, const double* __restrict__ velocity,
                                 double* __restrict__ integral) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < v.n_dual_edges) integral[j] = simplicial::edge_integral(v, j, traced, velocity);
}

__global__ void ks_circulation(View v, const double* __restrict__ integral, double* __restrict__ omega) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < v.n_edges) omega[e] = simplicial::circulation(v, e, integral);
}

__global__ void ks_density(View v, double dt, double decay, const double* __restrict__ dual_velocity,
                           const double* __restrict__ samples, const float* __restrict__ density,
                           float* __restrict__ out, int* error) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= v.n_primal) return;
    int e = 0;
    out[i] = simplicial::trace_density(v, i, dt, decay, dual_velocity, samples, density, &e);
    if (e) atomicOr(error, e);
}

// ---- preconditioned CG ----

// Iteration state in device memory.
enum CgSlot { kRz = 0, kAlpha, kBeta, kInitial, kResidual, kDone, kIterations, kBreakdown, kDot, kSlots };

// The Dirichlet potential operator, matrix-free, as the CPU solver applies
// it (SimplicialFluidSolver3D::applyLaplacian / laplacian): boundary entries
// of the input zeroed; per face the d1 sum of its three signed edges times
// star2; per vertex the signed star1-weighted sum of its edges in edge order,
// divided by star0 (zero on boundary vertices); per edge the d1-transpose sum
// over its faces in face order plus star1 times the d0 gradient of the vertex
// values; boundary edges pass the input through.
struct Laplacian {
    int n_edges, n_faces, n_vertices;
    const int* face_edges;        // 3 per face
    const int* face_signs;        // 3 per face
    const double* star0;
    const double* star1;
    const double* star2;
    const int* edge_vertices;     // 2 per edge
    const unsigned char* edge_boundary;
    const unsigned char* vertex_boundary;
    const int* edge_face_offsets; // per edge: its (face, slot) pairs in face order
    const int* edge_face_items;   // face * 3 + slot
    const int* vertex_edge_offsets;  // per vertex: its edges in edge order
    const int* vertex_edge_items;    // edge * 2 + (1 if the vertex is the edge's second end)
};

// c_f = star2_f d1(x)_f and the vertex values of the divergence term.
__global__ void ks_lap_faces_vertices(Laplacian L, const double* __restrict__ in, double* __restrict__ face_value,
                                      double* __restrict__ vertex_value, const double* status) {
    if (status && status[kDone] != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < L.n_faces) {
        double y = 0;
        for (int k = 0; k < 3; ++k) {
            const int e = L.face_edges[3 * i + k];
            y += L.face_signs[3 * i + k] * (L.edge_boundary[e] ? 0. : in[e]);
        }
        face_value[i] = y * L.star2[i];
    }
    if (i < L.n_vertices) {
        double d = 0;
        for (int j = L.vertex_edge_offsets[i]; j < L.vertex_edge_offsets[i + 1]; ++j) {
            const int code = L.vertex_edge_items[j], e = code >> 1;
            const double value = L.star1[e] * (L.edge_boundary[e] ? 0. : in[e]);
            if (code & 1)
                d += value;
            else
                d -= value;
        }
        vertex_value[i] = L.vertex_boundary[i] ? 0 : d / L.star0[i];
    }
}
__global__ void ks_lap_edges(Laplacian L, const double* __restrict__ in, const double* __restrict__ face_value,
                             const double* __restrict__ vertex_value, double* __restrict__ out, const double* status) {
    if (status && status[kDone] != 0) return;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= L.n_edges) return;
    if (L.edge_boundary[e]) {
        out[e] = in[e];
        return;
    }
    double y = 0;
    for (int j = L.edge_face_offsets[e]; j < L.edge_face_offsets[e + 1]; ++j) {
        const int code = L.edge_face_items[j];
        y += L.face_signs[code] * face_value[code / 3];
    }
    const double gradient = vertex_value[L.edge_vertices[2 * e + 1]] - vertex_value[L.edge_vertices[2 * e]];
    out[e] = y + L.star1[e] * gradient;
}

// Maximum that keeps a NaN (a non-finite residual must not read as converged).
__device__ __forceinline__ double max_nan(double a, double b) {
    return a != a ? a : (b != b ? b : (a < b ? b : a));
}

// Block sum and maximum, written as the block's partials.
__device__ __forceinline__ void block_partials(double sum, double maximum, double* partials, int blocks) {
    __shared__ double s_sum[kT / 32], s_max[kT / 32];
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        maximum = max_nan(maximum, __shfl_down_sync(0xffffffffu, maximum, o));
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_sum[warp] = sum;
        s_max[warp] = maximum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, m = 0;
        for (int w = 0; w < kT / 32; ++w) {
            a += s_sum[w];
            m = max_nan(m, s_max[w]);
        }
        partials[blockIdx.x] = a;
        partials[blocks + blockIdx.x] = m;
    }
}

// One block: the sum and maximum over all blocks' partials, in block order
// within each thread's stride and a fixed tree across threads.
__device__ __forceinline__ void reduce_partials(const double* partials, int blocks, double* sum_out, double* max_out) {
    double a = 0, m = 0;
    for (int j = threadIdx.x; j < blocks; j += kT) {
        a += partials[j];
        m = max_nan(m, partials[blocks + j]);
    }
    __shared__ double s_sum[kT], s_max[kT];
    s_sum[threadIdx.x] = a;
    s_max[threadIdx.x] = m;
    __syncthreads();
    for (int step = kT / 2; step > 0; step >>= 1) {
        if (int(threadIdx.x) < step) {
            s_sum[threadIdx.x] += s_sum[threadIdx.x + step];
            s_max[threadIdx.x] = max_nan(s_max[threadIdx.x], s_max[threadIdx.x + step]);
        }
        __syncthreads();
    }
    *sum_out = s_sum[0];
    *max_out = s_max[0];
}

// a.b into status[kDot]: in index order on one thread, as std::inner_product
// sums it (sequential), or by block partials and one reducing block (tree).
// One block: the products of a chunk are formed in parallel into shared
// memory, then one thread adds them in order.
__global__ void ks_dot_sequential(int n, const double* __restrict__ a, const double* __restrict__ b, double* status) {
    if (status[kDone] != 0) return;
    __shared__ double products[2048];
    double acc = 0;
    for (int base = 0; base < n; base += 2048) {
        const int count = min(2048, n - base);
        for (int k = threadIdx.x; k < count; k += blockDim.x) products[k] = a[base + k] * b[base + k];
        __syncthreads();
        if (threadIdx.x == 0)
            for (int k = 0; k < count; ++k) acc = acc + products[k];
        __syncthreads();
    }
    if (threadIdx.x == 0) status[kDot] = acc;
}
__global__ void ks_dot_partials(int n, const double* __restrict__ a, const double* __restrict__ b, double* partials,
                                int blocks, const double* status) {
    if (status[kDone] != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    block_partials(i < n ? a[i] * b[i] : 0., 0., partials, blocks);
}
__global__ void ks_dot_tree(const double* partials, int blocks, double* status) {
    if (status[kDone] != 0) return;
    double sum, maximum;
    reduce_partials(partials, blocks, &sum, &maximum);
    if (threadIdx.x == 0) status[kDot] = sum;
}

// The preconditioner M^-1 r: the inverse diagonal, or the solver's IC(0)
// factor (M = L L^T, L unit-free: rows of strictly lower entries plus a
// diagonal) applied by two triangular solves in level order.
struct Precond {
    int ic;
    const double* jacobi;  // diagonal (Jacobi)
    // forward solve: rows of L, strictly lower entries in ascending column
    // order; rows grouped by dependency level
    const int* l_offsets;
    const int* l_columns;
    const double* l_values;
    const double* l_diagonal;
    const int* f_level_offsets;
    const int* f_rows;
    int f_levels;
    // backward solve: the entries of each column of L, in descending row
    // order; columns grouped by dependency level
    const int* t_offsets;
    const int* t_rows;
    const double* t_values;
    const int* b_level_offsets;
    const int* b_columns;
    int b_levels;
    // the same rows in level order as (row, first entry, end) for one load
    const int4* f_table;
    const int4* b_table;
};

// r = b - A x (zero on boundary edges, as the CPU solver sets it); partials
// of max |r|.
__global__ void ks_cg_residual(int n, const unsigned char* __restrict__ boundary, const double* __restrict__ b,
                               const double* __restrict__ ax, double* __restrict__ r, double* partials, int blocks) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double maximum = 0;
    if (i < n) {
        const double ri = boundary[i] ? 0. : b[i] - ax[i];
        r[i] = ri;
        maximum = fabs(ri);
    }
    block_partials(0, maximum, partials, blocks);
}
__global__ void ks_cg_started(const double* partials, int blocks, double target, double* status) {
    double sum, maximum;
    reduce_partials(partials, blocks, &sum, &maximum);
    if (threadIdx.x == 0) {
        status[kInitial] = maximum;
        status[kResidual] = maximum;
        status[kDone] = maximum <= target ? 1 : 0;
        status[kIterations] = 0;
        status[kBreakdown] = 0;
    }
}
// z = r / diag.
__global__ void ks_jacobi(int n, const double* __restrict__ r, const double* __restrict__ diagonal,
                          double* __restrict__ z, const double* status) {
    if (status[kDone] != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) z[i] = r[i] / diagonal[i];
}
// z = L^-T (L^-1 r) in one block: each level's rows in parallel, a block
// barrier between levels. Each row keeps the CPU's operation order: the
// forward value subtracts its row's terms in column order, then divides; the
// backward value subtracts the terms of the later rows in descending order,
// then divides.
__global__ void __launch_bounds__(1024) ks_ic_solve(Precond m, const double* __restrict__ r, double* z,
                                                    const double* status) {
    if (status[kDone] != 0) return;
    for (int level = 0; level < m.f_levels; ++level) {
        for (int k = m.f_level_offsets[level] + threadIdx.x; k < m.f_level_offsets[level + 1]; k += blockDim.x) {
            const int i = m.f_rows[k];
            double acc = r[i];
            for (int j = m.l_offsets[i]; j < m.l_offsets[i + 1]; ++j) acc -= m.l_values[j] * z[m.l_columns[j]];
            z[i] = acc / m.l_diagonal[i];
        }
        __syncthreads();
    }
    for (int level = 0; level < m.b_levels; ++level) {
        for (int k = m.b_level_offsets[level] + threadIdx.x; k < m.b_level_offsets[level + 1]; k += blockDim.x) {
            const int c = m.b_columns[k];
            double acc = z[c];
            for (int j = m.t_offsets[c]; j < m.t_offsets[c + 1]; ++j) acc -= m.t_values[j] * z[m.t_rows[j]];
            z[c] = acc / m.l_diagonal[c];
        }
        __syncthreads();
    }
}
// ks_ic_solve with the vector in shared memory (n doubles) and one warp per
// row. The lanes hold a row's entries (up to 32 at a time) and form its
// products in parallel; one lane then subtracts them from the row's value in
// the CPU's order. The entries of a warp's row in the
// next level do not depend on the solve, so they are fetched before the
// barrier that ends the current level and arrive while it waits: a level
// costs the shared-memory gathers, the shuffles and the barrier, not round
// trips to L2. Same operations in the same order as the thread-per-row form.
struct IcRowFetch {
    int row, beg, end;  // row < 0: none
    int column;
    double value, init;
};
__device__ __forceinline__ IcRowFetch ic_fetch(int k, int k_end, const int4* __restrict__ table,
                                               const int* __restrict__ columns, const double* __restrict__ values,
                                               const double* init_global, int lane) {
    IcRowFetch f;
    f.row = -1;
    f.beg = f.end = 0;
    f.column = 0;
    f.value = 0.0;
    f.init = 0.0;
    if (k < k_end) {
        const int4 t = table[k];
        f.row = t.x;
        f.beg = t.y;
        f.end = t.z;
        const int j = f.beg + lane;
        if (j < f.end) {
            f.column = columns[j];
            f.value = values[j];
        }
        if (init_global) f.init = init_global[f.row];
    }
    return f;
}
// acc minus the row's products in order (the fetched first 32, then the
// rest): the lanes form the products into the warp's shared-memory slots and
// lane 0 subtracts them one after the other (its result is the one kept).
__device__ __forceinline__ double ic_apply(const IcRowFetch& f, double acc, const int* __restrict__ columns,
                                           const double* __restrict__ values, const double* zs, double* stage,
                                           int lane) {
    stage[lane] = f.beg + lane < f.end ? f.value * zs[f.column] : 0.0;
    __syncwarp();
    if (lane == 0) {
        const int count = min(32, f.end - f.beg);
        for (int t = 0; t < count; ++t) acc -= stage[t];
    }
    __syncwarp();
    for (int base = f.beg + 32; base < f.end; base += 32) {
        const int j = base + lane;
        stage[lane] = j < f.end ? values[j] * zs[columns[j]] : 0.0;
        __syncwarp();
        if (lane == 0) {
            const int count = min(32, f.end - base);
            for (int t = 0; t < count; ++t) acc -= stage[t];
        }
        __syncwarp();
    }
    return acc;
}
// One triangular solve over `levels` levels: each warp's first row of a level
// is fetched two levels ahead (its table entry, entries and initial value do
// not depend on the solve); further rows of the level are fetched in place.
__device__ __forceinline__ void ic_sweep(int levels, const int* __restrict__ level_offsets,
                                         const int4* __restrict__ table, const int* __restrict__ columns,
                                         const double* __restrict__ values, const double* __restrict__ diagonal,
                                         const double* init_global, double* zs, double* stage, int lane, int warp,
                                         int warps) {
    auto fetch = [&](int level) {
        if (level >= levels) return IcRowFetch{-1, 0, 0, 0, 0.0, 0.0};
        return ic_fetch(level_offsets[level] + warp, level_offsets[level + 1], table, columns, values, init_global,
                        lane);
    };
    IcRowFetch a = fetch(0), b = fetch(1);
    for (int level = 0; level < levels; ++level) {
        const IcRowFetch cur = a;
        a = b;
        b = fetch(level + 2);
        if (cur.row >= 0) {
            const double acc = ic_apply(cur, init_global ? cur.init : zs[cur.row], columns, values, zs, stage, lane);
            if (lane == 0) zs[cur.row] = acc / diagonal[cur.row];
        }
        for (int k = level_offsets[level] + warp + warps; k < level_offsets[level + 1]; k += warps) {
            const IcRowFetch f = ic_fetch(k, k + 1, table, columns, values, init_global, lane);
            const double acc = ic_apply(f, init_global ? f.init : zs[f.row], columns, values, zs, stage, lane);
            if (lane == 0) zs[f.row] = acc / diagonal[f.row];
        }
        __syncthreads();
    }
}
__global__ void __launch_bounds__(1024, 1) ks_ic_solve_shared(Precond m, int n, const double* __restrict__ r,
                                                              double* __restrict__ z, const double* status) {
    if (status[kDone] != 0) return;
    extern __shared__ double zs[];
    __shared__ double stages[32 * 32];  // per warp, the products of one row chunk
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    double* stage = stages + 32 * warp;
    // forward: zs[i] = (r[i] - sum L_ij zs[j]) / D_i
    ic_sweep(m.f_levels, m.f_level_offsets, m.f_table, m.l_columns, m.l_values, m.l_diagonal, r, zs, stage, lane,
             warp, warps);
    // backward: zs[c] = (zs[c] - sum over later rows i of L_ic zs[i]) / D_c
    ic_sweep(m.b_levels, m.b_level_offsets, m.b_table, m.t_rows, m.t_values, m.l_diagonal, nullptr, zs, stage, lane,
             warp, warps);
    for (int i = threadIdx.x; i < n; i += blockDim.x) z[i] = zs[i];
}
// rz of the start
__global__ void ks_cg_take_rz(double* status) {
    if (status[kDone] == 0) status[kRz] = status[kDot];
}
__global__ void ks_cg_copy(int n, const double* __restrict__ z, double* __restrict__ p, const double* status) {
    if (status[kDone] != 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i];
}
// alpha = rz / p.ap, or the breakdown the CPU reports
__global__ void ks_cg_alpha(double* status) {
    if (status[kDone] != 0) return;
    const double pap = status[kDot];
    if (!(pap > 0) || !(pap <= DBL_MAX)) {  // not positive, or not finite
        status[kDone] = 2;
        status[kBreakdown] = 1;
    } else {
        status[kAlpha] = status[kRz] / pap;
    }
}
// x += alpha p, r -= alpha ap; partials of max |r|.
__global__ void ks_cg_update(int n, double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                             const double* __restrict__ ap, double* partials, int blocks, const double* status) {
    if (status[kDone] != 0) return;
    const double alpha = status[kAlpha];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double maximum = 0;
    if (i < n) {
        x[i] += alpha * p[i];
        const double ri = r[i] - alpha * ap[i];
        r[i] = ri;
        maximum = fabs(ri);
    }
    block_partials(0, maximum, partials, blocks);
}
// the iteration counted; done once the updated residual meets the target
__global__ void ks_cg_check(const double* partials, int blocks, double target, double* status) {
    if (status[kDone] != 0) return;
    double sum, maximum;
    reduce_partials(partials, blocks, &sum, &maximum);
    if (threadIdx.x == 0) {
        status[kResidual] = maximum;
        status[kIterations] += 1;
        if (maximum <= target) status[kDone] = 1;
    }
}
__global__ void ks_cg_beta(double* status) {
    if (status[kDone] != 0) return;
    status[kBeta] = status[kDot] / status[kRz];
    status[kRz] = status[kDot];
}
__global__ void ks_cg_direction(int n, const double* __restrict__ z, double* __restrict__ p, const double* status) {
    if (status[kDone] != 0) return;
    const double beta = status[kBeta];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = z[i] + beta * p[i];
}
__global__ void ks_cg_final(const double* partials, int blocks, double target, double* status) {
    double sum, maximum;
    reduce_partials(partials, blocks, &sum, &maximum);
    if (threadIdx.x == 0) {
        status[kResidual] = maximum;
        status[kDone] = maximum <= target ? 1 : 0;
    }
}

template <class T>
void upload(DevArray<T>& d, const T* src, size_t count, cudaStream_t s) {
    d.allocate(std::max<size_t>(count, 1));
    if (count) VB_CUDA(cudaMemcpyAsync(d.p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
}
void upload_i(DevArray<uint32_t>& d, const int32_t* src, size_t count, cudaStream_t s) {
    upload(d, reinterpret_cast<const uint32_t*>(src), count, s);
}
const int* iptr(const DevArray<uint32_t>& d) { return reinterpret_cast<const int*>(d.p); }

void require_s(bool ok, const char* what) {
    if (!ok) fail(VAPOR_INVALID_ARGUMENT, std::string("simplicial mesh: ") + what);
}
// Every entry of idx[0..count) in [lo, hi).
void check_range(const int32_t* idx, long count, long lo, long hi, const char* what) {
    require_s(count == 0 || idx != nullptr, what);
    for (long k = 0; k < count; ++k) require_s(idx[k] >= lo && idx[k] < hi, what);
}
// Non-decreasing offsets from 0; returns the item count.
long check_offsets(const int32_t* off, long owners, const char* what) {
    require_s(off != nullptr && off[0] == 0, what);
    for (long k = 0; k < owners; ++k) require_s(off[k + 1] >= off[k], what);
    return off[owners];
}

}  // namespace

class SimplicialStages {
public:
    SimplicialStages(const vapor_simplicial3d_mesh& m, int site_search, int dot_order, int preconditioner) {
        validate(m);
        cudaStream_t s = st_.s;
        v_ = View{};
        v_.box = m.box_domain ? 1 : 0;
        v_.search = site_search == 1 ? 0 : site_search == 2 ? 1 : (m.n_primal <= 4096 ? 0 : 1);
        sequential_dots_ = dot_order == 1 || (dot_order == 0 && m.n_edges <= 262144);
        v_.size = m.size;
        v_.n_primal = m.n_primal;
        v_.n_dual = m.n_dual;
        v_.n_nodes = m.n_nodes;
        v_.n_edges = m.n_edges;
        v_.n_dual_edges = m.n_dual_edges;
        v_.n_tets = m.n_tets;
        v_.bins = m.bins;
        const long nb = std::max<long>(1, long(m.bins) * m.bins * m.bins);
        upload(dual_position_, m.dual_position, 3L * m.n_dual, s);
        upload(node_position_, m.node_position, 3L * m.n_nodes, s);
        upload(tet_geometry_, m.tet_geometry, 12L * m.n_tets, s);
        upload_i(tet_vertices_, m.tet_vertices, 4L * m.n_tets, s);
        upload_i(dual_hint_, m.dual_hint, m.n_dual, s);
        upload_i(primal_hint_, m.primal_hint, m.n_primal, s);
        upload_i(bin_offsets_, m.bin_offsets, nb + 1, s);
        upload_i(bin_items_, m.bin_items, m.bin_offsets[nb], s);
        upload_i(wall_offsets_, m.wall_offsets, nb + 1, s);
        upload_i(wall_items_, m.wall_items, m.wall_offsets[nb], s);
        upload(wall_geometry_, m.wall_geometry, 6L * m.n_faces, s);
        upload_i(wall_owner_, m.wall_owner, m.n_faces, s);
        upload_i(loop_offsets_, m.loop_offsets, m.n_edges + 1L, s);
        upload_i(loop_items_, m.loop_items, m.loop_offsets[m.n_edges], s);
        upload_i(dual_edges_, m.dual_edges, 2L * m.n_dual_edges, s);
        if (v_.box) {
            upload(box_planes_, m.box_planes, 4L * m.n_planes, s);
            upload_i(cell_corners_, m.cell_corners, m.n_primal + 1L, s);
            upload_i(corner_vertices_, m.corner_vertices, m.n_corners, s);
            upload_i(corner_cones_, m.corner_cones, m.n_corners + 1L, s);
            upload_i(cone_planes_, m.cone_planes, 3L * m.n_cones, s);
            upload_i(neighbor_offsets_, m.neighbor_offsets, m.n_primal + 1L, s);
            upload_i(neighbors_, m.neighbors, m.neighbor_offsets[m.n_primal], s);
        } else {
            upload_i(sub_offsets_, m.sub_offsets, m.n_tets + 1L, s);
            upload_i(sub_nodes_, m.sub_nodes, 4L * m.n_subtets, s);
            upload(sub_gradients_, m.sub_gradients, 9L * m.n_subtets, s);
        }
        v_.dual_position = dual_position_.p;
        v_.node_position = node_position_.p;
        v_.tet_geometry = tet_geometry_.p;
        v_.tet_vertices = iptr(tet_vertices_);
        v_.dual_hint = iptr(dual_hint_);
        v_.primal_hint = iptr(primal_hint_);
        v_.bin_offsets = iptr(bin_offsets_);
        v_.bin_items = iptr(bin_items_);
        v_.wall_offsets = iptr(wall_offsets_);
        v_.wall_items = iptr(wall_items_);
        v_.wall_geometry = wall_geometry_.p;
        v_.wall_owner = iptr(wall_owner_);
        v_.box_planes = box_planes_.p;
        v_.cell_corners = iptr(cell_corners_);
        v_.corner_vertices = iptr(corner_vertices_);
        v_.corner_cones = iptr(corner_cones_);
        v_.cone_planes = iptr(cone_planes_);
        v_.neighbor_offsets = iptr(neighbor_offsets_);
        v_.neighbors = iptr(neighbors_);
        v_.sub_offsets = iptr(sub_offsets_);
        v_.sub_nodes = iptr(sub_nodes_);
        v_.sub_gradients = sub_gradients_.p;
        v_.loop_offsets = iptr(loop_offsets_);
        v_.loop_items = iptr(loop_items_);
        v_.dual_edges = iptr(dual_edges_);
        setup_operator(m);
        setup_preconditioner(m, preconditioner == 1);
        dual_velocity_.allocate(3L * m.n_dual);
        samples_.allocate(3L * m.n_nodes);
        traced_.allocate(3L * m.n_dual);
        traced_velocity_.allocate(3L * m.n_dual);
        integral_.allocate(std::max(1, m.n_dual_edges));
        omega_.allocate(std::max(1, m.n_edges));
        density_in_.allocate(m.n_primal);
        density_out_.allocate(m.n_primal);
        error_.allocate(1);
        const long n = m.n_edges;
        for (DevArray<double>* a : {&b_, &x_, &r_, &z_, &p_, &ap_}) a->allocate(std::max<long>(1, n));
        cg_blocks_ = blocks_s(n);
        partials_.allocate(2L * cg_blocks_);
        status_.allocate(kSlots);
        VB_CUDA(cudaStreamSynchronize(s));
    }
    ~SimplicialStages() { cudaStreamSynchronize(st_.s); }

    void advect_circulation(double dt, const double* dual_velocity, const double* samples, double* omega) {
        require_s(dual_velocity != nullptr && omega != nullptr, "null velocity or output");
        require_s(v_.box || samples != nullptr, "general domains need the node samples");
        cudaStream_t s = st_.s;
        put_velocity(dual_velocity, samples);
        ks_trace_dual<<<blocks_s(v_.n_dual), kT, 0, s>>>(v_, dt, dual_velocity_.p, samples_.p, traced_.p,
                                                         traced_velocity_.p, reinterpret_cast<int*>(error_.p));
        ks_edge_integral<<<blocks_s(v_.n_dual_edges), kT, 0, s>>>(v_, traced_.p, traced_velocity_.p, integral_.p);
        ks_circulation<<<blocks_s(v_.n_edges), kT, 0, s>>>(v_, integral_.p, omega_.p);
        VB_CUDA(cudaGetLastError());
        if (v_.n_edges)
            VB_CUDA(cudaMemcpyAsync(omega, omega_.p, sizeof(double) * v_.n_edges, cudaMemcpyDeviceToHost, s));
        finish();
    }

    void advect_density(double dt, double decay, const double* dual_velocity, const double* samples,
                        const float* density, float* out) {
        require_s(dual_velocity != nullptr && density != nullptr && out != nullptr, "null input or output");
        require_s(v_.box || samples != nullptr, "general domains need the node samples");
        cudaStream_t s = st_.s;
        put_velocity(dual_velocity, samples);
        VB_CUDA(cudaMemcpyAsync(density_in_.p, density, sizeof(float) * v_.n_primal, cudaMemcpyHostToDevice, s));
        ks_density<<<blocks_s(v_.n_primal), kT, 0, s>>>(v_, dt, decay, dual_velocity_.p, samples_.p, density_in_.p,
                                                        density_out_.p, reinterpret_cast<int*>(error_.p));
        VB_CUDA(cudaGetLastError());
        VB_CUDA(cudaMemcpyAsync(out, density_out_.p, sizeof(float) * v_.n_primal, cudaMemcpyDeviceToHost, s));
        finish();
    }

    vapor_linear_solve_result recover(const double* rhs, const double* x0, int iterations, double absolute,
                                      double relative, double* x) {
        if (iterations < 0 || !std::isfinite(absolute) || absolute < 0 || !std::isfinite(relative) || relative < 0)
            fail(VAPOR_INVALID_ARGUMENT, "Invalid GPU CG parameters");
        require_s(rhs != nullptr && x0 != nullptr && x != nullptr, "null right-hand side, start or output");
        const int n = v_.n_edges;
        std::vector<double> b(rhs, rhs + n);
        double norm = 0;
        for (int i = 0; i < n; ++i) {
            if (!std::isfinite(b[i])) fail(VAPOR_RUNTIME_ERROR, "Non-finite GPU RHS");
            if (edge_boundary_[i]) b[i] = 0;
            norm = std::max(norm, std::abs(b[i]));
        }
        const double target = std::max(absolute, relative * norm);
        cudaStream_t s = st_.s;
        const int g = cg_blocks_;
        const unsigned char* boundary = lap_.edge_boundary;
        VB_CUDA(cudaMemcpyAsync(b_.p, b.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
        VB_CUDA(cudaMemcpyAsync(x_.p, x0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        apply(x_.p, ap_.p, false);
        ks_cg_residual<<<g, kT, 0, s>>>(n, boundary, b_.p, ap_.p, r_.p, partials_.p, g);
        ks_cg_started<<<1, kT, 0, s>>>(partials_.p, g, target, status_.p);
        precondition();
        dot(r_.p, z_.p);
        ks_cg_take_rz<<<1, 1, 0, s>>>(status_.p);
        ks_cg_copy<<<g, kT, 0, s>>>(n, z_.p, p_.p, status_.p);
        double st[kSlots];
        read_status(st);
        for (int done = 0; done < iterations && st[kDone] == 0;) {
            const int batch = std::min(8, iterations - done);
            for (int k = 0; k < batch; ++k) {
                apply(p_.p, ap_.p, true);
                dot(p_.p, ap_.p);
                ks_cg_alpha<<<1, 1, 0, s>>>(status_.p);
                ks_cg_update<<<g, kT, 0, s>>>(n, x_.p, r_.p, p_.p, ap_.p, partials_.p, g, status_.p);
                ks_cg_check<<<1, kT, 0, s>>>(partials_.p, g, target, status_.p);
                precondition();
                dot(r_.p, z_.p);
                ks_cg_beta<<<1, 1, 0, s>>>(status_.p);
                ks_cg_direction<<<g, kT, 0, s>>>(n, z_.p, p_.p, status_.p);
            }
            done += batch;
            read_status(st);
        }
        if (st[kBreakdown] != 0) fail(VAPOR_RUNTIME_ERROR, "GPU CG lost positive definiteness");
        vapor_linear_solve_result result{};
        result.initial_residual = st[kInitial];
        result.iterations = int(st[kIterations]);
        // the actual residual of x, not the recursively updated one
        apply(x_.p, ap_.p, false);
        ks_cg_residual<<<g, kT, 0, s>>>(n, boundary, b_.p, ap_.p, r_.p, partials_.p, g);
        ks_cg_final<<<1, kT, 0, s>>>(partials_.p, g, target, status_.p);
        read_status(st);
        result.final_residual = st[kResidual];
        result.converged = std::isfinite(st[kResidual]) && st[kDone] == 1 ? 1 : 0;
        if (n) VB_CUDA(cudaMemcpyAsync(x, x_.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        VB_CUDA(cudaStreamSynchronize(s));
        return result;
    }

private:
    void validate(const vapor_simplicial3d_mesh& m) {
        require_s(std::isfinite(m.size) && m.size > 0, "size");
        require_s(m.n_primal >= 4 && m.n_tets >= 1 && m.n_dual >= 1 && m.n_edges >= 1 && m.n_faces >= 1 &&
                      m.n_dual_edges >= 0 && m.n_nodes >= m.n_primal,
                  "counts");
        require_s(m.bins >= 0 && m.bins <= 512, "bins");
        const long nb = std::max<long>(1, long(m.bins) * m.bins * m.bins);
        require_s(m.dual_position && m.node_position && m.tet_geometry && m.wall_geometry, "geometry arrays");
        check_range(m.tet_vertices, 4L * m.n_tets, 0, m.n_primal, "tet vertices");
        check_range(m.dual_hint, m.n_dual, -1, m.n_tets, "dual hints");
        check_range(m.primal_hint, m.n_primal, -1, m.n_tets, "primal hints");
        check_range(m.bin_items, check_offsets(m.bin_offsets, nb, "bin offsets"), 0, m.n_tets, "bin items");
        check_range(m.wall_items, check_offsets(m.wall_offsets, nb, "wall offsets"), 0, m.n_faces, "wall items");
        check_range(m.wall_owner, m.n_faces, 0, m.n_tets, "wall owners");
        const long loops = check_offsets(m.loop_offsets, m.n_edges, "loop offsets");
        require_s(loops == 0 || m.loop_items != nullptr, "loop items");
        for (long k = 0; k < loops; ++k) {
            const int code = m.loop_items[k];
            require_s(code != 0 && std::abs(long(code)) <= m.n_dual_edges, "loop items");
        }
        check_range(m.dual_edges, 2L * m.n_dual_edges, 0, m.n_dual, "dual edges");
        if (m.box_domain) {
            require_s(m.n_planes >= 0 && m.n_corners >= 0 && m.n_cones >= 0 && (m.n_planes == 0 || m.box_planes),
                      "box cell counts");
            require_s(check_offsets(m.cell_corners, m.n_primal, "cell corners") == m.n_corners, "cell corners");
            check_range(m.corner_vertices, m.n_corners, 0, m.n_dual, "corner vertices");
            require_s(check_offsets(m.corner_cones, m.n_corners, "corner cones") == m.n_cones, "corner cones");
            check_range(m.cone_planes, 3L * m.n_cones, 0, m.n_planes, "cone planes");
            check_range(m.neighbors, check_offsets(m.neighbor_offsets, m.n_primal, "neighbour offsets"), 0,
                        m.n_primal, "neighbours");
        } else {
            require_s(m.n_subtets >= 0 && (m.n_subtets == 0 || m.sub_gradients), "subtets");
            require_s(check_offsets(m.sub_offsets, m.n_tets, "subtet offsets") == m.n_subtets, "subtet offsets");
            check_range(m.sub_nodes, 4L * m.n_subtets, 0, m.n_nodes, "subtet nodes");
        }
        check_range(m.face_edges, 3L * m.n_faces, 0, m.n_edges, "face edges");
        require_s(m.face_signs && m.star0 && m.star1 && m.star2 && m.edge_boundary && m.vertex_boundary,
                  "operator arrays");
        check_range(m.edge_vertices, 2L * m.n_edges, 0, m.n_primal, "edge vertices");
    }

    // The operator's gather lists (SimplicialFluidSolver3D::laplacian): per
    // edge its faces in face order, per vertex its edges in edge order, so
    // that every sum runs in the CPU loops' order.
    void setup_operator(const vapor_simplicial3d_mesh& m) {
        const int n = m.n_edges;
        cudaStream_t s = st_.s;
        edge_boundary_.assign(m.edge_boundary, m.edge_boundary + n);
        std::vector<int32_t> ef_off(n + 1, 0), ef(3L * m.n_faces);
        for (long k = 0; k < 3L * m.n_faces; ++k) ++ef_off[m.face_edges[k] + 1];
        for (int e = 0; e < n; ++e) ef_off[e + 1] += ef_off[e];
        std::vector<int32_t> fill(ef_off.begin(), ef_off.end() - 1);
        for (int f = 0; f < m.n_faces; ++f)
            for (int k = 0; k < 3; ++k) ef[fill[m.face_edges[3 * f + k]]++] = 3 * f + k;
        std::vector<int32_t> ve_off(m.n_primal + 1, 0), ve(2L * n);
        for (long k = 0; k < 2L * n; ++k) ++ve_off[m.edge_vertices[k] + 1];
        for (int v = 0; v < m.n_primal; ++v) ve_off[v + 1] += ve_off[v];
        fill.assign(ve_off.begin(), ve_off.end() - 1);
        for (int e = 0; e < n; ++e) {
            ve[fill[m.edge_vertices[2 * e]]++] = 2 * e;
            ve[fill[m.edge_vertices[2 * e + 1]]++] = 2 * e + 1;
        }
        upload_i(face_edges_, m.face_edges, 3L * m.n_faces, s);
        upload_i(face_signs_, m.face_signs, 3L * m.n_faces, s);
        upload_i(edge_vertices_, m.edge_vertices, 2L * n, s);
        upload(edge_boundary_d_, m.edge_boundary, n, s);
        upload(vertex_boundary_d_, m.vertex_boundary, m.n_primal, s);
        upload(star0_, m.star0, m.n_primal, s);
        upload(star1_, m.star1, n, s);
        upload(star2_, m.star2, m.n_faces, s);
        upload_i(edge_face_offsets_, ef_off.data(), ef_off.size(), s);
        upload_i(edge_face_items_, ef.data(), ef.size(), s);
        upload_i(vertex_edge_offsets_, ve_off.data(), ve_off.size(), s);
        upload_i(vertex_edge_items_, ve.data(), ve.size(), s);
        face_value_.allocate(m.n_faces);
        vertex_value_.allocate(m.n_primal);
        VB_CUDA(cudaStreamSynchronize(s));
        lap_ = Laplacian{n,
                         m.n_faces,
                         m.n_primal,
                         iptr(face_edges_),
                         iptr(face_signs_),
                         star0_.p,
                         star1_.p,
                         star2_.p,
                         iptr(edge_vertices_),
                         edge_boundary_d_.p,
                         vertex_boundary_d_.p,
                         iptr(edge_face_offsets_),
                         iptr(edge_face_items_),
                         iptr(vertex_edge_offsets_),
                         iptr(vertex_edge_items_)};
    }

    // out = A in; `gated`: skipped once the iteration is done.
    void apply(const double* in, double* out, bool gated) {
        cudaStream_t s = st_.s;
        const double* status = gated ? status_.p : nullptr;
        ks_lap_faces_vertices<<<blocks_s(std::max(lap_.n_faces, lap_.n_vertices)), kT, 0, s>>>(
            lap_, in, face_value_.p, vertex_value_.p, status);
        ks_lap_edges<<<blocks_s(lap_.n_edges), kT, 0, s>>>(lap_, in, face_value_.p, vertex_value_.p, out, status);
    }

    // status[kDot] = a.b in the chosen order.
    void dot(const double* a, const double* b) {
        cudaStream_t s = st_.s;
        if (sequential_dots_) {
            ks_dot_sequential<<<1, kT, 0, s>>>(v_.n_edges, a, b, status_.p);
        } else {
            ks_dot_partials<<<cg_blocks_, kT, 0, s>>>(v_.n_edges, a, b, partials_.p, cg_blocks_, status_.p);
            ks_dot_tree<<<1, kT, 0, s>>>(partials_.p, cg_blocks_, status_.p);
        }
    }

    // z = M^-1 r on the stream (skipped once the iteration is done).
    void precondition() {
        cudaStream_t s = st_.s;
        if (pc_.ic && ic_shared_bytes_)
            ks_ic_solve_shared<<<1, 1024, ic_shared_bytes_, s>>>(pc_, v_.n_edges, r_.p, z_.p, status_.p);
        else if (pc_.ic)
            ks_ic_solve<<<1, 1024, 0, s>>>(pc_, r_.p, z_.p, status_.p);
        else
            ks_jacobi<<<cg_blocks_, kT, 0, s>>>(v_.n_edges, r_.p, pc_.jacobi, z_.p, status_.p);
    }

    // The CPU solver's preconditioner: its IC(0) factor, with the level sets
    // of both triangular solves, or its diagonal.
    void setup_preconditioner(const vapor_simplicial3d_mesh& m, bool jacobi_only) {
        const int n = m.n_edges;
        cudaStream_t s = st_.s;
        pc_ = Precond{};
        if (m.jacobi_diagonal) {
            for (int i = 0; i < n; ++i)
                require_s(std::isfinite(m.jacobi_diagonal[i]) && m.jacobi_diagonal[i] != 0, "Jacobi diagonal");
            upload(jacobi_, m.jacobi_diagonal, n, s);
            pc_.jacobi = jacobi_.p;
        } else {
            require_s(m.ic_offsets != nullptr && !jacobi_only,
                      "the preconditioner needs the Jacobi diagonal or the IC factor");
        }
        if (!m.ic_offsets || jacobi_only) return;
        const long nnz = check_offsets(m.ic_offsets, n, "IC factor offsets");
        require_s(m.ic_diagonal && (nnz == 0 || (m.ic_columns && m.ic_values)), "IC factor arrays");
        for (int i = 0; i < n; ++i) {
            require_s(std::isfinite(m.ic_diagonal[i]) && m.ic_diagonal[i] > 0, "IC factor diagonal");
            for (int k = m.ic_offsets[i]; k < m.ic_offsets[i + 1]; ++k)
                require_s(m.ic_columns[k] >= 0 && m.ic_columns[k] < i &&
                              (k == m.ic_offsets[i] || m.ic_columns[k] > m.ic_columns[k - 1]),
                          "IC factor columns (strictly lower, ascending)");
        }
        // forward levels: a row after every row it reads
        std::vector<int> level(n, 0);
        int f_levels = 0;
        for (int i = 0; i < n; ++i) {
            int l = 0;
            for (int k = m.ic_offsets[i]; k < m.ic_offsets[i + 1]; ++k) l = std::max(l, level[m.ic_columns[k]] + 1);
            level[i] = l;
            f_levels = std::max(f_levels, l + 1);
        }
        auto group = [&](const std::vector<int>& lv, int levels, std::vector<int32_t>& off, std::vector<int32_t>& items) {
            off.assign(levels + 1, 0);
            for (int i = 0; i < n; ++i) ++off[lv[i] + 1];
            for (int l = 0; l < levels; ++l) off[l + 1] += off[l];
            items.assign(n, 0);
            std::vector<int32_t> fill(off.begin(), off.end() - 1);
            for (int i = 0; i < n; ++i) items[fill[lv[i]]++] = i;
        };
        std::vector<int32_t> f_off, f_rows;
        group(level, f_levels, f_off, f_rows);
        // the transpose: for each column c, (row, value) in descending row order
        std::vector<int32_t> t_off(n + 1, 0), t_rows(nnz);
        std::vector<double> t_values(nnz);
        for (long k = 0; k < nnz; ++k) ++t_off[m.ic_columns[k] + 1];
        for (int c = 0; c < n; ++c) t_off[c + 1] += t_off[c];
        std::vector<int32_t> fill(t_off.begin(), t_off.end() - 1);
        for (int i = n - 1; i >= 0; --i)
            for (int k = m.ic_offsets[i]; k < m.ic_offsets[i + 1]; ++k) {
                const int c = m.ic_columns[k];
                t_rows[fill[c]] = i;
                t_values[fill[c]++] = m.ic_values[k];
            }
        // backward levels: a column after every later row it reads
        std::fill(level.begin(), level.end(), 0);
        int b_levels = 0;
        for (int c = n - 1; c >= 0; --c) {
            int l = 0;
            for (int k = t_off[c]; k < t_off[c + 1]; ++k) l = std::max(l, level[t_rows[k]] + 1);
            level[c] = l;
            b_levels = std::max(b_levels, l + 1);
        }
        std::vector<int32_t> b_off, b_cols;
        group(level, b_levels, b_off, b_cols);
        upload_i(ic_offsets_, m.ic_offsets, n + 1L, s);
        upload_i(ic_columns_, m.ic_columns, nnz, s);
        upload(ic_values_, m.ic_values, nnz, s);
        upload(ic_diagonal_, m.ic_diagonal, n, s);
        upload_i(f_level_offsets_, f_off.data(), f_off.size(), s);
        upload_i(f_rows_, f_rows.data(), f_rows.size(), s);
        upload_i(t_offsets_, t_off.data(), t_off.size(), s);
        upload_i(t_rows_, t_rows.data(), t_rows.size(), s);
        upload(t_values_, t_values.data(), t_values.size(), s);
        upload_i(b_level_offsets_, b_off.data(), b_off.size(), s);
        upload_i(b_columns_, b_cols.data(), b_cols.size(), s);
        std::vector<int32_t> f_tab, b_tab;
        for (int k = 0; k < n; ++k) {
            const int i = f_rows[k];
            f_tab.insert(f_tab.end(), {i, m.ic_offsets[i], m.ic_offsets[i + 1], 0});
            const int c = b_cols[k];
            b_tab.insert(b_tab.end(), {c, t_off[c], t_off[c + 1], 0});
        }
        upload_i(f_table_, f_tab.data(), f_tab.size(), s);
        upload_i(b_table_, b_tab.data(), b_tab.size(), s);
        VB_CUDA(cudaStreamSynchronize(s));
        pc_.ic = 1;
        pc_.l_offsets = iptr(ic_offsets_);
        pc_.l_columns = iptr(ic_columns_);
        pc_.l_values = ic_values_.p;
        pc_.l_diagonal = ic_diagonal_.p;
        pc_.f_level_offsets = iptr(f_level_offsets_);
        pc_.f_rows = iptr(f_rows_);
        pc_.f_levels = f_levels;
        pc_.t_offsets = iptr(t_offsets_);
        pc_.t_rows = iptr(t_rows_);
        pc_.t_values = t_values_.p;
        pc_.b_level_offsets = iptr(b_level_offsets_);
        pc_.b_columns = iptr(b_columns_);
        pc_.b_levels = b_levels;
        pc_.f_table = reinterpret_cast<const int4*>(f_table_.p);
        pc_.b_table = reinterpret_cast<const int4*>(b_table_.p);
        // the shared-memory form when the vector fits the block's shared memory
        int device = 0, limit = 0;
        VB_CUDA(cudaGetDevice(&device));
        VB_CUDA(cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        const size_t need = sizeof(double) * size_t(n);
        ic_shared_bytes_ = 0;
        if (need + sizeof(double) * 32 * 32 <= size_t(limit)) {
            VB_CUDA(cudaFuncSetAttribute(ks_ic_solve_shared, cudaFuncAttributeMaxDynamicSharedMemorySize, int(need)));
            ic_shared_bytes_ = need;
        }
    }

    void put_velocity(const double* dual_velocity, const double* samples) {
        cudaStream_t s = st_.s;
        VB_CUDA(cudaMemcpyAsync(dual_velocity_.p, dual_velocity, sizeof(double) * 3 * v_.n_dual,
                                cudaMemcpyHostToDevice, s));
        if (samples)
            VB_CUDA(cudaMemcpyAsync(samples_.p, samples, sizeof(double) * 3 * v_.n_nodes, cudaMemcpyHostToDevice, s));
        VB_CUDA(cudaMemsetAsync(error_.p, 0, sizeof(int), s));
    }

    void finish() {
        int error = 0;
        VB_CUDA(cudaMemcpyAsync(&error, error_.p, sizeof(int), cudaMemcpyDeviceToHost, st_.s));
        VB_CUDA(cudaStreamSynchronize(st_.s));
        if (error & simplicial::kInvalidWeights) fail(VAPOR_RUNTIME_ERROR, "Invalid generalized barycentric weights");
        if (error & simplicial::kEscapedSubdivision)
            fail(VAPOR_RUNTIME_ERROR, "GPU sample escaped circumcentric subdivision");
    }

    void read_status(double* st) {
        VB_CUDA(cudaMemcpyAsync(st, status_.p, sizeof(double) * kSlots, cudaMemcpyDeviceToHost, st_.s));
        VB_CUDA(cudaStreamSynchronize(st_.s));
    }

    Stream st_;
    View v_{};
    DevArray<double> dual_position_, node_position_, tet_geometry_, wall_geometry_, box_planes_, sub_gradients_;
    DevArray<uint32_t> tet_vertices_, dual_hint_, primal_hint_, bin_offsets_, bin_items_, wall_offsets_, wall_items_,
        wall_owner_, cell_corners_, corner_vertices_, corner_cones_, cone_planes_, neighbor_offsets_, neighbors_,
        sub_offsets_, sub_nodes_, loop_offsets_, loop_items_, dual_edges_;
    Laplacian lap_{};
    DevArray<uint32_t> face_edges_, face_signs_, edge_vertices_, edge_face_offsets_, edge_face_items_,
        vertex_edge_offsets_, vertex_edge_items_;
    DevArray<uint8_t> edge_boundary_d_, vertex_boundary_d_;
    DevArray<double> star0_, star1_, star2_, face_value_, vertex_value_;
    bool sequential_dots_ = true;
    DevArray<double> dual_velocity_, samples_, traced_, traced_velocity_, integral_, omega_;
    DevArray<float> density_in_, density_out_;
    DevArray<uint32_t> error_;
    DevArray<double> b_, x_, r_, z_, p_, ap_, partials_, status_;
    std::vector<uint8_t> edge_boundary_;
    int cg_blocks_ = 1;
    Precond pc_{};
    size_t ic_shared_bytes_ = 0;
    DevArray<double> jacobi_, ic_values_, ic_diagonal_, t_values_;
    DevArray<uint32_t> ic_offsets_, ic_columns_, f_level_offsets_, f_rows_, t_offsets_, t_rows_, b_level_offsets_,
        b_columns_, f_table_, b_table_;
};

}  // namespace vb

// ---- C ABI ----

struct vapor_simplicial3d {
    vb::SimplicialStages stages;
    vapor_simplicial3d(const vapor_simplicial3d_mesh& m, int search, int dots, int precond)
        : stages(m, search, dots, precond) {}
};

#define VB_APIS extern "C" __attribute__((visibility("default")))

VB_APIS vapor_status vapor_simplicial3d_create(const vapor_simplicial3d_mesh* mesh, int32_t site_search,
                                               int32_t dot_order, int32_t preconditioner, vapor_simplicial3d** out) {
    return vb::guard([&] {
        if (!out || !mesh) vb::fail(VAPOR_INVALID_ARGUMENT, "null mesh or output");
        *out = nullptr;
        if (site_search < 0 || site_search > 2) vb::fail(VAPOR_INVALID_ARGUMENT, "site_search must be 0, 1 or 2");
        if (dot_order < 0 || dot_order > 2) vb::fail(VAPOR_INVALID_ARGUMENT, "dot_order must be 0, 1 or 2");
        if (preconditioner < 0 || preconditioner > 1) vb::fail(VAPOR_INVALID_ARGUMENT, "preconditioner must be 0 or 1");
        *out = new vapor_simplicial3d(*mesh, site_search, dot_order, preconditioner);
    });
}
VB_APIS vapor_status vapor_simplicial3d_destroy(vapor_simplicial3d* stages) {
    return vb::guard([&] { delete stages; });
}
VB_APIS vapor_status vapor_simplicial3d_advect_circulation(vapor_simplicial3d* stages, double dt,
                                                           const double* dual_velocity, const double* node_samples,
                                                           double* omega) {
    return vb::guard([&] {
        if (!stages) vb::fail(VAPOR_INVALID_ARGUMENT, "null handle");
        stages->stages.advect_circulation(dt, dual_velocity, node_samples, omega);
    });
}
VB_APIS vapor_status vapor_simplicial3d_advect_density(vapor_simplicial3d* stages, double dt, double decay,
                                                       const double* dual_velocity, const double* node_samples,
                                                       const float* vertex_density, float* density_out) {
    return vb::guard([&] {
        if (!stages) vb::fail(VAPOR_INVALID_ARGUMENT, "null handle");
        stages->stages.advect_density(dt, decay, dual_velocity, node_samples, vertex_density, density_out);
    });
}
VB_APIS vapor_status vapor_simplicial3d_recover(vapor_simplicial3d* stages, const double* rhs, const double* x0,
                                                int32_t iterations, double absolute_tolerance,
                                                double relative_tolerance, double* x,
                                                vapor_linear_solve_result* result) {
    return vb::guard([&] {
        if (!stages || !result) vb::fail(VAPOR_INVALID_ARGUMENT, "null handle or result");
        *result = stages->stages.recover(rhs, x0, iterations, absolute_tolerance, relative_tolerance, x);
    });
}
