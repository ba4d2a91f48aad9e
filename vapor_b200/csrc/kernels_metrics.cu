// Comparison metrics of a MAC state on the device: the quantities the
// reference's diagnostic harness prints for its Reflection / MacCormack
// comparison (tests/ReflectionComparison.hpp:32-75), computed on the host
// there. Per cell: density mass, square and the absolute differences to the
// +x, +y, +z neighbours; the squared divergence; and for smoke cells
// (density > 0.001) the CFL number of the velocity sampled at the cell centre
// and whether the forward or backward trace over one frame leaves the box.
// The per-cell arithmetic follows the harness's FP32 expressions; the sums are
// FP64 in a fixed tree (deterministic, within FP64 rounding of the harness's
// sequential sums); counts and maxima are exact.
#include "engine.hpp"
#include "kernels.hpp"

namespace vb {
namespace {

constexpr int kThreads = 256;

struct MetricsControl {
    unsigned long long smoke_cells, cfl_fallback, boundary_fallback;
    unsigned int max_div_bits, max_cfl_bits, nonfinite, reserved;
};

__global__ void k_metrics_begin(MetricsControl* m) {
    m->smoke_cells = m->cfl_fallback = m->boundary_fallback = 0ull;
    m->max_div_bits = m->max_cfl_bits = m->nonfinite = 0u;
}

__global__ void __launch_bounds__(kThreads) k_metrics(Grid g, float fps, float cfl_limit,
                                                      const float* __restrict__ d, const float* __restrict__ u,
                                                      const float* __restrict__ v, const float* __restrict__ w,
                                                      double* __restrict__ partials, MetricsControl* m) {
    __shared__ double s_sum[32];
    __shared__ float s_max[32];
    __shared__ unsigned long long s_cnt[32];
    const int n = g.n;
    const size_t cells = size_t(n) * n * n;
    const float box = g.box;
    double mass = 0.0, grad = 0.0, square = 0.0, divsq = 0.0;
    float dmax = 0.f, cmax = 0.f;
    unsigned long long smoke = 0, cfl_fb = 0, bnd_fb = 0;
    unsigned int bad = 0u;
    for (size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x; c < cells; c += size_t(gridDim.x) * blockDim.x) {
        const int z = int(c / (size_t(n) * n)), r = int(c - size_t(z) * n * n), y = r / n, x = r - y * n;
        const float dv = d[c];
        mass += dv;
        square += double(dv) * dv;
        if (x + 1 < n) grad += fabsf(dv - d[c + 1]);
        if (y + 1 < n) grad += fabsf(dv - d[c + n]);
        if (z + 1 < n) grad += fabsf(dv - d[c + size_t(n) * n]);
        const float div = (u[index_of(n, FACE_X, x + 1, y, z)] - u[index_of(n, FACE_X, x, y, z)] +
                           v[index_of(n, FACE_Y, x, y + 1, z)] - v[index_of(n, FACE_Y, x, y, z)] +
                           w[index_of(n, FACE_Z, x, y, z + 1)] - w[index_of(n, FACE_Z, x, y, z)]) /
                          g.h;
        if (!isfinite(div)) bad = 1u;
        divsq += double(div) * div;
        dmax = maxf_ref(dmax, fabsf(div));
        if (dv <= .001f) continue;
        ++smoke;
        // cell centre (x + .5) / n of the unit box, scaled to the box
        const float px = (float(x) + .5f) / float(n) * box, py = (float(y) + .5f) / float(n) * box,
                    pz = (float(z) + .5f) / float(n) * box;
        const Vel vel = velocity_at(u, v, w, n, g.h, px, py, pz);
        const float cfl = sqrtf(vel.x * vel.x + vel.y * vel.y + vel.z * vel.z) * float(n) / (box * fps);
        cmax = fmaxf(cmax, cfl);
        if (cfl > cfl_limit) ++cfl_fb;
        const float step = 1.f / fps;
        const float ax = px - vel.x * step, ay = py - vel.y * step, az = pz - vel.z * step;
        const float bx = px + vel.x * step, by = py + vel.y * step, bz = pz + vel.z * step;
        if (ax < 0.f || ax > box || ay < 0.f || ay > box || az < 0.f || az > box || bx < 0.f || bx > box ||
            by < 0.f || by > box || bz < 0.f || bz > box)
            ++bnd_fb;
    }
    const double sm = block_sum(mass, s_sum);
    const double sg = block_sum(grad, s_sum);
    const double ss = block_sum(square, s_sum);
    const double sd = block_sum(divsq, s_sum);
    const float bd = block_max(dmax, s_max);
    __syncthreads();
    const float bc = block_max(cmax, s_max);
    const unsigned long long nsm = block_sum(smoke, s_cnt);
    const unsigned long long ncf = block_sum(cfl_fb, s_cnt);
    const unsigned long long nbf = block_sum(bnd_fb, s_cnt);
    const int any_bad = __syncthreads_or(int(bad));
    if (threadIdx.x == 0) {
        double* p = partials + 4 * blockIdx.x;
        p[0] = sm;
        p[1] = sg;
        p[2] = ss;
        p[3] = sd;
        atomic_max_nonneg(&m->max_div_bits, bd);
        atomic_max_nonneg(&m->max_cfl_bits, bc);
        atomicAdd(&m->smoke_cells, nsm);
        atomicAdd(&m->cfl_fallback, ncf);
        atomicAdd(&m->boundary_fallback, nbf);
        if (any_bad) atomicOr(&m->nonfinite, 1u);
    }
}

__global__ void k_metrics_finish(const double* __restrict__ partials, int blocks, const MetricsControl* m,
                                 double cells, vapor_comparison_metrics* out) {
    __shared__ double s_sum[32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = threadIdx.x; i < blocks; i += blockDim.x)
        for (int k = 0; k < 4; ++k) acc[k] += partials[4 * i + k];
    double tot[4];
    for (int k = 0; k < 4; ++k) {
        tot[k] = block_sum(acc[k], s_sum);
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    out->mass_sum = tot[0];
    out->mass = tot[0] / cells;
    out->grad_per_mass = tot[1] / tot[0];
    out->square_per_mass = tot[2] / tot[0];
    out->rms_div = sqrt(tot[3] / cells);
    out->max_div = double(__uint_as_float(m->max_div_bits));
    out->smoke_cells = (long long)m->smoke_cells;
    out->cfl_fallback = (long long)m->cfl_fallback;
    out->boundary_fallback = (long long)m->boundary_fallback;
    out->max_cfl = double(__uint_as_float(m->max_cfl_bits));
    out->nonfinite = int(m->nonfinite);
}

}  // namespace

void comparison_metrics(const Grid& g, float fps, float cfl_limit, const float* d, const float* u, const float* v,
                        const float* w, vapor_comparison_metrics* out, cudaStream_t s) {
    const size_t cells = size_t(g.n) * g.n * g.n;
    const int blocks = reduction_blocks(cells);
    // one allocation: the block partials, the control block, the result
    constexpr size_t kCtrl = (sizeof(MetricsControl) + 7) / 8, kOut = (sizeof(vapor_comparison_metrics) + 7) / 8;
    DevArray<double> buf;
    buf.allocate(size_t(4) * blocks + kCtrl + kOut);
    double* partials = buf.p;
    auto* m = reinterpret_cast<MetricsControl*>(buf.p + size_t(4) * blocks);
    auto* dev = reinterpret_cast<vapor_comparison_metrics*>(buf.p + size_t(4) * blocks + kCtrl);
    count_launch();
    k_metrics_begin<<<1, 1, 0, s>>>(m);
    count_launch();
    k_metrics<<<blocks, kThreads, 0, s>>>(g, fps, cfl_limit, d, u, v, w, partials, m);
    count_launch();
    k_metrics_finish<<<1, 256, 0, s>>>(partials, blocks, m, double(cells), dev);
    VB_CUDA(cudaGetLastError());
    VB_CUDA(cudaMemcpyAsync(out, dev, sizeof(vapor_comparison_metrics), cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaStreamSynchronize(s));
    if (out->nonfinite) fail(VAPOR_NON_FINITE, "Non-finite MAC velocity");
}

}  // namespace vb
