// Host-side engine: buffers, projection orchestration, resident coordinator
// (GpuMacSimulation3D's role, gpu/GpuMacSimulation3D.cpp:49-264) and staged
// stages (GpuPressureSolver.cpp / GpuAdvection.cpp).
#include "engine.hpp"
#include "unet.hpp"

#include <algorithm>
#include <atomic>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>

namespace vb {

void fail(vapor_status code, const std::string& message) { throw Error(code, message); }

void cuda_check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const vapor_status code = e == cudaErrorMemoryAllocation ? VAPOR_OUT_OF_MEMORY : VAPOR_RUNTIME_ERROR;
    throw Error(code, std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}

template <class T>
void DevArray<T>::allocate(size_t count) {
    release();
    if (count == 0) return;
    void* ptr = nullptr;
    VB_CUDA(cudaMalloc(&ptr, count * sizeof(T)));
    p = static_cast<T*>(ptr);
    n = count;
}
template <class T>
void DevArray<T>::release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
}
template <class T>
void DevArray<T>::zero(cudaStream_t s) {
    if (p) VB_CUDA(cudaMemsetAsync(p, 0, bytes(), s));
}
template struct DevArray<float>;
template struct DevArray<double>;
template struct DevArray<uint32_t>;
template struct DevArray<uint16_t>;
template struct DevArray<uint8_t>;

Stream::Stream() { VB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
Stream::~Stream() {
    if (s) cudaStreamDestroy(s);
}

void validate_grid(int n, float box) {
    if (n <= 0) fail(VAPOR_INVALID_ARGUMENT, "MAC grid resolution must be positive");
    const size_t nn = size_t(n);
    const size_t limit = size_t(std::numeric_limits<int>::max());
    if (nn > limit / nn || nn * nn > limit / (nn + 1)) fail(VAPOR_LENGTH_ERROR, "MAC grid exceeds the supported index range");
    if (!std::isfinite(box) || box <= 0.f || box / float(n) <= 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "MAC grid requires a finite positive box size and spacing");
}

static bool valid_options(const vapor_linear_solve_options& o) {
    return o.max_iterations >= 0 && o.residual_check_interval > 0 && std::isfinite(o.absolute_tolerance) &&
           o.absolute_tolerance >= 0.0 && std::isfinite(o.relative_tolerance) && o.relative_tolerance >= 0.0;
}

// ---------------------------------------------------------------------------
// PhaseTimer
// ---------------------------------------------------------------------------
PhaseTimer::~PhaseTimer() {
    for (auto& p : pending_) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (auto e : pool_) cudaEventDestroy(e);
    for (auto e : open_)
        if (e) cudaEventDestroy(e);
}

cudaEvent_t PhaseTimer::take() {
    if (!pool_.empty()) {
        cudaEvent_t e = pool_.back();
        pool_.pop_back();
        return e;
    }
    cudaEvent_t e;
    VB_CUDA(cudaEventCreate(&e));
    return e;
}

void PhaseTimer::enable(bool on) {
    fold(true);
    on_ = on;
    acc_ = vapor_phase_timings{};
}

void PhaseTimer::begin(int phase) {
    if (!on_) return;
    cudaEvent_t e = take();
    VB_CUDA(cudaEventRecord(e, s_));
    if (open_[phase]) pool_.push_back(open_[phase]);
    open_[phase] = e;
}

void PhaseTimer::end(int phase, long long launches) {
    if (!on_ || !open_[phase]) return;
    cudaEvent_t e = take();
    VB_CUDA(cudaEventRecord(e, s_));
    pending_.push_back({phase, open_[phase], e, launches});
    open_[phase] = nullptr;
    if (pending_.size() > 4096) fold(true);
}

void PhaseTimer::fold(bool wait) {
    if (pending_.empty()) return;
    if (wait) VB_CUDA(cudaStreamSynchronize(s_));
    size_t keep = 0;
    for (size_t i = 0; i < pending_.size(); ++i) {
        Pending& p = pending_[i];
        if (!wait && cudaEventQuery(p.b) != cudaSuccess) {
            pending_[keep++] = p;
            continue;
        }
        float ms = 0.f;
        VB_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
        acc_.milliseconds[p.phase] += ms;
        acc_.launches[p.phase] += p.launches;
        acc_.intervals[p.phase] += 1;
        pool_.push_back(p.a);
        pool_.push_back(p.b);
    }
    pending_.resize(keep);
    (void)cudaGetLastError();  // clear cudaErrorNotReady from queries
}

vapor_phase_timings PhaseTimer::totals() {
    fold(true);
    return acc_;
}

// ---------------------------------------------------------------------------
// Workspace
// ---------------------------------------------------------------------------
Workspace::Workspace(int n, float box, cudaStream_t stream)
    : n_(n), box_(box), stream_(stream), timer_(stream) {
    validate_grid(n, box);
    const size_t faces = size_t(n) * n * (n + 1);
    const size_t slots = rb_count(n);  // red-black split storage
    b_.allocate(slots);
    p_.allocate(slots);
    if (sor_blocked_applies(n)) x_alt_.allocate(slots);  // out-of-place blocked sweeps
    fwd_.allocate(faces);
    partial_capacity_ = reduction_blocks(faces);
    partials_.allocate(size_t(partial_capacity_));
    VB_CUDA(cudaMalloc(&ctrl_, sizeof(ProjControl)));
    VB_CUDA(cudaMalloc(&diag_, sizeof(DiagControl)));
    VB_CUDA(cudaMallocHost(&ctrl_host_, sizeof(ProjControl)));
    VB_CUDA(cudaMallocHost(&diag_host_, sizeof(DiagControl)));
    VB_CUDA(cudaMallocHost(&done_host_, sizeof(int)));
    std::memset(ctrl_host_, 0, sizeof(ProjControl));
    reset_buffers();
    VB_CUDA(cudaStreamSynchronize(stream_));
}

Workspace::~Workspace() {
    if (stream_) cudaStreamSynchronize(stream_);
    if (ctrl_) cudaFree(ctrl_);
    if (cg_) cudaFree(cg_);
    if (diag_) cudaFree(diag_);
    if (ctrl_host_) cudaFreeHost(ctrl_host_);
    if (diag_host_) cudaFreeHost(diag_host_);
    if (done_host_) cudaFreeHost(done_host_);
}

void Workspace::reset_buffers() {
    b_.zero(stream_);
    p_.zero(stream_);
    fwd_.zero(stream_);
    VB_CUDA(cudaMemsetAsync(ctrl_, 0, sizeof(ProjControl), stream_));
    VB_CUDA(cudaMemsetAsync(diag_, 0, sizeof(DiagControl), stream_));
    total_iterations_ = 0;
    sticky_errors_ = 0u;
}

void Workspace::clear_errors() { VB_CUDA(cudaMemsetAsync(&ctrl_->sticky_nonfinite, 0, sizeof(unsigned int), stream_)); }

void Workspace::advect(int loc, float dt, float cfl, bool maccormack, const float* src, const float* u,
                       const float* v, const float* w, float* out, float post_scale) {
    timer_.begin(VAPOR_PHASE_ADVECT);
    launch_advect(grid(), loc, dt, cfl, maccormack, src, u, v, w, fwd_.p, out, post_scale, stream_);
    timer_.end(VAPOR_PHASE_ADVECT, maccormack ? 2 : 1);
    VB_CUDA(cudaGetLastError());
}

void Workspace::advect_velocity(float dt, float cfl, bool maccormack, const float* const src[3], const float* u,
                                const float* v, const float* w, float* const out[3]) {
    const size_t faces = size_t(n_) * n_ * (n_ + 1);
    if (maccormack) {
        if (capturing_ && fwd3_.n != 3 * faces) fail(VAPOR_RUNTIME_ERROR, "velocity advection scratch not prepared");
        ensure_velocity_scratch();
    }
    float* fwd[3] = {fwd3_.p, fwd3_.p + faces, fwd3_.p + 2 * faces};
    timer_.begin(VAPOR_PHASE_ADVECT);
    launch_advect_velocity(grid(), dt, cfl, maccormack, src, u, v, w, fwd, out, maccormack ? vel_cache_.p : nullptr,
                           stream_);
    timer_.end(VAPOR_PHASE_ADVECT, maccormack ? 2 : 1);
    VB_CUDA(cudaGetLastError());
}

void Workspace::ensure_velocity_scratch() {
    const size_t faces = size_t(n_) * n_ * (n_ + 1);
    if (fwd3_.n != 3 * faces) fwd3_.allocate(3 * faces);
    if (vel_cache_.n != 9 * faces) vel_cache_.allocate(9 * faces);
}

void Workspace::advect_smoke(float dt, float cfl, bool maccormack, const float* src, const float* u, const float* v,
                             const float* w, float* out, float post_scale) {
    // the velocity cache is free once the velocity has been advected; it
    // holds 9 face arrays, more than the smoke's 3 cell arrays
    float* cache = (maccormack && vel_cache_.p) ? vel_cache_.p : nullptr;
    timer_.begin(VAPOR_PHASE_ADVECT);
    launch_advect_smoke(grid(), dt, cfl, maccormack, src, u, v, w, fwd_.p, out, post_scale, cache, stream_);
    timer_.end(VAPOR_PHASE_ADVECT, maccormack ? 2 : 1);
    VB_CUDA(cudaGetLastError());
}

void Workspace::ensure_mixed() {
    const size_t cells = rb_count(n_);
    for (auto& x : x64_)
        if (x.n != cells) x.allocate(cells);
    if (r32_.n != cells) {
        r32_.allocate(cells);
        r32_.zero(stream_);  // padding slots stay zero (they enter the CG dot products)
    }
}

// Adds a while-loop node at the current capture position of stream `s` whose
// body is recorded by `body` on the workspace's body stream. The loop runs
// while the handle's value (set by a kernel before the node and by the body's
// last kernel) is nonzero.
template <class Body>
static void add_conditional(cudaStream_t s, cudaStream_t body_stream, cudaGraphConditionalHandle handle,
                            cudaGraphConditionalNodeType type, Body&& body) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    VB_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, &deps, &ndeps));
    if (status != cudaStreamCaptureStatusActive) fail(VAPOR_RUNTIME_ERROR, "stream is not capturing");
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = handle;
    params.conditional.type = type;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    VB_CUDA(cudaGraphAddNode(&node, graph, deps, ndeps, &params));
    VB_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body_graph = params.conditional.phGraph_out[0];
    VB_CUDA(cudaStreamBeginCaptureToGraph(body_stream, body_graph, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
    body(body_stream);
    cudaGraph_t captured = nullptr;
    VB_CUDA(cudaStreamEndCapture(body_stream, &captured));
}

template <class Body>
static void add_while_loop(cudaStream_t s, cudaStream_t body_stream, cudaGraphConditionalHandle handle,
                           Body&& body) {
    add_conditional(s, body_stream, handle, cudaGraphCondTypeWhile, body);
}

static cudaGraphConditionalHandle new_condition(cudaStream_t s) {
    cudaStreamCaptureStatus status;
    cudaGraph_t graph;
    VB_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &graph, nullptr, nullptr));
    if (status != cudaStreamCaptureStatusActive) fail(VAPOR_RUNTIME_ERROR, "stream is not capturing");
    cudaGraphConditionalHandle h;
    VB_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 0, 0));
    return h;
}

void Workspace::set_solid(const uint8_t* mask) {
    VB_CUDA(cudaStreamSynchronize(stream_));
    if (!mask) {
        solid_.release();
        solid_diag_.release();
        fluid_ = 0.0;
        return;
    }
    const int n = n_;
    const size_t cells = size_t(n) * n * n;
    const RBLayout L = rb_layout(n);
    auto solid = [&](int x, int y, int z) { return mask[(size_t(z) * n + y) * n + x] != 0; };
    std::vector<uint8_t> nat(cells), diag(rb_count(n), 0);
    size_t fluid = 0;
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const bool s = solid(x, y, z);
                nat[(size_t(z) * n + y) * n + x] = s ? 1 : 0;
                if (s) continue;
                ++fluid;
                diag[rb_index(L, x, y, z)] = uint8_t((x > 0 && !solid(x - 1, y, z)) + (x + 1 < n && !solid(x + 1, y, z)) +
                                                     (y > 0 && !solid(x, y - 1, z)) + (y + 1 < n && !solid(x, y + 1, z)) +
                                                     (z > 0 && !solid(x, y, z - 1)) + (z + 1 < n && !solid(x, y, z + 1)));
            }
    if (fluid == 0) fail(VAPOR_INVALID_ARGUMENT, "the solid mask leaves no fluid cell");
    solid_.allocate(cells);
    solid_diag_.allocate(diag.size());
    VB_CUDA(cudaMemcpy(solid_.p, nat.data(), cells, cudaMemcpyHostToDevice));
    VB_CUDA(cudaMemcpy(solid_diag_.p, diag.data(), diag.size(), cudaMemcpyHostToDevice));
    fluid_ = double(fluid);
}

namespace {
std::atomic<int> g_fpcg_sweeps{2};
std::atomic<float> g_fpcg_omega{1.2f};  // measured: 57 CG steps per 256^3 plume step against 59 at 1.0
}  // namespace

FpcgSmoothing fpcg_smoothing() { return {g_fpcg_sweeps.load(), g_fpcg_omega.load()}; }

void set_fpcg_smoothing(int sweeps, float omega) {
    if (sweeps < 1 || sweeps > 8 || !(omega > 0.0f && omega < 2.0f))
        fail(VAPOR_INVALID_ARGUMENT, "FPCG smoothing: 1..8 sweeps and 0 < omega < 2");
    g_fpcg_sweeps.store(sweeps);
    g_fpcg_omega.store(omega);
}

void Workspace::ensure_fpcg(bool coarse) {
    const size_t count = rb_count(n_);
    for (DevArray<float>* v : {&cg_p_, &cg_p2_, &cg_q_, &cg_z_})
        if (v->n != count) {
            v->allocate(count);
            v->zero(stream_);
        }
    if (cg_partials_.n < size_t(cg_partial_capacity(n_))) cg_partials_.allocate(cg_partial_capacity(n_));
    if (!cg_) VB_CUDA(cudaMalloc(&cg_, sizeof(CgControl)));
    if (coarse) {
        if (n_ % 16 != 0 || n_ < 32)
            fail(VAPOR_INVALID_ARGUMENT, "the coarse-grid network needs n divisible by 16 (n >= 32)");
        const size_t nc = size_t(n_ / 4);
        if (cg_rc_.n != nc * nc * nc) cg_rc_.allocate(nc * nc * nc);
        if (cg_rows_.n != size_t(n_) * n_ * nc) cg_rows_.allocate(size_t(n_) * n_ * nc);
    }
}

// Flexible PCG on the error equation with FP64 re-centring (x64 += e,
// r = float(b - A x64), e = 0) whenever the FP32 recurrence residual reaches
// the target or drops by kRecentreDrop; stops when the FP64 residual meets
// the target. Preconditioner: fpcg_smoothing() red-black relaxation sweeps,
// the coarse-grid correction when `coarse` is given, then the same sweeps in
// reverse colour order. Iterations count CG steps.
void Workspace::project_fpcg(const ProjectionArgs& a, unet::UNet* warm, unet::UNet* coarse, LoopCond cond,
                             cudaGraphConditionalHandle handle) {
    cudaStream_t s = stream_;
    PhaseTimer& t = timer_;
    const bool graph = capturing_;
    const size_t count = rb_count(n_);
    float* e = p_.p;
    float* r = r32_.p;
    const FpcgSmoothing sm = fpcg_smoothing();
    const int sweeps = sm.sweeps;
    // the smoothing sweeps keep the projection's obstacle mask, if any
    ProjectionArgs smooth = a;
    smooth.omega = sm.omega;
    smooth.diagonal_floor = 0.0f;
    const uint8_t* mask = a.diag;
    if (warm) warm->infer_into(n_, b_.p, ctrl_, nullptr, x64_[0].p);
    else VB_CUDA(cudaMemsetAsync(x64_[0].p, 0, x64_[0].bytes(), s));
    t.begin(VAPOR_PHASE_RESIDUAL);
    launch_refine_residual(a, b_.p, e, r, ctrl_, s);
    launch_check(ctrl_, 0, false, true, cond, s);
    t.end(VAPOR_PHASE_RESIDUAL, 2);
    // The preconditioner, z = M r, with one-colour sweeps (the temporally
    // blocked sweep measured slower at these sizes). With `dot`, the last
    // sweep also writes the partials of z.r and z.q for beta; returns their
    // block count, or 0 when they were not written.
    auto precondition = [&](cudaStream_t st, bool dot) {
        t.begin(VAPOR_PHASE_SOR);
        // the first colour sweep starts from z = 0 (and clears the other colour)
        const bool fused_start = sor_fuses_measure(n_);
        if (!fused_start) VB_CUDA(cudaMemsetAsync(cg_z_.p, 0, cg_z_.bytes(), st));
        for (int j = 0; j < sweeps; ++j) {
            launch_sor_color(smooth, 0, cg_z_.p, r, ctrl_, false, 0, false, st, false, false, fused_start && j == 0);
            launch_sor_color(smooth, 1, cg_z_.p, r, ctrl_, false, 0, false, st, false);
        }
        t.end(VAPOR_PHASE_SOR, 2 * sweeps);
        if (coarse) {
            t.begin(VAPOR_PHASE_COARSE);
            launch_restrict_residual(n_, r, cg_z_.p, cg_rows_.p, cg_rc_.p, st, mask);
            if (coarse_log_)
                launch_log_coarse(cg_rc_.p, cg_rc_.n, coarse_log_, coarse_log_capacity_, coarse_log_counter_, st);
            coarse->set_stream(st);
            const float* zc = coarse->precondition(n_ / 4, cg_rc_.p);
            coarse->set_stream(s);
            launch_coarse_correction(n_, cg_z_.p, zc, cg_rc_.p, cg_partials_.p, cg_, st, mask);
            t.end(VAPOR_PHASE_COARSE, 0);
        }
        t.begin(VAPOR_PHASE_SOR);
        int dot_blocks = 0;
        for (int j = 0; j < sweeps; ++j) {
            launch_sor_color(smooth, 1, cg_z_.p, r, ctrl_, false, 0, false, st, false);
            if (dot && j + 1 == sweeps)
                dot_blocks = launch_sor_color_dot(smooth, 0, cg_z_.p, r, cg_q_.p, cg_partials_.p,
                                                  int(cg_partials_.n), ctrl_, st);
            if (dot_blocks == 0) launch_sor_color(smooth, 0, cg_z_.p, r, ctrl_, false, 0, false, st, false);
        }
        t.end(VAPOR_PHASE_SOR, 2 * sweeps);
        return dot_blocks;
    };
    // n % 8 == 0 and no obstacles: the direction update, A p and the
    // deferred error update run as one pass (launch_cg_direction_apply), with
    // the direction in two buffers; same values as the separate passes
    const bool fused = n_ % 8 == 0 && mask == nullptr;
    float* const pbuf[2] = {cg_p_.p, cg_p2_.p};
    auto recentre_group = [&](cudaStream_t st) {
        if (fused) launch_cg_fold(count, e, pbuf, cg_, ctrl_, st);
        launch_refine_residual_gated(a, b_.p, e, r, ctrl_, st);
        launch_check_gated(ctrl_, LoopCond{}, st);
        launch_zero_error_gated(a, e, ctrl_, st);
    };
    auto update = [&](cudaStream_t st, LoopCond if_cond) {
        if (fused) launch_cg_update_r(count, r, cg_q_.p, cg_, ctrl_, if_cond, st);
        else launch_cg_update(count, e, r, cg_p_.p, cg_q_.p, cg_, ctrl_, if_cond, st);
    };
    auto iteration = [&](cudaStream_t st) {
        t.begin(VAPOR_PHASE_KRYLOV);
        if (fused) launch_cg_direction_apply(n_, cg_z_.p, pbuf, e, cg_q_.p, cg_partials_.p, cg_, st);
        else launch_apply_A_alpha(n_, cg_p_.p, cg_q_.p, cg_partials_.p, cg_, st, mask);
        t.end(VAPOR_PHASE_KRYLOV, 2);
        t.begin(VAPOR_PHASE_RESIDUAL);
        if (graph) {
            const cudaGraphConditionalHandle ifh = new_condition(st);
            LoopCond if_cond;
            if_cond.active = 1;
            if_cond.handle = (unsigned long long)ifh;
            update(st, if_cond);
            add_conditional(st, body_stream2_.s, ifh, cudaGraphCondTypeIf,
                            [&](cudaStream_t is) { recentre_group(is); });
        } else {
            update(st, LoopCond{});
            recentre_group(st);
        }
        t.end(VAPOR_PHASE_RESIDUAL, fused ? 7 : 5);
        const int dot_blocks = precondition(st, true);
        t.begin(VAPOR_PHASE_KRYLOV);
        if (dot_blocks > 0) launch_cg_beta_finish(cg_partials_.p, dot_blocks, cg_, st);
        else launch_cg_beta(count, cg_z_.p, r, cg_q_.p, cg_partials_.p, cg_, st);
        if (!fused) launch_cg_direction(count, cg_p_.p, cg_z_.p, cg_, st);
        t.end(VAPOR_PHASE_KRYLOV, (dot_blocks > 0 ? 1 : 2) + (fused ? 0 : 1));
        launch_loop_condition(ctrl_, cond, st);
    };
    precondition(s, false);
    launch_cg_rho(count, cg_z_.p, r, cg_partials_.p, cg_, s);
    if (!fused) VB_CUDA(cudaMemcpyAsync(cg_p_.p, cg_z_.p, cg_z_.bytes(), cudaMemcpyDeviceToDevice, s));
    if (graph) {
        add_while_loop(s, body_stream_.s, handle, iteration);
    } else {
        auto wait_done = [&]() {
            VB_CUDA(cudaMemcpyAsync(done_host_, &ctrl_->done, sizeof(int), cudaMemcpyDeviceToHost, s));
            VB_CUDA(cudaStreamSynchronize(s));
            t.fold(false);
            return *done_host_ != 0;
        };
        while (!wait_done()) iteration(s);
    }
}

void Workspace::project(const float* ui, const float* vi, const float* wi, float* uo, float* vo, float* wo,
                        float* uh, float* vh, float* wh, float dt, float omega, float diagonal_floor,
                        const vapor_linear_solve_options& o, int solver_kind, unet::UNet* warm,
                        unet::UNet* coarse, const float* rhs_field) {
    ProjectionArgs a{grid(), dt, omega, diagonal_floor, o};
    if (fluid_ > 0.0) {
        if (solver_kind != VAPOR_SOLVER_MIXED_REFINEMENT && solver_kind != VAPOR_SOLVER_FPCG)
            fail(VAPOR_INVALID_ARGUMENT,
                 "solid obstacles need the mixed-precision or the FPCG solver (VAPOR_SOLVER_MIXED_REFINEMENT, VAPOR_SOLVER_FPCG)");
        a.diag = solid_diag_.p;
        a.solid = solid_.p;
        a.fluid = fluid_;
    }
    cudaStream_t s = stream_;
    PhaseTimer& t = timer_;
    const bool fpcg = solver_kind == VAPOR_SOLVER_FPCG;
    const bool mixed = solver_kind == VAPOR_SOLVER_MIXED_REFINEMENT || fpcg;
    const bool graph = capturing_;
    const int interval = o.residual_check_interval;
    if (mixed) ensure_mixed();
    if (fpcg) ensure_fpcg(coarse != nullptr);
    // A device-side while loop is recorded only when the solve has one; a
    // conditional handle that no node uses makes graph instantiation fail.
    const bool loop = graph && (mixed || !o.fixed_iterations || o.max_iterations > interval);
    LoopCond cond;
    cudaGraphConditionalHandle handle = 0;
    if (loop) {
        handle = new_condition(s);
        cond.active = 1;
        cond.handle = (unsigned long long)handle;
    }
    auto wait_done = [&]() {
        VB_CUDA(cudaMemcpyAsync(done_host_, &ctrl_->done, sizeof(int), cudaMemcpyDeviceToHost, s));
        VB_CUDA(cudaStreamSynchronize(s));
        t.fold(false);
        return *done_host_ != 0;
    };
    // k guarded colour-pair sweeps on x (right-hand side rhs) on stream st.
    // Inner sweeps of the mixed solver use the divide-free relaxation.
    // With `measure`, the last colour-1 launch also records the FP32 residual.
    auto sweeps = [&](cudaStream_t st, int k, int first_index, float* x, const float* rhs, bool subtract_mean,
                      bool measure = false) {
        t.begin(VAPOR_PHASE_SOR);
        // Temporal blocking: launches of two (or one) red+black iterations,
        // out of place between x and its twin, an even number of them so
        // that the result ends in x; else one launch per colour, in place.
        const int per = sor_block_iterations(n_);
        int n2 = per == 2 ? k / 2 : 0, n1 = per == 2 ? k % 2 : k;
        if ((n2 + n1) % 2 == 1 && n2 > 0) {
            --n2;
            n1 += 2;
        }
        long long launches = 0;
        if (per > 0 && (n2 + n1) % 2 == 0 && x_alt_.p) {
            const float* src = x;
            float* dst = x_alt_.p;
            int j = 0;
            for (int l = 0; l < n2 + n1; ++l) {
                const int it = l < n2 ? 2 : 1;
                launch_sor_blocked(a, it, 0, src, dst, rhs, ctrl_, true, first_index + j, subtract_mean, st, !mixed,
                                   measure && j + it == k);
                j += it;
                src = dst;
                dst = dst == x ? x_alt_.p : x;
                ++launches;
            }
        } else {
            for (int j = 0; j < k; ++j) {
                launch_sor_color(a, 0, x, rhs, ctrl_, true, first_index + j, subtract_mean, st, !mixed);
                launch_sor_color(a, 1, x, rhs, ctrl_, true, first_index + j, subtract_mean, st, !mixed,
                                 measure && j + 1 == k);
            }
            launches = 2LL * k;
        }
        t.end(VAPOR_PHASE_SOR, launches);
    };

    t.begin(VAPOR_PHASE_RHS);
    LoopCond rhs_cond = cond;
    if (mixed) rhs_cond.active = 0;  // the mixed loop is decided by its first re-centring pass
    launch_rhs(a, ui, vi, wi, b_.p, partials_.p, partial_capacity_, ctrl_, mixed ? x64_[0].p : nullptr,
               mixed ? x64_[1].p : nullptr, rhs_cond, s, rhs_field);
    VB_CUDA(cudaMemsetAsync(p_.p, 0, p_.bytes(), s));
    t.end(VAPOR_PHASE_RHS, 3);

    if (fpcg) {
        project_fpcg(a, warm, coarse, cond, handle);
        t.begin(VAPOR_PHASE_GRADIENT);
        const int finish = launch_finish_projection64(a, b_.p, p_.p, partials_.p, partial_capacity_, ctrl_, ui, vi,
                                                      wi, uo, vo, wo, uh, vh, wh, s);
        t.end(VAPOR_PHASE_GRADIENT, finish);
    } else if (mixed) {
        // FP32 red-black sweeps on the error equation A e = r32. Every check
        // interval the FP32 residual of that equation decides whether to
        // re-centre in FP64 (x64 += e, r32 = b - A x64, e = 0) and test the FP64
        // residual against the target (the oracle's refinementSolve).
        if (warm) warm->infer_into(n_, b_.p, ctrl_, nullptr, x64_[0].p);  // x0 = network prediction
        else VB_CUDA(cudaMemsetAsync(x64_[0].p, 0, x64_[0].bytes(), s));
        t.begin(VAPOR_PHASE_RESIDUAL);
        launch_refine_residual(a, b_.p, p_.p, r32_.p, ctrl_, s);
        launch_check(ctrl_, 0, false, true, cond, s);
        t.end(VAPOR_PHASE_RESIDUAL, 2);
        const bool fused = sor_fuses_measure(n_);
        auto recentre_group = [&](cudaStream_t st, LoopCond loop_cond) {
            launch_refine_residual_gated(a, b_.p, p_.p, r32_.p, ctrl_, st);
            launch_check_gated(ctrl_, loop_cond, st);
            launch_zero_error_gated(a, p_.p, ctrl_, st);
        };
        auto chunk_then_check = [&](cudaStream_t st, int k) {
            sweeps(st, k, 0, p_.p, r32_.p, false, true);
            t.begin(VAPOR_PHASE_RESIDUAL);
            if (graph) {
                // the re-centring runs under a conditional if-node that the
                // decision kernel sets, so skipped re-centrings cost nothing
                const cudaGraphConditionalHandle ifh = new_condition(st);
                LoopCond if_cond;
                if_cond.active = 1;
                if_cond.handle = (unsigned long long)ifh;
                launch_error_check(a, p_.p, r32_.p, ctrl_, k, fused, LoopCond{}, if_cond, st);
                add_conditional(st, body_stream2_.s, ifh, cudaGraphCondTypeIf,
                                [&](cudaStream_t is) { recentre_group(is, LoopCond{}); });
                launch_loop_condition(ctrl_, cond, st);  // continue while !ctrl->done
            } else {
                launch_error_check(a, p_.p, r32_.p, ctrl_, k, fused, cond, LoopCond{}, st);
                recentre_group(st, cond);
            }
            t.end(VAPOR_PHASE_RESIDUAL, 6);
        };
        if (graph) {
            const int chunk = std::max(1, std::min(interval, o.max_iterations));
            add_while_loop(s, body_stream_.s, handle, [&](cudaStream_t bs) { chunk_then_check(bs, chunk); });
        } else {
            int it = 0;
            while (!wait_done()) {
                const int k = std::min(interval - it % interval, o.max_iterations - it);
                chunk_then_check(s, k);
                it += k;
            }
        }
        t.begin(VAPOR_PHASE_GRADIENT);
        const int finish = launch_finish_projection64(a, b_.p, p_.p, partials_.p, partial_capacity_, ctrl_, ui, vi,
                                                      wi, uo, vo, wo, uh, vh, wh, s);
        t.end(VAPOR_PHASE_GRADIENT, finish);
    } else {
        if (warm) warm->infer_into(n_, b_.p, ctrl_, p_.p, nullptr);  // x0 = network prediction
        if (o.fixed_iterations) {
            // Intermediate residual checks cannot change a fixed-budget solve:
            // the final residual and convergence are recomputed after the
            // pressure gauge (CpuPressureSolver3D.cpp:50-56).
            if (loop) {
                add_while_loop(s, body_stream_.s, handle, [&](cudaStream_t bs) {
                    sweeps(bs, interval, 0, p_.p, b_.p, true);
                    launch_check(ctrl_, interval, true, false, cond, bs);
                });
            } else {
                sweeps(s, o.max_iterations, 0, p_.p, b_.p, true);
                launch_check(ctrl_, o.max_iterations, false, false, LoopCond{}, s);
            }
        } else if (graph) {
            add_while_loop(s, body_stream_.s, handle, [&](cudaStream_t bs) {
                sweeps(bs, interval, 0, p_.p, b_.p, true);
                launch_residual(a, p_.p, b_.p, ctrl_, false, bs);
                launch_check(ctrl_, interval, true, false, cond, bs);
            });
        } else {
            int it = 0;
            bool stop = wait_done();
            while (!stop && it < o.max_iterations) {
                const int k = std::min(interval - it % interval, o.max_iterations - it);
                sweeps(s, k, 0, p_.p, b_.p, true);
                it += k;
                t.begin(VAPOR_PHASE_RESIDUAL);
                launch_residual(a, p_.p, b_.p, ctrl_, false, s);
                launch_check(ctrl_, k, true, false, LoopCond{}, s);
                t.end(VAPOR_PHASE_RESIDUAL, 2);
                stop = wait_done();
            }
        }
        t.begin(VAPOR_PHASE_GRADIENT);
        launch_pressure_mean(a, p_.p, partials_.p, partial_capacity_, ctrl_, s);
        launch_residual(a, p_.p, b_.p, ctrl_, true, s);
        launch_gradient(a, p_.p, ui, vi, wi, uo, vo, wo, uh, vh, wh, ctrl_, s);
        t.end(VAPOR_PHASE_GRADIENT, 5);
    }
    launch_finish_projection(ctrl_, s);
    VB_CUDA(cudaGetLastError());
    VB_CUDA(cudaMemcpyAsync(ctrl_host_, ctrl_, sizeof(ProjControl), cudaMemcpyDeviceToHost, s));
}

vapor_projection_result Workspace::last_result() {
    VB_CUDA(cudaStreamSynchronize(stream_));
    if (ctrl_host_->sticky_nonfinite & 1u) fail(VAPOR_NON_FINITE, "Non-finite divergence");
    if (ctrl_host_->sticky_nonfinite & 6u) fail(VAPOR_NON_FINITE, "Non-finite MAC velocity");
    return ctrl_host_->result;
}

long long Workspace::total_iterations() {
    VB_CUDA(cudaMemcpyAsync(ctrl_host_, ctrl_, sizeof(ProjControl), cudaMemcpyDeviceToHost, stream_));
    VB_CUDA(cudaStreamSynchronize(stream_));
    return ctrl_host_->total_iterations;
}

void Workspace::diagnostics(const float* u, const float* v, const float* w, vapor_fluid_diagnostics* out) {
    launch_diagnostics(grid(), u, v, w, partials_.p, partial_capacity_, diag_, stream_);
    VB_CUDA(cudaGetLastError());
    VB_CUDA(cudaMemcpyAsync(diag_host_, diag_, sizeof(DiagControl), cudaMemcpyDeviceToHost, stream_));
    VB_CUDA(cudaStreamSynchronize(stream_));
    if (diag_host_->nonfinite) fail(VAPOR_NON_FINITE, "Non-finite MAC velocity");
    const double dx = double(grid().h);
    out->kinetic_energy = float(0.5 * diag_host_->kinetic_sum * dx * dx * dx);
    uint32_t bits = diag_host_->max_velocity_bits;
    std::memcpy(&out->max_velocity, &bits, sizeof(float));
    bits = diag_host_->max_divergence_bits;
    std::memcpy(&out->max_divergence, &bits, sizeof(float));
}

// ---------------------------------------------------------------------------
// Resident simulation
// ---------------------------------------------------------------------------
Simulation::Simulation(int n, float box, const vapor_mac3d_params& p) : params(p), ws_(n, box, stream_.s) {
    const size_t cells = size_t(n) * n * n;
    const size_t faces = size_t(n) * n * (n + 1);
    for (auto& d : dens_) d.allocate(cells);
    for (auto& set : vel_)
        for (auto& c : set) c.allocate(faces);
    rng_.allocate(1);
    reset();
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
}

Simulation::~Simulation() {
    cudaStreamSynchronize(h2d_.s);
    cudaStreamSynchronize(d2h_.s);
    for (cudaEvent_t e : {in_ready_, in_taken_, out_ready_, out_done_})
        if (e) cudaEventDestroy(e);
    cudaStreamSynchronize(ws_.stream());
    release_graphs();
    if (warm_) warm_->use_own_stream();  // the networks outlive this simulation's stream
    if (coarse_) coarse_->use_own_stream();
}

void Simulation::reset() {
    cudaStream_t s = ws_.stream();
    for (auto& d : dens_) d.zero(s);
    for (auto& set : vel_)
        for (auto& c : set) c.zero(s);
    ws_.reset_buffers();
    const uint32_t seed = params.random_seed;
    VB_CUDA(cudaMemcpyAsync(rng_.p, &seed, sizeof(seed), cudaMemcpyHostToDevice, s));
    // The seed is a stack value: wait so the copy has read it.
    VB_CUDA(cudaStreamSynchronize(s));
    std::memset(ws_.ctrl_host_, 0, sizeof(ProjControl));
    cur_ = 0;
    S_ = 0;
    T_ = 1;
    U_ = 2;
}

void Simulation::set_box(float box) {
    if (!std::isfinite(box) || box <= 0.f || box / float(ws_.n()) <= 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "Invalid GPU box size");
    if (box != ws_.box()) {
        ws_.set_box(box);
        reset();
    }
}

vapor_linear_solve_options Simulation::solve_options(int iterations) const {
    if (params.use_solve_options) return params.solve;
    vapor_linear_solve_options o{};
    o.max_iterations = iterations;
    o.residual_check_interval = 8;
    o.absolute_tolerance = 1e-6;
    o.relative_tolerance = 1e-5;
    o.fixed_iterations = 1;
    return o;
}

// Emitter patch of MacGridFluidSolver3D::emit (MacGridFluidSolver3D.cpp:140-147),
// computed in the same FP32 operations. Returns false for an empty patch.
bool Simulation::emitter_box(float cxf, float cyf, float czf, float dt, EmitterBox& e) const {
    const Grid g = ws_.grid();
    const float dx = g.h;
    const float box = g.box;
    e = EmitterBox{};
    e.ec[0] = cxf * box;
    e.ec[1] = cyf * box;
    e.ec[2] = czf * box;
    e.erad = params.emitter_radius * box;
    const int R = int(e.erad / dx + 1);
    for (int a = 0; a < 3; ++a) {
        const int c = int(e.ec[a] / dx);
        e.lo[a] = std::max(0, c - R);
        e.size[a] = std::min(g.n, c + R) - e.lo[a];
    }
    if (e.size[0] <= 0 || e.size[1] <= 0 || e.size[2] <= 0) return false;
    e.kick = params.emitter_kick_multiplier * (params.emitter_kick_base + params.emitter_kick_scale * params.source_strength);
    e.apply_kick = params.emitter_kick_multiplier > 0.f;
    e.stir = params.stir_strength;
    e.dt_scale = dt * 60.0f;
    e.profile = params.emitter_profile;
    e.strength = params.source_strength;
    return true;
}

void Simulation::emit(float dt) {
    if (params.source_strength <= 0.f) return;
    const float centres[2][3] = {{params.emitter_center_x, params.emitter_center_y, params.emitter_center_z},
                                 {params.emitter2_center_x, params.emitter2_center_y, params.emitter2_center_z}};
    for (int k = 0; k < params.emitter_count; ++k) {
        EmitterBox e;
        if (!emitter_box(centres[k][0], centres[k][1], centres[k][2], dt, e)) continue;
        const size_t patch = size_t(e.size[0]) * e.size[1] * e.size[2];
        if (noise_.n < patch) fail(VAPOR_RUNTIME_ERROR, "emitter scratch not prepared");
        launch_emit(ws_.grid(), e, rng_.p, noise_.p, dens_[cur_].p, vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p,
                    ws_.stream());
    }
}

void Simulation::advect_velocity(float dt, int src, int flow, int out) {
    const float* srcs[3] = {vel_[src][0].p, vel_[src][1].p, vel_[src][2].p};
    float* outs[3] = {vel_[out][0].p, vel_[out][1].p, vel_[out][2].p};
    ws_.advect_velocity(dt, params.cfl_mc, params.mac_cormack_vel != 0, srcs, vel_[flow][0].p, vel_[flow][1].p,
                        vel_[flow][2].p, outs);
}

void Simulation::validate_step(float dt) const {
    const auto& p = params;
    if (!std::isfinite(p.emitter_kick_multiplier) || p.emitter_kick_multiplier < 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "Invalid emitter kick multiplier");
    // GpuMacSimulation3D::advance validation (GpuMacSimulation3D.cpp:226-233).
    if (!std::isfinite(dt) || dt <= 0.f || !std::isfinite(p.source_strength) || p.source_strength < 0.f ||
        !std::isfinite(p.emitter_radius) || p.emitter_radius <= 0.f || p.emitter_radius > 1.f ||
        !std::isfinite(p.buoyancy) || !std::isfinite(p.smoke_decay) || p.smoke_decay < 0.f ||
        !std::isfinite(p.sor_omega) || p.sor_omega <= 0.f || p.sor_omega >= 2.f || p.project_iterations < 0 ||
        !std::isfinite(p.stir_strength) || !std::isfinite(p.cfl_mc) || p.cfl_mc <= 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "Invalid resident GPU step parameters");
    if (p.use_solve_options && !valid_options(p.solve)) fail(VAPOR_INVALID_ARGUMENT, "Invalid linear solve options");
    if (p.solver_kind != VAPOR_SOLVER_RED_BLACK_SOR && p.solver_kind != VAPOR_SOLVER_MIXED_REFINEMENT &&
        p.solver_kind != VAPOR_SOLVER_FPCG)
        fail(VAPOR_INVALID_ARGUMENT, "Unknown solver kind");
    if (p.emitter_count < 1 || p.emitter_count > 2) fail(VAPOR_INVALID_ARGUMENT, "emitter_count must be 1 or 2");
    if (p.emitter_profile < 0 || p.emitter_profile > 1) fail(VAPOR_INVALID_ARGUMENT, "emitter_profile must be 0 or 1");
    const float scale = ws_.grid().h * ws_.grid().h / (p.reflection ? 0.5f * dt : dt);
    if (!std::isfinite(scale) || scale <= 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "Projection scale is outside the supported float range");
}

// One step of MacGridFluidSolver3D::step / stepNoReflect on the device,
// reading density from dens_[cur_] and writing dens_[1 - cur_].
void Simulation::record_step(float dt) {
    const auto& p = params;
    cudaStream_t s = ws_.stream();
    const Grid g = ws_.grid();
    ws_.timer().begin(VAPOR_PHASE_FORCING);
    emit(dt);
    launch_buoyancy_walls(g, p.buoyancy, dt, p.buoyancy_split, dens_[cur_].p, vel_[S_][0].p, vel_[S_][1].p,
                          vel_[S_][2].p, s);
    ws_.timer().end(VAPOR_PHASE_FORCING, 1);
    if (p.reflection) {
        // MacGridFluidSolver3D::step (MacGridFluidSolver3D.cpp:192-228).
        const float half = 0.5f * dt;
        const auto o = solve_options(std::max(1, p.project_iterations / 2));
        advect_velocity(half, S_, S_, T_);  // T = advected (tilde)
        ws_.project(vel_[T_][0].p, vel_[T_][1].p, vel_[T_][2].p, vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p,
                    vel_[U_][0].p, vel_[U_][1].p, vel_[U_][2].p, half, p.sor_omega, 6.f, o,
                    p.solver_kind, warm_, coarse_);  // S = projected, U = hat
        advect_velocity(half, U_, S_, T_);
        ws_.project(vel_[T_][0].p, vel_[T_][1].p, vel_[T_][2].p, vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p,
                    nullptr, nullptr, nullptr, half, p.sor_omega, 6.f, o, p.solver_kind, warm_, coarse_);
    } else {
        // MacGridFluidSolver3D::stepNoReflect (MacGridFluidSolver3D.cpp:230-245).
        advect_velocity(dt, S_, S_, T_);
        ws_.project(vel_[T_][0].p, vel_[T_][1].p, vel_[T_][2].p, vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p,
                    nullptr, nullptr, nullptr, dt, p.sor_omega, 6.f, solve_options(p.project_iterations),
                    p.solver_kind, warm_, coarse_);
    }
    // Smoke transport through the projected velocity, then dissipation
    // (MacGridFluidSolver3D.cpp:183-190) fused as a post-scale.
    const float factor = std::clamp(1.0f - p.smoke_decay * dt, 0.0f, 1.0f);
    ws_.advect_smoke(dt, p.cfl_mc, p.mac_cormack_smoke != 0, dens_[cur_].p, vel_[S_][0].p, vel_[S_][1].p,
                     vel_[S_][2].p, dens_[1 - cur_].p, factor);
}

void Simulation::set_warm_start(unet::UNet* net) {
    if (net && (ws_.n() % 4 != 0 || ws_.n() < 8))
        fail(VAPOR_INVALID_ARGUMENT, "the warm-start network needs n divisible by 4 (n >= 8)");
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
    release_graphs();
    if (warm_ && warm_ != net) warm_->use_own_stream();
    warm_ = net;
    if (warm_) {
        warm_->set_stream(ws_.stream());
        warm_->prepare(ws_.n());
    }
}

void Simulation::set_preconditioner(unet::UNet* net) {
    if (net && (ws_.n() % 16 != 0 || ws_.n() < 32))
        fail(VAPOR_INVALID_ARGUMENT, "the coarse-grid network needs n divisible by 16 (n >= 32)");
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
    release_graphs();
    if (coarse_ && coarse_ != net) coarse_->use_own_stream();
    coarse_ = net;
    if (coarse_) {
        coarse_->set_stream(ws_.stream());
        coarse_->prepare(ws_.n() / 4);
    }
}

void Simulation::set_solid(const uint8_t* mask) {
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
    release_graphs();
    ws_.set_solid(mask);
}

void Simulation::release_graphs() {
    for (auto& g : graphs_) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.exec = nullptr;
    }
}

void Simulation::prepare_step(float dt) {
    validate_step(dt);
    // Scratch that a captured step needs is allocated before any capture.
    {
        const float centres[2][3] = {{params.emitter_center_x, params.emitter_center_y, params.emitter_center_z},
                                     {params.emitter2_center_x, params.emitter2_center_y, params.emitter2_center_z}};
        size_t need = 0;
        for (int k = 0; k < params.emitter_count; ++k) {
            EmitterBox e;
            if (emitter_box(centres[k][0], centres[k][1], centres[k][2], dt, e))
                need = std::max(need, size_t(e.size[0]) * e.size[1] * e.size[2]);
        }
        if (noise_.n < need) {
            VB_CUDA(cudaStreamSynchronize(ws_.stream()));
            release_graphs();
            noise_.allocate(need);
        }
        if (params.solver_kind != VAPOR_SOLVER_RED_BLACK_SOR) ws_.ensure_mixed();
        if (params.mac_cormack_vel || params.mac_cormack_smoke) ws_.ensure_velocity_scratch();
        if (warm_) {
            warm_->set_stream(ws_.stream());
            warm_->prepare(ws_.n());
        }
        if (params.solver_kind == VAPOR_SOLVER_FPCG) ws_.ensure_fpcg(coarse_ != nullptr);
        if (coarse_) {
            coarse_->set_stream(ws_.stream());
            coarse_->prepare(ws_.n() / 4);
        }
    }
}

void Simulation::record_step_for_batch(float dt) {
    ws_.set_capturing(true);
    try {
        record_step(dt);
    } catch (...) {
        ws_.set_capturing(false);
        throw;
    }
    ws_.set_capturing(false);
}

void Simulation::advance(float dt) {
    prepare_step(dt);
    take_staged_upload();
    cudaStream_t s = ws_.stream();
    if (!use_graphs_ || ws_.timer().enabled()) {
        record_step(dt);
        cur_ = 1 - cur_;
        VB_CUDA(cudaGetLastError());
        return;
    }
    CachedGraph& slot = graphs_[cur_];
    GraphKey key{};
    key.dt = dt;
    key.box = ws_.box();
    key.params = params;
    key.warm = warm_;
    key.warm_buffers = warm_ ? warm_->generation() : 0ull;
    key.coarse = coarse_;
    key.coarse_buffers = coarse_ ? coarse_->generation() : 0ull;
    if (!slot.exec || std::memcmp(&slot.key, &key, sizeof(GraphKey)) != 0) {
        if (slot.exec) {
            cudaGraphExecDestroy(slot.exec);
            slot.exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        VB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        ws_.set_capturing(true);
        try {
            record_step(dt);
        } catch (...) {
            ws_.set_capturing(false);
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            throw;
        }
        ws_.set_capturing(false);
        VB_CUDA(cudaStreamEndCapture(s, &graph));
        const cudaError_t e = cudaGraphInstantiate(&slot.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            slot.exec = nullptr;
            (void)cudaGetLastError();  // do not leave the failure as the runtime's last error
            VB_CUDA(e);
        }
        slot.key = key;
    }
    VB_CUDA(cudaGraphLaunch(slot.exec, s));
    cur_ = 1 - cur_;
}

// ---- Batch: many scenes' steps in one CUDA graph -------------------------

Batch::Batch(std::vector<Simulation*> sims) : sims_(std::move(sims)) {
    if (sims_.empty()) fail(VAPOR_INVALID_ARGUMENT, "a batch needs at least one simulation");
    for (size_t i = 0; i < sims_.size(); ++i) {
        if (!sims_[i]) fail(VAPOR_INVALID_ARGUMENT, "null simulation in batch");
        for (size_t j = 0; j < i; ++j)
            if (sims_[j] == sims_[i]) fail(VAPOR_INVALID_ARGUMENT, "a simulation appears twice in the batch");
    }
    events_.resize(sims_.size() + 1, nullptr);
    for (auto& e : events_) VB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

Batch::~Batch() {
    if (stream_.s) cudaStreamSynchronize(stream_.s);
    for (auto& g : graphs_)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    for (auto& e : events_)
        if (e) cudaEventDestroy(e);
}

// Orders stream `after` behind everything enqueued so far on `before`.
void Batch::order(cudaStream_t before, cudaStream_t after, cudaEvent_t e) {
    VB_CUDA(cudaEventRecord(e, before));
    VB_CUDA(cudaStreamWaitEvent(after, e, 0));
}

void Batch::advance(float dt) {
    for (Simulation* sim : sims_) sim->prepare_step(dt);
    // Key: dt, and for every scene its step parity and graph key.
    std::vector<uint8_t> key(sizeof(float));
    std::memcpy(key.data(), &dt, sizeof(float));
    for (Simulation* sim : sims_) {
        const std::vector<uint8_t> k = sim->step_key(dt);
        key.insert(key.end(), k.begin(), k.end());
    }
    Slot* slot = nullptr;
    for (auto& g : graphs_)
        if (g.exec && g.key == key) slot = &g;
    cudaStream_t s = stream_.s;
    // the batch launch waits for each scene's earlier work (uploads, resets)
    for (size_t i = 0; i < sims_.size(); ++i) order(sims_[i]->stream(), s, events_[i]);
    if (!slot) {
        slot = &graphs_[next_];
        next_ = 1 - next_;
        if (slot->exec) {
            cudaGraphExecDestroy(slot->exec);
            slot->exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        VB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        try {
            // fork: every scene's stream joins the capture, records its step
            // as a parallel branch, and joins back
            VB_CUDA(cudaEventRecord(events_.back(), s));
            for (Simulation* sim : sims_) VB_CUDA(cudaStreamWaitEvent(sim->stream(), events_.back(), 0));
            for (Simulation* sim : sims_) sim->record_step_for_batch(dt);
            for (size_t i = 0; i < sims_.size(); ++i) order(sims_[i]->stream(), s, events_[i]);
        } catch (...) {
            cudaStreamEndCapture(s, &graph);
            if (graph) cudaGraphDestroy(graph);
            (void)cudaGetLastError();
            throw;
        }
        VB_CUDA(cudaStreamEndCapture(s, &graph));
        const cudaError_t e = cudaGraphInstantiate(&slot->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            slot->exec = nullptr;
            (void)cudaGetLastError();
            VB_CUDA(e);
        }
        slot->key = key;
    }
    VB_CUDA(cudaGraphLaunch(slot->exec, s));
    for (size_t i = 0; i < sims_.size(); ++i) {
        sims_[i]->flip_after_batch();
        order(s, sims_[i]->stream(), events_[i]);  // later per-scene work follows the batch
    }
}

void Batch::synchronize() { VB_CUDA(cudaStreamSynchronize(stream_.s)); }

std::vector<uint8_t> Simulation::step_key(float dt) const {
    GraphKey key{};
    key.dt = dt;
    key.box = ws_.box();
    key.params = params;
    key.warm = warm_;
    key.warm_buffers = warm_ ? warm_->generation() : 0ull;
    key.coarse = coarse_;
    key.coarse_buffers = coarse_ ? coarse_->generation() : 0ull;
    std::vector<uint8_t> out(sizeof(GraphKey) + sizeof(int));
    std::memcpy(out.data(), &key, sizeof(GraphKey));
    std::memcpy(out.data() + sizeof(GraphKey), &cur_, sizeof(int));
    return out;
}

void Simulation::upload(const float* d, const float* u, const float* v, const float* w) {
    // a synchronous upload replaces a staged one that no step took in yet
    VB_CUDA(cudaStreamSynchronize(h2d_.s));
    pending_in_ = false;
    cudaStream_t s = ws_.stream();
    const size_t cells = dens_[0].n, faces = vel_[0][0].n;
    VB_CUDA(cudaMemcpyAsync(dens_[cur_].p, d, cells * sizeof(float), cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaMemcpyAsync(vel_[S_][0].p, u, faces * sizeof(float), cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaMemcpyAsync(vel_[S_][1].p, v, faces * sizeof(float), cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaMemcpyAsync(vel_[S_][2].p, w, faces * sizeof(float), cudaMemcpyHostToDevice, s));
    VB_CUDA(cudaStreamSynchronize(s));
    uploaded += (cells + 3 * faces) * sizeof(float);
}

void Simulation::download(float* d, float* u, float* v, float* w) {
    cudaStream_t s = ws_.stream();
    const size_t cells = dens_[0].n, faces = vel_[0][0].n;
    VB_CUDA(cudaMemcpyAsync(d, dens_[cur_].p, cells * sizeof(float), cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaMemcpyAsync(u, vel_[S_][0].p, faces * sizeof(float), cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaMemcpyAsync(v, vel_[S_][1].p, faces * sizeof(float), cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaMemcpyAsync(w, vel_[S_][2].p, faces * sizeof(float), cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaStreamSynchronize(s));
    downloaded += (cells + 3 * faces) * sizeof(float);
}

namespace {
void ensure_event(cudaEvent_t& e) {
    if (!e) VB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}
void ensure_stage(DevArray<float>* stage, size_t cells, size_t faces) {
    if (stage[0].n != cells) stage[0].allocate(cells);
    for (int c = 1; c < 4; ++c)
        if (stage[c].n != faces) stage[c].allocate(faces);
}
}  // namespace

void Simulation::upload_async(const float* d, const float* u, const float* v, const float* w) {
    const size_t cells = dens_[0].n, faces = vel_[0][0].n;
    ensure_stage(in_stage_, cells, faces);
    for (cudaEvent_t* e : {&in_ready_, &in_taken_}) ensure_event(*e);
    // the staging copy is reused once the previous staged upload was taken in
    if (in_taken_recorded_) VB_CUDA(cudaStreamWaitEvent(h2d_.s, in_taken_, 0));
    const float* src[4] = {d, u, v, w};
    for (int c = 0; c < 4; ++c)
        VB_CUDA(cudaMemcpyAsync(in_stage_[c].p, src[c], in_stage_[c].bytes(), cudaMemcpyHostToDevice, h2d_.s));
    VB_CUDA(cudaEventRecord(in_ready_, h2d_.s));
    pending_in_ = true;
    uploaded += (cells + 3 * faces) * sizeof(float);
}

// At the start of a step: the staged snapshot becomes the state.
void Simulation::take_staged_upload() {
    if (!pending_in_) return;
    cudaStream_t s = ws_.stream();
    VB_CUDA(cudaStreamWaitEvent(s, in_ready_, 0));
    float* dst[4] = {dens_[cur_].p, vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p};
    for (int c = 0; c < 4; ++c)
        VB_CUDA(cudaMemcpyAsync(dst[c], in_stage_[c].p, in_stage_[c].bytes(), cudaMemcpyDeviceToDevice, s));
    VB_CUDA(cudaEventRecord(in_taken_, s));
    in_taken_recorded_ = true;
    pending_in_ = false;
}

void Simulation::download_async(float* d, float* u, float* v, float* w) {
    const size_t cells = dens_[0].n, faces = vel_[0][0].n;
    ensure_stage(out_stage_, cells, faces);
    for (cudaEvent_t* e : {&out_ready_, &out_done_}) ensure_event(*e);
    cudaStream_t s = ws_.stream();
    // the snapshot is rewritten once the previous one reached the host
    if (out_done_recorded_) VB_CUDA(cudaStreamWaitEvent(s, out_done_, 0));
    const float* src[4] = {dens_[cur_].p, vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p};
    for (int c = 0; c < 4; ++c)
        VB_CUDA(cudaMemcpyAsync(out_stage_[c].p, src[c], out_stage_[c].bytes(), cudaMemcpyDeviceToDevice, s));
    VB_CUDA(cudaEventRecord(out_ready_, s));
    VB_CUDA(cudaStreamWaitEvent(d2h_.s, out_ready_, 0));
    float* dst[4] = {d, u, v, w};
    for (int c = 0; c < 4; ++c)
        VB_CUDA(cudaMemcpyAsync(dst[c], out_stage_[c].p, out_stage_[c].bytes(), cudaMemcpyDeviceToHost, d2h_.s));
    VB_CUDA(cudaEventRecord(out_done_, d2h_.s));
    out_done_recorded_ = true;
    downloaded += (cells + 3 * faces) * sizeof(float);
}

void Simulation::wait_transfers() {
    VB_CUDA(cudaStreamSynchronize(h2d_.s));
    VB_CUDA(cudaStreamSynchronize(d2h_.s));
}

void Simulation::synchronize() { (void)last_projection(); }

vapor_projection_result Simulation::last_projection() {
    const vapor_projection_result r = ws_.last_result();
    // a network that ran inside the step reports its bounded waits here
    if (warm_) warm_->check_error();
    if (coarse_) coarse_->check_error();
    return r;
}

void Simulation::diagnostics(vapor_fluid_diagnostics* out) {
    ws_.diagnostics(vel_[S_][0].p, vel_[S_][1].p, vel_[S_][2].p, out);
}

void Simulation::render(const vapor_render_params& p, float* rgb_host) {
    const size_t count = size_t(3) * p.width * p.height;
    DevArray<float> rgb;
    rgb.allocate(count);
    render_volume(dens_[cur_].p, ws_.n(), ws_.box(), p, rgb.p, ws_.stream());
    VB_CUDA(cudaMemcpyAsync(rgb_host, rgb.p, count * sizeof(float), cudaMemcpyDeviceToHost, ws_.stream()));
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
}

void Simulation::comparison_metrics(float frames_per_second, vapor_comparison_metrics* out) {
    vb::comparison_metrics(ws_.grid(), frames_per_second, params.cfl_mc, dens_[cur_].p, vel_[S_][0].p,
                           vel_[S_][1].p, vel_[S_][2].p, out, ws_.stream());
}

// ---------------------------------------------------------------------------
// Staged stages
// ---------------------------------------------------------------------------
Stage::Stage(int n, float box) : ws_(n, box, stream_.s) {
    const size_t faces = size_t(n) * n * (n + 1);
    for (auto& a : in_) a.allocate(faces);
    for (auto& a : out_) a.allocate(faces);
    src_.allocate(faces);
    dst_.allocate(faces);
}

Stage::~Stage() { cudaStreamSynchronize(ws_.stream()); }

void Stage::reset() {
    ws_.reset_buffers();
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
}

static bool overlaps(const float* a, size_t na, const float* b, size_t nb) {
    if (!a || !b || na == 0 || nb == 0) return false;
    const uintptr_t a0 = uintptr_t(a), a1 = uintptr_t(a + na), b0 = uintptr_t(b), b1 = uintptr_t(b + nb);
    return a0 < b1 && b0 < a1;
}

// Projection3D::project contract (CpuPressureSolver3D.cpp:25-33, SOR.cpp:15-27).
void Stage::solve_rhs(const float* rhs_device, const vapor_projection_options& o, float floor_diag,
                      vapor_projection_result* result, float* pressure_device) {
    if (!rhs_device) fail(VAPOR_INVALID_ARGUMENT, "a right-hand side is required");
    if (!std::isfinite(o.relaxation) || o.relaxation <= 0.f || o.relaxation >= 2.f)
        fail(VAPOR_INVALID_ARGUMENT, "SOR relaxation factor must be between 0 and 2");
    if (!valid_options(o.linear_solve)) fail(VAPOR_INVALID_ARGUMENT, "Invalid linear solve options");
    ws_.clear_errors();
    ws_.ensure_mixed();
    ws_.project(nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 1.f, o.relaxation,
                floor_diag, o.linear_solve, VAPOR_SOLVER_MIXED_REFINEMENT, nullptr, nullptr, rhs_device);
    const vapor_projection_result r = ws_.last_result();
    if (pressure_device) {
        launch_unsplit_pressure(ws_.grid(), ws_.pressure(), ws_.control(), pressure_device, ws_.stream());
        VB_CUDA(cudaGetLastError());
    }
    VB_CUDA(cudaStreamSynchronize(ws_.stream()));
    if (result) *result = r;
}

void Stage::project(float* u, float* v, float* w, const vapor_projection_options& o, float floor_diag,
                    vapor_projection_result* result, float* pressure_out, bool device_pointers) {
    const Grid g = ws_.grid();
    if (!u || !v || !w) fail(VAPOR_INVALID_ARGUMENT, "Velocity fields are required");
    if (!std::isfinite(o.relaxation) || o.relaxation <= 0.f || o.relaxation >= 2.f)
        fail(VAPOR_INVALID_ARGUMENT, "SOR relaxation factor must be between 0 and 2");
    if (!std::isfinite(floor_diag) || floor_diag < 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "SOR diagonal floor must be finite and nonnegative");
    if (!std::isfinite(o.dt) || o.dt <= 0.f) fail(VAPOR_INVALID_ARGUMENT, "Projection time step must be finite and positive");
    const float scale = g.h * g.h / o.dt;
    if (!std::isfinite(scale) || scale <= 0.f)
        fail(VAPOR_INVALID_ARGUMENT, "Projection scale is outside the supported float range");
    if (!valid_options(o.linear_solve)) fail(VAPOR_INVALID_ARGUMENT, "Invalid linear solve options");
    cudaStream_t s = ws_.stream();
    const size_t faces = in_[0].n, bytes = faces * sizeof(float);
    float* user[3] = {u, v, w};
    const cudaMemcpyKind in_kind = device_pointers ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = device_pointers ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (int c = 0; c < 3; ++c) VB_CUDA(cudaMemcpyAsync(in_[c].p, user[c], bytes, in_kind, s));
    ws_.clear_errors();
    if (solver_kind != VAPOR_SOLVER_RED_BLACK_SOR && solver_kind != VAPOR_SOLVER_MIXED_REFINEMENT &&
        solver_kind != VAPOR_SOLVER_FPCG)
        fail(VAPOR_INVALID_ARGUMENT, "Unknown solver kind");
    unet::UNet* net = solver_kind == VAPOR_SOLVER_FPCG ? coarse : nullptr;
    if (net) {
        if (g.n % 16 != 0 || g.n < 32)
            fail(VAPOR_INVALID_ARGUMENT, "the coarse-grid network needs n divisible by 16 (n >= 32)");
        net->set_stream(s);
    }
    try {
        ws_.project(in_[0].p, in_[1].p, in_[2].p, out_[0].p, out_[1].p, out_[2].p, nullptr, nullptr, nullptr, o.dt,
                    o.relaxation, floor_diag, o.linear_solve, solver_kind, nullptr, net);
    } catch (...) {
        if (net) net->use_own_stream();
        throw;
    }
    const vapor_projection_result r = ws_.last_result();  // waits; raises on non-finite input
    for (int c = 0; c < 3; ++c) VB_CUDA(cudaMemcpyAsync(user[c], out_[c].p, bytes, out_kind, s));
    if (pressure_out) {
        // Zero-mean pressure in natural order (the reference subtracts the
        // mean in place; the same FP32 subtraction happens on the device).
        const size_t cells = size_t(g.n) * g.n * g.n;
        float* natural = device_pointers ? pressure_out : dst_.p;
        launch_unsplit_pressure(g, ws_.pressure(), ws_.control(), natural, s);
        VB_CUDA(cudaGetLastError());
        if (!device_pointers)
            VB_CUDA(cudaMemcpyAsync(pressure_out, natural, cells * sizeof(float), cudaMemcpyDeviceToHost, s));
    }
    VB_CUDA(cudaStreamSynchronize(s));
    if (net) net->use_own_stream();
    if (result) *result = r;
}

// Advection3D contract (AdvectionContext.cpp:15-67).
void Stage::advect(int loc, float dt, float cfl, int method, const float* src, const float* fu, const float* fv,
                   const float* fw, float* out, bool device_pointers) {
    const Grid g = ws_.grid();
    if (!std::isfinite(dt) || dt < 0.f || !std::isfinite(cfl) || cfl <= 0.f || !fu || !fv || !fw)
        fail(VAPOR_INVALID_ARGUMENT, "Invalid advection time step, CFL limit, or tracer field sizes");
    if (loc < CELL || loc > FACE_Z) fail(VAPOR_INVALID_ARGUMENT, "Invalid staggered field axis");
    if (method != VAPOR_SEMI_LAGRANGIAN && method != VAPOR_MACCORMACK)
        fail(VAPOR_INVALID_ARGUMENT, "Invalid advection method");
    const size_t faces = size_t(g.n) * g.n * (g.n + 1);
    const size_t count = count_of(g.n, loc);
    if (!src || !out) fail(VAPOR_INVALID_ARGUMENT, "Velocity fields must match their grid layout and not overlap");
    if (loc != CELL && overlaps(src, count, out, count))
        fail(VAPOR_INVALID_ARGUMENT, "Velocity fields must match their grid layout and not overlap");
    if (overlaps(out, count, fu, faces) || overlaps(out, count, fv, faces) || overlaps(out, count, fw, faces))
        fail(VAPOR_INVALID_ARGUMENT, "Advection output must not alias tracer velocities");
    cudaStream_t s = ws_.stream();
    const float* flow[3] = {fu, fv, fw};
    const float* dsrc = src;
    const float* dflow[3] = {fu, fv, fw};
    float* dout = out;
    if (!device_pointers) {
        for (int c = 0; c < 3; ++c) {
            VB_CUDA(cudaMemcpyAsync(in_[c].p, flow[c], faces * sizeof(float), cudaMemcpyHostToDevice, s));
            dflow[c] = in_[c].p;
        }
        VB_CUDA(cudaMemcpyAsync(src_.p, src, count * sizeof(float), cudaMemcpyHostToDevice, s));
        dsrc = src_.p;
        dout = dst_.p;
    } else if (loc == CELL && src == out) {
        // In-place scalar transport on device memory: stage through src_.
        VB_CUDA(cudaMemcpyAsync(src_.p, src, count * sizeof(float), cudaMemcpyDeviceToDevice, s));
        dsrc = src_.p;
    }
    ws_.advect(loc, dt, cfl, method == VAPOR_MACCORMACK, dsrc, dflow[0], dflow[1], dflow[2], dout, 1.f);
    if (!device_pointers) VB_CUDA(cudaMemcpyAsync(out, dst_.p, count * sizeof(float), cudaMemcpyDeviceToHost, s));
    VB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace vb
