// Host-side engine of the B200 MAC 3D step: device buffers, the projection
// orchestration, the resident coordinator (GpuMacSimulation3D's role) and the
// staged stage plugins (GpuPressureSolver / GpuAdvection's role).
#pragma once

#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.hpp"

namespace vb {
namespace unet {
class UNet;
}

// Error carried to the C ABI, where it becomes a vapor_status.
struct Error : std::runtime_error {
    vapor_status code;
    Error(vapor_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void fail(vapor_status code, const std::string& message);
// Runs f, turning exceptions into a vapor_status and the per-thread message
// returned by vapor_last_error (the C ABI's guard, capi.cu).
vapor_status guard(const std::function<void()>& f);
void cuda_check(cudaError_t e, const char* what);
#define VB_CUDA(call) ::vb::cuda_check((call), #call)

// Owning device allocation.
template <class T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    void allocate(size_t count);
    void release();
    void zero(cudaStream_t s);
    size_t bytes() const { return n * sizeof(T); }
};

// Owning non-blocking CUDA stream.
struct Stream {
    cudaStream_t s = nullptr;
    Stream();
    ~Stream();
    Stream(const Stream&) = delete;
    Stream& operator=(const Stream&) = delete;
};

// Opt-in CUDA-event timing of step phases on one stream.
class PhaseTimer {
public:
    explicit PhaseTimer(cudaStream_t s) : s_(s) {}
    ~PhaseTimer();
    PhaseTimer(const PhaseTimer&) = delete;
    PhaseTimer& operator=(const PhaseTimer&) = delete;
    void enable(bool on);
    bool enabled() const { return on_; }
    void begin(int phase);
    void end(int phase, long long launches);
    void fold(bool wait);  // accumulate finished intervals
    vapor_phase_timings totals();

private:
    cudaEvent_t take();
    struct Pending {
        int phase;
        cudaEvent_t a, b;
        long long launches;
    };
    cudaStream_t s_;
    bool on_ = false;
    std::vector<cudaEvent_t> pool_;
    std::vector<Pending> pending_;
    cudaEvent_t open_[VAPOR_PHASE_COUNT] = {};
    vapor_phase_timings acc_{};
};

// Red-black relaxation sweeps before (and, in reverse colour order, after)
// the coarse correction in the FPCG preconditioner, and their weight
// (1: Gauss-Seidel). Process-wide; read when a projection is recorded.
struct FpcgSmoothing {
    int sweeps;
    float omega;
};
FpcgSmoothing fpcg_smoothing();
void set_fpcg_smoothing(int sweeps, float omega);

// Validation shared by every entry point (MacGridDomain3D.cpp:7-22).
void validate_grid(int n, float box);

// Projection workspace: b, x, MacCormack scratch, reduction partials and the
// device control block. One per concurrent operation.
class Workspace {
public:
    Workspace(int n, float box, cudaStream_t stream);
    ~Workspace();
    Workspace(const Workspace&) = delete;
    Workspace& operator=(const Workspace&) = delete;

    Grid grid() const { return Grid{n_, box_, box_ / float(n_)}; }
    int n() const { return n_; }
    float box() const { return box_; }
    void set_box(float box) { box_ = box; }
    cudaStream_t stream() const { return stream_; }

    // Projects (ui,vi,wi) into (uo,vo,wo) (+ hat = 2 out - in when given).
    // Fixed-iteration solves never wait for the device; tolerance-driven
    // solves read the stop flag after each residual check.
    void project(const float* ui, const float* vi, const float* wi, float* uo, float* vo, float* wo, float* uh,
                 float* vh, float* wh, float dt, float omega, float diagonal_floor,
                 const vapor_linear_solve_options& options, int solver_kind = VAPOR_SOLVER_RED_BLACK_SOR,
                 unet::UNet* warm_start = nullptr, unet::UNet* coarse = nullptr,
                 const float* rhs_field = nullptr);
    // Logs every FPCG coarse right-hand side into a device ring (training data
    // for the coarse network); null disables. See launch_log_coarse.
    void set_coarse_log(float* log, int capacity, int* counter) {
        coarse_log_ = log;
        coarse_log_capacity_ = capacity;
        coarse_log_counter_ = counter;
    }
    float* rhs() { return b_.p; }
    void advect(int loc, float dt, float cfl, bool maccormack, const float* src, const float* u, const float* v,
                const float* w, float* out, float post_scale);
    // The three velocity components in one forward and one MacCormack launch
    // (their forward passes kept in a 3-face-array scratch).
    void advect_velocity(float dt, float cfl, bool maccormack, const float* const src[3], const float* u,
                         const float* v, const float* w, float* const out[3]);
    // The smoke through the flow, its forward pass's traced velocities cached
    // for the MacCormack pass when the velocity scratch exists.
    void advect_smoke(float dt, float cfl, bool maccormack, const float* src, const float* u, const float* v,
                      const float* w, float* out, float post_scale);
    // Waits for the stream and returns the last projection result; raises
    // VAPOR_NON_FINITE if a non-finite divergence or residual was seen since
    // the last clear_errors().
    vapor_projection_result last_result();
    void clear_errors();
    void reset_buffers();
    float* pressure() { return p_.p; }
    ProjControl* control() { return ctrl_; }
    const ProjControl* host_control() const { return ctrl_host_; }
    void diagnostics(const float* u, const float* v, const float* w, vapor_fluid_diagnostics* out);
    long long total_iterations();
    PhaseTimer& timer() { return timer_; }
    void ensure_mixed();
    void ensure_fpcg(bool coarse);
    void ensure_velocity_scratch();
    // Solid obstacles (extension): n^3 host mask, x fastest, nonzero = solid;
    // null clears. Faces touching a solid are closed, solid cells are not
    // unknowns, means run over fluid cells. Mixed-precision solver only.
    void set_solid(const uint8_t* mask);
    bool has_solid() const { return fluid_ > 0.0; }
    // While true, project() records CUDA-graph nodes (the solve loops become
    // conditional while nodes) instead of driving the loop from the host.
    void set_capturing(bool on) { capturing_ = on; }

private:
    void project_fpcg(const ProjectionArgs& a, unet::UNet* warm, unet::UNet* coarse, LoopCond cond,
                      cudaGraphConditionalHandle handle);

    int n_;
    float box_;
    cudaStream_t stream_;
    DevArray<float> b_, p_, fwd_;
    DevArray<float> fwd3_;  // forward passes of the three velocity components (allocated before capture)
    DevArray<float> vel_cache_;  // traced velocities of the forward passes (9 face arrays)
    DevArray<double> partials_;
    DevArray<double> x64_[2];           // mixed-precision pressure (ping-pong)
    DevArray<float> r32_;               // mixed-precision inner right-hand side (FPCG: the residual)
    DevArray<float> cg_p_, cg_q_, cg_z_;  // FPCG direction, A p, preconditioned residual
    DevArray<float> cg_p2_;             // second direction buffer of the fused step (n % 8 == 0)
    DevArray<float> x_alt_;             // twin of the iterate for out-of-place blocked sweeps
    DevArray<float> cg_rc_;             // FPCG coarse right-hand side ((n/4)^3, natural layout)
    DevArray<float> cg_rows_;           // FPCG restriction scratch (n^2 * n/4 row sums)
    DevArray<double> cg_partials_;
    DevArray<uint8_t> solid_;           // natural-layout solid mask (obstacles)
    DevArray<uint8_t> solid_diag_;      // split-layout fluid-neighbour counts, 0 = solid
    double fluid_ = 0.0;                // fluid cells when a mask is set, else 0
    float* coarse_log_ = nullptr;       // FPCG coarse right-hand-side ring (device), optional
    int coarse_log_capacity_ = 0;
    int* coarse_log_counter_ = nullptr;
    CgControl* cg_ = nullptr;           // device
    int partial_capacity_ = 0;
    ProjControl* ctrl_ = nullptr;       // device
    ProjControl* ctrl_host_ = nullptr;  // pinned mirror
    DiagControl* diag_ = nullptr;
    DiagControl* diag_host_ = nullptr;
    int* done_host_ = nullptr;          // pinned
    PhaseTimer timer_;
    Stream body_stream_;                // records conditional-loop bodies
    Stream body_stream2_;               // records conditional bodies nested in a loop
    bool capturing_ = false;
    long long total_iterations_ = 0;
    unsigned int sticky_errors_ = 0u;
    friend class Simulation;
};

// Resident coordinator: all fields on the device across steps.
class Simulation {
public:
    Simulation(int n, float box, const vapor_mac3d_params& params);
    ~Simulation();
    void release_graphs();
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;

    void reset();
    void set_box(float box);
    void advance(float dt);
    // Batched stepping (Batch): validation and scratch allocation before a
    // capture, the step recorded into the current capture, the step's cache
    // key, and the parity flip once a batch graph holding the step launched.
    void prepare_step(float dt);
    void record_step_for_batch(float dt);
    std::vector<uint8_t> step_key(float dt) const;
    void flip_after_batch() { cur_ = 1 - cur_; }
    void set_coarse_log(float* log, int capacity, int* counter) {
        VB_CUDA(cudaStreamSynchronize(ws_.stream()));
        release_graphs();
        ws_.set_coarse_log(log, capacity, counter);
    }
    void upload(const float* d, const float* u, const float* v, const float* w);
    void download(float* d, float* u, float* v, float* w);
    // Streamed host transfers. upload_async copies a host snapshot into a
    // device staging copy on its own stream and returns; the next advance
    // takes it in (one device-to-device copy at the start of the step).
    // download_async snapshots the fields on the step's stream and copies
    // the snapshot to the host on another stream. Both overlap the
    // neighbouring steps' compute; wait_transfers blocks until every staged
    // copy has finished (host buffers stay untouched and valid until then).
    void upload_async(const float* d, const float* u, const float* v, const float* w);
    void download_async(float* d, float* u, float* v, float* w);
    void wait_transfers();
    void synchronize();
    vapor_projection_result last_projection();
    void diagnostics(vapor_fluid_diagnostics* out);
    // The harness comparison metrics of the current state (waits).
    void comparison_metrics(float frames_per_second, vapor_comparison_metrics* out);
    // Ray-marched image of the current density into host memory (waits).
    void render(const vapor_render_params& p, float* rgb_host);
    long long total_iterations() { return ws_.total_iterations(); }
    PhaseTimer& timer() { return ws_.timer(); }

    vapor_mac3d_params params;
    uint64_t uploaded = 0, downloaded = 0;
    int n() const { return ws_.n(); }
    float box() const { return ws_.box(); }
    cudaStream_t stream() const { return ws_.stream(); }
    float* density() { return dens_[cur_].p; }
    float* velocity(int c) { return vel_[S_][c].p; }

    // CUDA-graph replay of whole steps (default on; phase timing uses the
    // eager path).
    void set_graphs(bool on) { use_graphs_ = on; }
    // Learned warm start for every projection (null: start from zero, the
    // reference's x = 0). The network is bound to this simulation's stream.
    void set_warm_start(unet::UNet* net);
    unet::UNet* warm_start() const { return warm_; }
    // Learned coarse-grid correction of the FPCG solver (VAPOR_SOLVER_FPCG;
    // null: smoothing-only preconditioner). Needs n divisible by 16.
    void set_preconditioner(unet::UNet* net);
    // Obstacle mask (n^3, x fastest, nonzero = solid; null clears) for every
    // later projection of this simulation; needs the mixed-precision or the
    // FPCG solver.
    void set_solid(const uint8_t* mask);
    unet::UNet* preconditioner() const { return coarse_; }
    Workspace& workspace() { return ws_; }

private:
    bool emitter_box(float cx, float cy, float cz, float dt, EmitterBox& e) const;
    void emit(float dt);
    void advect_velocity(float dt, int src_set, int flow_set, int out_set);
    void record_step(float dt);
    void validate_step(float dt) const;
    vapor_linear_solve_options solve_options(int iterations) const;

    struct GraphKey {
        float dt;
        float box;
        vapor_mac3d_params params;
        const void* warm;                 // warm-start network, if any
        unsigned long long warm_buffers;  // its buffer generation (reallocation re-records)
        const void* coarse;               // coarse-grid network of the FPCG solver, if any
        unsigned long long coarse_buffers;
    };
    struct CachedGraph {
        GraphKey key{};
        cudaGraphExec_t exec = nullptr;
    };
    CachedGraph graphs_[2];
    bool use_graphs_ = true;
    unet::UNet* warm_ = nullptr;
    unet::UNet* coarse_ = nullptr;

    // streamed transfers
    void take_staged_upload();
    Stream h2d_, d2h_;
    DevArray<float> in_stage_[4], out_stage_[4];
    cudaEvent_t in_ready_ = nullptr, in_taken_ = nullptr, out_ready_ = nullptr, out_done_ = nullptr;
    bool pending_in_ = false, in_taken_recorded_ = false, out_done_recorded_ = false;

    Stream stream_;
    Workspace ws_;
    DevArray<float> dens_[2];
    DevArray<float> vel_[3][3];
    DevArray<uint32_t> rng_;
    DevArray<float> noise_;
    int cur_ = 0;
    int S_ = 0, T_ = 1, U_ = 2;
};

// Staged stage plugins on caller-owned spans (host or device).
// Many scenes stepped by one CUDA-graph launch: each scene's whole step
// (solve loops included) is a parallel branch of one graph, recorded from
// the scenes' own streams, so independent grids of uneven sizes fill the GPU
// together. Graphs are cached per dt, scene parameters and parities. The
// batch does not own the simulations; destroy it first.
class Batch {
public:
    explicit Batch(std::vector<Simulation*> sims);
    ~Batch();
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    void advance(float dt);
    void synchronize();
    cudaStream_t stream() const { return stream_.s; }
    size_t size() const { return sims_.size(); }

private:
    static void order(cudaStream_t before, cudaStream_t after, cudaEvent_t e);
    struct Slot {
        std::vector<uint8_t> key;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<Simulation*> sims_;
    Stream stream_;
    std::vector<cudaEvent_t> events_;
    Slot graphs_[2];
    int next_ = 0;
};

class Stage {
public:
    Stage(int n, float box);
    ~Stage();
    Stage(const Stage&) = delete;
    Stage& operator=(const Stage&) = delete;

    void reset();
    int solver_kind = VAPOR_SOLVER_RED_BLACK_SOR;
    unet::UNet* coarse = nullptr;
    void set_solid(const uint8_t* mask) { ws_.set_solid(mask); }
    // Mixed-precision solve of A x = rhs for a given right-hand side (device,
    // natural layout, n^3); the pressure (zero mean) into pressure_device if
    // given. The workspace keeps (b, x) for network training.
    void solve_rhs(const float* rhs_device, const vapor_projection_options& o, float floor_diag,
                   vapor_projection_result* result, float* pressure_device);  // FPCG coarse-grid network (bound to this stage's stream per call)
    void project(float* u, float* v, float* w, const vapor_projection_options& options, float diagonal_floor,
                 vapor_projection_result* result, float* pressure_out, bool device_pointers);
    void advect(int loc, float dt, float cfl, int method, const float* src, const float* fu, const float* fv,
                const float* fw, float* out, bool device_pointers);
    cudaStream_t stream() const { return ws_.stream(); }
    int n() const { return ws_.n(); }
    Workspace& workspace() { return ws_; }

private:
    Stream stream_;
    Workspace ws_;
    DevArray<float> in_[3], out_[3], src_, dst_;
};

}  // namespace vb
