// extern "C" boundary of include/vapor_b200.h. Every entry point catches all
// C++ exceptions and turns them into a vapor_status plus a per-thread message.
#include <cmath>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "engine.hpp"
#include "unet.hpp"

struct vapor_mac3d {
    vb::Simulation sim;
    vapor_mac3d(int n, float box, const vapor_mac3d_params& p) : sim(n, box, p) {}
};
struct vapor_stage {
    vb::Stage stage;
    vapor_stage(int n, float box) : stage(n, box) {}
};
struct vapor_batch {
    vb::Batch batch;
    explicit vapor_batch(std::vector<vb::Simulation*> sims) : batch(std::move(sims)) {}
};
struct vapor_unet {
    vb::Stream stream;
    vb::unet::UNet net;
    vapor_unet() : net(stream.s) {}
};

namespace {
thread_local std::string g_last_error;

template <class F>
vapor_status guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return VAPOR_OK;
    } catch (const vb::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return VAPOR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return VAPOR_RUNTIME_ERROR;
    } catch (...) {
        g_last_error = "unknown error";
        return VAPOR_RUNTIME_ERROR;
    }
}

void require(bool ok, const char* message) {
    if (!ok) vb::fail(VAPOR_INVALID_ARGUMENT, message);
}

// The library targets sm_100a only; refuse other devices up front.
void require_device() {
    int dev = 0;
    VB_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    VB_CUDA(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) vb::fail(VAPOR_RUNTIME_ERROR, "vapor_b200 requires an sm_100 (B200) device");
}
}  // namespace

namespace vb {
vapor_status guard(const std::function<void()>& f) { return guarded(f); }
}  // namespace vb

#define VB_API extern "C" __attribute__((visibility("default")))

VB_API const char* vapor_last_error(void) { return g_last_error.c_str(); }
VB_API int32_t vapor_abi_version(void) { return VAPOR_B200_ABI_VERSION; }
VB_API int64_t vapor_kernel_launch_count(void) { return vb::launch_count(); }
VB_API vapor_status vapor_set_device(int32_t device) {
    return guarded([&] {
        int count = 0;
        VB_CUDA(cudaGetDeviceCount(&count));
        require(device >= 0 && device < count, "device index out of range");
        VB_CUDA(cudaSetDevice(device));
    });
}

VB_API vapor_status vapor_mac3d_default_params(vapor_mac3d_params* o) {
    return guarded([&] {
        require(o != nullptr, "null output");
        std::memset(o, 0, sizeof(*o));
        o->emitter_radius = 0.035f;
        o->emitter_center_x = 0.5f;
        o->emitter_center_y = 0.5f;
        o->emitter_center_z = 0.1f;
        o->emitter_kick_multiplier = 1.f;
        o->emitter_kick_base = 0.8f;
        o->emitter_kick_scale = 0.8f;
        o->stir_strength = 0.5f;
        o->random_seed = 0x9E3779B9u;
        o->sor_omega = 1.95f;
        o->buoyancy_split = 0.5f;
        o->cfl_mc = 3.0f;
        o->mac_cormack_smoke = 1;
        o->mac_cormack_vel = 1;
        o->smoke_decay = 0.06f;
        o->reflection = 1;
        o->buoyancy = 2.5f;
        o->source_strength = 1.f;
        o->project_iterations = 64;
        o->use_solve_options = 0;
        o->solve.max_iterations = 200;
        o->solve.residual_check_interval = 8;
        o->solve.absolute_tolerance = 1e-6;
        o->solve.relative_tolerance = 1e-5;
        o->solve.fixed_iterations = 0;
        o->solver_kind = VAPOR_SOLVER_RED_BLACK_SOR;
        o->emitter_profile = 0;
        o->emitter_count = 1;
        o->emitter2_center_x = 0.5f;
        o->emitter2_center_y = 0.5f;
        o->emitter2_center_z = 0.1f;
    });
}

VB_API vapor_status vapor_mac3d_algorithm_params(int32_t algorithm, vapor_mac3d_params* o) {
    return guarded([&] {
        require(algorithm >= 0 && algorithm <= 3, "Unknown MAC algorithm");
        require(o != nullptr, "null output");
        vapor_mac3d_default_params(o);
        o->reflection = algorithm >= 2;
        o->mac_cormack_smoke = algorithm & 1;
        o->mac_cormack_vel = o->mac_cormack_smoke;
        o->emitter_radius = 0.08f;
        o->source_strength = 4.f;
        o->buoyancy = 3.f;
        o->smoke_decay = 0.08f;
        o->project_iterations = 600;
        o->sor_omega = 1.9f;
    });
}

VB_API vapor_status vapor_default_projection_options(vapor_projection_options* o) {
    return guarded([&] {
        require(o != nullptr, "null output");
        o->dt = 1.f / 60.f;
        o->relaxation = 1.95f;
        o->linear_solve.max_iterations = 200;
        o->linear_solve.residual_check_interval = 8;
        o->linear_solve.absolute_tolerance = 1e-6;
        o->linear_solve.relative_tolerance = 1e-5;
        o->linear_solve.fixed_iterations = 0;
        o->linear_solve.reserved0 = 0;
    });
}

// ---- resident coordinator ----
VB_API vapor_status vapor_mac3d_create(int32_t n, float box, const vapor_mac3d_params* params, vapor_mac3d** out) {
    return guarded([&] {
        require(out != nullptr && params != nullptr, "null argument");
        *out = nullptr;
        vb::validate_grid(n, box);
        require_device();
        *out = new vapor_mac3d(n, box, *params);
    });
}

VB_API vapor_status vapor_mac3d_destroy(vapor_mac3d* sim) {
    return guarded([&] { delete sim; });
}

#define SIM_GUARD(body)                                           \
    return guarded([&] {                                          \
        require(sim != nullptr, "null simulation handle");       \
        body;                                                     \
    })

VB_API vapor_status vapor_mac3d_reset(vapor_mac3d* sim) { SIM_GUARD(sim->sim.reset()); }
VB_API vapor_status vapor_mac3d_set_box(vapor_mac3d* sim, float box) { SIM_GUARD(sim->sim.set_box(box)); }
VB_API vapor_status vapor_mac3d_get_params(const vapor_mac3d* sim, vapor_mac3d_params* out) {
    SIM_GUARD(require(out != nullptr, "null output"); *out = sim->sim.params);
}
VB_API vapor_status vapor_mac3d_set_params(vapor_mac3d* sim, const vapor_mac3d_params* params) {
    SIM_GUARD(require(params != nullptr, "null params"); sim->sim.params = *params);
}
VB_API vapor_status vapor_mac3d_advance(vapor_mac3d* sim, float dt) { SIM_GUARD(sim->sim.advance(dt)); }
VB_API vapor_status vapor_mac3d_advance_n(vapor_mac3d* sim, float dt, int32_t steps) {
    SIM_GUARD(require(steps >= 0, "negative step count"); for (int i = 0; i < steps; ++i) sim->sim.advance(dt));
}
VB_API vapor_status vapor_mac3d_synchronize(vapor_mac3d* sim) { SIM_GUARD(sim->sim.synchronize()); }
VB_API vapor_status vapor_mac3d_last_projection(vapor_mac3d* sim, vapor_projection_result* out) {
    SIM_GUARD(require(out != nullptr, "null output"); *out = sim->sim.last_projection());
}
VB_API vapor_status vapor_mac3d_total_iterations(vapor_mac3d* sim, int64_t* out) {
    SIM_GUARD(require(out != nullptr, "null output"); *out = sim->sim.total_iterations());
}
VB_API vapor_status vapor_mac3d_diagnostics(vapor_mac3d* sim, vapor_fluid_diagnostics* out) {
    SIM_GUARD(require(out != nullptr, "null output"); sim->sim.diagnostics(out));
}
VB_API vapor_status vapor_mac3d_comparison_metrics(vapor_mac3d* sim, float frames_per_second,
                                                   vapor_comparison_metrics* out) {
    SIM_GUARD(require(out != nullptr, "null output");
              require(std::isfinite(frames_per_second) && frames_per_second > 0.f, "Invalid frame rate");
              sim->sim.comparison_metrics(frames_per_second, out));
}
static void validate_render(const vapor_render_params* p) {
    require(p != nullptr, "null parameters");
    require(p->width > 0 && p->height > 0 && p->width <= 16384 && p->height <= 16384, "Invalid image size");
    const float v[] = {p->azimuth, p->elevation, p->distance, p->step_scale, p->alpha_mul, p->light[0],
                       p->light[1], p->light[2], p->shadow_strength, p->shadow_step};
    for (float x : v) require(std::isfinite(x), "Non-finite render parameter");
    require(p->step_scale > 0.f && p->distance > 0.f, "Invalid ray step or camera distance");
    require(p->shadow_strength <= 0.f || p->shadow_step > 0.f, "Invalid shadow step");
}
VB_API vapor_status vapor_render_volume(const float* density_device, int32_t n, float box,
                                        const vapor_render_params* params, float* rgb_device, void* stream) {
    return guarded([&] {
        vb::validate_grid(n, box);
        validate_render(params);
        require(density_device && rgb_device, "null buffer");
        vb::render_volume(density_device, n, box, *params, rgb_device, static_cast<cudaStream_t>(stream));
    });
}
VB_API vapor_status vapor_mac3d_render(vapor_mac3d* sim, const vapor_render_params* params, float* rgb_host) {
    SIM_GUARD(validate_render(params); require(rgb_host != nullptr, "null output"); sim->sim.render(*params, rgb_host));
}
VB_API vapor_status vapor_mac3d_upload(vapor_mac3d* sim, const float* d, const float* u, const float* v,
                                       const float* w) {
    SIM_GUARD(require(d && u && v && w, "null field"); sim->sim.upload(d, u, v, w));
}
VB_API vapor_status vapor_mac3d_download(vapor_mac3d* sim, float* d, float* u, float* v, float* w) {
    SIM_GUARD(require(d && u && v && w, "null field"); sim->sim.download(d, u, v, w));
}
VB_API vapor_status vapor_mac3d_upload_async(vapor_mac3d* sim, const float* d, const float* u, const float* v,
                                             const float* w) {
    SIM_GUARD(require(d && u && v && w, "null field"); sim->sim.upload_async(d, u, v, w));
}
VB_API vapor_status vapor_mac3d_download_async(vapor_mac3d* sim, float* d, float* u, float* v, float* w) {
    SIM_GUARD(require(d && u && v && w, "null field"); sim->sim.download_async(d, u, v, w));
}
VB_API vapor_status vapor_mac3d_wait_transfers(vapor_mac3d* sim) { SIM_GUARD(sim->sim.wait_transfers()); }
VB_API vapor_status vapor_mac3d_byte_counters(const vapor_mac3d* sim, uint64_t* up, uint64_t* down) {
    SIM_GUARD(if (up) *up = sim->sim.uploaded; if (down) *down = sim->sim.downloaded);
}
VB_API vapor_status vapor_mac3d_device_fields(vapor_mac3d* sim, float** d, float** u, float** v, float** w) {
    SIM_GUARD(if (d) *d = sim->sim.density(); if (u) *u = sim->sim.velocity(0); if (v) *v = sim->sim.velocity(1);
              if (w) *w = sim->sim.velocity(2));
}
VB_API vapor_status vapor_mac3d_stream(vapor_mac3d* sim, void** stream) {
    SIM_GUARD(require(stream != nullptr, "null output"); *stream = (void*)sim->sim.stream());
}
VB_API vapor_status vapor_mac3d_resolution(const vapor_mac3d* sim, int32_t* n, float* box) {
    SIM_GUARD(if (n) *n = sim->sim.n(); if (box) *box = sim->sim.box());
}

VB_API vapor_status vapor_mac3d_set_timing(vapor_mac3d* sim, int32_t enabled) {
    SIM_GUARD(sim->sim.timer().enable(enabled != 0));
}
VB_API vapor_status vapor_mac3d_timings(vapor_mac3d* sim, vapor_phase_timings* out) {
    SIM_GUARD(require(out != nullptr, "null output"); *out = sim->sim.timer().totals());
}

// ---- staged stages ----
VB_API vapor_status vapor_stage_create(int32_t n, float box, vapor_stage** out) {
    return guarded([&] {
        require(out != nullptr, "null output");
        *out = nullptr;
        vb::validate_grid(n, box);
        require_device();
        *out = new vapor_stage(n, box);
    });
}
VB_API vapor_status vapor_stage_destroy(vapor_stage* stage) {
    return guarded([&] { delete stage; });
}

#define STAGE_GUARD(body)                                     \
    return guarded([&] {                                      \
        require(stage != nullptr, "null stage handle");      \
        body;                                                 \
    })

VB_API vapor_status vapor_stage_reset(vapor_stage* stage) { STAGE_GUARD(stage->stage.reset()); }
VB_API vapor_status vapor_stage_project(vapor_stage* stage, float* u, float* v, float* w,
                                        const vapor_projection_options* options, float diagonal_floor,
                                        vapor_projection_result* result, float* pressure_out) {
    STAGE_GUARD(require(options != nullptr, "null options");
                stage->stage.project(u, v, w, *options, diagonal_floor, result, pressure_out, false));
}
VB_API vapor_status vapor_stage_project_device(vapor_stage* stage, float* u, float* v, float* w,
                                               const vapor_projection_options* options, float diagonal_floor,
                                               vapor_projection_result* result, float* pressure_out) {
    STAGE_GUARD(require(options != nullptr, "null options");
                stage->stage.project(u, v, w, *options, diagonal_floor, result, pressure_out, true));
}
VB_API vapor_status vapor_stage_advect_face(vapor_stage* stage, int32_t axis, float dt, float cfl_limit,
                                            int32_t method, const float* source, const float* fu,
                                            const float* fv, const float* fw, float* output) {
    STAGE_GUARD(require(axis >= 0 && axis <= 2, "Invalid staggered field axis");
                stage->stage.advect(1 + axis, dt, cfl_limit, method, source, fu, fv, fw, output, false));
}
VB_API vapor_status vapor_stage_advect_face_device(vapor_stage* stage, int32_t axis, float dt, float cfl_limit,
                                                   int32_t method, const float* source, const float* fu,
                                                   const float* fv, const float* fw, float* output) {
    STAGE_GUARD(require(axis >= 0 && axis <= 2, "Invalid staggered field axis");
                stage->stage.advect(1 + axis, dt, cfl_limit, method, source, fu, fv, fw, output, true));
}
VB_API vapor_status vapor_stage_advect_scalar(vapor_stage* stage, float dt, float cfl_limit, int32_t method,
                                              float* field, const float* fu, const float* fv, const float* fw) {
    STAGE_GUARD(stage->stage.advect(0, dt, cfl_limit, method, field, fu, fv, fw, field, false));
}
VB_API vapor_status vapor_stage_advect_scalar_device(vapor_stage* stage, float dt, float cfl_limit, int32_t method,
                                                     float* field, const float* fu, const float* fv,
                                                     const float* fw) {
    STAGE_GUARD(stage->stage.advect(0, dt, cfl_limit, method, field, fu, fv, fw, field, true));
}
VB_API vapor_status vapor_stage_set_solver_kind(vapor_stage* stage, int32_t kind) {
    STAGE_GUARD(require(kind == VAPOR_SOLVER_RED_BLACK_SOR || kind == VAPOR_SOLVER_MIXED_REFINEMENT ||
                            kind == VAPOR_SOLVER_FPCG,
                        "Unknown solver kind");
                stage->stage.solver_kind = kind);
}
VB_API vapor_status vapor_stage_set_solid(vapor_stage* stage, const uint8_t* mask) {
    STAGE_GUARD(stage->stage.set_solid(mask));
}
VB_API vapor_status vapor_stage_solve_rhs(vapor_stage* stage, const float* rhs_device,
                                          const vapor_projection_options* options, float diagonal_floor,
                                          vapor_projection_result* result, float* pressure_device) {
    STAGE_GUARD(require(options != nullptr, "null options");
                stage->stage.solve_rhs(rhs_device, *options, diagonal_floor, result, pressure_device));
}
VB_API vapor_status vapor_stage_stream(vapor_stage* stage, void** stream) {
    STAGE_GUARD(require(stream != nullptr, "null output"); *stream = (void*)stage->stage.stream());
}

VB_API vapor_status vapor_tune_sor_planes(int32_t n, int32_t planes) {
    return guarded([&] {
        require(n > 0 && planes >= 0 && planes <= 64, "invalid tuning value");
        vb::set_sor_planes(n, planes);
    });
}

VB_API vapor_status vapor_tune_conv_kernel(int32_t kind) {
    return guarded([&] {
        require(kind >= 0 && kind <= 3, "0, 1, 2 or 3");
        vb::unet::set_conv_kernel(kind);
    });
}
VB_API vapor_status vapor_tune_wgrad_kernel(int32_t kind) {
    return guarded([&] { vb::unet::set_wgrad_kernel(kind); });
}
VB_API vapor_status vapor_tune_fpcg_smoothing(int32_t sweeps, float omega) {
    return guarded([&] { vb::set_fpcg_smoothing(sweeps, omega); });
}
VB_API vapor_status vapor_fpcg_smoothing(int32_t* sweeps, float* omega) {
    return guarded([&] {
        require(sweeps != nullptr && omega != nullptr, "null output");
        const vb::FpcgSmoothing sm = vb::fpcg_smoothing();
        *sweeps = sm.sweeps;
        *omega = sm.omega;
    });
}
VB_API vapor_status vapor_tune_sor_blocking(int32_t iterations_per_launch) {
    return guarded([&] { vb::set_sor_block_iterations(iterations_per_launch); });
}
VB_API vapor_status vapor_tune_sor_blocked_chunks(int32_t n, int32_t chunks) {
    return guarded([&] {
        require(n > 0 && chunks >= 0 && chunks <= n, "invalid tuning value");
        vb::set_sor_blocked_chunks(n, chunks);
    });
}

// ---- batched scenes ----
VB_API vapor_status vapor_batch_create(int32_t count, vapor_mac3d* const* sims, vapor_batch** out) {
    return guarded([&] {
        require(out != nullptr, "null output");
        *out = nullptr;
        require(count > 0 && sims != nullptr, "a batch needs at least one simulation");
        std::vector<vb::Simulation*> v;
        for (int32_t i = 0; i < count; ++i) {
            require(sims[i] != nullptr, "null simulation in batch");
            v.push_back(&sims[i]->sim);
        }
        *out = new vapor_batch(std::move(v));
    });
}
VB_API vapor_status vapor_batch_destroy(vapor_batch* batch) {
    return guarded([&] { delete batch; });
}
VB_API vapor_status vapor_batch_advance(vapor_batch* batch, float dt) {
    return guarded([&] {
        require(batch != nullptr, "null batch handle");
        batch->batch.advance(dt);
    });
}
VB_API vapor_status vapor_batch_synchronize(vapor_batch* batch) {
    return guarded([&] {
        require(batch != nullptr, "null batch handle");
        batch->batch.synchronize();
    });
}
VB_API vapor_status vapor_batch_stream(vapor_batch* batch, void** stream) {
    return guarded([&] {
        require(batch != nullptr && stream != nullptr, "null handle or output");
        *stream = (void*)batch->batch.stream();
    });
}

// ---- learned warm start ----
namespace {
// Orders the network's work on the simulation's stream for one call; after it
// the network goes back to its own stream unless the simulation uses it as
// its warm start.
struct StreamBinding {
    vb::Simulation& sim;
    vb::unet::UNet& net;
    StreamBinding(vb::Simulation& s, vb::unet::UNet& n, cudaStream_t stream) : sim(s), net(n) {
        net.set_stream(stream);
    }
    ~StreamBinding() {
        if (sim.warm_start() != &net) net.use_own_stream();
    }
};
}  // namespace
VB_API int64_t vapor_unet_parameter_count(void) { return vb::unet::parameter_count(); }

VB_API vapor_status vapor_unet_create(vapor_unet** out) {
    return guarded([&] {
        require(out != nullptr, "null output");
        *out = nullptr;
        require_device();
        *out = new vapor_unet();
    });
}
VB_API vapor_status vapor_unet_destroy(vapor_unet* net) {
    return guarded([&] { delete net; });
}

#define NET_GUARD(body)                                      \
    return guarded([&] {                                     \
        require(net != nullptr, "null network handle");     \
        net->net.use_own_stream();                           \
        body;                                                \
    })

VB_API vapor_status vapor_unet_init(vapor_unet* net, uint32_t seed) {
    NET_GUARD(net->net.init_parameters(seed));
}
VB_API vapor_status vapor_unet_set_parameters(vapor_unet* net, const float* host, int64_t count) {
    NET_GUARD(require(host && count == vb::unet::parameter_count(), "parameter count mismatch");
              net->net.set_parameters(host));
}
VB_API vapor_status vapor_unet_get_parameters(vapor_unet* net, float* host, int64_t count) {
    NET_GUARD(require(host && count == vb::unet::parameter_count(), "parameter count mismatch");
              net->net.get_parameters(host));
}
VB_API vapor_status vapor_unet_forward_features(vapor_unet* net, int32_t n, const void* input_bf16, float* output) {
    NET_GUARD(require(input_bf16 && output, "null buffer");
              net->net.forward_features(n, static_cast<const __nv_bfloat16*>(input_bf16), output);
              VB_CUDA(cudaStreamSynchronize(net->stream.s));
              net->net.check_error());
}
VB_API vapor_status vapor_unet_backward(vapor_unet* net, int32_t n, const float* grad_output, float* grad_params) {
    NET_GUARD(require(grad_output && grad_params, "null buffer");
              net->net.backward_from_output(n, grad_output);
              VB_CUDA(cudaMemcpyAsync(grad_params, net->net.gradient(),
                                      vb::unet::parameter_count() * sizeof(float), cudaMemcpyDeviceToHost,
                                      net->stream.s));
              VB_CUDA(cudaStreamSynchronize(net->stream.s));
              net->net.check_error());
}
VB_API vapor_status vapor_unet_set_wait_probe(vapor_unet* net, int32_t iterations) {
    NET_GUARD(require(iterations >= 0, "iterations must be non-negative"); net->net.set_wait_probe(iterations));
}
VB_API vapor_status vapor_mac3d_set_warm_start(vapor_mac3d* sim, vapor_unet* net) {
    SIM_GUARD(sim->sim.set_warm_start(net ? &net->net : nullptr));
}
VB_API vapor_status vapor_mac3d_set_coarse_log(vapor_mac3d* sim, float* log_device, int32_t capacity,
                                               int32_t* counter_device) {
    SIM_GUARD(require((log_device == nullptr) == (counter_device == nullptr), "log and counter go together");
              require(log_device == nullptr || capacity > 0, "capacity must be positive");
              sim->sim.set_coarse_log(log_device, capacity, counter_device));
}
VB_API vapor_status vapor_mac3d_set_solid(vapor_mac3d* sim, const uint8_t* mask) {
    SIM_GUARD(sim->sim.set_solid(mask));
}
VB_API vapor_status vapor_mac3d_set_preconditioner(vapor_mac3d* sim, vapor_unet* net) {
    SIM_GUARD(sim->sim.set_preconditioner(net ? &net->net : nullptr));
}
VB_API vapor_status vapor_stage_set_preconditioner(vapor_stage* stage, vapor_unet* net) {
    STAGE_GUARD(if (net && (stage->stage.n() % 16 != 0 || stage->stage.n() < 32))
                    vb::fail(VAPOR_INVALID_ARGUMENT, "the coarse-grid network needs n divisible by 16 (n >= 32)");
                stage->stage.coarse = net ? &net->net : nullptr);
}
VB_API vapor_status vapor_mac3d_train_warm_start(vapor_mac3d* sim, vapor_unet* net, float learning_rate,
                                                 double* loss) {
    SIM_GUARD(require(net != nullptr, "null network handle");
              require(std::isfinite(learning_rate) && learning_rate > 0.f, "invalid learning rate");
              vb::Workspace& ws = sim->sim.workspace(); StreamBinding bind(sim->sim, net->net, ws.stream());
              const double l = net->net.train_step(ws.n(), ws.rhs(), ws.pressure(), ws.control(), learning_rate);
              if (loss) *loss = l);
}
VB_API vapor_status vapor_stage_train_network(vapor_stage* stage, vapor_unet* net, float learning_rate,
                                              double* loss) {
    STAGE_GUARD(require(net != nullptr, "null network handle");
                require(std::isfinite(learning_rate) && learning_rate > 0.f, "invalid learning rate");
                vb::Workspace& ws = stage->stage.workspace(); net->net.set_stream(ws.stream());
                double l = 0.0;
                try {
                    l = net->net.train_step(ws.n(), ws.rhs(), ws.pressure(), ws.control(), learning_rate);
                } catch (...) {
                    net->net.use_own_stream();
                    throw;
                }
                net->net.use_own_stream();
                if (loss) *loss = l);
}
VB_API vapor_status vapor_mac3d_evaluate_warm_start(vapor_mac3d* sim, vapor_unet* net, double* loss) {
    SIM_GUARD(require(net != nullptr, "null network handle"); vb::Workspace& ws = sim->sim.workspace();
              StreamBinding bind(sim->sim, net->net, ws.stream());
              const double l = net->net.evaluate(ws.n(), ws.rhs(), ws.pressure(), ws.control());
              if (loss) *loss = l);
}
