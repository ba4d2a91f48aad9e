// Advection entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc/cudaFree at the point where they advect
// a field: cudaFree synchronizes the whole device, which a frame loop with a
// hard time budget cannot afford; a host that owns all device memory itself
// (a renderer or engine with a fixed memory budget, or a plugin host that
// forbids a plugin from allocating) gives its plugins only the buffers it
// passes in. For those callers this entry point takes
// the MacCormack forward-pass scratch from a fixed array in this library's
// device image instead of allocating it.
//
// The array holds kNoAllocCapacity floats (4 MiB) on every GPU that loads
// the library, for as long as the process lives. The driver commits it when
// it loads this file's module into a context: at library load, or, under
// lazy module loading (CUDA_MODULE_LOADING=LAZY, the default of recent CUDA
// releases), during the first call in that context, which also looks up the
// array's address. Callers should therefore make one call during set-up,
// before any stream capture. The address is cached per CUDA context; a device
// reset (cudaDeviceReset) ends the context it belongs to, so this entry point
// must not be used after a reset in the same process. The largest field it can
// advect has kNoAllocCapacity values (face arrays up to n = 101).
// All calls share the one array: calls that overlap on the GPU (different
// streams, or different threads without ordering) race on it and must be
// serialized by the caller. No part of it needs clearing between calls: the
// forward pass writes every entry the correction pass reads.
#include <climits>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>

#include "engine.hpp"

namespace {

constexpr size_t kNoAllocCapacity = size_t(1) << 20;

// Fixed device scratch for the MacCormack forward pass. In host code this
// name is a host-side stand-in, not a device address: the device address is
// obtained with cudaGetSymbolAddress below.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocCapacity];

// The array's device address belongs to a CUDA context (the module holding
// it is loaded once per context), so looked-up addresses are cached per
// context: the runtime's primary context of each device, or any context the
// caller made current with the driver API.
using CtxGetCurrentFn = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)
std::mutex g_scratch_mutex;
std::map<void*, float*> g_scratch_ptr;

CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q);
        return (e == cudaSuccess && q == cudaDriverEntryPointSuccess) ? reinterpret_cast<CtxGetCurrentFn>(f)
                                                                        : nullptr;
    }();
    if (!fn) vb::fail(VAPOR_RUNTIME_ERROR, "cuCtxGetCurrent is not available from the CUDA driver");
    return fn;
}

// Device address of the scratch array in the current context. The first call
// in a context looks it up with that context current (under lazy module
// loading this also loads the module and commits the array) and caches it.
float* scratch_for_current_context() {
    void* ctx = nullptr;
    void* ptr = nullptr;
    if (ctx_get_current()(&ctx) != 0) vb::fail(VAPOR_RUNTIME_ERROR, "cuCtxGetCurrent failed");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (ctx) {
        const auto it = g_scratch_ptr.find(ctx);
        if (it != g_scratch_ptr.end()) return it->second;
    }
    // with no context current yet, this call makes the device's primary
    // context current (the runtime's implicit initialization)
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr)
        vb::fail(VAPOR_RUNTIME_ERROR, std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                          cudaGetErrorString(e));
    if (!ctx && (ctx_get_current()(&ctx) != 0 || !ctx)) vb::fail(VAPOR_RUNTIME_ERROR, "no current CUDA context");
    g_scratch_ptr[ctx] = static_cast<float*>(ptr);
    return static_cast<float*>(ptr);
}

bool overlaps(const float* a, size_t na, const float* b, size_t nb) {
    const uintptr_t a0 = uintptr_t(a), a1 = uintptr_t(a + na), b0 = uintptr_t(b), b1 = uintptr_t(b + nb);
    return a0 < b1 && b0 < a1;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) vapor_status vapor_advect_noalloc(
    int32_t n, float box, int32_t loc, float dt, float cfl_limit, int32_t method, const float* source,
    const float* flow_u, const float* flow_v, const float* flow_w, float* output, void* stream) {
    return vb::guard([&] {
        vb::validate_grid(n, box);
        if (loc < vb::CELL || loc > vb::FACE_Z) vb::fail(VAPOR_INVALID_ARGUMENT, "Invalid staggered field location");
        if (method != VAPOR_SEMI_LAGRANGIAN && method != VAPOR_MACCORMACK)
            vb::fail(VAPOR_INVALID_ARGUMENT, "Invalid advection method");
        if (!std::isfinite(dt) || dt < 0.f || !std::isfinite(cfl_limit) || cfl_limit <= 0.f)
            vb::fail(VAPOR_INVALID_ARGUMENT, "Invalid advection time step or CFL limit");
        if (!source || !flow_u || !flow_v || !flow_w || !output)
            vb::fail(VAPOR_INVALID_ARGUMENT, "Advection fields are required");
        const size_t count = vb::count_of(n, loc);
        const size_t faces = size_t(n) * n * (n + 1);
        if (count > kNoAllocCapacity)
            vb::fail(VAPOR_LENGTH_ERROR, "field of " + std::to_string(count) +
                                             " values exceeds the no-allocation scratch capacity of " +
                                             std::to_string(kNoAllocCapacity) + " values (n <= 101 for faces)");
        if (overlaps(source, count, output, count) || overlaps(output, count, flow_u, faces) ||
            overlaps(output, count, flow_v, faces) || overlaps(output, count, flow_w, faces))
            vb::fail(VAPOR_INVALID_ARGUMENT, "Advection output must not alias its source or the tracer velocities");
        float* scratch = scratch_for_current_context();
        const vb::Grid g{n, box, box / float(n)};
        vb::launch_advect(g, loc, dt, cfl_limit, method == VAPOR_MACCORMACK, source, flow_u, flow_v, flow_w, scratch,
                          output, 1.f, static_cast<cudaStream_t>(stream));
        VB_CUDA(cudaGetLastError());
    });
}
