// C++ host interface of vapor_b200 over the C ABI (include/vapor_b200.h).
//
// vapor_b200::CudaMacSimulation3D mirrors the reference's resident coordinator
// GpuMacSimulation3D (src/solvers/mac3d/gpu/GpuMacSimulation3D.hpp:9-46):
// construction from an algorithm preset or (n, box, parameters), advance,
// resetState, setBoxSize, parameters, lastProjection, upload/download and the
// byte counters. Status codes from the C ABI become the reference's exception
// types: std::invalid_argument, std::length_error, std::runtime_error.
//
// Header-only; link against vapor_b200/_lib/libvapor_b200.so.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/vapor_b200.h"

namespace vapor_b200 {

inline void check(vapor_status status) {
    if (status == VAPOR_OK) return;
    const std::string message = vapor_last_error();
    switch (status) {
        case VAPOR_INVALID_ARGUMENT:
        case VAPOR_NON_FINITE: throw std::invalid_argument(message);
        case VAPOR_LENGTH_ERROR: throw std::length_error(message);
        case VAPOR_OUT_OF_MEMORY: throw std::bad_alloc();
        default: throw std::runtime_error(message);
    }
}

inline vapor_mac3d_params defaultParameters() {
    vapor_mac3d_params p;
    check(vapor_mac3d_default_params(&p));
    return p;
}

inline vapor_mac3d_params algorithmParameters(vapor_mac_algorithm algorithm) {
    vapor_mac3d_params p;
    check(vapor_mac3d_algorithm_params(algorithm, &p));
    return p;
}

// Host snapshot of a MAC state in the reference layout.
struct HostState {
    int n = 0;
    float box = 0.f;
    std::vector<float> density, u, v, w;
    HostState() = default;
    HostState(int n_, float box_)
        : n(n_), box(box_), density(size_t(n_) * n_ * n_), u(size_t(n_) * n_ * (n_ + 1)),
          v(size_t(n_) * n_ * (n_ + 1)), w(size_t(n_) * n_ * (n_ + 1)) {}
};

class CudaMacSimulation3D {
public:
    explicit CudaMacSimulation3D(vapor_mac_algorithm algorithm)
        : CudaMacSimulation3D(32, 4.5f, algorithmParameters(algorithm)) {}
    CudaMacSimulation3D(int n, float box, const vapor_mac3d_params& parameters) : params_(parameters) {
        check(vapor_mac3d_create(n, box, &params_, &handle_));
    }
    ~CudaMacSimulation3D() {
        if (handle_) vapor_mac3d_destroy(handle_);
    }
    CudaMacSimulation3D(const CudaMacSimulation3D&) = delete;
    CudaMacSimulation3D& operator=(const CudaMacSimulation3D&) = delete;

    // parameters() is read on every advance, as in the reference.
    vapor_mac3d_params& parameters() { return params_; }
    void advance(float dt) {
        check(vapor_mac3d_set_params(handle_, &params_));
        check(vapor_mac3d_advance(handle_, dt));
    }
    void resetState() {
        check(vapor_mac3d_set_params(handle_, &params_));
        check(vapor_mac3d_reset(handle_));
    }
    void setBoxSize(float size) { check(vapor_mac3d_set_box(handle_, size)); }
    float boxSize() const {
        int32_t n;
        float b;
        check(vapor_mac3d_resolution(handle_, &n, &b));
        return b;
    }
    int resolution() const {
        int32_t n;
        float b;
        check(vapor_mac3d_resolution(handle_, &n, &b));
        return n;
    }
    vapor_projection_result lastProjection() const {
        vapor_projection_result r;
        check(vapor_mac3d_last_projection(handle_, &r));
        return r;
    }
    vapor_fluid_diagnostics diagnostics() const {
        vapor_fluid_diagnostics d;
        check(vapor_mac3d_diagnostics(handle_, &d));
        return d;
    }
    void upload(const HostState& s) {
        if (s.n != resolution() || s.box != boxSize()) throw std::invalid_argument("GPU snapshot box mismatch");
        check(vapor_mac3d_upload(handle_, s.density.data(), s.u.data(), s.v.data(), s.w.data()));
    }
    void download(HostState& s) const {
        if (s.n != resolution() || s.box != boxSize()) throw std::invalid_argument("GPU snapshot box mismatch");
        check(vapor_mac3d_download(handle_, s.density.data(), s.u.data(), s.v.data(), s.w.data()));
    }
    // Streamed transfers (vapor_mac3d_upload_async / _download_async): the
    // snapshot must stay alive and unchanged, and a downloaded one unread,
    // until waitTransfers() returns.
    void uploadAsync(const HostState& s) {
        if (s.n != resolution() || s.box != boxSize()) throw std::invalid_argument("GPU snapshot box mismatch");
        check(vapor_mac3d_upload_async(handle_, s.density.data(), s.u.data(), s.v.data(), s.w.data()));
    }
    void downloadAsync(HostState& s) {
        if (s.n != resolution() || s.box != boxSize()) throw std::invalid_argument("GPU snapshot box mismatch");
        check(vapor_mac3d_download_async(handle_, s.density.data(), s.u.data(), s.v.data(), s.w.data()));
    }
    void waitTransfers() { check(vapor_mac3d_wait_transfers(handle_)); }
    std::uint64_t uploadedBytes() const {
        uint64_t up, down;
        check(vapor_mac3d_byte_counters(handle_, &up, &down));
        return up;
    }
    std::uint64_t downloadedBytes() const {
        uint64_t up, down;
        check(vapor_mac3d_byte_counters(handle_, &up, &down));
        return down;
    }
    // renderData() analogue: borrowed device pointer of the density.
    const float* deviceDensity() const {
        float* d = nullptr;
        check(vapor_mac3d_device_fields(handle_, &d, nullptr, nullptr, nullptr));
        return d;
    }
    vapor_mac3d* handle() const { return handle_; }

private:
    vapor_mac3d_params params_;
    vapor_mac3d* handle_ = nullptr;
};

}  // namespace vapor_b200
