// TEST INFRASTRUCTURE — not part of the product. A C shim over the
// reference's own MAC 2D solver (taehwann/vapor src/solvers/mac2d/*.cpp,
// compiled from where they lie by oracle/Makefile into
// _ref/libvapor_ref2d.so), so that the tests can step the reference's CPU
// solver beside the device one on the same state and parameters.
#include "../include/vapor_b200.h"

#include "solvers/mac2d/MacGridFluidSolver2D.hpp"

#include <algorithm>
#include <exception>

#define REF2_EXPORT extern "C" __attribute__((visibility("default")))

namespace {
void to_params(const vapor_mac2d_params& p, MacGridParameters2D& r) {
    r.reflection = p.reflection != 0;
    r.sourceStrength = p.source_strength;
    r.emitterKickMultiplier = p.emitter_kick_multiplier;
    r.emitterRadius = p.emitter_radius;
    r.emitterCenterX = p.emitter_center_x;
    r.emitterCenterY = p.emitter_center_y;
    r.buoyancy = p.buoyancy;
    r.smokeDecay = p.smoke_decay;
    r.sorOmega = p.sor_omega;
    r.projectIterations = p.project_iterations;
}
void to_result(const ProjectionResult& r, vapor_projection_result* out) {
    *out = vapor_projection_result{};
    out->linear_solve.iterations = r.linearSolve.iterations;
    out->linear_solve.converged = r.linearSolve.converged ? 1 : 0;
    out->linear_solve.initial_residual = r.linearSolve.initialResidual;
    out->linear_solve.final_residual = r.linearSolve.finalResidual;
    out->residual_available = r.residualAvailable ? 1 : 0;
    out->divergence_before = r.divergenceBefore;
    out->divergence_after = r.divergenceAfter;
    out->removed_rhs_mean = r.removedRhsMean;
}
}  // namespace

// A solver on the given state (any field pointer may be null: zeros).
REF2_EXPORT void* ref2_create(int n, float box, const float* d, const float* u, const float* v) {
    try {
        MacGridState2D state(n, box);
        if (d) std::copy(d, d + state.density().size(), state.density().begin());
        if (u) std::copy(u, u + state.velocityX().size(), state.velocityX().begin());
        if (v) std::copy(v, v + state.velocityY().size(), state.velocityY().begin());
        return new MacGridFluidSolver2D(std::move(state));
    } catch (const std::exception&) {
        return nullptr;
    }
}
REF2_EXPORT void ref2_destroy(void* h) { delete static_cast<MacGridFluidSolver2D*>(h); }
REF2_EXPORT void ref2_set_params(void* h, const vapor_mac2d_params* p) {
    to_params(*p, static_cast<MacGridFluidSolver2D*>(h)->parameters());
}
// 0 on success, 1 if the reference threw.
REF2_EXPORT int ref2_advance(void* h, float dt) {
    try {
        static_cast<MacGridFluidSolver2D*>(h)->advance(dt);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}
REF2_EXPORT void ref2_get_fields(void* h, float* d, float* u, float* v) {
    const MacGridState2D& s = static_cast<MacGridFluidSolver2D*>(h)->state();
    std::copy(s.density().begin(), s.density().end(), d);
    std::copy(s.velocityX().begin(), s.velocityX().end(), u);
    std::copy(s.velocityY().begin(), s.velocityY().end(), v);
}
REF2_EXPORT void ref2_last_projection(void* h, vapor_projection_result* out) {
    to_result(static_cast<MacGridFluidSolver2D*>(h)->lastProjection(), out);
}
REF2_EXPORT void ref2_midpoint_projection(void* h, vapor_projection_result* out) {
    to_result(static_cast<MacGridFluidSolver2D*>(h)->midpointProjection(), out);
}
REF2_EXPORT void ref2_diagnostics(void* h, vapor_fluid_diagnostics* out) {
    const FluidDiagnostics d = static_cast<MacGridFluidSolver2D*>(h)->diagnostics();
    out->kinetic_energy = d.kineticEnergy;
    out->max_velocity = d.maxVelocity;
    out->max_divergence = d.maxDivergence;
}
