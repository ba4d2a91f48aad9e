// TEST INFRASTRUCTURE — not part of the product. A C shim over the
// reference's own MAC 2D solvers (taehwann/vapor src/solvers/mac2d/*.cpp and
// the header-only ReflectionMacFluidSolver2D.hpp, compiled from where they lie
// by oracle/Makefile into _ref/libvapor_ref2d.so), so that the tests can step
// the reference's CPU solvers beside the device ones on the same state and
// parameters; and over the reference's historical 2D plume
// (tests/fixtures/Ba20987Smoke2D.hpp), which its Historical2DTests.cpp
// replays against the reflection solver.
#include "../include/vapor_b200.h"

#include "solvers/mac2d/MacGridFluidSolver2D.hpp"
#include "solvers/mac2d/ReflectionMacFluidSolver2D.hpp"
#include "fixtures/Ba20987Smoke2D.hpp"

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

// ---- ReflectionMacFluidSolver2D ----
namespace {
using Refl = ReflectionMacFluidSolver2D;
void to_refl(const vapor_mac2d_refl_params& p, Refl& r) {
    r.macCormackSmoke = p.mac_cormack_smoke != 0;
    r.sourceStrength = p.source_strength;
    r.buoyancy = p.buoyancy;
    r.smokeDecay = p.smoke_decay;
    r.projectIterations = p.project_iterations;
    r.emitterRadius = p.emitter_radius;
    r.emitterCenterX = p.emitter_center_x;
    r.emitterCenterY = p.emitter_center_y;
    r.emitterKickMultiplier = p.emitter_kick_multiplier;
    r.stirStrength = p.stir_strength;
    r.sorOmega = p.sor_omega;
    r.randomSeed = p.random_seed;
}
void from_refl(const Refl& r, vapor_mac2d_refl_params* p) {
    p->mac_cormack_smoke = r.macCormackSmoke ? 1 : 0;
    p->source_strength = r.sourceStrength;
    p->buoyancy = r.buoyancy;
    p->smoke_decay = r.smokeDecay;
    p->project_iterations = r.projectIterations;
    p->emitter_radius = r.emitterRadius;
    p->emitter_center_x = r.emitterCenterX;
    p->emitter_center_y = r.emitterCenterY;
    p->emitter_kick_multiplier = r.emitterKickMultiplier;
    p->stir_strength = r.stirStrength;
    p->sor_omega = r.sorOmega;
    p->random_seed = r.randomSeed;
}
}  // namespace

// A solver of resolution n (null on the reference's exception) with the given
// fields, its stirring stream started at the seed as resetState() does.
REF2_EXPORT void* ref2r_create(int n, const vapor_mac2d_refl_params* p) {
    try {
        Refl* r = new Refl(n);
        if (p) to_refl(*p, *r);
        r->randomState = r->randomSeed;
        return r;
    } catch (const std::exception&) {
        return nullptr;
    }
}
// The solver built from an advection method (0 semi-Lagrangian, 1 MacCormack).
REF2_EXPORT void* ref2r_create_app(int method) {
    try {
        return new Refl(method == 0 ? AdvectionMethod::SemiLagrangian : AdvectionMethod::MacCormack);
    } catch (const std::exception&) {
        return nullptr;
    }
}
REF2_EXPORT void ref2r_destroy(void* h) { delete static_cast<Refl*>(h); }
REF2_EXPORT int ref2r_resolution(void* h) { return static_cast<Refl*>(h)->n; }
REF2_EXPORT void ref2r_get_params(void* h, vapor_mac2d_refl_params* out) { from_refl(*static_cast<Refl*>(h), out); }
REF2_EXPORT void ref2r_set_params(void* h, const vapor_mac2d_refl_params* p) { to_refl(*p, *static_cast<Refl*>(h)); }
REF2_EXPORT void ref2r_reset(void* h) { static_cast<Refl*>(h)->resetState(); }
REF2_EXPORT void ref2r_set_fields(void* h, const float* s, const float* u, const float* v) {
    Refl& r = *static_cast<Refl*>(h);
    if (s) std::copy(s, s + r.smoke.size(), r.smoke.begin());
    if (u) std::copy(u, u + r.vx.size(), r.vx.begin());
    if (v) std::copy(v, v + r.vy.size(), r.vy.begin());
}
// 0 on success, 1 if the reference threw.
REF2_EXPORT int ref2r_advance(void* h, float dt) {
    try {
        static_cast<Refl*>(h)->advance(dt);
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}
REF2_EXPORT void ref2r_get_fields(void* h, float* s, float* u, float* v, float* pressure) {
    const Refl& r = *static_cast<Refl*>(h);
    std::copy(r.smoke.begin(), r.smoke.end(), s);
    std::copy(r.vx.begin(), r.vx.end(), u);
    std::copy(r.vy.begin(), r.vy.end(), v);
    std::copy(r.pressure.begin(), r.pressure.end(), pressure);
}
REF2_EXPORT void ref2r_diagnostics(void* h, vapor_fluid_diagnostics* out) {
    const FluidDiagnostics d = static_cast<Refl*>(h)->diagnostics();
    out->kinetic_energy = d.kineticEnergy;
    out->max_velocity = d.maxVelocity;
    out->max_divergence = d.maxDivergence;
}

// ---- the historical plume (Ba20987Smoke2D.hpp), closed walls ----
// Random stirring is off: the fixture's stirring stream is one process-wide
// state, so only the first instance of a process could replay it.
REF2_EXPORT void* ref2h_create(int n) {
    auto* s = new ba20987::SmokeSim2D(n);
    s->stirStrength = 0.f;
    s->openLeft = s->openRight = s->openTop = s->openBottom = false;
    return s;
}
REF2_EXPORT void ref2h_destroy(void* h) { delete static_cast<ba20987::SmokeSim2D*>(h); }
REF2_EXPORT void ref2h_step(void* h, float dt, float buoyancy, float dissipation, float strength, int iterations) {
    static_cast<ba20987::SmokeSim2D*>(h)->step(dt, buoyancy, dissipation, strength, iterations);
}
REF2_EXPORT void ref2h_get_fields(void* h, float* s, float* u, float* v, float* pressure) {
    const ba20987::SmokeSim2D& r = *static_cast<ba20987::SmokeSim2D*>(h);
    std::copy(r.smoke.begin(), r.smoke.end(), s);
    std::copy(r.vx.begin(), r.vx.end(), u);
    std::copy(r.vy.begin(), r.vy.end(), v);
    std::copy(r.pressure.begin(), r.pressure.end(), pressure);
}
