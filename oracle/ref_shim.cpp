// TEST INFRASTRUCTURE — C entry points over the reference's own CPU MAC 3D
// classes (taehwann/vapor, src/solvers/mac3d/*.cpp), compiled together with
// those unmodified sources by oracle/Makefile into oracle/_ref/libvapor_ref.so.
// Only tests/ and bench.py's reference/CPU-baseline leg load it.
//
// Wrapped reference interfaces:
//   MacGridFluidSolver3D  ctor/advance/resetState/setBoxSize/parameters/
//                         diagnostics/lastProjection (MacGridFluidSolver3D.hpp:39-124)
//   CpuAdvection          advectScalar/advectFace (CpuAdvection.hpp:4-10)
//   CpuPressureSolver3D   project (CpuPressureSolver3D.hpp:12-29)
//   SOR                   solve (SOR.hpp:8-21) on an explicit StencilLinearSystem
//   MacGridSampler3D      sample* (MacGridSampler3D.hpp:8-18)
//   MacGridOperators3D    maxDivergence (MacGridOperators3D.hpp:5-11)
// Exceptions map to vapor_status codes: invalid_argument -> 1,
// length_error -> 2, anything else -> 3.

#include "../include/vapor_b200.h"

#include "solvers/mac3d/CpuAdvection.hpp"
#include "solvers/mac3d/CpuPressureSolver3D.hpp"
#include "solvers/mac3d/MacGridFluidSolver3D.hpp"
#include "solvers/mac3d/MacGridOperators3D.hpp"
#include "solvers/mac3d/MacGridSampler3D.hpp"
#include "solvers/mac3d/SOR.hpp"

#include <algorithm>
#include <cstring>
#include <memory>
#include <stdexcept>

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

template <class F>
int guarded(F&& f) {
    try {
        f();
        return VAPOR_OK;
    } catch (const std::invalid_argument&) {
        return VAPOR_INVALID_ARGUMENT;
    } catch (const std::length_error&) {
        return VAPOR_LENGTH_ERROR;
    } catch (...) {
        return VAPOR_RUNTIME_ERROR;
    }
}

LinearSolveOptions toOptions(const vapor_linear_solve_options& o) {
    LinearSolveOptions r;
    r.maxIterations = o.max_iterations;
    r.residualCheckInterval = o.residual_check_interval;
    r.absoluteTolerance = o.absolute_tolerance;
    r.relativeTolerance = o.relative_tolerance;
    r.fixedIterations = o.fixed_iterations != 0;
    return r;
}

void fromResult(const ProjectionResult& r, vapor_projection_result* out) {
    std::memset(out, 0, sizeof(*out));
    out->linear_solve.iterations = r.linearSolve.iterations;
    out->linear_solve.converged = r.linearSolve.converged;
    out->linear_solve.initial_residual = r.linearSolve.initialResidual;
    out->linear_solve.final_residual = r.linearSolve.finalResidual;
    out->residual_available = r.residualAvailable;
    out->divergence_before = r.divergenceBefore;
    out->divergence_after = r.divergenceAfter;
    out->removed_rhs_mean = r.removedRhsMean;
}

// The reference's own plugin hook for tolerance-driven projections: the
// coordinator forces fixed iterations (MacGridFluidSolver3D.cpp:131-138); a
// Projection3D installed with setPressureSolver replaces the solve options.
class ToleranceProjection final : public Projection3D {
public:
    explicit ToleranceProjection(LinearSolveOptions o) : options_(o) {}
    ProjectionResult project(MacGridState3D& state, const ProjectionOptions& options) override {
        ProjectionOptions adjusted = options;
        adjusted.linearSolve = options_;
        return cpu_.project(state, adjusted);
    }
    void reset() noexcept override { cpu_.reset(); }

private:
    LinearSolveOptions options_;
    CpuPressureSolver3D cpu_{6.f};
};

struct RefSim {
    std::unique_ptr<MacGridFluidSolver3D> solver;
};

MacGridState3D stateFrom(int n, float box, const float* d, const float* u, const float* v, const float* w) {
    MacGridState3D s(n, box);
    if (d) std::copy(d, d + s.density().size(), s.density().begin());
    if (u) std::copy(u, u + s.velocityX().size(), s.velocityX().begin());
    if (v) std::copy(v, v + s.velocityY().size(), s.velocityY().begin());
    if (w) std::copy(w, w + s.velocityZ().size(), s.velocityZ().begin());
    return s;
}

}  // namespace

REF_EXPORT int ref_sim_create(int n, float box, void** out) {
    return guarded([&] {
        auto* h = new RefSim;
        try {
            h->solver = std::make_unique<MacGridFluidSolver3D>(MacGridState3D(n, box));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

REF_EXPORT int ref_sim_create_algorithm(int algorithm, void** out) {
    return guarded([&] {
        auto* h = new RefSim;
        try {
            h->solver = std::make_unique<MacGridFluidSolver3D>(static_cast<MacAlgorithm>(algorithm));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

// MacGridFluidSolver3D(MacGridState3D): fields as given, no reset.
REF_EXPORT int ref_sim_create_from_fields(int n, float box, const float* d, const float* u, const float* v,
                                          const float* w, void** out) {
    return guarded([&] {
        auto* h = new RefSim;
        try {
            h->solver = std::make_unique<MacGridFluidSolver3D>(stateFrom(n, box, d, u, v, w));
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

REF_EXPORT void ref_sim_destroy(void* h) { delete static_cast<RefSim*>(h); }

// Reference fields only. use_solve_options installs ToleranceProjection; the
// other extensions have no reference counterpart and are rejected.
REF_EXPORT int ref_sim_set_params(void* h, const vapor_mac3d_params* p) {
    return guarded([&] {
        if (p->emitter_profile != 0 || p->emitter_count != 1 || p->solver_kind != VAPOR_SOLVER_RED_BLACK_SOR)
            throw std::invalid_argument("extension parameters have no reference counterpart");
        auto* s = static_cast<RefSim*>(h)->solver.get();
        auto& q = s->parameters();
        q.emitterRadius = p->emitter_radius;
        q.emitterCenterX = p->emitter_center_x;
        q.emitterCenterY = p->emitter_center_y;
        q.emitterCenterZ = p->emitter_center_z;
        q.emitterKickMultiplier = p->emitter_kick_multiplier;
        q.emitterKickBase = p->emitter_kick_base;
        q.emitterKickScale = p->emitter_kick_scale;
        q.stirStrength = p->stir_strength;
        q.randomSeed = p->random_seed;
        q.sorOmega = p->sor_omega;
        q.buoyancySplit = p->buoyancy_split;
        q.cflMc = p->cfl_mc;
        q.macCormackSmoke = p->mac_cormack_smoke != 0;
        q.macCormackVel = p->mac_cormack_vel != 0;
        q.smokeDecay = p->smoke_decay;
        q.reflection = p->reflection != 0;
        q.buoyancy = p->buoyancy;
        q.sourceStrength = p->source_strength;
        q.projectIterations = p->project_iterations;
        if (p->use_solve_options)
            s->setPressureSolver(std::make_unique<ToleranceProjection>(toOptions(p->solve)));
        else
            s->useDefaultPressureSolver();
    });
}

REF_EXPORT void ref_sim_get_params(void* h, vapor_mac3d_params* p) {
    const auto& q = static_cast<RefSim*>(h)->solver->parameters();
    vapor_mac3d_default_params(p);
    p->emitter_radius = q.emitterRadius;
    p->emitter_center_x = q.emitterCenterX;
    p->emitter_center_y = q.emitterCenterY;
    p->emitter_center_z = q.emitterCenterZ;
    p->emitter_kick_multiplier = q.emitterKickMultiplier;
    p->emitter_kick_base = q.emitterKickBase;
    p->emitter_kick_scale = q.emitterKickScale;
    p->stir_strength = q.stirStrength;
    p->random_seed = q.randomSeed;
    p->sor_omega = q.sorOmega;
    p->buoyancy_split = q.buoyancySplit;
    p->cfl_mc = q.cflMc;
    p->mac_cormack_smoke = q.macCormackSmoke;
    p->mac_cormack_vel = q.macCormackVel;
    p->smoke_decay = q.smokeDecay;
    p->reflection = q.reflection;
    p->buoyancy = q.buoyancy;
    p->source_strength = q.sourceStrength;
    p->project_iterations = q.projectIterations;
}

REF_EXPORT int ref_sim_reset(void* h) {
    return guarded([&] { static_cast<RefSim*>(h)->solver->resetState(); });
}
REF_EXPORT int ref_sim_set_box(void* h, float box) {
    return guarded([&] { static_cast<RefSim*>(h)->solver->setBoxSize(box); });
}
REF_EXPORT int ref_sim_advance(void* h, float dt) {
    return guarded([&] { static_cast<RefSim*>(h)->solver->advance(dt); });
}
REF_EXPORT void ref_sim_get_fields(void* h, float* d, float* u, float* v, float* w) {
    const auto& s = static_cast<RefSim*>(h)->solver->state();
    std::copy(s.density().begin(), s.density().end(), d);
    std::copy(s.velocityX().begin(), s.velocityX().end(), u);
    std::copy(s.velocityY().begin(), s.velocityY().end(), v);
    std::copy(s.velocityZ().begin(), s.velocityZ().end(), w);
}
REF_EXPORT int ref_sim_diagnostics(void* h, vapor_fluid_diagnostics* out) {
    return guarded([&] {
        const auto d = static_cast<RefSim*>(h)->solver->diagnostics();
        out->kinetic_energy = d.kineticEnergy;
        out->max_velocity = d.maxVelocity;
        out->max_divergence = d.maxDivergence;
    });
}
REF_EXPORT void ref_sim_last_projection(void* h, vapor_projection_result* out) {
    fromResult(static_cast<RefSim*>(h)->solver->lastProjection(), out);
}
REF_EXPORT int ref_sim_resolution(void* h) { return static_cast<RefSim*>(h)->solver->resolution(); }
REF_EXPORT float ref_sim_box(void* h) { return static_cast<RefSim*>(h)->solver->boxSize(); }

// ---- staged operations on explicit fields ----

// loc: 0 cell, 1/2/3 x/y/z faces. Flow spans are the tracer velocity.
REF_EXPORT int ref_advect(int n, float box, int loc, float dt, float cfl, int maccormack, const float* src,
                          const float* u, const float* v, const float* w, float* out) {
    return guarded([&] {
        MacGridState3D grid(n, box);
        const VelocityFieldView flow{{u, grid.velocityX().size()}, {v, grid.velocityY().size()},
                                     {w, grid.velocityZ().size()}};
        const AdvectionContext context{grid, flow, dt, cfl};
        AdvectionWorkspace workspace;
        CpuAdvection method;
        const auto selected = maccormack ? AdvectionMethod::MacCormack : AdvectionMethod::SemiLagrangian;
        if (loc == 0) {
            std::copy(src, src + grid.cellCount(), out);
            method.advectScalar(context, {out, grid.cellCount()}, workspace, selected);
        } else {
            const size_t count = grid.velocityX().size();
            method.advectFace(context, static_cast<FaceAxis>(loc - 1), {src, count}, {out, count}, workspace,
                              selected);
        }
    });
}

REF_EXPORT int ref_project(int n, float box, float* u, float* v, float* w, float dt, float omega,
                           float diagonalFloor, const vapor_linear_solve_options* o,
                           vapor_projection_result* result, float* pressureOut) {
    return guarded([&] {
        MacGridState3D state = stateFrom(n, box, nullptr, u, v, w);
        CpuPressureSolver3D solver(diagonalFloor);
        ProjectionOptions options;
        options.dt = dt;
        options.relaxation = omega;
        options.linearSolve = toOptions(*o);
        const auto r = solver.project(state, options);
        fromResult(r, result);
        std::copy(state.velocityX().begin(), state.velocityX().end(), u);
        std::copy(state.velocityY().begin(), state.velocityY().end(), v);
        std::copy(state.velocityZ().begin(), state.velocityZ().end(), w);
        if (pressureOut) std::copy(solver.pressure().begin(), solver.pressure().end(), pressureOut);
    });
}

// SOR::solve on an explicit seven-point system (rows diag/right/up/front).
REF_EXPORT int ref_sor_solve(int n, float omega, float diagonalFloor, const float* diag, const float* right,
                             const float* up, const float* front, float* x, const float* b,
                             const vapor_linear_solve_options* o, vapor_linear_solve_result* r) {
    return guarded([&] {
        StencilLinearSystem s;
        s.resize(n);
        for (size_t i = 0; i < s.x.size(); ++i) {
            s.matrix[i] = {diag[i], right[i], up[i], front[i]};
            s.x[i] = x[i];
            s.b[i] = b[i];
        }
        SOR sor(omega, diagonalFloor);
        const auto res = sor.solve(s, toOptions(*o));
        std::copy(s.x.begin(), s.x.end(), x);
        r->iterations = res.iterations;
        r->converged = res.converged;
        r->initial_residual = res.initialResidual;
        r->final_residual = res.finalResidual;
    });
}

REF_EXPORT double ref_sample(int n, float box, int loc, const float* f, float x, float y, float z) {
    MacGridState3D grid(n, box);
    MacGridSampler3D s(grid);
    const Vec3 p{x, y, z};
    switch (loc) {
        case 0: return s.sampleCell({f, grid.cellCount()}, p);
        case 1: return s.sampleVxField({f, grid.velocityX().size()}, p);
        case 2: return s.sampleVyField({f, grid.velocityY().size()}, p);
        default: return s.sampleVzField({f, grid.velocityZ().size()}, p);
    }
}

REF_EXPORT int ref_max_divergence(int n, float box, const float* u, const float* v, const float* w, float* out) {
    return guarded([&] {
        MacGridState3D state = stateFrom(n, box, nullptr, u, v, w);
        *out = MacGridOperators3D::maxDivergence(state);
    });
}

REF_EXPORT int ref_divergence(int n, float box, const float* u, const float* v, const float* w, float* out) {
    return guarded([&] {
        MacGridState3D state = stateFrom(n, box, nullptr, u, v, w);
        MacGridOperators3D::computeDivergence(state, {out, state.cellCount()});
    });
}

// Parameter presets, for the shim's own users (the shim does not link the oracle).
REF_EXPORT vapor_status vapor_mac3d_default_params(vapor_mac3d_params* o) {
    std::memset(o, 0, sizeof(*o));
    const MacGridParameters3D q;
    o->emitter_radius = q.emitterRadius;
    o->emitter_center_x = q.emitterCenterX;
    o->emitter_center_y = q.emitterCenterY;
    o->emitter_center_z = q.emitterCenterZ;
    o->emitter_kick_multiplier = q.emitterKickMultiplier;
    o->emitter_kick_base = q.emitterKickBase;
    o->emitter_kick_scale = q.emitterKickScale;
    o->stir_strength = q.stirStrength;
    o->random_seed = q.randomSeed;
    o->sor_omega = q.sorOmega;
    o->buoyancy_split = q.buoyancySplit;
    o->cfl_mc = q.cflMc;
    o->mac_cormack_smoke = q.macCormackSmoke;
    o->mac_cormack_vel = q.macCormackVel;
    o->smoke_decay = q.smokeDecay;
    o->reflection = q.reflection;
    o->buoyancy = q.buoyancy;
    o->source_strength = q.sourceStrength;
    o->project_iterations = q.projectIterations;
    const LinearSolveOptions l;
    o->solve.max_iterations = l.maxIterations;
    o->solve.residual_check_interval = l.residualCheckInterval;
    o->solve.absolute_tolerance = l.absoluteTolerance;
    o->solve.relative_tolerance = l.relativeTolerance;
    o->solve.fixed_iterations = l.fixedIterations;
    o->emitter_count = 1;
    o->emitter2_center_x = 0.5f;
    o->emitter2_center_y = 0.5f;
    o->emitter2_center_z = 0.1f;
    return VAPOR_OK;
}
