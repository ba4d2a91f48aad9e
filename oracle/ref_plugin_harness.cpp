// TEST INFRASTRUCTURE — drives the reference's own coordinator
// MacGridFluidSolver3D (taehwann/vapor, src/solvers/mac3d/, compiled from its
// sources by oracle/Makefile) with the product's drop-in CUDA stages
// (vapor_b200/host/VaporCudaStages.hpp) installed through the reference's
// plugin hooks setPressureSolver / setAdvection (MacGridFluidSolver3D.cpp:305-313).
// This is the staged-parity harness the reference runs for its OpenGL stages
// (tests/GraphicsSmokeTests.cpp:22-43), with CUDA in place of OpenGL. It also
// exercises the C++ resident wrapper vapor_b200::CudaMacSimulation3D.
// Built into oracle/_ref/libvapor_ref_plugins.so; only tests/ load it.

#include <algorithm>
#include <cstring>
#include <memory>

#include "VaporCudaStages.hpp"
#include "solvers/mac3d/MacGridFluidSolver3D.hpp"

#define HX extern "C" __attribute__((visibility("default")))

namespace {

void toReference(const vapor_mac3d_params& p, MacGridParameters3D& q) {
    q.emitterRadius = p.emitter_radius;
    q.emitterCenterX = p.emitter_center_x;
    q.emitterCenterY = p.emitter_center_y;
    q.emitterCenterZ = p.emitter_center_z;
    q.emitterKickMultiplier = p.emitter_kick_multiplier;
    q.emitterKickBase = p.emitter_kick_base;
    q.emitterKickScale = p.emitter_kick_scale;
    q.stirStrength = p.stir_strength;
    q.randomSeed = p.random_seed;
    q.sorOmega = p.sor_omega;
    q.buoyancySplit = p.buoyancy_split;
    q.cflMc = p.cfl_mc;
    q.macCormackSmoke = p.mac_cormack_smoke != 0;
    q.macCormackVel = p.mac_cormack_vel != 0;
    q.smokeDecay = p.smoke_decay;
    q.reflection = p.reflection != 0;
    q.buoyancy = p.buoyancy;
    q.sourceStrength = p.source_strength;
    q.projectIterations = p.project_iterations;
}

// Counts stage calls while delegating to a CUDA stage (BackendTests.cpp:18-60 pattern).
struct Counts {
    long long projections = 0, faces = 0, scalars = 0;
};

class CountingProjection final : public Projection3D {
public:
    CountingProjection(std::shared_ptr<vapor_b200::StageBackend> b, Counts* c) : inner_(6.f, std::move(b)), c_(c) {}
    ProjectionResult project(MacGridState3D& s, const ProjectionOptions& o) override {
        ++c_->projections;
        return inner_.project(s, o);
    }
    void reset() noexcept override { inner_.reset(); }

private:
    vapor_b200::CudaProjection3D inner_;
    Counts* c_;
};

class CountingAdvection final : public Advection3D {
public:
    CountingAdvection(std::shared_ptr<vapor_b200::StageBackend> b, Counts* c) : inner_(std::move(b)), c_(c) {}
    void advectScalar(const AdvectionContext& ctx, std::span<float> f, AdvectionWorkspace& ws,
                      AdvectionMethod m) const override {
        ++c_->scalars;
        inner_.advectScalar(ctx, f, ws, m);
    }
    void advectFace(const AdvectionContext& ctx, FaceAxis a, std::span<const float> s, std::span<float> o,
                    AdvectionWorkspace& ws, AdvectionMethod m) const override {
        ++c_->faces;
        inner_.advectFace(ctx, a, s, o, ws, m);
    }

private:
    vapor_b200::CudaAdvection3D inner_;
    Counts* c_;
};

}  // namespace

// Runs `frames` steps of the reference coordinator; cuda_projection /
// cuda_advection select the CUDA stages. counts (may be null) receives
// {projections, face advections, scalar advections} made through the plugins.
HX int harness_run(int n, float box, const vapor_mac3d_params* p, int frames, float dt, int cuda_projection,
                   int cuda_advection, float* d, float* u, float* v, float* w, long long* counts) {
    try {
        MacGridFluidSolver3D solver{MacGridState3D(n, box)};
        toReference(*p, solver.parameters());
        auto backend = std::make_shared<vapor_b200::StageBackend>();
        Counts c;
        if (cuda_projection) solver.setPressureSolver(std::make_unique<CountingProjection>(backend, &c));
        if (cuda_advection) solver.setAdvection(std::make_unique<CountingAdvection>(backend, &c));
        solver.resetState();
        for (int f = 0; f < frames; ++f) solver.advance(dt);
        const auto& s = solver.state();
        std::copy(s.density().begin(), s.density().end(), d);
        std::copy(s.velocityX().begin(), s.velocityX().end(), u);
        std::copy(s.velocityY().begin(), s.velocityY().end(), v);
        std::copy(s.velocityZ().begin(), s.velocityZ().end(), w);
        if (counts) {
            counts[0] = c.projections;
            counts[1] = c.faces;
            counts[2] = c.scalars;
        }
        return 0;
    } catch (const std::invalid_argument&) {
        return VAPOR_INVALID_ARGUMENT;
    } catch (...) {
        return VAPOR_RUNTIME_ERROR;
    }
}

// The C++ resident wrapper: construct, advance `frames` steps, download.
HX int harness_resident_cpp(int n, float box, const vapor_mac3d_params* p, int frames, float dt, float* d, float* u,
                            float* v, float* w, unsigned long long* uploaded, unsigned long long* downloaded) {
    try {
        vapor_b200::CudaMacSimulation3D sim(n, box, *p);
        for (int f = 0; f < frames; ++f) sim.advance(dt);
        vapor_b200::HostState s(n, box);
        sim.download(s);
        std::copy(s.density.begin(), s.density.end(), d);
        std::copy(s.u.begin(), s.u.end(), u);
        std::copy(s.v.begin(), s.v.end(), v);
        std::copy(s.w.begin(), s.w.end(), w);
        *uploaded = sim.uploadedBytes();
        *downloaded = sim.downloadedBytes();
        return 0;
    } catch (const std::invalid_argument&) {
        return VAPOR_INVALID_ARGUMENT;
    } catch (...) {
        return VAPOR_RUNTIME_ERROR;
    }
}
