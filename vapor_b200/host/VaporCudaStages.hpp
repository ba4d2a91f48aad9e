// Drop-in CUDA stage plugins for the reference's MAC 3D coordinator.
//
// Include this header from inside a taehwann/vapor source tree (it includes
// the reference's own interface headers) and install the stages with the
// reference's plugin hooks:
//
//   solver.setPressureSolver(std::make_unique<vapor_b200::CudaProjection3D>());
//   solver.setAdvection(std::make_unique<vapor_b200::CudaAdvection3D>());
//
// CudaProjection3D implements Projection3D (src/solvers/mac3d/Projection3D.hpp:6-11)
// and CudaAdvection3D implements Advection3D (src/solvers/mac3d/Advection3D.hpp:6-14),
// the two virtual stage interfaces MacGridFluidSolver3D dispatches through
// (MacGridFluidSolver3D.cpp:82-138). They take the place of the reference's
// OpenGL adapters GpuPressureSolver / GpuAdvection: each call copies its host
// spans to the device, runs the sm_100a kernels and copies back. Results are
// bit-identical to the reference's CPU stages (CpuPressureSolver3D with the
// same diagonal floor, CpuAdvection).
#pragma once

#include <memory>
#include <stdexcept>

#include "solvers/mac3d/Advection3D.hpp"
#include "solvers/mac3d/MacGridState3D.hpp"
#include "solvers/mac3d/Projection3D.hpp"
#include "vapor_b200.hpp"

namespace vapor_b200 {

// One device workspace, rebuilt when the grid changes (the reference's
// GpuMacBackend::validateGrid role).
class StageBackend {
public:
    StageBackend() = default;
    ~StageBackend() { release(); }
    StageBackend(const StageBackend&) = delete;
    StageBackend& operator=(const StageBackend&) = delete;
    vapor_stage* bind(const MacGridState3D& grid) {
        if (!stage_ || n_ != grid.resolution() || box_ != grid.boxSize()) {
            release();
            check(vapor_stage_create(grid.resolution(), grid.boxSize(), &stage_));
            n_ = grid.resolution();
            box_ = grid.boxSize();
        }
        return stage_;
    }
    void reset() {
        if (stage_) check(vapor_stage_reset(stage_));
    }

private:
    void release() {
        if (stage_) vapor_stage_destroy(stage_);
        stage_ = nullptr;
    }
    vapor_stage* stage_ = nullptr;
    int n_ = 0;
    float box_ = 0.f;
};

class CudaProjection3D final : public Projection3D {
public:
    // diagonalFloor 6 reproduces MacGridFluidSolver3D's own solver
    // (MacGridFluidSolver3D.hpp:118); 0 is CpuPressureSolver3D's default.
    explicit CudaProjection3D(float diagonalFloor = 6.f,
                              std::shared_ptr<StageBackend> backend = std::make_shared<StageBackend>())
        : floor_(diagonalFloor), backend_(std::move(backend)) {}

    ProjectionResult project(MacGridState3D& state, const ProjectionOptions& options) override {
        vapor_stage* stage = backend_->bind(state);
        vapor_projection_options o;
        o.dt = options.dt;
        o.relaxation = options.relaxation;
        o.linear_solve.max_iterations = options.linearSolve.maxIterations;
        o.linear_solve.residual_check_interval = options.linearSolve.residualCheckInterval;
        o.linear_solve.absolute_tolerance = options.linearSolve.absoluteTolerance;
        o.linear_solve.relative_tolerance = options.linearSolve.relativeTolerance;
        o.linear_solve.fixed_iterations = options.linearSolve.fixedIterations ? 1 : 0;
        o.linear_solve.reserved0 = 0;
        vapor_projection_result r;
        check(vapor_stage_project(stage, state.velocityX().data(), state.velocityY().data(),
                                  state.velocityZ().data(), &o, floor_, &r, nullptr));
        ProjectionResult out;
        out.linearSolve.iterations = r.linear_solve.iterations;
        out.linearSolve.initialResidual = r.linear_solve.initial_residual;
        out.linearSolve.finalResidual = r.linear_solve.final_residual;
        out.linearSolve.converged = r.linear_solve.converged != 0;
        out.residualAvailable = r.residual_available != 0;
        out.divergenceBefore = r.divergence_before;
        out.divergenceAfter = r.divergence_after;
        out.removedRhsMean = r.removed_rhs_mean;
        return out;
    }
    void reset() noexcept override {
        try {
            backend_->reset();
        } catch (...) {
        }
    }

private:
    float floor_;
    std::shared_ptr<StageBackend> backend_;
};

class CudaAdvection3D final : public Advection3D {
public:
    explicit CudaAdvection3D(std::shared_ptr<StageBackend> backend = std::make_shared<StageBackend>())
        : backend_(std::move(backend)) {}

    void advectScalar(const AdvectionContext& context, std::span<float> field, AdvectionWorkspace&,
                      AdvectionMethod method) const override {
        validateScalarAdvection(context, field);
        vapor_stage* stage = backend_->bind(context.grid);
        check(vapor_stage_advect_scalar(stage, context.dt, context.cflLimit,
                                        method == AdvectionMethod::MacCormack ? VAPOR_MACCORMACK
                                                                              : VAPOR_SEMI_LAGRANGIAN,
                                        field.data(), context.flow.x.data(), context.flow.y.data(),
                                        context.flow.z.data()));
    }
    void advectFace(const AdvectionContext& context, FaceAxis axis, std::span<const float> source,
                    std::span<float> output, AdvectionWorkspace&, AdvectionMethod method) const override {
        validateFaceAdvection(context, axis, source, output);
        vapor_stage* stage = backend_->bind(context.grid);
        check(vapor_stage_advect_face(stage, static_cast<int32_t>(axis), context.dt, context.cflLimit,
                                      method == AdvectionMethod::MacCormack ? VAPOR_MACCORMACK
                                                                            : VAPOR_SEMI_LAGRANGIAN,
                                      source.data(), context.flow.x.data(), context.flow.y.data(),
                                      context.flow.z.data(), output.data()));
    }

private:
    std::shared_ptr<StageBackend> backend_;
};

}  // namespace vapor_b200
