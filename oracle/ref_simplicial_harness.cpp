// TEST INFRASTRUCTURE — drives the reference's own simplicial 3D solver
// (taehwann/vapor src/solvers/simplicial3d/*.cpp, compiled from its sources by
// oracle/Makefile into _ref/libvapor_ref_simplicial.so) with the product's
// drop-in compute backend (vapor_b200/host/VaporSimplicial3D.hpp) installed
// through setComputeBackend, as the reference's tests/SimplicialGpu3DTests.cpp
// does with its OpenGL backend. Backends a solver can take:
//   0  none: the reference's CPU path
//   1  the CUDA stages (advection and recovery)
//   2  the stages' arithmetic (vapor_b200/csrc/simplicial_math.cuh) compiled
//      for the host, box meshes, no GPU; recovery copied from a partner
//      solver on the CPU path that was stepped first
//   3  the CUDA advection stages with the partner's recovery
// Modes 2 and 3 isolate the advection: with the partner's recovery, every
// field of the two solvers must stay bit-identical step after step.
// Only tests/ load this library.

#include <array>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "VaporSimplicial3D.hpp"
#include "simplicial_math.cuh"

#define HX extern "C" __attribute__((visibility("default")))

namespace {

std::string g_error;

vb::simplicial::View host_view(const vapor_b200::SimplicialPacked& k, int search) {
    vb::simplicial::View v{};
    const auto& m = k.mesh;
    v.box = m.box_domain;
    v.search = search;
    v.size = m.size;
    v.n_primal = m.n_primal;
    v.n_dual = m.n_dual;
    v.n_nodes = m.n_nodes;
    v.n_edges = m.n_edges;
    v.n_dual_edges = m.n_dual_edges;
    v.n_tets = m.n_tets;
    v.bins = m.bins;
    v.dual_position = m.dual_position;
    v.node_position = m.node_position;
    v.tet_geometry = m.tet_geometry;
    v.tet_vertices = m.tet_vertices;
    v.dual_hint = m.dual_hint;
    v.primal_hint = m.primal_hint;
    v.bin_offsets = m.bin_offsets;
    v.bin_items = m.bin_items;
    v.wall_offsets = m.wall_offsets;
    v.wall_items = m.wall_items;
    v.wall_geometry = m.wall_geometry;
    v.wall_owner = m.wall_owner;
    v.box_planes = m.box_planes;
    v.cell_corners = m.cell_corners;
    v.corner_vertices = m.corner_vertices;
    v.corner_cones = m.corner_cones;
    v.cone_planes = m.cone_planes;
    v.neighbor_offsets = m.neighbor_offsets;
    v.neighbors = m.neighbors;
    v.sub_offsets = m.sub_offsets;
    v.sub_nodes = m.sub_nodes;
    v.sub_gradients = m.sub_gradients;
    v.loop_offsets = m.loop_offsets;
    v.loop_items = m.loop_items;
    v.dual_edges = m.dual_edges;
    return v;
}

struct Solver;

// Recovery copied from the partner (stepped first on the CPU path).
LinearSolveResult partner_recovery(const Solver& partner, std::vector<double>& x);

// The stages' arithmetic on the host (mode 2).
class HostStages final : public SimplicialCompute3D {
public:
    HostStages(const Solver* partner, int search) : partner_(partner), search_(search) {}
    void advectCirculation(const SimplicialFluidSolver3D& s, double dt, std::vector<double>& omega) override {
        prepare(s);
        const auto v = host_view(packed_, search_);
        std::vector<double> traced(3 * size_t(v.n_dual)), velocity(traced.size()), integral(v.n_dual_edges);
        int error = 0;
        for (int i = 0; i < v.n_dual; ++i) {
            vb::simplicial::P3 t, u;
            vb::simplicial::trace_dual(v, i, dt, GpuSimplicial3D::velocities(s), GpuSimplicial3D::samples(s), &t,
                                       &u, &error);
            std::memcpy(&traced[3 * size_t(i)], &t, sizeof t);
            std::memcpy(&velocity[3 * size_t(i)], &u, sizeof u);
        }
        if (error) throw std::runtime_error("host stages: sampling error " + std::to_string(error));
        for (int j = 0; j < v.n_dual_edges; ++j)
            integral[j] = vb::simplicial::edge_integral(v, j, traced.data(), velocity.data());
        omega.resize(v.n_edges);
        for (int e = 0; e < v.n_edges; ++e) omega[e] = vb::simplicial::circulation(v, e, integral.data());
    }
    void advectDensity(const SimplicialFluidSolver3D& s, double dt, std::vector<float>& density) override {
        prepare(s);
        const auto v = host_view(packed_, search_);
        const double decay = std::exp(-s.parameters().smokeDecay * dt);
        density.resize(v.n_primal);
        int error = 0;
        for (int i = 0; i < v.n_primal; ++i)
            density[i] = vb::simplicial::trace_density(v, i, dt, decay, GpuSimplicial3D::velocities(s),
                                                       GpuSimplicial3D::samples(s), s.vertexDensity().data(), &error);
        if (error) throw std::runtime_error("host stages: sampling error " + std::to_string(error));
    }
    LinearSolveResult recover(const SimplicialFluidSolver3D&, std::span<const double>, std::vector<double>& x) override {
        return partner_recovery(*partner_, x);
    }

private:
    void prepare(const SimplicialFluidSolver3D& s) {
        if (key_ == s.domain().tets.data() && size_ == s.domain().size) return;
        GpuSimplicial3D::packSolver(s, packed_);
        key_ = s.domain().tets.data();
        size_ = s.domain().size;
    }
    const Solver* partner_;
    int search_;
    vapor_b200::SimplicialPacked packed_;
    const void* key_ = nullptr;
    double size_ = 0;
};

// The CUDA advection stages with the partner's recovery (mode 3).
class DeviceAdvection final : public SimplicialCompute3D {
public:
    DeviceAdvection(const Solver* partner, int search) : partner_(partner), gpu_(search) {}
    void advectCirculation(const SimplicialFluidSolver3D& s, double dt, std::vector<double>& omega) override {
        gpu_.advectCirculation(s, dt, omega);
    }
    void advectDensity(const SimplicialFluidSolver3D& s, double dt, std::vector<float>& density) override {
        gpu_.advectDensity(s, dt, density);
    }
    LinearSolveResult recover(const SimplicialFluidSolver3D&, std::span<const double>, std::vector<double>& x) override {
        return partner_recovery(*partner_, x);
    }

private:
    const Solver* partner_;
    GpuSimplicial3D gpu_;
};

struct Solver {
    std::unique_ptr<SimplicialFluidSolver3D> solver;
    std::unique_ptr<SimplicialCompute3D> backend;
};

LinearSolveResult partner_recovery(const Solver& partner, std::vector<double>& x) {
    x = partner.solver->potential();
    return partner.solver->lastRecovery();
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return 1;
    }
}

Solver& S(void* h) { return *static_cast<Solver*>(h); }

}  // namespace

HX const char* rs_error() { return g_error.c_str(); }

// The VAPOR_TET file read with stdio (the reference's std::ifstream reader,
// Mesh::loadDomain, faults in this toolchain's istream once the host process
// has loaded numpy), then built as loadBox / loadDomain build it: the
// public constructor on unit-box coordinates, then scaledBox(size), which
// multiplies by size / 1 (the same bits as loadDomain's p * size) and builds
// the spatial bins. loadBox's fill and boundary checks are not repeated.
simplicial3d::Mesh read_mesh(const char* path, bool box, double size) {
    FILE* f = std::fopen(path, "r");
    if (!f) throw std::invalid_argument(std::string("Cannot open ") + path);
    char magic[16] = {0};
    int version = 0, nv = 0, nt = 0;
    bool ok = std::fscanf(f, "%15s %d %d %d", magic, &version, &nv, &nt) == 4 &&
              std::string(magic) == "VAPOR_TET" && version == 1 && nv >= 4 && nt >= 1;
    std::vector<simplicial3d::Point> v(ok ? nv : 0);
    std::vector<std::array<int, 4>> cells(ok ? nt : 0);
    for (auto& p : v) ok = ok && std::fscanf(f, "%lf %lf %lf", &p.x, &p.y, &p.z) == 3;
    for (auto& t : cells) ok = ok && std::fscanf(f, "%d %d %d %d", &t[0], &t[1], &t[2], &t[3]) == 4;
    std::fclose(f);
    if (!ok) throw std::invalid_argument(std::string("Cannot read VAPOR_TET mesh: ") + path);
    simplicial3d::Mesh unit(std::move(v), std::move(cells));
    unit.size = 1;
    unit.boxDomain = box;
    return unit.scaledBox(size);
}

// A CPU solver on a VAPOR_TET mesh (box or general domain, scaled to size).
// Null on the reference's exception.
HX void* rs_create(const char* path, int box, double size) {
    Solver* out = nullptr;
    guarded([&] {
        auto mesh = read_mesh(path, box != 0, size);
        auto s = std::make_unique<Solver>();
        s->solver = std::make_unique<SimplicialFluidSolver3D>(std::move(mesh));
        out = s.release();
    });
    return out;
}
HX void rs_destroy(void* h) { delete static_cast<Solver*>(h); }

// Installs backend `mode` (see the header) with nearest-site search `search`
// and the recovery's dot-product order `dot_order` and preconditioner
// (vapor_simplicial3d_create).
HX int rs_attach(void* h, int mode, int search, int dot_order, int preconditioner, void* partner) {
    return guarded([&] {
        Solver& s = S(h);
        s.solver->setComputeBackend(nullptr);
        s.backend.reset();
        if (mode == 1) {
            auto gpu = std::make_unique<GpuSimplicial3D>(search, dot_order, preconditioner);
            gpu->initialize(*s.solver);
            s.backend = std::move(gpu);
        } else if (mode == 2) {
            s.backend = std::make_unique<HostStages>(static_cast<Solver*>(partner), search == 2 ? 1 : 0);
        } else if (mode == 3) {
            s.backend = std::make_unique<DeviceAdvection>(static_cast<Solver*>(partner), search);
        }
        s.solver->setComputeBackend(s.backend.get());
    });
}

// counts: vertices, edges, faces, tets, dual vertices
HX void rs_counts(void* h, int* out) {
    const auto& s = *S(h).solver;
    out[0] = int(s.domain().vertices.size());
    out[1] = int(s.domain().edges.size());
    out[2] = int(s.domain().faces.size());
    out[3] = int(s.domain().tets.size());
    out[4] = int(s.dual().vertices.size());
}

HX int rs_set_potential(void* h, const double* phi) {
    return guarded([&] {
        auto& s = *S(h).solver;
        s.setPotential(std::span<const double>(phi, s.domain().edges.size()));
    });
}
HX int rs_advect_vorticity(void* h, double dt) {
    return guarded([&] { S(h).solver->advectVorticity(dt); });
}
HX int rs_advance(void* h, float dt) {
    return guarded([&] { S(h).solver->advance(dt); });
}
HX int rs_set_box_size(void* h, float size) {
    return guarded([&] { S(h).solver->setBoxSize(size); });
}
HX int rs_reset(void* h) {
    return guarded([&] { S(h).solver->resetState(); });
}
// Parameters: emitter on/off, smoke decay, CG iteration cap and tolerances.
HX void rs_set_parameters(void* h, int emitter, float decay, int cg_iterations, double abs_tol, double rel_tol) {
    auto& p = S(h).solver->parameters();
    p.emitterEnabled = emitter != 0;
    p.smokeDecay = decay;
    p.cgIterations = cg_iterations;
    p.cgAbsoluteTolerance = abs_tol;
    p.cgRelativeTolerance = rel_tol;
}

HX void rs_vorticity(void* h, double* out) {
    const auto& v = S(h).solver->vorticity();
    std::copy(v.begin(), v.end(), out);
}
HX void rs_potential(void* h, double* out) {
    const auto& v = S(h).solver->potential();
    std::copy(v.begin(), v.end(), out);
}
HX void rs_flux(void* h, double* out) {
    const auto& v = S(h).solver->flux();
    std::copy(v.begin(), v.end(), out);
}
HX void rs_vertex_density(void* h, float* out) {
    const auto& v = S(h).solver->vertexDensity();
    std::copy(v.begin(), v.end(), out);
}
// Tet smoke (reconstructed from the vertex smoke).
HX void rs_density(void* h, float* out) {
    const auto& v = S(h).solver->density();
    std::copy(v.begin(), v.end(), out);
}
HX void rs_edge_midpoints(void* h, double* out) {
    const auto& m = S(h).solver->domain();
    for (size_t e = 0; e < m.edges.size(); ++e) {
        const auto a = m.vertices[m.edges[e].vertices[0]], b = m.vertices[m.edges[e].vertices[1]];
        out[6 * e] = a.x;
        out[6 * e + 1] = a.y;
        out[6 * e + 2] = a.z;
        out[6 * e + 3] = b.x;
        out[6 * e + 4] = b.y;
        out[6 * e + 5] = b.z;
    }
}
// maxDivergence, maxBoundaryFlux, kineticEnergy, maxSpeed, recoveryCurlError, smokeMass
HX void rs_diagnostics(void* h, double* out) {
    const auto d = S(h).solver->diagnostics();
    out[0] = d.maxDivergence;
    out[1] = d.maxBoundaryFlux;
    out[2] = d.kineticEnergy;
    out[3] = d.maxSpeed;
    out[4] = d.recoveryCurlError;
    out[5] = d.smokeMass;
}
HX void rs_last_recovery(void* h, int* iterations, int* converged, double* initial, double* final_residual) {
    const auto& r = S(h).solver->lastRecovery();
    *iterations = r.iterations;
    *converged = r.converged ? 1 : 0;
    *initial = r.initialResidual;
    *final_residual = r.finalResidual;
}
// The smoke's centre height and mass (SimplicialGpu3DTests.cpp's smokeCenter):
// tet smoke times volume, its height from the four vertices' mean z.
HX void rs_smoke_center(void* h, double* out) {
    const auto& s = *S(h).solver;
    double mass = 0, height = 0;
    for (size_t i = 0; i < s.domain().tets.size(); ++i) {
        const auto& tet = s.domain().tets[i];
        const double amount = s.density()[i] * tet.volume;
        mass += amount;
        for (int v : tet.vertices) height += .25 * amount * s.domain().vertices[v].z;
    }
    out[0] = mass > 0 ? height / mass : 0;
    out[1] = mass;
}
// CFL substeps of the last advance (SimplicialTimings3D::substeps).
HX int rs_substeps(void* h) { return S(h).solver->timings().substeps; }
// Dependency levels of the forward solve of the solver's IC(0) factor (0
// when it has none): the sequential steps of the preconditioner on a GPU.
HX int rs_ic_levels(void* h) {
    vapor_b200::SimplicialPacked k;
    GpuSimplicial3D::packSolver(*S(h).solver, k);
    if (k.ic_offsets.empty()) return 0;
    const int n = int(k.ic_offsets.size()) - 1;
    std::vector<int> level(n, 0);
    int levels = 0;
    for (int i = 0; i < n; ++i) {
        int l = 0;
        for (int j = k.ic_offsets[i]; j < k.ic_offsets[i + 1]; ++j) l = std::max(l, level[k.ic_columns[j]] + 1);
        level[i] = l;
        levels = std::max(levels, l + 1);
    }
    return levels;
}
// The rotating stir force and the emitter position/strength/radius.
HX void rs_set_stir(void* h, float strength, float radius, float frequency) {
    auto& p = S(h).solver->parameters();
    p.stirStrength = strength;
    p.stirRadius = radius;
    p.stirFrequency = frequency;
}
HX void rs_set_emitter(void* h, float x, float y, float z, float strength, float radius, float buoyancy) {
    auto& p = S(h).solver->parameters();
    p.emitterX = x;
    p.emitterY = y;
    p.emitterZ = z;
    p.sourceStrength = strength;
    p.emitterRadius = radius;
    p.buoyancy = buoyancy;
}
