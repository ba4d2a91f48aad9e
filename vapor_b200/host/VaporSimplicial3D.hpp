// Drop-in CUDA compute backend for the reference's simplicial 3D solver.
//
// The reference's SimplicialFluidSolver3D takes an optional compute backend
// through setComputeBackend(SimplicialCompute3D*)
// (src/solvers/simplicial3d/SimplicialCompute3D.hpp:7-13,
// SimplicialFluidSolver3D.hpp:34) and ships an OpenGL one, GpuSimplicial3D
// (gpu/GpuSimplicial3D.hpp), which the solver, the mesh and the dual declare
// a friend so that it can read their flattened structure. This header
// defines a class of that name with that public interface (initialize,
// advectCirculation, advectDensity, recover, device) on the CUDA stages of
// include/vapor_b200.h (vapor_simplicial3d_*): a build compiles this header
// in place of gpu/GpuSimplicial3D.cpp and needs no OpenGL context.
//
// initialize() flattens the mesh, the dual and the interpolation structure
// into vapor_simplicial3d_mesh (once per mesh and size); each stage call
// passes the solver's current dual velocities, subdivision samples and
// vertex smoke. Status codes become the reference's exception types.
//
// Header-only; include after the reference's solver headers are on the
// include path; link against vapor_b200/_lib/libvapor_b200.so.
#pragma once

#include <cmath>
#include <cstdint>
#include <span>
#include <string>
#include <vector>

#include "solvers/simplicial3d/SimplicialCompute3D.hpp"
#include "solvers/simplicial3d/SimplicialFluidSolver3D.hpp"
#include "vapor_b200.hpp"

namespace vapor_b200 {

// The flattened arrays behind a vapor_simplicial3d_mesh (whose pointers
// point into them: movable, not copyable).
struct SimplicialPacked {
    SimplicialPacked() = default;
    SimplicialPacked(const SimplicialPacked&) = delete;
    SimplicialPacked& operator=(const SimplicialPacked&) = delete;
    SimplicialPacked(SimplicialPacked&&) = default;
    SimplicialPacked& operator=(SimplicialPacked&&) = default;
    vapor_simplicial3d_mesh mesh{};
    std::vector<double> dual_position, node_position, tet_geometry, wall_geometry, box_planes, sub_gradients;
    std::vector<double> star0, star1, star2;
    std::vector<int32_t> tet_vertices, dual_hint, primal_hint, bin_offsets, bin_items, wall_offsets, wall_items,
        wall_owner, cell_corners, corner_vertices, corner_cones, cone_planes, neighbor_offsets, neighbors,
        sub_offsets, sub_nodes, loop_offsets, loop_items, dual_edges, face_edges, face_signs, edge_vertices;
    std::vector<uint8_t> edge_boundary, vertex_boundary;
    std::vector<double> jacobi, ic_values, ic_diagonal;
    std::vector<int32_t> ic_offsets, ic_columns;
};

}  // namespace vapor_b200

class GpuSimplicial3D final : public SimplicialCompute3D {
public:
    // site_search: 0 automatic, 1 scan of all sites, 2 descent; dot_order: 0
    // automatic, 1 index order, 2 tree; preconditioner: 0 the CPU solver's,
    // 1 Jacobi (vapor_simplicial3d_create).
    explicit GpuSimplicial3D(int site_search = 0, int dot_order = 0, int preconditioner = 0)
        : search_(site_search), dots_(dot_order), precond_(preconditioner) {}
    ~GpuSimplicial3D() override { release(); }
    GpuSimplicial3D(const GpuSimplicial3D&) = delete;
    GpuSimplicial3D& operator=(const GpuSimplicial3D&) = delete;

    void initialize(const SimplicialFluidSolver3D& solver) {
        const auto& mesh = solver.mesh_;
        if (stages_ && key_ == mesh.tets.data() && size_ == mesh.size) return;
        release();
        packSolver(solver, packed_);
        vapor_b200::check(vapor_simplicial3d_create(&packed_.mesh, search_, dots_, precond_, &stages_));
        key_ = mesh.tets.data();
        size_ = mesh.size;
    }

    void advectCirculation(const SimplicialFluidSolver3D& solver, double dt, std::vector<double>& omega) override {
        initialize(solver);
        omega.resize(solver.mesh_.edges.size());
        vapor_b200::check(vapor_simplicial3d_advect_circulation(stages_, dt, velocities(solver), samples(solver),
                                                                omega.data()));
    }

    void advectDensity(const SimplicialFluidSolver3D& solver, double dt, std::vector<float>& density) override {
        initialize(solver);
        density.resize(solver.vertexDensity_.size());
        const double decay = std::exp(-solver.parameters_.smokeDecay * dt);
        vapor_b200::check(vapor_simplicial3d_advect_density(stages_, dt, decay, velocities(solver), samples(solver),
                                                            solver.vertexDensity_.data(), density.data()));
    }

    LinearSolveResult recover(const SimplicialFluidSolver3D& solver, std::span<const double> rhs,
                              std::vector<double>& x) override {
        initialize(solver);
        const auto& p = solver.parameters_;
        if (rhs.size() != solver.mesh_.edges.size()) throw std::invalid_argument("GPU CG RHS size mismatch");
        x.resize(rhs.size());
        // the CPU solver's start: zero on boxes, the current potential elsewhere
        const std::vector<double> zero(solver.mesh_.boxDomain ? rhs.size() : 0, 0.0);
        const double* x0 = solver.mesh_.boxDomain ? zero.data() : solver.phi_.data();
        vapor_linear_solve_result r{};
        vapor_b200::check(vapor_simplicial3d_recover(stages_, rhs.data(), x0, p.cgIterations, p.cgAbsoluteTolerance,
                                                     p.cgRelativeTolerance, x.data(), &r));
        LinearSolveResult result;
        result.iterations = r.iterations;
        result.converged = r.converged != 0;
        result.initialResidual = r.initial_residual;
        result.finalResidual = r.final_residual;
        return result;
    }

    const std::string& device() const { return device_; }

    // The solver's current dual velocities and (general domains) subdivision
    // samples, as the stage calls take them.
    static const double* velocities(const SimplicialFluidSolver3D& solver) {
        return reinterpret_cast<const double*>(solver.dualVelocity_.data());
    }
    static const double* samples(const SimplicialFluidSolver3D& solver) {
        return solver.mesh_.boxDomain ? nullptr : reinterpret_cast<const double*>(solver.dual_.samples_.data());
    }

    // Flattens the solver's mesh, dual and interpolation structure.
    static void packSolver(const SimplicialFluidSolver3D& solver, vapor_b200::SimplicialPacked& k) {
        const auto& mesh = solver.mesh_;
        const auto& dual = solver.dual_;
        k = vapor_b200::SimplicialPacked{};
        if (mesh.boxDomain && dual.cells.size() != mesh.vertices.size())
            throw std::invalid_argument("Box dual needs one Voronoi cell per vertex");
        auto put = [](std::vector<double>& a, Point p) { a.insert(a.end(), {p.x, p.y, p.z}); };
        for (const auto& d : dual.vertices) put(k.dual_position, d.position);
        if (mesh.boxDomain)
            for (const auto& p : mesh.vertices) put(k.node_position, p);
        else
            for (const auto& node : dual.nodes_) put(k.node_position, node.position);
        for (const auto& t : mesh.tets) {
            put(k.tet_geometry, mesh.vertices[t.vertices[0]]);
            for (int c = 1; c < 4; ++c) put(k.tet_geometry, t.gradients[c]);
            k.tet_vertices.insert(k.tet_vertices.end(), t.vertices.begin(), t.vertices.end());
        }
        // hints: the tet of each sample's start
        if (mesh.boxDomain) {
            for (const auto& d : dual.vertices) k.dual_hint.push_back(mesh.locate(d.position, d.tet));
            k.primal_hint.assign(mesh.vertices.size(), -1);
            for (int t = 0; t < int(mesh.tets.size()); ++t)
                for (int v : mesh.tets[t].vertices) k.primal_hint[v] = t;
        } else {
            k.dual_hint.assign(solver.dualTets_.begin(), solver.dualTets_.end());
            k.primal_hint.assign(solver.primalTets_.begin(), solver.primalTets_.end());
        }
        // spatial bins of tets and of boundary faces
        auto flatten = [](const std::vector<std::vector<int>>& lists, std::vector<int32_t>& off,
                          std::vector<int32_t>& items) {
            off.assign(1, 0);
            for (const auto& l : lists) {
                items.insert(items.end(), l.begin(), l.end());
                off.push_back(int32_t(items.size()));
            }
        };
        if (mesh.binsPerAxis_ > 0) {
            flatten(mesh.bins_, k.bin_offsets, k.bin_items);
            flatten(mesh.boundaryBins_, k.wall_offsets, k.wall_items);
        } else {
            k.bin_offsets = {0, 0};
            std::vector<int> all;
            for (int f = 0; f < int(mesh.faces.size()); ++f)
                if (mesh.faces[f].boundary()) all.push_back(f);
            flatten({all}, k.wall_offsets, k.wall_items);
        }
        for (const auto& f : mesh.faces) {
            const bool inner0 = f.tets[0] >= 0;
            put(k.wall_geometry, f.areaNormal * (inner0 ? 1. : -1.));
            put(k.wall_geometry, mesh.vertices[f.vertices[0]]);
            k.wall_owner.push_back(inner0 ? f.tets[0] : f.tets[1]);
        }
        if (mesh.boxDomain) {
            // Voronoi cells: planes (global numbering), corners with their cones,
            // and each site's Delaunay neighbours (the far ends of its edges)
            k.cell_corners.push_back(0);
            k.corner_cones.push_back(0);
            k.neighbor_offsets.push_back(0);
            int plane_base = 0;
            for (int site = 0; site < int(dual.cells.size()); ++site) {
                const auto& cell = dual.cells[site];
                for (const auto& plane : cell.planes) {
                    put(k.box_planes, plane.normal);
                    k.box_planes.push_back(plane.offset);
                    if (plane.primalEdge >= 0) {
                        const auto ends = mesh.edges[plane.primalEdge].vertices;
                        k.neighbors.push_back(ends[0] == site ? ends[1] : ends[0]);
                    }
                }
                k.neighbor_offsets.push_back(int32_t(k.neighbors.size()));
                for (const auto& corner : cell.corners) {
                    k.corner_vertices.push_back(corner.vertex);
                    for (const auto& cone : corner.cones)
                        for (int p : cone) k.cone_planes.push_back(plane_base + p);
                    k.corner_cones.push_back(int32_t(k.cone_planes.size() / 3));
                }
                k.cell_corners.push_back(int32_t(k.corner_vertices.size()));
                plane_base += int(cell.planes.size());
            }
        } else {
            k.sub_offsets.push_back(0);
            for (const auto& subs : dual.subdivisions_) {
                for (const auto& sub : subs) {
                    k.sub_nodes.insert(k.sub_nodes.end(), sub.nodes.begin(), sub.nodes.end());
                    for (const auto& g : sub.gradients) put(k.sub_gradients, g);
                }
                k.sub_offsets.push_back(int32_t(k.sub_nodes.size() / 4));
            }
        }
        k.loop_offsets.push_back(0);
        for (const auto& loop : dual.loops) {
            for (const auto& side : loop) k.loop_items.push_back(side.sign * (side.edge + 1));
            k.loop_offsets.push_back(int32_t(k.loop_items.size()));
        }
        for (const auto& e : dual.edges) k.dual_edges.insert(k.dual_edges.end(), {e.a, e.b});
        // the operator's ingredients
        for (const auto& f : mesh.faces) {
            k.face_edges.insert(k.face_edges.end(), f.edges.begin(), f.edges.end());
            k.face_signs.insert(k.face_signs.end(), f.signs.begin(), f.signs.end());
        }
        for (const auto& e : mesh.edges) {
            k.edge_vertices.insert(k.edge_vertices.end(), e.vertices.begin(), e.vertices.end());
            k.edge_boundary.push_back(e.boundary ? 1 : 0);
        }
        for (bool b : mesh.boundaryVertices) k.vertex_boundary.push_back(b ? 1 : 0);
        k.star0 = mesh.star0;
        k.star1 = mesh.star1;
        k.star2 = mesh.star2;
        // the CPU solver's preconditioner: its diagonal, and its IC(0) factor
        // when it built one
        k.jacobi = solver.diagonal_;
        if (!solver.incompleteLower_.empty()) {
            k.ic_offsets.push_back(0);
            for (const auto& row : solver.incompleteLower_) {
                for (const auto& [j, value] : row) {
                    k.ic_columns.push_back(j);
                    k.ic_values.push_back(value);
                }
                k.ic_offsets.push_back(int32_t(k.ic_columns.size()));
            }
            k.ic_diagonal = solver.incompleteDiagonal_;
        }

        auto& m = k.mesh;
        m.box_domain = mesh.boxDomain ? 1 : 0;
        m.bins = mesh.binsPerAxis_;
        m.size = mesh.size;
        m.n_primal = int32_t(mesh.vertices.size());
        m.n_dual = int32_t(dual.vertices.size());
        m.n_nodes = int32_t(k.node_position.size() / 3);
        m.n_edges = int32_t(mesh.edges.size());
        m.n_dual_edges = int32_t(dual.edges.size());
        m.n_tets = int32_t(mesh.tets.size());
        m.n_faces = int32_t(mesh.faces.size());
        m.n_planes = int32_t(k.box_planes.size() / 4);
        m.n_corners = int32_t(k.corner_vertices.size());
        m.n_cones = int32_t(k.cone_planes.size() / 3);
        m.n_subtets = int32_t(k.sub_nodes.size() / 4);
        m.dual_position = k.dual_position.data();
        m.node_position = k.node_position.data();
        m.tet_geometry = k.tet_geometry.data();
        m.tet_vertices = k.tet_vertices.data();
        m.dual_hint = k.dual_hint.data();
        m.primal_hint = k.primal_hint.data();
        m.bin_offsets = k.bin_offsets.data();
        m.bin_items = k.bin_items.data();
        m.wall_offsets = k.wall_offsets.data();
        m.wall_items = k.wall_items.data();
        m.wall_geometry = k.wall_geometry.data();
        m.wall_owner = k.wall_owner.data();
        m.box_planes = k.box_planes.data();
        m.cell_corners = k.cell_corners.data();
        m.corner_vertices = k.corner_vertices.data();
        m.corner_cones = k.corner_cones.data();
        m.cone_planes = k.cone_planes.data();
        m.neighbor_offsets = k.neighbor_offsets.data();
        m.neighbors = k.neighbors.data();
        m.sub_offsets = k.sub_offsets.data();
        m.sub_nodes = k.sub_nodes.data();
        m.sub_gradients = k.sub_gradients.data();
        m.loop_offsets = k.loop_offsets.data();
        m.loop_items = k.loop_items.data();
        m.dual_edges = k.dual_edges.data();
        m.face_edges = k.face_edges.data();
        m.face_signs = k.face_signs.data();
        m.edge_vertices = k.edge_vertices.data();
        m.edge_boundary = k.edge_boundary.data();
        m.vertex_boundary = k.vertex_boundary.data();
        m.star0 = k.star0.data();
        m.star1 = k.star1.data();
        m.star2 = k.star2.data();
        m.jacobi_diagonal = k.jacobi.size() == mesh.edges.size() ? k.jacobi.data() : nullptr;
        m.ic_offsets = k.ic_offsets.empty() ? nullptr : k.ic_offsets.data();
        m.ic_columns = k.ic_columns.data();
        m.ic_values = k.ic_values.data();
        m.ic_diagonal = k.ic_diagonal.data();
    }

private:
    using Point = simplicial3d::Point;
    static_assert(sizeof(Point) == 3 * sizeof(double), "Point must be three packed doubles");

    void release() {
        if (stages_) vapor_simplicial3d_destroy(stages_);
        stages_ = nullptr;
    }

    int search_ = 0;
    int dots_ = 0;
    int precond_ = 0;
    vapor_simplicial3d* stages_ = nullptr;
    const void* key_ = nullptr;
    double size_ = 0;
    vapor_b200::SimplicialPacked packed_;
    std::string device_ = "CUDA sm_100a (vapor_b200)";
};
