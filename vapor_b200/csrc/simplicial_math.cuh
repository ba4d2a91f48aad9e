// FP64 sampling and tracing on a tetrahedral mesh and its circumcentric dual:
// the arithmetic of the reference's simplicial 3D solver
// (src/solvers/simplicial3d/), evaluated per sample point by the device
// stages of simplicial3d.cu and, compiled for the host, by the oracle's
// check of those stages. Every expression keeps the reference's operation
// order (the library builds with --fmad=false), so a host build of these
// functions reproduces the reference's CPU results bit for bit.
//
//   barycentric / locate      Mesh::barycentric, Mesh::locate (SimplicialMesh3D.cpp:166-185)
//   clip_segment              Mesh::clipSegment (SimplicialMesh3D.cpp:186-214)
//   box_velocity              DualMesh::interpolate + coordinates on a box
//                             (SimplicialDual3D.cpp:124-160): nearest site, then
//                             the rational weights of its Voronoi cell
//   domain_velocity           DualMesh::interpolate on a general domain: the
//                             circumcentric subdivision of the located tet
//   trace_*                   SimplicialFluidSolver3D::trace and the per-sample
//                             loops of advectVorticity / advectAndDecaySmoke
//                             (SimplicialFluidSolver3D.cpp:418-450, 594-616)
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define VB_SX __host__ __device__ __forceinline__
#else
#define VB_SX inline
#endif

namespace vb {
namespace simplicial {

struct P3 {
    double x, y, z;
};
VB_SX P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
VB_SX P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
VB_SX P3 mul(P3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
VB_SX double dot(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
VB_SX P3 cross(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
VB_SX double length(P3 a) { return sqrt(dot(a, a)); }
VB_SX double max_d(double a, double b) { return a < b ? b : a; }  // std::max(a, b)
VB_SX double clamp_d(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
VB_SX int min_i(int a, int b) { return b < a ? b : a; }
VB_SX P3 load3(const double* a, long i) { return {a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }

// Error bits a stage reports (the reference throws at the same points).
enum : int { kEscapedSubdivision = 1, kInvalidWeights = 2 };

// The mesh, dual and interpolation structure, flattened (device or host
// pointers). Offsets arrays have one entry more than their owners.
struct View {
    int box;       // 1: box domain (Voronoi cells), 0: general domain (subdivision)
    int search;    // box nearest site: 0 scan of all sites, 1 descent over Delaunay neighbours
    double size;
    int n_primal, n_dual, n_nodes, n_edges, n_dual_edges, n_tets, bins;
    const double* dual_position;  // 3 per dual vertex
    const double* node_position;  // 3 per node (box: the primal vertices)
    const double* tet_geometry;   // 12 per tet: vertex 0, gradients of barycentric 1..3
    const int* tet_vertices;      // 4 per tet
    const int* dual_hint;         // tet per dual vertex (general domains; -1 none)
    const int* primal_hint;       // tet per primal vertex
    const int* bin_offsets;       // bins^3 + 1
    const int* bin_items;         // tets per bin
    const int* wall_offsets;      // bins^3 + 1
    const int* wall_items;        // boundary faces per bin
    const double* wall_geometry;  // 6 per face: outward-oriented area normal, its first vertex
    const int* wall_owner;        // the face's one tet
    // box
    const double* box_planes;     // 4 per plane: normal, offset
    const int* cell_corners;      // per site: range of corners
    const int* corner_vertices;   // dual vertex of each corner
    const int* corner_cones;      // per corner: range of cones
    const int* cone_planes;       // 3 global plane indices per cone
    const int* neighbor_offsets;  // per site: range of Delaunay neighbours
    const int* neighbors;
    // general domain
    const int* sub_offsets;       // per tet: range of subtets
    const int* sub_nodes;         // 4 per subtet
    const double* sub_gradients;  // 9 per subtet
    // circulation
    const int* loop_offsets;      // per primal edge: range of oriented dual edges
    const int* loop_items;        // sign * (dual edge + 1)
    const int* dual_edges;        // 2 per dual edge
};

VB_SX double min4(const double w[4]) {  // *std::min_element
    double m = w[0];
    for (int k = 1; k < 4; ++k)
        if (w[k] < m) m = w[k];
    return m;
}

VB_SX void barycentric(const View& v, int t, P3 p, double w[4]) {
    const double* g = v.tet_geometry + 12L * t;
    const P3 q = sub(p, P3{g[0], g[1], g[2]});
    w[1] = dot(P3{g[3], g[4], g[5]}, q);
    w[2] = dot(P3{g[6], g[7], g[8]}, q);
    w[3] = dot(P3{g[9], g[10], g[11]}, q);
    w[0] = 1 - w[1] - w[2] - w[3];
}

VB_SX int locate(const View& v, P3 p, int hint) {
    double w[4];
    if (hint >= 0 && hint < v.n_tets) {
        barycentric(v, hint, p, w);
        if (min4(w) >= -1e-9) return hint;
    }
    if (v.bins > 0) {
        if (p.x < 0 || p.y < 0 || p.z < 0 || p.x > v.size || p.y > v.size || p.z > v.size) return -1;
        const int n = v.bins;
        const int x = min_i(n - 1, int(p.x / v.size * n)), y = min_i(n - 1, int(p.y / v.size * n)),
                  z = min_i(n - 1, int(p.z / v.size * n));
        const int b = x + n * (y + n * z);
        for (int j = v.bin_offsets[b]; j < v.bin_offsets[b + 1]; ++j) {
            const int t = v.bin_items[j];
            barycentric(v, t, p, w);
            if (min4(w) >= -1e-9) return t;
        }
        return -1;
    }
    for (int k = 0; k < v.n_tets; ++k) {
        const int t = ((hint > 0 ? hint : 0) + k) % v.n_tets;
        barycentric(v, t, p, w);
        if (min4(w) >= -1e-9) return t;
    }
    return -1;
}

VB_SX int bin_of(const View& v, double x) {
    const int n = v.bins;
    const int b = int(x / v.size * n);
    return b < 0 ? 0 : (n - 1 < b ? n - 1 : b);
}

// First crossing of a boundary face by the segment, backed off by 1e-8.
VB_SX P3 clip_segment(const View& v, P3 start, P3 end, int hint) {
    double w[4];
    if (hint >= 0 && hint < v.n_tets) {
        double a[4], b[4];
        barycentric(v, hint, start, a);
        barycentric(v, hint, end, b);
        if (min4(a) >= -1e-10 && min4(b) >= -1e-10) return end;
    }
    const P3 delta = sub(end, start);
    if (length(delta) < 1e-14 * v.size) return start;
    double first = 1;
    auto inspect = [&](int f) {
        const double* g = v.wall_geometry + 6L * f;
        const P3 normal{g[0], g[1], g[2]};
        const double denominator = dot(normal, delta);
        if (denominator <= 1e-15 * length(normal) * length(delta)) return;
        const double hit = dot(normal, sub(P3{g[3], g[4], g[5]}, start)) / denominator;
        if (hit < -1e-9 || hit > first) return;
        barycentric(v, v.wall_owner[f], add(start, mul(delta, hit)), w);
        if (min4(w) < -1e-8) return;
        first = max_d(0., hit);
    };
    // wall_offsets / wall_items list every boundary face per bin; without bins
    // the one pseudo-bin lists them all
    if (v.bins > 0) {
        const int n = v.bins;
        for (int z = bin_of(v, start.z < end.z ? start.z : end.z); z <= bin_of(v, start.z < end.z ? end.z : start.z); ++z)
            for (int y = bin_of(v, start.y < end.y ? start.y : end.y);
                 y <= bin_of(v, start.y < end.y ? end.y : start.y); ++y)
                for (int x = bin_of(v, start.x < end.x ? start.x : end.x);
                     x <= bin_of(v, start.x < end.x ? end.x : start.x); ++x) {
                    const int b = x + n * (y + n * z);
                    for (int j = v.wall_offsets[b]; j < v.wall_offsets[b + 1]; ++j) inspect(v.wall_items[j]);
                }
    } else {
        for (int j = v.wall_offsets[0]; j < v.wall_offsets[1]; ++j) inspect(v.wall_items[j]);
    }
    return first < 1 ? add(start, mul(delta, max_d(0., first - 1e-8))) : end;
}

// Nearest primal vertex (Voronoi site) of p: the lowest index at the least
// squared distance, by a scan of all sites, or by descent over Delaunay
// neighbours from `start` (a Voronoi cell is the intersection of its
// neighbour bisectors, so a site with no closer neighbour is the nearest).
VB_SX int nearest_site(const View& v, P3 p, int start) {
    if (v.search == 0) {
        int site = 0;
        double distance = DBL_MAX;
        for (int i = 0; i < v.n_primal; ++i) {
            const P3 d = sub(p, load3(v.node_position, i));
            const double squared = dot(d, d);
            if (squared < distance) {
                site = i;
                distance = squared;
            }
        }
        return site;
    }
    int site = start;
    P3 d = sub(p, load3(v.node_position, site));
    double nearest = dot(d, d);
    for (int step = 0; step < v.n_primal; ++step) {
        int next = site;
        for (int j = v.neighbor_offsets[site]; j < v.neighbor_offsets[site + 1]; ++j) {
            const int other = v.neighbors[j];
            const P3 e = sub(p, load3(v.node_position, other));
            const double squared = dot(e, e);
            if (squared < nearest || (squared == nearest && other < next)) {
                nearest = squared;
                next = other;
            }
        }
        if (next == site) break;
        site = next;
    }
    return site;
}

// Generalised barycentric interpolation of the dual velocities in the
// Voronoi cell of the nearest site.
VB_SX P3 box_velocity(const View& v, P3 p, int start_site, const double* values, int* error) {
    const int site = nearest_site(v, p, start_site);
    const int c0 = v.cell_corners[site], c1 = v.cell_corners[site + 1];
    P3 value{0, 0, 0};
    for (int c = c0; c < c1; ++c)
        if (length(sub(load3(v.dual_position, v.corner_vertices[c]), p)) < 1e-12 * v.size) {
            // the point is this corner: weight 1 here, 0 elsewhere
            for (int k = c0; k < c1; ++k) value = add(value, mul(load3(values, v.corner_vertices[k]), k == c ? 1. : 0.));
            return value;
        }
    // The weights are normalised by their sum before the values are
    // accumulated, as coordinates() returns them.
    double sum = 0;
    for (int c = c0; c < c1; ++c) {
        double weight = 0;
        for (int k = v.corner_cones[c]; k < v.corner_cones[c + 1]; ++k) {
            const double* a = v.box_planes + 4L * v.cone_planes[3 * k];
            const double* b = v.box_planes + 4L * v.cone_planes[3 * k + 1];
            const double* cc = v.box_planes + 4L * v.cone_planes[3 * k + 2];
            const P3 na{a[0], a[1], a[2]}, nb{b[0], b[1], b[2]}, nc{cc[0], cc[1], cc[2]};
            const double da = max_d(1e-13 * v.size, a[3] - dot(na, p));
            const double db = max_d(1e-13 * v.size, b[3] - dot(nb, p));
            const double dc = max_d(1e-13 * v.size, cc[3] - dot(nc, p));
            weight += fabs(dot(na, cross(nb, nc))) / (da * db * dc);
        }
        sum += weight;
    }
    if (!(sum <= DBL_MAX) || sum <= 0) {  // not finite, or not positive
        *error |= kInvalidWeights;
        return P3{0, 0, 0};
    }
    for (int c = c0; c < c1; ++c) {
        double weight = 0;
        for (int k = v.corner_cones[c]; k < v.corner_cones[c + 1]; ++k) {
            const double* a = v.box_planes + 4L * v.cone_planes[3 * k];
            const double* b = v.box_planes + 4L * v.cone_planes[3 * k + 1];
            const double* cc = v.box_planes + 4L * v.cone_planes[3 * k + 2];
            const P3 na{a[0], a[1], a[2]}, nb{b[0], b[1], b[2]}, nc{cc[0], cc[1], cc[2]};
            const double da = max_d(1e-13 * v.size, a[3] - dot(na, p));
            const double db = max_d(1e-13 * v.size, b[3] - dot(nb, p));
            const double dc = max_d(1e-13 * v.size, cc[3] - dot(nc, p));
            weight += fabs(dot(na, cross(nb, nc))) / (da * db * dc);
        }
        value = add(value, mul(load3(values, v.corner_vertices[c]), weight / sum));
    }
    return value;
}

// Piecewise-linear interpolation of the node samples on the subdivision of
// the located tet; zero outside the domain.
VB_SX P3 domain_velocity(const View& v, P3 p, int hint, const double* samples, int* error) {
    const int t = locate(v, p, hint);
    if (t < 0) return P3{0, 0, 0};
    for (int s = v.sub_offsets[t]; s < v.sub_offsets[t + 1]; ++s) {
        const int* ids = v.sub_nodes + 4L * s;
        const double* g = v.sub_gradients + 9L * s;
        const P3 delta = sub(p, load3(v.node_position, ids[0]));
        double w[4];
        w[1] = dot(P3{g[0], g[1], g[2]}, delta);
        w[2] = dot(P3{g[3], g[4], g[5]}, delta);
        w[3] = dot(P3{g[6], g[7], g[8]}, delta);
        w[0] = 1 - w[1] - w[2] - w[3];
        if (min4(w) >= -1e-8) {
            P3 r{0, 0, 0};
            for (int k = 0; k < 4; ++k) r = add(r, mul(load3(samples, ids[k]), w[k]));
            return r;
        }
    }
    *error |= kEscapedSubdivision;
    return P3{0, 0, 0};
}

VB_SX P3 clip_box(const View& v, P3 q) {
    return P3{clamp_d(q.x, 0., v.size), clamp_d(q.y, 0., v.size), clamp_d(q.z, 0., v.size)};
}

// The first vertex of a tet: where the descent toward the nearest site starts.
VB_SX int start_site(const View& v, int hint) { return hint >= 0 ? v.tet_vertices[4 * hint] : 0; }

// Midpoint trace of dual vertex i and the velocity at its foot
// (advectVorticity's first loop).
VB_SX void trace_dual(const View& v, int i, double dt, const double* dual_velocity, const double* samples, P3* traced,
                      P3* velocity, int* error) {
    const P3 p = load3(v.dual_position, i);
    const int hint = v.dual_hint[i];
    if (v.box) {
        const int s0 = start_site(v, hint);
        const P3 mid = clip_box(v, sub(p, mul(box_velocity(v, p, s0, dual_velocity, error), dt * .5)));
        *traced = clip_box(v, sub(p, mul(box_velocity(v, mid, s0, dual_velocity, error), dt)));
        *velocity = box_velocity(v, *traced, s0, dual_velocity, error);
        return;
    }
    const P3 mid = clip_segment(v, p, sub(p, mul(load3(dual_velocity, i), dt * .5)), hint);
    const P3 mv = domain_velocity(v, mid, hint, samples, error);
    *traced = clip_segment(v, p, sub(p, mul(mv, dt)), hint);
    *velocity = domain_velocity(v, *traced, hint, samples, error);
}

// .5 (v_a + v_b) . (x_b - x_a) of dual edge j (advectVorticity's second
// loop); traced points and their velocities, 3 doubles per dual vertex.
VB_SX double edge_integral(const View& v, int j, const double* traced, const double* velocity) {
    const int a = v.dual_edges[2 * j], b = v.dual_edges[2 * j + 1];
    return .5 * dot(add(load3(velocity, a), load3(velocity, b)), sub(load3(traced, b), load3(traced, a)));
}

// The circulation of primal edge e: its dual face's signed edge integrals,
// summed in loop order from zero (DualMesh::circulation).
VB_SX double circulation(const View& v, int e, const double* integral) {
    double omega = 0;
    for (int j = v.loop_offsets[e]; j < v.loop_offsets[e + 1]; ++j) {
        const int code = v.loop_items[j];
        const int sign = code > 0 ? 1 : -1, edge = (code > 0 ? code : -code) - 1;
        omega += sign * integral[edge];
    }
    return omega;
}

// Traced smoke of primal vertex i (advectAndDecaySmoke's loop), as the
// float the reference stores.
VB_SX float trace_density(const View& v, int i, double dt, double decay, const double* dual_velocity,
                          const double* samples, const float* density, int* error) {
    const P3 p = load3(v.node_position, i);
    double w[4];
    if (v.box) {
        const int hint = v.primal_hint[i];
        const int s0 = start_site(v, hint);
        const P3 mid = clip_box(v, sub(p, mul(box_velocity(v, p, s0, dual_velocity, error), dt * .5)));
        const P3 q = clip_box(v, sub(p, mul(box_velocity(v, mid, s0, dual_velocity, error), dt)));
        const int t = locate(v, q, -1);  // sampleDensity locates without a hint
        double sampled = 0;
        if (t >= 0) {
            barycentric(v, t, q, w);
            double value = 0, total = 0;
            for (int k = 0; k < 4; ++k) {
                const double weight = max_d(0., w[k]);
                value += weight * density[v.tet_vertices[4 * t + k]];
                total += weight;
            }
            sampled = value / total;
        }
        return float(sampled * decay);
    }
    const int hint = v.primal_hint[i];
    const P3 mid = clip_segment(v, p, sub(p, mul(load3(samples, i), dt * .5)), hint);
    const P3 vel = domain_velocity(v, mid, hint, samples, error);
    const P3 q = clip_segment(v, p, sub(p, mul(vel, dt)), hint);
    const int t = locate(v, q, hint);
    double value = 0, total = 0;
    if (t >= 0) {
        barycentric(v, t, q, w);
        for (int k = 0; k < 4; ++k) {
            const double weight = max_d(0., w[k]);
            value += weight * density[v.tet_vertices[4 * t + k]];
            total += weight;
        }
    }
    return total > 0 ? float(value / total * decay) : 0.f;
}

}  // namespace simplicial
}  // namespace vb
