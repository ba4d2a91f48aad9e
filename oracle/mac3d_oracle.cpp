// TEST INFRASTRUCTURE — the oracle. Nothing in the product links or calls this
// file; only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it,
// as the checker.
//
// CPU restatement of the MAC 3D smoke step of taehwann/vapor, templated on the
// arithmetic type T:
//   T = float  reproduces the reference's FP32 arithmetic operation for
//              operation (same evaluation order, no FMA contraction: build with
//              -ffp-contract=off), so it is bit-identical to the reference CPU
//              path. Pinned against the compiled reference (oracle/_ref) and the
//              reference's golden vectors (tests/SimulationTests.cpp:17-34).
//   T = double the FP64 oracle: the same formulas evaluated in double, used to
//              state the FP32 error of every field.
//
// Reference files followed (paths inside taehwann/vapor):
//   sampling           src/solvers/mac3d/MacGridSampler3D.cpp:5-75
//   advection          src/solvers/mac3d/CpuAdvectionKernels.cpp:18-269
//   divergence, walls, gradient   src/solvers/mac3d/MacGridOperators3D.cpp:8-67
//   Neumann system     src/solvers/mac3d/CpuPressureSolver3D.cpp:9-23
//   projection         src/solvers/mac3d/CpuPressureSolver3D.cpp:25-60
//   SOR                src/solvers/mac3d/SOR.cpp:22-64
//   residual           src/solvers/mac3d/StencilLinearSystem.cpp:53-70
//   emit/buoyancy/decay/step   src/solvers/mac3d/MacGridFluidSolver3D.cpp:140-245
//   diagnostics        src/solvers/mac3d/MacGridFluidSolver3D.cpp:247-269
//
// Extensions the reference does not have (profile emitter, second emitter,
// tolerance-driven projections inside the step, mixed-precision refinement)
// are implemented here the same way as in the CUDA path; for those the oracle
// is the only pin ("parity unpinned" against the reference).

#include "../include/vapor_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace {

// Staggered locations: cell centre, x-, y- and z-faces.
enum Loc : int { CELL = 0, FACE_X = 1, FACE_Y = 2, FACE_Z = 3 };

template <class T>
struct Grid {
    int n;
    T box;
    T h;  // box / n, computed once as MacGridDomain3D::cellSize does
    Grid(int n_, T box_) : n(n_), box(box_), h(box_ / T(n_)) {}
    int extent(int loc, int dim) const { return n + (loc == dim + 1 ? 1 : 0); }
    size_t count(int loc) const {
        return size_t(extent(loc, 0)) * size_t(extent(loc, 1)) * size_t(extent(loc, 2));
    }
    size_t index(int loc, int x, int y, int z) const {
        return size_t(x) + size_t(extent(loc, 0)) * (size_t(y) + size_t(extent(loc, 1)) * size_t(z));
    }
};

template <class T> struct V3 { T x, y, z; };

template <class T> inline T clampT(T v, T lo, T hi) { return v < lo ? lo : (hi < v ? hi : v); }
inline int clampI(int v, int lo, int hi) { return v < lo ? lo : (hi < v ? hi : v); }
template <class T> inline T minT(T a, T b) { return b < a ? b : a; }
template <class T> inline T maxT(T a, T b) { return a < b ? b : a; }

// One dimension of a clamped trilinear lookup (MacGridSampler3D.cpp:6-11).
template <class T>
struct Bracket { int i0, i1; T t; };

template <class T>
inline Bracket<T> bracket(T coord, T h, bool staggered, int n) {
    Bracket<T> b;
    if (staggered) {
        const T g = clampT(coord / h, T(0), T(n));
        b.i0 = std::min(int(g), n - 1);
        b.i1 = b.i0 + 1;
        b.t = g - T(b.i0);
    } else {
        const T g = clampT(coord / h - T(0.5), T(0), T(n - 1));
        b.i0 = int(g);
        b.i1 = std::min(b.i0 + 1, n - 1);
        b.t = g - T(b.i0);
    }
    return b;
}

// Fixed 8-term weight order of the reference sampler.
template <class T, class F>
inline T sample(const Grid<T>& g, int loc, const F* f, V3<T> p) {
    const Bracket<T> bx = bracket(p.x, g.h, loc == FACE_X, g.n);
    const Bracket<T> by = bracket(p.y, g.h, loc == FACE_Y, g.n);
    const Bracket<T> bz = bracket(p.z, g.h, loc == FACE_Z, g.n);
    const T ux = T(1) - bx.t, uy = T(1) - by.t, uz = T(1) - bz.t;
    const T tx = bx.t, ty = by.t, tz = bz.t;
    auto at = [&](int x, int y, int z) -> T { return T(f[g.index(loc, x, y, z)]); };
    return at(bx.i0, by.i0, bz.i0) * ux * uy * uz + at(bx.i1, by.i0, bz.i0) * tx * uy * uz +
           at(bx.i0, by.i1, bz.i0) * ux * ty * uz + at(bx.i1, by.i1, bz.i0) * tx * ty * uz +
           at(bx.i0, by.i0, bz.i1) * ux * uy * tz + at(bx.i1, by.i0, bz.i1) * tx * uy * tz +
           at(bx.i0, by.i1, bz.i1) * ux * ty * tz + at(bx.i1, by.i1, bz.i1) * tx * ty * tz;
}

template <class T, class F>
inline V3<T> velocityAt(const Grid<T>& g, const F* u, const F* v, const F* w, V3<T> p) {
    return {sample(g, FACE_X, u, p), sample(g, FACE_Y, v, p), sample(g, FACE_Z, w, p)};
}

// World position of a sample point: staggered axis at i*h, others at (i+.5)h.
template <class T>
inline V3<T> position(const Grid<T>& g, int loc, int x, int y, int z) {
    auto c = [&](int i, bool staggered) { return staggered ? T(i) * g.h : (T(i) + T(0.5)) * g.h; };
    return {c(x, loc == FACE_X), c(y, loc == FACE_Y), c(z, loc == FACE_Z)};
}

// Semi-Lagrangian / MacCormack transport of one staggered field
// (CpuAdvectionKernels.cpp:18-269). `out` must not alias `src` or the flow.
template <class T, class F>
void advect(const Grid<T>& g, int loc, T dt, T cflLimit, bool maccormack, const F* src, const F* u,
            const F* v, const F* w, F* out) {
    const int ex = g.extent(loc, 0), ey = g.extent(loc, 1), ez = g.extent(loc, 2);
    std::vector<T> fwd(g.count(loc));
    for (int z = 0; z < ez; ++z)
        for (int y = 0; y < ey; ++y)
            for (int x = 0; x < ex; ++x) {
                const V3<T> p = position(g, loc, x, y, z);
                const V3<T> vel = velocityAt(g, u, v, w, p);
                const V3<T> dep{p.x - vel.x * dt, p.y - vel.y * dt, p.z - vel.z * dt};
                fwd[g.index(loc, x, y, z)] = sample(g, loc, src, dep);
            }
    if (!maccormack) {
        for (size_t i = 0; i < fwd.size(); ++i) out[i] = F(fwd[i]);
        return;
    }
    const int hiX = ex - 1, hiY = ey - 1, hiZ = ez - 1;
    for (int z = 0; z < ez; ++z)
        for (int y = 0; y < ey; ++y)
            for (int x = 0; x < ex; ++x) {
                const size_t i = g.index(loc, x, y, z);
                const V3<T> p = position(g, loc, x, y, z);
                const V3<T> vel = velocityAt(g, u, v, w, p);
                const V3<T> pf{p.x - vel.x * dt, p.y - vel.y * dt, p.z - vel.z * dt};
                const V3<T> pb{p.x + vel.x * dt, p.y + vel.y * dt, p.z + vel.z * dt};
                const T cfl = std::sqrt(vel.x * vel.x + vel.y * vel.y + vel.z * vel.z) * dt / g.h;
                const bool leaves = pf.x < T(0) || pf.x > g.box || pf.y < T(0) || pf.y > g.box ||
                                    pf.z < T(0) || pf.z > g.box || pb.x < T(0) || pb.x > g.box ||
                                    pb.y < T(0) || pb.y > g.box || pb.z < T(0) || pb.z > g.box;
                if (leaves || cfl > cflLimit) {
                    out[i] = F(fwd[i]);
                    continue;
                }
                const T back = sample(g, loc, fwd.data(), pb);
                const T corrected = fwd[i] + T(0.5) * (T(src[i]) - back);
                auto donor = [&](T coord, bool staggered) {
                    return staggered ? clampI(int(coord / g.h), 0, g.n)
                                     : clampI(int(coord / g.h - T(0.5)), 0, g.n - 1);
                };
                const int gx = donor(pf.x, loc == FACE_X), gy = donor(pf.y, loc == FACE_Y),
                          gz = donor(pf.z, loc == FACE_Z);
                T lo = T(src[g.index(loc, gx, gy, gz)]), hi = lo;
                for (int dz = 0; dz <= 1; ++dz)
                    for (int dy = 0; dy <= 1; ++dy)
                        for (int dx = 0; dx <= 1; ++dx) {
                            const T s = T(src[g.index(loc, clampI(gx + dx, 0, hiX), clampI(gy + dy, 0, hiY),
                                                      clampI(gz + dz, 0, hiZ))]);
                            lo = minT(lo, s);
                            hi = maxT(hi, s);
                        }
                out[i] = F(clampT(corrected, lo, hi));
            }
}

// (u[x+1]-u[x] + v[y+1]-v[y] + w[z+1]-w[z]) / h, left to right.
template <class T, class F>
inline T divergenceAt(const Grid<T>& g, const F* u, const F* v, const F* w, int x, int y, int z) {
    return (T(u[g.index(FACE_X, x + 1, y, z)]) - T(u[g.index(FACE_X, x, y, z)]) +
            T(v[g.index(FACE_Y, x, y + 1, z)]) - T(v[g.index(FACE_Y, x, y, z)]) +
            T(w[g.index(FACE_Z, x, y, z + 1)]) - T(w[g.index(FACE_Z, x, y, z)])) /
           g.h;
}

template <class T, class F>
void enforceWalls(const Grid<T>& g, F* u, F* v, F* w) {
    const int n = g.n;
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y) u[g.index(FACE_X, 0, y, z)] = u[g.index(FACE_X, n, y, z)] = F(0);
    for (int z = 0; z < n; ++z)
        for (int x = 0; x < n; ++x) v[g.index(FACE_Y, x, 0, z)] = v[g.index(FACE_Y, x, n, z)] = F(0);
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) w[g.index(FACE_Z, x, y, 0)] = w[g.index(FACE_Z, x, y, n)] = F(0);
}

// max |div| with the reference's non-finite rejection; returns NaN when a
// non-finite divergence is found (the reference throws invalid_argument).
template <class T, class F>
T maxDivergence(const Grid<T>& g, const F* u, const F* v, const F* w) {
    T m = T(0);
    for (int z = 0; z < g.n; ++z)
        for (int y = 0; y < g.n; ++y)
            for (int x = 0; x < g.n; ++x) {
                const T d = divergenceAt(g, u, v, w, x, y, z);
                if (!std::isfinite(d)) return std::numeric_limits<T>::quiet_NaN();
                m = maxT(m, std::abs(d));
            }
    return m;
}

// u -= dt * (p_i - p_{i-1}) * (1/h) on interior faces (MacGridOperators3D.cpp:51-67).
template <class T, class F, class P>
void applyGradient(const Grid<T>& g, const P* p, T dt, F* u, F* v, F* w) {
    const int n = g.n;
    const T hInv = T(1) / g.h;
    auto pc = [&](int x, int y, int z) { return T(p[g.index(CELL, x, y, z)]); };
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 1; x < n; ++x) {
                F& f = u[g.index(FACE_X, x, y, z)];
                f = F(T(f) - dt * (pc(x, y, z) - pc(x - 1, y, z)) * hInv);
            }
    for (int z = 0; z < n; ++z)
        for (int y = 1; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                F& f = v[g.index(FACE_Y, x, y, z)];
                f = F(T(f) - dt * (pc(x, y, z) - pc(x, y - 1, z)) * hInv);
            }
    for (int z = 1; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                F& f = w[g.index(FACE_Z, x, y, z)];
                f = F(T(f) - dt * (pc(x, y, z) - pc(x, y, z - 1)) * hInv);
            }
}

// Gradient step with an FP64 pressure (mixed-precision refinement): the
// difference, scaling and subtraction run in double, then round to the field.
template <class T, class F>
void applyGradient64(const Grid<T>& g, const double* p, T dt, F* u, F* v, F* w) {
    const int n = g.n;
    const double hInv = 1.0 / double(g.h), dtd = double(dt);
    auto pc = [&](int x, int y, int z) { return p[g.index(CELL, x, y, z)]; };
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 1; x < n; ++x) {
                F& f = u[g.index(FACE_X, x, y, z)];
                f = F(double(f) - dtd * (pc(x, y, z) - pc(x - 1, y, z)) * hInv);
            }
    for (int z = 0; z < n; ++z)
        for (int y = 1; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                F& f = v[g.index(FACE_Y, x, y, z)];
                f = F(double(f) - dtd * (pc(x, y, z) - pc(x, y - 1, z)) * hInv);
            }
    for (int z = 1; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                F& f = w[g.index(FACE_Z, x, y, z)];
                f = F(double(f) - dtd * (pc(x, y, z) - pc(x, y, z - 1)) * hInv);
            }
}

// ---------------------------------------------------------------------------
// Closed-box Neumann system A = -h^2 Laplacian (CpuPressureSolver3D.cpp:9-23):
// diagonal = number of existing neighbours, every coupling -1. Stored
// implicitly; the operator order matches StencilLinearSystem.
// ---------------------------------------------------------------------------
// Solid obstacles (extension, no reference counterpart): while a projection
// with a solid mask runs, tSolid points at its n^3 mask (x fastest, nonzero =
// solid). Solid cells are not unknowns (pressure 0, residual excluded); the
// diagonal of a fluid cell counts its fluid neighbours; faces touching a
// solid are closed (velocity 0).
thread_local const uint8_t* tSolid = nullptr;
inline bool solidAt(int n, int x, int y, int z) {
    return tSolid && tSolid[size_t(x) + size_t(n) * (size_t(y) + size_t(n) * z)] != 0;
}

inline int neighbourCount(int n, int x, int y, int z) {
    if (!tSolid) return (x > 0) + (x + 1 < n) + (y > 0) + (y + 1 < n) + (z > 0) + (z + 1 < n);
    if (solidAt(n, x, y, z)) return 0;
    return (x > 0 && !solidAt(n, x - 1, y, z)) + (x + 1 < n && !solidAt(n, x + 1, y, z)) +
           (y > 0 && !solidAt(n, x, y - 1, z)) + (y + 1 < n && !solidAt(n, x, y + 1, z)) +
           (z > 0 && !solidAt(n, x, y, z - 1)) + (z + 1 < n && !solidAt(n, x, y, z + 1));
}

// Zero every face that touches a solid cell (no-op without a mask).
template <class T, class F>
void enforceSolids(const Grid<T>& g, F* u, F* v, F* w) {
    if (!tSolid) return;
    const int n = g.n;
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                if (!solidAt(n, x, y, z)) continue;
                u[g.index(FACE_X, x, y, z)] = u[g.index(FACE_X, x + 1, y, z)] = F(0);
                v[g.index(FACE_Y, x, y, z)] = v[g.index(FACE_Y, x, y + 1, z)] = F(0);
                w[g.index(FACE_Z, x, y, z)] = w[g.index(FACE_Z, x, y, z + 1)] = F(0);
            }
}

// FP64 infinity norm of b - A x (StencilLinearSystem.cpp:53-70).
template <class X, class B>
double residualInf(int n, const X* x, const B* b) {
    double r = 0.0;
    const size_t nn = size_t(n) * n;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const size_t id = size_t(i) + size_t(n) * (size_t(j) + size_t(n) * k);
                if (solidAt(n, i, j, k)) continue;
                double ax = double(float(neighbourCount(n, i, j, k))) * double(x[id]);
                if (i > 0) ax += -1.0 * double(x[id - 1]);
                if (i + 1 < n) ax += -1.0 * double(x[id + 1]);
                if (j > 0) ax += -1.0 * double(x[id - n]);
                if (j + 1 < n) ax += -1.0 * double(x[id + n]);
                if (k > 0) ax += -1.0 * double(x[id - nn]);
                if (k + 1 < n) ax += -1.0 * double(x[id + nn]);
                if (!std::isfinite(double(x[id])) || !std::isfinite(double(b[id])))
                    return std::numeric_limits<double>::quiet_NaN();
                r = std::max(r, std::abs(double(b[id]) - ax));
            }
    return r;
}

// One red-black SOR iteration (SOR.cpp:36-54): colour 0 (i+j+k even) first.
template <class T>
void sorIteration(int n, T omega, T floorDiag, T* x, const T* b) {
    const size_t nn = size_t(n) * n;
    for (int parity = 0; parity < 2; ++parity)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = (j + k + parity) & 1; i < n; i += 2) {
                    const size_t id = size_t(i) + size_t(n) * (size_t(j) + size_t(n) * k);
                    const T diag = T(neighbourCount(n, i, j, k));
                    if (diag == T(0)) continue;
                    T off = T(0);
                    if (i > 0) off += T(-1) * x[id - 1];
                    if (i + 1 < n) off += T(-1) * x[id + 1];
                    if (j > 0) off += T(-1) * x[id - n];
                    if (j + 1 < n) off += T(-1) * x[id + n];
                    if (k > 0) off += T(-1) * x[id - nn];
                    if (k + 1 < n) off += T(-1) * x[id + nn];
                    const T relax = maxT(diag, floorDiag);
                    x[id] += omega * (b[id] - off - diag * x[id]) / relax;
                }
}

// The mixed solver's inner sweep: the same red-black order with the
// divide-free relaxation x += (b - off - diag x) * w[diag], where
// w[d] = omega / max(d, floor) in FP32 (an extension; the reference's SOR is
// sorIteration above).
inline void sorIterationFast(int n, float omega, float floorDiag, float* x, const float* b) {
    float w[7];
    for (int d = 0; d < 7; ++d) w[d] = omega / maxT(float(d), floorDiag);
    const size_t nn = size_t(n) * n;
    for (int parity = 0; parity < 2; ++parity)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = (j + k + parity) & 1; i < n; i += 2) {
                    const size_t id = size_t(i) + size_t(n) * (size_t(j) + size_t(n) * k);
                    const int d = neighbourCount(n, i, j, k);
                    const float diag = float(d);
                    if (diag == 0.f) continue;
                    float off = 0.f;
                    if (i > 0) off += -1.f * x[id - 1];
                    if (i + 1 < n) off += -1.f * x[id + 1];
                    if (j > 0) off += -1.f * x[id - n];
                    if (j + 1 < n) off += -1.f * x[id + n];
                    if (k > 0) off += -1.f * x[id - nn];
                    if (k + 1 < n) off += -1.f * x[id + nn];
                    x[id] = x[id] + (b[id] - off - diag * x[id]) * w[d];
                }
}

inline bool validOptions(const vapor_linear_solve_options& o) {
    return o.max_iterations >= 0 && o.residual_check_interval > 0 && std::isfinite(o.absolute_tolerance) &&
           o.absolute_tolerance >= 0.0 && std::isfinite(o.relative_tolerance) && o.relative_tolerance >= 0.0;
}

// SOR::solve (SOR.cpp:22-64). Returns false on invalid input.
template <class T>
bool sorSolve(int n, T omega, T floorDiag, T* x, const T* b, const vapor_linear_solve_options& o,
              vapor_linear_solve_result& r) {
    if (!validOptions(o)) return false;
    r = {};
    r.initial_residual = r.final_residual = residualInf(n, x, b);
    if (std::isnan(r.initial_residual)) return false;
    const double target = std::max(o.absolute_tolerance, o.relative_tolerance * r.initial_residual);
    r.converged = r.final_residual <= target;
    if (r.converged && !o.fixed_iterations) return true;
    for (int it = 0; it < o.max_iterations; ++it) {
        sorIteration(n, omega, floorDiag, x, b);
        r.iterations = it + 1;
        if (r.iterations % o.residual_check_interval == 0 || r.iterations == o.max_iterations) {
            r.final_residual = residualInf(n, x, b);
            r.converged = r.final_residual <= target;
            if (r.converged && !o.fixed_iterations) break;
        }
    }
    return true;
}

// Mixed-precision refinement (extension). The pressure x64 is FP64; FP32
// red-black SOR sweeps run on the error equation A e = float(b - A x64) from
// e = 0. Every `residual_check_interval` sweeps (SOR.cpp:56-61) the FP32
// residual of the error equation is measured on the colour-1 cells (those
// the sweep updates last; the GPU measures it inside that sweep); the solver
// re-centres
// (x64 += e, new FP64 residual, e = 0) when that residual reaches the target,
// drops below kRecentreDrop times the FP64 residual of the last re-centring,
// after kRecentreSweeps sweeps, or at the iteration budget, and stops when the
// FP64 residual meets the target. For a stationary iteration this equals
// continuing SOR on x in exact arithmetic, but the iterate no longer stagnates
// at FP32 rounding (plain FP32 SOR stops near 1e-5 relative residual on a 32^3
// plume). The FP32 measure loses accuracy once the residual is ~1e3 below the
// last re-centring, which the 1e-2 threshold stays well clear of. `iterations`
// counts FP32 sweeps.
constexpr float kRecentreDrop = 1e-2f;
constexpr int kRecentreSweeps = 1024;

inline bool refinementSolve(int n, float omega, float floorDiag, std::vector<double>& x64,
                            const float* b, const vapor_linear_solve_options& o, vapor_linear_solve_result& r) {
    if (!validOptions(o)) return false;
    const size_t count = size_t(n) * n * n;
    r = {};
    std::vector<double> res(count);
    auto residual = [&]() {
        double m = 0.0;
        const size_t nn = size_t(n) * n;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    const size_t id = size_t(i) + size_t(n) * (size_t(j) + size_t(n) * k);
                    if (solidAt(n, i, j, k)) {
                        res[id] = 0.0;
                        continue;
                    }
                    double ax = double(neighbourCount(n, i, j, k)) * x64[id];
                    if (i > 0) ax -= x64[id - 1];
                    if (i + 1 < n) ax -= x64[id + 1];
                    if (j > 0) ax -= x64[id - n];
                    if (j + 1 < n) ax -= x64[id + n];
                    if (k > 0) ax -= x64[id - nn];
                    if (k + 1 < n) ax -= x64[id + nn];
                    res[id] = double(b[id]) - ax;
                    m = std::max(m, std::abs(res[id]));
                }
        return m;
    };
    r.initial_residual = r.final_residual = residual();
    const double target = std::max(o.absolute_tolerance, o.relative_tolerance * r.initial_residual);
    r.converged = r.final_residual <= target;
    if (r.converged && !o.fixed_iterations) return true;
    // FP32 sweeps on the error equation A e = rf; every check interval the FP32
    // residual max |rf - A e| (operation order: count * e, minus x-, x+, y-, y+,
    // z-, z+) decides whether to re-centre in FP64 and test the FP64 residual.
    std::vector<float> e(count, 0.f), rf(count);
    for (size_t i = 0; i < count; ++i) rf[i] = float(res[i]);
    double r0 = r.final_residual;
    int since = 0;
    const size_t nn = size_t(n) * n;
    while (true) {
        const int sweeps = std::min(o.residual_check_interval - r.iterations % o.residual_check_interval,
                                    o.max_iterations - r.iterations);
        for (int k = 0; k < sweeps; ++k) sorIterationFast(n, omega, floorDiag, e.data(), rf.data());
        r.iterations += sweeps;
        since += sweeps;
        // FP32 residual over the colour-1 cells ((i + j + k) odd, the colour a
        // sweep updates last), in the sweep's operation order.
        float rho = 0.f;
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    if (((i + j + k) & 1) == 0 || solidAt(n, i, j, k)) continue;
                    const size_t id = size_t(i) + size_t(n) * (size_t(j) + size_t(n) * k);
                    const float diag = float(neighbourCount(n, i, j, k));
                    float off = 0.f;
                    if (i > 0) off += -1.f * e[id - 1];
                    if (i + 1 < n) off += -1.f * e[id + 1];
                    if (j > 0) off += -1.f * e[id - n];
                    if (j + 1 < n) off += -1.f * e[id + n];
                    if (k > 0) off += -1.f * e[id - nn];
                    if (k + 1 < n) off += -1.f * e[id + nn];
                    rho = std::max(rho, std::abs(rf[id] - off - diag * e[id]));
                }
        const bool recentre = double(rho) <= target || double(rho) <= double(kRecentreDrop) * r0 ||
                              since >= kRecentreSweeps || r.iterations >= o.max_iterations;
        if (!recentre) continue;
        for (size_t i = 0; i < count; ++i) x64[i] += double(e[i]);
        r.final_residual = r0 = residual();
        since = 0;
        r.converged = r.final_residual <= target;
        if ((r.converged && !o.fixed_iterations) || r.iterations >= o.max_iterations) break;
        for (size_t i = 0; i < count; ++i) {
            rf[i] = float(res[i]);
            e[i] = 0.f;
        }
    }
    return true;
}

// CpuPressureSolver3D::project (CpuPressureSolver3D.cpp:25-60) over the fields
// u, v, w (FP type F) with arithmetic T. Returns a vapor_status.
template <class T, class F>
int project(const Grid<T>& g, F* u, F* v, F* w, T dt, T omega, T floorDiag, const vapor_linear_solve_options& o,
            int solverKind, vapor_projection_result& result, std::vector<T>& pressure) {
    if (!std::isfinite(double(omega)) || omega <= T(0) || omega >= T(2)) return VAPOR_INVALID_ARGUMENT;
    if (!std::isfinite(double(dt)) || dt <= T(0)) return VAPOR_INVALID_ARGUMENT;
    const T scale = g.h * g.h / dt;
    if (!std::isfinite(double(scale)) || scale <= T(0)) return VAPOR_INVALID_ARGUMENT;
    if (!validOptions(o)) return VAPOR_INVALID_ARGUMENT;
    const int n = g.n;
    const size_t count = size_t(n) * n * n;
    enforceWalls(g, u, v, w);
    enforceSolids(g, u, v, w);
    std::vector<T> b(count);
    result = {};
    size_t fluid = 0;
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const size_t i = g.index(CELL, x, y, z);
                if (solidAt(n, x, y, z)) {
                    b[i] = T(0);
                    continue;
                }
                ++fluid;
                const T d = divergenceAt(g, u, v, w, x, y, z);
                if (!std::isfinite(double(d))) return VAPOR_NON_FINITE;
                result.divergence_before = std::max(result.divergence_before, float(std::abs(d)));
                b[i] = -d * scale;
            }
    double sum = 0.0;
    for (size_t i = 0; i < count; ++i) sum += double(b[i]);
    result.removed_rhs_mean = sum / double(fluid);
    for (size_t i = 0; i < count; ++i)
        if (!tSolid || !tSolid[i]) b[i] -= T(result.removed_rhs_mean);
    pressure.assign(count, T(0));
    if (solverKind == VAPOR_SOLVER_MIXED_REFINEMENT && sizeof(T) == sizeof(float)) {
        std::vector<double> x64(count, 0.0);
        std::vector<float> bf(b.begin(), b.end());
        if (!refinementSolve(n, float(omega), float(floorDiag), x64, bf.data(), o, result.linear_solve))
            return VAPOR_INVALID_ARGUMENT;
        result.residual_available = 1;
        double pm = 0.0;
        for (double value : x64) pm += value;
        pm /= double(fluid);
        for (size_t i = 0; i < count; ++i)
            if (!tSolid || !tSolid[i]) x64[i] -= pm;
        result.linear_solve.final_residual = residualInf(n, x64.data(), bf.data());
        const double target = std::max(o.absolute_tolerance, o.relative_tolerance * result.linear_solve.initial_residual);
        result.linear_solve.converged = result.linear_solve.final_residual <= target;
        applyGradient64(g, x64.data(), dt, u, v, w);
        for (size_t i = 0; i < count; ++i) pressure[i] = T(x64[i]);
    } else {
        if (!sorSolve(n, omega, floorDiag, pressure.data(), b.data(), o, result.linear_solve))
            return VAPOR_INVALID_ARGUMENT;
        result.residual_available = 1;
        double pm = 0.0;
        for (size_t i = 0; i < count; ++i) pm += double(pressure[i]);
        pm /= double(fluid);
        for (size_t i = 0; i < count; ++i)
            if (!tSolid || !tSolid[i]) pressure[i] -= T(pm);
        result.linear_solve.final_residual = residualInf(n, pressure.data(), b.data());
        const double target = std::max(o.absolute_tolerance, o.relative_tolerance * result.linear_solve.initial_residual);
        result.linear_solve.converged = result.linear_solve.final_residual <= target;
        applyGradient(g, pressure.data(), dt, u, v, w);
    }
    enforceWalls(g, u, v, w);
    enforceSolids(g, u, v, w);
    const T after = maxDivergence(g, u, v, w);
    if (std::isnan(double(after))) return VAPOR_NON_FINITE;
    result.divergence_after = float(after);
    return VAPOR_OK;
}

// ---------------------------------------------------------------------------
// The coordinator: MacGridFluidSolver3D's step sequence.
// ---------------------------------------------------------------------------
template <class T>
struct Simulation {
    Grid<T> g;
    vapor_mac3d_params p{};
    uint32_t rng = 0x9E3779B9u;
    std::vector<T> d, u, v, w;
    vapor_projection_result last{};
    long long totalIterations = 0;
    std::vector<uint8_t> solid;  // n^3 obstacle mask used by every projection (empty: none)

    Simulation(int n, T box) : g(n, box) {
        vapor_mac3d_default_params(&p);
        p.project_iterations = 2 * n;  // MacGridFluidSolver3D(MacGridState3D) ctor
        allocate();
    }
    void allocate() {
        d.assign(g.count(CELL), T(0));
        u.assign(g.count(FACE_X), T(0));
        v.assign(g.count(FACE_Y), T(0));
        w.assign(g.count(FACE_Z), T(0));
    }
    void reset() {
        rng = p.random_seed;
        std::fill(d.begin(), d.end(), T(0));
        std::fill(u.begin(), u.end(), T(0));
        std::fill(v.begin(), v.end(), T(0));
        std::fill(w.begin(), w.end(), T(0));
        last = {};
        totalIterations = 0;
    }
    T randomUnit() {
        rng = rng * 1664525u + 1013904223u;
        return T(rng >> 8) * T(1.0f / 16777216.0f);
    }

    // emit (MacGridFluidSolver3D.cpp:140-165) for one emitter centre.
    void emitAt(T cxFrac, T cyFrac, T czFrac, T strength, T dt) {
        const T dx = g.h;
        const T dtScale = dt * T(60);
        const T ecx = cxFrac * g.box, ecy = cyFrac * g.box, ecz = czFrac * g.box;
        const T erad = T(p.emitter_radius) * g.box;
        const int R = int(erad / dx + T(1));
        const int cx = int(ecx / dx), cy = int(ecy / dx), cz = int(ecz / dx);
        const int n = g.n;
        const T kickMul = T(p.emitter_kick_multiplier);
        for (int z = std::max(0, cz - R); z < std::min(n, cz + R); ++z)
            for (int y = std::max(0, cy - R); y < std::min(n, cy + R); ++y)
                for (int x = std::max(0, cx - R); x < std::min(n, cx + R); ++x) {
                    const T px = (T(x) + T(0.5)) * dx, py = (T(y) + T(0.5)) * dx, pz = (T(z) + T(0.5)) * dx;
                    const T qx = (px - ecx) / erad, qy = (py - ecy) / erad, qz = (pz - ecz) / erad;
                    const T q2 = qx * qx + qy * qy + qz * qz;
                    if (q2 > T(1)) continue;
                    const size_t i = g.index(CELL, x, y, z);
                    if (p.emitter_profile == 1) {
                        const T profile = minT(T(1), strength * T(3) * T(std::exp(double(T(-3.5) * q2))));
                        d[i] = maxT(d[i], profile);
                    } else {
                        d[i] = T(1);
                    }
                    const T kick = kickMul * (T(p.emitter_kick_base) + T(p.emitter_kick_scale) * strength);
                    if (kickMul > T(0)) {
                        T& lo = w[g.index(FACE_Z, x, y, z)];
                        T& hi = w[g.index(FACE_Z, x, y, z + 1)];
                        lo = maxT(lo, kick);
                        hi = maxT(hi, kick);
                    }
                    const T j = (randomUnit() - T(0.5)) * T(p.stir_strength) * dtScale;
                    u[g.index(FACE_X, x, y, z)] += j;
                    u[g.index(FACE_X, x + 1, y, z)] += j;
                    v[g.index(FACE_Y, x, y, z)] += j;
                    v[g.index(FACE_Y, x, y + 1, z)] += j;
                }
    }
    void emit(T strength, T dt) {
        if (strength <= T(0)) return;
        emitAt(T(p.emitter_center_x), T(p.emitter_center_y), T(p.emitter_center_z), strength, dt);
        if (p.emitter_count > 1)
            emitAt(T(p.emitter2_center_x), T(p.emitter2_center_y), T(p.emitter2_center_z), strength, dt);
    }
    // applyBuoyancy (MacGridFluidSolver3D.cpp:167-181): two separate adds per face.
    void buoyancy(T dt, T b) {
        const int n = g.n;
        const T split = T(p.buoyancy_split);
        for (int z = 1; z < n; ++z)
            for (int y = 0; y < n; ++y)
                for (int x = 0; x < n; ++x) {
                    const T lower = b * d[g.index(CELL, x, y, z - 1)] * dt;
                    const T upper = b * d[g.index(CELL, x, y, z)] * dt;
                    T& f = w[g.index(FACE_Z, x, y, z)];
                    f += split * lower;
                    f += split * upper;
                }
    }
    void dissipate(T dt) {
        const T factor = clampT(T(1) - T(p.smoke_decay) * dt, T(0), T(1));
        for (auto& value : d) value *= factor;
    }
    void advectVelocity(T dt, const std::vector<T>& su, const std::vector<T>& sv, const std::vector<T>& sw,
                        const std::vector<T>& fu, const std::vector<T>& fv, const std::vector<T>& fw) {
        const T cfl = T(p.cfl_mc);
        const bool mc = p.mac_cormack_vel != 0;
        advect(g, FACE_X, dt, cfl, mc, su.data(), fu.data(), fv.data(), fw.data(), u.data());
        advect(g, FACE_Y, dt, cfl, mc, sv.data(), fu.data(), fv.data(), fw.data(), v.data());
        advect(g, FACE_Z, dt, cfl, mc, sw.data(), fu.data(), fv.data(), fw.data(), w.data());
    }
    int doProject(T dt, int iterations) {
        vapor_linear_solve_options o;
        if (p.use_solve_options) {
            o = p.solve;
        } else {
            o.max_iterations = iterations;
            o.residual_check_interval = 8;
            o.absolute_tolerance = 1e-6;
            o.relative_tolerance = 1e-5;
            o.fixed_iterations = 1;
            o.reserved0 = 0;
        }
        std::vector<T> pressure;
        tSolid = solid.empty() ? nullptr : solid.data();
        const int status = project(g, u.data(), v.data(), w.data(), dt, T(p.sor_omega), T(6), o,
                                   p.solver_kind, last, pressure);
        tSolid = nullptr;
        totalIterations += last.linear_solve.iterations;
        return status;
    }
    void advectSmoke(T dt) {
        std::vector<T> out(d.size());
        advect(g, CELL, dt, T(p.cfl_mc), p.mac_cormack_smoke != 0, d.data(), u.data(), v.data(), w.data(),
               out.data());
        d.swap(out);
    }
    int stepNoReflect(T dt) {
        emit(T(p.source_strength), dt);
        buoyancy(dt, T(p.buoyancy));
        enforceWalls(g, u.data(), v.data(), w.data());
        const std::vector<T> u0 = u, v0 = v, w0 = w;
        advectVelocity(dt, u0, v0, w0, u0, v0, w0);
        const int status = doProject(dt, p.project_iterations);
        if (status) return status;
        advectSmoke(dt);
        dissipate(dt);
        return VAPOR_OK;
    }
    int stepReflect(T dt) {
        const T half = T(0.5) * dt;
        const int halfIters = std::max(1, p.project_iterations / 2);
        emit(T(p.source_strength), dt);
        buoyancy(dt, T(p.buoyancy));
        enforceWalls(g, u.data(), v.data(), w.data());
        const std::vector<T> u0 = u, v0 = v, w0 = w;
        advectVelocity(half, u0, v0, w0, u0, v0, w0);
        const std::vector<T> ut = u, vt = v, wt = w;
        int status = doProject(half, halfIters);
        if (status) return status;
        const std::vector<T> ud = u, vd = v, wd = w;
        std::vector<T> uh(u.size()), vh(v.size()), wh(w.size());
        for (size_t i = 0; i < u.size(); ++i) uh[i] = T(2) * u[i] - ut[i];
        for (size_t i = 0; i < v.size(); ++i) vh[i] = T(2) * v[i] - vt[i];
        for (size_t i = 0; i < w.size(); ++i) wh[i] = T(2) * w[i] - wt[i];
        advectVelocity(half, uh, vh, wh, ud, vd, wd);
        status = doProject(half, halfIters);
        if (status) return status;
        advectSmoke(dt);
        dissipate(dt);
        return VAPOR_OK;
    }
    int advance(T dt) {
        if (!std::isfinite(p.emitter_kick_multiplier) || p.emitter_kick_multiplier < 0.f)
            return VAPOR_INVALID_ARGUMENT;
        return p.reflection ? stepReflect(dt) : stepNoReflect(dt);
    }
    // kineticEnergy / maxVelocity (MacGridFluidSolver3D.cpp:247-264).
    void diagnostics(vapor_fluid_diagnostics& out) const {
        double ke = 0.0;
        for (T f : u) ke += double(f) * double(f);
        for (T f : v) ke += double(f) * double(f);
        for (T f : w) ke += double(f) * double(f);
        const double dx = double(g.h);
        out.kinetic_energy = float(0.5 * ke * dx * dx * dx);
        T m = T(0);
        for (T f : u) m = maxT(m, std::abs(f));
        for (T f : v) m = maxT(m, std::abs(f));
        for (T f : w) m = maxT(m, std::abs(f));
        out.max_velocity = float(m);
        const T md = maxDivergence(g, u.data(), v.data(), w.data());
        out.max_divergence = float(md);
    }
};

}  // namespace

// ---------------------------------------------------------------------------
// C API of the oracle (loaded with ctypes by tests and bench.py's CPU leg).
// Functions are generated for T = float (suffix _f32) and T = double (_f64).
// ---------------------------------------------------------------------------
#define VO_EXPORT extern "C" __attribute__((visibility("default")))

VO_EXPORT vapor_status vapor_mac3d_default_params(vapor_mac3d_params* o) {
    std::memset(o, 0, sizeof(*o));
    o->emitter_radius = 0.035f;
    o->emitter_center_x = 0.5f;
    o->emitter_center_y = 0.5f;
    o->emitter_center_z = 0.1f;
    o->emitter_kick_multiplier = 1.f;
    o->emitter_kick_base = 0.8f;
    o->emitter_kick_scale = 0.8f;
    o->stir_strength = 0.5f;
    o->random_seed = 0x9E3779B9u;
    o->sor_omega = 1.95f;
    o->buoyancy_split = 0.5f;
    o->cfl_mc = 3.0f;
    o->mac_cormack_smoke = 1;
    o->mac_cormack_vel = 1;
    o->smoke_decay = 0.06f;
    o->reflection = 1;
    o->buoyancy = 2.5f;
    o->source_strength = 1.f;
    o->project_iterations = 64;
    o->use_solve_options = 0;
    o->solve.max_iterations = 200;
    o->solve.residual_check_interval = 8;
    o->solve.absolute_tolerance = 1e-6;
    o->solve.relative_tolerance = 1e-5;
    o->solve.fixed_iterations = 0;
    o->solver_kind = VAPOR_SOLVER_RED_BLACK_SOR;
    o->emitter_profile = 0;
    o->emitter_count = 1;
    o->emitter2_center_x = 0.5f;
    o->emitter2_center_y = 0.5f;
    o->emitter2_center_z = 0.1f;
    return VAPOR_OK;
}

#define VO_DEFINE(T, SUF)                                                                                   \
    VO_EXPORT double vo_sample_##SUF(int n, T box, int loc, const T* f, T x, T y, T z) {                    \
        Grid<T> g(n, box);                                                                                  \
        return double(sample(g, loc, f, V3<T>{x, y, z}));                                                   \
    }                                                                                                       \
    VO_EXPORT void vo_advect_##SUF(int n, T box, int loc, T dt, T cfl, int mc, const T* src, const T* u,    \
                                   const T* v, const T* w, T* out) {                                        \
        Grid<T> g(n, box);                                                                                  \
        advect(g, loc, dt, cfl, mc != 0, src, u, v, w, out);                                                \
    }                                                                                                       \
    VO_EXPORT void vo_divergence_##SUF(int n, T box, const T* u, const T* v, const T* w, T* out) {          \
        Grid<T> g(n, box);                                                                                  \
        for (int z = 0; z < n; ++z)                                                                         \
            for (int y = 0; y < n; ++y)                                                                     \
                for (int x = 0; x < n; ++x) out[g.index(CELL, x, y, z)] = divergenceAt(g, u, v, w, x, y, z); \
    }                                                                                                       \
    VO_EXPORT double vo_max_divergence_##SUF(int n, T box, const T* u, const T* v, const T* w) {            \
        Grid<T> g(n, box);                                                                                  \
        return double(maxDivergence(g, u, v, w));                                                           \
    }                                                                                                       \
    VO_EXPORT void vo_enforce_walls_##SUF(int n, T* u, T* v, T* w) {                                       \
        Grid<T> g(n, T(1));                                                                                 \
        enforceWalls(g, u, v, w);                                                                           \
    }                                                                                                       \
    VO_EXPORT void vo_apply_gradient_##SUF(int n, T box, const T* p, T dt, T* u, T* v, T* w) {              \
        Grid<T> g(n, box);                                                                                  \
        applyGradient(g, p, dt, u, v, w);                                                                   \
    }                                                                                                       \
    VO_EXPORT double vo_residual_##SUF(int n, const T* x, const T* b) { return residualInf(n, x, b); }      \
    VO_EXPORT int vo_sor_solve_##SUF(int n, T omega, T floorDiag, T* x, const T* b,                         \
                                     const vapor_linear_solve_options* o, vapor_linear_solve_result* r) {   \
        return sorSolve(n, omega, floorDiag, x, b, *o, *r) ? VAPOR_OK : VAPOR_INVALID_ARGUMENT;             \
    }                                                                                                       \
    VO_EXPORT void vo_sor_iteration_##SUF(int n, T omega, T floorDiag, T* x, const T* b) {                  \
        sorIteration(n, omega, floorDiag, x, b);                                                            \
    }                                                                                                       \
    VO_EXPORT int vo_project_##SUF(int n, T box, T* u, T* v, T* w, T dt, T omega, T floorDiag,              \
                                   const vapor_linear_solve_options* o, int solverKind,                     \
                                   vapor_projection_result* r, T* pressureOut) {                            \
        Grid<T> g(n, box);                                                                                  \
        std::vector<T> pressure;                                                                            \
        const int status = project(g, u, v, w, dt, omega, floorDiag, *o, solverKind, *r, pressure);         \
        if (pressureOut && pressure.size() == size_t(n) * n * n)                                            \
            std::copy(pressure.begin(), pressure.end(), pressureOut);                                       \
        return status;                                                                                      \
    }                                                                                                       \
    VO_EXPORT int vo_project_masked_##SUF(int n, T box, T* u, T* v, T* w, T dt, T omega, T floorDiag,       \
                                          const vapor_linear_solve_options* o, int solverKind,              \
                                          const uint8_t* solid, vapor_projection_result* r, T* pressureOut) {\
        tSolid = solid;                                                                                     \
        const int status = vo_project_##SUF(n, box, u, v, w, dt, omega, floorDiag, o, solverKind, r,        \
                                            pressureOut);                                                   \
        tSolid = nullptr;                                                                                   \
        return status;                                                                                      \
    }                                                                                                       \
    VO_EXPORT void* vo_sim_create_##SUF(int n, T box) { return new Simulation<T>(n, box); }                 \
    VO_EXPORT void vo_sim_destroy_##SUF(void* h) { delete static_cast<Simulation<T>*>(h); }                \
    VO_EXPORT void vo_sim_set_params_##SUF(void* h, const vapor_mac3d_params* p) {                          \
        static_cast<Simulation<T>*>(h)->p = *p;                                                             \
    }                                                                                                       \
    VO_EXPORT void vo_sim_get_params_##SUF(void* h, vapor_mac3d_params* p) {                                \
        *p = static_cast<Simulation<T>*>(h)->p;                                                             \
    }                                                                                                       \
    VO_EXPORT void vo_sim_reset_##SUF(void* h) { static_cast<Simulation<T>*>(h)->reset(); }                 \
    VO_EXPORT void vo_sim_set_solid_##SUF(void* h, const uint8_t* mask) {                                   \
        Simulation<T>* sim = static_cast<Simulation<T>*>(h);                                                \
        const size_t cells = size_t(sim->g.n) * sim->g.n * sim->g.n;                                        \
        if (mask) sim->solid.assign(mask, mask + cells);                                                    \
        else sim->solid.clear();                                                                            \
    }                                                                                                       \
    VO_EXPORT int vo_sim_advance_##SUF(void* h, T dt) { return static_cast<Simulation<T>*>(h)->advance(dt); } \
    VO_EXPORT void vo_sim_get_fields_##SUF(void* h, T* d, T* u, T* v, T* w) {                               \
        auto* s = static_cast<Simulation<T>*>(h);                                                           \
        std::copy(s->d.begin(), s->d.end(), d);                                                             \
        std::copy(s->u.begin(), s->u.end(), u);                                                             \
        std::copy(s->v.begin(), s->v.end(), v);                                                             \
        std::copy(s->w.begin(), s->w.end(), w);                                                             \
    }                                                                                                       \
    VO_EXPORT void vo_sim_set_fields_##SUF(void* h, const T* d, const T* u, const T* v, const T* w) {       \
        auto* s = static_cast<Simulation<T>*>(h);                                                           \
        std::copy(d, d + s->d.size(), s->d.begin());                                                       \
        std::copy(u, u + s->u.size(), s->u.begin());                                                       \
        std::copy(v, v + s->v.size(), s->v.begin());                                                       \
        std::copy(w, w + s->w.size(), s->w.begin());                                                       \
    }                                                                                                       \
    VO_EXPORT uint32_t vo_sim_rng_##SUF(void* h) { return static_cast<Simulation<T>*>(h)->rng; }            \
    VO_EXPORT void vo_sim_set_rng_##SUF(void* h, uint32_t s) { static_cast<Simulation<T>*>(h)->rng = s; }   \
    VO_EXPORT void vo_sim_diagnostics_##SUF(void* h, vapor_fluid_diagnostics* out) {                        \
        static_cast<Simulation<T>*>(h)->diagnostics(*out);                                                  \
    }                                                                                                       \
    VO_EXPORT void vo_sim_last_projection_##SUF(void* h, vapor_projection_result* out) {                    \
        *out = static_cast<Simulation<T>*>(h)->last;                                                        \
    }                                                                                                       \
    VO_EXPORT long long vo_sim_total_iterations_##SUF(void* h) {                                            \
        return static_cast<Simulation<T>*>(h)->totalIterations;                                             \
    }

VO_DEFINE(float, f32)
VO_DEFINE(double, f64)

// The comparison metrics of the reference's diagnostic harness
// (tests/ReflectionComparison.hpp:32-75) on an FP32 state of box `box`
// (positions (x + .5) / n scaled by the box, frame time 1 / fps), with the
// harness's sequential FP64 sums. out: mass_sum, grad_sum, square_sum,
// div_square_sum, max_div, smoke_cells, cfl_fallback, boundary_fallback,
// max_cfl.
VO_EXPORT void vo_comparison_metrics(int n, float box, float fps, float cflMc, const float* d, const float* u,
                                     const float* v, const float* w, double* out) {
    const Grid<float> g(n, box);
    double mass = 0, grad = 0, square = 0, divSquare = 0, maxCfl = 0;
    float maxDiv = 0.f;
    long long smokeCells = 0, cflFallback = 0, boundaryFallback = 0;
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const float div = divergenceAt(g, u, v, w, x, y, z);
                divSquare += double(div) * div;
                maxDiv = maxT(maxDiv, std::fabs(div));
            }
    for (int z = 0; z < n; ++z)
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const float dv = d[g.index(CELL, x, y, z)];
                mass += dv;
                square += double(dv) * dv;
                if (x + 1 < n) grad += std::fabs(dv - d[g.index(CELL, x + 1, y, z)]);
                if (y + 1 < n) grad += std::fabs(dv - d[g.index(CELL, x, y + 1, z)]);
                if (z + 1 < n) grad += std::fabs(dv - d[g.index(CELL, x, y, z + 1)]);
                if (dv <= .001f) continue;
                ++smokeCells;
                const V3<float> pos{(x + .5f) / n * box, (y + .5f) / n * box, (z + .5f) / n * box};
                const V3<float> vel = velocityAt(g, u, v, w, pos);
                const double cfl = std::sqrt(vel.x * vel.x + vel.y * vel.y + vel.z * vel.z) * n / (box * fps);
                maxCfl = std::max(maxCfl, cfl);
                if (cfl > cflMc) ++cflFallback;
                const float step = 1.f / fps;
                const V3<float> a{pos.x - vel.x * step, pos.y - vel.y * step, pos.z - vel.z * step};
                const V3<float> b{pos.x + vel.x * step, pos.y + vel.y * step, pos.z + vel.z * step};
                if (a.x < 0 || a.x > box || a.y < 0 || a.y > box || a.z < 0 || a.z > box || b.x < 0 ||
                    b.x > box || b.y < 0 || b.y > box || b.z < 0 || b.z > box)
                    ++boundaryFallback;
            }
    const double r[9] = {mass, grad, square, divSquare, double(maxDiv), double(smokeCells), double(cflFallback),
                         double(boundaryFallback), maxCfl};
    std::copy(r, r + 9, out);
}

// MacGridParameters3D(MacAlgorithm) presets (MacGridFluidSolver3D.cpp:11-26).
VO_EXPORT vapor_status vapor_mac3d_algorithm_params(int32_t algorithm, vapor_mac3d_params* o) {
    if (algorithm < 0 || algorithm > 3) return VAPOR_INVALID_ARGUMENT;
    vapor_mac3d_default_params(o);
    o->reflection = algorithm >= 2;
    o->mac_cormack_smoke = (algorithm & 1);
    o->mac_cormack_vel = o->mac_cormack_smoke;
    o->emitter_radius = 0.08f;
    o->source_strength = 4.f;
    o->buoyancy = 3.f;
    o->smoke_decay = 0.08f;
    o->project_iterations = 600;
    o->sor_omega = 1.9f;
    return VAPOR_OK;
}


// Headless restatement of the reference's volume shader
// (src/renderer/shaders/volume.frag:13-55) with its orbit camera
// (src/renderer/OrbitCamera.cpp:5-28): for each pixel centre, the ray from the
// camera, the box slab test, front-to-back compositing of the FP32 trilinear
// (linear filter, clamp to edge) density, and the shadow march towards the
// light. rgb is width x height x 3, row 0 at the bottom; pixels without smoke
// keep the clear colour.
VO_EXPORT void vo_render_volume(int n, float box, const float* d, const vapor_render_params* p, float* rgb) {
    const float cax = cosf(p->azimuth), sax = sinf(p->azimuth), cel = cosf(p->elevation), sel = sinf(p->elevation);
    const float half = box * 0.5f;
    const float ro[3] = {half + p->distance * cel * cax, half + p->distance * cel * sax, half + p->distance * sel};
    const float up[3] = {-sel * cax, -sel * sax, cel};
    float fw[3] = {half - ro[0], half - ro[1], half - ro[2]};
    const float fl = sqrtf(fw[0] * fw[0] + fw[1] * fw[1] + fw[2] * fw[2]);
    for (float& c : fw) c /= fl;
    const float rt[3] = {fw[1] * up[2] - fw[2] * up[1], fw[2] * up[0] - fw[0] * up[2], fw[0] * up[1] - fw[1] * up[0]};
    const float f = 1.0f / tanf(0.8f * 0.5f);
    const float inv_p0 = 1.f / (f / (float(p->width) / float(p->height))), inv_p5 = 1.f / f;
    const float nf = float(n);
    auto tex = [&](float sx, float sy, float sz) {
        auto axis = [&](float s, int& i0, int& i1, float& t) {
            const float g = clampT(s * nf - 0.5f, 0.f, nf - 1.f);
            i0 = int(g);
            i1 = std::min(i0 + 1, n - 1);
            t = g - float(i0);
        };
        int x0, x1, y0, y1, z0, z1;
        float tx, ty, tz;
        axis(sx, x0, x1, tx);
        axis(sy, y0, y1, ty);
        axis(sz, z0, z1, tz);
        auto at = [&](int x, int y, int z) { return d[(size_t(z) * n + y) * n + x]; };
        const float ux = 1.f - tx, uy = 1.f - ty, uz = 1.f - tz;
        float s = at(x0, y0, z0) * ux * uy * uz;
        s = s + at(x1, y0, z0) * tx * uy * uz;
        s = s + at(x0, y1, z0) * ux * ty * uz;
        s = s + at(x1, y1, z0) * tx * ty * uz;
        s = s + at(x0, y0, z1) * ux * uy * tz;
        s = s + at(x1, y0, z1) * tx * uy * tz;
        s = s + at(x0, y1, z1) * ux * ty * tz;
        s = s + at(x1, y1, z1) * tx * ty * tz;
        return s;
    };
    const float bg[3] = {0.03f, 0.04f, 0.07f}, smoke[3] = {0.9f, 0.85f, 0.75f};
    for (int j = 0; j < p->height; ++j)
        for (int i = 0; i < p->width; ++i) {
            float* out = rgb + 3 * (size_t(j) * p->width + i);
            for (int k = 0; k < 3; ++k) out[k] = bg[k];
            const float xn = (float(i) + 0.5f) / float(p->width) * 2.f - 1.f;
            const float yn = (float(j) + 0.5f) / float(p->height) * 2.f - 1.f;
            const float vx = xn * inv_p0, vy = yn * inv_p5;
            float rd[3];
            for (int k = 0; k < 3; ++k) rd[k] = rt[k] * vx + up[k] * vy + fw[k];
            const float len = sqrtf(rd[0] * rd[0] + rd[1] * rd[1] + rd[2] * rd[2]);
            for (float& c : rd) c = c / len;
            float tnear = -std::numeric_limits<float>::infinity(), tfar = std::numeric_limits<float>::infinity();
            for (int k = 0; k < 3; ++k) {
                const float t0 = (0.f - ro[k]) / rd[k], t1 = (box - ro[k]) / rd[k];
                tnear = std::fmax(tnear, std::fmin(t0, t1));
                tfar = std::fmin(tfar, std::fmax(t0, t1));
            }
            if (tnear < 0.f) tnear = 0.f;
            if (!(tnear < tfar)) continue;
            const float step = p->step_scale / nf;
            float col[4] = {0.f, 0.f, 0.f, 0.f};
            bool hit = false;
            for (float t = tnear; t < tfar; t += step) {
                const float px = ro[0] + rd[0] * t, py = ro[1] + rd[1] * t, pz = ro[2] + rd[2] * t;
                const float dv = tex(px / box, py / box, pz / box);
                if (dv > 0.001f) {
                    hit = true;
                    float shadow = 1.f;
                    if (p->shadow_strength > 0.f) {
                        float sa = 0.f;
                        for (float st = p->shadow_step; st < box * 2.f; st += p->shadow_step) {
                            const float sx = px + p->light[0] * st, sy = py + p->light[1] * st,
                                        sz = pz + p->light[2] * st;
                            if (sx < 0.f || sx > box || sy < 0.f || sy > box || sz < 0.f || sz > box) break;
                            sa += tex(sx / box, sy / box, sz / box) * p->shadow_step * p->alpha_mul *
                                  p->shadow_strength;
                            if (sa > 3.f) break;
                        }
                        shadow = std::exp(-sa);
                    }
                    const float alpha = clampT(dv * step * p->alpha_mul, 0.f, 1.f);
                    for (int k = 0; k < 3; ++k) col[k] += (1.f - col[3]) * smoke[k] * alpha * shadow;
                    col[3] += (1.f - col[3]) * alpha;
                }
                if (col[3] > 0.99f) break;
            }
            if (!hit) continue;
            for (int k = 0; k < 3; ++k) out[k] = bg[k] * (1.f - col[3]) + col[k];
        }
}
