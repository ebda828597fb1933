// Test infrastructure (oracle): a C-ABI harness around the reference's own explicit DG operator.
//
// This file is compiled together with the reference sources, where they lie, by oracle/Makefile
// into oracle/_ref/libfvedg_ref.so. It is only ever loaded by tests, by __graft_entry__.smoke()
// and by bench.py's CPU-baseline / reference legs; the product never links it.
//
// What it exposes:
//   * ComputingMesh(const DGMesh&)  (src/Mesh/ComputingMesh.cpp:268-298) built from flat arrays,
//     with periodic faces patched in place: the face is first built as a boundary face so that its
//     normal points out of cells[0] (ComputingMesh.cpp:47-60), then cells[1] and the side-1
//     natural coordinates are filled by the same rule as ComputingMesh.cpp:67-75, using the
//     translated partner nodes.
//   * ExplicitConvection<P, Flux, QuadC, QuadF>::eval / eval_cells / eval_internals /
//     eval_boundarys (src/DG/DG_Schemes/ExplicitConvection.cpp:21-272) for the quadrature pairs
//     that the configurations use.
//   * The diagonal mass of examples/Eular1D/Sod1D/Riemann1D.cpp:108-121 and an SSP-RK3 loop
//     written with LongVector operators in the style of examples/Vortex/123/VortexRK.cpp:264-271.
//   * The reference's quadrature tables and DGBasisEvaluator<P>::eval_all/grad_all, so that the
//     product's own tables can be pinned against them.
//   * PositiveLimiter<P, QuadC, OnlyNeigbAvg> (include/DG/DG_Schemes/PositiveLimiter.h:12-261) as the
//     drivers call it: constructMinMax(current, previous) then apply(current, previous)
//     (examples/Eular1D/Sod1D/Riemann1D.cpp:194-195).
//   * ExplicitDiffusion<P, QuadC, QuadF>::eval (include/DG/DG_Schemes/ExplicitDiffusion.h:133-626),
//     the explicit viscous operator (mu = 1, Pr = 1, gamma = 1.4 fixed there).
//   * Meshes made without the product: the periodic Kuhn box restated here (build_box), and the
//     reference's own route OrthHexMesh -> split_hex6_scan -> ComputingMesh(GeneralMesh)
//     (build_orthhex); their flat topology is exported so tests can give the product the same mesh.
//   * Initial data by the reference's DGBasisEvaluator<P>::func2coef (long double,
//     include/DG/DG_Basis/DG_Basis_Evaluator.h:33-59) for the vortex, density wave and Taylor-Green.
#include "DG/DG_Schemes/ExplicitConvection.h"
#include "DG/DG_Schemes/ExplicitDiffusion.h"
#include "DG/DG_Schemes/PositiveLimiter.h"
#include "src/DG/DG_Schemes/ExplicitConvection.cpp"

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <map>
#include <omp.h>
#include <random>

// ---------------------------------------------------------------------------------------------
// Problem hooks required by include/base/exact.h:32-52. The Dirichlet branch of eval_boundarys
// (ExplicitConvection.cpp:47-53) calls rho_Xi .. rhoe_Xi. Here they evaluate a travelling
// density wave rho = r0 + A sin(2 pi k.(x - u t)), constant velocity and pressure, with the
// parameters set by fveref_set_dirichlet().
// ---------------------------------------------------------------------------------------------
namespace {
double g_dw[10] = {1.0, 0.2, 1.0, 1.0, 1.0, 1.0, 0.5, 0.25, 1.0, 1.4};  // r0 A kx ky kz u v w p gamma

void dw_state(const CompTetrahedron& cell, const vector3f& Xi, double t, double out[5]) {
    const vector3f x = cell.transform_to_physical(Xi);
    const double r0 = g_dw[0], A = g_dw[1];
    const double u = g_dw[5], v = g_dw[6], w = g_dw[7], p = g_dw[8], gam = g_dw[9];
    const double ph = 2.0 * M_PI * (g_dw[2] * (x[0] - u * t) + g_dw[3] * (x[1] - v * t) +
                                    g_dw[4] * (x[2] - w * t));
    const double rho = r0 + A * std::sin(ph);
    out[0] = rho;
    out[1] = rho * u;
    out[2] = rho * v;
    out[3] = rho * w;
    out[4] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
}
}  // namespace

Scalar rho_Xi(const CompTetrahedron& cell, const vector3f& Xi, Scalar t) {
    double s[5]; dw_state(cell, Xi, t, s); return s[0];
}
Scalar rhou_Xi(const CompTetrahedron& cell, const vector3f& Xi, Scalar t) {
    double s[5]; dw_state(cell, Xi, t, s); return s[1];
}
Scalar rhov_Xi(const CompTetrahedron& cell, const vector3f& Xi, Scalar t) {
    double s[5]; dw_state(cell, Xi, t, s); return s[2];
}
Scalar rhow_Xi(const CompTetrahedron& cell, const vector3f& Xi, Scalar t) {
    double s[5]; dw_state(cell, Xi, t, s); return s[3];
}
Scalar rhoe_Xi(const CompTetrahedron& cell, const vector3f& Xi, Scalar t) {
    double s[5]; dw_state(cell, Xi, t, s); return s[4];
}

// ---------------------------------------------------------------------------------------------
// Quadrature ids shared with the product and the C restatement:
//   tet: 0 Degree2Points4, 1 Degree4Points11, 2 Degree5Points15, 3 Degree6Points23,
//        4 Degree7Points31, 5 Degree8Points44, 6 Degree9Points57
//   tri: 0 Degree3Points4, 1 Degree3Points6, 2 Degree4Points7, 3 Degree10Points24
// ---------------------------------------------------------------------------------------------
namespace T = GaussLegendreTet;
namespace F = GaussLegendreTri;

template <class Q>
static int copy_rule3(double* pts, double* w) {
    for (int g = 0; g < Q::num_points; ++g) {
        if (pts) { pts[3 * g] = Q::points[g][0]; pts[3 * g + 1] = Q::points[g][1]; pts[3 * g + 2] = Q::points[g][2]; }
        if (w) w[g] = Q::weights[g];
    }
    return Q::num_points;
}
template <class Q>
static int copy_rule2(double* pts, double* w) {
    for (int g = 0; g < Q::num_points; ++g) {
        if (pts) { pts[2 * g] = Q::points[g][0]; pts[2 * g + 1] = Q::points[g][1]; }
        if (w) w[g] = Q::weights[g];
    }
    return Q::num_points;
}

namespace {
// A reference ComputingMesh plus, for meshes built inside this harness, the flat topology it was
// built from (exported so that tests can hand the very same mesh to the product).
struct RefMesh {
    ComputingMesh* cm = nullptr;
    std::vector<double> pts;                                // [npts][3]
    std::vector<uint64_t> cells, cell_faces, cell_cells;    // [ncell][4]
    std::vector<uint64_t> faces, face_cells, face_nodes1;   // [nface][3], [nface][2], [nface][3]
    std::vector<uint8_t> periodic, bc;                      // [nface]
};

template <uInt P>
void to_lv(const double* U, size_t ncell, LongVector<5 * DGBasisEvaluator<P>::NumBasis>& lv) {
    constexpr uInt B = 5 * DGBasisEvaluator<P>::NumBasis;
    for (size_t c = 0; c < ncell; ++c)
        for (uInt i = 0; i < B; ++i) lv[c](i, 0) = U[c * B + i];
}
template <uInt P>
void from_lv(const LongVector<5 * DGBasisEvaluator<P>::NumBasis>& lv, size_t ncell, double* U) {
    constexpr uInt B = 5 * DGBasisEvaluator<P>::NumBasis;
    for (size_t c = 0; c < ncell; ++c)
        for (uInt i = 0; i < B; ++i) U[c * B + i] = lv[c](i, 0);
}

template <uInt P, class Flux, class QC, class QF>
int run_eval(const ComputingMesh& m, const double* U, double* R, double t, int part) {
    using EC = ExplicitConvection<P, Flux, QC, QF>;
    EC ec;
    const size_t nc = m.m_cells.size();
    LongVector<5 * DGBasisEvaluator<P>::NumBasis> x(nc);
    to_lv<P>(U, nc, x);
    if (part == 0) from_lv<P>(ec.eval(m, x, t), nc, R);
    else if (part == 1) from_lv<P>(ec.eval_cells(m, x, t), nc, R);
    else if (part == 2) from_lv<P>(ec.eval_internals(m, x, t), nc, R);
    else if (part == 3) from_lv<P>(ec.eval_boundarys(m, x, t), nc, R);
    else return -2;
    return 0;
}

// SSP-RK3 (Shu-Osher) with L(U) = -(1/b) * eval(U); the stage arithmetic is written with the
// reference's LongVector operators exactly as its RK4 driver does (VortexRK.cpp:264-271).
template <uInt P, class Flux, class QC, class QF>
int run_ssprk3(const ComputingMesh& m, double* U, const double* mass, double dt, int nsteps,
               double t0) {
    using EC = ExplicitConvection<P, Flux, QC, QF>;
    using LV = LongVector<5 * DGBasisEvaluator<P>::NumBasis>;
    EC ec;
    const size_t nc = m.m_cells.size();
    LV x(nc), b(nc);
    to_lv<P>(U, nc, x);
    to_lv<P>(mass, nc, b);
    double t = t0;
    for (int s = 0; s < nsteps; ++s) {
        const auto& x1 = x + dt * (-1 / b * ec.eval(m, x, t));
        const auto& x2 = 0.75 * x + 0.25 * (x1 + dt * (-1 / b * ec.eval(m, x1, t + dt)));
        x = (1.0 / 3.0) * x + (2.0 / 3.0) * (x2 + dt * (-1 / b * ec.eval(m, x2, t + 0.5 * dt)));
        t += dt;
    }
    from_lv<P>(x, nc, U);
    return 0;
}

// Diagonal mass, examples/Eular1D/Sod1D/Riemann1D.cpp:108-121.
template <uInt P, class QC>
int run_mass(const ComputingMesh& m, double* mass) {
    using Basis = DGBasisEvaluator<P>;
    constexpr uInt N = Basis::NumBasis;
    const size_t nc = m.m_cells.size();
    LongVector<5 * N> b(nc);
    for (size_t cid = 0; cid < nc; ++cid) {
        for (uInt g = 0; g < QC::num_points; ++g) {
            const auto& p = QC::points[g];
            auto phi = Basis::eval_all(p[0], p[1], p[2]);
            for (uInt i = 0; i < N; ++i)
                for (uInt k = 0; k < 5; ++k)
                    b[cid](5 * i + k, 0) += phi[i] * phi[i] * QC::weights[g] * m.m_cells[cid].compute_jacobian_det();
        }
    }
    from_lv<P>(b, nc, mass);
    return 0;
}

template <uInt P, class QC, class QF>
int run_diffusion(const ComputingMesh& m, const double* U, double* R, double t) {
    const size_t nc = m.m_cells.size();
    LongVector<5 * DGBasisEvaluator<P>::NumBasis> x(nc);
    to_lv<P>(U, nc, x);
    ExplicitDiffusion<P, QC, QF> d;
    from_lv<P>(d.eval(m, x, t), nc, R);
    return 0;
}

template <uInt P, class QC, bool OnlyAvg>
int run_limit(const ComputingMesh& m, double* Ucur, const double* Uprev, double gamma) {
    using LV = LongVector<5 * DGBasisEvaluator<P>::NumBasis>;
    const size_t nc = m.m_cells.size();
    LV cur(nc), prev(nc);
    to_lv<P>(Ucur, nc, cur);
    to_lv<P>(Uprev, nc, prev);
    PositiveLimiter<P, QC, OnlyAvg> lim(m, gamma);
    lim.constructMinMax(cur, prev);
    lim.apply(cur, prev);
    from_lv<P>(cur, nc, Ucur);
    return 0;
}

template <uInt P>
int run_basis(int npts, const double* xyz, double* phi, double* grad) {
    using Basis = DGBasisEvaluator<P>;
    constexpr uInt N = Basis::NumBasis;
    for (int g = 0; g < npts; ++g) {
        auto v = Basis::eval_all(xyz[3 * g], xyz[3 * g + 1], xyz[3 * g + 2]);
        auto d = Basis::grad_all(xyz[3 * g], xyz[3 * g + 1], xyz[3 * g + 2]);
        for (uInt i = 0; i < N; ++i) {
            if (phi) phi[g * N + i] = v[i];
            if (grad) for (int c = 0; c < 3; ++c) grad[(g * N + i) * 3 + c] = d[i][c];
        }
    }
    return 0;
}
}  // namespace

namespace {
// Flat mesh in the DGMesh layout (include/Mesh/MeshGenerator.h:46-57) through ComputingMesh(const
// DGMesh&) (src/Mesh/ComputingMesh.cpp:268-298). A face with periodic_cell[f] != UINT64_MAX is a
// periodic face: it is passed to ComputingMesh as a boundary face of cells[0] (so its normal is
// oriented by the boundary rule, ComputingMesh.cpp:47-60) and then patched: cells[1] and the side-1
// natural coordinates by the rule of ComputingMesh.cpp:67-75 with the translated partner nodes.
RefMesh* build_dgmesh(uint64_t npts, const double* pts, uint64_t ncell, const uint64_t* cells,
                      const uint64_t* cell_faces, const uint64_t* cell_cells, uint64_t nface,
                      const uint64_t* faces, const uint64_t* face_cells, const uint8_t* bc,
                      const uint64_t* periodic_cell, const uint64_t* periodic_nodes) {
    DGMesh d;
    d.points.resize(npts);
    for (uint64_t i = 0; i < npts; ++i) d.points[i] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
    d.cells.resize(ncell);
    d.cell_faces.resize(ncell);
    d.cell_cells.resize(ncell);
    for (uint64_t c = 0; c < ncell; ++c)
        for (int k = 0; k < 4; ++k) {
            d.cells[c][k] = cells[4 * c + k];
            d.cell_faces[c][k] = cell_faces[4 * c + k];
            d.cell_cells[c][k] = cell_cells[4 * c + k];
        }
    d.faces.resize(nface);
    d.face_cells.resize(nface);
    d.is_boundary_face.resize(nface);
    for (uint64_t f = 0; f < nface; ++f) {
        for (int k = 0; k < 3; ++k) d.faces[f][k] = faces[3 * f + k];
        const bool per = periodic_cell && periodic_cell[f] != UINT64_MAX;
        d.face_cells[f] = {face_cells[2 * f], per ? size_t(-1) : face_cells[2 * f + 1]};
        d.is_boundary_face[f] = d.face_cells[f][1] == size_t(-1);
    }
    RefMesh* h = new RefMesh;
    h->cm = new ComputingMesh(d);
    ComputingMesh& m = *h->cm;
    m.m_boundaryTypes.assign(nface, BoundaryType::Pseudo3DZ);
    for (uint64_t f = 0; f < nface; ++f) {
        if (bc) m.m_boundaryTypes[f] = static_cast<BoundaryType>(bc[f]);
        if (!periodic_cell || periodic_cell[f] == UINT64_MAX) continue;
        auto& face = m.m_faces[f];
        const uInt c1 = periodic_cell[f];
        face.m_neighbor_cells[1] = c1;
        for (uInt k = 0; k < 3; ++k) {
            face.m_natural_coords[1][k] = {0, 0, 0};
            for (uInt ki = 0; ki < 3; ++ki)
                if (periodic_nodes[3 * f + k] == m.m_cells[c1].m_nodes[ki + 1])
                    face.m_natural_coords[1][k][ki] = 1;
        }
    }
    return h;
}
}  // namespace

namespace {
// ---------------------------------------------------------------------------------------------
// The periodic Kuhn box, restated here so that the oracle's own runs (the reference's CPU
// timings, golden data) need nothing from the product. Same mesh as the product's generator
// (tests check the arrays are identical):
//   * points i + (n+1)(j + (n+1)k) on [lo, hi]^3, the last plane exactly at hi; points strictly
//     inside the box moved by jitter*h*U(-1,1) per axis, in point order, from std::mt19937_64(seed);
//   * cube (i,j,k) in k, j, i order cut into the six tetrahedra of the monotone lattice paths from
//     its corner (i,j,k) to (i+1,j+1,k+1), steps in the axis orders xyz, yzx, zxy, xzy, zyx, yxz;
//     the second and third node swapped in the last three (odd permutations) so every det J > 0;
//   * local face q omits local node q; a face is numbered when first met in (cell, q) order and
//     keeps that cell's node order;
//   * on a periodic axis, a boundary face pairs with its translate: the lower-numbered face of the
//     pair stays, its cells[1] becomes the partner's cell and its side-1 nodes the translated ones;
//     the partner is removed and the numbering closed up.
// Face identification is by sorting (sorted node triple, position) records, not hashing.
// ---------------------------------------------------------------------------------------------
RefMesh* build_box(int n, const double lo[3], const double hi[3], double jitter, uint64_t seed, const int per[3],
                   int bc) {
    const uint64_t nv = (uint64_t)n + 1;
    auto pid = [&](uint64_t i, uint64_t j, uint64_t k) { return i + nv * (j + nv * k); };
    RefMesh* h = new RefMesh;
    h->pts.resize(3 * nv * nv * nv);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    double hs[3];
    for (int d = 0; d < 3; ++d) hs[d] = (hi[d] - lo[d]) / n;
    for (uint64_t k = 0; k < nv; ++k)
        for (uint64_t j = 0; j < nv; ++j)
            for (uint64_t i = 0; i < nv; ++i) {
                const uint64_t ijk[3] = {i, j, k};
                double* x = &h->pts[3 * pid(i, j, k)];
                for (int d = 0; d < 3; ++d) x[d] = ijk[d] == (uint64_t)n ? hi[d] : lo[d] + hs[d] * (double)ijk[d];
                const bool inside = i > 0 && i < (uint64_t)n && j > 0 && j < (uint64_t)n && k > 0 && k < (uint64_t)n;
                if (inside && jitter > 0)
                    for (int d = 0; d < 3; ++d) x[d] += jitter * hs[d] * uni(rng);
            }
    static const int order[6][2] = {{0, 1}, {1, 2}, {2, 0}, {0, 2}, {2, 1}, {1, 0}};  // first two steps
    const uint64_t nc = 6ull * n * n * n;
    h->cells.resize(4 * nc);
    uint64_t c = 0;
    for (uint64_t k = 0; k < (uint64_t)n; ++k)
        for (uint64_t j = 0; j < (uint64_t)n; ++j)
            for (uint64_t i = 0; i < (uint64_t)n; ++i)
                for (int s = 0; s < 6; ++s, ++c) {
                    uint64_t a[3] = {i, j, k};
                    uint64_t* nd = &h->cells[4 * c];
                    nd[0] = pid(a[0], a[1], a[2]);
                    ++a[order[s][0]];
                    nd[1] = pid(a[0], a[1], a[2]);
                    ++a[order[s][1]];
                    nd[2] = pid(a[0], a[1], a[2]);
                    nd[3] = pid(i + 1, j + 1, k + 1);
                    if (s >= 3) std::swap(nd[1], nd[2]);
                }
    // faces by sorting (key, position); position = 4 cell + q
    struct Rec { std::array<uint64_t, 3> key; uint64_t pos; };
    std::vector<Rec> rec(4 * nc);
    for (uint64_t cc = 0; cc < nc; ++cc)
        for (int q = 0; q < 4; ++q) {
            std::array<uint64_t, 3> key;
            for (int t = 0, m = 0; t < 4; ++t)
                if (t != q) key[m++] = h->cells[4 * cc + t];
            std::sort(key.begin(), key.end());
            rec[4 * cc + q] = {key, 4 * cc + q};
        }
    std::sort(rec.begin(), rec.end(), [](const Rec& x, const Rec& y) { return x.key != y.key ? x.key < y.key : x.pos < y.pos; });
    std::vector<uint64_t> creator;  // position of the first instance of each distinct face
    std::vector<uint64_t> group(4 * nc);  // position -> index of its group
    for (size_t r = 0; r < rec.size(); ++r) {
        if (r == 0 || rec[r].key != rec[r - 1].key) creator.push_back(rec[r].pos);
        group[rec[r].pos] = creator.size() - 1;
    }
    std::vector<uint64_t> rank(creator.size());  // group -> face id in first-met order
    {
        std::vector<uint64_t> idx(creator.size());
        for (size_t g = 0; g < idx.size(); ++g) idx[g] = g;
        std::sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return creator[x] < creator[y]; });
        for (size_t r = 0; r < idx.size(); ++r) rank[idx[r]] = r;
    }
    const uint64_t nf0 = creator.size();
    std::vector<uint64_t> fn(3 * nf0), fc(2 * nf0, UINT64_MAX), cf(4 * nc);
    std::map<std::array<uint64_t, 3>, uint64_t> by_key;
    for (uint64_t pos = 0; pos < 4 * nc; ++pos) {
        const uint64_t f = rank[group[pos]], cc = pos / 4;
        const int q = (int)(pos % 4);
        cf[pos] = f;
        if (creator[group[pos]] == pos) {
            for (int t = 0, m = 0; t < 4; ++t)
                if (t != q) fn[3 * f + m++] = h->cells[4 * cc + t];
            fc[2 * f] = cc;
        } else {
            fc[2 * f + 1] = cc;
        }
    }
    for (size_t r = 0; r < rec.size(); ++r)
        if (creator[group[rec[r].pos]] == rec[r].pos) by_key[rec[r].key] = rank[group[rec[r].pos]];
    std::vector<uint64_t> fn1(fn);
    std::vector<uint8_t> isper(nf0, 0);
    std::vector<char> gone(nf0, 0);
    for (uint64_t f = 0; f < nf0; ++f) {
        if (fc[2 * f + 1] != UINT64_MAX || gone[f]) continue;
        uint64_t ijk[3][3];
        for (int t = 0; t < 3; ++t) {
            const uint64_t p = fn[3 * f + t];
            ijk[t][0] = p % nv; ijk[t][1] = (p / nv) % nv; ijk[t][2] = p / (nv * nv);
        }
        for (int d = 0; d < 3; ++d) {
            const bool low = ijk[0][d] == 0 && ijk[1][d] == 0 && ijk[2][d] == 0;
            const bool high = ijk[0][d] == (uint64_t)n && ijk[1][d] == (uint64_t)n && ijk[2][d] == (uint64_t)n;
            if (!(low || high) || !per[d]) continue;
            uint64_t moved[3];
            for (int t = 0; t < 3; ++t) {
                uint64_t a[3] = {ijk[t][0], ijk[t][1], ijk[t][2]};
                a[d] = low ? a[d] + n : a[d] - n;
                moved[t] = pid(a[0], a[1], a[2]);
            }
            std::array<uint64_t, 3> key = {moved[0], moved[1], moved[2]};
            std::sort(key.begin(), key.end());
            const uint64_t g = by_key.at(key);
            fc[2 * f + 1] = fc[2 * g];
            for (int t = 0; t < 3; ++t) fn1[3 * f + t] = moved[t];
            isper[f] = 1;
            gone[g] = 1;
            for (int q = 0; q < 4; ++q)
                if (cf[4 * fc[2 * g] + q] == g) cf[4 * fc[2 * g] + q] = f;
        }
    }
    std::vector<uint64_t> newid(nf0, UINT64_MAX);
    uint64_t nf = 0;
    for (uint64_t f = 0; f < nf0; ++f)
        if (!gone[f]) newid[f] = nf++;
    h->faces.resize(3 * nf); h->face_nodes1.resize(3 * nf); h->face_cells.resize(2 * nf);
    h->periodic.resize(nf); h->bc.assign(nf, (uint8_t)bc);
    for (uint64_t f = 0; f < nf0; ++f) {
        if (gone[f]) continue;
        const uint64_t r = newid[f];
        for (int t = 0; t < 3; ++t) { h->faces[3 * r + t] = fn[3 * f + t]; h->face_nodes1[3 * r + t] = fn1[3 * f + t]; }
        h->face_cells[2 * r] = fc[2 * f];
        h->face_cells[2 * r + 1] = fc[2 * f + 1];
        h->periodic[r] = isper[f];
    }
    h->cell_faces.resize(4 * nc); h->cell_cells.resize(4 * nc);
    for (uint64_t cc = 0; cc < nc; ++cc)
        for (int q = 0; q < 4; ++q) {
            const uint64_t r = newid[cf[4 * cc + q]];
            h->cell_faces[4 * cc + q] = r;
            const uint64_t a = h->face_cells[2 * r], b = h->face_cells[2 * r + 1];
            h->cell_cells[4 * cc + q] = b == UINT64_MAX ? UINT64_MAX : (a == cc ? b : a);
        }
    // through ComputingMesh(const DGMesh&) with the periodic faces patched
    std::vector<uint64_t> pcell(nf, UINT64_MAX);
    for (uint64_t f = 0; f < nf; ++f)
        if (h->periodic[f]) pcell[f] = h->face_cells[2 * f + 1];
    RefMesh* m = build_dgmesh(nv * nv * nv, h->pts.data(), nc, h->cells.data(), h->cell_faces.data(),
                              h->cell_cells.data(), nf, h->faces.data(), h->face_cells.data(), h->bc.data(),
                              pcell.data(), h->face_nodes1.data());
    h->cm = m->cm;
    m->cm = nullptr;
    delete m;
    return h;
}

// The reference's own mesh route, as its drivers build a box (examples/Vortex/123/Vortex.cpp:101-106):
// OrthHexMesh (include/Mesh/OrthHexMesh.h:7-106) -> split_hex6_scan (src/Mesh/GeneralMesh.cpp:78-129)
// -> rebuild_cell_topology (:4-52, cell node order from unordered_set iteration) -> validate_mesh ->
// ComputingMesh(const GeneralMesh&) (src/Mesh/ComputingMesh.cpp:205-263). Boundary faces whose unit
// normal has |n_z| > 0.5 get bc_z, the others bc_side (the driver's split of its boundary at
// Vortex.cpp:108-114). The topology of the resulting ComputingMesh is kept for export.
RefMesh* build_orthhex(int n, const double lo[3], const double hi[3], int bc_z, int bc_side) {
    GeneralMesh g = OrthHexMesh({lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}, {(uInt)n, (uInt)n, (uInt)n});
    g.split_hex6_scan();
    g.rebuild_cell_topology();
    g.validate_mesh();
    RefMesh* h = new RefMesh;
    h->cm = new ComputingMesh(g);
    ComputingMesh& m = *h->cm;
    const size_t nc = m.m_cells.size(), nf = m.m_faces.size();
    m.m_boundaryTypes.assign(nf, BoundaryType::Pseudo3DZ);
    h->pts.resize(3 * m.m_points.size());
    for (size_t i = 0; i < m.m_points.size(); ++i)
        for (int d = 0; d < 3; ++d) h->pts[3 * i + d] = m.m_points[i][d];
    h->cells.resize(4 * nc); h->cell_faces.resize(4 * nc); h->cell_cells.resize(4 * nc);
    for (size_t c = 0; c < nc; ++c)
        for (int q = 0; q < 4; ++q) {
            h->cells[4 * c + q] = m.m_cells[c].m_nodes[q];
            h->cell_faces[4 * c + q] = m.m_cells[c].m_faces[q];
            h->cell_cells[4 * c + q] = m.m_cells[c].m_neighbors[q];
        }
    h->faces.resize(3 * nf); h->face_cells.resize(2 * nf); h->bc.resize(nf); h->periodic.assign(nf, 0);
    for (size_t f = 0; f < nf; ++f) {
        const auto& F = m.m_faces[f];
        for (int t = 0; t < 3; ++t) h->faces[3 * f + t] = F.m_nodes[t];
        h->face_cells[2 * f] = F.m_neighbor_cells[0];
        h->face_cells[2 * f + 1] = F.m_neighbor_cells[1];
        if (F.m_neighbor_cells[1] == uInt(-1))
            m.m_boundaryTypes[f] = static_cast<BoundaryType>(std::abs(F.m_normal[2]) > 0.5 ? bc_z : bc_side);
        h->bc[f] = static_cast<uint8_t>(m.m_boundaryTypes[f]);
    }
    h->face_nodes1 = h->faces;
    return h;
}

// Initial data of the problems, evaluated at physical points (the product's problems are new; this
// is the oracle's own statement of them):
//   0 isentropic vortex  p = {cx,cy,cz, ax,ay,az, beta, gamma, ux,uy,uz, period (0: none)}
//   1 density wave       p = {A, kx,ky,kz, ux,uy,uz, p, gamma}
//   2 Taylor-Green       p = {Mach, gamma}
DenseMatrix<5, 1> problem_state(int id, const double* p, const vector3f& x) {
    double rho, u[3], pr, gam;
    if (id == 0) {
        double a[3] = {p[3], p[4], p[5]};
        const double an = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        for (double& v : a) v /= an;
        double d[3];
        for (int i = 0; i < 3; ++i) {
            d[i] = x[i] - p[i];
            if (p[11] > 0) d[i] -= p[11] * std::nearbyint(d[i] / p[11]);
        }
        const double dpa = d[0] * a[0] + d[1] * a[1] + d[2] * a[2];
        const double dp[3] = {d[0] - dpa * a[0], d[1] - dpa * a[1], d[2] - dpa * a[2]};
        const double r2 = dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2];
        const double sw[3] = {a[1] * dp[2] - a[2] * dp[1], a[2] * dp[0] - a[0] * dp[2], a[0] * dp[1] - a[1] * dp[0]};
        const double beta = p[6];
        gam = p[7];
        const double amp = beta / (2 * M_PI) * std::exp(0.5 * (1.0 - r2));
        for (int i = 0; i < 3; ++i) u[i] = p[8 + i] + amp * sw[i];
        const double T = 1.0 - (gam - 1.0) * beta * beta / (8.0 * gam * M_PI * M_PI) * std::exp(1.0 - r2);
        rho = std::pow(T, 1.0 / (gam - 1.0));
        pr = std::pow(rho, gam);
    } else if (id == 1) {
        rho = 1.0 + p[0] * std::sin(2 * M_PI * (p[1] * x[0] + p[2] * x[1] + p[3] * x[2]));
        for (int i = 0; i < 3; ++i) u[i] = p[4 + i];
        pr = p[7];
        gam = p[8];
    } else {
        gam = p[1];
        const double p0 = 1.0 / (gam * p[0] * p[0]);
        rho = 1.0;
        u[0] = std::sin(x[0]) * std::cos(x[1]) * std::cos(x[2]);
        u[1] = -std::cos(x[0]) * std::sin(x[1]) * std::cos(x[2]);
        u[2] = 0.0;
        pr = p0 + (std::cos(2 * x[0]) + std::cos(2 * x[1])) * (std::cos(2 * x[2]) + 2.0) / 16.0;
    }
    const double E = pr / (gam - 1.0) + 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    return {rho, rho * u[0], rho * u[1], rho * u[2], E};
}

// Initial coefficients by the reference's own L2 projection DGBasisEvaluator<P>::func2coef
// (include/DG/DG_Basis/DG_Basis_Evaluator.h:33-59: basis in long double on the Auto tet rule of the
// order), per cell with the state at transform_to_physical(Xi), as the drivers call it
// (examples/cylinder/cylinder_demo/cylinder.cpp:146).
template <uInt P>
int run_project(const ComputingMesh& m, int id, const double* prm, double* U) {
    constexpr uInt N = DGBasisEvaluator<P>::NumBasis;
    const int64_t nc = (int64_t)m.m_cells.size();
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nc; ++c) {
        const auto& cell = m.m_cells[c];
        const auto coef = DGBasisEvaluator<P>::func2coef(
            [&](vector3f Xi) -> DenseMatrix<5, 1> { return problem_state(id, prm, cell.transform_to_physical(Xi)); });
        for (uInt j = 0; j < N; ++j)
            for (uInt k = 0; k < 5; ++k) U[(size_t)c * 5 * N + 5 * j + k] = coef[j](k, 0);
    }
    return 0;
}
}  // namespace

// (order, tet rule, tri rule) combinations instantiated here. X(P, qv, qf, QC, QF)
#define FVEREF_COMBOS(X)                                   \
    X(0, 2, 2, T::Degree5Points15, F::Degree4Points7)      \
    X(1, 0, 1, T::Degree2Points4, F::Degree3Points6)       \
    X(1, 0, 0, T::Degree2Points4, F::Degree3Points4)       \
    X(1, 0, 2, T::Degree2Points4, F::Degree4Points7)       \
    X(1, 2, 2, T::Degree5Points15, F::Degree4Points7)      \
    X(2, 1, 2, T::Degree4Points11, F::Degree4Points7)      \
    X(2, 1, 3, T::Degree4Points11, F::Degree10Points24)    \
    X(2, 2, 3, T::Degree5Points15, F::Degree10Points24)    \
    X(3, 3, 3, T::Degree6Points23, F::Degree10Points24)    \
    X(3, 4, 3, T::Degree7Points31, F::Degree10Points24)    \
    X(4, 5, 3, T::Degree8Points44, F::Degree10Points24)    \
    X(4, 6, 3, T::Degree9Points57, F::Degree10Points24)    \
    X(5, 7, 4, T::Degree11Points94, F::Degree13Points36)

extern "C" {

int fveref_quad_tet(int id, double* pts, double* w) {
    switch (id) {
        case 0: return copy_rule3<T::Degree2Points4>(pts, w);
        case 1: return copy_rule3<T::Degree4Points11>(pts, w);
        case 2: return copy_rule3<T::Degree5Points15>(pts, w);
        case 3: return copy_rule3<T::Degree6Points23>(pts, w);
        case 4: return copy_rule3<T::Degree7Points31>(pts, w);
        case 5: return copy_rule3<T::Degree8Points44>(pts, w);
        case 6: return copy_rule3<T::Degree9Points57>(pts, w);
        case 7: return copy_rule3<T::Degree11Points94>(pts, w);
    }
    return -1;
}

int fveref_quad_tri(int id, double* pts, double* w) {
    switch (id) {
        case 0: return copy_rule2<F::Degree3Points4>(pts, w);
        case 1: return copy_rule2<F::Degree3Points6>(pts, w);
        case 2: return copy_rule2<F::Degree4Points7>(pts, w);
        case 3: return copy_rule2<F::Degree10Points24>(pts, w);
        case 4: return copy_rule2<F::Degree13Points36>(pts, w);
    }
    return -1;
}

int fveref_basis(int order, int npts, const double* xyz, double* phi, double* grad) {
    switch (order) {
        case 0: return run_basis<0>(npts, xyz, phi, grad);
        case 1: return run_basis<1>(npts, xyz, phi, grad);
        case 2: return run_basis<2>(npts, xyz, phi, grad);
        case 3: return run_basis<3>(npts, xyz, phi, grad);
        case 4: return run_basis<4>(npts, xyz, phi, grad);
        case 5: return run_basis<5>(npts, xyz, phi, grad);
    }
    return -1;
}

// Bytes of one element block of LongVector<5*Nb>, i.e. the reference's padded element stride.
size_t fveref_block_bytes(int order) {
    switch (order) {
        case 0: return sizeof(DenseMatrix<5 * DGBasisEvaluator<0>::NumBasis, 1>);
        case 1: return sizeof(DenseMatrix<5 * DGBasisEvaluator<1>::NumBasis, 1>);
        case 2: return sizeof(DenseMatrix<5 * DGBasisEvaluator<2>::NumBasis, 1>);
        case 3: return sizeof(DenseMatrix<5 * DGBasisEvaluator<3>::NumBasis, 1>);
        case 4: return sizeof(DenseMatrix<5 * DGBasisEvaluator<4>::NumBasis, 1>);
        case 5: return sizeof(DenseMatrix<5 * DGBasisEvaluator<5>::NumBasis, 1>);
    }
    return 0;
}

void fveref_set_dirichlet(const double* p10) { std::memcpy(g_dw, p10, sizeof(g_dw)); }
void fveref_set_threads(int n) { omp_set_num_threads(n); }
int fveref_get_threads(void) { return omp_get_max_threads(); }
int fveref_phy_cpu(void) { return get_phy_cpu(); }

// Flat mesh in the DGMesh layout (include/Mesh/MeshGenerator.h:46-57). A face with
// periodic_cell[f] != UINT64_MAX is a periodic face: it is passed to ComputingMesh as a boundary
// face of cells[0] (so its normal is oriented by the boundary rule) and then patched.
void* fveref_mesh_create(uint64_t npts, const double* pts, uint64_t ncell, const uint64_t* cells,
                         const uint64_t* cell_faces, const uint64_t* cell_cells, uint64_t nface,
                         const uint64_t* faces, const uint64_t* face_cells, const uint8_t* bc,
                         const uint64_t* periodic_cell, const uint64_t* periodic_nodes) {
    return build_dgmesh(npts, pts, ncell, cells, cell_faces, cell_cells, nface, faces, face_cells, bc, periodic_cell,
                        periodic_nodes);
}

void fveref_mesh_destroy(void* p) {
    RefMesh* h = static_cast<RefMesh*>(p);
    if (!h) return;
    delete h->cm;
    delete h;
}

void fveref_mesh_export(void* p, double* normals, double* areas, double* natc, uint64_t* fcells,
                        double* invjac, double* detj, double* centroid) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
    for (size_t f = 0; f < m.m_faces.size(); ++f) {
        const auto& fc = m.m_faces[f];
        for (int c = 0; c < 3; ++c) normals[3 * f + c] = fc.m_normal[c];
        areas[f] = fc.m_area;
        for (int s = 0; s < 2; ++s)
            for (int k = 0; k < 3; ++k)
                for (int c = 0; c < 3; ++c) natc[((f * 2 + s) * 3 + k) * 3 + c] = fc.m_natural_coords[s][k][c];
        fcells[2 * f] = fc.m_neighbor_cells[0];
        fcells[2 * f + 1] = fc.m_neighbor_cells[1];
    }
    for (size_t c = 0; c < m.m_cells.size(); ++c) {
        const auto& cl = m.m_cells[c];
        for (int i = 0; i < 9; ++i) invjac[9 * c + i] = cl.m_invJac[i];
        detj[c] = cl.compute_jacobian_det();
        for (int i = 0; i < 3; ++i) centroid[3 * c + i] = cl.m_centroid[i];
    }
}

// gamma_id: 0 = AirFluxC (7/5), 1 = MonatomicFluxC (5/3).
int fveref_eval(void* p, int order, int gamma_id, int qv, int qf, const double* U, double* R,
                double t, int part) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
#define X(P, QV, QF, QC_, QF_)                                                         \
    if (order == P && qv == QV && qf == QF)                                             \
        return gamma_id == 0 ? run_eval<P, AirFluxC, QC_, QF_>(m, U, R, t, part)        \
                             : run_eval<P, MonatomicFluxC, QC_, QF_>(m, U, R, t, part);
    FVEREF_COMBOS(X)
#undef X
    return -1;
}

int fveref_ssprk3(void* p, int order, int gamma_id, int qv, int qf, double* U, const double* mass,
                  double dt, int nsteps, double t0) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
#define X(P, QV, QF, QC_, QF_)                                                                   \
    if (order == P && qv == QV && qf == QF)                                                       \
        return gamma_id == 0 ? run_ssprk3<P, AirFluxC, QC_, QF_>(m, U, mass, dt, nsteps, t0)      \
                             : run_ssprk3<P, MonatomicFluxC, QC_, QF_>(m, U, mass, dt, nsteps, t0);
    FVEREF_COMBOS(X)
#undef X
    return -1;
}

int fveref_diffusion(void* p, int order, int qv, int qf, const double* U, double* R, double t) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
#define X(P, QV, QF, QC_, QF_) \
    if (order == P && qv == QV && qf == QF) return run_diffusion<P, QC_, QF_>(m, U, R, t);
    FVEREF_COMBOS(X)
#undef X
    return -1;
}

// The limiter over the volume rule qv; only_avg selects the neighbour-mean bounds.
int fveref_limit(void* p, int order, int qv, double* Ucur, const double* Uprev, double gamma, int only_avg) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
#define L(P, QC_)                                                                                  \
    return only_avg ? run_limit<P, QC_, true>(m, Ucur, Uprev, gamma) : run_limit<P, QC_, false>(m, Ucur, Uprev, gamma);
    switch (order * 16 + qv) {
        case 1 * 16 + 0: L(1, T::Degree2Points4)
        case 1 * 16 + 2: L(1, T::Degree5Points15)
        case 2 * 16 + 1: L(2, T::Degree4Points11)
        case 2 * 16 + 2: L(2, T::Degree5Points15)
        case 3 * 16 + 3: L(3, T::Degree6Points23)
        case 3 * 16 + 4: L(3, T::Degree7Points31)
        case 4 * 16 + 5: L(4, T::Degree8Points44)
        case 4 * 16 + 6: L(4, T::Degree9Points57)
    }
#undef L
    return -1;
}

int fveref_mass(void* p, int order, int qv, double* mass) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
    switch (order * 16 + qv) {
        case 0 * 16 + 2: return run_mass<0, T::Degree5Points15>(m, mass);
        case 1 * 16 + 0: return run_mass<1, T::Degree2Points4>(m, mass);
        case 1 * 16 + 2: return run_mass<1, T::Degree5Points15>(m, mass);
        case 2 * 16 + 1: return run_mass<2, T::Degree4Points11>(m, mass);
        case 2 * 16 + 2: return run_mass<2, T::Degree5Points15>(m, mass);
        case 3 * 16 + 3: return run_mass<3, T::Degree6Points23>(m, mass);
        case 3 * 16 + 4: return run_mass<3, T::Degree7Points31>(m, mass);
        case 4 * 16 + 5: return run_mass<4, T::Degree8Points44>(m, mass);
        case 4 * 16 + 6: return run_mass<4, T::Degree9Points57>(m, mass);
        case 5 * 16 + 7: return run_mass<5, T::Degree11Points94>(m, mass);
    }
    return -1;
}

// Periodic Kuhn box built by the oracle itself (see build_box), as a reference ComputingMesh.
void* fveref_box_create(int n, const double* lo, const double* hi, double jitter, uint64_t seed, const int* periodic,
                        int bc) {
    if (n < 1 || !lo || !hi || !periodic) return nullptr;
    return build_box(n, lo, hi, jitter, seed, periodic, bc);
}

// The reference's own route OrthHexMesh -> split_hex6_scan -> ComputingMesh(GeneralMesh) (see
// build_orthhex); bc_z / bc_side are BoundaryType values.
void* fveref_orthhex_create(int n, const double* lo, const double* hi, int bc_z, int bc_side) {
    if (n < 1 || !lo || !hi) return nullptr;
    return build_orthhex(n, lo, hi, bc_z, bc_side);
}

// Sizes of a mesh made by fveref_box_create / fveref_orthhex_create: npts, ncell, nface.
int fveref_mesh_sizes(void* p, uint64_t* sizes) {
    const RefMesh* h = static_cast<RefMesh*>(p);
    if (!h || h->cells.empty()) return -1;
    sizes[0] = h->pts.size() / 3;
    sizes[1] = h->cells.size() / 4;
    sizes[2] = h->face_cells.size() / 2;
    return 0;
}

// Its flat topology (DGMesh layout; uInt(-1) for a missing neighbour); any pointer may be NULL.
int fveref_mesh_topology(void* p, double* pts, uint64_t* cells, uint64_t* cell_faces, uint64_t* cell_cells,
                         uint64_t* faces, uint64_t* face_cells, uint64_t* face_nodes1, uint8_t* periodic, uint8_t* bc) {
    const RefMesh* h = static_cast<RefMesh*>(p);
    if (!h || h->cells.empty()) return -1;
    auto put = [](auto* dst, const auto& v) { if (dst) std::copy(v.begin(), v.end(), dst); };
    put(pts, h->pts); put(cells, h->cells); put(cell_faces, h->cell_faces); put(cell_cells, h->cell_cells);
    put(faces, h->faces); put(face_cells, h->face_cells); put(face_nodes1, h->face_nodes1);
    put(periodic, h->periodic); put(bc, h->bc);
    return 0;
}

// func2coef projection of problem `id` (see problem_state) onto the P-basis of every cell.
int fveref_project(void* p, int order, int id, const double* params, double* U) {
    const ComputingMesh& m = *static_cast<RefMesh*>(p)->cm;
    if (id < 0 || id > 2) return -2;
    switch (order) {
        case 0: return run_project<0>(m, id, params, U);
        case 1: return run_project<1>(m, id, params, U);
        case 2: return run_project<2>(m, id, params, U);
        case 3: return run_project<3>(m, id, params, U);
        case 4: return run_project<4>(m, id, params, U);
        case 5: return run_project<5>(m, id, params, U);
    }
    return -1;
}

}  // extern "C"
