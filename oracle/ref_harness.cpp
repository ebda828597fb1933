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
#include "DG/DG_Schemes/ExplicitConvection.h"
#include "DG/DG_Schemes/ExplicitDiffusion.h"
#include "DG/DG_Schemes/PositiveLimiter.h"
#include "src/DG/DG_Schemes/ExplicitConvection.cpp"

#include <cstdint>
#include <cstring>
#include <omp.h>

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
struct RefMesh {
    ComputingMesh* cm = nullptr;
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

// (order, tet rule, tri rule) combinations instantiated here. X(P, qv, qf, QC, QF)
#define FVEREF_COMBOS(X)                                   \
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
    X(4, 6, 3, T::Degree9Points57, F::Degree10Points24)

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
    }
    return -1;
}

int fveref_quad_tri(int id, double* pts, double* w) {
    switch (id) {
        case 0: return copy_rule2<F::Degree3Points4>(pts, w);
        case 1: return copy_rule2<F::Degree3Points6>(pts, w);
        case 2: return copy_rule2<F::Degree4Points7>(pts, w);
        case 3: return copy_rule2<F::Degree10Points24>(pts, w);
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
        case 1: return sizeof(DenseMatrix<5 * DGBasisEvaluator<1>::NumBasis, 1>);
        case 2: return sizeof(DenseMatrix<5 * DGBasisEvaluator<2>::NumBasis, 1>);
        case 3: return sizeof(DenseMatrix<5 * DGBasisEvaluator<3>::NumBasis, 1>);
        case 4: return sizeof(DenseMatrix<5 * DGBasisEvaluator<4>::NumBasis, 1>);
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
        case 1 * 16 + 0: return run_mass<1, T::Degree2Points4>(m, mass);
        case 1 * 16 + 2: return run_mass<1, T::Degree5Points15>(m, mass);
        case 2 * 16 + 1: return run_mass<2, T::Degree4Points11>(m, mass);
        case 2 * 16 + 2: return run_mass<2, T::Degree5Points15>(m, mass);
        case 3 * 16 + 3: return run_mass<3, T::Degree6Points23>(m, mass);
        case 3 * 16 + 4: return run_mass<3, T::Degree7Points31>(m, mass);
        case 4 * 16 + 5: return run_mass<4, T::Degree8Points44>(m, mass);
        case 4 * 16 + 6: return run_mass<4, T::Degree9Points57>(m, mass);
    }
    return -1;
}

}  // extern "C"
