// Test infrastructure: compiles the C++ drop-ins include/ExplicitConvectionGPU.h,
// ExplicitDiffusionGPU.h and PositiveLimiterGPU.h against the reference's own headers and checks
// them against the reference's ExplicitConvection, ExplicitDiffusion and PositiveLimiter on the same
// ComputingMesh, the way a driver would swap the classes: on Kuhn boxes passed through
// ComputingMesh(const DGMesh&), and on the reference's own OrthHexMesh + split_hex6_scan mesh passed
// through ComputingMesh(const GeneralMesh&). Built by `make -C oracle ref` into
// oracle/_ref/adaptor_check (linked to fve_dg_b200/libfvedg_b200.so); run by
// tests/test_gpu_adaptor.py on a GPU. Exit status 0 when every case agrees to 1e-12 (relative L2).
#include "DG/DG_Schemes/ExplicitConvection.h"
#include "DG/DG_Schemes/ExplicitDiffusion.h"
#include "DG/DG_Schemes/PositiveLimiter.h"
#include "src/DG/DG_Schemes/ExplicitConvection.cpp"

#include <cstdio>
#include <random>

#include "ExplicitConvectionGPU.h"
#include "ExplicitDiffusionGPU.h"
#include "PositiveLimiterGPU.h"

// Problem hooks of include/base/exact.h:32-52 (a travelling density wave) for Dirichlet faces.
namespace {
double wave(const CompTetrahedron& cell, const vector3f& Xi, double t, int k) {
    const vector3f x = cell.transform_to_physical(Xi);
    const double u = 1.0, v = 0.5, w = 0.25, p = 1.0, gam = 1.4;
    const double rho = 1.0 + 0.2 * std::sin(2.0 * M_PI * ((x[0] - u * t) + (x[1] - v * t) + (x[2] - w * t)));
    const double s[5] = {rho, rho * u, rho * v, rho * w, p / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w)};
    return s[k];
}
}  // namespace
Scalar rho_Xi(const CompTetrahedron& c, const vector3f& Xi, Scalar t) { return wave(c, Xi, t, 0); }
Scalar rhou_Xi(const CompTetrahedron& c, const vector3f& Xi, Scalar t) { return wave(c, Xi, t, 1); }
Scalar rhov_Xi(const CompTetrahedron& c, const vector3f& Xi, Scalar t) { return wave(c, Xi, t, 2); }
Scalar rhow_Xi(const CompTetrahedron& c, const vector3f& Xi, Scalar t) { return wave(c, Xi, t, 3); }
Scalar rhoe_Xi(const CompTetrahedron& c, const vector3f& Xi, Scalar t) { return wave(c, Xi, t, 4); }

namespace T = GaussLegendreTet;
namespace F = GaussLegendreTri;

static ComputingMesh* make_mesh(int n, BoundaryType bt) {
    const double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    const int periodic[3] = {0, 0, 0};
    int err = 0;
    dg_box_mesh* bm = dg_box_mesh_create(n, lo, hi, 0.1, 5, periodic, (int)bt, &err);
    if (!bm) return nullptr;
    dg_mesh_desc d{};
    const int64_t *cf = nullptr, *cc = nullptr;
    dg_box_mesh_view(bm, &d, &cf, &cc);
    DGMesh g;
    for (int64_t i = 0; i < d.npts; ++i) g.points.push_back({d.points[3 * i], d.points[3 * i + 1], d.points[3 * i + 2]});
    for (int64_t c = 0; c < d.ncell; ++c) {
        g.cells.push_back({(size_t)d.cell_nodes[4 * c], (size_t)d.cell_nodes[4 * c + 1], (size_t)d.cell_nodes[4 * c + 2],
                           (size_t)d.cell_nodes[4 * c + 3]});
        g.cell_faces.push_back({(size_t)cf[4 * c], (size_t)cf[4 * c + 1], (size_t)cf[4 * c + 2], (size_t)cf[4 * c + 3]});
        g.cell_cells.push_back({(size_t)cc[4 * c], (size_t)cc[4 * c + 1], (size_t)cc[4 * c + 2], (size_t)cc[4 * c + 3]});
    }
    for (int64_t f = 0; f < d.nface; ++f) {
        g.faces.push_back({(size_t)d.face_nodes[3 * f], (size_t)d.face_nodes[3 * f + 1], (size_t)d.face_nodes[3 * f + 2]});
        g.face_cells.push_back({(size_t)d.face_cells[2 * f], (size_t)d.face_cells[2 * f + 1]});
        g.is_boundary_face.push_back(d.face_cells[2 * f + 1] < 0);
    }
    dg_box_mesh_destroy(bm);
    ComputingMesh* m = new ComputingMesh(g);
    m->m_boundaryTypes.assign(m->m_faces.size(), bt);
    return m;
}

// The reference's own route, as its drivers build a box (examples/Vortex/123/Vortex.cpp:101-106):
// OrthHexMesh -> split_hex6_scan -> rebuild_cell_topology -> validate_mesh -> ComputingMesh(GeneralMesh);
// boundary faces with |n_z| > 0.5 get Pseudo3DZ, the others bt.
static ComputingMesh* make_mesh_orthhex(int n, BoundaryType bt) {
    GeneralMesh g = OrthHexMesh({0.0, 0.0, 0.0}, {1.0, 1.0, 0.5}, {(uInt)n, (uInt)n, (uInt)n});
    g.split_hex6_scan();
    g.rebuild_cell_topology();
    g.validate_mesh();
    ComputingMesh* m = new ComputingMesh(g);
    m->m_boundaryTypes.assign(m->m_faces.size(), BoundaryType::Pseudo3DZ);
    for (size_t f = 0; f < m->m_faces.size(); ++f)
        if (m->m_faces[f].m_neighbor_cells[1] == uInt(-1) && std::abs(m->m_faces[f].m_normal[2]) <= 0.5)
            m->m_boundaryTypes[f] = bt;
    return m;
}

template <uInt P, class QC, class QF>
static int check(const ComputingMesh& m, const char* name) {
    constexpr uInt N = DGBasisEvaluator<P>::NumBasis;
    LongVector<5 * N> U(m.m_cells.size());
    std::mt19937_64 rng(P * 17 + 3);
    std::uniform_real_distribution<double> uni(-1e-2, 1e-2);
    for (size_t c = 0; c < m.m_cells.size(); ++c) {
        U[c](0, 0) = 1.0;
        U[c](4, 0) = 2.5;
        for (uInt i = 0; i < 5 * N; ++i) U[c](i, 0) += uni(rng);
    }
    ExplicitConvection<P, AirFluxC, QC, QF> ref;
    ExplicitConvectionGPU<P, AirFluxC, QC, QF> gpu;
    int bad = 0;
    for (int part = 0; part < 4; ++part) {
        const double t = 0.125;
        LongVector<5 * N> a = part == 0 ? ref.eval(m, U, t) : part == 1 ? ref.eval_cells(m, U, t)
                              : part == 2 ? ref.eval_internals(m, U, t) : ref.eval_boundarys(m, U, t);
        LongVector<5 * N> b = part == 0 ? gpu.eval(m, U, t) : part == 1 ? gpu.eval_cells(m, U, t)
                              : part == 2 ? gpu.eval_internals(m, U, t) : gpu.eval_boundarys(m, U, t);
        double num = 0, den = 0;
        for (size_t c = 0; c < m.m_cells.size(); ++c)
            for (uInt i = 0; i < 5 * N; ++i) {
                const double d = a[c](i, 0) - b[c](i, 0);
                num += d * d;
                den += a[c](i, 0) * a[c](i, 0);
            }
        const double rel = den > 0 ? std::sqrt(num / den) : std::sqrt(num);
        std::printf("%s P%d part %d rel L2 %.3e\n", name, (int)P, part, rel);
        if (!(rel < 1e-12)) ++bad;
    }
    return bad;
}

template <uInt N>
static double rel_l2(const LongVector<5 * N>& a, const LongVector<5 * N>& b) {
    double num = 0, den = 0;
    for (size_t c = 0; c < a.size(); ++c)
        for (uInt i = 0; i < 5 * N; ++i) {
            const double d = a[c](i, 0) - b[c](i, 0);
            num += d * d;
            den += a[c](i, 0) * a[c](i, 0);
        }
    return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}

// ExplicitDiffusionGPU against ExplicitDiffusion (mu = Pr = 1, as the reference fixes them).
template <uInt P, class QC, class QF>
static int check_diffusion(const ComputingMesh& m, const char* name) {
    constexpr uInt N = DGBasisEvaluator<P>::NumBasis;
    LongVector<5 * N> U(m.m_cells.size());
    std::mt19937_64 rng(P * 29 + 5);
    std::uniform_real_distribution<double> uni(-1e-2, 1e-2);
    for (size_t c = 0; c < m.m_cells.size(); ++c) {
        U[c](0, 0) = 1.0;
        U[c](4, 0) = 2.5;
        for (uInt i = 0; i < 5 * N; ++i) U[c](i, 0) += uni(rng);
    }
    ExplicitDiffusion<P, QC, QF> ref;
    ExplicitDiffusionGPU<P, QC, QF> gpu;
    const double t = 0.125;
    const double rel = rel_l2<N>(ref.eval(m, U, t), gpu.eval(m, U, t));
    std::printf("%s diffusion P%d rel L2 %.3e\n", name, (int)P, rel);
    return rel < 1e-12 ? 0 : 1;
}

// PositiveLimiterGPU against PositiveLimiter: constructMinMax(current, previous), apply(current,
// previous) on a state whose modes leave the bounds and whose points go non-physical.
template <uInt P, class QC, bool Avg>
static int check_limiter(const ComputingMesh& m, const char* name) {
    constexpr uInt N = DGBasisEvaluator<P>::NumBasis;
    const size_t nc = m.m_cells.size();
    LongVector<5 * N> prev(nc), cur(nc);
    std::mt19937_64 rng(P * 31 + (Avg ? 7 : 3));
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    for (size_t c = 0; c < nc; ++c) {
        prev[c](0, 0) = 1.0 + 0.05 * uni(rng);
        prev[c](4, 0) = 2.5 + 0.05 * uni(rng);
        for (uInt i = 5; i < 5 * N; ++i) prev[c](i, 0) = 0.01 * uni(rng);
        cur[c] = prev[c];
        for (uInt i = 5; i < 5 * N; ++i) cur[c](i, 0) += 0.4 * uni(rng);
    }
    LongVector<5 * N> a = cur, b = cur;
    PositiveLimiter<P, QC, Avg> ref(m, 1.4);
    ref.constructMinMax(a, prev);
    ref.apply(a, prev);
    PositiveLimiterGPU<P, QC, Avg> gpu(m, 1.4);
    gpu.constructMinMax(b, prev);
    gpu.apply(b, prev);
    const double rel = rel_l2<N>(a, b), acted = rel_l2<N>(a, cur);
    std::printf("%s limiter P%d avg %d rel L2 %.3e (limited vs input %.3e)\n", name, (int)P, (int)Avg, rel, acted);
    return (rel < 1e-12 && acted > 1e-3) ? 0 : 1;
}

int main() {
    int bad = 0;
    for (int which = 0; which < 3; ++which) {
        const BoundaryType bt = which == 1 ? BoundaryType::Pseudo3DZ : BoundaryType::Dirichlet;
        ComputingMesh* m = which < 2 ? make_mesh(2, bt) : make_mesh_orthhex(3, bt);
        if (!m) return 2;
        const char* name = which == 0 ? "dirichlet" : which == 1 ? "pseudo3dz" : "orthhex-split6";
        bad += check<1, T::Degree2Points4, F::Degree3Points6>(*m, name);
        bad += check<2, T::Degree4Points11, F::Degree4Points7>(*m, name);
        bad += check<3, T::Degree6Points23, F::Degree10Points24>(*m, name);
        bad += check<4, T::Degree8Points44, F::Degree10Points24>(*m, name);
        bad += check<3, GaussLegendreTet::Auto, GaussLegendreTri::Auto>(*m, name);
        bad += check<0, GaussLegendreTet::Auto, GaussLegendreTri::Auto>(*m, name);
        bad += check<5, GaussLegendreTet::Auto, GaussLegendreTri::Auto>(*m, name);
        bad += check_diffusion<1, T::Degree2Points4, F::Degree3Points6>(*m, name);
        bad += check_diffusion<2, T::Degree4Points11, F::Degree4Points7>(*m, name);
        bad += check_diffusion<3, T::Degree6Points23, F::Degree10Points24>(*m, name);
        bad += check_limiter<2, T::Degree4Points11, false>(*m, name);
        bad += check_limiter<3, T::Degree6Points23, false>(*m, name);
        bad += check_limiter<3, T::Degree6Points23, true>(*m, name);
        delete m;
    }
    std::printf("%s\n", bad ? "FAIL" : "OK");
    return bad ? 1 : 0;
}
