// ExplicitConvectionGPU.h — drop-in for the reference's explicit convection operator.
//
// A driver that today writes
//     ExplicitConvection<Order, Flux, QuadC, QuadF> conv;            // ExplicitConvection.h:9-45
//     auto R = conv.eval(cmesh, U, t);                              // ExplicitConvection.cpp:136-141
// swaps the class name for ExplicitConvectionGPU and keeps the same call; eval_cells,
// eval_internals and eval_boundarys are there too. The operator runs on a B200 through the C ABI
// of dg_gpu.h. Include this header after the reference's DG and mesh headers (it uses
// ComputingMesh, LongVector, DenseMatrix, DGBasisEvaluator and the GaussQuadrature rule types).
//
// The first eval on a mesh uploads it with the geometry the reference's ComputingMesh already
// holds (m_neighbor_cells, m_natural_coords, m_normal, m_area, m_invJac, compute_jacobian_det),
// so the device sees exactly the reference's numbers. Dirichlet faces take U_D from the driver's
// rho_Xi .. rhoe_Xi hooks (include/base/exact.h:32-52) at every face point and time, as
// ExplicitConvection.cpp:47-53 does.
#pragma once
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "dg_gpu.h"

namespace fvedg_adaptor {

template <class Q> struct rule_id { static constexpr int value = -2; };  // unsupported rule
template <> struct rule_id<GaussLegendreTet::Auto> { static constexpr int value = -1; };
template <> struct rule_id<GaussLegendreTri::Auto> { static constexpr int value = -1; };
template <> struct rule_id<GaussLegendreTet::Degree2Points4> { static constexpr int value = DG_TET_D2P4; };
template <> struct rule_id<GaussLegendreTet::Degree4Points11> { static constexpr int value = DG_TET_D4P11; };
template <> struct rule_id<GaussLegendreTet::Degree5Points15> { static constexpr int value = DG_TET_D5P15; };
template <> struct rule_id<GaussLegendreTet::Degree6Points23> { static constexpr int value = DG_TET_D6P23; };
template <> struct rule_id<GaussLegendreTet::Degree7Points31> { static constexpr int value = DG_TET_D7P31; };
template <> struct rule_id<GaussLegendreTet::Degree8Points44> { static constexpr int value = DG_TET_D8P44; };
template <> struct rule_id<GaussLegendreTet::Degree9Points57> { static constexpr int value = DG_TET_D9P57; };
template <> struct rule_id<GaussLegendreTet::Degree11Points94> { static constexpr int value = DG_TET_D11P94; };
template <> struct rule_id<GaussLegendreTri::Degree3Points4> { static constexpr int value = DG_TRI_D3P4; };
template <> struct rule_id<GaussLegendreTri::Degree3Points6> { static constexpr int value = DG_TRI_D3P6; };
template <> struct rule_id<GaussLegendreTri::Degree4Points7> { static constexpr int value = DG_TRI_D4P7; };
template <> struct rule_id<GaussLegendreTri::Degree10Points24> { static constexpr int value = DG_TRI_D10P24; };
template <> struct rule_id<GaussLegendreTri::Degree13Points36> { static constexpr int value = DG_TRI_D13P36; };

inline void check(int rc, const char* what) {
    if (rc == DG_E_CUDA)
        throw std::runtime_error(std::string(what) + ": " + dg_status_string(rc) + " (" + dg_last_cuda_error() + ")");
    if (rc != DG_OK) throw std::runtime_error(std::string(what) + ": " + dg_status_string(rc));
}

}  // namespace fvedg_adaptor

template <uInt Order = 3, typename Flux = AirFluxC, typename GaussQuadCell = GaussLegendreTet::Auto,
          typename GaussQuadFace = GaussLegendreTri::Auto>
class ExplicitConvectionGPU {
    using Basis = DGBasisEvaluator<Order>;
    using QuadF = typename std::conditional_t<std::is_same_v<GaussQuadFace, GaussLegendreTri::Auto>,
                                              typename AutoQuadSelector<Order, GaussLegendreTri::Auto>::type,
                                              GaussQuadFace>;
    static constexpr int kVol = fvedg_adaptor::rule_id<GaussQuadCell>::value;
    static constexpr int kFace = fvedg_adaptor::rule_id<GaussQuadFace>::value;
    static_assert(kVol != -2 && kFace != -2, "quadrature rule not supported by the B200 operator");
    static_assert(Order <= 5, "the B200 operator covers P0..P5 (the orders ExplicitConvection.cpp:5-16 instantiates)");

public:
    static constexpr uInt N = Basis::NumBasis;

    explicit ExplicitConvectionGPU(int device = 0, int precision = DG_PREC_FP64, int flux = DG_FLUX_LF,
                                   double gamma = Flux::gamma)
        : device_(device), precision_(precision), flux_(flux), gamma_(gamma) {}
    ~ExplicitConvectionGPU() { release(); }
    ExplicitConvectionGPU(const ExplicitConvectionGPU&) = delete;
    ExplicitConvectionGPU& operator=(const ExplicitConvectionGPU&) = delete;

    LongVector<5 * N> eval(const ComputingMesh& mesh, const LongVector<5 * N>& U, const Scalar t = 0.0) {
        return run(mesh, U, t, 0);
    }
    LongVector<5 * N> eval_cells(const ComputingMesh& mesh, const LongVector<5 * N>& U, const Scalar t = 0.0) {
        return run(mesh, U, t, 1);
    }
    LongVector<5 * N> eval_internals(const ComputingMesh& mesh, const LongVector<5 * N>& U, const Scalar t = 0.0) {
        return run(mesh, U, t, 2);
    }
    LongVector<5 * N> eval_boundarys(const ComputingMesh& mesh, const LongVector<5 * N>& U, const Scalar t = 0.0) {
        return run(mesh, U, t, 3);
    }

    dg_ctx* context() { return ctx_; }
    // The context for `mesh` (made on the first call for a mesh) with the Dirichlet data at time t:
    // what eval does before it evaluates; ExplicitDiffusionGPU and PositiveLimiterGPU use it.
    void prepare(const ComputingMesh& mesh, Scalar t = 0.0) {
        if (!ctx_ || mesh_ != &mesh) upload(mesh);
        dirichlet(mesh, t);
    }

private:
    int device_, precision_, flux_;
    double gamma_;
    dg_ctx* ctx_ = nullptr;
    const ComputingMesh* mesh_ = nullptr;
    std::vector<int64_t> dirichlet_faces_;

    void release() {
        if (ctx_) dg_destroy(ctx_);
        ctx_ = nullptr;
        mesh_ = nullptr;
    }

    void upload(const ComputingMesh& mesh) {
        release();
        const size_t nf = mesh.m_faces.size(), nc = mesh.m_cells.size();
        std::vector<int64_t> fc(2 * nf);
        std::vector<uint8_t> bc(nf, DG_BC_PSEUDO3DZ);
        std::vector<double> nat(18 * nf), nrm(3 * nf), area(nf), invj(9 * nc), detj(nc);
        dirichlet_faces_.clear();
        for (size_t f = 0; f < nf; ++f) {
            const auto& F = mesh.m_faces[f];
            fc[2 * f] = (int64_t)F.m_neighbor_cells[0];
            fc[2 * f + 1] = F.m_neighbor_cells[1] == uInt(-1) ? DG_NO_CELL : (int64_t)F.m_neighbor_cells[1];
            if (f < mesh.m_boundaryTypes.size()) bc[f] = (uint8_t)mesh.m_boundaryTypes[f];
            if (fc[2 * f + 1] == DG_NO_CELL && bc[f] == DG_BC_DIRICHLET) dirichlet_faces_.push_back((int64_t)f);
            for (int s = 0; s < 2; ++s)
                for (int k = 0; k < 3; ++k)
                    for (int c = 0; c < 3; ++c) nat[18 * f + 9 * s + 3 * k + c] = F.m_natural_coords[s][k][c];
            for (int c = 0; c < 3; ++c) nrm[3 * f + c] = F.m_normal[c];
            area[f] = F.m_area;
        }
        for (size_t c = 0; c < nc; ++c) {
            const auto& C = mesh.m_cells[c];
            for (int i = 0; i < 9; ++i) invj[9 * c + i] = C.m_invJac[i];
            detj[c] = C.compute_jacobian_det();
        }
        dg_mesh_desc d{};
        d.ncell = (int64_t)nc;
        d.nface = (int64_t)nf;
        d.face_cells = fc.data();
        d.face_bc = bc.data();
        d.face_natural = nat.data();
        d.face_normal = nrm.data();
        d.face_area = area.data();
        d.cell_invjac = invj.data();
        d.cell_detj = detj.data();
        dg_config cfg{};
        cfg.order = (int)Order;
        cfg.flux = flux_;
        cfg.quad_vol = kVol;
        cfg.quad_face = kFace;
        cfg.gamma = gamma_;
        cfg.precision = precision_;
        cfg.device = device_;
        int err = DG_OK;
        ctx_ = dg_create(&d, &cfg, &err);
        fvedg_adaptor::check(err, "dg_create");
        mesh_ = &mesh;
    }

    // U_D at every face point of every Dirichlet face from the driver's hooks (exact.h:32-52),
    // evaluated where ExplicitConvection.cpp:34-53 evaluates them.
    void dirichlet(const ComputingMesh& mesh, Scalar t) {
        if (dirichlet_faces_.empty()) return;
        const size_t nq = QuadF::num_points;
        std::vector<double> UD(mesh.m_faces.size() * nq * 5, 0.0);
        for (int64_t f : dirichlet_faces_) {
            const auto& F = mesh.m_faces[f];
            const auto& cell = mesh.m_cells[F.m_neighbor_cells[0]];
            for (size_t g = 0; g < nq; ++g) {
                const auto& uv = QuadF::points[g];
                const auto& nc = F.m_natural_coords[0];
                const vector3f xi = nc[0] * (1 - uv[0] - uv[1]) + nc[1] * uv[0] + nc[2] * uv[1];
                double* o = &UD[(f * nq + g) * 5];
                o[0] = rho_Xi(cell, xi, t);
                o[1] = rhou_Xi(cell, xi, t);
                o[2] = rhov_Xi(cell, xi, t);
                o[3] = rhow_Xi(cell, xi, t);
                o[4] = rhoe_Xi(cell, xi, t);
            }
        }
        fvedg_adaptor::check(dg_set_dirichlet(ctx_, UD.data()), "dg_set_dirichlet");
    }

    LongVector<5 * N> run(const ComputingMesh& mesh, const LongVector<5 * N>& U, Scalar t, int part) {
        prepare(mesh, t);
        LongVector<5 * N> R(U.size());
        if (U.size() == 0) return R;
        fvedg_adaptor::check(dg_residual(ctx_, U[0].data_ptr(), R[0].data_ptr(), sizeof(DenseMatrix<5 * N, 1>), t, part),
                             "dg_residual");
        return R;
    }
};
