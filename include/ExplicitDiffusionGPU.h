// ExplicitDiffusionGPU.h — drop-in for the reference's explicit viscous operator.
//
// A driver that today writes
//     ExplicitDiffusion<Order, QuadC, QuadF> diffusion;                 // ExplicitDiffusion.h:10-626
//     auto k = 1/b * (diffusion.eval(cmesh, x) - convection.eval(cmesh, x));   // test_diffusion.cpp:381
// swaps the class name for ExplicitDiffusionGPU and keeps the call. eval(mesh, U, t) returns the
// interior-penalty viscous residual with the reference's sign and scaling, on a B200 through
// dg_viscous_residual (dg_gpu.h). The reference fixes mu = 1, Pr = 1 and gamma = 1.4; here mu and
// Pr are constructor arguments with those defaults. Dirichlet faces take U_D from the driver's
// rho_Xi .. rhoe_Xi hooks at the call's time, as the reference's eval does. Include after the
// reference's DG and mesh headers, like ExplicitConvectionGPU.h.
#pragma once
#include "ExplicitConvectionGPU.h"

template <uInt Order = 3, typename GaussQuadCell = GaussLegendreTet::Auto,
          typename GaussQuadFace = GaussLegendreTri::Auto>
class ExplicitDiffusionGPU {
public:
    static constexpr uInt N = DGBasisEvaluator<Order>::NumBasis;

    explicit ExplicitDiffusionGPU(int device = 0, double mu = 1.0, double prandtl = 1.0)
        : conv_(device), mu_(mu), prandtl_(prandtl) {}

    LongVector<5 * N> eval(const ComputingMesh& mesh, const LongVector<5 * N>& U, const Scalar t = 0.0) {
        conv_.prepare(mesh, t);
        LongVector<5 * N> R(U.size());
        if (U.size() == 0) return R;
        fvedg_adaptor::check(dg_viscous_residual(conv_.context(), U[0].data_ptr(), R[0].data_ptr(),
                                                 sizeof(DenseMatrix<5 * N, 1>), mu_, prandtl_),
                             "dg_viscous_residual");
        return R;
    }

    dg_ctx* context() { return conv_.context(); }

private:
    ExplicitConvectionGPU<Order, AirFluxC, GaussQuadCell, GaussQuadFace> conv_;  // owns the mesh context
    double mu_, prandtl_;
};
