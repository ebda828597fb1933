// PositiveLimiterGPU.h — drop-in for the reference's positivity-preserving limiter.
//
// A driver that today writes
//     PositiveLimiter<Order, QuadC, OnlyNeigbAvg> limiter(cmesh, gamma);   // PositiveLimiter.h:12-36
//     limiter.constructMinMax(ddx, dx);                                    // Riemann1D.cpp:194
//     limiter.apply(ddx, dx);                                              // Riemann1D.cpp:195
// swaps the class name for PositiveLimiterGPU and keeps the calls. As in the reference, the bounds
// come from the `previous` state given to constructMinMax (it keeps a copy here) and apply limits
// `current` in place; apply without an earlier constructMinMax takes them from its own `previous`.
// The three limiting steps run on a B200 through dg_limit (dg_gpu.h). Include after the
// reference's DG and mesh headers, like ExplicitConvectionGPU.h.
#pragma once
#include "ExplicitConvectionGPU.h"

template <uInt Order, typename QuadType, bool OnlyNeigbAvg = false>
class PositiveLimiterGPU {
public:
    static constexpr uInt N = DGBasisEvaluator<Order>::NumBasis;

    PositiveLimiterGPU(const ComputingMesh& mesh, Scalar gamma = 1.4, int device = 0)
        : mesh_(mesh), conv_(device, DG_PREC_FP64, DG_FLUX_LF, gamma) {}

    void constructMinMax(LongVector<5 * N>& /*current_coeffs*/, const LongVector<5 * N>& previous_coeffs) {
        bounds_ = previous_coeffs;
        have_bounds_ = true;
    }

    void apply(LongVector<5 * N>& current_coeffs, const LongVector<5 * N>& previous_coeffs) {
        if (current_coeffs.size() == 0) return;
        conv_.prepare(mesh_);
        const LongVector<5 * N>& from = have_bounds_ ? bounds_ : previous_coeffs;
        fvedg_adaptor::check(dg_limit(conv_.context(), current_coeffs[0].data_ptr(), from[0].data_ptr(),
                                      sizeof(DenseMatrix<5 * N, 1>), OnlyNeigbAvg ? 1 : 0),
                             "dg_limit");
    }

    dg_ctx* context() { return conv_.context(); }

private:
    const ComputingMesh& mesh_;
    ExplicitConvectionGPU<Order, AirFluxC, QuadType, GaussLegendreTri::Auto> conv_;  // owns the mesh context
    LongVector<5 * N> bounds_;
    bool have_bounds_ = false;
};
