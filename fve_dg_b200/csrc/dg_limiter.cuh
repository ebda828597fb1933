// Positivity-preserving two-step limiter, after include/DG/DG_Schemes/PositiveLimiter.h:12-261, as
// the reference's drivers call it: constructMinMax(current, previous) then apply(current, previous)
// (examples/Eular1D/Sod1D/Riemann1D.cpp:194-195). FP64 in both forms.
//
//   bounds (constructMinMax, :57-103): per face, both cells' previous states evaluated at the
//     volume rule's reference points; max over points of max(v1, v2) per variable, and - as the
//     reference computes it (:86) - the min is min(v1, v2) at the last point. With only_avg the
//     bounds are the max/min of the two cells' means. A boundary face uses its one cell twice.
//     Each cell's bounds are the max/min over its faces.
//   step 1 (apply_1_limitCell, :128-163): per variable, if the quadrature values leave the cell's
//     bounds, scale the modes l >= 1 by min(theta_min, theta_max, 1) with
//     theta_min = (avg - min_b) / (avg - v_min + 1e-32), theta_max = (max_b - avg) / (v_max - avg + 1e-32).
//   step 2 (apply_21_limitCell, :164-188): density kept >= 1e-16 at the points by scaling its modes.
//   step 3 (apply_22_limitCell, :189-258): for every point with negative pressure, 100 bisection
//     steps on t in [0, 1] for p((1 - t) avg + t U(x_g)) = 0; all modes l >= 1 scaled by the
//     smallest t.
// Means are never changed, so mass, momentum and energy are conserved exactly.
//
// Two passes, one warp per cell, lanes over the quadrature points (each point value summed over the
// modes in order, as the reference does): per-cell statistics of the previous state, then the bounds
// and the three steps. Warps never wait on one another.
#pragma once
#include <cfloat>

#include "dg_kernels_fp64.cuh"
#include "dg_kernels_mixed.cuh"

namespace fvedg {

__device__ __forceinline__ double ref_max(double a, double b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ double ref_min(double a, double b) { return (b < a) ? b : a; }  // std::min

__device__ __forceinline__ double warp_max(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = ref_max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = ref_min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <int NB>
__device__ __forceinline__ double point_value(const double* phi_g, const double* u, int k) {
    double v = 0.0;
    #pragma unroll 5
    for (int l = 0; l < NB; ++l) v = fma(phi_g[l], u[k + 5 * l], v);
    return v;
}

// PositiveLimiter.h:112-123
__device__ __forceinline__ double limiter_pressure(const double U[5], double gamma) {
    const double rho = U[0];
    if (rho <= 1e-16) return -1.0;
    const double ke = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / (2.0 * rho);
    return (gamma - 1.0) * (U[4] - ke);
}

constexpr int kLimWarps = 4;
constexpr int kLimMaxPts = 64;  // volume points a warp holds, two per lane (the largest rule has 57)

// The 5 conserved values at volume point g.
template <int NB>
__device__ __forceinline__ void point_values(const double* phi_g, const double* u, double v[5]) {
    #pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = 0.0;
    for (int l = 0; l < NB; ++l) {
        const double p = phi_g[l];
        #pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = fma(p, u[k + 5 * l], v[k]);
    }
}

// Per-cell statistics of the previous state for the bounds: the max over the volume points of
// each variable and the values at the last point. A face's bounds are max(v1, v2) over the points
// and min(v1, v2) at the last point (PositiveLimiter.h:77-88), i.e. the max of its two cells' maxima
// and the min of their last-point values; with only_avg both are the cell mean (:70-75).
template <int NB, int NQV>
__global__ void __launch_bounds__(kLimWarps * 32)
    limiter_cell_stats(const double* __restrict__ Up, const double* __restrict__ phi, int64_t ncell, int only_avg,
                       double* __restrict__ stats) {
    __shared__ double sphi[NQV * NB];
    __shared__ double scoef[kLimWarps][5 * NB];
    for (int i = threadIdx.x; i < NQV * NB; i += blockDim.x) sphi[i] = phi[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    double* su = scoef[threadIdx.x >> 5];
    for (int64_t c = (int64_t)blockIdx.x * kLimWarps + (threadIdx.x >> 5); c < ncell;
         c += (int64_t)gridDim.x * kLimWarps) {
        const double* ug = Up + c * (5 * NB);
        for (int i = lane; i < 5 * NB; i += 32) su[i] = ug[i];  // coalesced, then broadcast reads
        __syncwarp();
        const double* u = su;
        double* out = stats + c * 10;
        if (only_avg) {
            if (lane < 5) { out[lane] = u[lane]; out[5 + lane] = u[lane]; }
            __syncwarp();
            continue;
        }
        double mx[5], last[5];
        #pragma unroll
        for (int k = 0; k < 5; ++k) { mx[k] = -DBL_MAX; last[k] = 0.0; }
        for (int g = lane; g < NQV; g += 32) {
            double v[5];
            point_values<NB>(sphi + g * NB, u, v);
            #pragma unroll
            for (int k = 0; k < 5; ++k) {
                mx[k] = ref_max(mx[k], v[k]);
                if (g == NQV - 1) last[k] = v[k];
            }
        }
        #pragma unroll
        for (int k = 0; k < 5; ++k) {
            mx[k] = warp_max(mx[k]);
            last[k] = __shfl_sync(0xffffffffu, last[k], (NQV - 1) % 32);
        }
        if (lane < 5) {
            double a = mx[0], b = last[0];
            #pragma unroll
            for (int k = 1; k < 5; ++k)
                if (lane == k) { a = mx[k]; b = last[k]; }
            out[lane] = a;
            out[5 + lane] = b;
        }
        __syncwarp();
    }
}

// The three steps per element (PositiveLimiter.h:128-258). Point values are evaluated once; after a
// step scales the modes l >= 1 of a variable by theta, its point values become avg + theta (v - avg)
// (phi_0 = 1), which is what the reference re-evaluates. mir: when non-null, the element's split
// coefficient rows (A rows, [ncell][5][KB]) are rewritten if the limiter changed the element.
template <int NB, int NQV>
__global__ void __launch_bounds__(kLimWarps * 32)
    limiter_apply(double* __restrict__ U, const ElemFace* __restrict__ ef, const FaceInfo* __restrict__ fi,
                  const double* __restrict__ stats, const double* __restrict__ phi, int64_t ncell, double gamma,
                  uint32_t* __restrict__ mir) {
    constexpr int KB = pad8(NB - 1);
    constexpr int PPL = (NQV + 31) / 32;  // points per lane
    static_assert(NQV <= kLimMaxPts, "volume rule too large");
    __shared__ double sphi[NQV * NB];
    __shared__ double scoef[kLimWarps][5 * NB];
    for (int i = threadIdx.x; i < NQV * NB; i += blockDim.x) sphi[i] = phi[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    double* u = scoef[threadIdx.x >> 5];
    for (int64_t e = (int64_t)blockIdx.x * kLimWarps + (threadIdx.x >> 5); e < ncell;
         e += (int64_t)gridDim.x * kLimWarps) {
        double* ug = U + e * (5 * NB);
        for (int i = lane; i < 5 * NB; i += 32) u[i] = ug[i];  // coalesced, then broadcast reads
        __syncwarp();
        // the cell's bounds over its faces (constructMinMax, :92-102); a boundary face has one cell
        double gmax = -DBL_MAX, gmin = DBL_MAX;
        if (lane < 5) {
            #pragma unroll
            for (int q = 0; q < 4; ++q) {
                const FaceInfo& F = fi[ef[4 * e + q].face];
                const int64_t c0 = F.c0, c1 = F.c1 >= 0 ? F.c1 : F.c0;
                gmax = ref_max(gmax, ref_max(stats[c0 * 10 + lane], stats[c1 * 10 + lane]));
                gmin = ref_min(gmin, ref_min(stats[c0 * 10 + 5 + lane], stats[c1 * 10 + 5 + lane]));
            }
        }
        double avg[5], v[PPL][5];
        #pragma unroll
        for (int k = 0; k < 5; ++k) avg[k] = u[k];
        #pragma unroll
        for (int r = 0; r < PPL; ++r) {
            const int g = lane + 32 * r;
            if (g < NQV) point_values<NB>(sphi + g * NB, u, v[r]);
            else
                #pragma unroll
                for (int k = 0; k < 5; ++k) v[r][k] = avg[k];  // neutral for min/max and pressure
        }
        double scale[5] = {1.0, 1.0, 1.0, 1.0, 1.0};
        bool changed = false;
        // step 1: each variable within the cell's bounds
        #pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double bmax = __shfl_sync(0xffffffffu, gmax, k), bmin = __shfl_sync(0xffffffffu, gmin, k);
            double vmin = DBL_MAX, vmax = -DBL_MAX;
            #pragma unroll
            for (int r = 0; r < PPL; ++r)
                if (lane + 32 * r < NQV) { vmin = ref_min(vmin, v[r][k]); vmax = ref_max(vmax, v[r][k]); }
            vmin = warp_min(vmin);
            vmax = warp_max(vmax);
            if (vmin < bmin || vmax > bmax) {
                const double tmin = (avg[k] != vmin) ? (avg[k] - bmin) / (avg[k] - vmin + 1e-32) : 0.0;
                const double tmax = (avg[k] != vmax) ? (bmax - avg[k]) / (vmax - avg[k] + 1e-32) : 0.0;
                const double theta = ref_min(ref_min(tmin, tmax), 1.0);
                scale[k] *= theta;
                #pragma unroll
                for (int r = 0; r < PPL; ++r) v[r][k] = avg[k] + theta * (v[r][k] - avg[k]);
                changed = true;
            }
        }
        // step 2: density at the points >= 1e-16
        {
            const double eps = 1e-16;
            double rmin = DBL_MAX;
            #pragma unroll
            for (int r = 0; r < PPL; ++r)
                if (lane + 32 * r < NQV) rmin = ref_min(rmin, v[r][0]);
            rmin = warp_min(rmin);
            if (rmin < eps) {
                const double eff = ref_max(avg[0], eps);
                const double num = eff - eps, den = eff - rmin;
                const double theta = (den < 1e-32) ? 0.0 : ref_min(1.0, num / den);
                scale[0] *= theta;
                #pragma unroll
                for (int r = 0; r < PPL; ++r) v[r][0] = avg[0] + theta * (v[r][0] - avg[0]);
                changed = true;
            }
        }
        // step 3: pressure at the points >= 0 by bisection toward the mean
        double tp = 1.0;
        #pragma unroll
        for (int r = 0; r < PPL; ++r) {
            if (lane + 32 * r >= NQV || limiter_pressure(v[r], gamma) >= 0) continue;
            double lo = 0.0, hi = 1.0, mid = 0.5 * (lo + hi);
            for (int it = 0; it < 100; ++it) {
                mid = 0.5 * (lo + hi);
                double um[5];
                #pragma unroll
                for (int k = 0; k < 5; ++k) um[k] = (1.0 - mid) * avg[k] + mid * v[r][k];
                if (limiter_pressure(um, gamma) < 0) hi = mid;
                else lo = mid;
            }
            tp = ref_min(tp, mid);
        }
        tp = warp_min(tp);
        if (tp != 1.0) changed = true;
        if (changed) {  // modes l >= 1: c *= theta_1 [*= theta_rho] *= theta_p, in the reference's order
            for (int i = lane; i < 5 * (NB - 1); i += 32) {
                const int k = i % 5;
                double c = u[5 + i];
                if (scale[k] != 1.0 || (k == 0 && scale[0] != 1.0)) c *= scale[k];
                if (tp != 1.0) c *= tp;
                u[5 + i] = c;
                ug[5 + i] = c;
            }
            __syncwarp();
            if (mir) {  // refresh the split rows of the changed element
                for (int i = lane; i < 5 * (KB / 2); i += 32) {
                    const int k = i / (KB / 2), x = 2 * (i - k * (KB / 2));
                    const float v0 = x + 1 < NB ? (float)u[5 * (x + 1) + k] : 0.f;
                    const float v1 = x + 2 < NB ? (float)u[5 * (x + 2) + k] : 0.f;
                    uint32_t h, l;
                    split2(v0, v1, h, l);
                    uint32_t* row = mir + (e * 5 + k) * KB;
                    row[arow_hi_word<KB>(x)] = h;
                    row[arow_lo_word<KB>(x)] = l;
                }
            }
        }
        __syncwarp();
    }
}

// X(order, qv, NB, NQV)
#define FVEDG_LIMITER_COMBOS(X) \
    X(1, 0, 4, 4)               \
    X(1, 2, 4, 15)              \
    X(2, 1, 10, 11)             \
    X(2, 2, 10, 15)             \
    X(3, 3, 20, 23)             \
    X(3, 4, 20, 31)             \
    X(4, 5, 35, 44)             \
    X(4, 6, 35, 57)

inline bool limiter_supported(int order, int qv) {
#define X(P, QV, NB, NQV) \
    if (order == P && qv == QV) return true;
    FVEDG_LIMITER_COMBOS(X)
#undef X
    return false;
}

// Bounds from Uprev, then the three steps on U (in place) for cells [0, napply) (the owned cells;
// the statistics cover ghost cells too). stats: [ncell][10] scratch.
inline int launch_limiter(int order, int qv, double* U, const double* Uprev, const FaceInfo* fi, const ElemFace* ef,
                          const double* phi_v, int64_t ncell, int64_t napply, double gamma, int only_avg,
                          double* stats, uint32_t* mir, int sms, cudaStream_t s) {
#define X(P, QV, NB, NQV)                                                                                        \
    if (order == P && qv == QV) {                                                                                \
        const unsigned ge = (unsigned)std::min<int64_t>((ncell + kLimWarps - 1) / kLimWarps, (int64_t)sms * 16); \
        limiter_cell_stats<NB, NQV><<<ge, kLimWarps * 32, 0, s>>>(Uprev, phi_v, ncell, only_avg, stats);         \
        limiter_apply<NB, NQV><<<ge, kLimWarps * 32, 0, s>>>(U, ef, fi, stats, phi_v, napply, gamma, mir);      \
        return cudaGetLastError() == cudaSuccess ? DG_OK : DG_E_CUDA;                                            \
    }
    FVEDG_LIMITER_COMBOS(X)
#undef X
    return DG_E_ARG;
}

}  // namespace fvedg
