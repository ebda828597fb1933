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
// Per-cell statistics of the previous state (lanes over the quadrature points, each point value summed
// over the modes in order, as the reference does), then the bounds and the three steps with the cells
// of a warp side by side. In the time loop the statistics of each stage's limited output come out of
// the same launch and bound the next stage, so one launch per stage suffices. Warps never wait on one
// another.
#pragma once
#include <cfloat>

#include "dg_kernels_fp64.cuh"
#include "dg_status.cuh"
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

// PositiveLimiter.h:112-123
__device__ __forceinline__ double limiter_pressure(const double U[5], double gamma) {
    const double rho = U[0];
    if (rho <= 1e-16) return -1.0;
    const double ke = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / (2.0 * rho);
    return (gamma - 1.0) * (U[4] - ke);
}

constexpr int kLimWarps = 4;
constexpr int kLimMaxPts = 64;  // volume points a warp holds, two per lane (the largest rule has 57)

// The volume rule's basis values transposed to [l][g] in shared memory: lanes over points read
// consecutive doubles (conflict-free) for every mode l.
template <int NB, int NQV>
__device__ __forceinline__ void load_phi_t(double* sphi, const double* __restrict__ phi) {
    for (int i = threadIdx.x; i < NQV * NB; i += blockDim.x) {
        const int g = i / NB, l = i - g * NB;
        sphi[l * NQV + g] = phi[i];
    }
}

// The 5 conserved values at volume point g from the transposed table, summed over the modes in
// order, as the reference evaluates a point value.
template <int NB, int NQV>
__device__ __forceinline__ void point_values_t(const double* sphi, const double* u, int g, double v[5]) {
    #pragma unroll
    for (int k = 0; k < 5; ++k) v[k] = 0.0;
    #pragma unroll 4
    for (int l = 0; l < NB; ++l) {
        const double p = sphi[l * NQV + g];
        #pragma unroll
        for (int k = 0; k < 5; ++k) v[k] = fma(p, u[k + 5 * l], v[k]);
    }
}

// Lanes per cell in the apply pass: the cells of a warp are processed side by side by groups of G
// lanes (G a power of two), each lane holding ceil(NQV / G) points.
template <int NQV>
struct LimGroup {
    static constexpr int G = NQV <= 4 ? 4 : NQV <= 24 ? 8 : NQV <= 48 ? 16 : 32;
};

template <int G>
__device__ __forceinline__ double group_max(double v, unsigned mask) {
    #pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = ref_max(v, __shfl_xor_sync(mask, v, o));
    return v;
}
template <int G>
__device__ __forceinline__ double group_min(double v, unsigned mask) {
    #pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) v = ref_min(v, __shfl_xor_sync(mask, v, o));
    return v;
}
__device__ __forceinline__ bool group_any(bool p, unsigned mask) { return (__ballot_sync(mask, p) & mask) != 0u; }

// A cell's statistics from its point values v[PPL][5], held by a group of G lanes (lane gl holds
// points gl + G r): the max over the points of each variable and the values at the last point
// (with only_avg: the mean, twice).
template <int NQV, int G, int PPL>
__device__ __forceinline__ void write_stats(const double (&v)[PPL][5], const double (&avg)[5], int gl, unsigned mask,
                                            int only_avg, double* __restrict__ out) {
    if (only_avg) {
        #pragma unroll
        for (int k = 0; k < 5; ++k)
            if (gl == k % G) { out[k] = avg[k]; out[5 + k] = avg[k]; }
        return;
    }
    constexpr int LR = (NQV - 1) / G, LL = (NQV - 1) % G;
    if (gl == LL) {
        #pragma unroll
        for (int k = 0; k < 5; ++k) out[5 + k] = v[LR][k];
    }
    #pragma unroll
    for (int k = 0; k < 5; ++k) {
        double mx = -DBL_MAX;
        #pragma unroll
        for (int r = 0; r < PPL; ++r)
            if (gl + G * r < NQV) mx = ref_max(mx, v[r][k]);
        mx = group_max<G>(mx, mask);
        if (gl == 0) out[k] = mx;
    }
}

// Per-cell statistics of a state for the bounds, cells [c_begin, c_end): the max over the volume
// points of each variable and the values at the last point. A face's bounds are max(v1, v2) over the
// points and min(v1, v2) at the last point (PositiveLimiter.h:77-88), i.e. the max of its two cells'
// maxima and the min of their last-point values; with only_avg both are the cell mean (:70-75).
template <int NB, int NQV>
__global__ void __launch_bounds__(kLimWarps * 32)
    limiter_cell_stats(const double* __restrict__ Up, const double* __restrict__ phi, int64_t c_begin, int64_t c_end,
                       int only_avg, double* __restrict__ stats) {
    constexpr int PPL = (NQV + 31) / 32;
    __shared__ double sphi[NQV * NB];
    __shared__ double scoef[kLimWarps][5 * NB];
    load_phi_t<NB, NQV>(sphi, phi);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    double* u = scoef[threadIdx.x >> 5];
    for (int64_t c = c_begin + (int64_t)blockIdx.x * kLimWarps + (threadIdx.x >> 5); c < c_end;
         c += (int64_t)gridDim.x * kLimWarps) {
        const double* ug = Up + c * (5 * NB);
        for (int i = lane; i < 5 * NB; i += 32) u[i] = ug[i];  // coalesced, then broadcast reads
        __syncwarp();
        double avg[5], v[PPL][5];
        #pragma unroll
        for (int k = 0; k < 5; ++k) avg[k] = u[k];
        if (!only_avg) {
            #pragma unroll
            for (int r = 0; r < PPL; ++r) {
                const int g = lane + 32 * r;
                if (g < NQV) point_values_t<NB, NQV>(sphi, u, g, v[r]);
            }
        }
        write_stats<NQV, 32, PPL>(v, avg, lane, 0xffffffffu, only_avg, stats + c * 10);
        __syncwarp();
    }
}

// The three steps per element (PositiveLimiter.h:128-258) for cells [0, ncell), CPW = 32 / G cells
// per warp side by side (lanes over the points of their cell). Bounds: the max of the statistics'
// maxima and the min of their last-point values over the cell and its face neighbours (nbr
// [ncell][4], the cell itself across a boundary face), which is the max/min over the cell's faces of
// the face bounds. Point values are evaluated once; after a step scales the modes l >= 1 of a
// variable by theta, its point values become avg + theta (v - avg) (phi_0 = 1), which is what the
// reference re-evaluates. A step whose test passes at every point costs one vote. stats_out: when
// non-null, the statistics of the limited state (as
// limiter_cell_stats computes them: re-evaluated from the new coefficients where the limiter acted),
// the next stage's bounds.
template <int NB, int NQV>
__global__ void __launch_bounds__(kLimWarps * 32)
    limiter_apply(double* __restrict__ U, const int* __restrict__ nbr, const double* __restrict__ stats,
                  const double* __restrict__ phi, int64_t ncell, double gamma, int only_avg,
                  double* __restrict__ stats_out) {
    constexpr int G = LimGroup<NQV>::G, CPW = 32 / G;
    constexpr int PPL = (NQV + G - 1) / G;  // points per lane
    static_assert(NQV <= kLimMaxPts, "volume rule too large");
    __shared__ double sphi[NQV * NB];
    __shared__ double scoef[kLimWarps][CPW * 5 * NB];
    __shared__ double sbnd[kLimWarps][CPW][10];
    load_phi_t<NB, NQV>(sphi, phi);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int grp = lane / G, gl = lane - grp * G;
    const unsigned gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << (grp * G));
    double* u = scoef[w] + grp * (5 * NB);
    double* bnd = sbnd[w][grp];
    for (int64_t e0 = ((int64_t)blockIdx.x * kLimWarps + w) * CPW; e0 < ncell;
         e0 += (int64_t)gridDim.x * kLimWarps * CPW) {
        const int nc = (int)(ncell - e0 < CPW ? ncell - e0 : CPW);
        {   // the next iteration's cells into L2 while these are limited
            const int64_t en = e0 + (int64_t)gridDim.x * kLimWarps * CPW;
            if (en < ncell) {
                const int64_t bytes = (ncell - en < CPW ? ncell - en : CPW) * (5 * NB * 8);
                for (int64_t off = (int64_t)lane * 128; off < bytes; off += 32 * 128)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char*>(U + en * (5 * NB)) + off));
            }
        }
        const double* ug0 = U + e0 * (5 * NB);
        for (int i = lane; i < nc * 5 * NB; i += 32) scoef[w][i] = ug0[i];  // the warp's cells, coalesced
        __syncwarp();
        if (grp < nc) {
            const int64_t e = e0 + grp;
            double* ug = U + e * (5 * NB);
            for (int k = gl; k < 5; k += G) {  // the cell's bounds: max of maxima, min of last values
                const int4 n = reinterpret_cast<const int4*>(nbr)[e];
                const double* st = stats + k;
                double bx = st[e * 10], bn = st[e * 10 + 5];
                bx = ref_max(bx, st[(int64_t)n.x * 10]); bn = ref_min(bn, st[(int64_t)n.x * 10 + 5]);
                bx = ref_max(bx, st[(int64_t)n.y * 10]); bn = ref_min(bn, st[(int64_t)n.y * 10 + 5]);
                bx = ref_max(bx, st[(int64_t)n.z * 10]); bn = ref_min(bn, st[(int64_t)n.z * 10 + 5]);
                bx = ref_max(bx, st[(int64_t)n.w * 10]); bn = ref_min(bn, st[(int64_t)n.w * 10 + 5]);
                bnd[k] = bx;
                bnd[5 + k] = bn;
            }
            __syncwarp(gmask);
            double avg[5], v[PPL][5];
            #pragma unroll
            for (int k = 0; k < 5; ++k) avg[k] = u[k];
            #pragma unroll
            for (int r = 0; r < PPL; ++r) {
                const int g = gl + G * r;
                if (g < NQV) point_values_t<NB, NQV>(sphi, u, g, v[r]);
                else
                    #pragma unroll
                    for (int k = 0; k < 5; ++k) v[r][k] = avg[k];  // neutral for min/max and pressure
            }
            double s0 = 1.0, s1 = 1.0, s2 = 1.0, s3 = 1.0, s4 = 1.0;  // per-variable scale of modes l >= 1
            bool changed = false;
            // step 1: each variable within the cell's bounds
            #pragma unroll
            for (int k = 0; k < 5; ++k) {
                const double bmax = bnd[k], bmin = bnd[5 + k];
                bool out = false;
                #pragma unroll
                for (int r = 0; r < PPL; ++r) out |= (v[r][k] < bmin) | (v[r][k] > bmax);
                if (!group_any(out, gmask)) continue;
                double vmin = DBL_MAX, vmax = -DBL_MAX;
                #pragma unroll
                for (int r = 0; r < PPL; ++r)
                    if (gl + G * r < NQV) { vmin = ref_min(vmin, v[r][k]); vmax = ref_max(vmax, v[r][k]); }
                vmin = group_min<G>(vmin, gmask);
                vmax = group_max<G>(vmax, gmask);
                const double tmin = (avg[k] != vmin) ? (avg[k] - bmin) / (avg[k] - vmin + 1e-32) : 0.0;
                const double tmax = (avg[k] != vmax) ? (bmax - avg[k]) / (vmax - avg[k] + 1e-32) : 0.0;
                const double theta = ref_min(ref_min(tmin, tmax), 1.0);
                if (k == 0) s0 *= theta;
                else if (k == 1) s1 *= theta;
                else if (k == 2) s2 *= theta;
                else if (k == 3) s3 *= theta;
                else s4 *= theta;
                #pragma unroll
                for (int r = 0; r < PPL; ++r) v[r][k] = avg[k] + theta * (v[r][k] - avg[k]);
                changed = true;
            }
            // step 2: density at the points >= 1e-16
            {
                const double eps = 1e-16;
                bool low = false;
                #pragma unroll
                for (int r = 0; r < PPL; ++r) low |= v[r][0] < eps;
                if (group_any(low, gmask)) {
                    double rmin = DBL_MAX;
                    #pragma unroll
                    for (int r = 0; r < PPL; ++r)
                        if (gl + G * r < NQV) rmin = ref_min(rmin, v[r][0]);
                    rmin = group_min<G>(rmin, gmask);
                    const double eff = ref_max(avg[0], eps);
                    const double num = eff - eps, den = eff - rmin;
                    const double theta = (den < 1e-32) ? 0.0 : ref_min(1.0, num / den);
                    s0 *= theta;
                    #pragma unroll
                    for (int r = 0; r < PPL; ++r) v[r][0] = avg[0] + theta * (v[r][0] - avg[0]);
                    changed = true;
                }
            }
            // step 3: pressure at the points >= 0 by bisection toward the mean
            double tp = 1.0;
            bool neg = false;
            #pragma unroll
            for (int r = 0; r < PPL; ++r) neg |= (gl + G * r < NQV) && limiter_pressure(v[r], gamma) < 0;
            if (group_any(neg, gmask)) {
                #pragma unroll
                for (int r = 0; r < PPL; ++r) {
                    if (gl + G * r >= NQV || limiter_pressure(v[r], gamma) >= 0) continue;
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
                tp = group_min<G>(tp, gmask);
                if (tp != 1.0) changed = true;
            }
            if (changed) {  // modes l >= 1: c *= theta_1 [*= theta_rho] *= theta_p, in the reference's order
                __syncwarp(gmask);
                for (int i = gl; i < 5 * (NB - 1); i += G) {
                    const int k = i % 5;
                    const double sk = k == 0 ? s0 : k == 1 ? s1 : k == 2 ? s2 : k == 3 ? s3 : s4;
                    double c = u[5 + i];
                    if (sk != 1.0) c *= sk;
                    if (tp != 1.0) c *= tp;
                    u[5 + i] = c;
                    ug[5 + i] = c;
                }
                __syncwarp(gmask);
                if (stats_out && !only_avg) {  // the limited state's point values, re-evaluated
                    #pragma unroll
                    for (int r = 0; r < PPL; ++r) {
                        const int g = gl + G * r;
                        if (g < NQV) point_values_t<NB, NQV>(sphi, u, g, v[r]);
                    }
                }
            }
            if (stats_out) write_stats<NQV, G, PPL>(v, avg, gl, gmask, only_avg, stats_out + e * 10);
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
inline int launch_limiter(int order, int qv, double* U, const double* Uprev, const int* nbr, const double* phi_v,
                          int64_t ncell, int64_t napply, double gamma, int only_avg, double* stats, int sms,
                          cudaStream_t s) {
#define X(P, QV, NB, NQV)                                                                                        \
    if (order == P && qv == QV) {                                                                                \
        const unsigned ge = (unsigned)std::min<int64_t>((ncell + kLimWarps - 1) / kLimWarps, (int64_t)sms * 16); \
        limiter_cell_stats<NB, NQV><<<ge, kLimWarps * 32, 0, s>>>(Uprev, phi_v, 0, ncell, only_avg, stats);      \
        limiter_apply<NB, NQV><<<ge, kLimWarps * 32, 0, s>>>(U, nbr, stats, phi_v, napply, gamma, only_avg,       \
                                                             nullptr);                                           \
        return cuda_status(cudaGetLastError());                                            \
    }
    FVEDG_LIMITER_COMBOS(X)
#undef X
    return DG_E_ARG;
}

// Statistics of cells [c_begin, c_end) of U into stats.
inline int launch_limiter_stats(int order, int qv, const double* U, const double* phi_v, int64_t c_begin,
                                int64_t c_end, int only_avg, double* stats, int sms, cudaStream_t s,
                                std::atomic<int64_t>* launches) {
    if (c_begin >= c_end) return DG_OK;
#define X(P, QV, NB, NQV)                                                                                       \
    if (order == P && qv == QV) {                                                                               \
        const int64_t n = c_end - c_begin;                                                                      \
        const unsigned gs = (unsigned)std::min<int64_t>((n + kLimWarps - 1) / kLimWarps, (int64_t)sms * 16);    \
        limiter_cell_stats<NB, NQV><<<gs, kLimWarps * 32, 0, s>>>(U, phi_v, c_begin, c_end, only_avg, stats);   \
        ++*launches;                                                                                            \
        return cuda_status(cudaGetLastError());                                           \
    }
    FVEDG_LIMITER_COMBOS(X)
#undef X
    return DG_E_ARG;
}

// The limiter inside the time loop, one launch per stage: bounds from `stats_in` (the statistics
// of the stage input, which the previous stage's launch wrote), and the statistics of the limited
// output into `stats_out`. The statistics of cells [stats_begin, ncell) of the input are computed
// first (all cells after the state was set from outside, else the ghost cells, whose rows a halo
// exchange rewrote; none when stats_begin == ncell).
inline int launch_limiter_stage(int order, int qv, double* U, const double* Uin, const int* nbr, const double* phi_v,
                                int64_t ncell, int64_t napply, int64_t stats_begin, double gamma, int only_avg,
                                double* stats_in, double* stats_out, int sms, cudaStream_t s,
                                std::atomic<int64_t>* launches) {
    int rc = launch_limiter_stats(order, qv, Uin, phi_v, stats_begin, ncell, only_avg, stats_in, sms, s, launches);
    if (rc) return rc;
#define X(P, QV, NB, NQV)                                                                                         \
    if (order == P && qv == QV) {                                                                                 \
        const unsigned ge = (unsigned)std::min<int64_t>((napply + kLimWarps - 1) / kLimWarps, (int64_t)sms * 16); \
        limiter_apply<NB, NQV><<<ge, kLimWarps * 32, 0, s>>>(U, nbr, stats_in, phi_v, napply, gamma, only_avg,    \
                                                             stats_out);                                          \
        ++*launches;                                                                                              \
        return cuda_status(cudaGetLastError());                                             \
    }
    FVEDG_LIMITER_COMBOS(X)
#undef X
    return DG_E_ARG;
}

}  // namespace fvedg
