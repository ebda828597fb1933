// Deterministic reductions over the device state: conservation sums, the largest wave speed (for a
// CFL time step, cf. examples/TaylerGreenVortex/TGBatch.cpp:358-383) and the non-physical point
// count. Each is a fixed grid of per-block partials (a fixed assignment of elements to warps and of
// volume points to lanes) followed by one block that sums them in a fixed order, so results do not
// depend on scheduling.
#pragma once
#include <atomic>
#include <cstdint>

#include "dg_flux.cuh"

namespace fvedg {

constexpr int kRedBlocks = 592;  // 4 x 148 SMs
constexpr int kRedThreads = 256;

enum RedKind { RED_CONSERVATION = 0, RED_WAVESPEED = 1, RED_BADPOINTS = 2 };

__device__ __forceinline__ double red_combine(int kind, double a, double b) {
    return kind == RED_WAVESPEED ? fmax(a, b) : a + b;
}

// partial[block][0..5]
__global__ void __launch_bounds__(kRedThreads) state_reduce_kernel(const double* __restrict__ U,
        const double* __restrict__ geo, const double* __restrict__ phi_v, const double* __restrict__ w_v,
        int ncell, int nb, int nqv, double gamma, int kind, double* __restrict__ partial) {
    __shared__ double sh[kRedThreads][6];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    // one warp per element, its lanes over the volume points: the element's row is read by
    // broadcast loads (one transaction per warp and value) instead of one row per thread
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int e = blockIdx.x * wpb + (threadIdx.x >> 5); e < ncell; e += gridDim.x * wpb) {
        const double* c = U + (int64_t)e * 5 * nb;
        const double dj = geo ? geo[(int64_t)e * 10 + 9] : 0.0;
        if (kind == RED_CONSERVATION && lane == 0)
            for (int k = 0; k < 5; ++k) acc[k] += c[k] * dj / 6.0;
        for (int g = lane; g < nqv; g += 32) {
            double Ug[5] = {0, 0, 0, 0, 0};
            for (int b = 0; b < nb; ++b) {
                const double p = phi_v[g * nb + b];
                for (int k = 0; k < 5; ++k) Ug[k] = fma(p, c[5 * b + k], Ug[k]);
            }
            if (kind == RED_CONSERVATION) {
                const double rho = Phys<double>::positive(Ug[0]);
                acc[5] += w_v[g] * dj * 0.5 * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]) / rho;
            } else {
                const double rho = Ug[0];
                const double ke = 0.5 * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]) / rho;
                const double p = (gamma - 1.0) * (Ug[4] - ke);
                bool bad = !(rho > 0.0) || !(p > 0.0);
                for (int k = 0; k < 5; ++k) bad = bad || !isfinite(Ug[k]);
                if (kind == RED_BADPOINTS) {
                    acc[0] += bad ? 1.0 : 0.0;
                } else if (!bad) {
                    const double vel[3] = {Ug[1] / rho, Ug[2] / rho, Ug[3] / rho};
                    acc[0] = fmax(acc[0], Phys<double>::wave_speed(rho, vel, p, gamma));
                }
            }
        }
    }
    for (int k = 0; k < 6; ++k) sh[threadIdx.x][k] = acc[k];
    __syncthreads();
    for (int s = kRedThreads / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int k = 0; k < 6; ++k) sh[threadIdx.x][k] = red_combine(kind, sh[threadIdx.x][k], sh[threadIdx.x + s][k]);
        __syncthreads();
    }
    if (threadIdx.x < 6) partial[blockIdx.x * 6 + threadIdx.x] = sh[0][threadIdx.x];
}

__global__ void partial_sum_kernel(const double* __restrict__ partial, int nblk, int kind, double* __restrict__ out) {
    if (threadIdx.x < 6) {
        double s = 0.0;
        for (int b = 0; b < nblk; ++b) s = red_combine(kind, s, partial[b * 6 + threadIdx.x]);
        out[threadIdx.x] = s;
    }
}

inline int run_state_reduce(const double* U, const double* geo, const double* phi_v, const double* w_v, int ncell,
                            int nb, int nqv, double gamma, int kind, double* partial, double out[6],
                            cudaStream_t s, std::atomic<int64_t>* launches) {
    state_reduce_kernel<<<kRedBlocks, kRedThreads, 0, s>>>(U, geo, phi_v, w_v, ncell, nb, nqv, gamma, kind, partial);
    partial_sum_kernel<<<1, 32, 0, s>>>(partial, kRedBlocks, kind, partial + (size_t)kRedBlocks * 6);
    *launches += 2;
    if (cudaGetLastError() != cudaSuccess) return DG_E_CUDA;
    if (cudaMemcpyAsync(out, partial + (size_t)kRedBlocks * 6, 6 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return DG_E_CUDA;
    return cudaStreamSynchronize(s) == cudaSuccess ? DG_OK : DG_E_CUDA;
}

inline int reduce_conservation(const double* U, const double* geo, const double* phi_v, const double* w_v,
                               int ncell, int nb, int nqv, double* partial, double out[6], cudaStream_t s,
                               std::atomic<int64_t>* launches) {
    return run_state_reduce(U, geo, phi_v, w_v, ncell, nb, nqv, 1.4, RED_CONSERVATION, partial, out, s, launches);
}
inline int reduce_wave_speed(const double* U, const double* phi_v, int ncell, int nb, int nqv, double gamma,
                             double* partial, double* lam, cudaStream_t s, std::atomic<int64_t>* launches) {
    double o[6];
    int rc = run_state_reduce(U, nullptr, phi_v, nullptr, ncell, nb, nqv, gamma, RED_WAVESPEED, partial, o, s, launches);
    *lam = o[0];
    return rc;
}
inline int reduce_bad_points(const double* U, const double* phi_v, int ncell, int nb, int nqv, double gamma,
                             double* partial, double* nbad, cudaStream_t s, std::atomic<int64_t>* launches) {
    double o[6];
    int rc = run_state_reduce(U, nullptr, phi_v, nullptr, ncell, nb, nqv, gamma, RED_BADPOINTS, partial, o, s, launches);
    *nbad = o[0];
    return rc;
}

}  // namespace fvedg
