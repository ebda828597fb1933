// Mixed-precision form of the explicit DG operator.
//
// The four dense contractions of a stage run on the tensor cores as BF16 MMAs with FP32
// accumulation (mma.sync.m16n8k16), each operand split into hi + lo BF16 parts and the three
// products hi*hi + hi*lo + lo*hi accumulated (about 16 significant bits per product):
//   face traces      U'(x_g) = sum_{b>=1} phi_b(xi_g^perm) c_b          A = face-map table
//   volume values    U'(x_g) = sum_{b>=1} phi_b(x_g) c_b                A = volume table
//   volume integral  R_v[j]  = -sum_{g,d} w_g dphi_j,d(x_g) G'_d(x_g)   A = weighted gradients
//   face integral    R_f[j]  = +-sum_g w_g phi_j(xi_g^perm) F'(x_g)     A = weighted face-map table
// Only deviations go through the tensor cores: the mode-0 coefficient c_0 (phi_0 = 1) is added to
// the traces exactly, and the per-element/per-face means of G and F are integrated exactly in FP64
// against precomputed moments (sum_g w_g dphi_j and sum_g w_g phi_j). Large constant backgrounds
// (the p0 ~ 71 pressure of a Mach 0.1 flow) therefore never meet BF16 rounding. The pointwise flux
// and the Riemann solvers run in FP32; the RK stage update, the inverse mass and the state stay in
// FP64. Contractions follow ExplicitConvection.cpp:144-272 term by term.
#pragma once
#include <cuda_bf16.h>

#include <atomic>
#include <cstdint>
#include <vector>

#include "dg_flux.cuh"
#include "dg_internal.h"
#include "dg_kernels_fp64.cuh"

namespace fvedg {

__host__ __device__ constexpr int pad16(int x) { return (x + 15) / 16 * 16; }

struct MixedTables {  // device pointers
    const __nv_bfloat16 *tfa_hi, *tfa_lo;  // [24][MF][KB]   face traces
    const __nv_bfloat16 *tva_hi, *tva_lo;  // [MV][KB]       volume values
    const __nv_bfloat16 *tvp_hi, *tvp_lo;  // [MJ][KV]       volume integral
    const __nv_bfloat16 *tfl_hi, *tfl_lo;  // [24][MJ][KF]   face integral
    const double* mv;                      // [NB][3]  sum_g w_g dphi_j
    const double* mf;                      // [24][NB] sum_g w_g phi_j(xi_g^perm)
    const double* wf;                      // [NQF] face weights
};

struct MixedFaceArgs {
    const double* U;
    const FaceInfo* fi;
    const double* UD;
    float* Fj;        // [nface][nqf][5]: 2A * numerical flux at the face points (no quadrature weight)
    MixedTables t;
    int nface;
    float gamma;
    int flux;
    int faces_mask;
};

struct MixedElemArgs {
    const double* U;
    const double* U0;
    double* out;
    const float* Fj;
    const double* geo;
    const ElemFace* ef;
    const double* mass_ref;
    MixedTables t;
    int ncell;
    float gamma;
    double dt, a0, a1;
    int mode;
    int with_volume;
};

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo_k, __nv_bfloat16 hi_k) {
    return (uint32_t)__bfloat16_as_ushort(lo_k) | ((uint32_t)__bfloat16_as_ushort(hi_k) << 16);
}

// x = hi + lo with hi, lo in BF16
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment of tile (mt, kt) of a row-major BF16 table with leading dimension ld.
__device__ __forceinline__ void load_a(const __nv_bfloat16* T, int ld, int mt, int kt, int lane, uint32_t a[4]) {
    const int gid = lane >> 2, tig = lane & 3;
    const __nv_bfloat16* p = T + (mt * 16 + gid) * ld + kt * 16 + tig * 2;
    a[0] = __ldg((const unsigned int*)p);
    a[1] = __ldg((const unsigned int*)(p + 8 * ld));
    a[2] = __ldg((const unsigned int*)(p + 8));
    a[3] = __ldg((const unsigned int*)(p + 8 * ld + 8));
}

// B fragment (16 x 8, k-major) for k-tile kt from a value functor v(k, n) -> float, split hi/lo.
template <class V>
__device__ __forceinline__ void load_b(V v, int kt, int lane, uint32_t bh[2], uint32_t bl[2]) {
    const int gid = lane >> 2, tig = lane & 3;
    __nv_bfloat16 h[4], l[4];
    #pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int k = kt * 16 + tig * 2 + (r & 1) + (r >> 1) * 8;
        split_bf16(v(k, gid), h[r], l[r]);
    }
    bh[0] = pack_bf16(h[0], h[1]);
    bh[1] = pack_bf16(h[2], h[3]);
    bl[0] = pack_bf16(l[0], l[1]);
    bl[1] = pack_bf16(l[2], l[3]);
}

// acc += A * B with both operands split: hi*hi + hi*lo + lo*hi
__device__ __forceinline__ void mma3(float acc[4], const __nv_bfloat16* Th, const __nv_bfloat16* Tl, int ld,
                                     int mt, int kt, int lane, const uint32_t bh[2], const uint32_t bl[2]) {
    uint32_t ah[4], al[4];
    load_a(Th, ld, mt, kt, lane, ah);
    load_a(Tl, ld, mt, kt, lane, al);
    mma16816(acc, ah, bh);
    mma16816(acc, ah, bl);
    mma16816(acc, al, bh);
}

// One warp per face: trace deviations of both sides on the tensor cores, then one lane per face
// point adds the mode-0 coefficient and evaluates the numerical flux in FP32.
template <int NB, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) face_flux_mixed(MixedFaceArgs a) {
    constexpr int KB = pad16(NB - 1), MF = pad16(NQF);
    __shared__ float sU[WARPS][2][MF][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    for (int f = blockIdx.x * WARPS + warp; f < a.nface; f += gridDim.x * WARPS) {
        const FaceInfo fi = a.fi[f];
        const int p[2] = {fi.meta & 0xff, (fi.meta >> 8) & 0xff};
        const int bc = (fi.meta >> 16) & 0xff;
        const bool interior = fi.c1 >= 0;
        const bool active = interior ? (a.faces_mask & 1)
                                     : ((a.faces_mask & 2) && ((bc == 0 && a.UD != nullptr) || bc == 5));
        if (!active) {
            for (int i = lane; i < NQF * 5; i += 32) a.Fj[(int64_t)f * NQF * 5 + i] = 0.f;
            continue;
        }
        const int nside = interior ? 2 : 1;
        for (int s = 0; s < nside; ++s) {
            const double* coef = a.U + (int64_t)(s ? fi.c1 : fi.c0) * (5 * NB);
            uint32_t bh[KB / 16][2], bl[KB / 16][2];
            #pragma unroll
            for (int kt = 0; kt < KB / 16; ++kt)
                load_b([&](int k, int n) {
                    return (n < 5 && k + 1 < NB) ? (float)__ldg(coef + 5 * (k + 1) + n) : 0.f;
                }, kt, lane, bh[kt], bl[kt]);
            const __nv_bfloat16* th = a.t.tfa_hi + p[s] * MF * KB;
            const __nv_bfloat16* tl = a.t.tfa_lo + p[s] * MF * KB;
            #pragma unroll
            for (int mt = 0; mt < MF / 16; ++mt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                #pragma unroll
                for (int kt = 0; kt < KB / 16; ++kt) mma3(acc, th, tl, KB, mt, kt, lane, bh[kt], bl[kt]);
                sU[warp][s][mt * 16 + gid][tig * 2] = acc[0];
                sU[warp][s][mt * 16 + gid][tig * 2 + 1] = acc[1];
                sU[warp][s][mt * 16 + gid + 8][tig * 2] = acc[2];
                sU[warp][s][mt * 16 + gid + 8][tig * 2 + 1] = acc[3];
            }
        }
        __syncwarp();
        if (lane < NQF) {
            const int g = lane;
            const double* cL = a.U + (int64_t)fi.c0 * (5 * NB);
            float UL[5], UR[5];
            #pragma unroll
            for (int k = 0; k < 5; ++k) UL[k] = (float)(__ldg(cL + k) + (double)sU[warp][0][g][k]);
            if (interior) {
                const double* cR = a.U + (int64_t)fi.c1 * (5 * NB);
                #pragma unroll
                for (int k = 0; k < 5; ++k) UR[k] = (float)(__ldg(cR + k) + (double)sU[warp][1][g][k]);
            } else if (bc == 0) {
                const double* ud = a.UD + ((int64_t)f * NQF + g) * 5;
                #pragma unroll
                for (int k = 0; k < 5; ++k) UR[k] = (float)ud[k] + ((float)ud[k] - UL[k]);
            } else {
                #pragma unroll
                for (int k = 0; k < 5; ++k) UR[k] = UL[k];
                UR[3] = -UL[3];
            }
            const float n[3] = {(float)fi.n[0], (float)fi.n[1], (float)fi.n[2]};
            float Fh[5];
            if (a.flux == 1) Phys<float>::roe(UL, UR, n, a.gamma, Fh);
            else Phys<float>::lax_friedrichs(UL, UR, n, a.gamma, Fh);
            const float jw = (float)fi.jw;
            float* o = a.Fj + ((int64_t)f * NQF + g) * 5;
            #pragma unroll
            for (int k = 0; k < 5; ++k) o[k] = Fh[k] * jw;
        }
        __syncwarp();
    }
}

// One warp per element: volume values (MMA), FP32 flux, volume integral (MMA), the four face
// integrals (MMA), exact FP64 mean-part integrals, then the FP64 RK stage update.
template <int NB, int NQV, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) element_mixed(MixedElemArgs a) {
    constexpr int KB = pad16(NB - 1), MV = pad16(NQV), MJ = pad16(NB), KV = pad16(3 * NQV), KF = pad16(NQF);
    __shared__ float sU[WARPS][MV][8];
    __shared__ float sG[WARPS][NQV * 15];
    __shared__ float sF[WARPS][4][NQF * 5];
    __shared__ double sGbar[WARPS][15];
    __shared__ double sFbar[WARPS][4][5];
    __shared__ double sS0[WARPS][4][5];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gid = lane >> 2, tig = lane & 3;
    for (int e = blockIdx.x * WARPS + warp; e < a.ncell; e += gridDim.x * WARPS) {
        const double* coef = a.U + (int64_t)e * (5 * NB);
        const double* geo = a.geo + (int64_t)e * 10;
        float accv[MJ / 16][4], accf[MJ / 16][4];
        #pragma unroll
        for (int mt = 0; mt < MJ / 16; ++mt)
            #pragma unroll
            for (int r = 0; r < 4; ++r) accv[mt][r] = accf[mt][r] = 0.f;
        if (a.with_volume) {
            uint32_t bh[KB / 16][2], bl[KB / 16][2];
            #pragma unroll
            for (int kt = 0; kt < KB / 16; ++kt)
                load_b([&](int k, int n) {
                    return (n < 5 && k + 1 < NB) ? (float)__ldg(coef + 5 * (k + 1) + n) : 0.f;
                }, kt, lane, bh[kt], bl[kt]);
            #pragma unroll
            for (int mt = 0; mt < MV / 16; ++mt) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                #pragma unroll
                for (int kt = 0; kt < KB / 16; ++kt) mma3(acc, a.t.tva_hi, a.t.tva_lo, KB, mt, kt, lane, bh[kt], bl[kt]);
                sU[warp][mt * 16 + gid][tig * 2] = acc[0];
                sU[warp][mt * 16 + gid][tig * 2 + 1] = acc[1];
                sU[warp][mt * 16 + gid + 8][tig * 2] = acc[2];
                sU[warp][mt * 16 + gid + 8][tig * 2 + 1] = acc[3];
            }
            __syncwarp();
            float J[9];
            #pragma unroll
            for (int i = 0; i < 9; ++i) J[i] = (float)__ldg(geo + i);
            const float dj = (float)__ldg(geo + 9);
            for (int g = lane; g < NQV; g += 32) {
                float U[5], F[5][3];
                #pragma unroll
                for (int k = 0; k < 5; ++k) U[k] = (float)(__ldg(coef + k) + (double)sU[warp][g][k]);
                Phys<float>::flux(U, a.gamma - 1.f, F);
                #pragma unroll
                for (int k = 0; k < 5; ++k)
                    #pragma unroll
                    for (int d = 0; d < 3; ++d)
                        sG[warp][g * 15 + 3 * k + d] = dj * (F[k][0] * J[d] + F[k][1] * J[3 + d] + F[k][2] * J[6 + d]);
            }
            __syncwarp();
            if (lane < 15) {
                double s = 0.0;
                for (int g = 0; g < NQV; ++g) s += (double)sG[warp][g * 15 + lane];
                sGbar[warp][lane] = s / NQV;
            }
            __syncwarp();
            const float* G = sG[warp];
            const double* Gb = sGbar[warp];
            #pragma unroll
            for (int kt = 0; kt < KV / 16; ++kt) {
                uint32_t gh[2], gl[2];
                load_b([&](int k, int n) {
                    if (n >= 5 || k >= 3 * NQV) return 0.f;
                    const int g = k / 3, d = k - 3 * g;
                    return G[g * 15 + 3 * n + d] - (float)Gb[3 * n + d];
                }, kt, lane, gh, gl);
                #pragma unroll
                for (int mt = 0; mt < MJ / 16; ++mt) mma3(accv[mt], a.t.tvp_hi, a.t.tvp_lo, KV, mt, kt, lane, gh, gl);
            }
        }
        // face integrals
        for (int i = lane; i < 4 * NQF * 5; i += 32) {
            const int q = i / (NQF * 5), off = i - q * (NQF * 5);
            const int face = a.ef[(int64_t)e * 4 + q].face;
            sF[warp][q][off] = __ldcg(a.Fj + (int64_t)face * NQF * 5 + off);
        }
        __syncwarp();
        if (lane < 20) {
            // per face: the mean used for the deviations, and the exact mode-0 integral
            // sum_g w_g F (phi_0 = 1), summed in one fixed order so that the two sides of a face
            // receive exactly opposite contributions and the element means are conserved
            const int q = lane / 5, k = lane - 5 * q;
            double s = 0.0, s0 = 0.0;
            for (int g = 0; g < NQF; ++g) {
                const double v = (double)sF[warp][q][g * 5 + k];
                s += v;
                s0 += __ldg(a.t.wf + g) * v;
            }
            sFbar[warp][q][k] = s / NQF;
            sS0[warp][q][k] = s0;
        }
        __syncwarp();
        #pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int meta = a.ef[(int64_t)e * 4 + q].meta;
            const int perm = meta & 0xff;
            const float sgn = (meta >> 8) ? -1.f : 1.f;
            const float* Fq = sF[warp][q];
            const double* Fb = sFbar[warp][q];
            const __nv_bfloat16* th = a.t.tfl_hi + perm * MJ * KF;
            const __nv_bfloat16* tl = a.t.tfl_lo + perm * MJ * KF;
            #pragma unroll
            for (int kt = 0; kt < KF / 16; ++kt) {
                uint32_t fh[2], fl[2];
                load_b([&](int k, int n) {
                    return (n < 5 && k < NQF) ? sgn * (Fq[k * 5 + n] - (float)Fb[n]) : 0.f;
                }, kt, lane, fh, fl);
                #pragma unroll
                for (int mt = 0; mt < MJ / 16; ++mt) mma3(accf[mt], th, tl, KF, mt, kt, lane, fh, fl);
            }
        }
        // epilogue: this lane owns R[j][k] for j = mt*16 + gid (+8), k = 2 tig (+1)
        const double detj = __ldg(geo + 9);
        #pragma unroll
        for (int mt = 0; mt < MJ / 16; ++mt) {
            #pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int j = mt * 16 + gid + (r >> 1) * 8;
                const int k = tig * 2 + (r & 1);
                if (j >= NB || k >= 5) continue;
                double R = (double)accf[mt][r] - (double)accv[mt][r];
                if (j == 0) {  // grad phi_0 = 0: only the exact face sums
                    R = 0.0;
                    #pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const int meta = a.ef[(int64_t)e * 4 + q].meta;
                        R += (meta >> 8) ? -sS0[warp][q][k] : sS0[warp][q][k];
                    }
                } else {
                if (a.with_volume) {
                    const double* gb = sGbar[warp] + 3 * k;
                    const double* mv = a.t.mv + 3 * j;
                    R -= gb[0] * __ldg(mv) + gb[1] * __ldg(mv + 1) + gb[2] * __ldg(mv + 2);
                }
                #pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int meta = a.ef[(int64_t)e * 4 + q].meta;
                    const double m = __ldg(a.t.mf + (meta & 0xff) * NB + j) * sFbar[warp][q][k];
                    R += (meta >> 8) ? -m : m;
                }
                }
                double* o = a.out + (int64_t)e * (5 * NB) + 5 * j + k;
                if (a.mode == 0) {
                    *o = R;
                } else {
                    const double ib = 1.0 / (detj * __ldg(a.mass_ref + j));
                    const double u0 = a.U0[(int64_t)e * (5 * NB) + 5 * j + k];
                    *o = a.a0 * u0 + a.a1 * (__ldg(coef + 5 * j + k) + a.dt * (-R * ib));
                }
            }
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
struct MixedData {
    bool ready = false;
    int order = 0, qv = 0, qf = 0, nb = 0, nqv = 0, nqf = 0;
    int64_t ncell = 0, nface = 0;
    float gamma = 1.4f;
    int flux = 0;
    int sms = 148;
    std::vector<void*> bufs;
    MixedTables t{};
    const FaceInfo* fi = nullptr;
    const ElemFace* ef = nullptr;
    const double* geo = nullptr;
    const double* mass_ref = nullptr;
    const double* UD = nullptr;
    float* Fj = nullptr;
};

// X(order, qv, qf, NB, NQV, NQF)
#define FVEDG_MIXED_COMBOS(X)      \
    X(1, 0, 1, 4, 4, 6)            \
    X(1, 0, 0, 4, 4, 4)            \
    X(1, 0, 2, 4, 4, 7)            \
    X(1, 2, 2, 4, 15, 7)           \
    X(2, 1, 2, 10, 11, 7)          \
    X(2, 1, 3, 10, 11, 24)         \
    X(2, 2, 3, 10, 15, 24)         \
    X(3, 3, 3, 20, 23, 24)         \
    X(3, 4, 3, 20, 31, 24)         \
    X(4, 5, 3, 35, 44, 24)         \
    X(4, 6, 3, 35, 57, 24)

inline bool mixed_supported(int order, int qv, int qf) {
#define X(P, QV, QF, NB, NQV, NQF) \
    if (order == P && qv == QV && qf == QF) return true;
    FVEDG_MIXED_COMBOS(X)
#undef X
    return false;
}

template <typename T>
inline int mixed_upload(MixedData& m, const T** dst, const std::vector<T>& v) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * v.size()) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    if (cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess) return DG_E_CUDA;
    *dst = (const T*)p;
    return DG_OK;
}

inline void split_table(const std::vector<double>& x, std::vector<__nv_bfloat16>& hi, std::vector<__nv_bfloat16>& lo) {
    hi.resize(x.size());
    lo.resize(x.size());
    for (size_t i = 0; i < x.size(); ++i) {
        const float f = (float)x[i];
        hi[i] = __float2bfloat16_rn(f);
        lo[i] = __float2bfloat16_rn(f - __bfloat162float(hi[i]));
    }
}

inline int init_mixed(MixedData& m, const Tables& tab, const std::vector<double>&, const std::vector<FaceInfo>&,
                      const std::vector<ElemFace>&, int64_t ncell, int64_t nface, double gamma, int flux,
                      int qv, int qf, const double* d_geo, const FaceInfo* d_fi, const ElemFace* d_ef,
                      const double* d_mass_ref) {
    if (!mixed_supported(tab.order, qv, qf)) return DG_E_ARG;
    const int NB = tab.nb, NQV = tab.nqv, NQF = tab.nqf;
    const int KB = pad16(NB - 1), MF = pad16(NQF), MV = pad16(NQV), MJ = pad16(NB), KV = pad16(3 * NQV),
              KF = pad16(NQF);
    m.order = tab.order; m.qv = qv; m.qf = qf; m.nb = NB; m.nqv = NQV; m.nqf = NQF;
    m.ncell = ncell; m.nface = nface; m.gamma = (float)gamma; m.flux = flux;
    std::vector<double> tfa(24 * MF * KB, 0.0), tva(MV * KB, 0.0), tvp(MJ * KV, 0.0), tfl(24 * MJ * KF, 0.0);
    std::vector<double> mv(NB * 3, 0.0), mf(24 * NB, 0.0);
    for (int p = 0; p < 24; ++p)
        for (int g = 0; g < NQF; ++g)
            for (int b = 1; b < NB; ++b) tfa[(p * MF + g) * KB + (b - 1)] = tab.phi_f[((size_t)p * NQF + g) * NB + b];
    for (int g = 0; g < NQV; ++g)
        for (int b = 1; b < NB; ++b) tva[g * KB + (b - 1)] = tab.phi_v[g * NB + b];
    for (int j = 0; j < NB; ++j)
        for (int g = 0; g < NQV; ++g)
            for (int d = 0; d < 3; ++d) {
                const double v = tab.dphi_vw[(g * NB + j) * 3 + d];
                tvp[j * KV + 3 * g + d] = v;
                mv[j * 3 + d] += v;
            }
    for (int p = 0; p < 24; ++p)
        for (int j = 0; j < NB; ++j)
            for (int g = 0; g < NQF; ++g) {
                const double v = tab.w_f[g] * tab.phi_f[((size_t)p * NQF + g) * NB + j];
                tfl[(p * MJ + j) * KF + g] = v;
                mf[p * NB + j] += v;
            }
    std::vector<__nv_bfloat16> h, l;
    int rc;
    split_table(tfa, h, l);
    if ((rc = mixed_upload(m, &m.t.tfa_hi, h)) || (rc = mixed_upload(m, &m.t.tfa_lo, l))) return rc;
    split_table(tva, h, l);
    if ((rc = mixed_upload(m, &m.t.tva_hi, h)) || (rc = mixed_upload(m, &m.t.tva_lo, l))) return rc;
    split_table(tvp, h, l);
    if ((rc = mixed_upload(m, &m.t.tvp_hi, h)) || (rc = mixed_upload(m, &m.t.tvp_lo, l))) return rc;
    split_table(tfl, h, l);
    if ((rc = mixed_upload(m, &m.t.tfl_hi, h)) || (rc = mixed_upload(m, &m.t.tfl_lo, l))) return rc;
    if ((rc = mixed_upload(m, &m.t.mv, mv)) || (rc = mixed_upload(m, &m.t.mf, mf)) ||
        (rc = mixed_upload(m, &m.t.wf, tab.w_f)))
        return rc;
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(float) * (size_t)nface * NQF * 5) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    m.Fj = (float*)p;
    m.fi = d_fi; m.ef = d_ef; m.geo = d_geo; m.mass_ref = d_mass_ref;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&m.sms, cudaDevAttrMultiProcessorCount, dev);
    m.ready = true;
    return DG_OK;
}

inline void free_mixed(MixedData& m) {
    for (void* p : m.bufs) cudaFree(p);
    m.bufs.clear();
    m.ready = false;
}

inline void set_mixed_dirichlet(MixedData& m, const double* UD) { m.UD = UD; }
inline int mixed_launches_per_step(const MixedData&) { return 6; }

template <int NB, int NQV, int NQF, int kMixedWarps = (NB >= 35 ? 4 : 8)>
inline int mixed_launch(MixedData& m, int which, const double* U, const double* U0, double* out, int mode,
                        double dt, double a0, double a1, int face_mask, int with_volume, cudaStream_t s) {
    if (which == 0) {
        MixedFaceArgs fa;
        fa.U = U; fa.fi = m.fi; fa.UD = m.UD; fa.Fj = m.Fj; fa.t = m.t; fa.nface = (int)m.nface;
        fa.gamma = m.gamma; fa.flux = m.flux; fa.faces_mask = face_mask;
        const int gf = (int)std::min<int64_t>((m.nface + kMixedWarps - 1) / kMixedWarps, (int64_t)m.sms * 16);
        face_flux_mixed<NB, NQF, kMixedWarps><<<gf, kMixedWarps * 32, 0, s>>>(fa);
    } else {
        MixedElemArgs ea;
        ea.U = U; ea.U0 = U0; ea.out = out; ea.Fj = m.Fj; ea.geo = m.geo; ea.ef = m.ef; ea.mass_ref = m.mass_ref;
        ea.t = m.t; ea.ncell = (int)m.ncell; ea.gamma = m.gamma; ea.dt = dt; ea.a0 = a0; ea.a1 = a1;
        ea.mode = mode; ea.with_volume = with_volume;
        const int ge = (int)std::min<int64_t>((m.ncell + kMixedWarps - 1) / kMixedWarps, (int64_t)m.sms * 16);
        element_mixed<NB, NQV, NQF, kMixedWarps><<<ge, kMixedWarps * 32, 0, s>>>(ea);
    }
    return cudaGetLastError() == cudaSuccess ? DG_OK : DG_E_CUDA;
}

// which: 0 = face kernel, 1 = element kernel
inline int mixed_kernel(MixedData& m, int which, const double* U, const double* U0, double* out, int mode,
                        double dt, double a0, double a1, int face_mask, int with_volume, cudaStream_t s,
                        std::atomic<int64_t>* launches) {
    if (!m.ready) return DG_E_ARG;
    ++*launches;
#define X(P, QV, QF, NB, NQV, NQF)                                                                          \
    if (m.order == P && m.qv == QV && m.qf == QF)                                                           \
        return mixed_launch<NB, NQV, NQF>(m, which, U, U0, out, mode, dt, a0, a1, face_mask, with_volume, s);
    FVEDG_MIXED_COMBOS(X)
#undef X
    return DG_E_ARG;
}

inline int residual_mixed(MixedData& m, const double* U, double* R, int part, cudaStream_t s,
                          std::atomic<int64_t>* launches) {
    const int mask = part == 0 ? 3 : part == 1 ? 0 : part == 2 ? 1 : 2;
    const int rc = mixed_kernel(m, 0, U, U, R, 0, 0.0, 0.0, 0.0, mask, 0, s, launches);
    if (rc) return rc;
    return mixed_kernel(m, 1, U, U, R, 0, 0.0, 0.0, 0.0, mask, part == 0 || part == 1, s, launches);
}

// SSP-RK3 step; `timed(cls, fn)` runs fn (one launch) and may bracket it with timing events.
template <class Timed>
inline int step_mixed(MixedData& m, double* Un, double* Ua, double* Ub, double dt, cudaStream_t s,
                      std::atomic<int64_t>* launches, Timed&& timed) {
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {Un, Ua, Ub};
    double* out[3] = {Ua, Ub, Un};
    for (int st = 0; st < 3; ++st) {
        int rc = timed(0, [&] { return mixed_kernel(m, 0, in[st], Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, launches); });
        if (rc) return rc;
        rc = timed(1, [&] { return mixed_kernel(m, 1, in[st], Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, launches); });
        if (rc) return rc;
    }
    return DG_OK;
}

}  // namespace fvedg
