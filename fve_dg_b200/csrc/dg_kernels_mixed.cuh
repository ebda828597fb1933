// Mixed-precision form of the explicit DG operator.
//
// The four dense contractions of a stage run on the tensor cores as BF16 MMAs with FP32
// accumulation (mma.sync.m16n8k16). Both operands are split into hi + lo BF16 parts and the three
// products hi*hi + hi*lo + lo*hi are accumulated (about 16 significant bits per product):
//   face traces      U'(x_g) = sum_{b>=1} phi_b(xi_g^perm) c_b          B = face-map table
//   volume values    U'(x_g) = sum_{b>=1} phi_b(x_g) c_b                B = volume table
//   volume integral  R_v[j]  = -sum_{g,d} w_g dphi_j,d(x_g) G'_d(x_g)   B = weighted gradients
//   face integral    R_f[j]  = +-sum_g w_g phi_j(xi_g^perm) F'(x_g)     B = weighted face-map table
// The MMA's 16 rows hold (item, variable) pairs of three items (faces or elements) that share their
// face maps, so one table fragment serves three items. Items are grouped that way on the host.
//
// Three kernels per RK stage: face fluxes, volume integrals (independent of the faces, so the two
// run side by side), and the face integrals with the RK update. The face kernel writes its flux
// deviations already split into BF16 hi/lo in the order the lift's MMA fragments read them.
//
// Only deviations go through the tensor cores: the mode-0 coefficient c_0 (phi_0 = 1) is added to
// the traces exactly; the volume flux is taken relative to the flux of the element mean state and
// the face flux relative to its face mean, and those references are integrated exactly in FP64
// against precomputed moments (sum_g w_g dphi_j and sum_g w_g phi_j). The mode-0 face integral
// is summed in FP64 in one fixed order per face, so both sides receive exactly opposite amounts
// and the element means (mass, momentum, energy) are conserved to round-off. Large constant
// backgrounds (the p0 ~ 71 of a Mach 0.1 flow) never meet BF16 rounding. The pointwise flux and
// the Riemann solvers run in FP32; the RK stage update, the inverse mass and the state are FP64.
// The terms follow ExplicitConvection.cpp:144-272 one for one.
#pragma once
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <map>
#include <vector>

#include "dg_flux.cuh"
#include "dg_internal.h"
#include "dg_kernels_fp64.cuh"

namespace fvedg {

__host__ __device__ constexpr int pad16(int x) { return (x + 15) / 16 * 16; }
__host__ __device__ constexpr int pad8(int x) { return (x + 7) / 8 * 8; }

struct MixedTables {  // device pointers; every table row-major [n][k] (the MMA's B operand)
    const __nv_bfloat16 *tfa_hi, *tfa_lo;  // [24][MF][KB]   face traces:  n = face point, k = mode-1
    const __nv_bfloat16 *tva_hi, *tva_lo;  // [MV][KB]       volume values: n = volume point
    const __nv_bfloat16 *tvp_hi, *tvp_lo;  // [MJ][KV]       volume integral: n = mode, k = (point, dir)
    const __nv_bfloat16 *tfl_hi, *tfl_lo;  // [24][MJ][KF]   face integral: n = mode, k = face point
    const double* mv;                      // [NB][3]  sum_g w_g dphi_j
    const double* mf;                      // [24][NB] sum_g w_g phi_j(xi_g^perm)
    const double* wf;                      // [NQF]
    const float* wf32;                     // [NQF]
    const double* inv_mass;                // [NB] 1 / sum_g w_g phi_j^2
};

struct FaceGroup {   // up to three faces with equal (perm0, perm1, kind)
    int f[3];
    int n;
};
struct ElemGroup {   // up to three elements with equal face maps in canonical face order
    int e[3];
    int n;
    int face[3][4];  // face id of canonical local face q (the face opposite local vertex q)
    int meta[4];     // perm | side << 8, shared by the group
};

struct MixedFaceArgs {
    const double* U;
    const __nv_bfloat16* mir_hi;  // U's deviation coefficients c_b (b >= 1), split, [ncell][5][KB]
    const __nv_bfloat16* mir_lo;
    const FaceInfo* fi;
    const FaceGroup* groups;
    const double* UD;
    __nv_bfloat16* dev_hi;  // [nface][5][KF] flux deviation from the face mean, 2A * (F - mean)
    __nv_bfloat16* dev_lo;
    double* Fmean;          // [nface][5] face mean of 2A * F
    double* S0;             // [nface][5] sum_g w_g 2A F (the exact mode-0 face integral)
    MixedTables t;
    int ngroups;
    float gamma;
    int flux;
    int faces_mask;
};

struct MixedVolArgs {
    const double* U;
    const __nv_bfloat16* mir_hi;
    const __nv_bfloat16* mir_lo;
    const double* geo;
    const ElemGroup* groups;
    double* Rv;             // [ncell][5*NB] volume part of the residual
    MixedTables t;
    int ngroups;
    float gamma;
};

struct MixedLiftArgs {
    const double* U;
    const double* U0;
    double* out;
    const double* Rv;       // null when the volume term is left out (residual parts 2 and 3)
    const __nv_bfloat16* dev_hi;
    const __nv_bfloat16* dev_lo;
    const double* Fmean;
    const double* S0;
    const double* inv_detj; // [ncell]
    const ElemGroup* groups;
    MixedTables t;
    int ngroups;
    double dt, a0, a1;
    int mode;
    const double* dt_inst;  // optional per-instance time step (ensembles), indexed by elem_inst
    const int* elem_inst;   // [ncell] instance of each element
    __nv_bfloat16* out_mir_hi;  // RK mode: the new stage's split deviation coefficients
    __nv_bfloat16* out_mir_lo;
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

// A fragment (16 x 16, row-major) of k-tile kt from a value functor v(row, col) -> float, split.
template <class V>
__device__ __forceinline__ void build_a(V v, int kt, int lane, uint32_t ah[4], uint32_t al[4]) {
    const int gid = lane >> 2, tig = lane & 3;
    __nv_bfloat16 h[8], l[8];
    #pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int row = gid + ((r >> 1) & 1) * 8;
        const int col = kt * 16 + tig * 2 + (r & 1) + (r >> 2) * 8;
        split_bf16(v(row, col), h[r], l[r]);
    }
    #pragma unroll
    for (int i = 0; i < 4; ++i) {
        ah[i] = pack_bf16(h[2 * i], h[2 * i + 1]);
        al[i] = pack_bf16(l[2 * i], l[2 * i + 1]);
    }
}

// A fragment of k-tile kt straight from a split mirror [item][5][KB]: row r = (slot, var) of the
// 16 rows reads mirror row base[r / 5] * 5 + r % 5; rows >= nrows are zero.
template <int KB>
__device__ __forceinline__ void load_a_mirror(const __nv_bfloat16* hi, const __nv_bfloat16* lo, const int* item,
                                              int nrows, int kt, int lane, uint32_t ah[4], uint32_t al[4]) {
    const int gid = lane >> 2, tig = lane & 3;
    const int r0 = gid, r1 = gid + 8;
    const bool v0 = r0 < nrows, v1 = r1 < nrows;
    const int64_t o0 = v0 ? ((int64_t)item[r0 / 5] * 5 + r0 % 5) * KB + kt * 16 + tig * 2 : 0;
    const int64_t o1 = v1 ? ((int64_t)item[r1 / 5] * 5 + r1 % 5) * KB + kt * 16 + tig * 2 : 0;
    ah[0] = v0 ? __ldg((const unsigned int*)(hi + o0)) : 0u;
    ah[1] = v1 ? __ldg((const unsigned int*)(hi + o1)) : 0u;
    ah[2] = v0 ? __ldg((const unsigned int*)(hi + o0 + 8)) : 0u;
    ah[3] = v1 ? __ldg((const unsigned int*)(hi + o1 + 8)) : 0u;
    al[0] = v0 ? __ldg((const unsigned int*)(lo + o0)) : 0u;
    al[1] = v1 ? __ldg((const unsigned int*)(lo + o1)) : 0u;
    al[2] = v0 ? __ldg((const unsigned int*)(lo + o0 + 8)) : 0u;
    al[3] = v1 ? __ldg((const unsigned int*)(lo + o1 + 8)) : 0u;
}

// Writes the split deviation coefficients of a state into a mirror (after an upload, or for a
// residual of an arbitrary state): one thread per (element, var, column).
template <int NB>
__global__ void mirror_split(const double* __restrict__ U, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo, int64_t ncell) {
    constexpr int KB = pad16(NB - 1);
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell * 5 * KB) return;
    const int64_t row = i / KB;
    const int col = (int)(i - row * KB);
    const int64_t e = row / 5;
    const int k = (int)(row - e * 5);
    const float v = col + 1 < NB ? (float)U[e * (5 * NB) + 5 * (col + 1) + k] : 0.f;
    __nv_bfloat16 h, l;
    split_bf16(v, h, l);
    hi[i] = h;
    lo[i] = l;
}

// acc(16 x 8 tile nt) += A * B(nt, kt) with B read from a row-major [n][k] BF16 table of leading
// dimension ld; three products hi*hi + hi*lo + lo*hi.
__device__ __forceinline__ void mma3_b(float acc[4], const uint32_t ah[4], const uint32_t al[4],
                                       const __nv_bfloat16* Th, const __nv_bfloat16* Tl, int ld, int nt, int kt,
                                       int lane) {
    const int gid = lane >> 2, tig = lane & 3;
    const int off = (nt * 8 + gid) * ld + kt * 16 + tig * 2;
    uint32_t bh[2], bl[2];
    bh[0] = __ldg((const unsigned int*)(Th + off));
    bh[1] = __ldg((const unsigned int*)(Th + off + 8));
    bl[0] = __ldg((const unsigned int*)(Tl + off));
    bl[1] = __ldg((const unsigned int*)(Tl + off + 8));
    mma16816(acc, ah, bh);
    mma16816(acc, ah, bl);
    mma16816(acc, al, bh);
}

// ------------------------------------------------------------------------------------------------
// Face fluxes: one warp per face group. Trace deviations of each side for the three faces (rows
// (face, var)) on the tensor cores; one lane per face point adds c_0 and evaluates the FP32 flux;
// then the face mean, the exact mode-0 sum and the split deviations are written.
// ------------------------------------------------------------------------------------------------
template <int NQF>
struct FaceMixedSmem {
    double sC0[2][3][5];  // mode-0 coefficients of both sides of the three faces
    float sN[3][4];       // unit normal and 2A of the three faces
    float sU[2][16][pad8(NQF) + 1];
    float sFb[3][5];
};

template <int NB, int NQF>
__device__ __forceinline__ void face_group_mixed(const MixedFaceArgs& a, int gi, FaceMixedSmem<NQF>& sm, int lane) {
    constexpr int KB = pad16(NB - 1), MF = pad8(NQF), KF = pad16(NQF);
    auto& sU = sm.sU;
    const int gid = lane >> 2, tig = lane & 3;
    const FaceGroup grp = a.groups[gi];
    const FaceInfo f0 = a.fi[grp.f[0]];  // shares perms and kind with the others
    const int perm[2] = {f0.meta & 0xff, (f0.meta >> 8) & 0xff};
    const int bc = (f0.meta >> 16) & 0xff;
    const bool interior = f0.c1 >= 0;
    const bool active = interior ? (a.faces_mask & 1)
                                 : ((a.faces_mask & 2) && ((bc == 0 && a.UD != nullptr) || bc == 5));
    if (!active) {
        const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
        for (int i = lane; i < grp.n * 5 * NQF; i += 32) {
            const int fl = i / (5 * NQF), r = i - fl * 5 * NQF, k = r / NQF, g = r - k * NQF;
            const int64_t o = ((int64_t)grp.f[fl] * 5 + k) * KF + g;
            a.dev_hi[o] = z;
            a.dev_lo[o] = z;
        }
        for (int i = lane; i < grp.n * 5; i += 32) {
            a.Fmean[(int64_t)grp.f[i / 5] * 5 + i % 5] = 0.0;
            a.S0[(int64_t)grp.f[i / 5] * 5 + i % 5] = 0.0;
        }
        return;
    }
    const int nside = interior ? 2 : 1;
    if (lane < 3 * nside * 5) {  // per-face data of the point loop, staged once
        const int s = lane / 15, r = lane - 15 * s, fl = r / 5, k = r - 5 * fl;
        const FaceInfo& F = a.fi[grp.f[fl]];
        sm.sC0[s][fl][k] = __ldg(a.U + (int64_t)(s ? F.c1 : F.c0) * (5 * NB) + k);
        if (s == 0 && k < 4) sm.sN[fl][k] = k < 3 ? (float)F.n[k] : (float)F.jw;
    }
    for (int s = 0; s < nside; ++s) {
        int cell[3];
        #pragma unroll
        for (int i = 0; i < 3; ++i) {
            const FaceInfo& F = a.fi[grp.f[i]];
            cell[i] = s ? F.c1 : F.c0;
        }
        uint32_t ah[KB / 16][4], al[KB / 16][4];
        #pragma unroll
        for (int kt = 0; kt < KB / 16; ++kt) load_a_mirror<KB>(a.mir_hi, a.mir_lo, cell, 5 * grp.n, kt, lane, ah[kt], al[kt]);
        const __nv_bfloat16* th = a.t.tfa_hi + perm[s] * MF * KB;
        const __nv_bfloat16* tl = a.t.tfa_lo + perm[s] * MF * KB;
        #pragma unroll
        for (int nt = 0; nt < MF / 8; ++nt) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            #pragma unroll
            for (int kt = 0; kt < KB / 16; ++kt) mma3_b(acc, ah[kt], al[kt], th, tl, KB, nt, kt, lane);
            sU[s][gid][nt * 8 + tig * 2] = acc[0];
            sU[s][gid][nt * 8 + tig * 2 + 1] = acc[1];
            sU[s][gid + 8][nt * 8 + tig * 2] = acc[2];
            sU[s][gid + 8][nt * 8 + tig * 2 + 1] = acc[3];
        }
    }
    __syncwarp();
    for (int p = lane; p < grp.n * NQF; p += 32) {
        const int fl = p / NQF, g = p - fl * NQF;
        const int f = grp.f[fl];
        float UL[5], UR[5];
        #pragma unroll
        for (int k = 0; k < 5; ++k) UL[k] = (float)(sm.sC0[0][fl][k] + (double)sU[0][fl * 5 + k][g]);
        if (interior) {
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = (float)(sm.sC0[1][fl][k] + (double)sU[1][fl * 5 + k][g]);
        } else if (bc == 0) {
            const double* ud = a.UD + ((int64_t)f * NQF + g) * 5;
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = (float)ud[k] + ((float)ud[k] - UL[k]);
        } else {
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = UL[k];
            UR[3] = -UL[3];
        }
        const float n[3] = {sm.sN[fl][0], sm.sN[fl][1], sm.sN[fl][2]};
        float Fh[5];
        if (a.flux == 1) Phys<float>::roe(UL, UR, n, a.gamma, Fh);
        else Phys<float>::lax_friedrichs(UL, UR, n, a.gamma, Fh);
        const float jw = sm.sN[fl][3];
        // side-1 deviations are no longer needed: keep the face flux there
        #pragma unroll
        for (int k = 0; k < 5; ++k) sU[1][fl * 5 + k][g] = Fh[k] * jw;
    }
    __syncwarp();
    if (lane < 5 * grp.n) {
        // face mean (any per-face constant serves as the reference) and the mode-0 integral
        // sum_g w_g F, in one fixed order: both sides of the face then use the same number, which
        // is what makes the element means conserved exactly
        const int fl = lane / 5, k = lane - 5 * fl;
        float s[2] = {0.f, 0.f}, s0[2] = {0.f, 0.f};
        #pragma unroll
        for (int g = 0; g < NQF; ++g) {
            const float v = sU[1][fl * 5 + k][g];
            s[g & 1] += v;
            s0[g & 1] += __ldg(a.t.wf32 + g) * v;
        }
        const float mean = (s[0] + s[1]) * (1.f / NQF);
        a.Fmean[(int64_t)grp.f[fl] * 5 + k] = (double)mean;
        a.S0[(int64_t)grp.f[fl] * 5 + k] = (double)(s0[0] + s0[1]);
        sm.sFb[fl][k] = mean;
    }
    __syncwarp();
    for (int i = lane; i < grp.n * 5 * NQF; i += 32) {  // deviations, split, in [face][var][point] order
        const int fl = i / (5 * NQF), r = i - fl * 5 * NQF, k = r / NQF, g = r - k * NQF;
        __nv_bfloat16 h, l;
        split_bf16(sU[1][fl * 5 + k][g] - sm.sFb[fl][k], h, l);
        const int64_t o = ((int64_t)grp.f[fl] * 5 + k) * KF + g;
        a.dev_hi[o] = h;
        a.dev_lo[o] = l;
    }
    __syncwarp();
}

template <int NB, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) face_flux_mixed(MixedFaceArgs a) {
    __shared__ FaceMixedSmem<NQF> sm[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int gi = blockIdx.x * WARPS + warp; gi < a.ngroups; gi += gridDim.x * WARPS)
        face_group_mixed<NB, NQF>(a, gi, sm[warp], lane);
}

// ------------------------------------------------------------------------------------------------
// Volume integrals: one warp per element group. Volume values on the tensor cores, FP32 flux,
// deviations from the flux of the element mean state, the integral on the tensor cores, and the
// FP64 mean part; writes R_v.
// ------------------------------------------------------------------------------------------------
template <int NB, int NQV>
struct VolMixedSmem {
    static constexpr int MV = pad8(NQV), KV = pad16(3 * NQV);
    double sGb[3][15];               // flux of the element mean state, times detJ J^-T
    float sJ[3][10];                 // J^-T and detJ, FP32
    float sU[16][MV + 1];            // volume deviations, rows (element, var), cols point
    float sG[16][KV + 2];            // G - G(c_0), rows (element, var), cols (point, dir)
};

template <int NB, int NQV>
__device__ __forceinline__ void volume_group_mixed(const MixedVolArgs& a, int gi, VolMixedSmem<NB, NQV>& sm, int lane) {
    using S = VolMixedSmem<NB, NQV>;
    constexpr int KB = pad16(NB - 1), MV = S::MV, MJ = pad8(NB), KV = S::KV;
    const int gid = lane >> 2, tig = lane & 3;
    const ElemGroup grp = a.groups[gi];
    const int ne = grp.n;
    const double* coef[3];
    #pragma unroll
    for (int i = 0; i < 3; ++i) coef[i] = a.U + (int64_t)grp.e[i] * (5 * NB);
    if (lane < ne) {  // G(c_0), FP64
        const double* geo = a.geo + (int64_t)grp.e[lane] * 10;
        double c0[5], F[5][3], J[9];
        #pragma unroll
        for (int k = 0; k < 5; ++k) c0[k] = __ldg(coef[lane] + k);
        #pragma unroll
        for (int i = 0; i < 9; ++i) J[i] = __ldg(geo + i);
        const double dj = __ldg(geo + 9);
        Phys<double>::flux(c0, (double)a.gamma - 1.0, F);
        #pragma unroll
        for (int k = 0; k < 5; ++k)
            #pragma unroll
            for (int d = 0; d < 3; ++d)
                sm.sGb[lane][3 * k + d] = dj * (F[k][0] * J[d] + F[k][1] * J[3 + d] + F[k][2] * J[6 + d]);
        #pragma unroll
        for (int i = 0; i < 9; ++i) sm.sJ[lane][i] = (float)J[i];
        sm.sJ[lane][9] = (float)dj;
    }
    {
        uint32_t ah[KB / 16][4], al[KB / 16][4];
        #pragma unroll
        for (int kt = 0; kt < KB / 16; ++kt) load_a_mirror<KB>(a.mir_hi, a.mir_lo, grp.e, 5 * ne, kt, lane, ah[kt], al[kt]);
        #pragma unroll
        for (int nt = 0; nt < MV / 8; ++nt) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            #pragma unroll
            for (int kt = 0; kt < KB / 16; ++kt) mma3_b(acc, ah[kt], al[kt], a.t.tva_hi, a.t.tva_lo, KB, nt, kt, lane);
            sm.sU[gid][nt * 8 + tig * 2] = acc[0];
            sm.sU[gid][nt * 8 + tig * 2 + 1] = acc[1];
            sm.sU[gid + 8][nt * 8 + tig * 2] = acc[2];
            sm.sU[gid + 8][nt * 8 + tig * 2 + 1] = acc[3];
        }
    }
    __syncwarp();
    for (int p = lane; p < ne * NQV; p += 32) {
        const int el = p / NQV, g = p - el * NQV;
        float U[5], F[5][3];
        #pragma unroll
        for (int k = 0; k < 5; ++k) U[k] = (float)(__ldg(coef[el] + k) + (double)sm.sU[el * 5 + k][g]);
        Phys<float>::flux(U, a.gamma - 1.f, F);
        const float* J = sm.sJ[el];
        #pragma unroll
        for (int k = 0; k < 5; ++k)
            #pragma unroll
            for (int d = 0; d < 3; ++d)
                sm.sG[el * 5 + k][3 * g + d] =
                    J[9] * (F[k][0] * J[d] + F[k][1] * J[3 + d] + F[k][2] * J[6 + d]) - (float)sm.sGb[el][3 * k + d];
    }
    __syncwarp();
    float accv[MJ / 8][4];
    #pragma unroll
    for (int nt = 0; nt < MJ / 8; ++nt)
        #pragma unroll
        for (int r = 0; r < 4; ++r) accv[nt][r] = 0.f;
    #pragma unroll
    for (int kt = 0; kt < KV / 16; ++kt) {
        uint32_t ah[4], al[4];
        build_a([&](int row, int col) { return (row < 5 * ne && col < 3 * NQV) ? sm.sG[row][col] : 0.f; },
                kt, lane, ah, al);
        #pragma unroll
        for (int nt = 0; nt < MJ / 8; ++nt) mma3_b(accv[nt], ah, al, a.t.tvp_hi, a.t.tvp_lo, KV, nt, kt, lane);
    }
    #pragma unroll
    for (int nt = 0; nt < MJ / 8; ++nt) {
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int row = gid + (r >> 1) * 8;
            const int j = nt * 8 + tig * 2 + (r & 1);
            if (row >= 5 * ne || j >= NB) continue;
            const int el = row / 5, k = row - 5 * el;
            double R = 0.0;  // grad phi_0 = 0
            if (j > 0) {
                const double* gb = sm.sGb[el] + 3 * k;
                const double* mv = a.t.mv + 3 * j;
                R = -(double)accv[nt][r] - (gb[0] * __ldg(mv) + gb[1] * __ldg(mv + 1) + gb[2] * __ldg(mv + 2));
            }
            a.Rv[(int64_t)grp.e[el] * (5 * NB) + 5 * j + k] = R;
        }
    }
    __syncwarp();
}

template <int NB, int NQV, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) volume_mixed(MixedVolArgs a) {
    using S = VolMixedSmem<NB, NQV>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S& sm = reinterpret_cast<S*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    for (int gi = blockIdx.x * WARPS + (threadIdx.x >> 5); gi < a.ngroups; gi += gridDim.x * WARPS)
        volume_group_mixed<NB, NQV>(a, gi, sm, lane);
}

// ------------------------------------------------------------------------------------------------
// Face integrals and the RK update: one warp per element group. The flux deviations arrive split,
// in fragment order, so the four face integrals are MMAs straight from memory; then the FP64 mean
// parts, the volume part and the stage combination.
// ------------------------------------------------------------------------------------------------
struct LiftMixedSmem {
    double sFb[3][4][5];   // face means
    double sS0[3][4][5];   // exact mode-0 face sums
};

template <int NB, int NQF>
__device__ __forceinline__ void lift_group_mixed(const MixedLiftArgs& a, int gi, LiftMixedSmem& sm, int lane) {
    constexpr int MJ = pad8(NB), KF = pad16(NQF);
    const int gid = lane >> 2, tig = lane & 3;
    const ElemGroup grp = a.groups[gi];
    const int ne = grp.n;
    for (int i = lane; i < ne * 20; i += 32) {
        const int el = i / 20, r = i - el * 20, q = r / 5, k = r - 5 * q;
        const int f = grp.face[el][q];
        sm.sFb[el][q][k] = __ldcg(a.Fmean + (int64_t)f * 5 + k);
        sm.sS0[el][q][k] = __ldcg(a.S0 + (int64_t)f * 5 + k);
    }
    float accf[MJ / 8][4];
    #pragma unroll
    for (int nt = 0; nt < MJ / 8; ++nt)
        #pragma unroll
        for (int r = 0; r < 4; ++r) accf[nt][r] = 0.f;
    // rows gid and gid + 8 of the A fragments: (element, var) -> the face's deviation row
    const int r0 = gid, r1 = gid + 8;
    const int el0 = r0 / 5, k0 = r0 - 5 * el0, el1 = r1 / 5, k1 = r1 - 5 * el1;
    const bool v0 = r0 < 5 * ne, v1 = r1 < 5 * ne;
    #pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int perm = grp.meta[q] & 0xff;
        const uint32_t flip = (grp.meta[q] >> 8) ? 0x80008000u : 0u;  // exact negation of both halves
        const int64_t o0 = v0 ? ((int64_t)grp.face[el0][q] * 5 + k0) * KF : 0;
        const int64_t o1 = v1 ? ((int64_t)grp.face[el1][q] * 5 + k1) * KF : 0;
        const __nv_bfloat16* th = a.t.tfl_hi + perm * MJ * KF;
        const __nv_bfloat16* tl = a.t.tfl_lo + perm * MJ * KF;
        #pragma unroll
        for (int kt = 0; kt < KF / 16; ++kt) {
            const int c = kt * 16 + tig * 2;
            uint32_t ah[4], al[4];
            ah[0] = v0 ? (__ldcg((const unsigned int*)(a.dev_hi + o0 + c)) ^ flip) : 0u;
            ah[1] = v1 ? (__ldcg((const unsigned int*)(a.dev_hi + o1 + c)) ^ flip) : 0u;
            ah[2] = v0 ? (__ldcg((const unsigned int*)(a.dev_hi + o0 + c + 8)) ^ flip) : 0u;
            ah[3] = v1 ? (__ldcg((const unsigned int*)(a.dev_hi + o1 + c + 8)) ^ flip) : 0u;
            al[0] = v0 ? (__ldcg((const unsigned int*)(a.dev_lo + o0 + c)) ^ flip) : 0u;
            al[1] = v1 ? (__ldcg((const unsigned int*)(a.dev_lo + o1 + c)) ^ flip) : 0u;
            al[2] = v0 ? (__ldcg((const unsigned int*)(a.dev_lo + o0 + c + 8)) ^ flip) : 0u;
            al[3] = v1 ? (__ldcg((const unsigned int*)(a.dev_lo + o1 + c + 8)) ^ flip) : 0u;
            #pragma unroll
            for (int nt = 0; nt < MJ / 8; ++nt) mma3_b(accf[nt], ah, al, th, tl, KF, nt, kt, lane);
        }
    }
    __syncwarp();
    // epilogue: this lane owns rows (element, var) gid and gid + 8, modes nt*8 + 2 tig (+1)
    #pragma unroll
    for (int nt = 0; nt < MJ / 8; ++nt) {
        #pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int row = gid + (r >> 1) * 8;
            const int j = nt * 8 + tig * 2 + (r & 1);
            if (row >= 5 * ne || j >= NB) continue;
            const int el = row / 5, k = row - 5 * el;
            double R;
            if (j == 0) {  // only the exact face sums
                R = 0.0;
                #pragma unroll
                for (int q = 0; q < 4; ++q) R += (grp.meta[q] >> 8) ? -sm.sS0[el][q][k] : sm.sS0[el][q][k];
            } else {
                R = (double)accf[nt][r];
                #pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double m = __ldg(a.t.mf + (grp.meta[q] & 0xff) * NB + j) * sm.sFb[el][q][k];
                    R += (grp.meta[q] >> 8) ? -m : m;
                }
            }
            const int e = grp.e[el];
            const int64_t idx = (int64_t)e * (5 * NB) + 5 * j + k;
            if (a.Rv) R += __ldcg(a.Rv + idx);
            if (a.mode == 0) {
                a.out[idx] = R;
            } else {
                const double ib = __ldg(a.inv_detj + e) * __ldg(a.t.inv_mass + j);
                const double dt = a.dt_inst ? __ldg(a.dt_inst + __ldg(a.elem_inst + e)) : a.dt;
                const double un = a.a0 * a.U0[idx] + a.a1 * (__ldg(a.U + idx) + dt * (-R * ib));
                a.out[idx] = un;
                if (j > 0) {
                    constexpr int KBm = pad16(NB - 1);
                    __nv_bfloat16 h, l;
                    split_bf16((float)un, h, l);
                    const int64_t mo = ((int64_t)e * 5 + k) * KBm + (j - 1);
                    a.out_mir_hi[mo] = h;
                    a.out_mir_lo[mo] = l;
                }
            }
        }
    }
    __syncwarp();
}

template <int NB, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, 4) lift_mixed(MixedLiftArgs a) {
    __shared__ LiftMixedSmem sm[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int gi = blockIdx.x * WARPS + warp; gi < a.ngroups; gi += gridDim.x * WARPS)
        lift_group_mixed<NB, NQF>(a, gi, sm[warp], lane);
}

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
struct MixedData {
    bool ready = false;
    int order = 0, qv = 0, qf = 0, nb = 0, nqv = 0, nqf = 0;
    int64_t ncell = 0, nface = 0;
    int nfgroups = 0, negroups = 0;
    float gamma = 1.4f;
    int flux = 0;
    int sms = 148;
    std::vector<void*> bufs;
    MixedTables t{};
    const FaceInfo* fi = nullptr;
    const FaceGroup* fgroups = nullptr;
    const ElemGroup* egroups = nullptr;
    const double* geo = nullptr;
    const double* inv_detj = nullptr;
    const double* UD = nullptr;
    __nv_bfloat16* dev_hi = nullptr;
    __nv_bfloat16* dev_lo = nullptr;
    double* Fmean = nullptr;
    double* S0 = nullptr;
    double* Rv = nullptr;
    const double* dt_inst = nullptr;  // ensembles: per-instance dt (device), else null
    const int* elem_inst = nullptr;
    // split deviation coefficients of the states Un, Ua, Ub and of a residual input, [ncell][5][KB]
    __nv_bfloat16* mir_hi[4] = {nullptr, nullptr, nullptr, nullptr};
    __nv_bfloat16* mir_lo[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t side = nullptr;      // second stream: the volume kernel beside the face kernel
    cudaEvent_t fork = nullptr, join = nullptr;
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
    if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(v.size(), 1)) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    if (!v.empty() && cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return DG_E_CUDA;
    *dst = (const T*)p;
    return DG_OK;
}

template <typename T>
inline int mixed_alloc(MixedData& m, T** dst, size_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    if (cudaMemset(p, 0, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) return DG_E_CUDA;
    *dst = (T*)p;
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

// Faces with equal (perm0, perm1, kind) and elements with equal face maps (in canonical face
// order: local face q is the one opposite local vertex q) are grouped in threes, in mesh order.
// A partial group repeats its first member in the unused slots (never read as a row: rows of
// unused slots are masked by the group size).
inline void build_groups(const std::vector<FaceInfo>& hfi, const std::vector<ElemFace>& hef, int64_t ncell,
                         std::vector<FaceGroup>& fg, std::vector<ElemGroup>& eg) {
    std::map<int64_t, FaceGroup> open_f;
    for (int64_t f = 0; f < (int64_t)hfi.size(); ++f) {
        const FaceInfo& F = hfi[f];
        const int64_t key = (int64_t)(F.meta & 0xffffff) * 2 + (F.c1 >= 0 ? 1 : 0);
        FaceGroup& g = open_f[key];
        g.f[g.n++] = (int)f;
        if (g.n == 3) { fg.push_back(g); g = FaceGroup{}; }
    }
    for (auto& kv : open_f)
        if (kv.second.n > 0) {
            for (int i = kv.second.n; i < 3; ++i) kv.second.f[i] = kv.second.f[0];
            fg.push_back(kv.second);
        }
    std::map<std::vector<int>, ElemGroup> open_e;
    for (int64_t e = 0; e < ncell; ++e) {
        int face[4] = {-1, -1, -1, -1}, meta[4] = {0, 0, 0, 0};
        for (int i = 0; i < 4; ++i) {
            const ElemFace& ef = hef[4 * e + i];
            const int p = ef.meta & 0xff;
            const int q = 6 - kPermSlots[p][0] - kPermSlots[p][1] - kPermSlots[p][2];  // missing vertex
            face[q] = ef.face;
            meta[q] = ef.meta;
        }
        std::vector<int> key(meta, meta + 4);
        ElemGroup& g = open_e[key];
        g.e[g.n] = (int)e;
        for (int q = 0; q < 4; ++q) { g.face[g.n][q] = face[q]; g.meta[q] = meta[q]; }
        ++g.n;
        if (g.n == 3) { eg.push_back(g); g = ElemGroup{}; }
    }
    for (auto& kv : open_e)
        if (kv.second.n > 0) {
            ElemGroup g = kv.second;
            for (int i = g.n; i < 3; ++i) {
                g.e[i] = g.e[0];
                for (int q = 0; q < 4; ++q) g.face[i][q] = g.face[0][q];
            }
            eg.push_back(g);
        }
}

inline int init_mixed(MixedData& m, const Tables& tab, const std::vector<double>& hgeo,
                      const std::vector<FaceInfo>& hfi, const std::vector<ElemFace>& hef, int64_t ncell,
                      int64_t nface, double gamma, int flux, int qv, int qf, const double* d_geo,
                      const FaceInfo* d_fi, const ElemFace*, const double*) {
    if (!mixed_supported(tab.order, qv, qf)) return DG_E_ARG;
    const int NB = tab.nb, NQV = tab.nqv, NQF = tab.nqf;
    const int KB = pad16(NB - 1), MF = pad8(NQF), MV = pad8(NQV), MJ = pad8(NB), KV = pad16(3 * NQV),
              KF = pad16(NQF);
    m.order = tab.order; m.qv = qv; m.qf = qf; m.nb = NB; m.nqv = NQV; m.nqf = NQF;
    m.ncell = ncell; m.nface = nface; m.gamma = (float)gamma; m.flux = flux;
    std::vector<double> tfa(24 * MF * KB, 0.0), tva(MV * KB, 0.0), tvp(MJ * KV, 0.0), tfl(24 * MJ * KF, 0.0);
    std::vector<double> mv(NB * 3, 0.0), mf(24 * NB, 0.0), inv_mass(NB, 0.0), inv_detj(ncell, 0.0);
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
    for (int j = 0; j < NB; ++j) inv_mass[j] = 1.0 / tab.mass_ref[j];
    for (int64_t e = 0; e < ncell; ++e) inv_detj[e] = 1.0 / hgeo[10 * e + 9];
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
        (rc = mixed_upload(m, &m.t.wf, tab.w_f)) || (rc = mixed_upload(m, &m.t.inv_mass, inv_mass)) ||
        (rc = mixed_upload(m, &m.t.wf32, std::vector<float>(tab.w_f.begin(), tab.w_f.end()))) ||
        (rc = mixed_upload(m, &m.inv_detj, inv_detj)))
        return rc;
    std::vector<FaceGroup> fg;
    std::vector<ElemGroup> eg;
    build_groups(hfi, hef, ncell, fg, eg);
    m.nfgroups = (int)fg.size();
    m.negroups = (int)eg.size();
    if ((rc = mixed_upload(m, &m.fgroups, fg)) || (rc = mixed_upload(m, &m.egroups, eg))) return rc;
    // the deviation buffers' padding columns stay zero: allocation clears them, kernels never write them
    if ((rc = mixed_alloc(m, &m.dev_hi, (size_t)nface * 5 * KF)) || (rc = mixed_alloc(m, &m.dev_lo, (size_t)nface * 5 * KF)) ||
        (rc = mixed_alloc(m, &m.Fmean, (size_t)nface * 5)) || (rc = mixed_alloc(m, &m.S0, (size_t)nface * 5)) ||
        (rc = mixed_alloc(m, &m.Rv, (size_t)ncell * 5 * NB)))
        return rc;
    for (int i = 0; i < 4; ++i)
        if ((rc = mixed_alloc(m, &m.mir_hi[i], (size_t)ncell * 5 * KB)) ||
            (rc = mixed_alloc(m, &m.mir_lo[i], (size_t)ncell * 5 * KB)))
            return rc;
    m.fi = d_fi; m.geo = d_geo;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&m.sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaStreamCreateWithFlags(&m.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&m.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&m.join, cudaEventDisableTiming) != cudaSuccess)
        return DG_E_CUDA;
    m.ready = true;
    return DG_OK;
}

inline void free_mixed(MixedData& m) {
    for (void* p : m.bufs) cudaFree(p);
    m.bufs.clear();
    if (m.side) cudaStreamDestroy(m.side);
    if (m.fork) cudaEventDestroy(m.fork);
    if (m.join) cudaEventDestroy(m.join);
    m.side = nullptr;
    m.fork = m.join = nullptr;
    m.ready = false;
}

inline void set_mixed_dirichlet(MixedData& m, const double* UD) { m.UD = UD; }

// Launch classes used for timing: 0 face fluxes, 3 volume integrals, 1 face integrals + update.
template <int NB, int NQV, int NQF, int W = 8>
inline int mixed_launch(MixedData& m, int which, const double* U, const double* U0, double* out, int mode,
                        double dt, double a0, double a1, int face_mask, int with_volume, cudaStream_t s,
                        int mir_in, int mir_out) {
    if (which == 4) {  // split U into mirror mir_in
        const int64_t n = m.ncell * 5 * pad16(NB - 1);
        mirror_split<NB><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(U, m.mir_hi[mir_in], m.mir_lo[mir_in], m.ncell);
    } else if (which == 0) {
        MixedFaceArgs fa;
        fa.U = U; fa.mir_hi = m.mir_hi[mir_in]; fa.mir_lo = m.mir_lo[mir_in]; fa.fi = m.fi; fa.groups = m.fgroups; fa.UD = m.UD; fa.dev_hi = m.dev_hi; fa.dev_lo = m.dev_lo;
        fa.Fmean = m.Fmean; fa.S0 = m.S0; fa.t = m.t; fa.ngroups = m.nfgroups; fa.gamma = m.gamma; fa.flux = m.flux;
        fa.faces_mask = face_mask;
        const int g = (int)std::min<int64_t>((m.nfgroups + W - 1) / W, (int64_t)m.sms * 32);
        face_flux_mixed<NB, NQF, W><<<g, W * 32, 0, s>>>(fa);
    } else if (which == 3) {
        constexpr size_t smem = sizeof(VolMixedSmem<NB, NQV>) * W;
        static bool attr = false;
        if (!attr) {
            if (cudaFuncSetAttribute(volume_mixed<NB, NQV, W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem) != cudaSuccess)
                return DG_E_CUDA;
            attr = true;
        }
        MixedVolArgs va;
        va.U = U; va.mir_hi = m.mir_hi[mir_in]; va.mir_lo = m.mir_lo[mir_in]; va.geo = m.geo; va.groups = m.egroups; va.Rv = m.Rv; va.t = m.t; va.ngroups = m.negroups;
        va.gamma = m.gamma;
        const int g = (int)std::min<int64_t>((m.negroups + W - 1) / W, (int64_t)m.sms * 32);
        volume_mixed<NB, NQV, W><<<g, W * 32, smem, s>>>(va);
    } else {
        MixedLiftArgs la;
        la.U = U; la.U0 = U0; la.out = out; la.Rv = with_volume ? m.Rv : nullptr; la.dev_hi = m.dev_hi;
        la.dev_lo = m.dev_lo; la.Fmean = m.Fmean; la.S0 = m.S0; la.inv_detj = m.inv_detj; la.groups = m.egroups;
        la.t = m.t; la.ngroups = m.negroups; la.dt = dt; la.a0 = a0; la.a1 = a1; la.mode = mode;
        la.dt_inst = mode == 1 ? m.dt_inst : nullptr; la.elem_inst = m.elem_inst;
        la.out_mir_hi = mir_out >= 0 ? m.mir_hi[mir_out] : nullptr;
        la.out_mir_lo = mir_out >= 0 ? m.mir_lo[mir_out] : nullptr;
        const int g = (int)std::min<int64_t>((m.negroups + W - 1) / W, (int64_t)m.sms * 32);
        lift_mixed<NB, NQF, W><<<g, W * 32, 0, s>>>(la);
    }
    return cudaGetLastError() == cudaSuccess ? DG_OK : DG_E_CUDA;
}

// which: 0 = face fluxes, 3 = volume integrals, 1 = face integrals + update, 4 = mirror split.
// mir_in: mirror of U (0..3); mir_out: mirror the update writes (RK mode), or -1.
inline int mixed_kernel(MixedData& m, int which, const double* U, const double* U0, double* out, int mode,
                        double dt, double a0, double a1, int face_mask, int with_volume, cudaStream_t s,
                        std::atomic<int64_t>* launches, int mir_in, int mir_out) {
    if (!m.ready) return DG_E_ARG;
    ++*launches;
#define X(P, QV, QF, NB, NQV, NQF)                                                                          \
    if (m.order == P && m.qv == QV && m.qf == QF)                                                           \
        return mixed_launch<NB, NQV, NQF>(m, which, U, U0, out, mode, dt, a0, a1, face_mask, with_volume, s, \
                                          mir_in, mir_out);
    FVEDG_MIXED_COMBOS(X)
#undef X
    return DG_E_ARG;
}

// One stage: face fluxes on s, volume integrals on the side stream (forked from and joined back to
// s, which a CUDA graph capture turns into two parallel branches), then face integrals + update.
template <class Timed>
inline int mixed_stage(MixedData& m, const double* U, const double* U0, double* out, int mode, double dt, double a0,
                       double a1, int face_mask, int with_volume, cudaStream_t s, std::atomic<int64_t>* launches,
                       Timed&& timed, bool overlap, int mir_in, int mir_out) {
    int rc;
    auto K = [&](int which, int wv, cudaStream_t st) {
        return mixed_kernel(m, which, U, U0, out, mode, dt, a0, a1, face_mask, wv, st, launches, mir_in, mir_out);
    };
    if (with_volume && overlap) {
        if (cudaEventRecord(m.fork, s) != cudaSuccess || cudaStreamWaitEvent(m.side, m.fork, 0) != cudaSuccess)
            return DG_E_CUDA;
        if ((rc = K(3, 1, m.side))) return rc;
        if (cudaEventRecord(m.join, m.side) != cudaSuccess) return DG_E_CUDA;
        if ((rc = timed(0, [&] { return K(0, 1, s); }))) return rc;
        if (cudaStreamWaitEvent(s, m.join, 0) != cudaSuccess) return DG_E_CUDA;
    } else {
        if ((rc = timed(0, [&] { return K(0, 1, s); }))) return rc;
        if (with_volume && (rc = timed(3, [&] { return K(3, 1, s); }))) return rc;
    }
    return timed(1, [&] { return K(1, with_volume, s); });
}

// The mirror of an arbitrary state (the upload, the residual input) is written by a split kernel.
inline int mixed_mirror(MixedData& m, const double* U, int mir, cudaStream_t s, std::atomic<int64_t>* launches) {
    return mixed_kernel(m, 4, U, U, nullptr, 0, 0.0, 0.0, 0.0, 0, 0, s, launches, mir, -1);
}

inline int residual_mixed(MixedData& m, const double* U, double* R, int part, cudaStream_t s,
                          std::atomic<int64_t>* launches) {
    const int mask = part == 0 ? 3 : part == 1 ? 0 : part == 2 ? 1 : 2;
    int rc = mixed_mirror(m, U, 3, s, launches);
    if (rc) return rc;
    return mixed_stage(m, U, U, R, 0, 0.0, 0.0, 0.0, mask, part == 0 || part == 1, s, launches,
                       [](int, auto&& fn) { return fn(); }, false, 3, -1);
}

inline int mixed_launches_per_step(const MixedData&) { return 9; }

// SSP-RK3 step; `timed(cls, fn)` runs fn (one launch) and may bracket it with timing events. When
// timing, the volume kernel runs in line so each launch has its own interval. The mirror of Un
// must be current (the upload writes it, and stage 3 of every step rewrites it).
template <class Timed>
inline int step_mixed(MixedData& m, double* Un, double* Ua, double* Ub, double dt, cudaStream_t s,
                      std::atomic<int64_t>* launches, Timed&& timed, bool overlap = true) {
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {Un, Ua, Ub};
    double* out[3] = {Ua, Ub, Un};
    const int mi[3] = {0, 1, 2}, mo[3] = {1, 2, 0};
    for (int st = 0; st < 3; ++st) {
        const int rc = mixed_stage(m, in[st], Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, launches, timed, overlap,
                                   mi[st], mo[st]);
        if (rc) return rc;
    }
    return DG_OK;
}

}  // namespace fvedg
