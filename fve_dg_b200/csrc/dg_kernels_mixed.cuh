// Mixed-precision form of the explicit DG operator.
//
// The four dense contractions of a stage run on the tensor cores as BF16 MMAs with FP32
// accumulation (mma.sync m16n8k16, plus an m16n8k8 tail so every K is padded to 8, not 16). Both
// operands are split into hi + lo BF16 parts and the three products hi*hi + hi*lo + lo*hi are
// accumulated (about 16 significant bits per product):
//   face traces      U'(x_g) = sum_{b>=1} phi_b(xi_g^perm) c_b          B = face-map table
//   volume values    U'(x_g) = sum_{b>=1} phi_b(x_g) c_b                B = volume table
//   volume integral  R_v[j]  = -sum_{g,d} w_g dphi_j,d(x_g) G'_d(x_g)   B = weighted gradients
//   face integral    R_f[j]  = +-sum_g w_g phi_j(xi_g^perm) F'(x_g)     B = weighted face-map table
// The MMA's 16 rows hold (item, variable) pairs of three items (faces or elements) that share their
// face maps, so one table fragment serves three items. Items are grouped that way on the host.
//
// Two kernels per RK stage. The face kernel interpolates both traces, evaluates the Riemann flux
// and stores the flux deviations already split and in the element kernel's fragment order. The
// element kernel does the volume term (values, flux, integral) and the four face integrals into
// the same accumulators, then the FP64 parts and the RK update (FP64 state only: both kernels split
// the FP64 coefficient rows they read into BF16 hi/lo A fragments in registers, load_afrag_state).
//
// Operands kept in memory are in fragment order ("A rows" of the face records, "B fragments" of
// the tables, below): a lane fetches its MMA registers for one 16-wide K tile, hi and lo, with one
// 128-bit load.
//
// Only deviations go through the tensor cores: the mode-0 coefficient c_0 (phi_0 = 1) is added to
// the traces in FP32 after the MMA; the volume flux is taken relative to the flux of the element
// mean state and the face flux relative to a per-face reference (the physical flux of the
// cells[0] mean state), and those references are integrated in FP64 against precomputed moments
// (sum_g w_g dphi_j and sum_g w_g phi_j). The mode-0 face integral of each face is formed once, in
// the face kernel, so both sides receive exactly opposite amounts and the element means (mass,
// momentum, energy) are conserved to round-off. Large constant backgrounds (the p0 ~ 71 of a Mach
// 0.1 flow) never meet BF16 rounding. The pointwise flux and the Riemann solvers run in FP32; the
// RK stage update, the inverse mass and the state are FP64. The terms follow
// ExplicitConvection.cpp:144-272 one for one.
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
#include "dg_tma.cuh"

namespace fvedg {

__host__ __device__ constexpr int pad8(int x) { return (x + 7) / 8 * 8; }
__host__ __device__ constexpr int pad16(int x) { return (x + 15) / 16 * 16; }
// A shared-memory row stride >= n that is 8 (mod 16) floats: the 64-bit accesses of the MMA
// fragment pattern (4 rows x 4 column pairs per half warp) then touch 32 distinct banks.
__host__ __device__ constexpr int frag_ld(int n) { return n + ((8 - n % 16) + 16) % 16; }

// K tiling of one contraction: K / 16 full tiles and, when K = 8 (mod 16), one 8-wide tail.
template <int K>
struct KTiles {
    static_assert(K % 8 == 0, "K is padded to a multiple of 8");
    static constexpr int N16 = K / 16;
    static constexpr bool TAIL = (K % 16) != 0;
    static constexpr int NT_U32 = N16 * 128 + (TAIL ? 64 : 0);  // 32-bit words of one n-tile of a B table
};

// ---- A rows ---------------------------------------------------------------------------------------
// One MMA row of K values split into BF16 hi/lo, stored as K 32-bit words in fragment order: in a
// full 16-column tile, lane quad t (columns 2t, 2t+1, 2t+8, 2t+9) owns the 4 words
// {hi(2t,2t+1), hi(2t+8,2t+9), lo(2t,2t+1), lo(2t+8,2t+9)}; in the 8-column tail, quad t owns
// {hi(2t,2t+1), lo(2t,2t+1)}. Each word holds the lower column in its low half.
template <int K>
__host__ __device__ __forceinline__ int arow_hi_word(int x) {
    constexpr int N16 = K / 16;
    const int t = x >> 4;
    if (t < N16) {
        const int w = x & 15;
        return t * 16 + ((w & 7) >> 1) * 4 + (w >> 3);
    }
    return N16 * 16 + ((x - N16 * 16) >> 1) * 2;
}
template <int K>
__host__ __device__ __forceinline__ int arow_lo_word(int x) {
    return arow_hi_word<K>(x) + ((x >> 4) < K / 16 ? 2 : 1);
}

// Face record of the mixed form, written by the face kernel and read by both elements of the face:
//   words [0, 5 KF)        A rows (one per variable) of the split flux deviations 2A F(x_g) - Fref
//   doubles [0, 5) after   Fref: the reference flux 2A F(c_0 of cells[0]) . n
//   doubles [5, 10) after  S0: the mode-0 face integral sum_g w_g 2A F
// face_rec_words(NQF) 32-bit words per face, a multiple of 4 (16 bytes) so that a face record is
// one bulk copy.
__host__ __device__ constexpr int face_rec_words(int nqf) { return 5 * pad8(nqf) + 20; }
template <int NQF>
__host__ __device__ __forceinline__ double* face_rec_fs(uint32_t* rec) {
    return reinterpret_cast<double*>(rec + 5 * pad8(NQF));
}
template <int NQF>
__host__ __device__ __forceinline__ const double* face_rec_fs(const uint32_t* rec) {
    return reinterpret_cast<const double*>(rec + 5 * pad8(NQF));
}

struct MixedTables {  // device pointers
    const uint32_t* tfa;     // [24 maps] B fragments of the face traces: n = face point, k = mode - 1
    const uint32_t* tva;     // B fragments of the volume values: n = volume point, k = mode - 1
    const uint32_t* tvp;     // B fragments of the volume integral: n = mode, k = (point, dir), w dphi
    const uint32_t* tfl;     // [24 maps] B fragments of the face integral: n = mode, k = face point, w phi
    const double* mv;        // [NB][3]  sum_g w_g dphi_j
    const double* mf;        // [24][NB] sum_g w_g phi_j(xi_g^perm)
    const float* wf32;       // [NQF] face weights
    const double* inv_mass;  // [NB] 1 / sum_g w_g phi_j^2
    double wsum;             // sum_g w_g of the face rule
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
    const FaceInfo* fi;
    const FaceGroup* groups;
    const double* UD;
    uint32_t* dev;          // [nface][face_rec_words] face records (layout at face_rec_words)
    MixedTables t;
    int ngroups;
    float gamma;
    int flux;
    int faces_mask;
};

struct MixedElemArgs {
    const double* U;
    const double* U0;
    double* out;
    const uint32_t* dev;     // face records (written by the face kernel)
    const double* geo;       // [ncell][10] J^-T row-major, detJ
    const double* inv_detj;  // [ncell]
    const ElemGroup* groups;
    MixedTables t;
    int ngroups;
    float gamma;
    int volume;              // 0: leave the volume term out (residual parts 2 and 3)
    double dt, a0, a1;
    int mode;                // 0: out = R; 1: out = a0 U0 + a1 (U - dt M^-1 R)
    const double* dt_inst;   // optional per-instance time step (ensembles), indexed by elem_inst
    const int* elem_inst;    // [ncell] instance of each element
    const double* Rv;        // RK mode: viscous residual subtracted from R (Navier-Stokes), or null
    int* err;                // device status word (DG_E_WATCHDOG when a bounded wait ran out), or null
};

// ---- MMA helpers ----------------------------------------------------------------------------------
__device__ __forceinline__ void mma16816(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ void mma1688(float d[4], const uint32_t a[2], uint32_t b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(b));
}

__device__ __forceinline__ uint32_t bf2_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// (x0, x1) = hi + lo, both pairs packed BF16 (x0 in the low half)
__device__ __forceinline__ void split2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
    hi = bf2_bits(h);
    lo = bf2_bits(__floats2bfloat162_rn(x0 - __low2float(h), x1 - __high2float(h)));
}
__device__ __forceinline__ void split1(float x, unsigned short& hi, unsigned short& lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(__float2bfloat16_rn(x - __bfloat162float(h)));
}

// A operand registers of a K-wide contraction (per full tile: the 4 hi and 4 lo MMA registers).
template <int K>
struct AFrag {
    static constexpr int N = KTiles<K>::N16 > 0 ? KTiles<K>::N16 : 1;
    uint32_t h[N][4], l[N][4];
    uint32_t th[2], tl[2];
};

// Rows gid and gid + 8 from A rows in global memory (null: a zero row). `Coherent` reads through
// L2 only, for data written earlier in the same launch (the persistent schedule).
template <int K, bool Coherent>
__device__ __forceinline__ void load_afrag(AFrag<K>& A, const uint32_t* r0, const uint32_t* r1, int lane,
                                           uint32_t flip = 0u) {
    const int tq = lane & 3;
    #pragma unroll
    for (int t = 0; t < KTiles<K>::N16; ++t) {
        uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
        if (r0) v0 = Coherent ? __ldcg(reinterpret_cast<const uint4*>(r0 + t * 16 + tq * 4))
                              : __ldg(reinterpret_cast<const uint4*>(r0 + t * 16 + tq * 4));
        if (r1) v1 = Coherent ? __ldcg(reinterpret_cast<const uint4*>(r1 + t * 16 + tq * 4))
                              : __ldg(reinterpret_cast<const uint4*>(r1 + t * 16 + tq * 4));
        A.h[t][0] = v0.x ^ flip; A.h[t][1] = v1.x ^ flip; A.h[t][2] = v0.y ^ flip; A.h[t][3] = v1.y ^ flip;
        A.l[t][0] = v0.z ^ flip; A.l[t][1] = v1.z ^ flip; A.l[t][2] = v0.w ^ flip; A.l[t][3] = v1.w ^ flip;
    }
    if constexpr (KTiles<K>::TAIL) {
        constexpr int o = KTiles<K>::N16 * 16;
        uint2 u0 = make_uint2(0u, 0u), u1 = u0;
        if (r0) u0 = Coherent ? __ldcg(reinterpret_cast<const uint2*>(r0 + o + tq * 2))
                              : __ldg(reinterpret_cast<const uint2*>(r0 + o + tq * 2));
        if (r1) u1 = Coherent ? __ldcg(reinterpret_cast<const uint2*>(r1 + o + tq * 2))
                              : __ldg(reinterpret_cast<const uint2*>(r1 + o + tq * 2));
        A.th[0] = u0.x ^ flip; A.th[1] = u1.x ^ flip;
        A.tl[0] = u0.y ^ flip; A.tl[1] = u1.y ^ flip;
    }
}

// Rows gid and gid + 8 of an A operand straight from FP64 state rows (null: a zero row): r points
// at a cell's variable-k coefficients, mode b at r[5 b]; column x of the row is mode x + 1 (the
// deviation modes), split into BF16 hi/lo in registers exactly as a stored split row would be.
template <int K, int NB, bool SMEM = false>
__device__ __forceinline__ void load_afrag_state(AFrag<K>& A, const double* r0, const double* r1, int lane) {
    const int tq = lane & 3;
    auto v = [&](const double* r, int x) -> float {
        if (!r || x + 1 >= NB) return 0.f;
        if constexpr (SMEM) return (float)r[5 * (x + 1)];
        else return (float)__ldg(r + 5 * (x + 1));
    };
    #pragma unroll
    for (int t = 0; t < KTiles<K>::N16; ++t) {
        const int c = t * 16 + 2 * tq;
        split2(v(r0, c), v(r0, c + 1), A.h[t][0], A.l[t][0]);
        split2(v(r1, c), v(r1, c + 1), A.h[t][1], A.l[t][1]);
        split2(v(r0, c + 8), v(r0, c + 9), A.h[t][2], A.l[t][2]);
        split2(v(r1, c + 8), v(r1, c + 9), A.h[t][3], A.l[t][3]);
    }
    if constexpr (KTiles<K>::TAIL) {
        const int c = KTiles<K>::N16 * 16 + 2 * tq;
        split2(v(r0, c), v(r0, c + 1), A.th[0], A.tl[0]);
        split2(v(r1, c), v(r1, c + 1), A.th[1], A.tl[1]);
    }
}

// acc += A(full tile t) * B(n-tile at tbn, tile t): three products
__device__ __forceinline__ void mma3_tile(float acc[4], const uint32_t h[4], const uint32_t l[4], const uint32_t* tbn,
                                          int t, int lane) {
    const uint4 b = __ldg(reinterpret_cast<const uint4*>(tbn + t * 128 + lane * 4));
    mma16816(acc, h, b.x, b.y);
    mma16816(acc, h, b.z, b.w);
    mma16816(acc, l, b.x, b.y);
}
template <int K>
__device__ __forceinline__ void mma3_tail(float acc[4], const uint32_t h[2], const uint32_t l[2], const uint32_t* tbn,
                                          int lane) {
    const uint2 b = __ldg(reinterpret_cast<const uint2*>(tbn + KTiles<K>::N16 * 128 + lane * 2));
    mma1688(acc, h, b.x);
    mma1688(acc, h, b.y);
    mma1688(acc, l, b.x);
}

// acc += A * B(n-tile nt) over the whole K of a fragment-ordered table tb
template <int K>
__device__ __forceinline__ void mma_bt(float acc[4], const AFrag<K>& A, const uint32_t* tb, int nt, int lane) {
    const uint32_t* tbn = tb + nt * KTiles<K>::NT_U32;
    #pragma unroll
    for (int t = 0; t < KTiles<K>::N16; ++t) mma3_tile(acc, A.h[t], A.l[t], tbn, t, lane);
    if constexpr (KTiles<K>::TAIL) mma3_tail<K>(acc, A.th, A.tl, tbn, lane);
}

// ------------------------------------------------------------------------------------------------
// Face fluxes: one warp per face group. Trace deviations of each side for the three faces (rows
// (face, var)) on the tensor cores, c_0 added in FP32; one lane per face point evaluates the FP32
// Riemann flux and writes 2A F - Fref, split, into the element kernel's A rows; then the mode-0
// integral of each face.
// ------------------------------------------------------------------------------------------------
template <int NQF>
struct alignas(16) FaceMixedSmem {
    static constexpr int MF = pad8(NQF), LD = frag_ld(MF);
    float sU[2][16][LD];  // traces of side 0 / 1, rows (face, var), cols face point
    float sC0[2][16];     // c_0 of the rows
    float sRef[3][5];     // reference flux of each face
    float sN[3][4];       // unit normal and 2A
};

template <int NB, int NQF>
__device__ __forceinline__ void face_group_mixed(const MixedFaceArgs& a, int gi, FaceMixedSmem<NQF>& sm, int lane) {
    using S = FaceMixedSmem<NQF>;
    constexpr int KB = pad8(NB - 1), MF = S::MF, KF = pad8(NQF);
    const int gid = lane >> 2, tq = lane & 3;
    const FaceGroup grp = a.groups[gi];
    const FaceInfo f0 = a.fi[grp.f[0]];  // shares perms and kind with the others
    const int perm[2] = {f0.meta & 0xff, (f0.meta >> 8) & 0xff};
    const int bc = (f0.meta >> 16) & 0xff;
    const bool interior = f0.c1 >= 0;
    const bool active = interior ? (a.faces_mask & 1)
                                 : ((a.faces_mask & 2) && ((bc == 0 && a.UD != nullptr) || bc == 5));
    constexpr int FR = face_rec_words(NQF);
    if (!active) {
        for (int i = lane; i < grp.n * FR; i += 32) {
            const int fl = i / FR;
            a.dev[(int64_t)grp.f[fl] * FR + (i - fl * FR)] = 0u;
        }
        return;
    }
    const int nside = interior ? 2 : 1;
    if (lane < 16 * nside) {
        const int s = lane >> 4, r = lane & 15;
        float v = 0.f;
        if (r < 5 * grp.n) {
            const FaceInfo& F = a.fi[grp.f[r / 5]];
            v = (float)__ldg(a.U + (int64_t)(s ? F.c1 : F.c0) * (5 * NB) + r % 5);
        }
        sm.sC0[s][r] = v;
    }
    if (lane < grp.n) {  // normal, 2A and the reference flux 2A F(c_0 of cells[0]) . n of each face
        const FaceInfo& F = a.fi[grp.f[lane]];
        float c0[5], n[3], Fn[5], rho, vel[3], p;
        #pragma unroll
        for (int k = 0; k < 5; ++k) c0[k] = (float)__ldg(a.U + (int64_t)F.c0 * (5 * NB) + k);
        #pragma unroll
        for (int i = 0; i < 3; ++i) n[i] = (float)F.n[i];
        const float jw = (float)F.jw;
        Phys<float>::flux_n(c0, n, a.gamma - 1.f, Fn, rho, vel, p);
        #pragma unroll
        for (int k = 0; k < 5; ++k) sm.sRef[lane][k] = Fn[k] * jw;
        sm.sN[lane][0] = n[0]; sm.sN[lane][1] = n[1]; sm.sN[lane][2] = n[2]; sm.sN[lane][3] = jw;
    }
    __syncwarp();
    for (int s = 0; s < nside; ++s) {
        const double* p0 = nullptr;
        const double* p1 = nullptr;
        if (gid < 5 * grp.n) {
            const FaceInfo& F = a.fi[grp.f[gid / 5]];
            p0 = a.U + (int64_t)(s ? F.c1 : F.c0) * (5 * NB) + gid % 5;
        }
        if (gid + 8 < 5 * grp.n) {
            const FaceInfo& F = a.fi[grp.f[(gid + 8) / 5]];
            p1 = a.U + (int64_t)(s ? F.c1 : F.c0) * (5 * NB) + (gid + 8) % 5;
        }
        AFrag<KB> A;
        load_afrag_state<KB, NB>(A, p0, p1, lane);
        const uint32_t* tb = a.t.tfa + perm[s] * (MF / 8) * KTiles<KB>::NT_U32;
        const float c00 = sm.sC0[s][gid], c01 = sm.sC0[s][gid + 8];
        #pragma unroll
        for (int nt = 0; nt < MF / 8; ++nt) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            mma_bt<KB>(acc, A, tb, nt, lane);
            *reinterpret_cast<float2*>(&sm.sU[s][gid][nt * 8 + 2 * tq]) = make_float2(acc[0] + c00, acc[1] + c00);
            *reinterpret_cast<float2*>(&sm.sU[s][gid + 8][nt * 8 + 2 * tq]) = make_float2(acc[2] + c01, acc[3] + c01);
        }
    }
    __syncwarp();
    for (int p = lane; p < grp.n * NQF; p += 32) {
        const int fl = p / NQF, g = p - fl * NQF;
        const int f = grp.f[fl];
        float UL[5], UR[5];
        #pragma unroll
        for (int k = 0; k < 5; ++k) UL[k] = sm.sU[0][fl * 5 + k][g];
        if (interior) {
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = sm.sU[1][fl * 5 + k][g];
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
        if (a.flux == 1) roe_f32(UL, UR, n, a.gamma, Fh);
        else lax_friedrichs_f32(UL, UR, n, a.gamma, Fh);
        const float jw = sm.sN[fl][3], w = __ldg(a.t.wf32 + g);
        unsigned short* drow = reinterpret_cast<unsigned short*>(a.dev + (int64_t)f * FR);
        const int hw = 2 * arow_hi_word<KF>(g) + (g & 1), lw = 2 * arow_lo_word<KF>(g) + (g & 1);
        #pragma unroll
        for (int k = 0; k < 5; ++k) {
            const float d = Fh[k] * jw - sm.sRef[fl][k];
            unsigned short h, l;
            split1(d, h, l);
            drow[2 * k * KF + hw] = h;
            drow[2 * k * KF + lw] = l;
            sm.sU[0][fl * 5 + k][g] = w * d;  // side 0 is no longer needed: keep w_g d_g for the sums
        }
    }
    __syncwarp();
    {   // mode-0 integral sum_g w_g 2A F = Fref sum_g w_g + sum_g w_g d_g, summed in one fixed order
        // per face: both sides of the face then use the same number, which is what makes the
        // element means conserved exactly
        constexpr int NH = (NQF + 1) / 2;
        const int r = lane >> 1, h = lane & 1;
        float s = 0.f;
        if (r < 5 * grp.n) {
            const int g1 = h ? NQF : NH;
            for (int g = h ? NH : 0; g < g1; ++g) s += sm.sU[0][r][g];
        }
        const float tot = s + __shfl_xor_sync(0xffffffffu, s, 1);
        if (h == 0 && r < 5 * grp.n) {
            const int fl = r / 5, k = r - 5 * fl;
            double* fs = face_rec_fs<NQF>(a.dev + (int64_t)grp.f[fl] * FR);
            const double ref = (double)sm.sRef[fl][k];
            fs[k] = ref;
            fs[5 + k] = ref * a.t.wsum + (double)tot;
        }
    }
    __syncwarp();
}

template <int NB, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, NB <= 20 ? 36 / WARPS : 24 / WARPS) face_flux_mixed(MixedFaceArgs a) {
    __shared__ FaceMixedSmem<NQF> sm[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int gi = blockIdx.x * WARPS + warp; gi < a.ngroups; gi += gridDim.x * WARPS)
        face_group_mixed<NB, NQF>(a, gi, sm[warp], lane);
}

// ------------------------------------------------------------------------------------------------
// Elements: one warp per element group. Volume values on the tensor cores, FP32 flux, deviations
// from the flux of the element mean state, the volume integral and the four face integrals into
// one set of accumulators; then the FP64 parts, the RK update and the new stage's A rows.
// ------------------------------------------------------------------------------------------------
template <int NB, int NQV, int NQF>
struct alignas(16) ElemMixedSmem {
    static constexpr int MV = pad8(NQV), KV = pad8(3 * NQV), MJ = pad8(NB);
    static constexpr int LDU = frag_ld(MV), LDG = frag_ld(KV);
    // FP64 residual rows: stride = 8 (mod 16) doubles, so the 16-byte stores of the accumulator
    // pattern (two rows x four column pairs per quarter warp) hit 32 distinct banks
    static constexpr int LDR = MJ + ((8 - MJ % 16) + 16) % 16;
    // 15 rows hold (element, var) pairs (row 15 is never a valid row); the FP64 residual [16][LDR]
    // reuses the space once the volume integral is done
    static constexpr int GROWS = 15 * LDG >= 32 * LDR ? 15 : (32 * LDR + LDG - 1) / LDG;
    float sU[16][LDU];       // volume values (c_0 added), rows (element, var), cols point
    float sG[GROWS][LDG];    // Gb - G, rows (element, var), cols (point, dir), padding columns zero
    double sGb[3][15];       // detJ F(c_0) J^-T of each element (FP64)
    double sDT[3];           // dt / detJ of each element
    float sJ[3][9];          // detJ J^-T, FP32
    float sGbf[3][15];
    float sC0[16];
    int sE[3];
};

// Per-block tables of the element kernel's epilogue: for DOF r = 5 j + k of an element, (j, k); and
// the inverse reference mass.
template <int NB>
struct ElemTables {
    int2 dof[5 * NB];
    double inv_mass[NB];
};

template <int NB>
__device__ __forceinline__ void element_tables_init(ElemTables<NB>& T, const double* inv_mass) {
    for (int r = threadIdx.x; r < 5 * NB; r += blockDim.x) {
        const int j = r / 5, k = r - 5 * j;
        T.dof[r] = make_int2(j, k);
    }
    for (int j = threadIdx.x; j < NB; j += blockDim.x) T.inv_mass[j] = inv_mass[j];
    __syncthreads();
}

// One DOF of the SSP-RK3 stage update, a0 U^n + a1 (U - s R) with s = dt / (det J M_j), every
// product and sum rounded explicitly, so that every element kernel computes it bit for bit alike
// (left to the compiler, the contraction into FMAs may differ between kernels).
__device__ __forceinline__ double rk_update(bool with_u0, double a0, double u0, double a1, double u, double s,
                                            double R) {
    const double x = __fma_rn(-s, R, u);
    return with_u0 ? __fma_rn(a1, x, __dmul_rn(a0, u0)) : __dmul_rn(a1, x);
}

__device__ __forceinline__ void dmma884(double d[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// The element kernel's B tables (fragment order): volume values, volume integral, the 24 face-integral
// tables.
struct ElemBTabs {
    const uint32_t* tva;
    const uint32_t* tvp;
    const uint32_t* tfl;
};

template <int NB, int NQV, int NQF>
__device__ __forceinline__ void element_group_mixed(const MixedElemArgs& a, int gi, ElemMixedSmem<NB, NQV, NQF>& sm,
                                                    const ElemTables<NB>& T, int lane, const ElemBTabs& bt) {
    using S = ElemMixedSmem<NB, NQV, NQF>;
    constexpr int KB = pad8(NB - 1), MV = S::MV, KV = S::KV, MJ = S::MJ, KF = pad8(NQF), NT = MJ / 8, LDR = S::LDR;
    const int gid = lane >> 2, tq = lane & 3;
    const ElemGroup& grp = a.groups[gi];  // read in place (a copy would live in local memory)
    const int ne = grp.n;
    const int r0 = gid, r1 = gid + 8;
    const bool v0 = r0 < 5 * ne, v1 = r1 < 5 * ne;
    // Pull the group's face records and stage input rows into L2 first (the addresses are known
    // from the group record): they arrive while the earlier phases run, instead of one dependent
    // DRAM round trip per phase. Prefetches take no registers; every address lies inside its row.
    constexpr int FR = face_rec_words(NQF);
    {
        constexpr int NL = (FR * 4 + 127) / 128;
        for (int i = lane; i < ne * 4 * NL; i += 32) {
            const int fq = i / NL, part = i - fq * NL;
            const int64_t f = grp.face[fq >> 2][fq & 3];
            const char* addr = reinterpret_cast<const char*>(a.dev + f * FR) + part * 128;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(addr));
        }
    }
    {
        constexpr int MB = 5 * NB * 8, ML = (MB + 127) / 128;
        for (int i = lane; i < ne * ML; i += 32) {
            const int el = i / ML, part = i - el * ML;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(
                reinterpret_cast<const char*>(a.U + (int64_t)grp.e[el] * 5 * NB) + part * 128));
        }
    }
    if (lane < 16) sm.sC0[lane] = lane < 5 * ne ? (float)__ldg(a.U + (int64_t)grp.e[lane / 5] * (5 * NB) + lane % 5) : 0.f;
    if (lane < ne) {
        const int e = grp.e[lane];
        sm.sE[lane] = e;
        const double dt = a.dt_inst ? __ldg(a.dt_inst + __ldg(a.elem_inst + e)) : a.dt;
        sm.sDT[lane] = dt * __ldg(a.inv_detj + e);
    }
    if (a.volume && lane < 5 * ne) {  // row k of G(c_0) = detJ F(c_0) J^-T, FP64, one lane per (element, var)
        const int el = lane / 5, k = lane - 5 * el;
        const int64_t e = grp.e[el];
        const double* geo = a.geo + e * 10;
        double c[5], J[9];
        #pragma unroll
        for (int i = 0; i < 5; ++i) c[i] = __ldg(a.U + e * (5 * NB) + i);
        #pragma unroll
        for (int i = 0; i < 9; ++i) J[i] = __ldg(geo + i);
        const double dj = __ldg(geo + 9);
        const double rho = c[0] > 1e-16 ? c[0] : 1e-16, ir = 1.0 / rho;
        const double u[3] = {c[1] * ir, c[2] * ir, c[3] * ir}, en = c[4] * ir;
        const double p = ((double)a.gamma - 1.0) * (rho * en - 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        double F[3];
        if (k == 0) {
            F[0] = rho * u[0]; F[1] = rho * u[1]; F[2] = rho * u[2];
        } else if (k < 4) {
            #pragma unroll
            for (int i = 0; i < 3; ++i) F[i] = rho * u[i] * u[k - 1] + (i == k - 1 ? p : 0.0);
        } else {
            #pragma unroll
            for (int i = 0; i < 3; ++i) F[i] = u[i] * (rho * en + p);
        }
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double gb = dj * (F[0] * J[d] + F[1] * J[3 + d] + F[2] * J[6 + d]);
            sm.sGb[el][3 * k + d] = gb;
            sm.sGbf[el][3 * k + d] = (float)gb;
        }
        if (k == 0) {
            #pragma unroll
            for (int i = 0; i < 9; ++i) sm.sJ[el][i] = (float)(dj * J[i]);
        }
    }
    __syncwarp();
    float acc[NT][4];
    #pragma unroll
    for (int nt = 0; nt < NT; ++nt)
        #pragma unroll
        for (int r = 0; r < 4; ++r) acc[nt][r] = 0.f;
    if (a.volume) {
        {   // values at the volume points
            AFrag<KB> A;
            load_afrag_state<KB, NB>(A, v0 ? a.U + (int64_t)grp.e[r0 / 5] * (5 * NB) + r0 % 5 : nullptr,
                                     v1 ? a.U + (int64_t)grp.e[r1 / 5] * (5 * NB) + r1 % 5 : nullptr, lane);
            const float c00 = sm.sC0[r0], c01 = sm.sC0[r1];
            #pragma unroll
            for (int nt = 0; nt < MV / 8; ++nt) {
                float o[4] = {0.f, 0.f, 0.f, 0.f};
                mma_bt<KB>(o, A, bt.tva, nt, lane);
                *reinterpret_cast<float2*>(&sm.sU[r0][nt * 8 + 2 * tq]) = make_float2(o[0] + c00, o[1] + c00);
                *reinterpret_cast<float2*>(&sm.sU[r1][nt * 8 + 2 * tq]) = make_float2(o[2] + c01, o[3] + c01);
            }
        }
        // the MMA reads columns up to KV: the padding past 3 NQV must be zero (the FP64 residual of
        // the previous group shares this memory)
        if constexpr (KV > 3 * NQV) {
            constexpr int w = KV - 3 * NQV;
            for (int i = lane; i < 15 * w; i += 32) sm.sG[i / w][3 * NQV + i % w] = 0.f;
        }
        __syncwarp();
        const float gm1 = a.gamma - 1.f;
        for (int p = lane; p < ne * NQV; p += 32) {
            const int el = p / NQV, g = p - el * NQV;
            float U[5], F[5][3];
            #pragma unroll
            for (int k = 0; k < 5; ++k) U[k] = sm.sU[el * 5 + k][g];
            flux_f32(U, gm1, F);
            const float* J = sm.sJ[el];
            #pragma unroll
            for (int k = 0; k < 5; ++k)
                #pragma unroll
                for (int d = 0; d < 3; ++d)
                    sm.sG[el * 5 + k][3 * g + d] =
                        fmaf(-F[k][0], J[d], fmaf(-F[k][1], J[3 + d], fmaf(-F[k][2], J[6 + d], sm.sGbf[el][3 * k + d])));
        }
        __syncwarp();
        // volume integral: acc += (Gb - G) * (w dphi), split on the fly
        #pragma unroll
        for (int t = 0; t < KTiles<KV>::N16; ++t) {
            const int c = t * 16 + 2 * tq;
            uint32_t h[4] = {0u, 0u, 0u, 0u}, l[4] = {0u, 0u, 0u, 0u};
            if (v0) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r0][c]);
                const float2 y = *reinterpret_cast<const float2*>(&sm.sG[r0][c + 8]);
                split2(x.x, x.y, h[0], l[0]);
                split2(y.x, y.y, h[2], l[2]);
            }
            if (v1) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r1][c]);
                const float2 y = *reinterpret_cast<const float2*>(&sm.sG[r1][c + 8]);
                split2(x.x, x.y, h[1], l[1]);
                split2(y.x, y.y, h[3], l[3]);
            }
            #pragma unroll
            for (int nt = 0; nt < NT; ++nt) mma3_tile(acc[nt], h, l, bt.tvp + nt * KTiles<KV>::NT_U32, t, lane);
        }
        if constexpr (KTiles<KV>::TAIL) {
            const int c = KTiles<KV>::N16 * 16 + 2 * tq;
            uint32_t h[2] = {0u, 0u}, l[2] = {0u, 0u};
            if (v0) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r0][c]);
                split2(x.x, x.y, h[0], l[0]);
            }
            if (v1) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r1][c]);
                split2(x.x, x.y, h[1], l[1]);
            }
            #pragma unroll
            for (int nt = 0; nt < NT; ++nt) mma3_tail<KV>(acc[nt], h, l, bt.tvp + nt * KTiles<KV>::NT_U32, lane);
        }
    }
    // face integrals: the flux deviations arrive split, in fragment order; side 1 negated exactly
    auto face_rows = [&](AFrag<KF>& A, int q) {
        const uint32_t flip = (grp.meta[q] >> 8) ? 0x80008000u : 0u;
        load_afrag<KF, true>(A, v0 ? a.dev + (int64_t)grp.face[r0 / 5][q] * FR + (r0 % 5) * KF : nullptr,
                             v1 ? a.dev + (int64_t)grp.face[r1 / 5][q] * FR + (r1 % 5) * KF : nullptr, lane, flip);
    };
    #pragma unroll
    for (int q = 0; q < 4; ++q) {
        AFrag<KF> A;
        face_rows(A, q);
        const uint32_t* tb = bt.tfl + (grp.meta[q] & 0xff) * NT * KTiles<KF>::NT_U32;
        #pragma unroll
        for (int nt = 0; nt < NT; ++nt) mma_bt<KF>(acc[nt], A, tb, nt, lane);
    }
    __syncwarp();  // sG is free
    // FP64 parts on the FP64 tensor cores, in the accumulators' own layout (rows gid / gid + 8,
    // columns 2 tq, 2 tq + 1 of each n-tile): R = acc + [Fr_q, Gb_d] x [+-mf_q(j), -mv_d(j)], K = 8
    // (four face references, three volume reference components, one zero)
    {
        double* sR = reinterpret_cast<double*>(&sm.sG[0][0]);
        const int mq = grp.meta[tq];  // face q = tq: its map and side
        const double sq = (mq >> 8) ? -1.0 : 1.0;
        double am[2][2], s0[2] = {0.0, 0.0};  // A(row gid + 8 mt, column 4 kt + tq); mode-0 sums
        #pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int row = gid + 8 * mt, el = row / 5, k = row - 5 * el;
            const bool ok = row < 5 * ne;
            am[mt][0] = ok ? __ldcg(face_rec_fs<NQF>(a.dev + (int64_t)grp.face[el][tq] * FR) + k) : 0.0;
            am[mt][1] = (ok && a.volume && tq < 3) ? sm.sGb[el][3 * k + tq] : 0.0;
            if (ok && tq == 0) {  // the exact mode-0 face sums, in a fixed order
                #pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double v = __ldcg(face_rec_fs<NQF>(a.dev + (int64_t)grp.face[el][q] * FR) + 5 + k);
                    s0[mt] += (grp.meta[q] >> 8) ? -v : v;
                }
            }
        }
        #pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int jb = nt * 8 + gid;  // B(k = 4 kt + tq, n = jb)
            const double b0 = jb < NB ? sq * __ldg(a.t.mf + (mq & 0xff) * NB + jb) : 0.0;
            const double b1 = (jb < NB && tq < 3) ? -__ldg(a.t.mv + 3 * jb + tq) : 0.0;
            #pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                double d[2] = {(double)acc[nt][2 * mt], (double)acc[nt][2 * mt + 1]};
                dmma884(d, am[mt][0], b0);
                dmma884(d, am[mt][1], b1);
                const int row = gid + 8 * mt;
                if (nt == 0 && tq == 0) d[0] = s0[mt];  // mode 0 (grad phi_0 = 0): the exact face sums only
                *reinterpret_cast<double2*>(sR + row * LDR + nt * 8 + 2 * tq) = make_double2(d[0], d[1]);
            }
        }
    }
    __syncwarp();
    // epilogue over the group's DOFs in memory order (coalesced FP64 traffic)
    const double* sR = reinterpret_cast<const double*>(&sm.sG[0][0]);
    if (a.mode == 0) {
        for (int i = lane; i < ne * 5 * NB; i += 32) {
            const int el = i / (5 * NB), r = i - el * (5 * NB);
            const int2 d = T.dof[r];
            const int64_t idx = (int64_t)sm.sE[el] * (5 * NB) + r;
            const double R = sR[(el * 5 + d.y) * LDR + d.x];
            a.out[idx] = a.Rv ? R - a.Rv[idx] : R;
        }
    } else {
        // RK update. The state rows are read in batches of EB DOFs per lane, every load of a batch
        // issued before its first use, so a group pays two dependent round trips for them instead
        // of one per round of 32 DOFs. Stage 1 has a0 = 0: U^n is not read twice. U^n may be the
        // output buffer (stage 3) and is read through the coherent path.
        constexpr int NPL = (15 * NB + 31) / 32, EB = (NPL + 1) / 2;
        const int ndof = ne * 5 * NB;
        const bool u0 = a.a0 != 0.0;
        #pragma unroll
        for (int b0 = 0; b0 < NPL; b0 += EB) {
            double uu[EB], vv[EB];
            int64_t ix[EB];
            #pragma unroll
            for (int j = 0; j < EB; ++j) {
                const int i = lane + 32 * (b0 + j);
                const int el = i / (5 * NB), r = i - el * (5 * NB);
                ix[j] = i < ndof ? (int64_t)sm.sE[el] * (5 * NB) + r : -1;
                uu[j] = ix[j] >= 0 ? __ldg(a.U + ix[j]) : 0.0;
                vv[j] = (ix[j] >= 0 && u0) ? a.U0[ix[j]] : 0.0;
            }
            #pragma unroll
            for (int j = 0; j < EB; ++j) {
                if (ix[j] < 0) continue;
                const int i = lane + 32 * (b0 + j);
                const int el = i / (5 * NB), r = i - el * (5 * NB);
                const int2 d = T.dof[r];  // mode j, variable k
                const double R = a.Rv ? sR[(el * 5 + d.y) * LDR + d.x] - a.Rv[ix[j]] : sR[(el * 5 + d.y) * LDR + d.x];
                const double un = rk_update(u0, a.a0, vv[j], a.a1, uu[j], __dmul_rn(sm.sDT[el], T.inv_mass[d.x]), R);
                a.out[ix[j]] = un;
            }
        }
    }
    __syncwarp();
}

// ------------------------------------------------------------------------------------------------
// Staged element kernel. The plain element kernel issues its global loads phase by phase (the
// stage input rows, the face records, the FP64 parts, then the state rows of the update), so a
// group waits for several dependent L2/DRAM round trips. Here lane 0 of the warp issues TMA bulk
// copies of every row the group reads (the four face records of each element, the stage input and
// U^n rows, the geometry) into the warp's staging area as soon as the group record is known; the
// warp waits once on its mbarrier and every later phase reads shared memory.
// State rows must be whole 16-byte units (5 NB doubles: P1..P3).
// ------------------------------------------------------------------------------------------------
template <int NB, int NQF>
struct alignas(16) ElemStage {
    static constexpr int KB = pad8(NB - 1), FR = face_rec_words(NQF);
    static constexpr unsigned FRB = FR * 4, UB = 5 * NB * 8, GEOB = 80;
    uint32_t face[3][4][FR];  // the face records of each element's faces, canonical face order
    double U[3][5 * NB];      // stage input rows
    double U0[3][5 * NB];     // U^n rows (stages with a0 != 0)
    double geo[3][10];        // J^-T row-major, det J
    uint64_t bar;             // completion of the group's copies (one phase per group)
};

template <int K>
__device__ __forceinline__ void load_afrag_smem(AFrag<K>& A, const uint32_t* r0, const uint32_t* r1, int lane,
                                                uint32_t flip = 0u) {
    const int tq = lane & 3;
    #pragma unroll
    for (int t = 0; t < KTiles<K>::N16; ++t) {
        uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
        if (r0) v0 = *reinterpret_cast<const uint4*>(r0 + t * 16 + tq * 4);
        if (r1) v1 = *reinterpret_cast<const uint4*>(r1 + t * 16 + tq * 4);
        A.h[t][0] = v0.x ^ flip; A.h[t][1] = v1.x ^ flip; A.h[t][2] = v0.y ^ flip; A.h[t][3] = v1.y ^ flip;
        A.l[t][0] = v0.z ^ flip; A.l[t][1] = v1.z ^ flip; A.l[t][2] = v0.w ^ flip; A.l[t][3] = v1.w ^ flip;
    }
    if constexpr (KTiles<K>::TAIL) {
        constexpr int o = KTiles<K>::N16 * 16;
        uint2 u0 = make_uint2(0u, 0u), u1 = u0;
        if (r0) u0 = *reinterpret_cast<const uint2*>(r0 + o + tq * 2);
        if (r1) u1 = *reinterpret_cast<const uint2*>(r1 + o + tq * 2);
        A.th[0] = u0.x ^ flip; A.th[1] = u1.x ^ flip;
        A.tl[0] = u0.y ^ flip; A.tl[1] = u1.y ^ flip;
    }
}

// One element group from the staging area; returns false when the copies did not land within the
// poll limit (the status word is set and the warp stops).
template <int NB, int NQV, int NQF>
__device__ __forceinline__ bool element_group_staged(const MixedElemArgs& a, int gi, ElemMixedSmem<NB, NQV, NQF>& sm,
                                                     ElemStage<NB, NQF>& st, const ElemTables<NB>& T, int lane,
                                                     const ElemBTabs& bt, unsigned parity) {
    using S = ElemMixedSmem<NB, NQV, NQF>;
    using G = ElemStage<NB, NQF>;
    static_assert((5 * NB * 8) % 16 == 0, "state rows must be whole 16-byte units for the bulk copies");
    constexpr int KB = pad8(NB - 1), MV = S::MV, KV = S::KV, MJ = S::MJ, KF = pad8(NQF), NT = MJ / 8, LDR = S::LDR;
    const int gid = lane >> 2, tq = lane & 3;
    const ElemGroup& grp = a.groups[gi];
    const int ne = grp.n;
    const int r0 = gid, r1 = gid + 8;
    const bool v0 = r0 < 5 * ne, v1 = r1 < 5 * ne;
    const bool need_u0 = a.mode != 0 && a.a0 != 0.0;
    if (lane == 0) {
        // the warp's reads of the previous group (generic proxy) are ordered before the copies'
        // writes (async proxy) by the __syncwarp that ended that group and this fence
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const unsigned per = 4u * G::FRB + G::UB + (need_u0 ? G::UB : 0u) + G::GEOB;
        mbar_arrive_expect_tx(&st.bar, per * (unsigned)ne);
        for (int el = 0; el < ne; ++el) {
            const int64_t e = grp.e[el];
            #pragma unroll
            for (int q = 0; q < 4; ++q)
                bulk_copy_g2s(st.face[el][q], a.dev + (int64_t)grp.face[el][q] * G::FR, G::FRB, &st.bar);
            bulk_copy_g2s(st.U[el], a.U + e * 5 * NB, G::UB, &st.bar);
            if (need_u0) bulk_copy_g2s(st.U0[el], a.U0 + e * 5 * NB, G::UB, &st.bar);
            bulk_copy_g2s(st.geo[el], a.geo + e * 10, G::GEOB, &st.bar);
        }
    }
    if (lane < ne) {
        const int e = grp.e[lane];
        sm.sE[lane] = e;
        const double dt = a.dt_inst ? __ldg(a.dt_inst + __ldg(a.elem_inst + e)) : a.dt;
        sm.sDT[lane] = dt * __ldg(a.inv_detj + e);
    }
    if (!mbar_wait_bounded(&st.bar, parity, kBulkSpinLimit)) {
        if (lane == 0 && a.err) atomicExch(a.err, DG_E_WATCHDOG);
        mbar_wait_bounded(&st.bar, parity, kBulkSpinLimit);  // copies in flight land before the warp leaves
        return false;
    }
    if (lane < 16) sm.sC0[lane] = lane < 5 * ne ? (float)st.U[lane / 5][lane % 5] : 0.f;
    if (a.volume && lane < 5 * ne) {  // row k of G(c_0) = detJ F(c_0) J^-T, FP64, one lane per (element, var)
        const int el = lane / 5, k = lane - 5 * el;
        const double* geo = st.geo[el];
        double c[5], J[9];
        #pragma unroll
        for (int i = 0; i < 5; ++i) c[i] = st.U[el][i];
        #pragma unroll
        for (int i = 0; i < 9; ++i) J[i] = geo[i];
        const double dj = geo[9];
        const double rho = c[0] > 1e-16 ? c[0] : 1e-16, ir = 1.0 / rho;
        const double u[3] = {c[1] * ir, c[2] * ir, c[3] * ir}, en = c[4] * ir;
        const double p = ((double)a.gamma - 1.0) * (rho * en - 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        double F[3];
        if (k == 0) {
            F[0] = rho * u[0]; F[1] = rho * u[1]; F[2] = rho * u[2];
        } else if (k < 4) {
            #pragma unroll
            for (int i = 0; i < 3; ++i) F[i] = rho * u[i] * u[k - 1] + (i == k - 1 ? p : 0.0);
        } else {
            #pragma unroll
            for (int i = 0; i < 3; ++i) F[i] = u[i] * (rho * en + p);
        }
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double gb = dj * (F[0] * J[d] + F[1] * J[3 + d] + F[2] * J[6 + d]);
            sm.sGb[el][3 * k + d] = gb;
            sm.sGbf[el][3 * k + d] = (float)gb;
        }
        if (k == 0) {
            #pragma unroll
            for (int i = 0; i < 9; ++i) sm.sJ[el][i] = (float)(dj * J[i]);
        }
    }
    __syncwarp();
    float acc[NT][4];
    #pragma unroll
    for (int nt = 0; nt < NT; ++nt)
        #pragma unroll
        for (int r = 0; r < 4; ++r) acc[nt][r] = 0.f;
    if (a.volume) {
        {   // values at the volume points
            AFrag<KB> A;
            load_afrag_state<KB, NB, true>(A, v0 ? st.U[r0 / 5] + r0 % 5 : nullptr,
                                           v1 ? st.U[r1 / 5] + r1 % 5 : nullptr, lane);
            const float c00 = sm.sC0[r0], c01 = sm.sC0[r1];
            #pragma unroll
            for (int nt = 0; nt < MV / 8; ++nt) {
                float o[4] = {0.f, 0.f, 0.f, 0.f};
                mma_bt<KB>(o, A, bt.tva, nt, lane);
                *reinterpret_cast<float2*>(&sm.sU[r0][nt * 8 + 2 * tq]) = make_float2(o[0] + c00, o[1] + c00);
                *reinterpret_cast<float2*>(&sm.sU[r1][nt * 8 + 2 * tq]) = make_float2(o[2] + c01, o[3] + c01);
            }
        }
        if constexpr (KV > 3 * NQV) {
            constexpr int w = KV - 3 * NQV;
            for (int i = lane; i < 15 * w; i += 32) sm.sG[i / w][3 * NQV + i % w] = 0.f;
        }
        __syncwarp();
        const float gm1 = a.gamma - 1.f;
        for (int p = lane; p < ne * NQV; p += 32) {
            const int el = p / NQV, g = p - el * NQV;
            float U[5], F[5][3];
            #pragma unroll
            for (int k = 0; k < 5; ++k) U[k] = sm.sU[el * 5 + k][g];
            flux_f32(U, gm1, F);
            const float* J = sm.sJ[el];
            #pragma unroll
            for (int k = 0; k < 5; ++k)
                #pragma unroll
                for (int d = 0; d < 3; ++d)
                    sm.sG[el * 5 + k][3 * g + d] =
                        fmaf(-F[k][0], J[d], fmaf(-F[k][1], J[3 + d], fmaf(-F[k][2], J[6 + d], sm.sGbf[el][3 * k + d])));
        }
        __syncwarp();
        #pragma unroll
        for (int t = 0; t < KTiles<KV>::N16; ++t) {
            const int c = t * 16 + 2 * tq;
            uint32_t h[4] = {0u, 0u, 0u, 0u}, l[4] = {0u, 0u, 0u, 0u};
            if (v0) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r0][c]);
                const float2 y = *reinterpret_cast<const float2*>(&sm.sG[r0][c + 8]);
                split2(x.x, x.y, h[0], l[0]);
                split2(y.x, y.y, h[2], l[2]);
            }
            if (v1) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r1][c]);
                const float2 y = *reinterpret_cast<const float2*>(&sm.sG[r1][c + 8]);
                split2(x.x, x.y, h[1], l[1]);
                split2(y.x, y.y, h[3], l[3]);
            }
            #pragma unroll
            for (int nt = 0; nt < NT; ++nt) mma3_tile(acc[nt], h, l, bt.tvp + nt * KTiles<KV>::NT_U32, t, lane);
        }
        if constexpr (KTiles<KV>::TAIL) {
            const int c = KTiles<KV>::N16 * 16 + 2 * tq;
            uint32_t h[2] = {0u, 0u}, l[2] = {0u, 0u};
            if (v0) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r0][c]);
                split2(x.x, x.y, h[0], l[0]);
            }
            if (v1) {
                const float2 x = *reinterpret_cast<const float2*>(&sm.sG[r1][c]);
                split2(x.x, x.y, h[1], l[1]);
            }
            #pragma unroll
            for (int nt = 0; nt < NT; ++nt) mma3_tail<KV>(acc[nt], h, l, bt.tvp + nt * KTiles<KV>::NT_U32, lane);
        }
    }
    // face integrals from the staged face records; side 1 negated exactly
    #pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int perm = grp.meta[q] & 0xff;
        const uint32_t flip = (grp.meta[q] >> 8) ? 0x80008000u : 0u;
        AFrag<KF> A;
        load_afrag_smem<KF>(A, v0 ? st.face[r0 / 5][q] + (r0 % 5) * KF : nullptr,
                            v1 ? st.face[r1 / 5][q] + (r1 % 5) * KF : nullptr, lane, flip);
        const uint32_t* tb = bt.tfl + perm * NT * KTiles<KF>::NT_U32;
        #pragma unroll
        for (int nt = 0; nt < NT; ++nt) mma_bt<KF>(acc[nt], A, tb, nt, lane);
    }
    __syncwarp();  // sG is free
    {
        double* sR = reinterpret_cast<double*>(&sm.sG[0][0]);
        const int mq = grp.meta[tq];
        const double sq = (mq >> 8) ? -1.0 : 1.0;
        double am[2][2], s0[2] = {0.0, 0.0};
        #pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int row = gid + 8 * mt, el = row / 5, k = row - 5 * el;
            const bool ok = row < 5 * ne;
            am[mt][0] = ok ? face_rec_fs<NQF>(st.face[el][tq])[k] : 0.0;
            am[mt][1] = (ok && a.volume && tq < 3) ? sm.sGb[el][3 * k + tq] : 0.0;
            if (ok && tq == 0) {
                #pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const double v = face_rec_fs<NQF>(st.face[el][q])[5 + k];
                    s0[mt] += (grp.meta[q] >> 8) ? -v : v;
                }
            }
        }
        #pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int jb = nt * 8 + gid;
            const double b0 = jb < NB ? sq * __ldg(a.t.mf + (mq & 0xff) * NB + jb) : 0.0;
            const double b1 = (jb < NB && tq < 3) ? -__ldg(a.t.mv + 3 * jb + tq) : 0.0;
            #pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                double d[2] = {(double)acc[nt][2 * mt], (double)acc[nt][2 * mt + 1]};
                dmma884(d, am[mt][0], b0);
                dmma884(d, am[mt][1], b1);
                const int row = gid + 8 * mt;
                if (nt == 0 && tq == 0) d[0] = s0[mt];
                *reinterpret_cast<double2*>(sR + row * LDR + nt * 8 + 2 * tq) = make_double2(d[0], d[1]);
            }
        }
    }
    __syncwarp();
    const double* sR = reinterpret_cast<const double*>(&sm.sG[0][0]);
    for (int i = lane; i < ne * 5 * NB; i += 32) {
        const int el = i / (5 * NB), r = i - el * (5 * NB);
        const int2 d = T.dof[r];
        const int64_t e = sm.sE[el];
        const int64_t idx = e * (5 * NB) + r;
        const double R = a.Rv ? sR[(el * 5 + d.y) * LDR + d.x] - a.Rv[idx] : sR[(el * 5 + d.y) * LDR + d.x];
        if (a.mode == 0) {
            a.out[idx] = R;
        } else {
            const double un = rk_update(need_u0, a.a0, need_u0 ? st.U0[el][r] : 0.0, a.a1, st.U[el][r],
                                        __dmul_rn(sm.sDT[el], T.inv_mass[d.x]), R);
            a.out[idx] = un;
        }
    }
    __syncwarp();
    return true;
}

template <int NB, int NQV, int NQF, int WARPS, int MINB>
__global__ void __launch_bounds__(WARPS * 32, MINB) element_mixed_staged(MixedElemArgs a) {
    using S = ElemMixedSmem<NB, NQV, NQF>;
    using G = ElemStage<NB, NQF>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ElemTables<NB> tabs;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    S& sm = reinterpret_cast<S*>(smem_raw)[warp];
    G& st = reinterpret_cast<G*>(smem_raw + sizeof(S) * WARPS)[warp];
    if (lane == 0) mbar_init(&st.bar, 1);
    element_tables_init(tabs, a.t.inv_mass);  // ends in __syncthreads: the barriers are initialised
    const ElemBTabs bt{a.t.tva, a.t.tvp, a.t.tfl};
    unsigned parity = 0;
    for (int gi = blockIdx.x * WARPS + warp; gi < a.ngroups; gi += gridDim.x * WARPS) {
        if (!element_group_staged<NB, NQV, NQF>(a, gi, sm, st, tabs, lane, bt, parity)) break;
        parity ^= 1u;
    }
}

template <int NB, int NQV, int NQF>
__host__ __device__ constexpr size_t elem_staged_warp_smem() {
    return sizeof(ElemMixedSmem<NB, NQV, NQF>) + sizeof(ElemStage<NB, NQF>);
}
// Warps per CTA of the staged kernel with `ctas` resident CTAs per SM: what fits in the SM's 228 KB
// (1 KB reserved per CTA, 3 KB for the static tables), at most 11 (one CTA) or 5 (two CTAs).
template <int NB, int NQV, int NQF>
__host__ __device__ constexpr int elem_staged_warps(int ctas) {
    const long long per_cta = 233472ll / ctas - 1024 - 3072;
    const long long w = per_cta / (long long)elem_staged_warp_smem<NB, NQV, NQF>();
    const int cap = ctas == 1 ? 11 : 5;
    return w > cap ? cap : (w < 1 ? 1 : (int)w);
}

// 8 warps: three CTAs per SM, at most 85 registers a thread (80 without spills; four CTAs at 64
// registers spill 20 bytes and measured 3 % slower with the batched update loads); 4 warps (P4):
// six CTAs, at most 85 registers
template <int NB, int NQV, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, WARPS == 8 ? 3 : 6) element_mixed(MixedElemArgs a) {
    using S = ElemMixedSmem<NB, NQV, NQF>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ElemTables<NB> tabs;
    element_tables_init(tabs, a.t.inv_mass);
    S& sm = reinterpret_cast<S*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const ElemBTabs bt{a.t.tva, a.t.tvp, a.t.tfl};
    for (int gi = blockIdx.x * WARPS + (threadIdx.x >> 5); gi < a.ngroups; gi += gridDim.x * WARPS)
        element_group_mixed<NB, NQV, NQF>(a, gi, sm, tabs, lane, bt);
}

// ------------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------------
struct MixedData {
    bool ready = false;
    int order = 0, qv = 0, qf = 0, nb = 0, nqv = 0, nqf = 0;
    int64_t ncell = 0, nface = 0;
    int nfgroups = 0, negroups = 0;
    int nfgroups_inner = 0;  // face groups [0, nfgroups_inner) touch no ghost element
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
    uint32_t* dev = nullptr;          // face records [nface][face_rec_words(nqf)]
    const double* dt_inst = nullptr;  // ensembles: per-instance dt (device), else null
    const int* elem_inst = nullptr;
    const double* Rv = nullptr;       // Navier-Stokes stepping: the stage input's viscous residual
    int* err = nullptr;               // device status word of the mixed kernels (bounded waits)
    // element kernel: 0 = loads phase by phase (8-warp CTAs, four per SM), 2 = each group's rows
    // staged by TMA bulk copies (P1..P3, 16-byte aligned state buffers); chosen by dg_autotune
    int elem_kernel = 0;
    int elem_ctas = 1;                // resident CTAs per SM of the staged kernel: 1 or 2
    // host copies the tile schedule of the persistent form is built from
    std::vector<FaceGroup> hfg;
    std::vector<ElemGroup> heg;
    std::vector<int> hface_cells;  // [nface][2]
};

// X(order, qv, qf, NB, NQV, NQF, W): W warps per block of the element kernel
#define FVEDG_MIXED_COMBOS(X)      \
    X(1, 0, 1, 4, 4, 6, 8)         \
    X(1, 0, 0, 4, 4, 4, 8)         \
    X(1, 0, 2, 4, 4, 7, 8)         \
    X(1, 2, 2, 4, 15, 7, 8)        \
    X(2, 1, 2, 10, 11, 7, 8)       \
    X(2, 1, 3, 10, 11, 24, 8)      \
    X(2, 2, 3, 10, 15, 24, 8)      \
    X(3, 3, 3, 20, 23, 24, 8)      \
    X(3, 4, 3, 20, 31, 24, 8)      \
    X(4, 5, 3, 35, 44, 24, 4)      \
    X(4, 6, 3, 35, 57, 24, 4)

inline bool mixed_supported(int order, int qv, int qf) {
#define X(P, QV, QF, NB, NQV, NQF, W) \
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

// B operand of one contraction in fragment order. T is N x K row-major (N, K multiples of 8). Per
// n-tile: for each full K tile, 32 lanes x {hi(c,c+1), hi(c+8,c+9), lo(c,c+1), lo(c+8,c+9)} of
// row n = 8 nt + lane / 4, c = 16 t + 2 (lane % 4); then the tail, 32 lanes x {hi(c,c+1), lo(c,c+1)}.
inline void append_frag_table(const std::vector<double>& T, int N, int K, std::vector<uint32_t>& out) {
    const int n16 = K / 16;
    const bool tail = (K % 16) != 0;
    auto half = [&](int n, int k, bool lo) -> uint32_t {
        const float f = (float)T[(size_t)n * K + k];
        const __nv_bfloat16 h = __float2bfloat16_rn(f);
        return (uint32_t)__bfloat16_as_ushort(lo ? __float2bfloat16_rn(f - __bfloat162float(h)) : h);
    };
    auto word = [&](int n, int c, bool lo) { return half(n, c, lo) | (half(n, c + 1, lo) << 16); };
    for (int nt = 0; nt < N / 8; ++nt) {
        for (int t = 0; t < n16; ++t)
            for (int lane = 0; lane < 32; ++lane) {
                const int n = nt * 8 + lane / 4, c = t * 16 + 2 * (lane % 4);
                out.push_back(word(n, c, false));
                out.push_back(word(n, c + 8, false));
                out.push_back(word(n, c, true));
                out.push_back(word(n, c + 8, true));
            }
        if (tail)
            for (int lane = 0; lane < 32; ++lane) {
                const int n = nt * 8 + lane / 4, c = n16 * 16 + 2 * (lane % 4);
                out.push_back(word(n, c, false));
                out.push_back(word(n, c, true));
            }
    }
}

// Faces with equal (perm0, perm1, kind) and elements with equal face maps (in canonical face
// order: local face q is the one opposite local vertex q) are grouped in threes, in mesh order.
// A partial group repeats its first member in the unused slots (never read as a row: rows of
// unused slots are masked by the group size).
// Face groups: faces of the same kind in threes, first the faces between owned elements, then
// (from *nf_inner on) the faces touching a ghost element (cells >= ncell), whose fluxes need the
// ghost rows of a halo exchange. Element groups: the owned elements [0, ncell).
inline void build_groups(const std::vector<FaceInfo>& hfi, const std::vector<ElemFace>& hef, int64_t ncell,
                         std::vector<FaceGroup>& fg, std::vector<ElemGroup>& eg, int* nf_inner) {
    for (int halo = 0; halo < 2; ++halo) {
        std::map<int64_t, FaceGroup> open_f;
        for (int64_t f = 0; f < (int64_t)hfi.size(); ++f) {
            const FaceInfo& F = hfi[f];
            if ((F.c0 >= ncell || F.c1 >= ncell) != (halo == 1)) continue;
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
        if (halo == 0) *nf_inner = (int)fg.size();
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
                      int64_t nowned, int64_t nface, double gamma, int flux, int qv, int qf, const double* d_geo,
                      const FaceInfo* d_fi, const ElemFace*, const double*) {
    if (!mixed_supported(tab.order, qv, qf)) return DG_E_ARG;
    const int NB = tab.nb, NQV = tab.nqv, NQF = tab.nqf;
    const int KB = pad8(NB - 1), MF = pad8(NQF), MV = pad8(NQV), MJ = pad8(NB), KV = pad8(3 * NQV), KF = pad8(NQF);
    m.order = tab.order; m.qv = qv; m.qf = qf; m.nb = NB; m.nqv = NQV; m.nqf = NQF;
    m.ncell = ncell; m.nface = nface; m.gamma = (float)gamma; m.flux = flux;
    std::vector<double> tva(MV * KB, 0.0), tvp(MJ * KV, 0.0);
    std::vector<double> mv(NB * 3, 0.0), mf(24 * NB, 0.0), inv_mass(NB, 0.0), inv_detj(ncell, 0.0);
    std::vector<uint32_t> ftfa, ftva, ftvp, ftfl;
    for (int p = 0; p < 24; ++p) {
        std::vector<double> tfa(MF * KB, 0.0), tfl(MJ * KF, 0.0);
        for (int g = 0; g < NQF; ++g)
            for (int b = 1; b < NB; ++b) tfa[g * KB + (b - 1)] = tab.phi_f[((size_t)p * NQF + g) * NB + b];
        for (int j = 0; j < NB; ++j)
            for (int g = 0; g < NQF; ++g) {
                const double v = tab.w_f[g] * tab.phi_f[((size_t)p * NQF + g) * NB + j];
                tfl[j * KF + g] = v;
                mf[p * NB + j] += v;
            }
        append_frag_table(tfa, MF, KB, ftfa);
        append_frag_table(tfl, MJ, KF, ftfl);
    }
    for (int g = 0; g < NQV; ++g)
        for (int b = 1; b < NB; ++b) tva[g * KB + (b - 1)] = tab.phi_v[g * NB + b];
    for (int j = 0; j < NB; ++j)
        for (int g = 0; g < NQV; ++g)
            for (int d = 0; d < 3; ++d) {
                const double v = tab.dphi_vw[(g * NB + j) * 3 + d];
                tvp[j * KV + 3 * g + d] = v;
                mv[j * 3 + d] += v;
            }
    append_frag_table(tva, MV, KB, ftva);
    append_frag_table(tvp, MJ, KV, ftvp);
    for (int j = 0; j < NB; ++j) inv_mass[j] = 1.0 / tab.mass_ref[j];
    for (int64_t e = 0; e < ncell; ++e) inv_detj[e] = 1.0 / hgeo[10 * e + 9];
    double wsum = 0.0;
    for (int g = 0; g < NQF; ++g) wsum += tab.w_f[g];
    m.t.wsum = wsum;
    int rc;
    if ((rc = mixed_upload(m, &m.t.tfa, ftfa)) || (rc = mixed_upload(m, &m.t.tva, ftva)) ||
        (rc = mixed_upload(m, &m.t.tvp, ftvp)) || (rc = mixed_upload(m, &m.t.tfl, ftfl)))
        return rc;
    if ((rc = mixed_upload(m, &m.t.mv, mv)) || (rc = mixed_upload(m, &m.t.mf, mf)) ||
        (rc = mixed_upload(m, &m.t.inv_mass, inv_mass)) ||
        (rc = mixed_upload(m, &m.t.wf32, std::vector<float>(tab.w_f.begin(), tab.w_f.end()))) ||
        (rc = mixed_upload(m, &m.inv_detj, inv_detj)))
        return rc;
    std::vector<FaceGroup> fg;
    std::vector<ElemGroup> eg;
    build_groups(hfi, hef, nowned, fg, eg, &m.nfgroups_inner);  // element groups: owned cells only
    m.nfgroups = (int)fg.size();
    m.negroups = (int)eg.size();
    if ((rc = mixed_upload(m, &m.fgroups, fg)) || (rc = mixed_upload(m, &m.egroups, eg))) return rc;
    m.hfg = fg;
    m.heg = eg;
    m.hface_cells.resize(2 * hfi.size());
    for (size_t f = 0; f < hfi.size(); ++f) {
        m.hface_cells[2 * f] = hfi[f].c0;
        m.hface_cells[2 * f + 1] = hfi[f].c1;
    }
    // padding columns of the A rows stay zero: allocation clears them and no kernel writes them
    if ((rc = mixed_alloc(m, &m.dev, (size_t)nface * face_rec_words(NQF)))) return rc;
    if ((rc = mixed_alloc(m, &m.err, 1))) return rc;
    m.fi = d_fi; m.geo = d_geo;
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

inline MixedFaceArgs face_args(const MixedData& m, const double* U, int face_mask, int g0 = 0, int g1 = -1) {
    MixedFaceArgs fa;
    fa.U = U; fa.fi = m.fi; fa.groups = m.fgroups; fa.UD = m.UD; fa.dev = m.dev;
    fa.t = m.t; fa.ngroups = m.nfgroups; fa.gamma = m.gamma; fa.flux = m.flux;
    if (g1 >= 0) {  // face groups [g0, g1) only
        fa.groups = m.fgroups + g0;
        fa.ngroups = g1 - g0;
    }
    fa.faces_mask = face_mask;
    return fa;
}

inline MixedElemArgs elem_args(const MixedData& m, const double* U, const double* U0, double* out, int mode,
                               double dt, double a0, double a1, int with_volume) {
    MixedElemArgs ea;
    ea.U = U; ea.U0 = U0; ea.out = out;
    ea.dev = m.dev; ea.geo = m.geo; ea.inv_detj = m.inv_detj; ea.groups = m.egroups;
    ea.t = m.t; ea.ngroups = m.negroups; ea.gamma = m.gamma; ea.volume = with_volume;
    ea.dt = dt; ea.a0 = a0; ea.a1 = a1; ea.mode = mode;
    ea.dt_inst = mode == 1 ? m.dt_inst : nullptr; ea.elem_inst = m.elem_inst;
    ea.Rv = mode == 1 ? m.Rv : nullptr;
    ea.err = m.err;
    return ea;
}

// Opt a kernel into `smem` bytes of dynamic shared memory once per device.
template <class Kernel>
inline int ensure_smem(Kernel k, size_t smem, unsigned long long& done_mask) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DG_E_CUDA;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done_mask & bit) return DG_OK;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return DG_E_CUDA;
    done_mask |= bit;
    return DG_OK;
}

// which: 0 = face fluxes, 1 = element kernel (volume + face integrals + update).
template <int NB, int NQV, int NQF, int WE>
inline int mixed_launch(MixedData& m, int which, const double* U, const double* U0, double* out, int mode,
                        double dt, double a0, double a1, int face_mask, int with_volume, cudaStream_t s, int g0,
                        int g1) {
    if (which == 0) {
        constexpr int W = 4;  // 4-warp CTAs: finer-grained scheduling than 8 at the same occupancy
        const int n = g1 < 0 ? m.nfgroups : g1 - g0;
        const int g = (int)std::min<int64_t>((n + W - 1) / W, (int64_t)m.sms * 64);
        face_flux_mixed<NB, NQF, W><<<g, W * 32, 0, s>>>(face_args(m, U, face_mask, g0, g1));
    } else if (m.elem_kernel == 2 && (5 * NB * 8) % 16 == 0 && ((uintptr_t)U & 15) == 0 &&
               ((uintptr_t)U0 & 15) == 0) {
        if constexpr ((5 * NB * 8) % 16 == 0) {
            const auto ea = elem_args(m, U, U0, out, mode, dt, a0, a1, with_volume);
            if (m.elem_ctas == 2) {
                constexpr int W = elem_staged_warps<NB, NQV, NQF>(2);
                constexpr size_t smem = elem_staged_warp_smem<NB, NQV, NQF>() * W;
                static unsigned long long done = 0;
                int rc = ensure_smem(element_mixed_staged<NB, NQV, NQF, W, 2>, smem, done);
                if (rc) return rc;
                const int g = (int)std::min<int64_t>((m.negroups + W - 1) / W, (int64_t)m.sms * 2);
                element_mixed_staged<NB, NQV, NQF, W, 2><<<g, W * 32, smem, s>>>(ea);
            } else {
                constexpr int W = elem_staged_warps<NB, NQV, NQF>(1);
                constexpr size_t smem = elem_staged_warp_smem<NB, NQV, NQF>() * W;
                static unsigned long long done = 0;
                int rc = ensure_smem(element_mixed_staged<NB, NQV, NQF, W, 1>, smem, done);
                if (rc) return rc;
                const int g = (int)std::min<int64_t>((m.negroups + W - 1) / W, (int64_t)m.sms);
                element_mixed_staged<NB, NQV, NQF, W, 1><<<g, W * 32, smem, s>>>(ea);
            }
        }
    } else {
        constexpr size_t smem = sizeof(ElemMixedSmem<NB, NQV, NQF>) * WE;
        static unsigned long long done = 0;
        int rc = ensure_smem(element_mixed<NB, NQV, NQF, WE>, smem, done);
        if (rc) return rc;
        const int g = (int)std::min<int64_t>((m.negroups + WE - 1) / WE, (int64_t)m.sms * 32);
        element_mixed<NB, NQV, NQF, WE><<<g, WE * 32, smem, s>>>(
            elem_args(m, U, U0, out, mode, dt, a0, a1, with_volume));
    }
    return cuda_status(cudaGetLastError());
}

// Element-kernel shapes of the two-launch schedule that dg_autotune times: the kernel (0: loads
// phase by phase, 2: rows staged by bulk copies), warps per CTA (three elements each) and resident
// CTAs per SM. Returns how many apply to this order and rule pair.
struct ElemShape {
    int kernel, warps, ctas;
};
inline int mixed_elem_shapes(const MixedData& m, ElemShape out[3]) {
#define X(P, QV, QF, NB, NQV, NQF, W)                                                 \
    if (m.order == P && m.qv == QV && m.qf == QF) {                                   \
        int n = 0;                                                                    \
        out[n++] = ElemShape{0, W, W == 8 ? 3 : 6};                                   \
        if ((5 * NB * 8) % 16 == 0) {                                                 \
            out[n++] = ElemShape{2, elem_staged_warps<NB, NQV, NQF>(1), 1};           \
            out[n++] = ElemShape{2, elem_staged_warps<NB, NQV, NQF>(2), 2};           \
        }                                                                             \
        return n;                                                                     \
    }
    FVEDG_MIXED_COMBOS(X)
#undef X
    return 0;
}

// Face launches (which 0) cover face groups [g0, g1) (g1 < 0: all of them).
inline int mixed_kernel(MixedData& m, int which, const double* U, const double* U0, double* out, int mode,
                        double dt, double a0, double a1, int face_mask, int with_volume, cudaStream_t s,
                        std::atomic<int64_t>* launches, int g0 = 0, int g1 = -1) {
    if (!m.ready) return DG_E_ARG;
    if (which == 0 && g1 >= 0 && g1 <= g0) return DG_OK;  // an empty range: nothing to launch
    ++*launches;
#define X(P, QV, QF, NB, NQV, NQF, W)                                                                           \
    if (m.order == P && m.qv == QV && m.qf == QF)                                                               \
        return mixed_launch<NB, NQV, NQF, W>(m, which, U, U0, out, mode, dt, a0, a1, face_mask, with_volume, s, \
                                             g0, g1);
    FVEDG_MIXED_COMBOS(X)
#undef X
    return DG_E_ARG;
}

// One stage: face fluxes, then the element kernel.
template <class Timed>
inline int mixed_stage(MixedData& m, const double* U, const double* U0, double* out, int mode, double dt, double a0,
                       double a1, int face_mask, int with_volume, cudaStream_t s, std::atomic<int64_t>* launches,
                       Timed&& timed) {
    auto K = [&](int which) {
        return mixed_kernel(m, which, U, U0, out, mode, dt, a0, a1, face_mask, with_volume, s, launches);
    };
    const int rc = timed(0, [&] { return K(0); });
    if (rc) return rc;
    return timed(1, [&] { return K(1); });
}

inline int residual_mixed(MixedData& m, const double* U, double* R, int part, cudaStream_t s,
                          std::atomic<int64_t>* launches) {
    const int mask = part == 0 ? 3 : part == 1 ? 0 : part == 2 ? 1 : 2;
    return mixed_stage(m, U, U, R, 0, 0.0, 0.0, 0.0, mask, part == 0 || part == 1, s, launches,
                       [](int, auto&& fn) { return fn(); });
}

inline int mixed_launches_per_step(const MixedData&) { return 6; }

// SSP-RK3 step; `timed(cls, fn)` runs fn (one launch) and may bracket it with timing events.
// `post(in, out, st)` runs after every stage st (the limiter, or nothing). Stages st0..st1-1 only
// (one stage at a time when a halo exchange runs between stages).
template <class Timed, class Post>
inline int step_mixed(MixedData& m, double* Un, double* Ua, double* Ub, double dt, cudaStream_t s,
                      std::atomic<int64_t>* launches, Timed&& timed, Post&& post, int st0 = 0, int st1 = 3) {
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {Un, Ua, Ub};
    double* out[3] = {Ua, Ub, Un};
    for (int st = st0; st < st1; ++st) {
        int rc = mixed_stage(m, in[st], Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, launches, timed);
        if (rc || (rc = post(in[st], out[st], st))) return rc;
    }
    return DG_OK;
}

}  // namespace fvedg
