// Explicit viscous operator, after ExplicitDiffusion<Order, QuadC, QuadF>::eval
// (include/DG/DG_Schemes/ExplicitDiffusion.h:133-626): an interior-penalty discretisation of the
// Navier-Stokes viscous terms in homogeneity-tensor form G_m = sum_n K_mn(U) dU/dx_n, with
// K_mn = dG_m / d(dU/dx_n) for G_m = (0, tau_{.m}, u . tau_{.m} - q_m), tau the Stokes stress with
// viscosity mu, q = -mu gamma/Pr grad(e - |u|^2/2) (the reference's ExplicitDiffusion.h:28-66,
// with its fixed mu = 1, Pr = 1 made parameters). FP64.
//
// The terms and their pairing follow the reference exactly (ExplicitDiffusion.h:158-612):
//   volume     R_j -= sum_g w_g detJ sum_{m,n} (grad phi_j)_n K_mn(U) (dU/dx_m)
//   face       F = 1/2 sum_{m,n} n_n K_mn (grad U_L + grad U_R)_m - beta sum_{m,n} n_m n_n K_mn (U_L - U_R),
//              K at (U_L + U_R)/2, beta = (P+1)^2 / h(cells[0]), h = volume / sum of face areas;
//              R_L[j] += phi_j^L F 2A w_g, R_R[j] -= phi_j^R F 2A w_g
//   symmetric  S_j = 1/2 sum_{m,n} n_n K_mn[:, 4] ((grad phi_j^L)_m + (grad phi_j^R)_m) (U_R - U_L)_4,
//              added to L and subtracted from R (the reference keeps only the energy column of
//              K (U_R - U_L), ExplicitDiffusion.h:588-593; since K_mn[:, 4] is zero outside the
//              energy row, S_j is 1/2 mu gamma/Pr / rho (U_R - U_L)_4 n . (grad phi_j^L + grad phi_j^R)
//              in the energy equation only)
//   boundary   Dirichlet: ghost 2 U_D - U, K at (U + ghost)/2, F from the inner gradient without the
//              1/2 and the penalty on the inner values only, S_j with (ghost - U)_4 and the inner
//              gradient; Pseudo3DZ: ghost (1, 1, 1, -1, 1) U, otherwise the same; other types
//              contribute nothing.
// Every contraction of K with a 5 x 3 input X (a gradient, or a state times the normal) reduces to
// the velocity-like rows Y_a,m = (X_{a+1,m} - u_a X_{0,m}) / rho and Ye_m = (X_{4,m} - e X_{0,m}) / rho:
//   H_n[1+a] = sum_m sum_b K_mn[1+a, b] X_{b,m} = mu (Y_a,n + delta_an tr Y - 2/3 Y_n,a)
//   H_n[4]   = sum_a u_a H_n[1+a] + mu gamma/Pr (Ye_n - sum_k u_k Y_k,n),   H_n[0] = 0
// with u = U_1..3 / U_0, e = U_4 / U_0 and rho = max(U_0, 1e-8), as ExplicitDiffusion.h:28-31,69-73.
//
// Two launches, FP64:
//   viscous_face     one warp per face: both traces (values and reference gradients at the face
//                    points, on the FP64 tensor cores: points x variables over modes) once per face;
//                    then lanes over the points: the averaged flux with its penalty (stored per point
//                    as Fl w 2A); then the energy-only symmetric term per mode,
//                    T_j = sum_g sfac_g w_g 2A n . (grad phi_j^L + grad phi_j^R), written as
//                    (J_L^T n) . dphi^L + (J_R^T n) . dphi^R (the same for both sides, up to sign).
//   viscous_element  one warp per element: the volume term (lanes over the volume points: J^T H w detJ
//                    per point), then the contractions on the FP64 tensor cores (mma m8n8k4, modes x
//                    variables): the volume term with the reference gradients over (point, direction),
//                    and each of the four faces' fluxes with its side's basis values over the face
//                    points; plus T_j in the energy column. Each element writes its own residual: no
//                    atomics, a deterministic result.
#pragma once
#include "dg_kernels_fp64.cuh"
#include "dg_status.cuh"

namespace fvedg {

struct ViscArgs {
    const double* U;
    double* R;
    const double* geo;      // [ncell][10]: J^-T row-major, detJ
    const double* h;        // [ncell] volume / sum of face areas
    const FaceInfo* fi;
    const ElemFace* ef;     // [ncell][4]
    const double* phi_v;    // [nqv][nb]
    const double* dphi_v;   // [nqv][nb][3]
    const double* w_v;      // [nqv]
    const double* phi_f;    // [24][nqf][nb]
    const double* dphi_f;   // [24][nqf][nb][3]
    const double* w_f;      // [nqf]
    const double* UD;       // [nface][nqf][5] Dirichlet data, or null
    const double* phiT_v;   // [nb][nqv] the volume tables transposed (lanes over points read rows)
    const double* dphiT_v;  // [nb][3][nqv]
    const double* Pt;       // [24][4][gp][kpb] A of the face traces: phi_f, then dphi_f[.][.][.][d], zero-padded
    const double* Av;       // [kpv][mp] A of the volume contraction: dphi_v[k/3][j][k%3], zero-padded
    const double* Pf;       // [24][kpf][mp] A of the face contraction: phi_f[p][g][j], zero-padded
    double* vf;             // [nface][5 nqf + nb] per face: Fl w 2A [5][nqf], then T_j [nb]
    int64_t ncell, nface;
    int nqv, nqf, order, kpv, kpf, mp, gp, kpb;
    double mu, cq;          // viscosity and gamma / Pr
};

constexpr int kViscWarps = 4;
constexpr int kViscMaxQv = 64;  // volume points an element warp stages (the largest rule has 57)
constexpr int kViscMaxQf = 32;  // face points, one per lane (the largest rule has 24)
constexpr int kViscMaxGp = 24;  // face points padded to the 8-row tiles of the trace products

inline int visc_mp(int nb) { return 8 * ((nb + 7) / 8); }  // modes padded to the 8-row tiles
inline int visc_kp(int k) { return 4 * ((k + 3) / 4); }     // contraction length padded to 4
inline int visc_gp(int nqf) { return 8 * ((nqf + 7) / 8); }  // face points padded to 8

// d (one 8 x 8 FP64 tile of D, two entries per lane) += A (8 x 4) B (4 x 8); lane l holds
// A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2 (l % 4) + {0, 1}].
__device__ __forceinline__ void visc_dmma(double d[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

struct ViscState {  // what K needs of the state it is taken at
    double u[3], e, irho;
};

__device__ __forceinline__ ViscState visc_state(const double U[5]) {
    ViscState s;
    const double inv = 1.0 / U[0];  // one division: the quotients below to within an ulp
    s.irho = U[0] > 1e-8 ? inv : 1e8;
    s.u[0] = U[1] * inv;
    s.u[1] = U[2] * inv;
    s.u[2] = U[3] * inv;
    s.e = U[4] * inv;
    return s;
}

// out[i] = sum_n d_n H_n[i] for X given as X[b][m] (b = variable, m = direction)
__device__ __forceinline__ void visc_contract(const ViscState& s, double mu, double cq, const double X[5][3],
                                              const double d[3], double out[5]) {
    double Y[3][3], Ye[3];
    #pragma unroll
    for (int m = 0; m < 3; ++m) {
        #pragma unroll
        for (int a = 0; a < 3; ++a) Y[a][m] = (X[a + 1][m] - s.u[a] * X[0][m]) * s.irho;
        Ye[m] = (X[4][m] - s.e * X[0][m]) * s.irho;
    }
    const double tr = Y[0][0] + Y[1][1] + Y[2][2];
    out[0] = 0.0;
    double o4 = 0.0;
    #pragma unroll
    for (int a = 0; a < 3; ++a) {
        double v = 0.0;
        #pragma unroll
        for (int n = 0; n < 3; ++n) v += d[n] * mu * (Y[a][n] + (a == n ? tr : 0.0) - (2.0 / 3.0) * Y[n][a]);
        out[1 + a] = v;
        o4 += s.u[a] * v;
    }
    #pragma unroll
    for (int n = 0; n < 3; ++n)
        o4 += d[n] * mu * cq * (Ye[n] - (s.u[0] * Y[0][n] + s.u[1] * Y[1][n] + s.u[2] * Y[2][n]));
    out[4] = o4;
}

// Value and physical gradient of the state at point g from transposed tables (phiT [nb][nq],
// dphiT [nb][3][nq]): Uv[k], G[k][m] = sum_d J[m][d] (sum_b c_bk dphi_bd).
template <int NB>
__device__ __forceinline__ void visc_trace_t(const double* c, const double* __restrict__ phiT,
                                             const double* __restrict__ dphiT, int nq, int g, const double J[9],
                                             double Uv[5], double G[5][3]) {
    double R[5][3];
    #pragma unroll
    for (int k = 0; k < 5; ++k) { Uv[k] = 0.0; R[k][0] = R[k][1] = R[k][2] = 0.0; }
    #pragma unroll 2
    for (int b = 0; b < NB; ++b) {
        const double p = phiT[b * nq + g];
        const double d0 = dphiT[(3 * b) * nq + g], d1 = dphiT[(3 * b + 1) * nq + g], d2 = dphiT[(3 * b + 2) * nq + g];
        #pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double cb = c[5 * b + k];
            Uv[k] = fma(p, cb, Uv[k]);
            R[k][0] = fma(d0, cb, R[k][0]);
            R[k][1] = fma(d1, cb, R[k][1]);
            R[k][2] = fma(d2, cb, R[k][2]);
        }
    }
    #pragma unroll
    for (int k = 0; k < 5; ++k)
        #pragma unroll
        for (int m = 0; m < 3; ++m) G[k][m] = J[3 * m] * R[k][0] + J[3 * m + 1] * R[k][1] + J[3 * m + 2] * R[k][2];
}

// One side's traces at the face points on the tensor cores: sd[t][g][i] = sum_b pt[t][g][b] c[b][i]
// for t = 0 (values) and t = 1..3 (reference gradient components), g < gp, i < 5.
template <int NB>
__device__ __forceinline__ void visc_face_traces(const double* c, const double* __restrict__ pt, int gp, int kpb,
                                                 double* sd, int lane) {
    constexpr int KT = (NB + 3) / 4, MTMAX = kViscMaxGp / 8;
    const int gid = lane >> 2, tq = lane & 3, mtn = gp / 8;
    double d[4][MTMAX][2];
    #pragma unroll
    for (int t = 0; t < 4; ++t)
        #pragma unroll
        for (int mt = 0; mt < MTMAX; ++mt) d[t][mt][0] = d[t][mt][1] = 0.0;
    #pragma unroll
    for (int kt = 0; kt < KT; ++kt) {
        const int b = kt * 4 + tq;
        const double bv = (gid < 5 && b < NB) ? c[5 * b + gid] : 0.0;
        #pragma unroll
        for (int t = 0; t < 4; ++t)
            #pragma unroll
            for (int mt = 0; mt < MTMAX; ++mt)
                if (mt < mtn) visc_dmma(d[t][mt], pt[((t * gp) + mt * 8 + gid) * kpb + b], bv);
    }
    const int i0 = 2 * tq;
    #pragma unroll
    for (int t = 0; t < 4; ++t)
        #pragma unroll
        for (int mt = 0; mt < MTMAX; ++mt)
            if (mt < mtn) {
                double* row = sd + ((t * gp) + mt * 8 + gid) * 5;
                if (i0 < 5) row[i0] = d[t][mt][0];
                if (i0 + 1 < 5) row[i0 + 1] = d[t][mt][1];
            }
}

// A point's value and physical gradient from traces staged by visc_face_traces.
__device__ __forceinline__ void visc_trace_smem(const double* sd, int gp, int g, const double J[9], double Uv[5],
                                                double G[5][3]) {
    #pragma unroll
    for (int k = 0; k < 5; ++k) {
        Uv[k] = sd[g * 5 + k];
        const double r0 = sd[(gp + g) * 5 + k], r1 = sd[(2 * gp + g) * 5 + k], r2 = sd[(3 * gp + g) * 5 + k];
        #pragma unroll
        for (int m = 0; m < 3; ++m) G[k][m] = J[3 * m] * r0 + J[3 * m + 1] * r1 + J[3 * m + 2] * r2;
    }
}

// Faces whose viscous terms act: interior, Dirichlet with data, Pseudo3DZ (ExplicitDiffusion.h:380-612).
__device__ __forceinline__ bool visc_face_active(const FaceInfo& F, const double* UD) {
    const int bc = (F.meta >> 16) & 0xff;
    return F.c1 >= 0 || bc == 5 || (bc == 0 && UD != nullptr);
}

template <int NB>
__global__ void __launch_bounds__(kViscWarps * 32, 4) viscous_face(ViscArgs a) {
    __shared__ double sc[kViscWarps][2][5 * NB];
    __shared__ double ssf[kViscWarps][kViscMaxQf];  // sfac w 2A per face point
    __shared__ double str[kViscWarps][2][4 * kViscMaxGp * 5];  // traces per side: [t][g][i]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* cL = sc[w][0];
    double* cR = sc[w][1];
    double* ss = ssf[w];
    const int nqf = a.nqf, bs = 5 * nqf + NB, gp = a.gp, kpb = a.kpb;
    const double beta_base = (double)((a.order + 1) * (a.order + 1));
    for (int64_t f = (int64_t)blockIdx.x * kViscWarps + w; f < a.nface; f += (int64_t)gridDim.x * kViscWarps) {
        const FaceInfo F = a.fi[f];
        {   // the next face's state rows into L2 while this face is computed
            constexpr int NL = (5 * NB * 8 + 127) / 128;
            const int64_t fn = f + (int64_t)gridDim.x * kViscWarps;
            if (fn < a.nface && lane < 2 * NL) {
                const int side = lane / NL, part = lane - side * NL;
                const int64_t cn = side ? a.fi[fn].c1 : a.fi[fn].c0;
                if (cn >= 0)
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(
                        reinterpret_cast<const char*>(a.U + cn * (5 * NB)) + part * 128));
            }
        }
        if (!visc_face_active(F, a.UD)) continue;  // warp-uniform
        const bool interior = F.c1 >= 0;
        const int bc = (F.meta >> 16) & 0xff;
        const double* gL = a.U + (int64_t)F.c0 * (5 * NB);
        for (int i = lane; i < 5 * NB; i += 32) cL[i] = gL[i];
        if (interior) {
            const double* gR = a.U + (int64_t)F.c1 * (5 * NB);
            for (int i = lane; i < 5 * NB; i += 32) cR[i] = gR[i];
        }
        __syncwarp();
        {
            const int pL0 = F.meta & 0xff, pR0 = (F.meta >> 8) & 0xff;
            visc_face_traces<NB>(cL, a.Pt + (int64_t)pL0 * 4 * gp * kpb, gp, kpb, str[w][0], lane);
            if (interior) visc_face_traces<NB>(cR, a.Pt + (int64_t)pR0 * 4 * gp * kpb, gp, kpb, str[w][1], lane);
        }
        __syncwarp();
        if (lane < nqf) {
            const int g = lane;
            const double n[3] = {F.n[0], F.n[1], F.n[2]};
            double J[9];
            #pragma unroll
            for (int i = 0; i < 9; ++i) J[i] = a.geo[(int64_t)F.c0 * 10 + i];
            double UL[5], UR[5], X[5][3];
            visc_trace_smem(str[w][0], gp, g, J, UL, X);
            if (interior) {
                #pragma unroll
                for (int i = 0; i < 9; ++i) J[i] = a.geo[(int64_t)F.c1 * 10 + i];
                double GR[5][3];
                visc_trace_smem(str[w][1], gp, g, J, UR, GR);
                #pragma unroll
                for (int k = 0; k < 5; ++k)
                    #pragma unroll
                    for (int m = 0; m < 3; ++m) X[k][m] = 0.5 * (X[k][m] + GR[k][m]);
            } else if (bc == 0) {
                const double* ud = a.UD + (f * nqf + g) * 5;
                #pragma unroll
                for (int k = 0; k < 5; ++k) UR[k] = ud[k] + (ud[k] - UL[k]);  // ghost 2 U_D - U
            } else {
                #pragma unroll
                for (int k = 0; k < 5; ++k) UR[k] = UL[k];
                UR[3] = -UL[3];
            }
            double Um[5];
            #pragma unroll
            for (int k = 0; k < 5; ++k) Um[k] = 0.5 * (UL[k] + UR[k]);
            const ViscState st = visc_state(Um);
            double Fa[5], Fb[5];
            visc_contract(st, a.mu, a.cq, X, n, Fa);  // averaged (boundary: inner) gradient flux
            #pragma unroll
            for (int k = 0; k < 5; ++k) {
                const double dU = interior ? UL[k] - UR[k] : UL[k];
                #pragma unroll
                for (int m = 0; m < 3; ++m) X[k][m] = dU * n[m];
            }
            visc_contract(st, a.mu, a.cq, X, n, Fb);  // penalty
            const double beta = beta_base / a.h[F.c0];
            const double jw = a.w_f[g] * F.jw;
            double* out = a.vf + f * bs;
            #pragma unroll
            for (int k = 0; k < 5; ++k) out[k * nqf + g] = (Fa[k] - beta * Fb[k]) * jw;
            ss[g] = (interior ? 0.5 : 1.0) * a.mu * a.cq * st.irho * (UR[4] - UL[4]) * jw;
        }
        __syncwarp();
        // symmetric term per mode: T_j = sum_g ss_g ((J_L^T n) . dphi_j^L(g) + (J_R^T n) . dphi_j^R(g))
        double nL[3], nR[3] = {0.0, 0.0, 0.0};
        {
            const double* JL = a.geo + (int64_t)F.c0 * 10;
            #pragma unroll
            for (int d = 0; d < 3; ++d) nL[d] = JL[d] * F.n[0] + JL[3 + d] * F.n[1] + JL[6 + d] * F.n[2];
            if (interior) {
                const double* JR = a.geo + (int64_t)F.c1 * 10;
                #pragma unroll
                for (int d = 0; d < 3; ++d) nR[d] = JR[d] * F.n[0] + JR[3 + d] * F.n[1] + JR[6 + d] * F.n[2];
            }
        }
        const int pL = F.meta & 0xff, pR = (F.meta >> 8) & 0xff;
        for (int j = lane; j < NB; j += 32) {
            double t = 0.0;
            for (int g = 0; g < nqf; ++g) {
                const double* dl = a.dphi_f + (((int64_t)pL * nqf + g) * NB + j) * 3;
                double sj = nL[0] * dl[0] + nL[1] * dl[1] + nL[2] * dl[2];
                if (interior) {
                    const double* dr = a.dphi_f + (((int64_t)pR * nqf + g) * NB + j) * 3;
                    sj += nR[0] * dr[0] + nR[1] * dr[1] + nR[2] * dr[2];
                }
                t = fma(ss[g], sj, t);
            }
            a.vf[f * bs + 5 * nqf + j] = t;
        }
        __syncwarp();
    }
}

template <int NB>
__global__ void __launch_bounds__(kViscWarps * 32, 5) viscous_element(ViscArgs a) {
    constexpr int MT = (NB + 7) / 8;  // 8-mode tiles of the contractions
    __shared__ double sc[kViscWarps][5 * NB];
    __shared__ double sh[kViscWarps][kViscMaxQv * 15];     // per volume point: (J^T H)[d][i] w detJ
    __shared__ double sv[kViscWarps][5 * kViscMaxQf + NB];  // the face block
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, gid = lane >> 2, tq = lane & 3;
    const int nqv = a.nqv, nqf = a.nqf, kv = 3 * nqv, mp = a.mp, bs = 5 * nqf + NB;
    double* c = sc[w];
    double* hs = sh[w];
    double* vb = sv[w];
    for (int64_t e = (int64_t)blockIdx.x * kViscWarps + w; e < a.ncell; e += (int64_t)gridDim.x * kViscWarps) {
        const double* ge = a.U + e * (5 * NB);
        for (int i = lane; i < 5 * NB; i += 32) c[i] = ge[i];
        double J[9];
        #pragma unroll
        for (int i = 0; i < 9; ++i) J[i] = a.geo[e * 10 + i];
        const double detj = a.geo[e * 10 + 9];
        __syncwarp();
        // volume term: per point the flux H_n (n = x, y, z) pulled back to reference directions,
        // hs[k = 3 g + d][i]
        for (int g = lane; g < nqv; g += 32) {
            double Uv[5], G[5][3];
            visc_trace_t<NB>(c, a.phiT_v, a.dphiT_v, nqv, g, J, Uv, G);
            const ViscState s = visc_state(Uv);
            double H[3][5];
            #pragma unroll
            for (int n = 0; n < 3; ++n) {
                const double d[3] = {n == 0 ? 1.0 : 0.0, n == 1 ? 1.0 : 0.0, n == 2 ? 1.0 : 0.0};
                visc_contract(s, a.mu, a.cq, G, d, H[n]);
            }
            const double wj = a.w_v[g] * detj;
            #pragma unroll
            for (int d = 0; d < 3; ++d)
                #pragma unroll
                for (int i = 0; i < 5; ++i)
                    hs[g * 15 + d * 5 + i] = (J[d] * H[0][i] + J[3 + d] * H[1][i] + J[6 + d] * H[2][i]) * wj;
        }
        __syncwarp();
        // R[j][i] = -sum_k Av[k][j] hs[k][i] on the tensor cores (B negated: exact)
        double acc[MT][2];
        #pragma unroll
        for (int mt = 0; mt < MT; ++mt) acc[mt][0] = acc[mt][1] = 0.0;
        for (int k0 = 0; k0 < kv; k0 += 4) {
            const int k = k0 + tq;
            const double b = (gid < 5 && k < kv) ? -hs[k * 5 + gid] : 0.0;
            const double* ar = a.Av + (int64_t)k * mp + gid;
            #pragma unroll
            for (int mt = 0; mt < MT; ++mt) visc_dmma(acc[mt], ar[mt * 8], b);
        }
        // the element's faces: R[j][i] += sgn sum_g phi_j^side(g) (Fl w 2A)[i][g], R[j][4] += sgn T_j
        for (int q = 0; q < 4; ++q) {
            const ElemFace E = a.ef[4 * e + q];
            const FaceInfo F = a.fi[E.face];
            if (!visc_face_active(F, a.UD)) continue;  // warp-uniform
            __syncwarp();
            const double* src = a.vf + (int64_t)E.face * bs;
            for (int i = lane; i < bs; i += 32) vb[i] = src[i];
            __syncwarp();
            const double sg = (E.meta >> 8) == 0 ? 1.0 : -1.0;
            const double* pt = a.Pf + (int64_t)(E.meta & 0xff) * a.kpf * mp;  // this side's basis values
            for (int g0 = 0; g0 < nqf; g0 += 4) {
                const int g = g0 + tq;
                const double b = (gid < 5 && g < nqf) ? sg * vb[gid * nqf + g] : 0.0;
                const double* ar = pt + (int64_t)g * mp + gid;
                #pragma unroll
                for (int mt = 0; mt < MT; ++mt) visc_dmma(acc[mt], ar[mt * 8], b);
            }
            if (tq == 2) {  // lanes holding column i = 4
                #pragma unroll
                for (int mt = 0; mt < MT; ++mt) {
                    const int j = mt * 8 + gid;
                    if (j < NB) acc[mt][0] += sg * vb[5 * nqf + j];
                }
            }
        }
        double* out = a.R + e * (5 * NB);
        #pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            const int j = mt * 8 + gid, i0 = 2 * tq;
            if (j < NB) {
                if (i0 < 5) out[5 * j + i0] = acc[mt][0];
                if (i0 + 1 < 5) out[5 * j + i0 + 1] = acc[mt][1];
            }
        }
        __syncwarp();
    }
}

inline int launch_viscous(int order, const ViscArgs& a, int sms, cudaStream_t s) {
    if (a.nqv > kViscMaxQv || a.nqf > kViscMaxQf) return DG_E_ARG;
    const unsigned gf = (unsigned)std::min<int64_t>((a.nface + kViscWarps - 1) / kViscWarps, (int64_t)sms * 32);
    const unsigned ge = (unsigned)std::min<int64_t>((a.ncell + kViscWarps - 1) / kViscWarps, (int64_t)sms * 32);
#define VISC_LAUNCH(NB)                                                 \
    viscous_face<NB><<<gf, kViscWarps * 32, 0, s>>>(a);                 \
    viscous_element<NB><<<ge, kViscWarps * 32, 0, s>>>(a);              \
    break;
    switch (order) {
        case 1: VISC_LAUNCH(4)
        case 2: VISC_LAUNCH(10)
        case 3: VISC_LAUNCH(20)
        case 4: VISC_LAUNCH(35)
        default: return DG_E_ARG;
    }
#undef VISC_LAUNCH
    return cuda_status(cudaGetLastError());
}

}  // namespace fvedg
