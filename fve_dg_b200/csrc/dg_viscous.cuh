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
//   viscous_face     one warp per face, lanes over the face points: both traces (values and physical
//                    gradients) once per face, the averaged flux with its penalty and the symmetric
//                    term's scalar; stored per point as Fl w 2A (5 values) and sfac w 2A.
//   viscous_element  one warp per element: the volume term (lanes over the volume points: J^T H w detJ
//                    per point; then lanes over the outputs (mode j, variable i) contract it with the
//                    reference gradients), then the element's four faces gathered with its side's basis
//                    values, plus the energy-only symmetric term n . (grad phi_j^L + grad phi_j^R),
//                    written as (J_L^T n) . dphi^L + (J_R^T n) . dphi^R. Each element writes its own
//                    residual: no atomics, a deterministic result.
#pragma once
#include "dg_kernels_fp64.cuh"

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
    const double* phiT_f;   // [24][nb][nqf]
    const double* dphiT_f;  // [24][nb][3][nqf]
    double* vf;             // [nface][6][nqf] per face point: Fl w 2A (5), sfac w 2A
    int64_t ncell, nface;
    int nqv, nqf, order;
    double mu, cq;          // viscosity and gamma / Pr
};

constexpr int kViscWarps = 4;
constexpr int kViscMaxQv = 64;  // volume points an element warp stages (the largest rule has 57)
constexpr int kViscMaxQf = 32;  // face points, one per lane (the largest rule has 24)

struct ViscState {  // what K needs of the state it is taken at
    double u[3], e, irho;
};

__device__ __forceinline__ ViscState visc_state(const double U[5]) {
    ViscState s;
    const double rho = U[0] > 1e-8 ? U[0] : 1e-8;
    s.irho = 1.0 / rho;
    s.u[0] = U[1] / U[0];
    s.u[1] = U[2] / U[0];
    s.u[2] = U[3] / U[0];
    s.e = U[4] / U[0];
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

// Faces whose viscous terms act: interior, Dirichlet with data, Pseudo3DZ (ExplicitDiffusion.h:380-612).
__device__ __forceinline__ bool visc_face_active(const FaceInfo& F, const double* UD) {
    const int bc = (F.meta >> 16) & 0xff;
    return F.c1 >= 0 || bc == 5 || (bc == 0 && UD != nullptr);
}

template <int NB>
__global__ void __launch_bounds__(kViscWarps * 32) viscous_face(ViscArgs a) {
    __shared__ double sc[kViscWarps][2][5 * NB];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double* cL = sc[w][0];
    double* cR = sc[w][1];
    const int nqf = a.nqf;
    const double beta_base = (double)((a.order + 1) * (a.order + 1));
    for (int64_t f = (int64_t)blockIdx.x * kViscWarps + w; f < a.nface; f += (int64_t)gridDim.x * kViscWarps) {
        const FaceInfo F = a.fi[f];
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
        if (lane < nqf) {
            const int g = lane;
            const int pL = F.meta & 0xff, pR = (F.meta >> 8) & 0xff;
            const double n[3] = {F.n[0], F.n[1], F.n[2]};
            double J[9];
            #pragma unroll
            for (int i = 0; i < 9; ++i) J[i] = a.geo[(int64_t)F.c0 * 10 + i];
            double UL[5], UR[5], X[5][3];
            visc_trace_t<NB>(cL, a.phiT_f + (int64_t)pL * NB * nqf, a.dphiT_f + (int64_t)pL * NB * 3 * nqf, nqf, g, J,
                             UL, X);
            if (interior) {
                #pragma unroll
                for (int i = 0; i < 9; ++i) J[i] = a.geo[(int64_t)F.c1 * 10 + i];
                double GR[5][3];
                visc_trace_t<NB>(cR, a.phiT_f + (int64_t)pR * NB * nqf, a.dphiT_f + (int64_t)pR * NB * 3 * nqf, nqf,
                                 g, J, UR, GR);
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
            double* out = a.vf + f * 6 * nqf;
            #pragma unroll
            for (int k = 0; k < 5; ++k) out[k * nqf + g] = (Fa[k] - beta * Fb[k]) * jw;
            out[5 * nqf + g] = (interior ? 0.5 : 1.0) * a.mu * a.cq * st.irho * (UR[4] - UL[4]) * jw;
        }
        __syncwarp();
    }
}

template <int NB>
__global__ void __launch_bounds__(kViscWarps * 32) viscous_element(ViscArgs a) {
    constexpr int NO = 5 * NB, OPL = (NO + 31) / 32;  // outputs (mode, variable) per lane
    __shared__ double sc[kViscWarps][5 * NB];
    __shared__ double sh[kViscWarps][kViscMaxQv * 15];  // per volume point: (J^T H)[d][i] w detJ
    __shared__ double sv[kViscWarps][6 * kViscMaxQf];   // the face block
    __shared__ double st_[kViscWarps][NB];              // symmetric term per mode
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nqv = a.nqv, nqf = a.nqf;
    double* c = sc[w];
    double* hs = sh[w];
    double* vb = sv[w];
    double* ts = st_[w];
    for (int64_t e = (int64_t)blockIdx.x * kViscWarps + w; e < a.ncell; e += (int64_t)gridDim.x * kViscWarps) {
        const double* ge = a.U + e * (5 * NB);
        for (int i = lane; i < 5 * NB; i += 32) c[i] = ge[i];
        double J[9];
        #pragma unroll
        for (int i = 0; i < 9; ++i) J[i] = a.geo[e * 10 + i];
        const double detj = a.geo[e * 10 + 9];
        __syncwarp();
        // volume term: per point the flux H_n (n = x, y, z) pulled back to reference directions
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
        double acc[OPL];
        #pragma unroll
        for (int r = 0; r < OPL; ++r) {
            acc[r] = 0.0;
            const int o = lane + 32 * r;
            if (o < NO) {
                const int j = o / 5, i = o - 5 * (o / 5);
                double v = 0.0;
                for (int g = 0; g < nqv; ++g) {
                    const double* dp = a.dphi_v + ((int64_t)g * NB + j) * 3;
                    const double* hg = hs + g * 15 + i;
                    v = fma(dp[0], hg[0], v);
                    v = fma(dp[1], hg[5], v);
                    v = fma(dp[2], hg[10], v);
                }
                acc[r] = -v;
            }
        }
        // the element's faces
        for (int q = 0; q < 4; ++q) {
            const ElemFace E = a.ef[4 * e + q];
            const FaceInfo F = a.fi[E.face];
            if (!visc_face_active(F, a.UD)) continue;  // warp-uniform
            const bool interior = F.c1 >= 0;
            __syncwarp();
            const double* src = a.vf + (int64_t)E.face * 6 * nqf;
            for (int i = lane; i < 6 * nqf; i += 32) vb[i] = src[i];
            // symmetric term T_j = sum_g sfac_g ((J_L^T n) . dphi_j^L(g) + (J_R^T n) . dphi_j^R(g))
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
            __syncwarp();
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
                    t = fma(vb[5 * nqf + g], sj, t);
                }
                ts[j] = t;
            }
            __syncwarp();
            const double sgn = (E.meta >> 8) == 0 ? 1.0 : -1.0;
            const double* ph = a.phi_f + (int64_t)(E.meta & 0xff) * nqf * NB;  // this side's basis values
            #pragma unroll
            for (int r = 0; r < OPL; ++r) {
                const int o = lane + 32 * r;
                if (o < NO) {
                    const int j = o / 5, i = o - 5 * (o / 5);
                    double v = 0.0;
                    for (int g = 0; g < nqf; ++g) v = fma(ph[g * NB + j], vb[i * nqf + g], v);
                    if (i == 4) v += ts[j];
                    acc[r] += sgn * v;
                }
            }
        }
        double* out = a.R + e * (5 * NB);
        #pragma unroll
        for (int r = 0; r < OPL; ++r) {
            const int o = lane + 32 * r;
            if (o < NO) out[o] = acc[r];
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
    return cudaGetLastError() == cudaSuccess ? DG_OK : DG_E_CUDA;
}

}  // namespace fvedg
