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
// One thread per element owns that element's residual: the volume term and its share of each of
// its four faces (the neighbour's trace is recomputed), so no atomics and a deterministic result.
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
    int64_t ncell;
    int nqv, nqf, order;
    double mu, cq;          // viscosity and gamma / Pr
};

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

// Value and physical gradient of the state at a point: Uv[k], G[k][m].
template <int NB>
__device__ __forceinline__ void visc_trace(const double* c, const double* phi, const double* dphi, const double J[9],
                                           double Uv[5], double G[5][3]) {
    #pragma unroll
    for (int k = 0; k < 5; ++k) {
        Uv[k] = 0.0;
        G[k][0] = G[k][1] = G[k][2] = 0.0;
    }
    for (int b = 0; b < NB; ++b) {
        const double gr[3] = {J[0] * dphi[3 * b] + J[1] * dphi[3 * b + 1] + J[2] * dphi[3 * b + 2],
                              J[3] * dphi[3 * b] + J[4] * dphi[3 * b + 1] + J[5] * dphi[3 * b + 2],
                              J[6] * dphi[3 * b] + J[7] * dphi[3 * b + 1] + J[8] * dphi[3 * b + 2]};
        #pragma unroll
        for (int k = 0; k < 5; ++k) {
            const double cb = c[5 * b + k];
            Uv[k] += phi[b] * cb;
            G[k][0] += gr[0] * cb;
            G[k][1] += gr[1] * cb;
            G[k][2] += gr[2] * cb;
        }
    }
}

__device__ __forceinline__ double grad_phi_dot(const double J[9], const double* dphi_b, const double d[3]) {
    const double g0 = J[0] * dphi_b[0] + J[1] * dphi_b[1] + J[2] * dphi_b[2];
    const double g1 = J[3] * dphi_b[0] + J[4] * dphi_b[1] + J[5] * dphi_b[2];
    const double g2 = J[6] * dphi_b[0] + J[7] * dphi_b[1] + J[8] * dphi_b[2];
    return g0 * d[0] + g1 * d[1] + g2 * d[2];
}

template <int NB>
__global__ void __launch_bounds__(128) viscous_residual(ViscArgs a) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.ncell) return;
    double acc[5 * NB];
    for (int i = 0; i < 5 * NB; ++i) acc[i] = 0.0;
    double J[9];
    for (int i = 0; i < 9; ++i) J[i] = a.geo[e * 10 + i];
    const double detj = a.geo[e * 10 + 9];
    const double* c = a.U + e * (5 * NB);
    // volume term
    for (int g = 0; g < a.nqv; ++g) {
        double Uv[5], G[5][3];
        visc_trace<NB>(c, a.phi_v + g * NB, a.dphi_v + g * NB * 3, J, Uv, G);
        const ViscState st = visc_state(Uv);
        double H[3][5];  // H_n for unit directions n
        #pragma unroll
        for (int n = 0; n < 3; ++n) {
            const double d[3] = {n == 0 ? 1.0 : 0.0, n == 1 ? 1.0 : 0.0, n == 2 ? 1.0 : 0.0};
            visc_contract(st, a.mu, a.cq, G, d, H[n]);
        }
        const double wj = a.w_v[g] * detj;
        for (int j = 0; j < NB; ++j) {
            const double* dp = a.dphi_v + (g * NB + j) * 3;
            const double gj[3] = {J[0] * dp[0] + J[1] * dp[1] + J[2] * dp[2], J[3] * dp[0] + J[4] * dp[1] + J[5] * dp[2],
                                  J[6] * dp[0] + J[7] * dp[1] + J[8] * dp[2]};
            #pragma unroll
            for (int i = 0; i < 5; ++i) acc[5 * j + i] -= (gj[0] * H[0][i] + gj[1] * H[1][i] + gj[2] * H[2][i]) * wj;
        }
    }
    // faces
    const double beta_base = (double)((a.order + 1) * (a.order + 1));
    for (int q = 0; q < 4; ++q) {
        const ElemFace E = a.ef[4 * e + q];
        const FaceInfo F = a.fi[E.face];
        const int side = E.meta >> 8;
        const int bc = (F.meta >> 16) & 0xff;
        const bool interior = F.c1 >= 0;
        if (!interior && bc != 0 && bc != 5) continue;
        if (!interior && bc == 0 && !a.UD) continue;
        const double n[3] = {F.n[0], F.n[1], F.n[2]};
        const double beta = beta_base / a.h[F.c0];
        const int pL = F.meta & 0xff, pR = (F.meta >> 8) & 0xff;
        double JL[9], JR[9];
        for (int i = 0; i < 9; ++i) JL[i] = a.geo[(int64_t)F.c0 * 10 + i];
        if (interior)
            for (int i = 0; i < 9; ++i) JR[i] = a.geo[(int64_t)F.c1 * 10 + i];
        const double* cL = a.U + (int64_t)F.c0 * (5 * NB);
        const double* cR = interior ? a.U + (int64_t)F.c1 * (5 * NB) : cL;
        for (int g = 0; g < a.nqf; ++g) {
            const double jw = a.w_f[g] * F.jw;
            const double* phL = a.phi_f + ((int64_t)pL * a.nqf + g) * NB;
            const double* dpL = a.dphi_f + ((int64_t)pL * a.nqf + g) * NB * 3;
            double UL[5], GL[5][3], UR[5], GR[5][3];
            visc_trace<NB>(cL, phL, dpL, JL, UL, GL);
            const double* phR = nullptr;
            const double* dpR = nullptr;
            if (interior) {
                phR = a.phi_f + ((int64_t)pR * a.nqf + g) * NB;
                dpR = a.dphi_f + ((int64_t)pR * a.nqf + g) * NB * 3;
                visc_trace<NB>(cR, phR, dpR, JR, UR, GR);
            } else if (bc == 0) {
                const double* ud = a.UD + ((int64_t)E.face * a.nqf + g) * 5;
                for (int k = 0; k < 5; ++k) UR[k] = ud[k] + (ud[k] - UL[k]);  // ghost
            } else {
                for (int k = 0; k < 5; ++k) UR[k] = UL[k];
                UR[3] = -UL[3];
            }
            double Um[5];
            for (int k = 0; k < 5; ++k) Um[k] = 0.5 * (UL[k] + UR[k]);
            const ViscState st = visc_state(Um);
            // averaged flux and penalty
            double X[5][3], Fa[5], Fb[5];
            for (int k = 0; k < 5; ++k)
                for (int m = 0; m < 3; ++m) X[k][m] = interior ? 0.5 * (GL[k][m] + GR[k][m]) : GL[k][m];
            visc_contract(st, a.mu, a.cq, X, n, Fa);
            for (int k = 0; k < 5; ++k) {
                const double dU = interior ? UL[k] - UR[k] : UL[k];
                for (int m = 0; m < 3; ++m) X[k][m] = dU * n[m];
            }
            visc_contract(st, a.mu, a.cq, X, n, Fb);
            double Fl[5];
            for (int k = 0; k < 5; ++k) Fl[k] = Fa[k] - beta * Fb[k];
            // symmetric term, energy equation only
            const double sfac = (interior ? 0.5 : 1.0) * a.mu * a.cq * st.irho * (UR[4] - UL[4]);
            const double sgn = side == 0 ? 1.0 : -1.0;
            const double* phS = side == 0 ? phL : phR;
            for (int j = 0; j < NB; ++j) {
                double sj = grad_phi_dot(JL, dpL + 3 * j, n);
                if (interior) sj += grad_phi_dot(JR, dpR + 3 * j, n);
                const double pj = phS[j];
                #pragma unroll
                for (int i = 0; i < 5; ++i) acc[5 * j + i] += sgn * pj * Fl[i] * jw;
                acc[5 * j + 4] += sgn * sfac * sj * jw;
            }
        }
    }
    double* r = a.R + e * (5 * NB);
    for (int i = 0; i < 5 * NB; ++i) r[i] = acc[i];
}

inline int launch_viscous(int order, const ViscArgs& a, cudaStream_t s) {
    const unsigned g = (unsigned)((a.ncell + 127) / 128);
    switch (order) {
        case 1: viscous_residual<4><<<g, 128, 0, s>>>(a); break;
        case 2: viscous_residual<10><<<g, 128, 0, s>>>(a); break;
        case 3: viscous_residual<20><<<g, 128, 0, s>>>(a); break;
        case 4: viscous_residual<35><<<g, 128, 0, s>>>(a); break;
        default: return DG_E_ARG;
    }
    return cudaGetLastError() == cudaSuccess ? DG_OK : DG_E_CUDA;
}

}  // namespace fvedg
