// Pointwise Euler physics shared by the kernels, templated on the arithmetic type so the FP64 form
// and the mixed form (FP32 flux) use one definition.
//
// Physical flux, pressure and wave speed follow src/DG/DG_Flux/EulerPhysicalFlux.cpp:7-89,
// including the positivity clamp max(rho, 1e-16) (:59-61) and c = sqrt(gamma max(p/rho, 1e-16))
// (:70-73). Local Lax-Friedrichs follows ExplicitConvection.cpp:232-240. The Roe flux is new (the
// reference declares one in tests/test_flux/RiemannSolvers.h:21-27 but never defines it): Roe
// averages, the five characteristic waves of 3D Euler, Harten's entropy fix on the acoustic waves
// with delta = 0.1 c_roe.
#pragma once
#include "dg_status.cuh"

namespace fvedg {

// Division and square root: IEEE in FP64 (the plain form's parity), the fast hardware
// approximations in FP32 (a few ulp; the mixed form's flux is FP32 by design).
__device__ __forceinline__ double dg_div(double a, double b) { return a / b; }
__device__ __forceinline__ float dg_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double dg_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dg_sqrt(float x) { return x > 0.f ? x * rsqrtf(x) : 0.f; }

template <typename T>
struct Phys {
    static __device__ __forceinline__ T positive(T v) { return v > T(1e-16) ? v : T(1e-16); }

    // F . n for the state U (the 5x3 physical flux contracted with the unit normal), plus the
    // primitive quantities the Riemann solvers reuse.
    static __device__ __forceinline__ void flux_n(const T U[5], const T n[3], T gm1, T Fn[5], T& rho,
                                                  T vel[3], T& p) {
        rho = positive(U[0]);
        const T ir = dg_div(T(1), rho);
        vel[0] = U[1] * ir;
        vel[1] = U[2] * ir;
        vel[2] = U[3] * ir;
        const T e = U[4] * ir;
        p = gm1 * (rho * e - T(0.5) * rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]));
        const T un = vel[0] * n[0] + vel[1] * n[1] + vel[2] * n[2];
        Fn[0] = rho * un;
        Fn[1] = rho * vel[0] * un + p * n[0];
        Fn[2] = rho * vel[1] * un + p * n[1];
        Fn[3] = rho * vel[2] * un + p * n[2];
        Fn[4] = un * (rho * e + p);
    }

    // Full 5x3 flux, row = variable, column = direction (EulerPhysicalFlux.cpp:8-18).
    static __device__ __forceinline__ void flux(const T U[5], T gm1, T F[5][3]) {
        const T rho = positive(U[0]);
        const T ir = dg_div(T(1), rho);
        const T u = U[1] * ir, v = U[2] * ir, w = U[3] * ir, e = U[4] * ir;
        const T p = gm1 * (rho * e - T(0.5) * rho * (u * u + v * v + w * w));
        F[0][0] = rho * u;         F[0][1] = rho * v;         F[0][2] = rho * w;
        F[1][0] = rho * u * u + p; F[1][1] = rho * v * u;     F[1][2] = rho * w * u;
        F[2][0] = rho * u * v;     F[2][1] = rho * v * v + p; F[2][2] = rho * w * v;
        F[3][0] = rho * u * w;     F[3][1] = rho * v * w;     F[3][2] = rho * w * w + p;
        const T h = rho * e + p;
        F[4][0] = u * h;           F[4][1] = v * h;           F[4][2] = w * h;
    }

    static __device__ __forceinline__ T wave_speed(T rho, const T vel[3], T p, T gam) {
        const T c = dg_sqrt(gam * positive(dg_div(p, rho)));
        return dg_sqrt(vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]) + c;
    }

    static __device__ __forceinline__ void lax_friedrichs(const T UL[5], const T UR[5], const T n[3],
                                                          T gam, T Fh[5]) {
        T FL[5], FR[5], vL[3], vR[3], rL, rR, pL, pR;
        flux_n(UL, n, gam - T(1), FL, rL, vL, pL);
        flux_n(UR, n, gam - T(1), FR, rR, vR, pR);
        const T a = wave_speed(rL, vL, pL, gam), b = wave_speed(rR, vR, pR, gam);
        const T lam = a > b ? a : b;
        #pragma unroll
        for (int k = 0; k < 5; ++k) Fh[k] = T(0.5) * (FL[k] + FR[k] + lam * (UL[k] - UR[k]));
    }

    static __device__ __forceinline__ void roe(const T UL[5], const T UR[5], const T n[3], T gam, T Fh[5]) {
        T FL[5], FR[5], uL[3], uR[3], rL, rR, pL, pR;
        const T gm1 = gam - T(1);
        flux_n(UL, n, gm1, FL, rL, uL, pL);
        flux_n(UR, n, gm1, FR, rR, uR, pR);
        const T HL = dg_div(UL[4] + pL, rL), HR = dg_div(UR[4] + pR, rR);
        const T sL = dg_sqrt(rL), sR = dg_sqrt(rR), iden = dg_div(T(1), sL + sR);
        T ut[3];
        #pragma unroll
        for (int i = 0; i < 3; ++i) ut[i] = (sL * uL[i] + sR * uR[i]) * iden;
        const T Ht = (sL * HL + sR * HR) * iden;
        const T q2 = ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2];
        const T c2 = positive(gm1 * (Ht - T(0.5) * q2));
        const T ct = dg_sqrt(c2);
        const T ic2 = dg_div(T(1), c2);
        const T rt = sL * sR;
        const T unt = ut[0] * n[0] + ut[1] * n[1] + ut[2] * n[2];
        const T dr = rR - rL, dp = pR - pL;
        T du[3];
        #pragma unroll
        for (int i = 0; i < 3; ++i) du[i] = uR[i] - uL[i];
        const T dun = du[0] * n[0] + du[1] * n[1] + du[2] * n[2];
        T l1 = fabs(unt - ct), l2 = fabs(unt), l5 = fabs(unt + ct);
        const T delta = T(0.1) * ct;
        if (l1 < delta) l1 = dg_div(l1 * l1 + delta * delta, T(2) * delta);
        if (l5 < delta) l5 = dg_div(l5 * l5 + delta * delta, T(2) * delta);
        const T a1 = (dp - rt * ct * dun) * (T(0.5) * ic2);
        const T a5 = (dp + rt * ct * dun) * (T(0.5) * ic2);
        const T a2 = dr - dp * ic2;
        const T w1 = l1 * a1, w5 = l5 * a5, w2 = l2 * a2;
        T D[5];
        D[0] = w1 + w5 + w2;
        T uds = T(0);
        #pragma unroll
        for (int i = 0; i < 3; ++i) {
            const T sh = du[i] - dun * n[i];
            D[1 + i] = w1 * (ut[i] - ct * n[i]) + w5 * (ut[i] + ct * n[i]) + w2 * ut[i] + l2 * rt * sh;
            uds += ut[i] * sh;
        }
        D[4] = w1 * (Ht - ct * unt) + w5 * (Ht + ct * unt) + w2 * T(0.5) * q2 + l2 * rt * uds;
        #pragma unroll
        for (int k = 0; k < 5; ++k) Fh[k] = T(0.5) * (FL[k] + FR[k]) - T(0.5) * D[k];
    }
};

// FP64 forms for the tensor-core FP64 kernels: the same fluxes as Phys<double> with fewer divisions
// and square roots (each costs a multi-instruction sequence in FP64). One reciprocal square root per
// state gives both sqrt(rho) = rho q and 1/rho = q^2 (q = rsqrt(rho)); H = (E + p)/rho uses that
// reciprocal; the Roe sound speed and 1/c^2 come from one rsqrt of c^2; the LF wave speeds from
// rsqrt as well. Agreement with Phys<double> is a few ulp per point, far inside the 1e-12 parity bar.
struct StateF64 {
    double r, ir, u[3], p, e, un, mn;  // clamped density, 1/rho, velocity, pressure, E + p, u.n, m.n
};

__device__ __forceinline__ StateF64 state_f64(const double U[5], const double n[3], double gm1, double& q) {
    StateF64 s;
    s.r = U[0] > 1e-16 ? U[0] : 1e-16;
    q = rsqrt(s.r);
    s.ir = q * q;
    #pragma unroll
    for (int i = 0; i < 3; ++i) s.u[i] = U[1 + i] * s.ir;
    const double k = s.u[0] * U[1] + s.u[1] * U[2] + s.u[2] * U[3];  // rho |u|^2
    s.p = gm1 * fma(-0.5, k, U[4]);
    s.e = U[4] + s.p;
    s.mn = U[1] * n[0] + U[2] * n[1] + U[3] * n[2];
    s.un = s.mn * s.ir;
    return s;
}

__device__ __forceinline__ void roe_f64(const double UL[5], const double UR[5], const double n[3], double gam,
                                        double Fh[5]) {
    const double gm1 = gam - 1.0;
    double qL, qR;
    const StateF64 L = state_f64(UL, n, gm1, qL), R = state_f64(UR, n, gm1, qR);
    const double sL = L.r * qL, sR = R.r * qR;  // sqrt(rho)
    const double iden = 1.0 / (sL + sR);
    const double wL = sL * iden, wR = sR * iden;
    double ut[3];
    #pragma unroll
    for (int i = 0; i < 3; ++i) ut[i] = fma(wL, L.u[i], wR * R.u[i]);
    const double Ht = fma(wL, L.e * L.ir, wR * (R.e * R.ir));
    const double q2 = ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2];
    const double c2r = gm1 * fma(-0.5, q2, Ht);
    const double c2 = c2r > 1e-16 ? c2r : 1e-16;
    const double qc = rsqrt(c2);
    const double ct = c2 * qc, ic2 = qc * qc;
    const double rt = sL * sR;
    const double unt = ut[0] * n[0] + ut[1] * n[1] + ut[2] * n[2];
    const double dr = R.r - L.r, dp = R.p - L.p, dun = R.un - L.un;
    double l1 = fabs(unt - ct), l5 = fabs(unt + ct);
    const double l2 = fabs(unt);
    const double delta = 0.1 * ct, d2 = delta * delta;
    if (l1 < delta || l5 < delta) {  // Harten's fix, rarely active
        const double ihd = 0.5 / delta;
        if (l1 < delta) l1 = fma(l1, l1, d2) * ihd;
        if (l5 < delta) l5 = fma(l5, l5, d2) * ihd;
    }
    const double rcd = rt * ct * dun, h2 = 0.5 * ic2;
    const double w1 = l1 * ((dp - rcd) * h2), w5 = l5 * ((dp + rcd) * h2), w2 = l2 * fma(-dp, ic2, dr);
    const double W = w1 + w5 + w2, cw = ct * (w5 - w1), lrt = l2 * rt;
    double uds = 0.0, D[5];
    D[0] = W;
    #pragma unroll
    for (int i = 0; i < 3; ++i) {
        const double sh = fma(-dun, n[i], R.u[i] - L.u[i]);
        uds = fma(ut[i], sh, uds);
        D[1 + i] = fma(W, ut[i], fma(cw, n[i], lrt * sh));
    }
    D[4] = fma(w1 + w5, Ht, fma(cw, unt, fma(0.5 * w2, q2, lrt * uds)));
    const double ps = L.p + R.p;
    Fh[0] = 0.5 * (L.mn + R.mn - D[0]);
    #pragma unroll
    for (int i = 0; i < 3; ++i) Fh[1 + i] = 0.5 * (fma(UL[1 + i], L.un, fma(UR[1 + i], R.un, ps * n[i])) - D[1 + i]);
    Fh[4] = 0.5 * (fma(L.un, L.e, R.un * R.e) - D[4]);
}

__device__ __forceinline__ void lax_friedrichs_f64(const double UL[5], const double UR[5], const double n[3],
                                                   double gam, double Fh[5]) {
    const double gm1 = gam - 1.0;
    double qL, qR;
    const StateF64 L = state_f64(UL, n, gm1, qL), R = state_f64(UR, n, gm1, qR);
    auto speed = [&](const StateF64& s) {  // |u| + sqrt(gamma max(p/rho, 1e-16)) (EulerPhysicalFlux.cpp:70-81)
        const double v2 = s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2];
        const double pr = s.p * s.ir;
        const double c2 = gam * (pr > 1e-16 ? pr : 1e-16);
        const double v = v2 > 0.0 ? v2 * rsqrt(v2) : 0.0;
        return v + c2 * rsqrt(c2);
    };
    const double a = speed(L), b = speed(R);
    const double lam = a > b ? a : b;
    Fh[0] = 0.5 * fma(lam, UL[0] - UR[0], L.mn + R.mn);
    const double ps = L.p + R.p;
    #pragma unroll
    for (int i = 0; i < 3; ++i)
        Fh[1 + i] = 0.5 * fma(lam, UL[1 + i] - UR[1 + i], fma(UL[1 + i], L.un, fma(UR[1 + i], R.un, ps * n[i])));
    Fh[4] = 0.5 * fma(lam, UL[4] - UR[4], fma(L.un, L.e, R.un * R.e));
}

// FP32 forms for the mixed-precision kernels: the same fluxes as Phys<float>, reorganised for fewer
// instructions. The momenta are used directly (rho u = m, rho u.n = m.n, rho e = E), each state
// costs one reciprocal, square roots come from the hardware reciprocal square root (the arguments
// are clamped positive), and the Roe dissipation shares its subexpressions:
//   D_0 = W, D_{1+i} = W u~_i + c~ (w5 - w1) n_i + |u~.n| r~ (du_i - du.n n_i),
//   D_4 = (w1 + w5) H~ + c~ (w5 - w1) u~.n + w2 |u~|^2 / 2 + |u~.n| r~ u~.(du - du.n n),
// with W = w1 + w2 + w5, which is the wave sum of Phys::roe term by term.
struct StateF32 {
    float r, ir, u[3], p, e, un, mn;  // clamped density, 1/rho, velocity, pressure, E + p, u.n, m.n
};

__device__ __forceinline__ float rcp_f32(float x) { return __fdividef(1.f, x); }

__device__ __forceinline__ StateF32 state_f32(const float U[5], const float n[3], float gm1) {
    StateF32 s;
    s.r = fmaxf(U[0], 1e-16f);
    s.ir = rcp_f32(s.r);
    #pragma unroll
    for (int i = 0; i < 3; ++i) s.u[i] = U[1 + i] * s.ir;
    const float k = s.u[0] * U[1] + s.u[1] * U[2] + s.u[2] * U[3];  // rho |u|^2
    s.p = gm1 * fmaf(-0.5f, k, U[4]);
    s.e = U[4] + s.p;
    s.mn = U[1] * n[0] + U[2] * n[1] + U[3] * n[2];
    s.un = s.mn * s.ir;
    return s;
}

__device__ __forceinline__ void roe_f32(const float UL[5], const float UR[5], const float n[3], float gam, float Fh[5]) {
    const float gm1 = gam - 1.f;
    const StateF32 L = state_f32(UL, n, gm1), R = state_f32(UR, n, gm1);
    const float qL = rsqrtf(L.r), qR = rsqrtf(R.r);
    const float sL = L.r * qL, sR = R.r * qR;  // sqrt(rho)
    const float iden = rcp_f32(sL + sR);
    const float wL = sL * iden, wR = sR * iden;
    float ut[3];
    #pragma unroll
    for (int i = 0; i < 3; ++i) ut[i] = fmaf(wL, L.u[i], wR * R.u[i]);
    const float Ht = fmaf(wL, L.e * L.ir, wR * (R.e * R.ir));
    const float q2 = ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2];
    const float c2 = fmaxf(gm1 * fmaf(-0.5f, q2, Ht), 1e-16f);
    const float qc = rsqrtf(c2);
    const float ct = c2 * qc, ic2 = qc * qc;
    const float rt = sL * sR;
    const float unt = ut[0] * n[0] + ut[1] * n[1] + ut[2] * n[2];
    const float dr = R.r - L.r, dp = R.p - L.p, dun = R.un - L.un;
    float l1 = fabsf(unt - ct), l5 = fabsf(unt + ct);
    const float l2 = fabsf(unt);
    const float delta = 0.1f * ct, d2 = delta * delta, ihd = __fdividef(0.5f, delta);
    if (l1 < delta) l1 = fmaf(l1, l1, d2) * ihd;
    if (l5 < delta) l5 = fmaf(l5, l5, d2) * ihd;
    const float rcd = rt * ct * dun, h2 = 0.5f * ic2;
    const float w1 = l1 * ((dp - rcd) * h2), w5 = l5 * ((dp + rcd) * h2), w2 = l2 * fmaf(-dp, ic2, dr);
    const float W = w1 + w5 + w2, cw = ct * (w5 - w1), lrt = l2 * rt;
    float uds = 0.f, D[5];
    D[0] = W;
    #pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float sh = fmaf(-dun, n[i], R.u[i] - L.u[i]);
        uds = fmaf(ut[i], sh, uds);
        D[1 + i] = fmaf(W, ut[i], fmaf(cw, n[i], lrt * sh));
    }
    D[4] = fmaf(w1 + w5, Ht, fmaf(cw, unt, fmaf(0.5f * w2, q2, lrt * uds)));
    const float ps = L.p + R.p;
    Fh[0] = 0.5f * (L.mn + R.mn - D[0]);
    #pragma unroll
    for (int i = 0; i < 3; ++i) Fh[1 + i] = 0.5f * (fmaf(UL[1 + i], L.un, fmaf(UR[1 + i], R.un, ps * n[i])) - D[1 + i]);
    Fh[4] = 0.5f * (fmaf(L.un, L.e, R.un * R.e) - D[4]);
}

__device__ __forceinline__ void lax_friedrichs_f32(const float UL[5], const float UR[5], const float n[3], float gam,
                                                   float Fh[5]) {
    const float gm1 = gam - 1.f;
    const StateF32 L = state_f32(UL, n, gm1), R = state_f32(UR, n, gm1);
    auto speed = [&](const StateF32& s) {
        const float v2 = s.u[0] * s.u[0] + s.u[1] * s.u[1] + s.u[2] * s.u[2];
        const float c2 = fmaxf(gam * fmaxf(s.p * s.ir, 1e-16f), 1e-16f);
        const float v = v2 > 0.f ? v2 * rsqrtf(v2) : 0.f;
        return v + c2 * rsqrtf(c2);
    };
    const float lam = fmaxf(speed(L), speed(R));
    Fh[0] = 0.5f * fmaf(lam, UL[0] - UR[0], L.mn + R.mn);
    const float ps = L.p + R.p;
    #pragma unroll
    for (int i = 0; i < 3; ++i)
        Fh[1 + i] = 0.5f * fmaf(lam, UL[1 + i] - UR[1 + i], fmaf(UL[1 + i], L.un, fmaf(UR[1 + i], R.un, ps * n[i])));
    Fh[4] = 0.5f * fmaf(lam, UL[4] - UR[4], fmaf(L.un, L.e, R.un * R.e));
}

// Full 5 x 3 flux in FP32 (row = variable, column = direction), momenta used directly.
__device__ __forceinline__ void flux_f32(const float U[5], float gm1, float F[5][3]) {
    const float r = fmaxf(U[0], 1e-16f), ir = rcp_f32(r);
    const float u[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
    const float p = gm1 * fmaf(-0.5f, u[0] * U[1] + u[1] * U[2] + u[2] * U[3], U[4]);
    const float e = U[4] + p;
    #pragma unroll
    for (int d = 0; d < 3; ++d) {
        F[0][d] = U[1 + d];
        #pragma unroll
        for (int i = 0; i < 3; ++i) F[1 + i][d] = U[1 + i] * u[d] + (i == d ? p : 0.f);
        F[4][d] = u[d] * e;
    }
}

}  // namespace fvedg
