/* Test infrastructure (oracle): plain-C restatement of the reference's explicit DG Euler operator.
 * See dg_oracle.h for the role of this file and the mesh arguments. Every routine cites the
 * reference lines it follows. Single-threaded and written for clarity, not speed.
 */
#include "dg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "quad_tables.inc"

#define MAXNB 56
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#define EPS_POS 1e-16

/* ------------------------------------------------------------------------------------------ */
/* Basis: the orthogonal modal (Dubiner-type, unnormalised) basis of                            */
/* include/DG/DG_Basis/DG_Basis_Func.h (generated by scripts/codegen/Basis.py:57-...), restated */
/* from its definition on the reference tet {(0,0,0),(1,0,0),(0,1,0),(0,0,1)}:                  */
/*   psi_pqr = P_p^{(2q+2r+2,0)}(2x-1) * (1-x)^q P_q^{(2r+1,0)}(2y/(1-x)-1)                     */
/*             * (1-x-y)^r P_r^{(0,0)}(2z/(1-x-y)-1)                                              */
/* ordered by total degree n, then r = 0..n, then q = 0..n-r (p = n-q-r).                       */
/* The collapsed factors are evaluated in homogeneous form s^n P_n((2y-s)/s) through the        */
/* three-term Jacobi recurrence, so no division by s occurs.                                    */
/* ------------------------------------------------------------------------------------------ */
int orc_num_basis(int order) { return (order + 1) * (order + 2) * (order + 3) / 6; }

/* Q_n(y, s) = s^n P_n^{(a,0)}((2y - s)/s) and its partial derivatives in y and s, n = 0..N. */
static void jac_homog(int N, double a, double y, double s, double* Q, double* Qy, double* Qs) {
    Q[0] = 1.0; Qy[0] = 0.0; Qs[0] = 0.0;
    if (N == 0) return;
    /* P_1 = ((a+2) t + a) / 2  ->  Q_1 = ((a+2)(2y - s) + a s) / 2 = (a+2) y - s */
    Q[1] = (a + 2.0) * y - s;
    Qy[1] = a + 2.0;
    Qs[1] = -1.0;
    for (int n = 1; n < N; ++n) {
        /* 2(n+1)(n+a+1)(2n+a) P_{n+1} = (2n+a+1)[(2n+a+2)(2n+a) t + a^2] P_n
                                          - 2 n (n+a)(2n+a+2) P_{n-1}                      */
        const double d = 2.0 * (n + 1) * (n + a + 1) * (2 * n + a);
        const double c1 = (2 * n + a + 1) * (2 * n + a + 2) * (2 * n + a) / d; /* times t */
        const double c2 = (2 * n + a + 1) * a * a / d;
        const double c3 = 2.0 * n * (n + a) * (2 * n + a + 2) / d;
        const double lin = c1 * (2.0 * y - s) + c2 * s; /* homogenised (c1 t + c2) * s */
        Q[n + 1] = lin * Q[n] - c3 * s * s * Q[n - 1];
        Qy[n + 1] = 2.0 * c1 * Q[n] + lin * Qy[n] - c3 * s * s * Qy[n - 1];
        Qs[n + 1] = (c2 - c1) * Q[n] + lin * Qs[n] - 2.0 * c3 * s * Q[n - 1] - c3 * s * s * Qs[n - 1];
    }
}

static void basis_point(int order, double x, double y, double z, double* phi, double* grad) {
    int idx = 0;
    for (int n = 0; n <= order; ++n) {
        for (int r = 0; r <= n; ++r) {
            for (int q = 0; q <= n - r; ++q) {
                const int p = n - q - r;
                double X[12], Xy[12], Xs[12], Y[12], Yy[12], Ys[12], Z[12], Zy[12], Zs[12];
                /* x factor: P_p^{(2q+2r+2,0)}(2x-1) = Q_p(x, 1) */
                jac_homog(p, 2.0 * q + 2.0 * r + 2.0, x, 1.0, X, Xy, Xs);
                /* y factor with s = 1 - x */
                jac_homog(q, 2.0 * r + 1.0, y, 1.0 - x, Y, Yy, Ys);
                /* z factor with s = 1 - x - y */
                jac_homog(r, 0.0, z, 1.0 - x - y, Z, Zy, Zs);
                const double fx = X[p], fy = Y[q], fz = Z[r];
                if (phi) phi[idx] = fx * fy * fz;
                if (grad) {
                    const double dfx = Xy[p];             /* d/dx of the x factor */
                    const double dfy_dx = -Ys[q];         /* s = 1 - x            */
                    const double dfy_dy = Yy[q];
                    const double dfz_dx = -Zs[r];         /* s = 1 - x - y        */
                    const double dfz_dy = -Zs[r];
                    const double dfz_dz = Zy[r];
                    grad[3 * idx + 0] = dfx * fy * fz + fx * dfy_dx * fz + fx * fy * dfz_dx;
                    grad[3 * idx + 1] = fx * dfy_dy * fz + fx * fy * dfz_dy;
                    grad[3 * idx + 2] = fx * fy * dfz_dz;
                }
                ++idx;
            }
        }
    }
}

int orc_basis(int order, int npts, const double* xyz, double* phi, double* grad) {
    const int nb = orc_num_basis(order);
    if (order < 0 || order > 5) return -1;
    for (int g = 0; g < npts; ++g)
        basis_point(order, xyz[3 * g], xyz[3 * g + 1], xyz[3 * g + 2], phi ? phi + g * nb : NULL,
                    grad ? grad + 3 * g * nb : NULL);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Geometry: src/Mesh/ComputingMesh.cpp:27-171. Arithmetic is written in the same order as the  */
/* reference (vec_dot of include/base/vector_op.h:121-141 sums left to right from 0 for N=3;    */
/* the 3x3 inverse is DenseMatrix.h:519-538), and this file is built with -ffp-contract=off,    */
/* so the results agree with the reference to the last bit.                                     */
/* ------------------------------------------------------------------------------------------ */
static double dot3(const double* a, const double* b) {
    double s = 0.0;
    s += a[0] * b[0];
    s += a[1] * b[1];
    s += a[2] * b[2];
    return s;
}
static void cross3(const double* a, const double* b, double* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
static void sub3(const double* a, const double* b, double* c) {
    c[0] = a[0] - b[0]; c[1] = a[1] - b[1]; c[2] = a[2] - b[2];
}

static void tet_geometry(const orc_mesh* m, int64_t c, double* invj, double* detj, double* cen) {
    const double* p0 = m->pts + 3 * m->cells[4 * c + 0];
    const double* p1 = m->pts + 3 * m->cells[4 * c + 1];
    const double* p2 = m->pts + 3 * m->cells[4 * c + 2];
    const double* p3 = m->pts + 3 * m->cells[4 * c + 3];
    for (int i = 0; i < 3; ++i) cen[i] = (((p0[i] + p1[i]) + p2[i]) + p3[i]) / 4.0; /* :120 */
    double v1[3], v2[3], v3[3], cr[3];
    sub3(p1, p0, v1); sub3(p2, p0, v2); sub3(p3, p0, v3);
    cross3(v2, v3, cr);
    const double vol = fabs(dot3(v1, cr)) / 6.0; /* :121-122 */
    *detj = vol * 6.0;                          /* :145-147 */
    /* inverse of A = rows {v1, v2, v3}, DenseMatrix.h:519-538 */
    const double A[3][3] = {{v1[0], v1[1], v1[2]}, {v2[0], v2[1], v2[2]}, {v3[0], v3[1], v3[2]}};
    double r[3][3];
    r[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
    r[1][0] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
    r[2][0] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
    r[0][1] = A[2][1] * A[0][2] - A[2][2] * A[0][1];
    r[1][1] = A[2][2] * A[0][0] - A[2][0] * A[0][2];
    r[2][1] = A[2][0] * A[0][1] - A[2][1] * A[0][0];
    r[0][2] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
    r[1][2] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
    r[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
    double det = 0.0;
    det += A[0][0] * r[0][0];
    det += A[1][0] * r[0][1];
    det += A[2][0] * r[0][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) invj[3 * i + j] = r[i][j] / det;
}

/* natural coordinates of face node k in cell c: e_{slot-1}, or 0 for slot 0 (:67-75) */
static void natural(const orc_mesh* m, int64_t cell, const int64_t* fnodes, double nc[3][3]) {
    for (int k = 0; k < 3; ++k) {
        nc[k][0] = nc[k][1] = nc[k][2] = 0.0;
        for (int ki = 0; ki < 3; ++ki)
            if (fnodes[k] == m->cells[4 * cell + ki + 1]) nc[k][ki] = 1.0;
    }
}

static void face_geometry(const orc_mesh* m, int64_t f, const double* cen, double* n, double* area,
                          double nc[2][3][3]) {
    const int64_t* fn = m->faces + 3 * f;
    const int64_t c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
    const double* p0 = m->pts + 3 * fn[0];
    const double* p1 = m->pts + 3 * fn[1];
    const double* p2 = m->pts + 3 * fn[2];
    double e1[3], e2[3];
    sub3(p1, p0, e1); sub3(p2, p0, e2);
    cross3(e1, e2, n);                                   /* :46 */
    const int boundary_rule = (c1 < 0) || (m->periodic && m->periodic[f]);
    if (boundary_rule) {                                 /* :47-60 */
        const double* p3 = NULL;
        for (int k = 0; k < 4; ++k) {
            const int64_t v = m->cells[4 * c0 + k];
            if (v == fn[0] || v == fn[1] || v == fn[2]) continue;
            p3 = m->pts + 3 * v;
        }
        double v3[3], cr[3];
        sub3(p3, p0, v3);
        cross3(e1, e2, cr);
        if (dot3(cr, v3) * dot3(cr, n) > 0) { n[0] *= -1; n[1] *= -1; n[2] *= -1; }
    } else {                                             /* :61-64 */
        double d[3];
        sub3(cen + 3 * c1, cen + 3 * c0, d);
        if (dot3(n, d) < 0) { n[0] *= -1; n[1] *= -1; n[2] *= -1; }
    }
    const double len = sqrt(dot3(n, n));
    *area = len * 0.5;                                    /* :65 */
    const double len2 = sqrt(dot3(n, n));
    n[0] = n[0] / len2; n[1] = n[1] / len2; n[2] = n[2] / len2; /* :66 vec_unit */
    natural(m, c0, fn, nc[0]);
    if (c1 >= 0) natural(m, c1, m->face_nodes1 + 3 * f, nc[1]);
    else memset(nc[1], 0, sizeof(double) * 9);
}

int orc_geometry(const orc_mesh* m, double* normals, double* areas, double* natc, double* invjac,
                 double* detj, double* centroid) {
    for (int64_t c = 0; c < m->ncell; ++c) tet_geometry(m, c, invjac + 9 * c, detj + c, centroid + 3 * c);
    for (int64_t f = 0; f < m->nface; ++f) {
        double nc[2][3][3];
        face_geometry(m, f, centroid, normals + 3 * f, areas + f, nc);
        memcpy(natc + 18 * f, nc, sizeof(nc));
    }
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Euler flux, src/DG/DG_Flux/EulerPhysicalFlux.cpp:7-89                                        */
/* ------------------------------------------------------------------------------------------ */
static double positive(double v) { return v > EPS_POS ? v : EPS_POS; }  /* :59-61 */

static double pressure(const double* U, double gam) {                    /* :84-89 */
    const double rho = positive(U[0]);
    const double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho, e = U[4] / rho;
    return (gam - 1) * (rho * e - 0.5 * rho * (u * u + v * v + w * w));
}

static void phys_flux(const double* U, double gam, double F[5][3]) {     /* :8-18 */
    const double rho = positive(U[0]);
    const double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho, e = U[4] / rho;
    const double p = pressure(U, gam);
    F[0][0] = rho * u;         F[0][1] = rho * v;         F[0][2] = rho * w;
    F[1][0] = rho * u * u + p; F[1][1] = rho * v * u;     F[1][2] = rho * w * u;
    F[2][0] = rho * u * v;     F[2][1] = rho * v * v + p; F[2][2] = rho * w * v;
    F[3][0] = rho * u * w;     F[3][1] = rho * v * w;     F[3][2] = rho * w * w + p;
    F[4][0] = u * (rho * e + p); F[4][1] = v * (rho * e + p); F[4][2] = w * (rho * e + p);
}

static double wave_speed(const double* U, double gam) {                  /* :70-81 */
    const double rho = positive(U[0]);
    const double u = U[1] / rho, v = U[2] / rho, w = U[3] / rho;
    const double c = sqrt(gam * positive(pressure(U, gam) / positive(U[0])));
    return sqrt(u * u + v * v + w * w) + c;
}

static void flux_normal(const double* U, const double* n, double gam, double Fn[5]) {
    double F[5][3];
    phys_flux(U, gam, F);
    for (int k = 0; k < 5; ++k) Fn[k] = F[k][0] * n[0] + F[k][1] * n[1] + F[k][2] * n[2];
}

/* Local Lax-Friedrichs, ExplicitConvection.cpp:232-240 */
static void flux_lf(const double* UL, const double* UR, const double* n, double gam, double Fh[5]) {
    double FL[5], FR[5];
    flux_normal(UL, n, gam, FL);
    flux_normal(UR, n, gam, FR);
    const double a = wave_speed(UL, gam), b = wave_speed(UR, gam);
    const double lam = a > b ? a : b;
    for (int k = 0; k < 5; ++k) Fh[k] = 0.5 * (FL[k] + FR[k] + lam * (UL[k] - UR[k]));
}

/* Roe flux (new: the reference declares but never defines one, tests/test_flux/RiemannSolvers.h).
 * Textbook Roe averages; F = (FnL + FnR)/2 - (1/2) sum_i |lambda_i| alpha_i r_i with the
 * acoustic, entropy and shear waves of the 3D Euler equations, and Harten's entropy fix on the
 * two acoustic waves: |lambda| -> (lambda^2 + delta^2) / (2 delta) when |lambda| < delta,
 * delta = 0.1 * c_roe. Densities and pressures use the same positivity clamp as the reference
 * flux. */
static void flux_roe(const double* UL, const double* UR, const double* n, double gam, double Fh[5]) {
    double FL[5], FR[5];
    flux_normal(UL, n, gam, FL);
    flux_normal(UR, n, gam, FR);
    const double rL = positive(UL[0]), rR = positive(UR[0]);
    const double uL[3] = {UL[1] / rL, UL[2] / rL, UL[3] / rL};
    const double uR[3] = {UR[1] / rR, UR[2] / rR, UR[3] / rR};
    const double pL = pressure(UL, gam), pR = pressure(UR, gam);
    const double HL = (UL[4] + pL) / rL, HR = (UR[4] + pR) / rR;
    const double sL = sqrt(rL), sR = sqrt(rR), den = sL + sR;
    double ut[3];
    for (int i = 0; i < 3; ++i) ut[i] = (sL * uL[i] + sR * uR[i]) / den;
    const double Ht = (sL * HL + sR * HR) / den;
    const double q2 = ut[0] * ut[0] + ut[1] * ut[1] + ut[2] * ut[2];
    const double c2 = positive((gam - 1) * (Ht - 0.5 * q2));
    const double ct = sqrt(c2);
    const double rt = sL * sR;
    const double unt = ut[0] * n[0] + ut[1] * n[1] + ut[2] * n[2];
    const double dr = rR - rL, dp = pR - pL;
    double du[3];
    for (int i = 0; i < 3; ++i) du[i] = uR[i] - uL[i];
    const double dun = du[0] * n[0] + du[1] * n[1] + du[2] * n[2];
    double l1 = fabs(unt - ct), l2 = fabs(unt), l5 = fabs(unt + ct);
    const double delta = 0.1 * ct;
    if (l1 < delta) l1 = (l1 * l1 + delta * delta) / (2 * delta);
    if (l5 < delta) l5 = (l5 * l5 + delta * delta) / (2 * delta);
    const double a1 = (dp - rt * ct * dun) / (2 * c2);
    const double a5 = (dp + rt * ct * dun) / (2 * c2);
    const double a2 = dr - dp / c2;
    double D[5];
    /* acoustic - */
    D[0] = l1 * a1;
    for (int i = 0; i < 3; ++i) D[1 + i] = l1 * a1 * (ut[i] - ct * n[i]);
    D[4] = l1 * a1 * (Ht - ct * unt);
    /* acoustic + */
    D[0] += l5 * a5;
    for (int i = 0; i < 3; ++i) D[1 + i] += l5 * a5 * (ut[i] + ct * n[i]);
    D[4] += l5 * a5 * (Ht + ct * unt);
    /* entropy */
    D[0] += l2 * a2;
    for (int i = 0; i < 3; ++i) D[1 + i] += l2 * a2 * ut[i];
    D[4] += l2 * a2 * 0.5 * q2;
    /* shear */
    double uds = 0.0;
    for (int i = 0; i < 3; ++i) {
        const double sh = du[i] - dun * n[i];
        D[1 + i] += l2 * rt * sh;
        uds += ut[i] * sh;
    }
    D[4] += l2 * rt * uds;
    for (int k = 0; k < 5; ++k) Fh[k] = 0.5 * (FL[k] + FR[k]) - 0.5 * D[k];
}

static void num_flux(int kind, const double* UL, const double* UR, const double* n, double gam,
                     double Fh[5]) {
    if (kind == ORC_FLUX_ROE) flux_roe(UL, UR, n, gam, Fh);
    else flux_lf(UL, UR, n, gam, Fh);
}

int orc_numerical_flux(int kind, const double* UL, const double* UR, const double* n, double gamma,
                       double* Fh) {
    if (!UL || !UR || !n || !Fh || (kind != ORC_FLUX_LF && kind != ORC_FLUX_ROE)) return -1;
    num_flux(kind, UL, UR, n, gamma, Fh);
    return 0;
}

/* ------------------------------------------------------------------------------------------ */
/* Residual R = R_cells + R_internal + R_boundary, ExplicitConvection.cpp:136-272               */
/* ------------------------------------------------------------------------------------------ */
static void density_wave(const double* prm, const double* x, double t, double* out) {
    const double r0 = prm[0], A = prm[1], u = prm[5], v = prm[6], w = prm[7], p = prm[8], gam = prm[9];
    const double ph = 2.0 * M_PI * (prm[2] * (x[0] - u * t) + prm[3] * (x[1] - v * t) + prm[4] * (x[2] - w * t));
    const double rho = r0 + A * sin(ph);
    out[0] = rho; out[1] = rho * u; out[2] = rho * v; out[3] = rho * w;
    out[4] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
}

int orc_residual(const orc_mesh* m, int order, double gam, int flux, int qv, int qf,
                 const double* U, double* R, double t, const double* dirichlet10, int part) {
    if (order < 0 || order > 5 || qv < 0 || qv >= FVEDG_NUM_TET_RULES || qf < 0 || qf >= FVEDG_NUM_TRI_RULES)
        return -1;
    const int nb = orc_num_basis(order), B = 5 * nb;
    const int nqv = fvedg_tet_npts[qv], nqf = fvedg_tri_npts[qf];
    const double* rv = fvedg_tet_rules[qv];
    const double* rf = fvedg_tri_rules[qf];
    double* invj = malloc(sizeof(double) * 9 * m->ncell);
    double* detj = malloc(sizeof(double) * m->ncell);
    double* cen = malloc(sizeof(double) * 3 * m->ncell);
    double* phiv = malloc(sizeof(double) * nqv * nb);
    double* gradv = malloc(sizeof(double) * nqv * nb * 3);
    for (int64_t c = 0; c < m->ncell; ++c) tet_geometry(m, c, invj + 9 * c, detj + c, cen + 3 * c);
    memset(R, 0, sizeof(double) * B * m->ncell);

    /* eval_cells, :144-198 */
    if (part == 0 || part == 1) {
        for (int g = 0; g < nqv; ++g)
            basis_point(order, rv[4 * g], rv[4 * g + 1], rv[4 * g + 2], phiv + g * nb, gradv + 3 * g * nb);
        for (int64_t c = 0; c < m->ncell; ++c) {
            const double* coef = U + c * B;
            const double* J = invj + 9 * c;
            for (int g = 0; g < nqv; ++g) {
                double Ug[5] = {0, 0, 0, 0, 0}, F[5][3];
                for (int b = 0; b < nb; ++b)
                    for (int k = 0; k < 5; ++k) Ug[k] += phiv[g * nb + b] * coef[5 * b + k];
                phys_flux(Ug, gam, F);
                const double jw = rv[4 * g + 3] * detj[c];
                for (int j = 0; j < nb; ++j) {
                    const double* gr = gradv + 3 * (g * nb + j);
                    double pg[3];
                    for (int i = 0; i < 3; ++i) pg[i] = J[3 * i] * gr[0] + J[3 * i + 1] * gr[1] + J[3 * i + 2] * gr[2];
                    for (int k = 0; k < 5; ++k)
                        R[c * B + 5 * j + k] -= (F[k][0] * pg[0] + F[k][1] * pg[1] + F[k][2] * pg[2]) * jw;
                }
            }
        }
    }

    /* eval_internals :201-272 and eval_boundarys :21-128 */
    if (part == 0 || part == 2 || part == 3) {
        for (int64_t f = 0; f < m->nface; ++f) {
            const int64_t c0 = m->face_cells[2 * f], c1 = m->face_cells[2 * f + 1];
            const int interior = c1 >= 0;
            if (interior && part == 3) continue;
            if (!interior && part == 2) continue;
            const int bct = (!interior && m->bc) ? m->bc[f] : 5;
            if (!interior && bct != 0 && bct != 5) continue; /* only Dirichlet and Pseudo3DZ act */
            double n[3], area, nc[2][3][3];
            face_geometry(m, f, cen, n, &area, nc);
            for (int g = 0; g < nqf; ++g) {
                const double u = rf[3 * g], v = rf[3 * g + 1];
                const double jw = rf[3 * g + 2] * (area * 2.0);
                double xiL[3], xiR[3], phL[MAXNB], phR[MAXNB];
                for (int i = 0; i < 3; ++i) {
                    xiL[i] = nc[0][0][i] * (1 - u - v) + nc[0][1][i] * u + nc[0][2][i] * v; /* :129-134 */
                    xiR[i] = nc[1][0][i] * (1 - u - v) + nc[1][1][i] * u + nc[1][2][i] * v;
                }
                basis_point(order, xiL[0], xiL[1], xiL[2], phL, NULL);
                double UL[5] = {0, 0, 0, 0, 0}, UR[5] = {0, 0, 0, 0, 0}, Fh[5];
                for (int b = 0; b < nb; ++b)
                    for (int k = 0; k < 5; ++k) UL[k] += phL[b] * U[c0 * B + 5 * b + k];
                if (interior) {
                    basis_point(order, xiR[0], xiR[1], xiR[2], phR, NULL);
                    for (int b = 0; b < nb; ++b)
                        for (int k = 0; k < 5; ++k) UR[k] += phR[b] * U[c1 * B + 5 * b + k];
                } else if (bct == 0) { /* Dirichlet ghost 2 U_D - U_in, :47-53 */
                    const double* p0 = m->pts + 3 * m->cells[4 * c0 + 0];
                    const double* p1 = m->pts + 3 * m->cells[4 * c0 + 1];
                    const double* p2 = m->pts + 3 * m->cells[4 * c0 + 2];
                    const double* p3 = m->pts + 3 * m->cells[4 * c0 + 3];
                    double x[3], UD[5];
                    for (int i = 0; i < 3; ++i)
                        x[i] = p0[i] * (1 - xiL[0] - xiL[1] - xiL[2]) + p1[i] * xiL[0] + p2[i] * xiL[1] + p3[i] * xiL[2];
                    if (!dirichlet10) return -3;
                    density_wave(dirichlet10, x, t, UD);
                    for (int k = 0; k < 5; ++k) UR[k] = UD[k] + (UD[k] - UL[k]);
                } else { /* Pseudo3DZ mirror, :90-92 */
                    for (int k = 0; k < 5; ++k) UR[k] = UL[k];
                    UR[3] = -UL[3];
                }
                num_flux(flux, UL, UR, n, gam, Fh);
                for (int j = 0; j < nb; ++j) {
                    for (int k = 0; k < 5; ++k) {
                        R[c0 * B + 5 * j + k] += Fh[k] * phL[j] * jw;
                        if (interior) R[c1 * B + 5 * j + k] -= Fh[k] * phR[j] * jw;
                    }
                }
            }
        }
    }
    free(invj); free(detj); free(cen); free(phiv); free(gradv);
    return 0;
}

/* Diagonal mass b[e][5i+k] = detJ sum_g w_g phi_i(x_g)^2, examples/Eular1D/Sod1D/Riemann1D.cpp:108-121 */
int orc_mass(const orc_mesh* m, int order, int qv, double* mass) {
    const int nb = orc_num_basis(order), B = 5 * nb;
    const int nqv = fvedg_tet_npts[qv];
    const double* rv = fvedg_tet_rules[qv];
    double phi[MAXNB];
    double* diag = calloc(nb, sizeof(double));
    for (int g = 0; g < nqv; ++g) {
        basis_point(order, rv[4 * g], rv[4 * g + 1], rv[4 * g + 2], phi, NULL);
        for (int i = 0; i < nb; ++i) diag[i] += phi[i] * phi[i] * rv[4 * g + 3];
    }
    for (int64_t c = 0; c < m->ncell; ++c) {
        double invj[9], detj, cen[3];
        tet_geometry(m, c, invj, &detj, cen);
        for (int i = 0; i < nb; ++i)
            for (int k = 0; k < 5; ++k) mass[c * B + 5 * i + k] = diag[i] * detj;
    }
    free(diag);
    return 0;
}

/* Shu-Osher SSP-RK3 with L(U) = -R(U)/b (the drivers' convention, VortexRK.cpp:264-271). */
int orc_ssprk3(const orc_mesh* m, int order, double gam, int flux, int qv, int qf, double* U,
               const double* mass, double dt, int nsteps, double t0, const double* dirichlet10) {
    const int64_t N = (int64_t)5 * orc_num_basis(order) * m->ncell;
    double* R = malloc(sizeof(double) * N);
    double* U1 = malloc(sizeof(double) * N);
    double* U2 = malloc(sizeof(double) * N);
    double t = t0;
    int rc = 0;
    for (int s = 0; s < nsteps && rc == 0; ++s) {
        rc |= orc_residual(m, order, gam, flux, qv, qf, U, R, t, dirichlet10, 0);
        for (int64_t i = 0; i < N; ++i) U1[i] = U[i] + dt * (-R[i] / mass[i]);
        rc |= orc_residual(m, order, gam, flux, qv, qf, U1, R, t + dt, dirichlet10, 0);
        for (int64_t i = 0; i < N; ++i) U2[i] = 0.75 * U[i] + 0.25 * (U1[i] + dt * (-R[i] / mass[i]));
        rc |= orc_residual(m, order, gam, flux, qv, qf, U2, R, t + 0.5 * dt, dirichlet10, 0);
        for (int64_t i = 0; i < N; ++i) U[i] = U[i] / 3.0 + (2.0 / 3.0) * (U2[i] + dt * (-R[i] / mass[i]));
        t += dt;
    }
    free(R); free(U1); free(U2);
    return rc;
}

/* Conservation sums (new): integrals of rho, rho u, rho v, rho w, rho E over the mesh (exactly
 * c_0 * |V| because every higher mode integrates to zero against phi_0 = 1) and the kinetic
 * energy integral of rho |u|^2 / 2 with the volume rule qv. */
int orc_conservation(const orc_mesh* m, int order, int qv, double gam, const double* U, double out6[6]) {
    (void)gam;
    const int nb = orc_num_basis(order), B = 5 * nb;
    const int nqv = fvedg_tet_npts[qv];
    const double* rv = fvedg_tet_rules[qv];
    double* phiv = malloc(sizeof(double) * nqv * nb);
    for (int g = 0; g < nqv; ++g) basis_point(order, rv[4 * g], rv[4 * g + 1], rv[4 * g + 2], phiv + g * nb, NULL);
    for (int k = 0; k < 6; ++k) out6[k] = 0.0;
    for (int64_t c = 0; c < m->ncell; ++c) {
        double invj[9], detj, cen[3];
        tet_geometry(m, c, invj, &detj, cen);
        for (int k = 0; k < 5; ++k) out6[k] += U[c * B + k] * detj / 6.0;
        for (int g = 0; g < nqv; ++g) {
            double Ug[5] = {0, 0, 0, 0, 0};
            for (int b = 0; b < nb; ++b)
                for (int k = 0; k < 5; ++k) Ug[k] += phiv[g * nb + b] * U[c * B + 5 * b + k];
            const double rho = positive(Ug[0]);
            out6[5] += rv[4 * g + 3] * detj * 0.5 * (Ug[1] * Ug[1] + Ug[2] * Ug[2] + Ug[3] * Ug[3]) / rho;
        }
    }
    free(phiv);
    return 0;
}
