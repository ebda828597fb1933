// Host side: modal basis, quadrature rule access and the constant tables the kernels read.
#include <cmath>

#include "dg_internal.h"
#include "quad_tables.inc"

namespace fvedg {

int auto_tet_rule(int order) {  // AutoQuadSelectorTet.h:2-30
    switch (order) {
        case 0: case 1: case 2: return DG_TET_D5P15;
        case 3: return DG_TET_D7P31;
        case 4: return DG_TET_D9P57;
        case 5: return DG_TET_D11P94;
    }
    return -1;
}
int auto_tri_rule(int order) {  // AutoQuadSelectorTri.h:1-27
    switch (order) {
        case 0: case 1: return DG_TRI_D4P7;
        case 2: case 3: case 4: return DG_TRI_D10P24;
        case 5: return DG_TRI_D13P36;
    }
    return -1;
}
int tet_rule_npts(int id) { return (id >= 0 && id < FVEDG_NUM_TET_RULES) ? fvedg_tet_npts[id] : 0; }
int tri_rule_npts(int id) { return (id >= 0 && id < FVEDG_NUM_TRI_RULES) ? fvedg_tri_npts[id] : 0; }
const double* tet_rule(int id) { return (id >= 0 && id < FVEDG_NUM_TET_RULES) ? fvedg_tet_rules[id] : nullptr; }
const double* tri_rule(int id) { return (id >= 0 && id < FVEDG_NUM_TRI_RULES) ? fvedg_tri_rules[id] : nullptr; }

namespace {
// Homogenised Jacobi polynomials J_n(y, s) = s^n P_n^{(a,0)}(2y/s - 1), n = 0..N, with their
// y- and s-derivatives, from the standard three-term recurrence in t = 2y/s - 1.
struct Jacobi {
    double v[kMaxOrder + 2], dy[kMaxOrder + 2], ds[kMaxOrder + 2];
    Jacobi(int N, double a, double y, double s) {
        v[0] = 1.0; dy[0] = 0.0; ds[0] = 0.0;
        if (N >= 1) { v[1] = (a + 2.0) * y - s; dy[1] = a + 2.0; ds[1] = -1.0; }
        for (int n = 1; n < N; ++n) {
            const double k = 2.0 * (n + 1) * (n + a + 1) * (2 * n + a);
            const double A = (2 * n + a + 1) * (2 * n + a + 2) * (2 * n + a) / k;  // coefficient of t
            const double B = (2 * n + a + 1) * a * a / k;
            const double C = 2.0 * n * (n + a) * (2 * n + a + 2) / k;
            const double l = A * (2.0 * y - s) + B * s;
            v[n + 1] = l * v[n] - C * s * s * v[n - 1];
            dy[n + 1] = 2.0 * A * v[n] + l * dy[n] - C * s * s * dy[n - 1];
            ds[n + 1] = (B - A) * v[n] + l * ds[n] - 2.0 * C * s * v[n - 1] - C * s * s * ds[n - 1];
        }
    }
};
}  // namespace

// psi_{pqr}(x,y,z) = P_p^{(2q+2r+2,0)}(2x-1) (1-x)^q P_q^{(2r+1,0)}(2y/(1-x)-1)
//                    (1-x-y)^r P_r^{(0,0)}(2z/(1-x-y)-1),
// ordered by total degree n, then r ascending, then q ascending (p = n - q - r): the ordering
// and scaling of DGBasis<0..> in include/DG/DG_Basis/DG_Basis_Func.h.
void basis_eval(int order, double x, double y, double z, double* phi, double* grad) {
    int idx = 0;
    for (int n = 0; n <= order; ++n)
        for (int r = 0; r <= n; ++r)
            for (int q = 0; q <= n - r; ++q, ++idx) {
                const int p = n - q - r;
                const Jacobi X(p, 2.0 * (q + r) + 2.0, x, 1.0);
                const Jacobi Y(q, 2.0 * r + 1.0, y, 1.0 - x);
                const Jacobi Z(r, 0.0, z, 1.0 - x - y);
                const double fx = X.v[p], fy = Y.v[q], fz = Z.v[r];
                if (phi) phi[idx] = fx * fy * fz;
                if (grad) {
                    grad[3 * idx + 0] = X.dy[p] * fy * fz - fx * Y.ds[q] * fz - fx * fy * Z.ds[r];
                    grad[3 * idx + 1] = fx * Y.dy[q] * fz - fx * fy * Z.ds[r];
                    grad[3 * idx + 2] = fx * fy * Z.dy[r];
                }
            }
}

void build_tables(int order, int qv, int qf, Tables* t) {
    const int nb = num_basis(order);
    const int nqv = tet_rule_npts(qv), nqf = tri_rule_npts(qf);
    const double* rv = tet_rule(qv);
    const double* rf = tri_rule(qf);
    t->order = order;
    t->nb = nb;
    t->nqv = nqv;
    t->nqf = nqf;
    t->phi_v.assign(nqv * nb, 0.0);
    t->dphi_vw.assign(nqv * nb * 3, 0.0);
    t->dphi_v.assign(nqv * nb * 3, 0.0);
    t->w_v.assign(nqv, 0.0);
    t->mass_ref.assign(nb, 0.0);
    double phi[64], grad[192];
    for (int g = 0; g < nqv; ++g) {
        basis_eval(order, rv[4 * g], rv[4 * g + 1], rv[4 * g + 2], phi, grad);
        const double w = rv[4 * g + 3];
        t->w_v[g] = w;
        for (int b = 0; b < nb; ++b) {
            t->phi_v[g * nb + b] = phi[b];
            for (int c = 0; c < 3; ++c) {
                t->dphi_vw[(g * nb + b) * 3 + c] = grad[3 * b + c] * w;
                t->dphi_v[(g * nb + b) * 3 + c] = grad[3 * b + c];
            }
            t->mass_ref[b] += phi[b] * phi[b] * w;
        }
    }
    // Face point of face map p at face parameters (u, v): xi = V[s0](1-u-v) + V[s1] u + V[s2] v
    // with V[0] = 0 and V[i] = e_{i-1}; the same point as ExplicitConvection.cpp:129-134.
    t->phi_f.assign((size_t)kNumPerms * nqf * nb, 0.0);
    t->dphi_f.assign((size_t)kNumPerms * nqf * nb * 3, 0.0);
    t->w_f.assign(nqf, 0.0);
    for (int g = 0; g < nqf; ++g) t->w_f[g] = rf[3 * g + 2];
    for (int p = 0; p < kNumPerms; ++p)
        for (int g = 0; g < nqf; ++g) {
            const double u = rf[3 * g], v = rf[3 * g + 1];
            const double coef[3] = {1 - u - v, u, v};
            double xi[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < 3; ++k) {
                const int s = kPermSlots[p][k];
                if (s > 0) xi[s - 1] = coef[k];
            }
            basis_eval(order, xi[0], xi[1], xi[2], phi, grad);
            for (int b = 0; b < nb; ++b) {
                t->phi_f[((size_t)p * nqf + g) * nb + b] = phi[b];
                for (int c = 0; c < 3; ++c) t->dphi_f[(((size_t)p * nqf + g) * nb + b) * 3 + c] = grad[3 * b + c];
            }
        }
    t->phi_vT.assign(nb * nqv, 0.0);
    for (int g = 0; g < nqv; ++g)
        for (int b = 0; b < nb; ++b) t->phi_vT[b * nqv + g] = t->phi_v[g * nb + b];
    t->phi_fT.assign(t->phi_f.size(), 0.0);
    for (int p = 0; p < kNumPerms; ++p)
        for (int g = 0; g < nqf; ++g)
            for (int b = 0; b < nb; ++b)
                t->phi_fT[((size_t)p * nb + b) * nqf + g] = t->phi_f[((size_t)p * nqf + g) * nb + b];
}

}  // namespace fvedg

using namespace fvedg;

extern "C" int dg_basis(int order, int npts, const double* xyz, double* phi, double* grad) {
    if (order < 0 || order > kMaxOrder || npts < 0 || (npts > 0 && !xyz)) return DG_E_ARG;
    const int nb = num_basis(order);
    for (int g = 0; g < npts; ++g)
        basis_eval(order, xyz[3 * g], xyz[3 * g + 1], xyz[3 * g + 2], phi ? phi + (size_t)g * nb : nullptr,
                   grad ? grad + (size_t)g * nb * 3 : nullptr);
    return DG_OK;
}

extern "C" int dg_quad_rule(int kind, int id, double* pts, double* w) {
    const int n = kind == 0 ? tet_rule_npts(id) : tri_rule_npts(id);
    if (n <= 0) return DG_E_ARG;
    const int dim = kind == 0 ? 3 : 2;
    const double* r = kind == 0 ? tet_rule(id) : tri_rule(id);
    for (int g = 0; g < n; ++g) {
        for (int c = 0; c < dim; ++c)
            if (pts) pts[dim * g + c] = r[(dim + 1) * g + c];
        if (w) w[g] = r[(dim + 1) * g + dim];
    }
    return n;
}

extern "C" int dg_auto_rules(int order, int* quad_vol, int* quad_face) {
    if (order < 0 || order > kMaxOrder) return DG_E_ARG;
    if (quad_vol) *quad_vol = auto_tet_rule(order);
    if (quad_face) *quad_face = auto_tri_rule(order);
    return DG_OK;
}
