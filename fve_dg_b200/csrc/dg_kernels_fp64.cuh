// FP64 kernels of the explicit DG operator (the plain form).
//
// One RK stage is two launches:
//   face_flux_fp64   one thread per (face, face point): two-sided trace through the face-map
//                    tables, numerical flux, times w_g * 2A; writes Fh[face][g][5].
//                    Replaces eval_internals + eval_boundarys' point loop
//                    (ExplicitConvection.cpp:21-128, 201-272) minus the scatter.
//   element_fp64     a CTA owns E elements: volume integral (eval_cells, :144-198) plus an
//                    element-owned gather of its four faces' Fh (the atomic-free replacement of
//                    the reference's omp atomic scatter), then either stores R or applies the
//                    inverse diagonal mass and the SSP-RK3 stage combination in place.
#pragma once
#include <cstdint>

#include "dg_flux.cuh"

namespace fvedg {

struct FaceInfo {     // 48 bytes
    double n[3];      // unit normal out of cells[0]
    double jw;        // 2A (the face Jacobian of CompTriangleFace::compute_jacobian_det)
    int c0, c1;       // c1 < 0: boundary face
    int meta;         // perm0 | perm1 << 8 | bc << 16 | flags << 24 (bit 0: periodic)
    int pad;
};

struct ElemFace {     // one of the four faces of an element
    int face;         // face id
    int meta;         // perm | side << 8
};

struct StageArgs {
    const double* U;      // stage input state [ncell][5*NB]
    const double* U0;     // U^n (RK base), may alias U
    double* out;          // R (residual mode) or the new stage state
    const double* Fh;     // [nface][nqf][5]
    const double* geo;    // [ncell][10]: invJ (9, row-major) then detJ
    const ElemFace* ef;   // [ncell][4]
    const double* phi_vT; // [NB][nqv] (point index fastest)
    const double* dphi_vw;// [nqv][NB][3]
    const double* phi_f;  // [24][nqf][NB]
    const double* mass_ref; // [NB]
    int ncell, nqv, nqf;
    double gamma;
    double dt, a0, a1;    // out = a0 * U0 + a1 * (U + dt * (-R / b))
    int mode;             // 0 = store R, 1 = RK stage
    int with_volume;      // 0 skips the volume term (eval_internals / eval_boundarys only)
    const double* dt_inst;  // optional per-instance time step (ensembles), indexed by elem_inst
    const int* elem_inst;   // [ncell] instance of each element
    const double* Rv;       // RK stage: viscous residual subtracted from R (Navier-Stokes), or null
};

struct FaceArgs {
    const double* U;
    const FaceInfo* fi;
    const double* phi_fT; // [24][NB][nqf] (point index fastest: coalesced across a face's threads)
    const double* w_f;    // [nqf]
    const double* UD;     // Dirichlet data [nface][nqf][5] or nullptr
    double* Fh;
    int nface, nqf;
    double gamma;
    int flux;             // 0 = LF, 1 = Roe
    int faces_mask;       // bit 0: interior faces, bit 1: boundary faces
};

template <int NB>
__global__ void __launch_bounds__(256) face_flux_fp64(FaceArgs a) {
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t total = (int64_t)a.nface * a.nqf;
    if (tid >= total) return;
    const int f = (int)(tid / a.nqf);
    const int g = (int)(tid - (int64_t)f * a.nqf);
    const FaceInfo fi = a.fi[f];
    const int p0 = fi.meta & 0xff, p1 = (fi.meta >> 8) & 0xff, bc = (fi.meta >> 16) & 0xff;
    const bool interior = fi.c1 >= 0;
    double* out = a.Fh + ((int64_t)f * a.nqf + g) * 5;
    const bool active = interior ? (a.faces_mask & 1)
                                 : ((a.faces_mask & 2) && ((bc == 0 && a.UD != nullptr) || bc == 5));
    if (!active) {
        #pragma unroll
        for (int k = 0; k < 5; ++k) out[k] = 0.0;
        return;
    }
    const double* phL = a.phi_fT + (int64_t)p0 * NB * a.nqf + g;
    const double* cL = a.U + (int64_t)fi.c0 * (5 * NB);
    double UL[5] = {0, 0, 0, 0, 0}, UR[5] = {0, 0, 0, 0, 0};
    #pragma unroll 5
    for (int b = 0; b < NB; ++b) {
        const double ph = __ldg(phL + b * a.nqf);
        #pragma unroll
        for (int k = 0; k < 5; ++k) UL[k] = fma(ph, __ldg(cL + 5 * b + k), UL[k]);
    }
    if (interior) {
        const double* phR = a.phi_fT + (int64_t)p1 * NB * a.nqf + g;
        const double* cR = a.U + (int64_t)fi.c1 * (5 * NB);
        #pragma unroll 5
        for (int b = 0; b < NB; ++b) {
            const double ph = __ldg(phR + b * a.nqf);
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = fma(ph, __ldg(cR + 5 * b + k), UR[k]);
        }
    } else if (bc == 0) {  // Dirichlet ghost 2 U_D - U_in (ExplicitConvection.cpp:53)
        const double* ud = a.UD + ((int64_t)f * a.nqf + g) * 5;
        #pragma unroll
        for (int k = 0; k < 5; ++k) UR[k] = ud[k] + (ud[k] - UL[k]);
    } else {               // Pseudo3DZ mirror (:92)
        #pragma unroll
        for (int k = 0; k < 5; ++k) UR[k] = UL[k];
        UR[3] = -UL[3];
    }
    double Fh[5];
    if (a.flux == 1) Phys<double>::roe(UL, UR, fi.n, a.gamma, Fh);
    else Phys<double>::lax_friedrichs(UL, UR, fi.n, a.gamma, Fh);
    const double jw = __ldg(a.w_f + g) * fi.jw;
    #pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = Fh[k] * jw;
}

// E elements per CTA; dynamic shared memory holds the stage state of the tile and the
// flux-times-inverse-Jacobian values G at every volume point.
template <int NB, int E>
__global__ void __launch_bounds__(256) element_fp64(StageArgs a) {
    extern __shared__ double smem[];
    double* sC = smem;                      // [E][5*NB]
    double* sG = smem + E * 5 * NB;         // [E][nqv][15]
    const int e0 = blockIdx.x * E;
    const int ne = min(E, a.ncell - e0);
    const int nqv = a.nqv;
    // stage the tile's coefficients (contiguous, coalesced)
    {
        const double* src = a.U + (int64_t)e0 * (5 * NB);
        const int n = ne * 5 * NB;
        for (int i = threadIdx.x; i < n; i += blockDim.x) sC[i] = src[i];
    }
    __syncthreads();
    if (a.with_volume) {
        // phase 1: (element, volume point) -> G = detJ * F(U(x_g)) . J^{-T}
        for (int it = threadIdx.x; it < ne * nqv; it += blockDim.x) {
            const int e = it / nqv, g = it - e * nqv;
            const double* c = sC + e * 5 * NB;
            const double* ph = a.phi_vT + g;
            double U[5] = {0, 0, 0, 0, 0};
            #pragma unroll 5
            for (int b = 0; b < NB; ++b) {
                const double p = __ldg(ph + b * nqv);
                #pragma unroll
                for (int k = 0; k < 5; ++k) U[k] = fma(p, c[5 * b + k], U[k]);
            }
            double F[5][3];
            Phys<double>::flux(U, a.gamma - 1.0, F);
            const double* geo = a.geo + (int64_t)(e0 + e) * 10;
            double J[9];
            #pragma unroll
            for (int i = 0; i < 9; ++i) J[i] = __ldg(geo + i);
            const double dj = __ldg(geo + 9);
            double* G = sG + (e * nqv + g) * 15;
            #pragma unroll
            for (int k = 0; k < 5; ++k)
                #pragma unroll
                for (int cdir = 0; cdir < 3; ++cdir)
                    G[3 * k + cdir] = dj * (F[k][0] * J[0 * 3 + cdir] + F[k][1] * J[1 * 3 + cdir] + F[k][2] * J[2 * 3 + cdir]);
        }
        __syncthreads();
    }
    // phase 2: (element, basis function j)
    for (int it = threadIdx.x; it < ne * NB; it += blockDim.x) {
        const int e = it / NB, j = it - e * NB;
        const int ge = e0 + e;
        double acc[5] = {0, 0, 0, 0, 0};
        if (a.with_volume) {
            const double* G = sG + e * nqv * 15;
            for (int g = 0; g < nqv; ++g) {
                const double* d = a.dphi_vw + (g * NB + j) * 3;
                const double d0 = __ldg(d), d1 = __ldg(d + 1), d2 = __ldg(d + 2);
                const double* Gg = G + g * 15;
                #pragma unroll
                for (int k = 0; k < 5; ++k) acc[k] -= Gg[3 * k] * d0 + Gg[3 * k + 1] * d1 + Gg[3 * k + 2] * d2;
            }
        }
        #pragma unroll
        for (int q = 0; q < 4; ++q) {
            const ElemFace ef = a.ef[(int64_t)ge * 4 + q];
            const int perm = ef.meta & 0xff;
            const double sgn = (ef.meta >> 8) ? -1.0 : 1.0;
            const double* F = a.Fh + (int64_t)ef.face * a.nqf * 5;
            const double* ph = a.phi_f + (int64_t)perm * a.nqf * NB + j;
            double s[5] = {0, 0, 0, 0, 0};
            for (int g = 0; g < a.nqf; ++g) {
                const double p = __ldg(ph + g * NB);
                #pragma unroll
                for (int k = 0; k < 5; ++k) s[k] = fma(p, __ldg(F + 5 * g + k), s[k]);
            }
            #pragma unroll
            for (int k = 0; k < 5; ++k) acc[k] = fma(sgn, s[k], acc[k]);
        }
        double* o = a.out + (int64_t)ge * 5 * NB + 5 * j;
        if (a.mode == 0) {
            #pragma unroll
            for (int k = 0; k < 5; ++k) o[k] = acc[k];
        } else {
            const double ib = 1.0 / (__ldg(a.geo + (int64_t)ge * 10 + 9) * __ldg(a.mass_ref + j));
            const double* u0 = a.U0 + (int64_t)ge * 5 * NB + 5 * j;
            const double* us = sC + e * 5 * NB + 5 * j;
            const double dt = a.dt_inst ? __ldg(a.dt_inst + __ldg(a.elem_inst + ge)) : a.dt;
            const double* rv = a.Rv ? a.Rv + (int64_t)ge * 5 * NB + 5 * j : nullptr;
            #pragma unroll
            for (int k = 0; k < 5; ++k) {
                const double L = -(rv ? acc[k] - rv[k] : acc[k]) * ib;
                o[k] = a.a0 * u0[k] + a.a1 * (us[k] + dt * L);
            }
        }
    }
}

}  // namespace fvedg

namespace fvedg {

// ------------------------------------------------------------------------------------------------
// Fixed-size variants for the quadrature pairs in common use: the point counts are compile-time
// constants (fully unrollable loops, independent loads in flight), the coefficient blocks of a
// face tile and the face fluxes of an element tile are staged in shared memory with coalesced
// copies first, and every later read is a shared-memory broadcast.
// ------------------------------------------------------------------------------------------------

// FT faces per CTA, NQF threads per face.
template <int NB, int NQF, int FT>
__global__ void __launch_bounds__(FT * NQF) face_flux_fp64_fixed(FaceArgs a) {
    constexpr int B5 = 5 * NB;
    __shared__ double sC[2 * FT * B5];
    __shared__ int sCell[2 * FT];
    const int f0 = blockIdx.x * FT;
    const int nf = min(FT, a.nface - f0);
    for (int i = threadIdx.x; i < 2 * nf; i += blockDim.x) {
        const FaceInfo* fi = a.fi + f0 + (i >> 1);
        sCell[i] = (i & 1) ? fi->c1 : fi->c0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * nf * B5; i += blockDim.x) {
        const int s = i / B5, off = i - s * B5;
        const int cell = sCell[s];
        sC[i] = cell >= 0 ? __ldg(a.U + (int64_t)cell * B5 + off) : 0.0;
    }
    __syncthreads();
    const int fl = threadIdx.x / NQF, g = threadIdx.x - fl * NQF;
    if (fl >= nf) return;
    const int f = f0 + fl;
    const FaceInfo fi = a.fi[f];
    const int p0 = fi.meta & 0xff, p1 = (fi.meta >> 8) & 0xff, bc = (fi.meta >> 16) & 0xff;
    const bool interior = fi.c1 >= 0;
    double* out = a.Fh + ((int64_t)f * NQF + g) * 5;
    const bool active = interior ? (a.faces_mask & 1)
                                 : ((a.faces_mask & 2) && ((bc == 0 && a.UD != nullptr) || bc == 5));
    if (!active) {
        #pragma unroll
        for (int k = 0; k < 5; ++k) out[k] = 0.0;
        return;
    }
    const double* cL = sC + (2 * fl) * B5;
    const double* cR = cL + B5;
    const double* phL = a.phi_fT + p0 * NB * NQF + g;
    const double* phR = a.phi_fT + p1 * NB * NQF + g;
    double UL[5] = {0, 0, 0, 0, 0}, UR[5] = {0, 0, 0, 0, 0};
    #pragma unroll
    for (int b = 0; b < NB; ++b) {
        const double pl = __ldg(phL + b * NQF);
        #pragma unroll
        for (int k = 0; k < 5; ++k) UL[k] = fma(pl, cL[5 * b + k], UL[k]);
    }
    if (interior) {
        #pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double pr = __ldg(phR + b * NQF);
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = fma(pr, cR[5 * b + k], UR[k]);
        }
    } else if (bc == 0) {
        const double* ud = a.UD + ((int64_t)f * NQF + g) * 5;
        #pragma unroll
        for (int k = 0; k < 5; ++k) UR[k] = ud[k] + (ud[k] - UL[k]);
    } else {
        #pragma unroll
        for (int k = 0; k < 5; ++k) UR[k] = UL[k];
        UR[3] = -UL[3];
    }
    double Fh[5];
    if (a.flux == 1) Phys<double>::roe(UL, UR, fi.n, a.gamma, Fh);
    else Phys<double>::lax_friedrichs(UL, UR, fi.n, a.gamma, Fh);
    const double jw = __ldg(a.w_f + g) * fi.jw;
    #pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = Fh[k] * jw;
}

template <int NB, int NQV, int NQF, int E>
constexpr size_t element_fixed_smem() {
    return sizeof(double) * ((size_t)E * 5 * NB + (size_t)E * NQV * 15 + (size_t)E * 4 * NQF * 5) + sizeof(int) * E * 4;
}

// E elements per CTA of NT threads.
template <int NB, int NQV, int NQF, int E, int NT>
__global__ void __launch_bounds__(NT) element_fp64_fixed(StageArgs a) {
    constexpr int B5 = 5 * NB;
    extern __shared__ double smem[];
    double* sC = smem;                    // [E][5NB]
    double* sG = sC + E * B5;             // [E][NQV][15]
    double* sF = sG + E * NQV * 15;       // [E][4][NQF][5]
    int* sMeta = (int*)(sF + E * 4 * NQF * 5);  // [E][4]: perm | side << 8
    const int e0 = blockIdx.x * E;
    const int ne = min(E, a.ncell - e0);
    {
        const double* src = a.U + (int64_t)e0 * B5;
        for (int i = threadIdx.x; i < ne * B5; i += NT) sC[i] = __ldg(src + i);
    }
    for (int i = threadIdx.x; i < ne * 4; i += NT) sMeta[i] = a.ef[(int64_t)e0 * 4 + i].meta;
    for (int i = threadIdx.x; i < ne * 4 * NQF * 5; i += NT) {
        const int eq = i / (NQF * 5), off = i - eq * (NQF * 5);
        const int face = a.ef[(int64_t)e0 * 4 + eq].face;
        sF[i] = a.Fh[(int64_t)face * NQF * 5 + off];
    }
    __syncthreads();
    if (a.with_volume) {
        for (int it = threadIdx.x; it < ne * NQV; it += NT) {
            const int e = it / NQV, g = it - e * NQV;
            const double* c = sC + e * B5;
            double U[5] = {0, 0, 0, 0, 0};
            #pragma unroll
            for (int b = 0; b < NB; ++b) {
                const double p = __ldg(a.phi_vT + b * NQV + g);
                #pragma unroll
                for (int k = 0; k < 5; ++k) U[k] = fma(p, c[5 * b + k], U[k]);
            }
            double F[5][3];
            Phys<double>::flux(U, a.gamma - 1.0, F);
            const double* geo = a.geo + (int64_t)(e0 + e) * 10;
            double J[9];
            #pragma unroll
            for (int i = 0; i < 9; ++i) J[i] = __ldg(geo + i);
            const double dj = __ldg(geo + 9);
            double* G = sG + (e * NQV + g) * 15;
            #pragma unroll
            for (int k = 0; k < 5; ++k)
                #pragma unroll
                for (int d = 0; d < 3; ++d)
                    G[3 * k + d] = dj * (F[k][0] * J[d] + F[k][1] * J[3 + d] + F[k][2] * J[6 + d]);
        }
        __syncthreads();
    }
    for (int it = threadIdx.x; it < ne * NB; it += NT) {
        const int e = it / NB, j = it - e * NB;
        const int ge = e0 + e;
        double acc[5] = {0, 0, 0, 0, 0};
        if (a.with_volume) {
            const double* G = sG + e * NQV * 15;
            #pragma unroll 4
            for (int g = 0; g < NQV; ++g) {
                const double* d = a.dphi_vw + (g * NB + j) * 3;
                const double d0 = __ldg(d), d1 = __ldg(d + 1), d2 = __ldg(d + 2);
                const double* Gg = G + g * 15;
                #pragma unroll
                for (int k = 0; k < 5; ++k) acc[k] -= Gg[3 * k] * d0 + Gg[3 * k + 1] * d1 + Gg[3 * k + 2] * d2;
            }
        }
        #pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int meta = sMeta[e * 4 + q];
            const double* ph = a.phi_f + (meta & 0xff) * NQF * NB + j;
            const double* F = sF + (e * 4 + q) * NQF * 5;
            double s[5] = {0, 0, 0, 0, 0};
            #pragma unroll 4
            for (int g = 0; g < NQF; ++g) {
                const double p = __ldg(ph + g * NB);
                #pragma unroll
                for (int k = 0; k < 5; ++k) s[k] = fma(p, F[5 * g + k], s[k]);
            }
            if (meta >> 8) {
                #pragma unroll
                for (int k = 0; k < 5; ++k) acc[k] -= s[k];
            } else {
                #pragma unroll
                for (int k = 0; k < 5; ++k) acc[k] += s[k];
            }
        }
        double* o = a.out + (int64_t)ge * B5 + 5 * j;
        if (a.mode == 0) {
            #pragma unroll
            for (int k = 0; k < 5; ++k) o[k] = acc[k];
        } else {
            const double ib = 1.0 / (__ldg(a.geo + (int64_t)ge * 10 + 9) * __ldg(a.mass_ref + j));
            const double* u0 = a.U0 + (int64_t)ge * B5 + 5 * j;
            const double* us = sC + e * B5 + 5 * j;
            const double dt = a.dt_inst ? __ldg(a.dt_inst + __ldg(a.elem_inst + ge)) : a.dt;
            const double* rv = a.Rv ? a.Rv + (int64_t)ge * B5 + 5 * j : nullptr;
            #pragma unroll
            for (int k = 0; k < 5; ++k)
                o[k] = a.a0 * u0[k] + a.a1 * (us[k] + dt * (-(rv ? acc[k] - rv[k] : acc[k]) * ib));
        }
    }
}

}  // namespace fvedg
