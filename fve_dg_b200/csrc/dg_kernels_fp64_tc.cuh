// FP64 form of the explicit DG operator on the FP64 tensor cores (mma.sync m8n8k4 f64).
//
// The contractions of ExplicitConvection::eval (ExplicitConvection.cpp:144-198 and 201-272) are
// dense products that every item of a group shares one table for:
//   face traces      T[r][g] = sum_b C[r][b] phi_f[perm][g][b]          r = (face, variable)
//   volume values    V[r][g] = sum_b C[r][b] phi_v[g][b]                r = (element, variable)
//   volume integral  R[r][j] -= sum_(g,d) G[r][(g,d)] w_g dphi_j,d(x_g)
//   face integrals   R[r][j] += +-sum_g Fh[face_q][k][g] phi_f[perm_q][g][j]
// Items are grouped in threes on the host: faces with equal (perm0, perm1, kind), elements with
// equal face maps in canonical face order (the grouping of the mixed form). The 15 rows of a group
// (3 items x 5 variables, padded to 16) are the M dimension of two 8-row MMA tiles; the table is
// the B operand, shared by all rows. One warp owns one group.
//
// Two launches per RK stage, as the scalar form:
//   face_flux_tc     both traces on the tensor cores, the numerical flux (LF or Roe, FP64) at
//                    every face point, Fh[face][k][g] = F^(x_g) w_g 2A written variable-major
//   element_tc       volume values on the tensor cores; the flux G = det J F J^-T at the volume
//                    points in chunks of eight points, each chunk's slice of the volume integral
//                    on the tensor cores; the four face integrals; the inverse mass and the SSP-RK3
//                    stage update, coalesced, in memory order
// Every product and sum is FP64; the results match the scalar kernels and the reference to
// round-off (the order of the sums differs).
#pragma once
#include <cstdint>
#include <vector>

#include "dg_flux.cuh"
#include "dg_kernels_fp64.cuh"
#include "dg_kernels_mixed.cuh"

namespace fvedg {

__host__ __device__ constexpr int pad4(int x) { return (x + 3) / 4 * 4; }
// A shared-memory row stride >= n with stride % 16 == 8 doubles: the 16-byte stores of the
// accumulator pattern (two rows x four column pairs per quarter warp) touch all 32 banks once.
__host__ __device__ constexpr int ld_acc(int n) { return n % 16 == 8 ? n : n + ((8 - n % 16) + 16) % 16; }
// The smallest stride >= n with stride % 16 == 4 or 12 doubles: the A-fragment loads (four rows x
// four consecutive doubles per half warp) then touch all 32 banks once.
__host__ __device__ constexpr int ld_afrag(int n) {
    return (n % 16 == 4 || n % 16 == 12) ? n : ld_afrag(n + 1);
}

// Launch bounds. The face kernel asks for five resident 4-warp CTAs per SM up to P3 (96 registers,
// 3 % faster than the compiler's own 106-register choice on the Taylor-Green P3 mesh). The element
// kernel gives only the block size: capping it at 72 or 64 registers (7 or 8 CTAs) spilled and took
// 2.57 / 2.75 ms per launch against 1.66 ms. (An explicit minimum of one CTA per SM makes the compiler
// spend up to 255 registers on unrolled loads, so the one-argument form is the default.)
// FVEDG_TC_FACE_MINB = 0 / FVEDG_TC_ELEM_MINB select other budgets at build time.
#ifndef FVEDG_TC_FACE_MINB
#define FVEDG_TC_FACE_MINB 5
#endif
#if FVEDG_TC_FACE_MINB > 0
#define TC_FACE_BOUNDS(W, NB) __launch_bounds__(W * 32, NB <= 20 ? FVEDG_TC_FACE_MINB : 4)
#else
#define TC_FACE_BOUNDS(W, NB) __launch_bounds__(W * 32)
#endif
#ifdef FVEDG_TC_ELEM_MINB
#define TC_ELEM_BOUNDS(W, NB) __launch_bounds__(W * 32, NB <= 20 ? FVEDG_TC_ELEM_MINB : 4)
#else
#define TC_ELEM_BOUNDS(W, NB) __launch_bounds__(W * 32)
#endif

// Debug builds (-DFVEDG_TC_CHECK) check every global index against its buffer's length and every
// 16-byte shared store for alignment: the first failure is recorded in a device word and the access
// goes to index 0 instead. Product builds compile the checks away.
struct TcCheck {
    int* err;               // [2]: code of the first failing check (0 = none) and its index
    int64_t nU, nfi, nUD, nFh, ntf, ntv, ntw, ntl, njd, ncell, nout;  // buffer lengths (elements)
};
#ifdef FVEDG_TC_CHECK
__device__ __forceinline__ int64_t tc_chk(const TcCheck& c, int64_t i, int64_t n, int code) {
    if (i < 0 || i >= n) {
        if (atomicCAS(c.err, 0, code) == 0) c.err[1] = (int)i;
        return 0;
    }
    return i;
}
#define TCK(i, n, code) tc_chk(a.chk, (int64_t)(i), (int64_t)(n), code)
#define TCA(p, code) \
    do { if (((uintptr_t)(p)) & 15) { if (atomicCAS(a.chk.err, 0, code) == 0) a.chk.err[1] = (int)(((uintptr_t)(p)) & 0xffff); } } while (0)
#else
#define TCK(i, n, code) (i)
#define TCA(p, code) do {} while (0)
#endif

__device__ __forceinline__ void dmma(double d[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

struct TcTables {          // device pointers; zero padding everywhere
    const double* tf;      // [24][GP][BP]  phi_f[perm][g][b]            (trace B operand, k = b)
    const double* tv;      // [VP][BP]      phi_v[g][b]                  (volume values, k = b)
    const double* tw;      // [VP/8][JP][24] w_g dphi_{j,d}(x_g) at kk = 3 (g - 8 c) + d (chunk c)
    const double* tl;      // [24][JP][GP]  phi_f[perm][g][j]            (face integral, k = g)
    const double* inv_mass;// [NB] 1 / sum_g w_g phi_j^2
    const double* wf;      // [NQF] face weights
};

struct TcFaceArgs {
    const double* U;
    const FaceInfo* fi;
    const FaceGroup* groups;
    int ngroups;
    const double* UD;      // Dirichlet data [nface][nqf][5] or null
    double* Fh;            // [nface][5][GP]
    TcTables t;
    double gamma;
    int flux;
    int faces_mask;        // bit 0: interior faces, bit 1: boundary faces
    TcCheck chk;
};

struct TcElemArgs {
    const double* U;       // stage input
    const double* U0;      // U^n
    double* out;           // R (mode 0) or the new stage (mode 1)
    const double* Fh;
    const double* jd;      // [ncell][9] det J * J^-T, row-major (c, d)
    const double* inv_detj;// [ncell]
    const ElemGroup* groups;
    int ngroups;
    TcTables t;
    double gamma;
    int with_volume;
    int mode;
    double dt, a0, a1;     // out = a0 U0 + a1 (U + dt (-(R - Rv) / b))
    const double* dt_inst; // ensembles: per-instance dt, indexed by elem_inst
    const int* elem_inst;
    const double* Rv;      // Navier-Stokes stepping: viscous residual of the stage input, or null
    TcCheck chk;
};

// ---- faces -----------------------------------------------------------------------------------
template <int NB, int NQF>
struct alignas(16) TcFaceSmem {
    static constexpr int GP = pad8(NQF), LDT = ld_acc(GP);
    double sT[2][16][LDT];  // traces of side 0 / 1, rows (face, var), columns face point
    double sN[3][4];        // unit normal and 2A of each face
};

template <int NB, int NQF>
__device__ __forceinline__ void face_group_tc(const TcFaceArgs& a, int gi, TcFaceSmem<NB, NQF>& sm, int lane) {
    using S = TcFaceSmem<NB, NQF>;
    constexpr int GP = S::GP, BP = pad4(NB), KT = BP / 4, NT = GP / 8;
    const int gid = lane >> 2, tq = lane & 3;
    const FaceGroup grp = a.groups[gi];
    const FaceInfo f0 = a.fi[TCK(grp.f[0], a.chk.nfi, 1)];
    const int perm0 = f0.meta & 0xff, perm1 = (f0.meta >> 8) & 0xff;
    const int bc = (f0.meta >> 16) & 0xff;
    const bool interior = f0.c1 >= 0;
    const bool active = interior ? (a.faces_mask & 1)
                                 : ((a.faces_mask & 2) && ((bc == 0 && a.UD != nullptr) || bc == 5));
    if (!active) {  // faces that contribute nothing (inactive kind or boundary type): zero fluxes
        for (int i = lane; i < grp.n * 5 * NQF; i += 32) {
            const int fl = i / (5 * NQF), r = i - fl * 5 * NQF, k = r / NQF, g = r - k * NQF;
            a.Fh[TCK(((int64_t)grp.f[fl] * 5 + k) * GP + g, a.chk.nFh, 2)] = 0.0;
        }
        return;
    }
    if (lane < grp.n) {
        const FaceInfo& F = a.fi[TCK(grp.f[lane], a.chk.nfi, 3)];
        sm.sN[lane][0] = F.n[0]; sm.sN[lane][1] = F.n[1]; sm.sN[lane][2] = F.n[2]; sm.sN[lane][3] = F.jw;
    }
    const int nside = interior ? 2 : 1;
    for (int s = 0; s < nside; ++s) {
        double A[2][KT];
        #pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r = 8 * mt + gid;
            const double* row = nullptr;
            if (r < 5 * grp.n) {
                const FaceInfo& F = a.fi[TCK(grp.f[r / 5], a.chk.nfi, 4)];
                row = a.U + TCK((int64_t)(s ? F.c1 : F.c0), a.chk.ncell, 5) * (5 * NB) + r % 5;
            }
            #pragma unroll
            for (int kt = 0; kt < KT; ++kt) {
                const int b = 4 * kt + tq;
                A[mt][kt] = (row && b < NB) ? __ldg(a.U + TCK(row - a.U + 5 * b, a.chk.nU, 6)) : 0.0;
            }
        }
        const double* tb = a.t.tf + (int64_t)(s ? perm1 : perm0) * GP * BP;
        #pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            double d[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
            #pragma unroll
            for (int kt = 0; kt < KT; ++kt) {
                const double b = __ldg(a.t.tf + TCK(tb - a.t.tf + (8 * nt + gid) * BP + 4 * kt + tq, a.chk.ntf, 7));
                dmma(d[0], A[0][kt], b);
                dmma(d[1], A[1][kt], b);
            }
            #pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                TCA(&sm.sT[s][8 * mt + gid][8 * nt + 2 * tq], 8);
                *reinterpret_cast<double2*>(&sm.sT[s][8 * mt + gid][8 * nt + 2 * tq]) = make_double2(d[mt][0], d[mt][1]);
            }
        }
    }
    __syncwarp();
    for (int p = lane; p < grp.n * NQF; p += 32) {
        const int fl = p / NQF, g = p - fl * NQF;
        const int f = grp.f[fl];
        double UL[5], UR[5];
        #pragma unroll
        for (int k = 0; k < 5; ++k) UL[k] = sm.sT[0][5 * fl + k][g];
        if (interior) {
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = sm.sT[1][5 * fl + k][g];
        } else if (bc == 0) {  // Dirichlet ghost 2 U_D - U_in (ExplicitConvection.cpp:53)
            const double* ud = a.UD + TCK(((int64_t)f * NQF + g) * 5 + 4, a.chk.nUD, 9) - 4;
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = ud[k] + (ud[k] - UL[k]);
        } else {               // Pseudo3DZ mirror (:92)
            #pragma unroll
            for (int k = 0; k < 5; ++k) UR[k] = UL[k];
            UR[3] = -UL[3];
        }
        const double n[3] = {sm.sN[fl][0], sm.sN[fl][1], sm.sN[fl][2]};
        double Fh[5];
        if (a.flux == 1) roe_f64(UL, UR, n, a.gamma, Fh);
        else lax_friedrichs_f64(UL, UR, n, a.gamma, Fh);
        const double jw = __ldg(a.t.wf + g) * sm.sN[fl][3];
        double* o = a.Fh + TCK((int64_t)f * 5 * GP + g + 4 * GP, a.chk.nFh, 10) - 4 * GP;
        #pragma unroll
        for (int k = 0; k < 5; ++k) o[k * GP] = Fh[k] * jw;
    }
    __syncwarp();
}

template <int NB, int NQF, int W>
__global__ void TC_FACE_BOUNDS(W, NB) face_flux_tc(TcFaceArgs a) {
    __shared__ TcFaceSmem<NB, NQF> sm[W];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int gi = blockIdx.x * W + warp; gi < a.ngroups; gi += gridDim.x * W)
        face_group_tc<NB, NQF>(a, gi, sm[warp], lane);
}

// ---- elements ----------------------------------------------------------------------------------
template <int NB, int NQV>
struct alignas(16) TcElemSmem {
    static constexpr int VP = pad8(NQV), JP = pad8(NB);
    static constexpr int LDV = ld_acc(VP), LDG = ld_afrag(24), LDR = ld_acc(JP);
    static constexpr int VROWS = (16 * LDV >= 16 * LDR) ? 16 : (16 * LDR + LDV - 1) / LDV;
    double sV[VROWS][LDV];  // volume values, rows (element, var), columns point; the residual R[r][j] later
    double sG[16][LDG];     // -G of one chunk of eight points, columns (point, direction)
    double sJ[3][9];        // det J J^-T of each element
    double sDT[3];          // dt / det J of each element
    int sE[3];
};

template <int NB, int NQV, int NQF>
__device__ __forceinline__ void element_group_tc(const TcElemArgs& a, int gi, TcElemSmem<NB, NQV>& sm,
                                                 const double* s_inv_mass, int lane) {
    using S = TcElemSmem<NB, NQV>;
    constexpr int BP = pad4(NB), KT = BP / 4, VP = S::VP, JP = S::JP, NJ = JP / 8, GP = pad8(NQF);
    constexpr int LDG = S::LDG, LDR = S::LDR;
    const int gid = lane >> 2, tq = lane & 3;
    const ElemGroup& grp = a.groups[gi];
    const int ne = grp.n;
    if (lane < ne) {
        const int e = grp.e[lane];
        sm.sE[lane] = e;
        const double dt = a.dt_inst ? __ldg(a.dt_inst + __ldg(a.elem_inst + e)) : a.dt;
        sm.sDT[lane] = dt * __ldg(a.inv_detj + e);
    }
    if (lane < 27) {
        const int el = lane / 9;
        sm.sJ[el][lane - 9 * el] = __ldg(a.jd + TCK((int64_t)grp.e[el] * 9 + lane - 9 * el, a.chk.njd, 11));
    }
    double acc[2][NJ][2];
    #pragma unroll
    for (int mt = 0; mt < 2; ++mt)
        #pragma unroll
        for (int nt = 0; nt < NJ; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
    if (a.with_volume) {
        {   // volume values V[r][g] on the tensor cores
            double A[2][KT];
            #pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int r = 8 * mt + gid;
                const double* row = r < 5 * ne ? a.U + (int64_t)grp.e[r / 5] * (5 * NB) + r % 5 : nullptr;
                #pragma unroll
                for (int kt = 0; kt < KT; ++kt) {
                    const int b = 4 * kt + tq;
                    A[mt][kt] = (row && b < NB) ? __ldg(a.U + TCK(row - a.U + 5 * b, a.chk.nU, 12)) : 0.0;
                }
            }
            #pragma unroll
            for (int nt = 0; nt < VP / 8; ++nt) {
                double d[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
                #pragma unroll
                for (int kt = 0; kt < KT; ++kt) {
                    const double b = __ldg(a.t.tv + TCK((8 * nt + gid) * BP + 4 * kt + tq, a.chk.ntv, 13));
                    dmma(d[0], A[0][kt], b);
                    dmma(d[1], A[1][kt], b);
                }
                #pragma unroll
                for (int mt = 0; mt < 2; ++mt) {
                    TCA(&sm.sV[8 * mt + gid][8 * nt + 2 * tq], 14);
                    *reinterpret_cast<double2*>(&sm.sV[8 * mt + gid][8 * nt + 2 * tq]) = make_double2(d[mt][0], d[mt][1]);
                }
            }
        }
        __syncwarp();
        const double gm1 = a.gamma - 1.0;
        #pragma unroll 1
        for (int c = 0; c < VP / 8; ++c) {
            // -G = -(det J F J^-T) at the chunk's points: lane = (element, point), 24 of 32 lanes;
            // with v = u (det J J^-T): G_0d = rho v_d, G_(1+i)d = rho u_i v_d + p (det J J^-T)_id,
            // G_4d = (E + p) v_d (the rows of EulerPhysicalFlux.cpp:8-18 contracted with det J J^-T)
            if (lane < 24) {
                const int el = lane >> 3, g = 8 * c + (lane & 7);
                double* Gr = &sm.sG[5 * el][3 * (lane & 7)];
                if (el < ne && g < NQV) {
                    double U[5];
                    #pragma unroll
                    for (int k = 0; k < 5; ++k) U[k] = sm.sV[5 * el + k][g];
                    const double rho = Phys<double>::positive(U[0]);
                    const double ir = 1.0 / rho;
                    const double u[3] = {U[1] * ir, U[2] * ir, U[3] * ir};
                    const double p = gm1 * (U[4] - 0.5 * rho * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
                    const double h = U[4] + p;
                    const double* J = sm.sJ[el];
                    #pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        const double v = u[0] * J[d] + u[1] * J[3 + d] + u[2] * J[6 + d];
                        Gr[d] = -rho * v;
                        #pragma unroll
                        for (int i = 0; i < 3; ++i) Gr[(1 + i) * LDG + d] = -(rho * u[i] * v + p * J[3 * i + d]);
                        Gr[4 * LDG + d] = -h * v;
                    }
                } else {
                    #pragma unroll
                    for (int k = 0; k < 5; ++k)
                        #pragma unroll
                        for (int d = 0; d < 3; ++d) Gr[k * LDG + d] = 0.0;
                }
            }
            __syncwarp();
            // acc[r][j] += (-G)[r][kk] W[kk][j] with W = w dphi: the volume term enters R with a
            // minus (ExplicitConvection.cpp:190-196)
            const double* tw = a.t.tw + (int64_t)c * JP * 24;
            #pragma unroll
            for (int kt = 0; kt < 6; ++kt) {
                const double a0 = sm.sG[gid][4 * kt + tq];
                const double a1 = sm.sG[8 + gid][4 * kt + tq];
                #pragma unroll
                for (int nt = 0; nt < NJ; ++nt) {
                    const double b = __ldg(a.t.tw + TCK(tw - a.t.tw + (8 * nt + gid) * 24 + 4 * kt + tq, a.chk.ntw, 15));
                    dmma(acc[0][nt], a0, b);
                    dmma(acc[1][nt], a1, b);
                }
            }
            __syncwarp();
        }
    }
    // face integrals: acc[r][j] += +-sum_g Fh[face_q(r)][k(r)][g] phi_f[perm_q][g][j]; the group shares
    // the face maps and the sides (+ on cells[0], - on cells[1], ExplicitConvection.cpp:247-266)
    const double* rowp[2][4];
    #pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int r = 8 * mt + gid;
        #pragma unroll
        for (int q = 0; q < 4; ++q)
            rowp[mt][q] = r < 5 * ne ? a.Fh + ((int64_t)grp.face[r / 5][q] * 5 + r % 5) * GP : nullptr;
    }
    #pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int meta = grp.meta[q];
        const double sgn = (meta >> 8) ? -1.0 : 1.0;
        const double* tl = a.t.tl + (int64_t)(meta & 0xff) * JP * GP;
        #pragma unroll
        for (int kt = 0; kt < GP / 4; ++kt) {
            const double a0 = rowp[0][q] ? sgn * __ldg(a.Fh + TCK(rowp[0][q] - a.Fh + 4 * kt + tq, a.chk.nFh, 16)) : 0.0;
            const double a1 = rowp[1][q] ? sgn * __ldg(a.Fh + TCK(rowp[1][q] - a.Fh + 4 * kt + tq, a.chk.nFh, 17)) : 0.0;
            #pragma unroll
            for (int nt = 0; nt < NJ; ++nt) {
                const double b = __ldg(a.t.tl + TCK(tl - a.t.tl + (8 * nt + gid) * GP + 4 * kt + tq, a.chk.ntl, 18));
                dmma(acc[0][nt], a0, b);
                dmma(acc[1][nt], a1, b);
            }
        }
    }
    // R[r][j] to shared memory (over the volume values), then the update in memory order
    double* sR = &sm.sV[0][0];
    #pragma unroll
    for (int mt = 0; mt < 2; ++mt)
        #pragma unroll
        for (int nt = 0; nt < NJ; ++nt) {
            TCA(sR + (8 * mt + gid) * LDR + 8 * nt + 2 * tq, 19);
            *reinterpret_cast<double2*>(sR + (8 * mt + gid) * LDR + 8 * nt + 2 * tq) = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
        }
    __syncwarp();
    for (int i = lane; i < ne * 5 * NB; i += 32) {
        const int el = i / (5 * NB), rr = i - el * (5 * NB), j = rr / 5, k = rr - 5 * j;
        const int64_t idx = TCK((int64_t)sm.sE[el] * (5 * NB) + rr, a.chk.nout, 20);
        double R = sR[(5 * el + k) * LDR + j];
        if (a.mode == 0) {
            a.out[idx] = R;
        } else {
            if (a.Rv) R -= __ldg(a.Rv + idx);
            const double u0 = a.a0 != 0.0 ? a.a0 * __ldg(a.U0 + idx) : 0.0;
            a.out[idx] = u0 + a.a1 * (__ldg(a.U + idx) - sm.sDT[el] * s_inv_mass[j] * R);
        }
    }
    __syncwarp();
}

template <int NB, int NQV, int NQF, int W>
__global__ void TC_ELEM_BOUNDS(W, NB) element_tc(TcElemArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double s_inv_mass[NB];
    for (int j = threadIdx.x; j < NB; j += blockDim.x) s_inv_mass[j] = a.t.inv_mass[j];
    __syncthreads();
    auto& sm = reinterpret_cast<TcElemSmem<NB, NQV>*>(smem_raw)[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    for (int gi = blockIdx.x * W + (threadIdx.x >> 5); gi < a.ngroups; gi += gridDim.x * W)
        element_group_tc<NB, NQV, NQF>(a, gi, sm, s_inv_mass, lane);
}

// ---- host side ---------------------------------------------------------------------------------
struct TcData {
    bool ready = false;
    int order = 0, qv = 0, qf = 0;
    int nfgroups = 0, negroups = 0, nfgroups_inner = 0;
    int sms = 148;
    std::vector<void*> bufs;
    TcTables t{};
    const FaceGroup* fgroups = nullptr;
    const ElemGroup* egroups = nullptr;
    const double* jd = nullptr;
    const double* inv_detj = nullptr;
    double* Fh = nullptr;  // [nface][5][GP]
    TcCheck chk{};         // buffer lengths for checked builds (err allocated only there)
};

// (order, tet rule, tri rule) combinations with tensor-core FP64 kernels: X(P, QV, QF, NB, NQV, NQF)
#define FVEDG_TC_COMBOS(X)      \
    X(1, 0, 1, 4, 4, 6)         \
    X(1, 0, 0, 4, 4, 4)         \
    X(1, 0, 2, 4, 4, 7)         \
    X(1, 2, 2, 4, 15, 7)        \
    X(2, 1, 2, 10, 11, 7)       \
    X(2, 1, 3, 10, 11, 24)      \
    X(2, 2, 3, 10, 15, 24)      \
    X(3, 3, 3, 20, 23, 24)      \
    X(3, 4, 3, 20, 31, 24)      \
    X(4, 5, 3, 35, 44, 24)      \
    X(4, 6, 3, 35, 57, 24)

inline bool tc_supported(int order, int qv, int qf) {
#define X(P, QV, QF, NB, NQV, NQF) \
    if (order == P && qv == QV && qf == QF) return true;
    FVEDG_TC_COMBOS(X)
#undef X
    return false;
}

template <typename T>
inline int tc_upload(TcData& m, const T** dst, const std::vector<T>& v) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * std::max<size_t>(v.size(), 1)) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    if (!v.empty() && cudaMemcpy(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return DG_E_CUDA;
    *dst = (const T*)p;
    return DG_OK;
}

inline int init_tc(TcData& m, const Tables& tab, const std::vector<double>& hgeo, const std::vector<FaceInfo>& hfi,
                   const std::vector<ElemFace>& hef, int64_t ncell, int64_t nowned, int64_t nface, int qv, int qf) {
    if (!tc_supported(tab.order, qv, qf)) return DG_E_ARG;
    const int NB = tab.nb, NQV = tab.nqv, NQF = tab.nqf;
    const int BP = pad4(NB), GP = pad8(NQF), VP = pad8(NQV), JP = pad8(NB);
    m.order = tab.order; m.qv = qv; m.qf = qf;
    std::vector<double> tf((size_t)24 * GP * BP, 0.0), tl((size_t)24 * JP * GP, 0.0);
    std::vector<double> tv((size_t)VP * BP, 0.0), tw((size_t)(VP / 8) * JP * 24, 0.0);
    for (int p = 0; p < 24; ++p)
        for (int g = 0; g < NQF; ++g)
            for (int b = 0; b < NB; ++b) {
                const double v = tab.phi_f[((size_t)p * NQF + g) * NB + b];
                tf[((size_t)p * GP + g) * BP + b] = v;
                tl[((size_t)p * JP + b) * GP + g] = v;
            }
    for (int g = 0; g < NQV; ++g)
        for (int b = 0; b < NB; ++b) tv[(size_t)g * BP + b] = tab.phi_v[(size_t)g * NB + b];
    // chunk c = g / 8, column kk = 3 (g % 8) + d
    for (int g = 0; g < NQV; ++g)
        for (int j = 0; j < NB; ++j)
            for (int d = 0; d < 3; ++d)
                tw[((size_t)(g / 8) * JP + j) * 24 + 3 * (g % 8) + d] = tab.dphi_vw[((size_t)g * NB + j) * 3 + d];
    std::vector<double> inv_mass(NB), jd(9 * ncell), inv_detj(ncell);
    for (int j = 0; j < NB; ++j) inv_mass[j] = 1.0 / tab.mass_ref[j];
    for (int64_t e = 0; e < ncell; ++e) {
        const double dj = hgeo[10 * e + 9];
        for (int i = 0; i < 9; ++i) jd[9 * e + i] = dj * hgeo[10 * e + i];
        inv_detj[e] = 1.0 / dj;
    }
    int rc;
    if ((rc = tc_upload(m, &m.t.tf, tf)) || (rc = tc_upload(m, &m.t.tl, tl)) || (rc = tc_upload(m, &m.t.tv, tv)) ||
        (rc = tc_upload(m, &m.t.tw, tw)) || (rc = tc_upload(m, &m.t.inv_mass, inv_mass)) ||
        (rc = tc_upload(m, &m.t.wf, tab.w_f)) || (rc = tc_upload(m, &m.jd, jd)) ||
        (rc = tc_upload(m, &m.inv_detj, inv_detj)))
        return rc;
    std::vector<FaceGroup> fg;
    std::vector<ElemGroup> eg;
    build_groups(hfi, hef, nowned, fg, eg, &m.nfgroups_inner);
    m.nfgroups = (int)fg.size();
    m.negroups = (int)eg.size();
    if ((rc = tc_upload(m, &m.fgroups, fg)) || (rc = tc_upload(m, &m.egroups, eg))) return rc;
    // face fluxes; the padding columns g >= NQF stay zero (no kernel writes them)
    void* p = nullptr;
    const size_t nfh = (size_t)nface * 5 * GP;
    if (cudaMalloc(&p, sizeof(double) * std::max<size_t>(nfh, 1)) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    if (cudaMemset(p, 0, sizeof(double) * std::max<size_t>(nfh, 1)) != cudaSuccess) return DG_E_CUDA;
    m.Fh = (double*)p;
    m.chk.nU = m.chk.nout = ncell * 5 * NB;
    m.chk.nfi = nface;
    m.chk.nUD = nface * NQF * 5;
    m.chk.nFh = (int64_t)nfh;
    m.chk.ntf = (int64_t)tf.size(); m.chk.ntv = (int64_t)tv.size(); m.chk.ntw = (int64_t)tw.size();
    m.chk.ntl = (int64_t)tl.size(); m.chk.njd = (int64_t)jd.size(); m.chk.ncell = ncell;
#ifdef FVEDG_TC_CHECK
    if (cudaMalloc(&p, 2 * sizeof(int)) != cudaSuccess) return DG_E_NOMEM;
    m.bufs.push_back(p);
    if (cudaMemset(p, 0, 2 * sizeof(int)) != cudaSuccess) return DG_E_CUDA;
    m.chk.err = (int*)p;
#endif
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&m.sms, cudaDevAttrMultiProcessorCount, dev);
    m.ready = true;
    return DG_OK;
}

inline void free_tc(TcData& m) {
    for (void* p : m.bufs) cudaFree(p);
    m.bufs.clear();
    m.ready = false;
}

template <int NB, int NQV, int NQF>
inline int tc_launch(TcData& m, int which, const TcFaceArgs& fa, const TcElemArgs& ea, cudaStream_t s) {
    constexpr int W = 4;
    if (which == 0) {
        const int g = (int)std::min<int64_t>((fa.ngroups + W - 1) / W, (int64_t)m.sms * 32);
        if (g > 0) face_flux_tc<NB, NQF, W><<<g, W * 32, 0, s>>>(fa);
    } else {
        constexpr size_t smem = sizeof(TcElemSmem<NB, NQV>) * W;
        static unsigned long long done = 0;
        int rc = ensure_smem(element_tc<NB, NQV, NQF, W>, smem, done);
        if (rc) return rc;
        const int g = (int)std::min<int64_t>((ea.ngroups + W - 1) / W, (int64_t)m.sms * 32);
        if (g > 0) element_tc<NB, NQV, NQF, W><<<g, W * 32, smem, s>>>(ea);
    }
    return cuda_status(cudaGetLastError());
}

inline int tc_kernel(TcData& m, int which, const TcFaceArgs& fa, const TcElemArgs& ea, cudaStream_t s) {
    if (!m.ready) return DG_E_ARG;
#define X(P, QV, QF, NB, NQV, NQF) \
    if (m.order == P && m.qv == QV && m.qf == QF) return tc_launch<NB, NQV, NQF>(m, which, fa, ea, s);
    FVEDG_TC_COMBOS(X)
#undef X
    return DG_E_ARG;
}

}  // namespace fvedg
