// C ABI of the B200 explicit DG operator: context management, uploads, launches, RK loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <mutex>
#include <string>
#include <vector>

#include "dg_internal.h"
#include "dg_kernels_fp64.cuh"
#include "dg_kernels_mixed.cuh"
#include "dg_kernels_fp64_tc.cuh"
#include "dg_persistent.cuh"
#include "dg_limiter.cuh"
#include "dg_viscous.cuh"
#include "dg_reduce.cuh"

using namespace fvedg;

namespace {
std::atomic<int64_t> g_launches{0};

inline int cuda_ok(cudaError_t e) { return cuda_status(e); }
#define DG_CUDA(x)                                   \
    do {                                             \
        cudaError_t e_ = (x);                        \
        if (e_ != cudaSuccess) return cuda_status(e_); \
    } while (0)

template <typename T>
int dev_alloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return DG_OK;
    return cudaMalloc((void**)p, n * sizeof(T)) == cudaSuccess ? DG_OK : DG_E_NOMEM;
}
template <typename T>
int upload(T** p, const std::vector<T>& v) {
    int rc = dev_alloc(p, v.size());
    if (rc) return rc;
    if (v.empty()) return DG_OK;
    return cuda_ok(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
}
}  // namespace

struct dg_ctx {
    dg_config cfg{};
    int qv = 0, qf = 0;
    int64_t ncell = 0, nface = 0;
    Tables tab;
    cudaStream_t stream = nullptr;
    // device data
    double* d_geo = nullptr;       // [ncell][10]
    FaceInfo* d_fi = nullptr;      // [nface]
    ElemFace* d_ef = nullptr;      // [ncell][4]
    double* d_phi_v = nullptr;
    double* d_dphi_vw = nullptr;
    double* d_w_v = nullptr;
    double* d_phi_f = nullptr;
    double* d_phi_fT = nullptr;
    double* d_phi_vT = nullptr;
    double* d_w_f = nullptr;
    double* d_mass_ref = nullptr;
    double* d_UD = nullptr;        // Dirichlet data
    double* d_Fh = nullptr;        // [nface][nqf][5] FP64 face fluxes
    double* d_Un = nullptr;        // state U^n
    double* d_Ua = nullptr;        // stage buffers
    double* d_Ub = nullptr;
    double* d_io = nullptr;        // residual input staging
    double* d_R = nullptr;         // residual output staging
    double* d_red = nullptr;       // reduction partials
    double* d_red_out = nullptr;
    MixedData mixed;               // mixed-precision form buffers
    TcData tc;                     // FP64 form on the FP64 tensor cores (the configurations' rules)
    bool have_state = false;
    bool has_dirichlet = false;    // some boundary face is Dirichlet: U_D must be set first
    cudaGraphExec_t graph = nullptr;
    double graph_dt = 0.0;
    // optional per-launch event timing (dg_ssprk3_timed)
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    std::vector<int> ev_cls;
    size_t ev_used = 0;
    // persistent schedule (mixed form): queue state and tile parameters (chosen by dg_autotune)
    QueueState* d_queue = nullptr;
    PersistentParams pp;
    QueueSchedule qs;
    // limiter: per-cell statistics [ncell][10] and a staging buffer for host calls
    double* d_lim_bnd = nullptr;
    double* d_lim_prev = nullptr;
    double* d_lim_stats[3] = {nullptr, nullptr, nullptr};  // limiter statistics of state buffer 0, 1, 2
    int* d_lim_nbr = nullptr;                              // [ncell][4] face neighbours (self across a boundary)
    bool lim_valid = false;                                // d_lim_stats[0] describes U^n's owned cells
    // viscous operator: reference gradients at the volume and face points, cell size h
    double* d_dphi_v = nullptr;
    double* d_dphi_f = nullptr;
    double* d_h = nullptr;
    // viscous operator, allocated by its first call: transposed basis tables, per-face-point fluxes
    double* d_visc_phiT_v = nullptr;
    double* d_visc_dphiT_v = nullptr;
    double* d_visc_Pt = nullptr;
    double* d_visc_Av = nullptr;
    double* d_visc_Pf = nullptr;
    double* d_visc_vf = nullptr;
    double* d_Rv = nullptr;  // viscous residual of the current stage input (dg_config.mu > 0)
    int sms = 148;
    // ensembles: instance element offsets, per-instance dt on the device, instance of each element
    int ninst = 1;
    int64_t nowned = 0;  // cells [nowned, ncell) are ghosts (dg_mesh_desc.nghost)
    std::vector<int64_t> inst_off;
    double* d_dt_inst = nullptr;
    int* d_elem_inst = nullptr;
};

namespace {

size_t elem_smem_bytes(int nb, int e, int nqv) { return sizeof(double) * (size_t)e * (5 * nb + 15 * nqv); }

template <int NB, int E>
int launch_element(const StageArgs& a, cudaStream_t s) {
    const size_t smem = elem_smem_bytes(NB, E, a.nqv);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(element_fp64<NB, E>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
            return DG_E_CUDA;
        attr = true;
    }
    const int grid = (a.ncell + E - 1) / E;
    element_fp64<NB, E><<<grid, 128, smem, s>>>(a);
    ++g_launches;
    return cuda_ok(cudaGetLastError());
}

template <int NB>
int launch_face(const FaceArgs& a, cudaStream_t s) {
    const int64_t total = (int64_t)a.nface * a.nqf;
    const int grid = (int)((total + 255) / 256);
    face_flux_fp64<NB><<<grid, 256, 0, s>>>(a);
    ++g_launches;
    return cuda_ok(cudaGetLastError());
}

// Fixed-size kernels for the (order, tet rule, tri rule) combinations in common use; any other
// combination runs the runtime-size kernels above.
template <int NB, int NQV, int NQF, int E, int NT>
int launch_element_fixed(const StageArgs& a, cudaStream_t s) {
    constexpr size_t smem = element_fixed_smem<NB, NQV, NQF, E>();
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(element_fp64_fixed<NB, NQV, NQF, E, NT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return DG_E_CUDA;
        attr = true;
    }
    const int grid = (a.ncell + E - 1) / E;
    element_fp64_fixed<NB, NQV, NQF, E, NT><<<grid, NT, smem, s>>>(a);
    ++g_launches;
    return cuda_ok(cudaGetLastError());
}

template <int NB, int NQF, int FT>
int launch_face_fixed(const FaceArgs& a, cudaStream_t s) {
    const int grid = (a.nface + FT - 1) / FT;
    face_flux_fp64_fixed<NB, NQF, FT><<<grid, FT * NQF, 0, s>>>(a);
    ++g_launches;
    return cuda_ok(cudaGetLastError());
}

// X(order, qv, qf, NB, NQV, NQF, E, NT, FT)
#define FVEDG_FIXED_COMBOS(X)                    \
    X(1, 0, 1, 4, 4, 6, 16, 128, 32)             \
    X(1, 0, 0, 4, 4, 4, 16, 128, 32)             \
    X(1, 0, 2, 4, 4, 7, 16, 128, 32)             \
    X(1, 2, 2, 4, 15, 7, 16, 128, 32)            \
    X(2, 1, 2, 10, 11, 7, 16, 256, 32)           \
    X(2, 1, 3, 10, 11, 24, 8, 128, 8)            \
    X(2, 2, 3, 10, 15, 24, 8, 128, 8)            \
    X(3, 3, 3, 20, 23, 24, 8, 192, 8)            \
    X(3, 4, 3, 20, 31, 24, 8, 192, 8)            \
    X(4, 5, 3, 35, 44, 24, 4, 192, 8)            \
    X(4, 6, 3, 35, 57, 24, 4, 192, 8)

int dispatch_face(int order, int qv, int qf, const FaceArgs& a, cudaStream_t s) {
#define X(P, QV, QF, NB, NQV, NQF, E, NT, FT) \
    if (order == P && qv == QV && qf == QF) return launch_face_fixed<NB, NQF, FT>(a, s);
    FVEDG_FIXED_COMBOS(X)
#undef X
    switch (order) {
        case 0: return launch_face<1>(a, s);
        case 1: return launch_face<4>(a, s);
        case 2: return launch_face<10>(a, s);
        case 3: return launch_face<20>(a, s);
        case 4: return launch_face<35>(a, s);
        case 5: return launch_face<56>(a, s);
    }
    return DG_E_ARG;
}
int dispatch_element(int order, int qv, int qf, const StageArgs& a, cudaStream_t s) {
#define X(P, QV, QF, NB, NQV, NQF, E, NT, FT) \
    if (order == P && qv == QV && qf == QF) return launch_element_fixed<NB, NQV, NQF, E, NT>(a, s);
    FVEDG_FIXED_COMBOS(X)
#undef X
    switch (order) {
        case 0: return launch_element<1, 32>(a, s);
        case 1: return launch_element<4, 32>(a, s);
        case 2: return launch_element<10, 16>(a, s);
        case 3: return launch_element<20, 8>(a, s);
        case 4: return launch_element<35, 4>(a, s);
        case 5: return launch_element<56, 4>(a, s);
    }
    return DG_E_ARG;
}

FaceArgs face_args(dg_ctx* c, const double* U, int mask) {
    FaceArgs a;
    a.U = U;
    a.fi = c->d_fi;
    a.phi_fT = c->d_phi_fT;
    a.w_f = c->d_w_f;
    a.UD = c->d_UD;
    a.Fh = c->d_Fh;
    a.nface = (int)c->nface;
    a.nqf = c->tab.nqf;
    a.gamma = c->cfg.gamma;
    a.flux = c->cfg.flux;
    a.faces_mask = mask;
    return a;
}

StageArgs stage_args(dg_ctx* c, const double* U, const double* U0, double* out, int mode, double dt,
                     double a0, double a1, int with_volume) {
    StageArgs a;
    a.U = U;
    a.U0 = U0;
    a.out = out;
    a.Fh = c->d_Fh;
    a.geo = c->d_geo;
    a.ef = c->d_ef;
    a.phi_vT = c->d_phi_vT;
    a.dphi_vw = c->d_dphi_vw;
    a.phi_f = c->d_phi_f;
    a.mass_ref = c->d_mass_ref;
    a.ncell = (int)c->nowned;  // ghosts get no residual
    a.nqv = c->tab.nqv;
    a.nqf = c->tab.nqf;
    a.gamma = c->cfg.gamma;
    a.dt = dt;
    a.a0 = a0;
    a.a1 = a1;
    a.mode = mode;
    a.with_volume = with_volume;
    a.dt_inst = mode == 1 ? c->d_dt_inst : nullptr;
    a.elem_inst = c->d_elem_inst;
    a.Rv = nullptr;
    return a;
}

TcFaceArgs tc_face_args(dg_ctx* c, const double* U, int mask) {
    TcFaceArgs a;
    a.U = U; a.fi = c->d_fi; a.groups = c->tc.fgroups; a.ngroups = c->tc.nfgroups; a.UD = c->d_UD; a.Fh = c->tc.Fh;
    a.t = c->tc.t; a.gamma = c->cfg.gamma; a.flux = c->cfg.flux; a.faces_mask = mask; a.chk = c->tc.chk;
    return a;
}

TcElemArgs tc_elem_args(dg_ctx* c, const double* U, const double* U0, double* out, int mode, double dt, double a0,
                        double a1, int with_volume) {
    TcElemArgs a;
    a.U = U; a.U0 = U0; a.out = out; a.Fh = c->tc.Fh; a.jd = c->tc.jd; a.inv_detj = c->tc.inv_detj;
    a.groups = c->tc.egroups; a.ngroups = c->tc.negroups; a.t = c->tc.t; a.gamma = c->cfg.gamma;
    a.with_volume = with_volume; a.mode = mode; a.dt = dt; a.a0 = a0; a.a1 = a1;
    a.dt_inst = mode == 1 ? c->d_dt_inst : nullptr; a.elem_inst = c->d_elem_inst;
    a.Rv = (mode == 1 && c->cfg.mu > 0.0) ? c->d_Rv : nullptr;
    a.chk = c->tc.chk;
    return a;
}

// Face-flux launch of the FP64 form (tensor-core kernels where the rules have them).
int fp64_face(dg_ctx* c, const double* U, int mask, cudaStream_t s) {
    if (c->tc.ready) {
        ++g_launches;
        return tc_kernel(c->tc, 0, tc_face_args(c, U, mask), TcElemArgs{}, s);
    }
    return dispatch_face(c->cfg.order, c->qv, c->qf, face_args(c, U, mask), s);
}

// Element launch of the FP64 form: R (mode 0) or the RK stage out = a0 U0 + a1 (U + dt L) (mode 1).
int fp64_element(dg_ctx* c, const double* U, const double* U0, double* out, int mode, double dt, double a0,
                 double a1, int with_volume, cudaStream_t s) {
    if (c->tc.ready) {
        ++g_launches;
        return tc_kernel(c->tc, 1, TcFaceArgs{}, tc_elem_args(c, U, U0, out, mode, dt, a0, a1, with_volume), s);
    }
    StageArgs sa = stage_args(c, U, U0, out, mode, dt, a0, a1, with_volume);
    sa.Rv = (mode == 1 && c->cfg.mu > 0.0) ? c->d_Rv : nullptr;
    return dispatch_element(c->cfg.order, c->qv, c->qf, sa, s);
}

// One residual evaluation on device buffers (packed layout), FP64 form.
int residual_fp64(dg_ctx* c, const double* U, double* R, int part, cudaStream_t s) {
    if (c->cfg.flux != DG_FLUX_LF && c->cfg.flux != DG_FLUX_ROE) return DG_E_ARG;
    if (c->has_dirichlet && !c->d_UD) return DG_E_STATE;
    const int mask = part == 0 ? 3 : part == 1 ? 0 : part == 2 ? 1 : 2;
    int rc = fp64_face(c, U, mask, s);
    if (rc) return rc;
    return fp64_element(c, U, U, R, 0, 0.0, 0.0, 0.0, part == 0 || part == 1, s);
}

// Launch `fn` (which enqueues one kernel on stream s), bracketed by timing events when enabled.
template <class F>
int timed(dg_ctx* c, int cls, cudaStream_t s, F&& fn) {
    if (!c->timing) return fn();
    if (c->ev_used + 2 > c->ev.size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return DG_E_CUDA;
            c->ev.push_back(e);
        }
        c->ev_cls.resize(c->ev.size() / 2);
    }
    const size_t i = c->ev_used;
    if (cudaEventRecord(c->ev[i], s) != cudaSuccess) return DG_E_CUDA;
    const int rc = fn();
    if (cudaEventRecord(c->ev[i + 1], s) != cudaSuccess) return DG_E_CUDA;
    c->ev_cls[i / 2] = cls;
    c->ev_used += 2;
    return rc;
}

// One SSP-RK3 step (Shu-Osher) on the device state, FP64 form:
//   U1 = U + dt L(U);  U2 = 3/4 U + 1/4 (U1 + dt L(U1));  U = 1/3 U + 2/3 (U2 + dt L(U2)).
// The viscous operator's tables (the volume ones transposed so that lanes over points read rows,
// the A operands of its tensor-core products) and its per-face buffer; made by the first call.
int viscous_buffers(dg_ctx* c) {
    if (c->d_visc_vf) return DG_OK;
    const Tables& t = c->tab;
    const int nb = t.nb, nqv = t.nqv, nqf = t.nqf;
    std::vector<double> pv((size_t)nb * nqv), dpv((size_t)nb * 3 * nqv);  // volume tables, transposed
    for (int g = 0; g < nqv; ++g)
        for (int b = 0; b < nb; ++b) {
            pv[(size_t)b * nqv + g] = t.phi_v[(size_t)g * nb + b];
            for (int d = 0; d < 3; ++d) dpv[((size_t)b * 3 + d) * nqv + g] = t.dphi_v[((size_t)g * nb + b) * 3 + d];
        }
    // A operands of the tensor-core contractions, rows padded to 4 and modes to 8 (zeros)
    const int mp = visc_mp(nb), kpv = visc_kp(3 * nqv), kpf = visc_kp(nqf), gp = visc_gp(nqf), kpb = visc_kp(nb);
    if (gp > kViscMaxGp) return DG_E_ARG;
    std::vector<double> apt((size_t)24 * 4 * gp * kpb, 0.0);  // face traces: [p][t][g][b]
    for (int p = 0; p < 24; ++p)
        for (int g = 0; g < nqf; ++g)
            for (int b = 0; b < nb; ++b) {
                apt[(((size_t)p * 4 + 0) * gp + g) * kpb + b] = t.phi_f[((size_t)p * nqf + g) * nb + b];
                for (int d = 0; d < 3; ++d)
                    apt[(((size_t)p * 4 + 1 + d) * gp + g) * kpb + b] = t.dphi_f[(((size_t)p * nqf + g) * nb + b) * 3 + d];
            }
    std::vector<double> av((size_t)kpv * mp, 0.0), apf((size_t)24 * kpf * mp, 0.0);
    for (int k = 0; k < 3 * nqv; ++k)
        for (int j = 0; j < nb; ++j) av[(size_t)k * mp + j] = t.dphi_v[((size_t)(k / 3) * nb + j) * 3 + k % 3];
    for (int p = 0; p < 24; ++p)
        for (int g = 0; g < nqf; ++g)
            for (int j = 0; j < nb; ++j)
                apf[((size_t)p * kpf + g) * mp + j] = t.phi_f[((size_t)p * nqf + g) * nb + j];
    int rc;
    if ((rc = upload(&c->d_visc_phiT_v, pv)) || (rc = upload(&c->d_visc_dphiT_v, dpv)) ||
        (rc = upload(&c->d_visc_Av, av)) || (rc = upload(&c->d_visc_Pf, apf)) || (rc = upload(&c->d_visc_Pt, apt)) ||
        (rc = dev_alloc(&c->d_visc_vf, (size_t)c->nface * (5 * nqf + nb))))
        return rc;
    return DG_OK;
}

int viscous_launch(dg_ctx* c, const double* U, double* R, double mu, double prandtl, cudaStream_t s);

// Navier-Stokes stepping (dg_config.mu > 0): the viscous residual of the stage input, which the
// element kernels' update subtracts from the convective one: L = (R_visc - R_conv) / b, as the
// reference's viscous driver steps (tests/test_diffusion.cpp:381-382).
int viscous_stage(dg_ctx* c, const double* in, cudaStream_t s) {
    if (!(c->cfg.mu > 0.0)) return DG_OK;
    return timed(c, 3, s, [&] { return viscous_launch(c, in, c->d_Rv, c->cfg.mu, c->cfg.prandtl, s); });
}

// Limiter after stage st (dg_config.limiter): bounds from the stage input's statistics, the output
// limited in place and its statistics written for the next stage. The input's statistics come from
// the previous stage's launch, except after the state was set from outside (computed here at stage
// 0) and for ghost cells (computed here every stage: a halo exchange rewrote their rows).
int limit_stage(dg_ctx* c, int st, const double* in, double* out, cudaStream_t s) {
    if (!c->cfg.limiter) return DG_OK;
    const int64_t stats_begin = (st == 0 && !c->lim_valid) ? 0 : c->nowned;
    const int rc = timed(c, 4, s, [&] {
        return launch_limiter_stage(c->cfg.order, c->qv, out, in, c->d_lim_nbr, c->d_phi_v, c->ncell, c->nowned,
                                    stats_begin, c->cfg.gamma, c->cfg.limiter == 2, c->d_lim_stats[st],
                                    c->d_lim_stats[(st + 1) % 3], c->sms, s, &g_launches);
    });
    if (rc == DG_OK && st != 1) c->lim_valid = true;  // stage 0 made them valid, stage 2 rewrote them
    return rc;
}

// Before a CUDA graph of whole steps is captured or replayed: the statistics of U^n, so that the
// graph never needs the full statistics pass.
int ensure_limiter_stats(dg_ctx* c, cudaStream_t s) {
    if (!c->cfg.limiter || c->lim_valid) return DG_OK;
    const int rc = launch_limiter_stats(c->cfg.order, c->qv, c->d_Un, c->d_phi_v, 0, c->ncell, c->cfg.limiter == 2,
                                        c->d_lim_stats[0], c->sms, s, &g_launches);
    if (rc == DG_OK) c->lim_valid = true;
    return rc;
}

int step_fp64(dg_ctx* c, double dt, cudaStream_t s, int st0, int st1) {
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {c->d_Un, c->d_Ua, c->d_Ub};
    double* out[3] = {c->d_Ua, c->d_Ub, c->d_Un};
    for (int st = st0; st < st1; ++st) {
        int rc = viscous_stage(c, in[st], s);
        if (rc) return rc;
        rc = timed(c, 0, s, [&] { return fp64_face(c, in[st], 3, s); });
        if (rc) return rc;
        rc = timed(c, 1, s, [&] { return fp64_element(c, in[st], c->d_Un, out[st], 1, dt, A0[st], A1[st], 1, s); });
        if (rc) return rc;
        if ((rc = limit_stage(c, st, in[st], out[st], s))) return rc;
    }
    return DG_OK;
}

// Stages st0..st1-1 of one step (all three by default).
int step(dg_ctx* c, double dt, cudaStream_t s, int st0 = 0, int st1 = 3) {
    if (c->has_dirichlet && !c->d_UD) return DG_E_STATE;
    auto tm = [&](int cls, auto&& fn) { return timed(c, cls, s, fn); };
    if (c->cfg.precision == DG_PREC_MIXED) {
        auto post = [&](const double* in, double* out, int st) { return limit_stage(c, st, in, out, s); };
        auto stages = [&](int a0, int a1) {
            if (c->cfg.schedule == 1)
                return step_persistent(c->mixed, c->d_queue, c->qs, c->pp, c->d_Un, c->d_Ua, c->d_Ub, dt, s,
                                       &g_launches, tm, post, a0, a1);
            return step_mixed(c->mixed, c->d_Un, c->d_Ua, c->d_Ub, dt, s, &g_launches, tm, post, a0, a1);
        };
        if (!(c->cfg.mu > 0.0)) return stages(st0, st1);
        const double* in[3] = {c->d_Un, c->d_Ua, c->d_Ub};
        for (int st = st0; st < st1; ++st) {  // the element kernels read the stage's viscous residual
            int rc = viscous_stage(c, in[st], s);
            if (rc || (rc = stages(st, st + 1))) return rc;
        }
        return DG_OK;
    }
    return step_fp64(c, dt, s, st0, st1);
}

// Stage st of the mixed two-launch form in two phases around a halo exchange (a mesh with ghost
// elements): phase 0 the fluxes of the faces between owned elements, which read no ghost row;
// phase 1 the viscous residual, the faces touching ghosts, the element kernel and the limiter.
// Together they launch what step() launches for the stage, with the same arguments.
int stage_phase_mixed(dg_ctx* c, double dt, int st, int phase, cudaStream_t s) {
    if (c->has_dirichlet && !c->d_UD) return DG_E_STATE;
    MixedData& m = c->mixed;
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {c->d_Un, c->d_Ua, c->d_Ub};
    double* out[3] = {c->d_Ua, c->d_Ub, c->d_Un};
    auto K = [&](int which, int g0, int g1) {
        return mixed_kernel(m, which, in[st], c->d_Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, &g_launches, g0, g1);
    };
    if (phase == 0) return timed(c, 0, s, [&] { return K(0, 0, m.nfgroups_inner); });
    int rc = viscous_stage(c, in[st], s);
    if (rc || (rc = timed(c, 0, s, [&] { return K(0, m.nfgroups_inner, m.nfgroups); }))) return rc;
    if ((rc = timed(c, 1, s, [&] { return K(1, 0, -1); }))) return rc;
    return limit_stage(c, st, in[st], out[st], s);
}

int launches_per_step(const dg_ctx* c) {
    const int lim = (c->cfg.limiter ? (c->nowned < c->ncell ? 6 : 3) : 0) + (c->cfg.mu > 0.0 ? 6 : 0);
    if (c->cfg.precision == DG_PREC_MIXED) return (c->cfg.schedule == 1 ? 3 : mixed_launches_per_step(c->mixed)) + lim;
    return 6 + lim;
}

// After a synchronize: the watchdog words of the persistent queue and of the mixed kernels' bounded
// waits (DG_OK or DG_E_WATCHDOG); a set word is cleared.
int check_queue(dg_ctx* c) {
    int err = 0;
    if (c->mixed.err) {
        if (cudaMemcpy(&err, c->mixed.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return DG_E_CUDA;
        if (err != DG_OK) {
            cudaMemset(c->mixed.err, 0, sizeof(int));
            return DG_E_WATCHDOG;
        }
    }
    if (!c->d_queue) return DG_OK;
    if (cudaMemcpy(&err, &c->d_queue->error, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return DG_E_CUDA;
    if (err == DG_OK) return DG_OK;
    cudaMemset(c->d_queue, 0, sizeof(QueueState));
    return DG_E_WATCHDOG;
}

// copy between a host buffer with element stride `stride` and a packed device buffer
int copy_in(dg_ctx* c, double* dev, const double* host, size_t stride, cudaStream_t s) {
    const size_t blk = sizeof(double) * 5 * c->tab.nb;
    if (stride == 0) stride = blk;
    if (stride < blk) return DG_E_ARG;
    if (stride == blk) return cuda_ok(cudaMemcpyAsync(dev, host, blk * c->ncell, cudaMemcpyHostToDevice, s));
    return cuda_ok(cudaMemcpy2DAsync(dev, blk, host, stride, blk, c->ncell, cudaMemcpyHostToDevice, s));
}
int copy_out(dg_ctx* c, double* host, const double* dev, size_t stride, cudaStream_t s) {
    const size_t blk = sizeof(double) * 5 * c->tab.nb;
    if (stride == 0) stride = blk;
    if (stride < blk) return DG_E_ARG;
    if (stride == blk) return cuda_ok(cudaMemcpyAsync(host, dev, blk * c->ncell, cudaMemcpyDeviceToHost, s));
    return cuda_ok(cudaMemcpy2DAsync(host, stride, dev, blk, blk, c->ncell, cudaMemcpyDeviceToHost, s));
}

void free_ctx(dg_ctx* c) {
    if (!c) return;
    if (c->graph) cudaGraphExecDestroy(c->graph);
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    void* ptrs[] = {c->d_geo, c->d_fi, c->d_ef, c->d_phi_v, c->d_dphi_vw, c->d_w_v, c->d_phi_f, c->d_w_f,
                    c->d_phi_fT, c->d_phi_vT,
                    c->d_mass_ref, c->d_UD, c->d_Fh, c->d_Un, c->d_Ua, c->d_Ub, c->d_io, c->d_R,
                    c->d_red, c->d_red_out};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    free_schedule(c->qs);
    free_mixed(c->mixed);
    free_tc(c->tc);
    if (c->d_queue) cudaFree(c->d_queue);
    if (c->d_dt_inst) cudaFree(c->d_dt_inst);
    if (c->d_lim_bnd) cudaFree(c->d_lim_bnd);
    for (double* p : c->d_lim_stats)
        if (p) cudaFree(p);
    if (c->d_lim_nbr) cudaFree(c->d_lim_nbr);
    if (c->d_dphi_v) cudaFree(c->d_dphi_v);
    if (c->d_dphi_f) cudaFree(c->d_dphi_f);
    if (c->d_h) cudaFree(c->d_h);
    for (double* p : {c->d_visc_phiT_v, c->d_visc_dphiT_v, c->d_visc_Pt,
                      c->d_visc_Av, c->d_visc_Pf, c->d_visc_vf, c->d_Rv})
        if (p) cudaFree(p);
    if (c->d_lim_prev) cudaFree(c->d_lim_prev);
    if (c->d_elem_inst) cudaFree(c->d_elem_inst);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

}  // namespace

extern "C" {

const char* dg_status_string(int s) {
    switch (s) {
        case DG_OK: return "ok";
        case DG_E_ARG: return "bad argument";
        case DG_E_MESH: return "malformed mesh";
        case DG_E_CUDA: return "CUDA runtime error";
        case DG_E_NOMEM: return "out of memory";
        case DG_E_NONPHYSICAL: return "non-physical state (NaN/Inf, rho <= 0 or p <= 0)";
        case DG_E_WATCHDOG: return "bounded device wait expired";
        case DG_E_STATE: return "call out of order";
        case DG_E_IO: return "file error (open, read, write or checksum)";
    }
    return "unknown status";
}

int64_t dg_launch_count(void) { return g_launches.load(); }

const char* dg_last_cuda_error(void) {
    const int e = last_cuda_error_slot().load();
    return e ? cudaGetErrorName((cudaError_t)e) : "cudaSuccess";
}

}  // extern "C"

namespace {
dg_ctx* create_impl(const dg_mesh_desc* mesh, const dg_config* cfg, int* err, const std::vector<int64_t>* inst_off) {
    auto fail = [&](dg_ctx* c, int e) -> dg_ctx* {
        if (err) *err = e;
        free_ctx(c);
        return nullptr;
    };
    if (!mesh || !cfg) return fail(nullptr, DG_E_ARG);
    if (cfg->order < 0 || cfg->order > kMaxOrder || !(cfg->gamma > 1.0)) return fail(nullptr, DG_E_ARG);
    if (cfg->flux != DG_FLUX_LF && cfg->flux != DG_FLUX_ROE) return fail(nullptr, DG_E_ARG);
    if (cfg->precision != DG_PREC_FP64 && cfg->precision != DG_PREC_MIXED) return fail(nullptr, DG_E_ARG);
    if (cfg->schedule != 0 && !(cfg->schedule == 1 && cfg->precision == DG_PREC_MIXED)) return fail(nullptr, DG_E_ARG);
    const int qv = cfg->quad_vol < 0 ? auto_tet_rule(cfg->order) : cfg->quad_vol;
    const int qf = cfg->quad_face < 0 ? auto_tri_rule(cfg->order) : cfg->quad_face;
    if (tet_rule_npts(qv) <= 0 || tri_rule_npts(qf) <= 0) return fail(nullptr, DG_E_ARG);
    if (cfg->limiter < 0 || cfg->limiter > 2 || (cfg->limiter && !limiter_supported(cfg->order, qv)))
        return fail(nullptr, DG_E_ARG);
    if (!(cfg->mu >= 0.0) || (cfg->mu > 0.0 && !(cfg->prandtl > 0.0))) return fail(nullptr, DG_E_ARG);
    if (cfg->mu > 0.0 && (cfg->order < 1 || cfg->order > 4)) return fail(nullptr, DG_E_ARG);  // viscous kernels: P1..P4
    if (mesh->ncell <= 0 || mesh->ncell > (int64_t)1 << 30 || mesh->nface <= 0 || mesh->nface > (int64_t)1 << 30)
        return fail(nullptr, DG_E_ARG);
    Geometry geo;
    int rc = build_geometry(mesh, &geo);
    if (rc) return fail(nullptr, rc);
    dg_ctx* c = new (std::nothrow) dg_ctx;
    if (!c) return fail(nullptr, DG_E_NOMEM);
    c->cfg = *cfg;
    c->qv = qv;
    c->qf = qf;
    c->cfg.quad_vol = qv;
    c->cfg.quad_face = qf;
    c->ncell = mesh->ncell;
    c->nowned = mesh->ncell - mesh->nghost;
    c->nface = mesh->nface;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return fail(c, DG_E_CUDA);
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(c, DG_E_CUDA);
    build_tables(cfg->order, qv, qf, &c->tab);
    const int nb = c->tab.nb, nqf = c->tab.nqf;
    // element geometry and element -> face lists
    std::vector<double> hgeo(10 * c->ncell);
    for (int64_t e = 0; e < c->ncell; ++e) {
        for (int i = 0; i < 9; ++i) hgeo[10 * e + i] = geo.invjac[9 * e + i];
        hgeo[10 * e + 9] = geo.detj[e];
    }
    std::vector<FaceInfo> hfi(c->nface);
    std::vector<ElemFace> hef(4 * c->ncell);
    std::vector<int> fill(c->ncell, 0);
    for (int64_t f = 0; f < c->nface; ++f) {
        FaceInfo& fi = hfi[f];
        for (int i = 0; i < 3; ++i) fi.n[i] = geo.normal[3 * f + i];
        fi.jw = geo.area[f] * 2.0;
        fi.c0 = (int)mesh->face_cells[2 * f];
        fi.c1 = mesh->face_cells[2 * f + 1] == DG_NO_CELL ? -1 : (int)mesh->face_cells[2 * f + 1];
        const int bc = mesh->face_bc ? mesh->face_bc[f] : DG_BC_PSEUDO3DZ;
        const int per = mesh->face_periodic ? (mesh->face_periodic[f] ? 1 : 0) : 0;
        const int p0 = geo.perm[2 * f], p1 = fi.c1 >= 0 ? geo.perm[2 * f + 1] : 0;
        fi.meta = p0 | (p1 << 8) | (bc << 16) | (per << 24);
        if (fi.c1 < 0 && bc == DG_BC_DIRICHLET) c->has_dirichlet = true;
        fi.pad = 0;
        hef[4 * fi.c0 + fill[fi.c0]++] = ElemFace{(int)f, p0};
        if (fi.c1 >= 0) hef[4 * fi.c1 + fill[fi.c1]++] = ElemFace{(int)f, p1 | (1 << 8)};
    }
    // h = volume / sum of the face areas (ComputingMesh.cpp:289-297), for the viscous penalty
    std::vector<double> hh(c->ncell);
    for (int64_t e = 0; e < c->ncell; ++e) {
        double area = 0.0;
        if (fill[e] == 4 || !mesh->points || !mesh->cell_nodes) {
            for (int q = 0; q < fill[e]; ++q) area += geo.area[hef[4 * e + q].face];
        } else {  // a ghost without all its faces: the areas of its four sides from its vertices
            const int64_t* cn = mesh->cell_nodes + 4 * e;
            for (int o = 0; o < 4; ++o) {
                const double* p[3];
                for (int k = 0, m = 0; k < 4; ++k)
                    if (k != o) p[m++] = mesh->points + 3 * cn[k];
                const double a[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
                const double b[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
                const double n[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
                area += std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]) * 0.5;
            }
        }
        hh[e] = geo.detj[e] / 6.0 / area;
    }
    const size_t nstate = (size_t)c->ncell * 5 * nb;
    if ((rc = upload(&c->d_h, hh)) || (rc = upload(&c->d_dphi_v, c->tab.dphi_v)) ||
        (rc = upload(&c->d_dphi_f, c->tab.dphi_f)))
        return fail(c, rc);
    if ((rc = upload(&c->d_geo, hgeo)) || (rc = upload(&c->d_fi, hfi)) || (rc = upload(&c->d_ef, hef)) ||
        (rc = upload(&c->d_phi_v, c->tab.phi_v)) || (rc = upload(&c->d_dphi_vw, c->tab.dphi_vw)) ||
        (rc = upload(&c->d_w_v, c->tab.w_v)) || (rc = upload(&c->d_phi_f, c->tab.phi_f)) ||
        (rc = upload(&c->d_phi_fT, c->tab.phi_fT)) || (rc = upload(&c->d_phi_vT, c->tab.phi_vT)) ||
        (rc = upload(&c->d_w_f, c->tab.w_f)) || (rc = upload(&c->d_mass_ref, c->tab.mass_ref)) ||
        (rc = dev_alloc(&c->d_Fh, (cfg->precision == DG_PREC_FP64 && !tc_supported(cfg->order, qv, qf))
                                      ? (size_t)c->nface * nqf * 5 : 0)) ||
        (rc = dev_alloc(&c->d_Un, nstate)) ||
        (rc = dev_alloc(&c->d_Ua, nstate)) || (rc = dev_alloc(&c->d_Ub, nstate)) ||
        (rc = dev_alloc(&c->d_red, (size_t)kRedBlocks * 8)) || (rc = dev_alloc(&c->d_red_out, 8)))
        return fail(c, rc);
    if (inst_off && inst_off->size() >= 2) {
        c->ninst = (int)inst_off->size() - 1;
        c->inst_off = *inst_off;
        std::vector<int> inst(c->ncell);
        for (int i = 0; i < c->ninst; ++i)
            for (int64_t e = (*inst_off)[i]; e < (*inst_off)[i + 1]; ++e) inst[e] = i;
        std::vector<double> dts(c->ninst, 0.0);
        if ((rc = upload(&c->d_elem_inst, inst)) || (rc = upload(&c->d_dt_inst, dts))) return fail(c, rc);
    }
    if (cfg->precision == DG_PREC_FP64 && tc_supported(cfg->order, qv, qf)) {
        if ((rc = init_tc(c->tc, c->tab, hgeo, hfi, hef, c->ncell, c->nowned, c->nface, qv, qf))) return fail(c, rc);
    }
    if (cfg->precision == DG_PREC_MIXED) {
        rc = init_mixed(c->mixed, c->tab, hgeo, hfi, hef, c->ncell, c->nowned, c->nface, cfg->gamma, cfg->flux, qv, qf,
                        c->d_geo, c->d_fi, c->d_ef, c->d_mass_ref);
        if (rc) return fail(c, rc);
        c->mixed.dt_inst = c->d_dt_inst;
        c->mixed.elem_inst = c->d_elem_inst;
        if (cudaMalloc((void**)&c->d_queue, sizeof(QueueState)) != cudaSuccess) return fail(c, DG_E_NOMEM);
        if (cudaMemset(c->d_queue, 0, sizeof(QueueState)) != cudaSuccess) return fail(c, DG_E_CUDA);
        // the region order of the face groups (the persistent schedule's tiles; the two-launch face
        // kernel runs them in any order), except where a two-launch context with ghost elements keeps
        // the faces between owned elements first (dg_ssprk3_stage_phase)
        if (cfg->schedule == 1 || c->nowned == c->ncell)
            if ((rc = build_schedule(c->mixed, c->qs, c->pp))) return fail(c, rc);
    }
    {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
            c->sms = sms;
    }
    // Navier-Stokes stepping: the viscous buffers now, so that no step allocates (graph capture)
    if (cfg->mu > 0.0) {
        if ((rc = viscous_buffers(c)) || (rc = dev_alloc(&c->d_Rv, (size_t)c->ncell * 5 * nb))) return fail(c, rc);
        c->mixed.Rv = c->d_Rv;
    }
    // the limiter's per-cell statistics, allocated here so that no step allocates (graph capture)
    if (cfg->limiter) {
        for (double*& p : c->d_lim_stats)
            if ((rc = dev_alloc(&p, (size_t)c->ncell * 10))) return fail(c, rc);
    }
    {  // the limiter's neighbour table: the cell across each face, the cell itself on a boundary
        std::vector<int> nbr(4 * c->ncell);
        for (int64_t e = 0; e < c->ncell; ++e)
            for (int q = 0; q < 4; ++q) {
                int o = (int)e;
                if (q < fill[e]) {
                    const FaceInfo& F = hfi[hef[4 * e + q].face];
                    o = F.c0 == (int)e ? F.c1 : F.c0;
                    if (o < 0) o = (int)e;
                }
                nbr[4 * e + q] = o;
            }
        if ((rc = upload(&c->d_lim_nbr, nbr))) return fail(c, rc);
    }
    if (err) *err = DG_OK;
    return c;
}
}  // namespace

extern "C" {

dg_ctx* dg_create(const dg_mesh_desc* mesh, const dg_config* cfg, int* err) {
    return create_impl(mesh, cfg, err, nullptr);
}

dg_ctx* dg_create_ensemble(const dg_mesh_desc* meshes, int ninst, const dg_config* cfg, int* err) {
    if (!meshes || ninst < 1 || !cfg) {
        if (err) *err = DG_E_ARG;
        return nullptr;
    }
    // lay the instances end to end as one disconnected mesh
    const bool given = meshes[0].face_natural != nullptr;
    int64_t nc = 0, nf = 0, np = 0;
    for (int i = 0; i < ninst; ++i) {
        const dg_mesh_desc& d = meshes[i];
        const bool gi = d.face_natural != nullptr;
        if (gi != given || !d.face_cells || (!gi && (!d.points || !d.cell_nodes || !d.face_nodes)) || d.nghost != 0) {
            if (err) *err = DG_E_ARG;
            return nullptr;
        }
        nc += d.ncell;
        nf += d.nface;
        np += d.npts;
    }
    std::vector<int64_t> fc(2 * nf), cn, fn, fn1;
    std::vector<uint8_t> bc(nf, DG_BC_PSEUDO3DZ), per(nf, 0);
    std::vector<double> pts, nat, nrm, area, invj, detj;
    if (given) { nat.reserve(18 * nf); nrm.reserve(3 * nf); area.reserve(nf); invj.reserve(9 * nc); detj.reserve(nc); }
    else { pts.reserve(3 * np); cn.reserve(4 * nc); fn.reserve(3 * nf); fn1.reserve(3 * nf); }
    std::vector<int64_t> off(1, 0);
    int64_t co = 0, fo = 0, po = 0;
    for (int i = 0; i < ninst; ++i) {
        const dg_mesh_desc& d = meshes[i];
        for (int64_t f = 0; f < d.nface; ++f) {
            fc[2 * (fo + f)] = d.face_cells[2 * f] + co;
            fc[2 * (fo + f) + 1] = d.face_cells[2 * f + 1] == DG_NO_CELL ? DG_NO_CELL : d.face_cells[2 * f + 1] + co;
            if (d.face_bc) bc[fo + f] = d.face_bc[f];
            if (d.face_periodic) per[fo + f] = d.face_periodic[f];
        }
        if (given) {
            nat.insert(nat.end(), d.face_natural, d.face_natural + 18 * d.nface);
            nrm.insert(nrm.end(), d.face_normal, d.face_normal + 3 * d.nface);
            area.insert(area.end(), d.face_area, d.face_area + d.nface);
            invj.insert(invj.end(), d.cell_invjac, d.cell_invjac + 9 * d.ncell);
            detj.insert(detj.end(), d.cell_detj, d.cell_detj + d.ncell);
        } else {
            pts.insert(pts.end(), d.points, d.points + 3 * d.npts);
            for (int64_t k = 0; k < 4 * d.ncell; ++k) cn.push_back(d.cell_nodes[k] + po);
            for (int64_t k = 0; k < 3 * d.nface; ++k) {
                fn.push_back(d.face_nodes[k] + po);
                fn1.push_back((d.face_nodes1 ? d.face_nodes1[k] : d.face_nodes[k]) + po);
            }
        }
        co += d.ncell;
        fo += d.nface;
        po += d.npts;
        off.push_back(co);
    }
    dg_mesh_desc u{};
    u.ncell = nc;
    u.nface = nf;
    u.face_cells = fc.data();
    u.face_bc = bc.data();
    if (given) {
        u.face_natural = nat.data(); u.face_normal = nrm.data(); u.face_area = area.data();
        u.cell_invjac = invj.data(); u.cell_detj = detj.data();
    } else {
        u.npts = np; u.points = pts.data(); u.cell_nodes = cn.data(); u.face_nodes = fn.data();
        u.face_nodes1 = fn1.data(); u.face_periodic = per.data();
    }
    return create_impl(&u, cfg, err, &off);
}

int dg_ensemble_offsets(const dg_ctx* c, int64_t* elem_offsets) {
    if (!c || !elem_offsets) return DG_E_ARG;
    if (c->inst_off.empty()) { elem_offsets[0] = 0; elem_offsets[1] = c->ncell; return 1; }
    for (size_t i = 0; i < c->inst_off.size(); ++i) elem_offsets[i] = c->inst_off[i];
    return c->ninst;
}

void dg_destroy(dg_ctx* c) {
    if (c) cudaSetDevice(c->cfg.device);
    free_ctx(c);
}

int dg_info(const dg_ctx* c, int* nb, int* nqv, int* nqf, int* qv, int* qf) {
    if (!c) return DG_E_ARG;
    if (nb) *nb = c->tab.nb;
    if (nqv) *nqv = c->tab.nqv;
    if (nqf) *nqf = c->tab.nqf;
    if (qv) *qv = c->qv;
    if (qf) *qf = c->qf;
    return DG_OK;
}

int dg_residual_device(dg_ctx* c, const double* U, double* R, double t, int part, void* stream) {
    (void)t;
    if (!c || !U || !R || part < 0 || part > 3) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    cudaStream_t s = (cudaStream_t)stream;
    if (c->cfg.precision == DG_PREC_MIXED) return residual_mixed(c->mixed, U, R, part, s, &g_launches);
    return residual_fp64(c, U, R, part, s);
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Residual without any allocation: the face-flux scratch lives in a fixed device array of this
// library instead of the context's buffer. For callers that must not allocate device memory at the
// point of the call (see dg_residual_device_static in dg_gpu.h).
// ------------------------------------------------------------------------------------------------
constexpr size_t kStaticScratchDoubles = (size_t)4 << 20;  // 32 MiB of FP64 face fluxes
static __device__ __align__(256) double g_static_face_scratch[kStaticScratchDoubles];

namespace {
std::mutex g_static_mu;
double* g_static_ptr[64] = {};

// Device address of this device's copy of the array, looked up once per device with that device
// current (the name is only a host-side stand-in for it).
int static_scratch(int dev, double** out) {
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (dev < 0 || dev >= 64) return DG_E_ARG;
    if (!g_static_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_static_face_scratch) != cudaSuccess || !p) return DG_E_CUDA;
        g_static_ptr[dev] = (double*)p;
    }
    *out = g_static_ptr[dev];
    return DG_OK;
}
}  // namespace

extern "C" {

int64_t dg_static_scratch_capacity(void) { return (int64_t)kStaticScratchDoubles; }

int dg_residual_device_static(dg_ctx* c, const double* U, double* R, int part, void* stream) {
    if (!c || !U || !R || part < 0 || part > 3) return DG_E_ARG;
    if ((size_t)c->nface * c->tab.nqf * 5 > kStaticScratchDoubles) return DG_E_ARG;  // mesh too large
    if (c->has_dirichlet && !c->d_UD) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    double* scratch = nullptr;
    int rc = static_scratch(c->cfg.device, &scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    const int mask = part == 0 ? 3 : part == 1 ? 0 : part == 2 ? 1 : 2;
    FaceArgs fa = face_args(c, U, mask);
    fa.Fh = scratch;  // every face's entries are written (zeros for faces that contribute nothing)
    StageArgs sa = stage_args(c, U, U, R, 0, 0.0, 0.0, 0.0, part == 0 || part == 1);
    sa.Fh = scratch;
    if ((rc = dispatch_face(c->cfg.order, c->qv, c->qf, fa, s))) return rc;
    return dispatch_element(c->cfg.order, c->qv, c->qf, sa, s);
}

int dg_residual(dg_ctx* c, const double* U, double* R, size_t stride, double t, int part) {
    if (!c || !U || !R || part < 0 || part > 3) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const size_t nstate = (size_t)c->ncell * 5 * c->tab.nb;
    int rc;
    if (!c->d_io && (rc = dev_alloc(&c->d_io, nstate))) return rc;
    if (!c->d_R && (rc = dev_alloc(&c->d_R, nstate))) return rc;
    if ((rc = copy_in(c, c->d_io, U, stride, c->stream))) return rc;
    if ((rc = dg_residual_device(c, c->d_io, c->d_R, t, part, c->stream))) return rc;
    if ((rc = copy_out(c, R, c->d_R, stride, c->stream))) return rc;
    return cuda_ok(cudaStreamSynchronize(c->stream));
}

int dg_viscous_residual_device(dg_ctx* c, const double* U, double* R, double mu, double prandtl, void* stream) {
    if (!c || !U || !R || !(mu >= 0.0) || !(prandtl > 0.0)) return DG_E_ARG;
    if (c->has_dirichlet && !c->d_UD) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    int rc = viscous_buffers(c);
    if (rc) return rc;
    return viscous_launch(c, U, R, mu, prandtl, (cudaStream_t)stream);
}

}  // extern "C"

namespace {
// The viscous residual of U into R (two launches on stream s); the buffers exist.
int viscous_launch(dg_ctx* c, const double* U, double* R, double mu, double prandtl, cudaStream_t s) {
    ViscArgs a;
    a.U = U; a.R = R; a.geo = c->d_geo; a.h = c->d_h; a.fi = c->d_fi; a.ef = c->d_ef;
    a.phi_v = c->d_phi_v; a.dphi_v = c->d_dphi_v; a.w_v = c->d_w_v;
    a.phi_f = c->d_phi_f; a.dphi_f = c->d_dphi_f; a.w_f = c->d_w_f; a.UD = c->d_UD;
    a.phiT_v = c->d_visc_phiT_v; a.dphiT_v = c->d_visc_dphiT_v;
    a.vf = c->d_visc_vf;
    a.Av = c->d_visc_Av; a.Pf = c->d_visc_Pf; a.Pt = c->d_visc_Pt;
    a.mp = visc_mp(c->tab.nb); a.kpv = visc_kp(3 * c->tab.nqv); a.kpf = visc_kp(c->tab.nqf);
    a.gp = visc_gp(c->tab.nqf); a.kpb = visc_kp(c->tab.nb);
    a.ncell = c->nowned; a.nface = c->nface; a.nqv = c->tab.nqv; a.nqf = c->tab.nqf; a.order = c->cfg.order;
    a.mu = mu; a.cq = c->cfg.gamma / prandtl;
    g_launches += 2;
    return launch_viscous(c->cfg.order, a, c->sms, s);
}

// dg_autotune for the two-launch mixed schedule: times each element-kernel shape (mixed_elem_shapes:
// the kernel, warps per CTA, CTAs per SM) over two SSP-RK3 steps after one warm-up step, keeps the
// fastest, restores U^n from `save` (which it frees) and writes the JSON record.
int autotune_two_launch(dg_ctx* c, double dt, double* save, size_t nstate, char* report, size_t len) {
    ElemShape shapes[3];
    const int ns = mixed_elem_shapes(c->mixed, shapes);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::string js = "{\"schedule\": \"two-launch\", \"order\": " + std::to_string(c->cfg.order) +
                     ", \"quad_vol\": " + std::to_string(c->qv) + ", \"quad_face\": " + std::to_string(c->qf) +
                     ", \"ncell\": " + std::to_string(c->ncell) + ", \"knob\": \"element kernel shape\", \"candidates\": [";
    const int keep_k = c->mixed.elem_kernel, keep_c = c->mixed.elem_ctas;
    float best = 1e30f;
    int bi = -1, rc = DG_OK;
    auto name = [](const ElemShape& e) { return std::string(e.kernel == 2 ? "rows staged by TMA bulk copies" : "loads phase by phase"); };
    for (int i = 0; i < ns && rc == DG_OK; ++i) {
        c->mixed.elem_kernel = shapes[i].kernel;
        c->mixed.elem_ctas = shapes[i].ctas;
        rc = step(c, dt, c->stream);  // warm-up
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 2 && rc == DG_OK; ++r) rc = step(c, dt, c->stream);
        cudaEventRecord(e1, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = DG_E_CUDA;
        if (rc == DG_OK) rc = check_queue(c);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms *= 0.5f;
        js += std::string(i ? ", " : "") + "{\"element_kernel\": \"" + name(shapes[i]) + "\", \"warps_per_cta\": " +
              std::to_string(shapes[i].warps) + ", \"elements_per_cta\": " + std::to_string(3 * shapes[i].warps) +
              ", \"ctas_per_sm\": " + std::to_string(shapes[i].ctas) + ", \"ms_per_step\": " + std::to_string(ms) + "}";
        if (rc == DG_OK && ms < best) { best = ms; bi = i; }
    }
    c->mixed.elem_kernel = bi >= 0 ? shapes[bi].kernel : keep_k;
    c->mixed.elem_ctas = bi >= 0 ? shapes[bi].ctas : keep_c;
    js += "], \"chosen\": ";
    js += bi >= 0 ? "{\"element_kernel\": \"" + name(shapes[bi]) + "\", \"elements_per_cta\": " +
                        std::to_string(3 * shapes[bi].warps) + ", \"ctas_per_sm\": " + std::to_string(shapes[bi].ctas) +
                        ", \"ms_per_step\": " + std::to_string(best) + "}}"
                  : std::string("null}");
    cudaMemcpyAsync(c->d_Un, save, nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    c->lim_valid = false;
    cudaStreamSynchronize(c->stream);
    cudaFree(save);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    if (report && len > 0) {
        const size_t n = std::min(len - 1, js.size());
        std::memcpy(report, js.data(), n);
        report[n] = 0;
    }
    return rc;
}
}  // namespace

extern "C" {

int dg_viscous_residual(dg_ctx* c, const double* U, double* R, size_t stride, double mu, double prandtl) {
    if (!c || !U || !R) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const size_t nstate = (size_t)c->ncell * 5 * c->tab.nb;
    int rc;
    if (!c->d_io && (rc = dev_alloc(&c->d_io, nstate))) return rc;
    if (!c->d_R && (rc = dev_alloc(&c->d_R, nstate))) return rc;
    if ((rc = copy_in(c, c->d_io, U, stride, c->stream))) return rc;
    if ((rc = dg_viscous_residual_device(c, c->d_io, c->d_R, mu, prandtl, c->stream))) return rc;
    if ((rc = copy_out(c, R, c->d_R, stride, c->stream))) return rc;
    return cuda_ok(cudaStreamSynchronize(c->stream));
}

int dg_limit_device(dg_ctx* c, double* U, const double* Uprev, int only_avg, void* stream) {
    if (!c || !U || !Uprev) return DG_E_ARG;
    if (!limiter_supported(c->cfg.order, c->qv)) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    int rc;
    if (!c->d_lim_bnd && (rc = dev_alloc(&c->d_lim_bnd, (size_t)c->ncell * 10))) return rc;
    g_launches += 2;
    return launch_limiter(c->cfg.order, c->qv, U, Uprev, c->d_lim_nbr, c->d_phi_v, c->ncell, c->nowned,
                          c->cfg.gamma, only_avg != 0, c->d_lim_bnd, c->sms, (cudaStream_t)stream);
}

int dg_limit(dg_ctx* c, double* U, const double* Uprev, size_t stride, int only_avg) {
    if (!c || !U || !Uprev) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const size_t nstate = (size_t)c->ncell * 5 * c->tab.nb;
    int rc;
    if (!c->d_io && (rc = dev_alloc(&c->d_io, nstate))) return rc;
    if (!c->d_lim_prev && (rc = dev_alloc(&c->d_lim_prev, nstate))) return rc;
    if ((rc = copy_in(c, c->d_io, U, stride, c->stream)) || (rc = copy_in(c, c->d_lim_prev, Uprev, stride, c->stream)))
        return rc;
    if ((rc = dg_limit_device(c, c->d_io, c->d_lim_prev, only_avg, c->stream))) return rc;
    if ((rc = copy_out(c, U, c->d_io, stride, c->stream))) return rc;
    return cuda_ok(cudaStreamSynchronize(c->stream));
}

int dg_set_state(dg_ctx* c, const double* U, size_t stride) {
    if (!c || !U) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    c->lim_valid = false;
    int rc = copy_in(c, c->d_Un, U, stride, c->stream);
    if (rc) return rc;
    c->have_state = true;
    return cuda_ok(cudaStreamSynchronize(c->stream));
}

int dg_get_state(dg_ctx* c, double* U, size_t stride) {
    if (!c || !U) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    int rc = copy_out(c, U, c->d_Un, stride, c->stream);
    if (rc) return rc;
    return cuda_ok(cudaStreamSynchronize(c->stream));
}

int dg_ssprk3(dg_ctx* c, double dt, int nsteps) {
    if (!c || nsteps < 0 || !(dt >= 0)) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    for (int i = 0; i < nsteps; ++i) {
        int rc = step(c, dt, c->stream);
        if (rc) return rc;
    }
    DG_CUDA(cudaStreamSynchronize(c->stream));
    return check_queue(c);
}

int dg_ssprk3_graph(dg_ctx* c, double dt, int nsteps) {
    if (!c || nsteps < 0 || !(dt >= 0)) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    if (const int lrc = ensure_limiter_stats(c, c->stream)) return lrc;
    if (!c->graph || c->graph_dt != dt) {
        if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
        cudaGraph_t g = nullptr;
        DG_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t before = g_launches.load();
        int rc = step(c, dt, c->stream);
        cudaError_t ce = cudaStreamEndCapture(c->stream, &g);
        if (rc || ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return rc ? rc : DG_E_CUDA; }
        g_launches.store(before);  // captured launches are counted when the graph replays
        ce = cudaGraphInstantiate(&c->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) { c->graph = nullptr; return DG_E_CUDA; }
        c->graph_dt = dt;
    }
    const int per_step = launches_per_step(c);
    for (int i = 0; i < nsteps; ++i) {
        DG_CUDA(cudaGraphLaunch(c->graph, c->stream));
        g_launches += per_step;
    }
    DG_CUDA(cudaStreamSynchronize(c->stream));
    return check_queue(c);
}

int dg_ssprk3_ensemble(dg_ctx* c, const double* dt, int nsteps, int use_graph) {
    if (!c || !dt || nsteps < 0) return DG_E_ARG;
    if (!c->d_dt_inst) return DG_E_STATE;
    for (int i = 0; i < c->ninst; ++i)
        if (!(dt[i] >= 0)) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    DG_CUDA(cudaMemcpyAsync(c->d_dt_inst, dt, sizeof(double) * c->ninst, cudaMemcpyHostToDevice, c->stream));
    // the kernels read the per-instance dt from device memory; the uniform dt argument is unused
    return use_graph ? dg_ssprk3_graph(c, 0.0, nsteps) : dg_ssprk3(c, 0.0, nsteps);
}

void* dg_stream(dg_ctx* c) { return c ? (void*)c->stream : nullptr; }

double* dg_state_device(dg_ctx* c, int which) {
    if (!c || which < 0 || which > 2) return nullptr;
    return which == 0 ? c->d_Un : which == 1 ? c->d_Ua : c->d_Ub;
}

}  // extern "C"

namespace {
// Whole element rows (5 Nb doubles) between a state buffer and a packed exchange buffer: pack
// copies rows[i] of the state to slot i of buf, unpack copies slot i into rows[i]. Rows outside
// [0, ncell) are skipped. One thread per double, consecutive threads along a row.
__global__ void halo_rows(double* __restrict__ state, double* __restrict__ buf, const int64_t* __restrict__ rows,
                          int64_t n, int row_len, int64_t ncell, int unpack) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * row_len) return;
    const int64_t slot = i / row_len;
    const int j = (int)(i - slot * row_len);
    const int64_t r = rows[slot];
    if (r < 0 || r >= ncell) return;
    if (unpack) state[r * row_len + j] = buf[i];
    else buf[i] = state[r * row_len + j];
}

int halo_copy(dg_ctx* c, int which, const int64_t* rows, int64_t n, double* buf, void* stream, int unpack) {
    if (!c || which < 0 || which > 2 || n < 0 || (n > 0 && (!rows || !buf))) return DG_E_ARG;
    if (n == 0) return DG_OK;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    const int row_len = 5 * c->tab.nb;
    const int64_t total = n * row_len;
    halo_rows<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(dg_state_device(c, which), buf, rows, n, row_len,
                                                             c->ncell, unpack);
    ++g_launches;
    return cuda_ok(cudaGetLastError());
}
}  // namespace

extern "C" {

int dg_halo_pack(dg_ctx* c, int which, const int64_t* rows_dev, int64_t n, double* buf_dev, void* stream) {
    return halo_copy(c, which, rows_dev, n, buf_dev, stream, 0);
}

int dg_halo_unpack(dg_ctx* c, int which, const int64_t* rows_dev, int64_t n, const double* buf_dev, void* stream) {
    return halo_copy(c, which, rows_dev, n, const_cast<double*>(buf_dev), stream, 1);
}

int dg_refresh_split(dg_ctx* c, int which, const int64_t* elems, int64_t n, void* stream) {
    (void)stream;
    if (!c || which < 0 || which > 2 || n < 0 || (n > 0 && !elems)) return DG_E_ARG;
    return DG_OK;  // the mixed kernels split the FP64 rows as they load them: no copy to refresh
}

int dg_ssprk3_stage_phase(dg_ctx* c, double dt, int stage, int phase) {
    if (!c || stage < 0 || stage > 2 || phase < 0 || phase > 1 || !(dt >= 0)) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const bool split = c->cfg.precision == DG_PREC_MIXED && c->cfg.schedule == 0 && c->nowned < c->ncell;
    if (!split) return phase == 0 ? DG_OK : step(c, dt, c->stream, stage, stage + 1);
    return stage_phase_mixed(c, dt, stage, phase, c->stream);
}

int dg_ssprk3_stage(dg_ctx* c, double dt, int stage) {
    if (!c || stage < 0 || stage > 2 || !(dt >= 0)) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    return step(c, dt, c->stream, stage, stage + 1);
}

int dg_ssprk3_timed(dg_ctx* c, double dt, int nsteps, double* out, int nclass) {
    if (!c || nsteps < 0 || !(dt >= 0) || !out || nclass <= 0) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    c->timing = true;
    c->ev_used = 0;
    int rc = DG_OK;
    for (int i = 0; i < nsteps && rc == DG_OK; ++i) rc = step(c, dt, c->stream);
    c->timing = false;
    if (rc) return rc;
    DG_CUDA(cudaStreamSynchronize(c->stream));
    if ((rc = check_queue(c))) return rc;
    for (int k = 0; k < 2 * nclass; ++k) out[k] = 0.0;
    for (size_t i = 0; i + 1 < c->ev_used; i += 2) {
        float ms = 0.f;
        DG_CUDA(cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]));
        const int k = c->ev_cls[i / 2];
        if (k < nclass) { out[2 * k] += ms; out[2 * k + 1] += 1.0; }
    }
    return DG_OK;
}

#ifdef FVEDG_TC_CHECK
// Checked builds only: the first failed bounds or alignment check of the tensor-core FP64 kernels
// (code, index), cleared on read.
int dg_debug_tc_check(dg_ctx* c, int* out) {
    if (!c || !c->tc.chk.err) return DG_E_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return DG_E_CUDA;
    if (cudaMemcpy(out, c->tc.chk.err, 2 * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return DG_E_CUDA;
    return cudaMemset(c->tc.chk.err, 0, 2 * sizeof(int)) == cudaSuccess ? DG_OK : DG_E_CUDA;
}
#endif

int dg_watchdog_selftest(dg_ctx* c, int64_t polls) {
    if (!c || polls < 1) return DG_E_ARG;
    if (c->cfg.precision != DG_PREC_MIXED || c->cfg.schedule != 1 || !c->qs.ready || c->qs.nregions < 1)
        return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    DG_CUDA(cudaStreamSynchronize(c->stream));
    unsigned int need = 0;
    DG_CUDA(cudaMemcpy(&need, c->qs.total, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    const unsigned int never = need + 1u;  // one face group more than region 0 has: no wait on it can end
    DG_CUDA(cudaMemcpy(c->qs.total, &never, sizeof(unsigned int), cudaMemcpyHostToDevice));
    PersistentParams pp = c->pp;
    pp.spin_limit = polls;
    auto untimed = [&](int, auto&& fn) { return fn(); };
    auto no_post = [&](const double*, double*, int) { return DG_OK; };
    int rc = step_persistent(c->mixed, c->d_queue, c->qs, pp, c->d_Un, c->d_Ua, c->d_Ub, 0.0, c->stream, &g_launches,
                             untimed, no_post, 0, 1);
    const cudaError_t se = cudaStreamSynchronize(c->stream);
    const cudaError_t re = cudaMemcpy(c->qs.total, &need, sizeof(unsigned int), cudaMemcpyHostToDevice);
    if (rc) return rc;
    if (se != cudaSuccess || re != cudaSuccess) return DG_E_CUDA;
    return check_queue(c);
}

int dg_set_element_shape(dg_ctx* c, int staged, int ctas_per_sm) {
    if (!c || c->cfg.precision != DG_PREC_MIXED || (staged != 0 && staged != 1)) return DG_E_ARG;
    if (staged && ctas_per_sm != 1 && ctas_per_sm != 2) return DG_E_ARG;
    if (staged && (5 * c->tab.nb * 8) % 16 != 0) return DG_E_ARG;  // state rows not whole 16-byte units
    DG_CUDA(cudaSetDevice(c->cfg.device));
    c->mixed.elem_kernel = staged ? 2 : 0;
    c->mixed.elem_ctas = staged ? ctas_per_sm : 1;
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }  // a captured step used the old shape
    return DG_OK;
}

int dg_autotune(dg_ctx* c, double dt, char* report, size_t len) {
    if (!c || !(dt >= 0)) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    if (c->cfg.precision != DG_PREC_MIXED) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const size_t nstate = (size_t)c->ncell * 5 * c->tab.nb;
    double* save = nullptr;
    if (dev_alloc(&save, nstate)) return DG_E_NOMEM;
    DG_CUDA(cudaMemcpyAsync(save, c->d_Un, nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (c->cfg.schedule == 0) return autotune_two_launch(c, dt, save, nstate, report, len);
    // {face groups per tile, element groups per tile, CTAs per SM cap, regions, lag}
    static const int cand[][5] = {{32, 16, 0, 32, 1}, {16, 8, 0, 32, 1}, {64, 32, 0, 32, 1}, {32, 16, 0, 16, 1},
                                  {32, 16, 0, 64, 1}, {64, 32, 0, 64, 1}, {32, 16, 0, 32, 2}, {32, 16, 0, 64, 2},
                                  {16, 8, 0, 64, 1},  {128, 64, 0, 64, 1}, {32, 16, 0, 8, 1}, {32, 16, 0, 1, 0}};
    const int ncand = (int)(sizeof(cand) / sizeof(cand[0]));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::string js = "{\"order\": " + std::to_string(c->cfg.order) + ", \"quad_vol\": " + std::to_string(c->qv) +
                     ", \"quad_face\": " + std::to_string(c->qf) + ", \"ncell\": " + std::to_string(c->ncell) +
                     ", \"face_groups\": " + std::to_string(c->mixed.nfgroups) +
                     ", \"element_groups\": " + std::to_string(c->mixed.negroups) + ", \"candidates\": [";
    float best = 1e30f;
    PersistentParams bestp = c->pp;
    int rc = DG_OK;
    for (int i = 0; i < ncand && rc == DG_OK; ++i) {
        c->pp.tile_f = cand[i][0];
        c->pp.tile_e = cand[i][1];
        c->pp.max_blocks = cand[i][2];
        c->pp.regions = cand[i][3];
        c->pp.lag = cand[i][4];
        rc = build_schedule(c->mixed, c->qs, c->pp);
        if (rc == DG_OK) rc = step(c, dt, c->stream);  // warm-up
        cudaEventRecord(e0, c->stream);
        for (int r = 0; r < 2 && rc == DG_OK; ++r) rc = step(c, dt, c->stream);
        cudaEventRecord(e1, c->stream);
        if (cudaStreamSynchronize(c->stream) != cudaSuccess) rc = DG_E_CUDA;
        if (rc == DG_OK) rc = check_queue(c);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms *= 0.5f;
        js += std::string(i ? ", " : "") + "{\"tile_f\": " + std::to_string(cand[i][0]) + ", \"tile_e\": " +
              std::to_string(cand[i][1]) + ", \"max_blocks_per_sm\": " + std::to_string(cand[i][2]) +
              ", \"regions\": " + std::to_string(c->qs.nregions) + ", \"lag\": " + std::to_string(cand[i][4]) +
              ", \"ms_per_step\": " + std::to_string(ms) + "}";
        if (rc == DG_OK && ms < best) { best = ms; bestp = c->pp; }
    }
    c->pp = bestp;
    {
        const int brc = build_schedule(c->mixed, c->qs, c->pp);
        if (rc == DG_OK) rc = brc;
    }
    js += "], \"chosen\": {\"tile_f\": " + std::to_string(bestp.tile_f) + ", \"tile_e\": " +
          std::to_string(bestp.tile_e) + ", \"max_blocks_per_sm\": " + std::to_string(bestp.max_blocks) +
          ", \"regions\": " + std::to_string(c->qs.nregions) + ", \"lag\": " + std::to_string(bestp.lag) +
          ", \"ms_per_step\": " + std::to_string(best) + "}}";
    cudaMemcpyAsync(c->d_Un, save, nstate * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    c->lim_valid = false;
    cudaStreamSynchronize(c->stream);
    cudaFree(save);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    if (report && len > 0) {
        const size_t n = std::min(len - 1, js.size());
        std::memcpy(report, js.data(), n);
        report[n] = 0;
    }
    return rc;
}

// ------------------------------------------------------------------------------------------------
// Binary checkpoint / restart (new: the reference writes text solution files only). Layout:
//   96-byte header: "FVEDGCK1", version, order, quad_vol, quad_face, flux, precision, ncell,
//   nface, num_basis, gamma, t, step, reserved; then the state U^n, [ncell][5*Nb] FP64 packed;
//   then the FNV-1a 64-bit hash of the state bytes. Little-endian, as the host writes it.
// ------------------------------------------------------------------------------------------------
namespace {
struct CkptHeader {
    char magic[8];
    uint32_t version, order, quad_vol, quad_face, flux, precision;
    int64_t ncell, nface;
    uint32_t num_basis, reserved0;
    double gamma, t;
    int64_t step;
    uint64_t reserved1[2];
};
static_assert(sizeof(CkptHeader) == 96, "checkpoint header layout");

uint64_t fnv1a(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}
}  // namespace

int dg_save_checkpoint(dg_ctx* c, const char* path, double t, int64_t step) {
    if (!c || !path) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    const size_t n = (size_t)c->ncell * 5 * c->tab.nb;
    std::vector<double> U(n);
    int rc = dg_get_state(c, U.data(), 0);
    if (rc) return rc;
    CkptHeader h{};
    std::memcpy(h.magic, "FVEDGCK1", 8);
    h.version = 1;
    h.order = (uint32_t)c->cfg.order;
    h.quad_vol = (uint32_t)c->qv;
    h.quad_face = (uint32_t)c->qf;
    h.flux = (uint32_t)c->cfg.flux;
    h.precision = (uint32_t)c->cfg.precision;
    h.ncell = c->ncell;
    h.nface = c->nface;
    h.num_basis = (uint32_t)c->tab.nb;
    h.gamma = c->cfg.gamma;
    h.t = t;
    h.step = step;
    const uint64_t sum = fnv1a(U.data(), n * sizeof(double));
    FILE* f = std::fopen(path, "wb");
    if (!f) return DG_E_IO;
    const bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(U.data(), sizeof(double), n, f) == n &&
                    std::fwrite(&sum, sizeof(sum), 1, f) == 1;
    return (std::fclose(f) == 0 && ok) ? DG_OK : DG_E_IO;
}

int dg_load_checkpoint(dg_ctx* c, const char* path, double* t, int64_t* step) {
    if (!c || !path) return DG_E_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return DG_E_IO;
    CkptHeader h{};
    const size_t n = (size_t)c->ncell * 5 * c->tab.nb;
    std::vector<double> U;
    uint64_t sum = 0;
    int rc = DG_OK;
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, "FVEDGCK1", 8) != 0 || h.version != 1) {
        rc = DG_E_IO;
    } else if (h.order != (uint32_t)c->cfg.order || h.quad_vol != (uint32_t)c->qv || h.ncell != c->ncell ||
               h.nface != c->nface || h.num_basis != (uint32_t)c->tab.nb) {
        rc = DG_E_MESH;  // written by a context of another mesh, order or volume rule
    } else {
        U.resize(n);
        if (std::fread(U.data(), sizeof(double), n, f) != n || std::fread(&sum, sizeof(sum), 1, f) != 1 ||
            sum != fnv1a(U.data(), n * sizeof(double)))
            rc = DG_E_IO;
    }
    std::fclose(f);
    if (rc) return rc;
    if ((rc = dg_set_state(c, U.data(), 0))) return rc;
    if (t) *t = h.t;
    if (step) *step = h.step;
    return DG_OK;
}

int dg_mass(dg_ctx* c, double* mass, size_t stride) {
    if (!c || !mass) return DG_E_ARG;
    const int nb = c->tab.nb;
    const size_t blk = sizeof(double) * 5 * nb;
    if (stride == 0) stride = blk;
    if (stride < blk) return DG_E_ARG;
    // detJ * sum_g w_g phi_i^2, Riemann1D.cpp:108-121; host copy of the geometry is not kept, so
    // read detJ back from the device table.
    std::vector<double> geo(10 * c->ncell);
    DG_CUDA(cudaSetDevice(c->cfg.device));
    DG_CUDA(cudaMemcpy(geo.data(), c->d_geo, sizeof(double) * geo.size(), cudaMemcpyDeviceToHost));
    for (int64_t e = 0; e < c->ncell; ++e) {
        double* row = (double*)((char*)mass + stride * e);
        for (int i = 0; i < nb; ++i)
            for (int k = 0; k < 5; ++k) row[5 * i + k] = c->tab.mass_ref[i] * geo[10 * e + 9];
    }
    return DG_OK;
}

int dg_set_dirichlet(dg_ctx* c, const double* UD) {
    if (!c || !UD) return DG_E_ARG;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    const size_t n = (size_t)c->nface * c->tab.nqf * 5;
    int rc;
    if (!c->d_UD && (rc = dev_alloc(&c->d_UD, n))) return rc;
    DG_CUDA(cudaMemcpy(c->d_UD, UD, n * sizeof(double), cudaMemcpyHostToDevice));
    if (c->cfg.precision == DG_PREC_MIXED) set_mixed_dirichlet(c->mixed, c->d_UD);
    if (c->graph) { cudaGraphExecDestroy(c->graph); c->graph = nullptr; }
    return DG_OK;
}

int dg_conservation(dg_ctx* c, double out[6]) {
    if (!c || !out) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    return reduce_conservation(c->d_Un, c->d_geo, c->d_phi_v, c->d_w_v, (int)c->nowned, c->tab.nb, c->tab.nqv,
                               c->d_red, out, c->stream, &g_launches);
}

int dg_max_wave_speed(dg_ctx* c, double* lam) {
    if (!c || !lam) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    return reduce_wave_speed(c->d_Un, c->d_phi_v, (int)c->nowned, c->tab.nb, c->tab.nqv, c->cfg.gamma, c->d_red,
                             lam, c->stream, &g_launches);
}

int dg_check_state(dg_ctx* c, int64_t* bad) {
    if (!c) return DG_E_ARG;
    if (!c->have_state) return DG_E_STATE;
    DG_CUDA(cudaSetDevice(c->cfg.device));
    double nbad = 0;
    int rc = reduce_bad_points(c->d_Un, c->d_phi_v, (int)c->nowned, c->tab.nb, c->tab.nqv, c->cfg.gamma, c->d_red,
                               &nbad, c->stream, &g_launches);
    if (rc) return rc;
    if (bad) *bad = (int64_t)nbad;
    return nbad > 0 ? DG_E_NONPHYSICAL : DG_OK;
}

}  // extern "C"
