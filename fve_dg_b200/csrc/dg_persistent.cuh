// Persistent form of one RK stage: a single cooperative launch whose CTAs pull tiles of work from
// two queues — face groups first, then element groups — separated by a grid-wide barrier. The
// queues are plain atomic tickets, so CTAs that finish early take more tiles and uneven work (an
// ensemble of meshes of different sizes laid end to end) balances itself. Each RK stage is one
// launch; a CUDA graph captures the three launches of a step.
//
// Every wait is bounded: a CTA that spins at the barrier longer than kSpinLimit polls records
// DG_E_WATCHDOG in the queue state and continues, the host reads that word after the step and
// reports the error. The launch is cooperative, so all CTAs are co-resident by construction.
#pragma once
#include "dg_kernels_mixed.cuh"

namespace fvedg {

struct QueueState {
    unsigned int ctr[2];     // tickets of the face and element queues
    unsigned int bar_count;  // grid barrier: arrivals
    unsigned int bar_gen;    // grid barrier: generation
    int error;               // DG_OK or DG_E_WATCHDOG
    int pad[3];
};

constexpr long long kSpinLimit = 1ll << 24;  // about a second of 64 ns naps

__device__ __forceinline__ void grid_barrier(QueueState* q, unsigned int nblocks) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = &q->bar_gen;
        const unsigned int gen = *vgen;
        __threadfence();
        const unsigned int arrived = atomicAdd(&q->bar_count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&q->bar_count, 0u);
            __threadfence();
            atomicAdd(&q->bar_gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == gen) {
                __nanosleep(64);
                if (++spins > kSpinLimit) {
                    atomicExch(&q->error, DG_E_WATCHDOG);
                    break;
                }
            }
        }
        __threadfence();
    }
    __syncthreads();
}

template <int NB, int NQV, int NQF>
__host__ __device__ constexpr size_t persistent_warp_smem() {
    constexpr size_t a = sizeof(FaceMixedSmem<NQF>), b = sizeof(ElemMixedSmem<NB, NQV, NQF>);
    return ((a > b ? a : b) + 15) / 16 * 16;
}

// Phase 1 takes tickets over face-group tiles; phase 2 takes tickets over element-group tiles
// (volume term, face integrals and the update).
template <int NB, int NQV, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
    stage_persistent_mixed(MixedFaceArgs fa, MixedElemArgs ea, QueueState* q, int tile_f, int tile_e) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_tile;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wsm = smem_raw + persistent_warp_smem<NB, NQV, NQF>() * warp;
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(&q->ctr[0], 1u);
        __syncthreads();
        const int g0 = s_tile * tile_f;
        __syncthreads();
        if (g0 >= fa.ngroups) break;
        const int g1 = min(g0 + tile_f, fa.ngroups);
        for (int gi = g0 + warp; gi < g1; gi += WARPS)
            face_group_mixed<NB, NQF>(fa, gi, *reinterpret_cast<FaceMixedSmem<NQF>*>(wsm), lane);
    }
    grid_barrier(q, gridDim.x);
    auto& esm = *reinterpret_cast<ElemMixedSmem<NB, NQV, NQF>*>(wsm);
    __shared__ ElemTables<NB> tabs;
    element_tables_init(tabs, ea.t.inv_mass);
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(&q->ctr[1], 1u);
        __syncthreads();
        const int g0 = s_tile * tile_e;
        __syncthreads();
        if (g0 >= ea.ngroups) break;
        const int g1 = min(g0 + tile_e, ea.ngroups);
        for (int gi = g0 + warp; gi < g1; gi += WARPS) element_group_mixed<NB, NQV, NQF>(ea, gi, esm, tabs, lane);
    }
    grid_barrier(q, gridDim.x);
    if (blockIdx.x == 0 && threadIdx.x == 0) {  // every CTA is past both queues: rearm them
        q->ctr[0] = 0u;
        q->ctr[1] = 0u;
        __threadfence();
    }
}

struct PersistentParams {
    int tile_f = 16;     // face groups per ticket
    int tile_e = 8;      // element groups per ticket
    int max_blocks = 0;  // CTAs per SM cap (0 = as many as fit)
};

template <int NB, int NQV, int NQF, int W = 8>
inline int persistent_launch(MixedData& m, QueueState* q, const PersistentParams& pp, const double* U,
                             const double* U0, double* out, int mode, double dt, double a0, double a1, int face_mask,
                             int with_volume, cudaStream_t s, int mir_in, int mir_out) {
    auto kern = stage_persistent_mixed<NB, NQV, NQF, W>;
    constexpr size_t smem = persistent_warp_smem<NB, NQV, NQF>() * W;
    static unsigned long long done = 0;
    static int per_sm[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DG_E_CUDA;
    if (!(done & (1ull << (dev & 63)))) {
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
            return DG_E_CUDA;
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, W * 32, smem) != cudaSuccess || n < 1)
            return DG_E_CUDA;
        per_sm[dev & 63] = n;
        done |= 1ull << (dev & 63);
    }
    const int bps = pp.max_blocks > 0 ? std::min(per_sm[dev & 63], pp.max_blocks) : per_sm[dev & 63];
    const MixedFaceArgs fa = face_args(m, U, mir_in, face_mask);
    const MixedElemArgs ea = elem_args(m, U, U0, out, mode, dt, a0, a1, with_volume, mir_in, mir_out);
    int tf = pp.tile_f, te = pp.tile_e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(m.sms * bps);
    cfg.blockDim = dim3(W * 32);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kern, fa, ea, q, tf, te) != cudaSuccess) return DG_E_CUDA;
    return DG_OK;
}

inline int persistent_kernel(MixedData& m, QueueState* q, const PersistentParams& pp, const double* U,
                             const double* U0, double* out, int mode, double dt, double a0, double a1, int face_mask,
                             int with_volume, cudaStream_t s, std::atomic<int64_t>* launches, int mir_in, int mir_out) {
    if (!m.ready) return DG_E_ARG;
    ++*launches;
#define X(P, QV, QF, NB, NQV, NQF, W)                                                                             \
    if (m.order == P && m.qv == QV && m.qf == QF)                                                                 \
        return persistent_launch<NB, NQV, NQF>(m, q, pp, U, U0, out, mode, dt, a0, a1, face_mask, with_volume, s, \
                                               mir_in, mir_out);
    FVEDG_MIXED_COMBOS(X)
#undef X
    return DG_E_ARG;
}

template <class Timed>
inline int step_persistent(MixedData& m, QueueState* q, const PersistentParams& pp, double* Un, double* Ua,
                           double* Ub, double dt, cudaStream_t s, std::atomic<int64_t>* launches, Timed&& timed) {
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {Un, Ua, Ub};
    double* out[3] = {Ua, Ub, Un};
    const int mi[3] = {0, 1, 2}, mo[3] = {1, 2, 0};
    for (int st = 0; st < 3; ++st) {
        const int rc = timed(2, [&] {
            return persistent_kernel(m, q, pp, in[st], Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, launches, mi[st],
                                     mo[st]);
        });
        if (rc) return rc;
    }
    return DG_OK;
}

}  // namespace fvedg
