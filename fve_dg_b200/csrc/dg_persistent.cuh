// Persistent, dependency-driven form of one RK stage: one launch whose CTAs take tickets over a
// single list of tiles in which face tiles and element tiles are interleaved region by region, so
// the face work (instruction-bound: traces, Riemann solver) and the element work (bound by memory
// latency: face data, state, update) share the SMs instead of running one after the other.
//
// The element groups are cut into R regions of consecutive groups. A face group belongs to the
// lowest region among the cells of its faces. An element tile of region r may start once every
// face region its elements read is complete; the host places it in the list `lag` face regions
// after the last of those, so by the time a CTA takes it the faces are normally done. Face tiles
// wait for nothing. Since a tile is taken only by a running CTA and every tile an element tile
// waits for was taken before it, every wait ends; no cooperative launch is needed, and uneven work
// (an ensemble of meshes of different sizes laid end to end) balances itself.
//
// Every wait is bounded: a CTA that spins longer than the poll limit (kSpinLimit unless the context
// sets another) records DG_E_WATCHDOG in the queue state and goes on; the host reads that word after
// the step and reports the error. The
// last CTA to leave re-arms the ticket and the completion counters for the next launch, so a CUDA
// graph replays the three launches of a step as they are.
#pragma once
#include "dg_kernels_mixed.cuh"

namespace fvedg {

constexpr int kMaxRegions = 64;

struct QueueState {
    unsigned int ticket;              // next tile of the list
    unsigned int exits;               // CTAs that have left this launch
    int error;                        // DG_OK or DG_E_WATCHDOG
    int pad;
    unsigned int done[kMaxRegions];   // face groups completed, per region
};

constexpr long long kSpinLimit = 1ll << 24;  // about a second of 64 ns naps

struct PersistentParams {
    int tile_f = 32;     // face groups per tile
    int tile_e = 16;     // element groups per tile
    int max_blocks = 0;  // CTAs per SM cap (0 = as many as fit)
    int regions = 32;    // element regions (1 .. kMaxRegions)
    int lag = 1;         // face regions between an element tile's last dependency and its place
    long long spin_limit = kSpinLimit;  // polls before a wait gives up (not part of the tile list)
    bool operator==(const PersistentParams& o) const {
        return tile_f == o.tile_f && tile_e == o.tile_e && regions == o.regions && lag == o.lag;
    }
};

struct QueueSchedule {
    int4* tiles = nullptr;              // {kind (0 face, 1 element), first group, end group, region}
    unsigned long long* deps = nullptr; // [R] face regions each element region reads
    unsigned int* total = nullptr;      // [R] face groups per region
    int ntiles = 0, nregions = 0;
    PersistentParams built{};
    bool ready = false;
};

template <int NB, int NQV, int NQF>
__host__ __device__ constexpr size_t persistent_warp_smem() {
    constexpr size_t a = sizeof(FaceMixedSmem<NQF>), b = sizeof(ElemMixedSmem<NB, NQV, NQF>);
    return ((a > b ? a : b) + 15) / 16 * 16;
}

#ifndef FVEDG_PERSIST_MINB8
#define FVEDG_PERSIST_MINB8 4
#endif
template <int NB, int NQV, int NQF, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, WARPS == 8 ? FVEDG_PERSIST_MINB8 : 6)
    stage_persistent_mixed(MixedFaceArgs fa, MixedElemArgs ea, QueueState* q, const int4* __restrict__ tiles,
                           int ntiles, const unsigned long long* __restrict__ deps,
                           const unsigned int* __restrict__ total, long long spin_limit) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ElemTables<NB> tabs;
    __shared__ int4 s_tile;
    element_tables_init(tabs, ea.t.inv_mass);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* wsm = smem_raw + persistent_warp_smem<NB, NQV, NQF>() * warp;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned int t = atomicAdd(&q->ticket, 1u);
            int4 tl = t < (unsigned int)ntiles ? tiles[t] : make_int4(-1, 0, 0, 0);
            if (tl.x == 1) {  // element tile: wait until the face regions it reads are complete
                unsigned long long need = deps[tl.w];
                while (need) {
                    const int f = __ffsll((long long)need) - 1;
                    const volatile unsigned int* d = &q->done[f];
                    long long spins = 0;
                    while (*d < total[f]) {
                        __nanosleep(64);
                        if (++spins > spin_limit) {
                            atomicExch(&q->error, DG_E_WATCHDOG);
                            break;
                        }
                    }
                    need &= need - 1;
                }
                __threadfence();
            }
            s_tile = tl;
        }
        __syncthreads();
        const int4 tl = s_tile;
        if (tl.x < 0) break;
        if (tl.x == 0) {
            for (int gi = tl.y + warp; gi < tl.z; gi += WARPS)
                face_group_mixed<NB, NQF>(fa, gi, *reinterpret_cast<FaceMixedSmem<NQF>*>(wsm), lane);
            __threadfence();  // this CTA's face data is visible before the region count moves
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(&q->done[tl.w], (unsigned int)(tl.z - tl.y));
        } else {
            auto& esm = *reinterpret_cast<ElemMixedSmem<NB, NQV, NQF>*>(wsm);
            const ElemBTabs bt{ea.t.tva, ea.t.tvp, ea.t.tfl};
            for (int gi = tl.y + warp; gi < tl.z; gi += WARPS) element_group_mixed<NB, NQV, NQF>(ea, gi, esm, tabs, lane, bt);
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {  // the last CTA out re-arms the queue
        __threadfence();
        if (atomicAdd(&q->exits, 1u) == gridDim.x - 1) {
            q->ticket = 0u;
            for (int r = 0; r < kMaxRegions; ++r) q->done[r] = 0u;
            __threadfence();
            q->exits = 0u;
        }
    }
}

// Builds the tile list for `pp`: reorders the face groups by region (the face kernel of the
// two-launch form does not depend on their order) and uploads the list. Synchronous: call outside
// any stream capture (context creation, the autotuner).
inline int build_schedule(MixedData& m, QueueSchedule& qs, const PersistentParams& pp) {
    const int ne = m.negroups, nf = m.nfgroups;
    if (ne < 1 || nf < 1) return DG_E_ARG;
    const int R = std::max(1, std::min({pp.regions, kMaxRegions, ne}));
    const int tf = std::max(1, pp.tile_f), te = std::max(1, pp.tile_e), lag = std::max(0, pp.lag);
    std::vector<int> ereg(m.ncell, R), greg(ne);  // ghost cells (in no element group) stay at R
    for (int g = 0; g < ne; ++g) {
        greg[g] = (int)((int64_t)g * R / ne);
        for (int i = 0; i < m.heg[g].n; ++i) ereg[m.heg[g].e[i]] = greg[g];
    }
    // face groups by region (lowest region among their cells), stable within a region
    std::vector<int> freg(nf);
    for (int g = 0; g < nf; ++g) {
        int r = R;
        for (int i = 0; i < m.hfg[g].n; ++i) {
            const int f = m.hfg[g].f[i];
            r = std::min(r, ereg[m.hface_cells[2 * f]]);
            if (m.hface_cells[2 * f + 1] >= 0) r = std::min(r, ereg[m.hface_cells[2 * f + 1]]);
        }
        freg[g] = std::min(r, R - 1);
    }
    std::vector<int> order(nf);
    for (int g = 0; g < nf; ++g) order[g] = g;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return freg[x] < freg[y]; });
    std::vector<FaceGroup> fg(nf);
    std::vector<int> fg_reg(nf), face_reg(m.nface, 0);
    std::vector<unsigned int> total(R, 0u);
    for (int i = 0; i < nf; ++i) {
        fg[i] = m.hfg[order[i]];
        fg_reg[i] = freg[order[i]];
        ++total[fg_reg[i]];
        for (int k = 0; k < fg[i].n; ++k) face_reg[fg[i].f[k]] = fg_reg[i];
    }
    std::vector<unsigned long long> deps(R, 0ull);
    for (int g = 0; g < ne; ++g)
        for (int i = 0; i < m.heg[g].n; ++i)
            for (int q = 0; q < 4; ++q) deps[greg[g]] |= 1ull << face_reg[m.heg[g].face[i][q]];
    // element region r goes after face region min(last dependency + lag, R - 1)
    std::vector<std::vector<int>> after(R);
    for (int r = 0; r < R; ++r) {
        int last = 0;
        for (int b = 0; b < R; ++b)
            if (deps[r] >> b & 1ull) last = b;
        after[std::min(last + lag, R - 1)].push_back(r);
    }
    std::vector<int> ebeg(R + 1, ne), fbeg(R + 1, nf);
    for (int g = ne - 1; g >= 0; --g) ebeg[greg[g]] = g;
    for (int i = nf - 1; i >= 0; --i) fbeg[fg_reg[i]] = i;
    for (int r = R - 1; r >= 0; --r) {
        ebeg[r] = std::min(ebeg[r], ebeg[r + 1]);
        fbeg[r] = std::min(fbeg[r], fbeg[r + 1]);
    }
    std::vector<int4> tiles;
    for (int x = 0; x < R; ++x) {
        for (int g = fbeg[x]; g < fbeg[x + 1]; g += tf) tiles.push_back(make_int4(0, g, std::min(g + tf, fbeg[x + 1]), x));
        for (int r : after[x])
            for (int g = ebeg[r]; g < ebeg[r + 1]; g += te)
                tiles.push_back(make_int4(1, g, std::min(g + te, ebeg[r + 1]), r));
    }
    // upload: the reordered face groups into the existing buffer, the schedule into fresh ones
    if (cudaMemcpy((void*)m.fgroups, fg.data(), sizeof(FaceGroup) * nf, cudaMemcpyHostToDevice) != cudaSuccess)
        return DG_E_CUDA;
    m.hfg = fg;
    if (qs.tiles) cudaFree(qs.tiles);
    if (qs.deps) cudaFree(qs.deps);
    if (qs.total) cudaFree(qs.total);
    qs.tiles = nullptr; qs.deps = nullptr; qs.total = nullptr;
    qs.ready = false;
    if (cudaMalloc((void**)&qs.tiles, sizeof(int4) * tiles.size()) != cudaSuccess ||
        cudaMalloc((void**)&qs.deps, sizeof(unsigned long long) * R) != cudaSuccess ||
        cudaMalloc((void**)&qs.total, sizeof(unsigned int) * R) != cudaSuccess)
        return DG_E_NOMEM;
    if (cudaMemcpy(qs.tiles, tiles.data(), sizeof(int4) * tiles.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(qs.deps, deps.data(), sizeof(unsigned long long) * R, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(qs.total, total.data(), sizeof(unsigned int) * R, cudaMemcpyHostToDevice) != cudaSuccess)
        return DG_E_CUDA;
    qs.ntiles = (int)tiles.size();
    qs.nregions = R;
    qs.built = pp;
    qs.ready = true;
    return DG_OK;
}

inline void free_schedule(QueueSchedule& qs) {
    if (qs.tiles) cudaFree(qs.tiles);
    if (qs.deps) cudaFree(qs.deps);
    if (qs.total) cudaFree(qs.total);
    qs = QueueSchedule{};
}

template <int NB, int NQV, int NQF, int W = 8>
inline int persistent_launch(MixedData& m, QueueState* q, const QueueSchedule& qs, const PersistentParams& pp,
                             const double* U, const double* U0, double* out, int mode, double dt, double a0, double a1,
                             int face_mask, int with_volume, cudaStream_t s) {
    if (!qs.ready || !(qs.built == pp)) return DG_E_STATE;
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
    const MixedFaceArgs fa = face_args(m, U, face_mask);
    const MixedElemArgs ea = elem_args(m, U, U0, out, mode, dt, a0, a1, with_volume);
    kern<<<m.sms * bps, W * 32, smem, s>>>(fa, ea, q, qs.tiles, qs.ntiles, qs.deps, qs.total,
                                           pp.spin_limit > 0 ? pp.spin_limit : kSpinLimit);
    return cuda_status(cudaGetLastError());
}

inline int persistent_kernel(MixedData& m, QueueState* q, const QueueSchedule& qs, const PersistentParams& pp,
                             const double* U, const double* U0, double* out, int mode, double dt, double a0, double a1,
                             int face_mask, int with_volume, cudaStream_t s, std::atomic<int64_t>* launches) {
    if (!m.ready) return DG_E_ARG;
    ++*launches;
#define X(P, QV, QF, NB, NQV, NQF, W)                                                                              \
    if (m.order == P && m.qv == QV && m.qf == QF)                                                                  \
        return persistent_launch<NB, NQV, NQF, W>(m, q, qs, pp, U, U0, out, mode, dt, a0, a1, face_mask,           \
                                                  with_volume, s);
    FVEDG_MIXED_COMBOS(X)
#undef X
    return DG_E_ARG;
}

template <class Timed, class Post>
inline int step_persistent(MixedData& m, QueueState* q, const QueueSchedule& qs, const PersistentParams& pp,
                           double* Un, double* Ua, double* Ub, double dt, cudaStream_t s,
                           std::atomic<int64_t>* launches, Timed&& timed, Post&& post, int st0 = 0,
                           int st1 = 3) {
    const double A0[3] = {0.0, 0.75, 1.0 / 3.0};
    const double A1[3] = {1.0, 0.25, 2.0 / 3.0};
    const double* in[3] = {Un, Ua, Ub};
    double* out[3] = {Ua, Ub, Un};
    for (int st = st0; st < st1; ++st) {
        int rc = timed(2, [&] {
            return persistent_kernel(m, q, qs, pp, in[st], Un, out[st], 1, dt, A0[st], A1[st], 3, 1, s, launches);
        });
        if (rc) return rc;
        if ((rc = post(in[st], out[st], st))) return rc;
    }
    return DG_OK;
}

}  // namespace fvedg
