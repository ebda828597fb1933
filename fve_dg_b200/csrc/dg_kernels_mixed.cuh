// Mixed-precision form (placeholder until the tensor-core kernels land).
#pragma once
#include <atomic>
#include <cstdint>
#include <vector>

#include "dg_internal.h"
#include "dg_kernels_fp64.cuh"

namespace fvedg {

struct MixedData {
    bool ready = false;
};

inline int init_mixed(MixedData&, const Tables&, const std::vector<double>&, const std::vector<FaceInfo>&,
                      const std::vector<ElemFace>&, int64_t, int64_t, double, int) {
    return DG_E_ARG;
}
inline void free_mixed(MixedData&) {}
inline void set_mixed_dirichlet(MixedData&, const double*) {}
inline int mixed_launches_per_step(const MixedData&) { return 0; }
inline int residual_mixed(MixedData&, const double*, double*, int, cudaStream_t, std::atomic<int64_t>*) {
    return DG_E_ARG;
}
inline int step_mixed(MixedData&, double*, double*, double*, double, cudaStream_t, std::atomic<int64_t>*) {
    return DG_E_ARG;
}

}  // namespace fvedg
