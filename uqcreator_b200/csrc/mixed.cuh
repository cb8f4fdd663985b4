// Mixed-precision closure pipeline (tensor-core Hessian). Planning and
// dispatch interface used by solver.cu.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "ipm_kernels.cuh"

namespace uqc {

struct MixedPlan {
    bool ok = false;
    std::string why = "mixed precision is not available for this configuration";
};

inline MixedPlan plan_mixed( int, int, int, int, int, int ) { return MixedPlan{}; }
inline void alloc_mixed( MixedPlan&, size_t ) {}
inline void free_mixed( MixedPlan& ) {}
inline int launch_mixed_closure( MixedPlan&, KParams&, int, int, cudaStream_t ) { return 0; }

}    // namespace uqc
