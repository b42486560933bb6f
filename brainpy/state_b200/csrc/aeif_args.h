// aeif_args.h -- per-step engine (aeif_cond_alpha RKF45 and plastic
// projections): launched step by step from the host loop.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

struct bspk_plan;

namespace bspk {
int run_per_step(bspk_plan *p, int64_t n_steps, cudaStream_t st);
}  // namespace bspk
