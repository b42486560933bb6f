// per_step.cu -- per-step engine for aeif_cond_alpha and plastic networks.
#include "../../../include/bspk.h"
#include "aeif_args.h"

namespace bspk {
int run_per_step(bspk_plan *, int64_t, cudaStream_t) { return BSPK_ERR_UNSUPPORTED; }
}  // namespace bspk
