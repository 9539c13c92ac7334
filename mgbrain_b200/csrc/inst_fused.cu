// Instantiations of the fused step kernel k_fused (one launch per step,
// deferred method, minimum delay >= 2), in a translation unit of their own
// so that the library's kernels compile in parallel.
#include "sim.h"

namespace mgc {

StepKernel fused_kernel(const mgc_sim* s, int v)
{
    if (s->a.has_cur) return v == 0 ? k_fused<true, 2> : k_fused<true, 3>;
    return v == 0 ? k_fused<false, 2> : k_fused<false, 3>;
}

}  // namespace mgc
