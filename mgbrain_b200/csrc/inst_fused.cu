// Instantiations of the fused step kernel k_fused (one launch per step,
// deferred method, minimum delay >= 2), in a translation unit of their own
// so that the library's kernels compile in parallel.  Instances: with or
// without LIF/LIFE currents x 2 or 3 resident blocks per SM x fp32 or
// fixed-point accumulation.
#include "sim.h"

namespace mgc {

template <bool FX>
static StepKernel fused_of(bool cur, int v)
{
    if (cur) return v == 0 ? k_fused<true, 2, FX> : k_fused<true, 3, FX>;
    return v == 0 ? k_fused<false, 2, FX> : k_fused<false, 3, FX>;
}

StepKernel fused_kernel(const mgc_sim* s, int v)
{
    return s->a.fx ? fused_of<true>(s->a.has_cur, v) : fused_of<false>(s->a.has_cur, v);
}

}  // namespace mgc
