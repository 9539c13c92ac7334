// Instantiations of the step groups with a grid barrier per step (k_steps,
// minimum delay >= 2) and per phase (k_steps1, minimum delay 1), and the
// selector of every step-group form.
#include "sim.h"

namespace mgc {

template <bool FX>
static GroupKernel steps_of(bool fused, bool cur, int v)
{
    if (!fused) return cur ? k_steps1<true, FX> : k_steps1<false, FX>;  // minimum delay 1
    if (cur) return v == 0 ? k_steps<true, 2, FX> : k_steps<true, 3, FX>;
    return v == 0 ? k_steps<false, 2, FX> : k_steps<false, 3, FX>;
}

GroupKernel steps_kernel(const mgc_sim* s, int p, int v)
{
    if (s->fused && p == 2) return pipe_kernel(s, v);
    return s->a.fx ? steps_of<true>(s->fused, s->a.has_cur, v) : steps_of<false>(s->fused, s->a.has_cur, v);
}

}  // namespace mgc
