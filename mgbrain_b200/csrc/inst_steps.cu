// Instantiations of the step groups with a grid barrier per step (k_steps,
// minimum delay >= 2) and per phase (k_steps1, minimum delay 1), and the
// selector of every step-group form.
#include "sim.h"

namespace mgc {

GroupKernel steps_kernel(const mgc_sim* s, int p, int v)
{
    if (!s->fused) return s->a.has_cur ? k_steps1<true> : k_steps1<false>;  // minimum delay 1
    if (p == 2) return pipe_kernel(s, v);
    if (s->a.has_cur) return v == 0 ? k_steps<true, 2> : k_steps<true, 3>;
    return v == 0 ? k_steps<false, 2> : k_steps<false, 3>;
}

}  // namespace mgc
