// Instantiations of the pipelined step group k_pipe (minimum delay >= 4).
#include "sim.h"

namespace mgc {

template <bool FX>
static GroupKernel pipe_of(bool cur, int v)
{
    if (cur) return v == 0 ? k_pipe<true, 2, FX> : k_pipe<true, 3, FX>;
    return v == 0 ? k_pipe<false, 2, FX> : k_pipe<false, 3, FX>;
}

GroupKernel pipe_kernel(const mgc_sim* s, int v)
{
    return s->a.fx ? pipe_of<true>(s->a.has_cur, v) : pipe_of<false>(s->a.has_cur, v);
}

}  // namespace mgc
