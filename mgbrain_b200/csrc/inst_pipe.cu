// Instantiations of the pipelined step group k_pipe (minimum delay >= 4).
#include "sim.h"

namespace mgc {

GroupKernel pipe_kernel(const mgc_sim* s, int v)
{
    if (s->a.has_cur) return v == 0 ? k_pipe<true, 2> : k_pipe<true, 3>;
    return v == 0 ? k_pipe<false, 2> : k_pipe<false, 3>;
}

}  // namespace mgc
