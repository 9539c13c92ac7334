// Instantiations of the windowed step group k_window (minimum delay >= 2).
#include "sim.h"

namespace mgc {

WindowKernel window_kernel(const mgc_sim* s, int v)
{
    if (s->a.has_cur) return v == 0 ? k_window<true, 2> : k_window<true, 3>;
    return v == 0 ? k_window<false, 2> : k_window<false, 3>;
}

}  // namespace mgc
