// Instantiations of the windowed step group k_window (minimum delay >= 2).
#include "sim.h"

namespace mgc {

template <bool FX>
static WindowKernel window_of(bool cur, int v)
{
    if (cur) return v == 0 ? k_window<true, 2, FX> : k_window<true, 3, FX>;
    return v == 0 ? k_window<false, 2, FX> : k_window<false, 3, FX>;
}

WindowKernel window_kernel(const mgc_sim* s, int v)
{
    return s->a.fx ? window_of<true>(s->a.has_cur, v) : window_of<false>(s->a.has_cur, v);
}

}  // namespace mgc
