// Instantiations of the windowed step group k_window (minimum delay >= 2).
#include "sim.h"

namespace mgc {

template <bool FX, int WMAX>
static WindowKernel window_of(bool cur, int v)
{
    if (cur) return v == 0 ? k_window<true, 2, FX, WMAX> : k_window<true, 3, FX, WMAX>;
    return v == 0 ? k_window<false, 2, FX, WMAX> : k_window<false, 3, FX, WMAX>;
}

WindowKernel window_kernel(const mgc_sim* s, int v, bool wide)
{
    if (wide)
        return s->a.fx ? window_of<true, kMaxWindow>(s->a.has_cur, v) : window_of<false, kMaxWindow>(s->a.has_cur, v);
    return s->a.fx ? window_of<true, kAccBuffers>(s->a.has_cur, v) : window_of<false, kAccBuffers>(s->a.has_cur, v);
}

}  // namespace mgc
