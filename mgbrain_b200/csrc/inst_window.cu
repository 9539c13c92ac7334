// Instantiations of the windowed step group k_window (minimum delay >= 2), with
// and without pull steps.
#include "sim.h"

namespace mgc {

template <bool FX, int WMAX, bool PULL>
static WindowKernel window_of(bool cur, int v)
{
    if (cur) return v == 0 ? k_window<true, 2, FX, WMAX, PULL> : k_window<true, 3, FX, WMAX, PULL>;
    return v == 0 ? k_window<false, 2, FX, WMAX, PULL> : k_window<false, 3, FX, WMAX, PULL>;
}

template <bool PULL>
static WindowKernel window_pick(const mgc_sim* s, int v, bool wide)
{
    if (wide)
        return s->a.fx ? window_of<true, kMaxWindow, PULL>(s->a.has_cur, v)
                       : window_of<false, kMaxWindow, PULL>(s->a.has_cur, v);
    return s->a.fx ? window_of<true, kAccBuffers, PULL>(s->a.has_cur, v)
                   : window_of<false, kAccBuffers, PULL>(s->a.has_cur, v);
}

// Pull steps (mgc_set_pull) take their own instantiations, so that the plain
// ones keep their register allocation.
WindowKernel window_kernel(const mgc_sim* s, int v, bool wide, bool pull)
{
    return pull ? window_pick<true>(s, v, wide) : window_pick<false>(s, v, wide);
}

}  // namespace mgc
