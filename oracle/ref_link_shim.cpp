/*
 * Test infrastructure: link shim for the reference build in oracle/_ref/.
 * src/simulator/mgsim/adj/mgnet.h:14-15 declares
 *   init_gsubnet_neus(GSubNet*, int, int) and init_gsubnet_syns(GSubNet*, int)
 * while mgnet.cpp:5,23 defines them with size_t counts, so mgsim.cpp's calls
 * (mgsim.cpp:93,105) bind to declarations that nothing defines.  These two
 * forwarders supply the declared signatures.
 */
#include <cstddef>
namespace MGBrain {
struct GSubNet;
void init_gsubnet_neus(GSubNet* cnet, size_t num, int max_delay);
void init_gsubnet_syns(GSubNet* cnet, size_t num);
void init_gsubnet_neus(GSubNet* cnet, int num, int max_delay)
{
    init_gsubnet_neus(cnet, (size_t)num, max_delay);
}
void init_gsubnet_syns(GSubNet* cnet, int num) { init_gsubnet_syns(cnet, (size_t)num); }
}  // namespace MGBrain
