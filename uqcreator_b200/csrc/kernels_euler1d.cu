// Kernels of the 1-D Euler problem: the entropy closure (kind 6) and the
// linear closures with its three states (kind 7).
#include "kernels_inst.cuh"

namespace uqc {
void* kernel_euler1d( int cl, int group, int which ) {
    if( cl == 6 ) return kernel_of<6>( group, which );
    if( cl == 7 ) return kernel_of<7>( group, which );
    return nullptr;
}
}    // namespace uqc
