// Kernels of the 2-D Euler closure (closure kind 1).
#include "kernels_inst.cuh"

namespace uqc {
void* kernel_euler2d( int group, int which ) { return kernel_of<1>( group, which ); }
}    // namespace uqc
