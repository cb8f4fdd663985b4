// Kernels of the shallow water closure (closure kind 2).
#include "kernels_inst.cuh"

namespace uqc {
void* kernel_shallow_water( int group, int which ) { return kernel_of<2>( group, which ); }
}    // namespace uqc
