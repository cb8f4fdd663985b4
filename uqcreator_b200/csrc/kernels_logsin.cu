// Kernels of the LogSin closure (kind 8, one state, with the Burgers problem).
#include "kernels_inst.cuh"

namespace uqc {
void* kernel_logsin( int group, int which ) { return kernel_of<8>( group, which ); }
}    // namespace uqc
