// Kernels of the bounded barrier (Burgers) closure (closure kind 0).
#include "kernels_inst.cuh"

namespace uqc {
void* kernel_bounded_barrier( int group, int which ) { return kernel_of<0>( group, which ); }
}    // namespace uqc
