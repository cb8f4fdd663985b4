// Kernels of the linear closures (stochastic Galerkin and the moment filters)
// with the states of Burgers (kind 3), 2-D Euler (kind 4) and shallow water
// (kind 5).
#include "kernels_inst.cuh"

namespace uqc {
void* kernel_linear( int cl, int group, int which ) {
    if( cl == 3 ) return kernel_of<3>( group, which );
    if( cl == 4 ) return kernel_of<4>( group, which );
    if( cl == 5 ) return kernel_of<5>( group, which );
    return nullptr;
}
}    // namespace uqc
