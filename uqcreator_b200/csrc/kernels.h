// Kernel addresses per closure kind. The kernels are instantiated in one
// translation unit per closure kind (kernels_bb.cu, kernels_euler2d.cu,
// kernels_sw.cu); the host code launches them through these addresses.
#pragma once

namespace uqc {

// `which`: the kernel; `group`: threads per cell where the kernel has variants.
enum KernelId {
    KERNEL_CLOSURE       = 0,    // k_closure, FP64 (group 32, 64 or 256)
    KERNEL_UPDATE        = 1,    // k_update with the next step's convergence test
    KERNEL_INIT          = 2,    // k_init (group 32 or 256)
    KERNEL_MEANVAR       = 3,    // k_meanvar (group 32 or 256)
    KERNEL_CLOSURE_MIXED = 4,    // k_closure, mixed form (group 32 or 64)
    KERNEL_UPDATE_PLAIN  = 5,    // k_update without it
    KERNEL_CHECK         = 6,    // k_check
    KERNEL_PHASE_COUNTERS = 7,   // device address of this unit's phase counters (diagnostic builds), else nullptr
    KERNEL_CHORD         = 8,    // k_chord (mixed form in rounds; 2-D Euler only)
    KERNEL_HESS_TC       = 9,    // k_hess_tc
    KERNEL_INVERT_RAW    = 10,   // k_invert from k_hess_tc's values
    KERNEL_INVERT        = 11,   // k_invert with the Hessian on CUDA cores
    KERNEL_INVERT_SWEEP  = 12,   // k_invert_sweep (from k_hess_tc's values, n <= 84)
    KERNEL_UPDATE_WALL   = 13,   // k_update for meshes with wall cells (2-D Euler)
    KERNEL_UPDATE_PLAIN_WALL = 14,
    KERNEL_CLOSURE_TINY      = 15,   // k_closure with the register Newton of tiny systems
    KERNEL_UPDATE_SPLIT      = 16,   // k_update (with / without the test) whose projection splits
    KERNEL_UPDATE_PLAIN_SPLIT = 17   // the nodes of a small last block of basis functions
};

// nullptr when there is no such variant
void* kernel_bounded_barrier( int group, int which );
void* kernel_euler2d( int group, int which );
void* kernel_shallow_water( int group, int which );
void* kernel_linear( int cl, int group, int which );    // kinds 3-5
void* kernel_euler1d( int cl, int group, int which );   // kinds 6, 7
void* kernel_logsin( int group, int which );            // kind 8

}    // namespace uqc
