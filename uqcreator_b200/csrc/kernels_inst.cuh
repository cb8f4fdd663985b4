// Instantiation of every kernel of one closure kind (included once per kind
// by kernels_<kind>.cu) and the table of their addresses.
#pragma once
#include "chord.cuh"
#include "ipm_kernels.cuh"
#include "kernels.h"

namespace uqc {

template <int CL> void* kernel_of( int group, int which ) {
    if constexpr( Closure<CL>::LINEAR ) {
        // linear closures: no Newton, so no mixed, register-Newton or rounds kernels
        if( which == KERNEL_CLOSURE_MIXED || which == KERNEL_CLOSURE_TINY || which == KERNEL_CHORD || which == KERNEL_HESS_TC ||
            which == KERNEL_INVERT_RAW || which == KERNEL_INVERT || which == KERNEL_INVERT_SWEEP )
            return nullptr;
    }
    switch( which ) {
        case KERNEL_CLOSURE:
            if( group == 32 ) return (void*)&k_closure<CL, 32, double>;
            if( group == 64 ) return (void*)&k_closure<CL, 64, double>;
            if( group == 256 ) return (void*)&k_closure<CL, 256, double>;
            return nullptr;
        case KERNEL_CLOSURE_TINY:
            if constexpr( !Closure<CL>::LINEAR ) return (void*)&k_closure<CL, 32, double, true>;
            return nullptr;
        case KERNEL_CLOSURE_MIXED:
            if constexpr( !Closure<CL>::LINEAR ) {
                if( group == 32 ) return (void*)&k_closure<CL, 32, float>;
                if( group == 64 ) return (void*)&k_closure<CL, 64, float>;
            }
            return nullptr;
        case KERNEL_UPDATE: return (void*)&k_update<CL, true, false, false>;
        case KERNEL_UPDATE_PLAIN: return (void*)&k_update<CL, false, false, false>;
        case KERNEL_UPDATE_SPLIT: return (void*)&k_update<CL, true, false, true>;
        case KERNEL_UPDATE_PLAIN_SPLIT: return (void*)&k_update<CL, false, false, true>;
        case KERNEL_UPDATE_WALL:
            if constexpr( Closure<CL>::NS == 4 ) return (void*)&k_update<CL, true, true, false>;
            return nullptr;
        case KERNEL_UPDATE_PLAIN_WALL:
            if constexpr( Closure<CL>::NS == 4 ) return (void*)&k_update<CL, false, true, false>;
            return nullptr;
        case KERNEL_INIT:
            if( group == 32 ) return (void*)&k_init<CL, 32>;
            if( group == 256 ) return (void*)&k_init<CL, 256>;
            return nullptr;
        case KERNEL_MEANVAR:
            if( group == 32 ) return (void*)&k_meanvar<CL, 32>;
            if( group == 256 ) return (void*)&k_meanvar<CL, 256>;
            return nullptr;
        case KERNEL_CHECK: return (void*)&k_check<CL>;
        case KERNEL_PHASE_COUNTERS: {
#ifdef UQC_PHASE_TIMERS
            void* p = nullptr;
            return cudaGetSymbolAddress( &p, g_phaseCycles ) == cudaSuccess ? p : nullptr;
#else
            return nullptr;
#endif
        }
        case KERNEL_CHORD:
        case KERNEL_HESS_TC:
        case KERNEL_INVERT_RAW:
        case KERNEL_INVERT:
        case KERNEL_INVERT_SWEEP:
            if constexpr( CL == 1 ) {    // the mixed form in rounds serves the 2-D Euler closure
                if( which == KERNEL_CHORD ) return (void*)&k_chord<CL>;
                if( which == KERNEL_INVERT_SWEEP ) return (void*)&k_invert_sweep<CL>;
                if( which == KERNEL_HESS_TC ) return (void*)&k_hess_tc<CL>;
                if( which == KERNEL_INVERT_RAW ) return (void*)&k_invert<CL, true>;
                return (void*)&k_invert<CL, false>;
            }
            return nullptr;
        default: return nullptr;
    }
}

}    // namespace uqc
