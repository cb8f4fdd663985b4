// GpuClosure: the drop-in binding a UQCreator maintainer adds so that the
// reference's own MomentSolver (momentsolver.cpp:4-30, 79-162) solves its dual
// problems on the GPU through the C ABI of include/uqc.h.
//
// MomentSolver builds its closure with Closure::Create (closure.cpp:94-131) and
// calls SolveClosure(lambda, u, nTotal, nQTotal) per cell inside an OpenMP loop
// (momentsolver.cpp:83-89). The adapter subclasses the reference's closure
// classes (so U, DU, DS, EvaluateLambda* and the tables stay the reference's)
// and overrides SolveClosure with one uqc_closure_solve_host call on the cell's
// Matrix storage (column-major nStates x nTotal, UQC_LAYOUT_REF). The factory
// below stands for the one-line change in Closure::Create that selects it; the
// Makefile renames the reference's own factory symbol in a copy of closure.o
// (objcopy) so this definition is the one MomentSolver calls.
//
// Built by oracle/ref/Makefile as oracle/_ref/libuqcref_gpu.so (the reference
// harness plus this file, linked against uqcreator_b200/libuqc_b200.so); used
// by tests/test_gpu_adapter.py only.
#include <mutex>
#include <stdexcept>
#include <string>

#include "boundedbarrier.h"
#include "closure.h"
#include "eulerclosure2d.h"
#include "settings.h"
#include "shallowwaterclosure.h"
#include "uqc.h"

// the reference's own factory, renamed in closure_gpu.o
extern "C" Closure* uqcref_closure_create_reference( Settings* settings );

namespace {

template <class Base> class GpuClosure : public Base {
    uqc_solver* _h = nullptr;
    std::mutex _mutex;    // one handle: calls from the OpenMP loop are serialised

  public:
    explicit GpuClosure( Settings* s ) : Base( s ) {
        char err[512] = {0};
        if( uqc_create_from_file( s->GetInputFile().c_str(), nullptr, &_h, err, int( sizeof err ) ) != UQC_OK )
            throw std::runtime_error( std::string( "GpuClosure: " ) + err );
    }
    ~GpuClosure() override { uqc_destroy( _h ); }

    // closure.cpp:133-193, same signature and in-place semantics
    void SolveClosure( Matrix& lambda, const Matrix& u, unsigned nTotal, unsigned ) override {
        std::lock_guard<std::mutex> lock( _mutex );
        int status   = 0;
        unsigned nt  = nTotal;
        const int rc = uqc_closure_solve_host( _h, 1, lambda.GetPointer(), const_cast<Matrix&>( u ).GetPointer(), &nt, UQC_LAYOUT_REF, &status );
        // the reference logs and exits on a failed closure (closure.cpp:180-192)
        if( rc != UQC_OK || status != UQC_CELL_CONVERGED ) throw std::runtime_error( std::string( "GpuClosure: " ) + uqc_last_error( _h ) );
    }
};

}    // namespace

// Closure::Create with the GPU closure selected for the closures the C ABI serves.
Closure* Closure::Create( Settings* settings ) {
    switch( settings->GetClosureType() ) {
        case ClosureType::C_BOUNDEDBARRIER: return new GpuClosure<BoundedBarrier>( settings );
        case ClosureType::C_EULER_2D: return new GpuClosure<EulerClosure2D>( settings );
        case ClosureType::C_SHALLOWWATER_1D: return new GpuClosure<ShallowWaterClosure>( settings );
        default: return uqcref_closure_create_reference( settings );
    }
}
