// GpuMomentSolver: the drop-in for MomentSolver (momentsolver.h:139-147) that a
// UQCreator maintainer adds to run the whole time loop on the GPU through the
// C ABI of include/uqc.h. Same constructor (Settings*, Mesh*, Problem*) and
// Solve(); main.cpp (:205-207) constructs it instead of MomentSolver.
//
// Solve() does what MomentSolver::Solve (momentsolver.cpp:36-229) leaves behind:
// - the initial state, including a restart from the previous run's files and
//   configuration echo (DetermineMoments / SetDuals, :418-523): uqc_init_state;
// - the time loop to tEnd or minResidual (:79-162): uqc_step in slices;
// - the mean and variance after the steps with timeIndex % writeFrequency == 1
//   (:156-160), exported through the reference's Mesh as "_<timeIndex>";
// - the final mean and variance (WriteMeanAndVar, Mesh::Export(.., ""), :224);
// - the final moments and duals through the "moments" and "duals" loggers in
//   MomentSolver::Export's format (:565-588).
// Not reproduced: the per-step "t residual" log lines, error files against a
// reference solution (WriteErrors) and the refinement-indicator exports.
//
// Built by oracle/ref/Makefile into oracle/_ref/libuqcref_gpu.so with
// gpuclosure.cpp; uqcref_gpu_moment_solver_run is the harness's entry
// (tests/test_gpu_adapter.py).
#include <algorithm>
#include <cstring>
#include <iomanip>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "mesh.h"
#include "problem.h"
#include "settings.h"
#include "spdlog/spdlog.h"
#include "typedefs.h"
#include "uqc.h"

namespace {

class GpuMomentSolver {
    Settings* _settings;
    Mesh* _mesh;
    Problem* _problem;
    uqc_solver* _h = nullptr;
    uqc_info _info{};

    // every error, a failed closure included, ends the solve (the reference
    // exits on a failed closure, closure.cpp:180-192)
    void check( int rc ) const {
        if( rc != UQC_OK ) throw std::runtime_error( std::string( "GpuMomentSolver: " ) + uqc_last_error( _h ) );
    }

    Matrix mean_and_var() const {
        const unsigned nS = unsigned( _info.n_states ), N = unsigned( _info.n_cells );
        std::vector<double> mv( size_t( N ) * 2 * nS );
        check( uqc_mean_var( _h, mv.data() ) );
        Matrix out( 2 * nS, N, 0.0 );
        for( unsigned j = 0; j < N; ++j )
            for( unsigned r = 0; r < 2 * nS; ++r ) out( r, j ) = mv[size_t( j ) * 2 * nS + r];
        return out;
    }

  public:
    GpuMomentSolver( Settings* settings, Mesh* mesh, Problem* problem ) : _settings( settings ), _mesh( mesh ), _problem( problem ) {
        char err[512] = {0};
        if( uqc_create_from_file( settings->GetInputFile().c_str(), nullptr, &_h, err, int( sizeof err ) ) != UQC_OK )
            throw std::runtime_error( std::string( "GpuMomentSolver: " ) + err );
        uqc_get_info( _h, &_info );
        if( unsigned( _info.n_cells ) != mesh->GetNumCells() ) throw std::runtime_error( "GpuMomentSolver: the mesh differs from the input file's" );
    }
    ~GpuMomentSolver() { uqc_destroy( _h ); }
    GpuMomentSolver( const GpuMomentSolver& ) = delete;
    GpuMomentSolver& operator=( const GpuMomentSolver& ) = delete;

    void Solve() {
        check( uqc_init_state( _h ) );
        const long long wf = std::max( 1, _settings->GetWriteFrequency() );
        long long timeIndex = 0;
        uqc_step_info si{};
        for( ;; ) {
            // the next step after which the reference exports: timeIndex % wf == 1
            long long next = wf == 1 ? -1 : ( timeIndex < 1 ? 1 : ( ( timeIndex - 1 ) / wf + 1 ) * wf + 1 );
            const long long slice = next < 0 ? 256 : std::min<long long>( 256, next - timeIndex );
            check( uqc_step( _h, int( slice ), &si ) );
            timeIndex += si.steps;
            if( si.steps == slice && timeIndex == next ) _mesh->Export( mean_and_var(), "_" + std::to_string( timeIndex ) );
            if( !si.running ) break;
        }
        _mesh->Export( mean_and_var(), "" );
        // MomentSolver::Export: one line per cell, the (state, moment) entries
        // with 15 significant digits, each followed by a comma
        const size_t N = size_t( _info.n_cells ), nS = size_t( _info.n_states ), nT = size_t( _info.n_total );
        std::vector<double> u( N * nS * nT ), lam( N * nS * nT );
        std::vector<unsigned> level( N );
        check( uqc_download_state( _h, u.data(), lam.data(), level.data(), UQC_LAYOUT_REF ) );
        for( int which = 0; which < 2; ++which ) {
            auto writer           = spdlog::get( which == 0 ? "moments" : "duals" );
            const std::vector<double>& v = which == 0 ? u : lam;
            for( size_t i = 0; i < N; ++i ) {
                std::stringstream line;
                for( size_t j = 0; j < nS; ++j )
                    for( size_t k = 0; k < nT; ++k )
                        line << std::setprecision( std::numeric_limits<double>::digits10 ) << v[i * nS * nT + k * nS + j] << ",";
                writer->info( line.str() );
            }
            writer->flush();
        }
    }
};

}    // namespace

// The harness's entry: GpuMomentSolver(settings, mesh, problem).Solve().
extern "C" int uqcref_gpu_moment_solver_run( Settings* settings, Mesh* mesh, Problem* problem, char* err, int errlen ) {
    try {
        GpuMomentSolver solver( settings, mesh, problem );
        solver.Solve();
        return 0;
    } catch( const std::exception& e ) {
        if( err && errlen > 0 ) {
            std::strncpy( err, e.what(), size_t( errlen - 1 ) );
            err[errlen - 1] = 0;
        }
        return -1;
    }
}
