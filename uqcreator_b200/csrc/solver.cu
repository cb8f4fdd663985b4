// Host orchestration and C ABI (include/uqc.h) of the B200 IPM solver.
//
// One uqc_solver = the reference's Settings + Mesh + Problem + Closure +
// MomentSolver for one run, with the whole state resident in HBM:
//   u, lambda   cell-major, state-major inside a cell (nS * nT doubles per cell)
//   uQ          nodal states, nS * nQ doubles per cell (FP64)
//   geometry    structure-of-arrays per cell / face
// A time step is two kernel launches (k_closure in step mode, k_update); the
// loop condition, dt and residual live in a device Control block, so steps
// need no host synchronisation and are captured into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <chrono>
#include <deque>
#include <map>
#include <new>
#include <string>
#include <vector>

#include "host.h"
#include "chord.cuh"
#include "ipm_kernels.cuh"
#include "kernels.h"
#include "uqc.h"

using namespace uqc;

struct uqc_solver {
    Config cfg;
    Tables tab;
    Mesh mesh;
    cudaStream_t stream     = nullptr;
    cudaStream_t userStream = nullptr;
    bool ownStream          = false;
    bool deviceReady        = false;
    int nS = 1, ld = 1, group = 32, numSMs = 148;
    int closureGroup = 32, closureGroupOverride = 0;    // threads per cell in k_closure (32, 64 or 256)
    int tinyOpt = -1;                  // option closure_tiny: -1 automatic, 0 off, 1 on where it applies
    int updateWarpsOpt = 0, checkWarpsOpt = 0, chordWarpsOpt = 0;    // options update_warps, check_warps, chord_warps (0: automatic)
    int blockPartialCap = 0;           // doubles in d_blockPartial
    double* d_chunkPartial = nullptr;  // uqc_step_host's chunked update: a partial per CTA and launch
    int chunkPartialCap    = 0;
    bool closureTiny = false;          // planned: the register Newton of tiny systems (k_closure TINY)
    int tinyGrid     = 0;
    size_t ldc = 1;
    // device buffers
    double *d_phi = nullptr, *d_phiWf = nullptr, *d_xi = nullptr;
    double *d_area = nullptr, *d_dx = nullptr, *d_center = nullptr, *d_unitN = nullptr, *d_scaledN = nullptr;
    int *d_nbr = nullptr, *d_boundary = nullptr;
    double* d_bndNormal = nullptr;    // wall meshes only
    double *d_u = nullptr, *d_lam = nullptr, *d_uQ = nullptr, *d_uOld0 = nullptr, *d_blockPartial = nullptr;
    unsigned* d_level = nullptr;
    int *d_status = nullptr, *d_iters = nullptr;
    Control* d_ctl = nullptr;
    Control* h_ctl = nullptr;    // pinned mirror
    // closure-only scratch for caller-owned batches (grow-only)
    double *d_xLam = nullptr, *d_xU = nullptr;
    unsigned* d_xNt = nullptr;
    int *d_xStatus = nullptr, *d_xIters = nullptr;
    size_t xCap = 0;
    // launch shapes
    int closureBlock = 256, closureGrid = 0, updateBlock = 256, updateGrid = 0, auxGrid = 0, auxBlock = 256;
    size_t closureSmem = 0, updateSmem = 0, initSmem = 0, mvSmem = 0, checkSmem = 0;
    int checkBlock = 256, checkGrid = 0;
    int* d_activeList = nullptr;    // cells that need Newton: two lists (running step, next step)
    double* d_cellDt  = nullptr;    // per cell: CFL step of its nodal states
    double* d_uRe     = nullptr;    // moments re-projected by the closure epilogue (input of k_update)
    int* d_checkList  = nullptr;    // two lists: converged cells whose level changes (k_check's epilogue)
    unsigned char* d_finFlag = nullptr;    // per cell: finished by k_update for the next step
    bool tablesInSmem        = false;    // check / update / init kernels stage the tables in shared memory
    bool closureTablesInSmem = false;    // ... the FP64 closure kernel
    int closureTablesOpt     = -1;       // option closure_tables_smem: -1 automatic, 0 read through L1, 1 stage
    // mixed form: FP32 Hessian / factor / solves, FP64 gradient and update
    float* d_phiF        = nullptr;    // phi rounded to FP32, row stride ld
    int* d_fallbackList  = nullptr;    // cells the mixed form hands to the FP64 form
    bool mixedOk         = false;
    std::string mixedWhy = "not planned";
    int mixedGroup = 64, mixedBlock = 256, mixedGrid = 0;
    int mixedMaxIter = 0;    // Newton iterations of the FP32 pass before the FP64 form takes over (0: the configured limit)
    // mixed form: each cell's last FP32 factor, reused by the chord Newton of later iterations and steps
    float* d_factorStore = nullptr;
    int* d_factorLevel   = nullptr;
    int factorStride     = 0;
    bool chord           = true;
    bool chordInverse    = false;    // planned: the mixed workspace holds the packed factor inverse
    bool chordInverseOpt = true;     // option mixed_chord_inverse
    double chordTheta    = 0.0;      // option mixed_chord_theta; 0: automatic (0.2 with rounds, 0.1 in the single kernel)
    size_t mixedSmem       = 0;
    bool mixedTablesInSmem = false;
    // mixed form in rounds (chord.cuh; 2-D Euler with one refinement level):
    // k_chord, then per round k_hess_tc / k_invert and k_chord again
    int roundsOpt   = -1;    // option mixed_hessian: -1 automatic, 0 single kernel, 1 CUDA-core Hessian, 2 tensor cores
    int v2Mode      = 0;     // planned: 0 off, 1 rounds with the CUDA-core Hessian, 2 with the tensor-core Hessian
    int v2Rounds    = 2;     // option mixed_rounds
    std::string v2Why;       // why the rounds (or the tensor cores) are not used
    double* d_gStore        = nullptr;
    int gStride             = 0;
    int* d_v2Lists          = nullptr;
    int* d_chordIters       = nullptr;
    unsigned short* d_qTiles = nullptr;
    int chordBlock = 512, chordGrid = 0, hessGrid = 0, invBlock = 256, invGrid = 0;
    size_t chordSmem = 0, hessSmem = 0, invSmem = 0;
    bool chordTablesInSmem = false;
    bool invSweep          = false;    // the inverse kernel is k_invert_sweep
    // bookkeeping
    bool stateReady = false;
    int precision   = 0;
    int launches    = 0;
    unsigned long long lastIters = 0, lastLs = 0, lastFallback = 0;
    int lastFailed = 0;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t asyncEv   = nullptr;    // end of the last uqc_step_async batch
    bool asyncPending     = false;
    int asyncStepsBefore  = 0;
    std::vector<cudaEvent_t> stepEvents;
    cudaStream_t copyStream = nullptr;       // uqc_step_host: the uploads beside the kernels
    cudaStream_t copyStreamOut = nullptr;    // ... and the downloads (the other copy direction)
    cudaStream_t checkStream   = nullptr;    // ... and its chunks' convergence checks
    std::vector<cudaEvent_t> hostEvents;     // uqc_step_host: chunk arrivals and phase ends
    int hostChunks = 6;                      // uqc_step_host: chunks of cells (option host_chunks; 2-D Euler,
                                             // 200k cells: 9.55 / 9.32 / 9.58 / 11.1 / 11.7 ms per step at 4 / 6 / 8 / 12 / 16)
    float lastMs[3] = {0, 0, 0};
    // CUDA graphs of n whole time steps (uqc_run, uqc_step_async), rebuilt
    // when anything the kernels' arguments hold changes (planGen)
    std::map<int, std::pair<cudaGraphExec_t, int>> graphs;    // n -> (graph, kernel launches)
    int planGen = 0, graphGen = 0;
    bool useGraphs = true;
    int finishInUpdateOpt = -1;    // option update_test: 1 on, 0 off, -1 automatic
    std::vector<double> padPhi, padPhiWf;    // host tables in the device layout
    std::vector<double> padWt;               // w_k / 2^dimXi per node
    double* d_wt = nullptr;
    std::string cfgText;                     // the input file's text (echoed by uqc_export_state)
    std::string cfgName = "uqcreator_b200";  // the input file's path, when created from a file
    double area0 = 0.0;                      // area of the global mesh's first cell (TimeSolver's fixed dt)
    // linear closures: the filter factors (host, device)
    std::vector<double> filterHost, lassoParamHost, lassoL1Host;
    double *d_filter = nullptr, *d_lassoParam = nullptr, *d_lassoL1 = nullptr;
    // spatial sharding (uqc_partition): the mesh is this rank's owned cells and halo
    bool sharded = false;
    ShardPlan shard;
    int* d_sendCells = nullptr;
    std::string err;
};

namespace {

struct CudaError : public std::runtime_error {
    explicit CudaError( const std::string& m ) : std::runtime_error( m ) {}
};
#define CK( x )                                                                                                                      \
    do {                                                                                                                             \
        cudaError_t e_ = ( x );                                                                                                      \
        if( e_ != cudaSuccess ) throw CudaError( std::string( #x ) + ": " + cudaGetErrorName( e_ ) + " " + cudaGetErrorString( e_ ) ); \
    } while( 0 )

int fail( uqc_solver* h, int code, const std::string& m ) {
    if( h ) h->err = m;
    return code;
}

template <class F> int guarded( uqc_solver* h, F&& f ) {
    try {
        return f();
    } catch( const ConfigError& e ) {
        return fail( h, UQC_ERR_CONFIG, e.what() );
    } catch( const CudaError& e ) {
        std::string m = e.what();
        return fail( h, m.find( "MemoryAllocation" ) != std::string::npos ? UQC_ERR_MEMORY : UQC_ERR_CUDA, m );
    } catch( const std::bad_alloc& ) {
        return fail( h, UQC_ERR_MEMORY, "host allocation failed" );
    } catch( const std::exception& e ) {
        return fail( h, UQC_ERR_ARGUMENT, e.what() );
    }
}

void ensure_device( uqc_solver* h );
void build_filters( uqc_solver* h );

// guarded() for entry points that touch the device
template <class F> int guarded_dev( uqc_solver* h, F&& f ) {
    return guarded( h, [&] {
        ensure_device( h );
        return f();
    } );
}

template <class T> T* dalloc( size_t n ) {
    T* p = nullptr;
    CK( cudaMalloc( &p, std::max<size_t>( n, 1 ) * sizeof( T ) ) );
    return p;
}
template <class T> T* dupload( const std::vector<T>& v, size_t extra = 0 ) {
    T* p = dalloc<T>( v.size() + extra );
    if( extra ) CK( cudaMemset( p, 0, ( v.size() + extra ) * sizeof( T ) ) );
    if( !v.empty() ) CK( cudaMemcpy( p, v.data(), v.size() * sizeof( T ), cudaMemcpyHostToDevice ) );
    return p;
}

// Whether k_update tests the next step's convergence (option update_test;
// automatic: with a single refinement level. With several, cells whose level
// flips every step still need the check kernel's epilogue, which then costs
// as much as testing every cell there).
bool update_test_on( const uqc_solver* h ) {
    const bool on = h->finishInUpdateOpt == -1 ? h->tab.nLevels == 1 : h->finishInUpdateOpt != 0;
    // a linear closure's duals follow the new moments: every cell goes through k_check
    return h->cfg.newtonMode != 2 && on && !closure_linear( h->cfg.closure );
}

// The update kernel instance: with or without the next step's test (fin),
// for meshes with walls, or (no walls) with the node-split projection when a
// level's last block of 32 basis functions holds 1-16 of them.
int update_kernel_id( const uqc_solver* h, bool fin ) {
    if( h->d_bndNormal != nullptr ) return fin ? KERNEL_UPDATE_WALL : KERNEL_UPDATE_PLAIN_WALL;
    bool split = false;
    for( int n : h->tab.nTLevel ) split = split || ( n % 32 >= 1 && n % 32 <= 16 );
    if( split ) return fin ? KERNEL_UPDATE_SPLIT : KERNEL_UPDATE_PLAIN_SPLIT;
    return fin ? KERNEL_UPDATE : KERNEL_UPDATE_PLAIN;
}

KParams make_params( const uqc_solver* h ) {
    KParams P{};
    P.nS      = h->nS;
    P.nT      = h->tab.nT;
    P.nQ      = h->tab.nQ;
    P.ld      = h->ld;
    P.nLevels = h->tab.nLevels;
    for( int l = 0; l < h->tab.nLevels; ++l ) P.nTLevel[l] = h->tab.nTLevel[l];
    P.filterKind   = h->cfg.filterKind;
    P.filter       = h->d_filter;
    P.lassoParam   = h->d_lassoParam;
    P.lassoL1      = h->d_lassoL1;
    P.refIndicator = h->cfg.refIndicator;
    P.refDown      = h->cfg.refDown;
    P.refUp        = h->cfg.refUp;
    P.nRet         = int( h->cfg.retResiduals.size() );
    for( int k = 0; k < P.nRet; ++k ) P.retRes[k] = h->cfg.retResiduals[k];
    for( int k = 0; k < int( h->cfg.retLevels.size() ); ++k ) P.retLev[k] = h->cfg.retLevels[k];
    P.nCells     = h->mesh.nCells;
    P.nWork      = h->mesh.nCells;    // a time step works on the owned cells only (step_lists)
    P.nFaces     = h->mesh.nFaces;
    P.dimXi      = h->tab.dimXi;
    P.eps        = h->cfg.epsilon;
    P.maxIter    = h->cfg.maxIterations;
    P.newtonMode = h->cfg.newtonMode;
    PhysParams& ph = P.phys;
    ph.bbMinus     = h->cfg.bbMinus;
    ph.bbPlus      = h->cfg.bbPlus;
    ph.gamma       = h->cfg.gamma;
    ph.eulerA      = 1.0 / ( 1.0 - h->cfg.gamma );
    ph.cfl         = h->cfg.cfl;
    for( size_t i = 0; i < h->cfg.ic.size() && i < 8; ++i ) ph.ic[i] = h->cfg.ic[i];
    ph.nIc = int( std::min<size_t>( h->cfg.ic.size(), 8 ) );
    for( size_t i = 0; i < h->cfg.sigma.size() && i < 4; ++i ) ph.sigma[i] = h->cfg.sigma[i];
    ph.dimXi   = h->tab.dimXi;
    ph.dtFixed = h->area0 * h->cfg.cfl / 12.0;    // TimeSolver (timesolver.cpp:4-9)
    P.phi          = h->d_phi;
    P.phiWf        = h->d_phiWf;
    P.xi           = h->d_xi;
    P.wt           = h->d_wt;
    P.phiF         = h->d_phiF;
    P.tablesInSmem = h->tablesInSmem;
    P.area         = h->d_area;
    P.dx           = h->d_dx;
    P.center       = h->d_center;
    P.unitN        = h->d_unitN;
    P.scaledN      = h->d_scaledN;
    P.nbr          = h->d_nbr;
    P.boundary     = h->d_boundary;
    P.bndNormal    = h->d_bndNormal;
    P.u            = h->d_u;
    P.lam          = h->d_lam;
    P.uQ           = h->d_uQ;
    P.uOld0        = h->d_uOld0;
    P.cellDt       = h->d_cellDt;
    // re-projected moments: a buffer of their own when k_update tests the next
    // step's convergence (it needs them next to u_new), else u itself (in place)
    P.uRe          = update_test_on( h ) ? h->d_uRe : h->d_u;
    P.level        = h->d_level;
    P.nTotalCell   = nullptr;
    P.status       = h->d_status;
    P.iters        = h->d_iters;
    P.blockPartial  = h->d_blockPartial;
    P.updChunk      = 0;
    P.updChunks     = 1;
    P.ctl           = h->d_ctl;
    P.workCounter   = h->d_ctl ? &h->d_ctl->workCounter : nullptr;
    P.fallbackList  = h->d_fallbackList;
    const bool useStore = h->precision == UQC_MIXED && h->chord && h->d_factorStore;
    P.factorStore       = useStore ? h->d_factorStore : nullptr;
    P.factorLevel       = useStore ? h->d_factorLevel : nullptr;
    P.factorStride      = h->factorStride;
    P.chordInverse      = useStore && h->chordInverse ? 1 : 0;
    P.chordTheta        = h->chordTheta > 0.0 ? h->chordTheta : ( h->v2Mode ? 0.2 : 0.1 );
    // the mixed form in rounds: k_check / k_update store the gradient of the
    // cells they list (gStore non-null) only when the rounds run
    const bool rounds = useStore && h->v2Mode && h->d_gStore;
    P.gStore          = rounds ? h->d_gStore : nullptr;
    P.gStride         = h->gStride;
    P.v2Lists         = rounds ? h->d_v2Lists : nullptr;
    P.v2Rounds        = h->v2Rounds;
    P.chordIters      = rounds ? h->d_chordIters : nullptr;
    P.qTiles          = h->d_qTiles;
    P.fallbackCount = h->d_ctl ? &h->d_ctl->nFallback : nullptr;
    return P;
}

// ---- kernel dispatch on (closure kind, group size) ------------------------
// The kernels are instantiated per closure kind in kernels_<kind>.cu (three
// translation units compiled in parallel); each exports its kernel addresses.
void* pick( int cl, int group, int which ) {
    void* fn = nullptr;
    if( cl == 0 ) fn = kernel_bounded_barrier( group, which );
    if( cl == 1 ) fn = kernel_euler2d( group, which );
    if( cl == 2 ) fn = kernel_shallow_water( group, which );
    if( closure_linear( cl ) && cl != CL_LINEAR_EULER1D ) fn = kernel_linear( cl, group, which );
    if( cl == CL_EULER1D || cl == CL_LINEAR_EULER1D ) fn = kernel_euler1d( cl, group, which );
    if( cl == CL_LOGSIN ) fn = kernel_logsin( group, which );
    if( !fn ) throw ConfigError( "no kernel for this closure" );
    return fn;
}

void* pick_check( int cl ) { return pick( cl, 32, KERNEL_CHECK ); }

int closure_np( int cl ) {
    const int ns = closure_states( cl );
    return ns * ( ns + 1 ) / 2;
}

// Dynamic shared memory limit of a kernel: the attribute belongs to the
// kernel function, for the whole process, so every handle sets it to the
// device's opt-in maximum (a handle that set its own smaller need would break
// another handle's larger launch of the same kernel).
void allow_dynamic_smem( const void* fn ) {
    int dev = 0, maxSmem = 0;
    CK( cudaGetDevice( &dev ) );
    CK( cudaDeviceGetAttribute( &maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev ) );
    cudaFuncAttributes fa;
    CK( cudaFuncGetAttributes( &fa, fn ) );    // the limit counts static shared memory too
    CK( cudaFuncSetAttribute( fn, cudaFuncAttributeMaxDynamicSharedMemorySize, maxSmem - int( fa.sharedSizeBytes ) ) );
}

void launch( uqc_solver* h, void* fn, int grid, int block, size_t smem, void** args ) {
    CK( cudaLaunchKernel( fn, dim3( grid ), dim3( block ), args, smem, h->stream ) );
    ++h->launches;
}

// Factor store of the mixed form: floats per cell (tiles + pivot inverses of
// the finest level, padded to 16 bytes) and its total bytes.
// Floats per cell of the factor store: the factor tiles and inverse pivots,
// or the packed inverse (whichever is larger, so the planner may switch).
int factor_stride( const uqc_solver* h ) {
    const int n = h->nS * h->tab.nT;
    size_t f    = std::max<size_t>( hess_doubles( n ) + size_t( hnb( n ) ) * 8, size_t( xpacked( n ) ) );
    if( h->cfg.closure == 1 ) {    // the rounds' inverse (n x n) and tensor-core values (pairs x blocks)
        const size_t pairs = size_t( h->tab.nT ) * ( h->tab.nT + 1 ) / 2;
        f                  = std::max( f, std::max( size_t( n ) * n, pairs * size_t( closure_np( 1 ) ) ) );
    }
    return int( ( f + 3 ) & ~size_t( 3 ) );
}
unsigned long long factor_store_bytes( const uqc_solver* h ) {
    const unsigned long long N = (unsigned long long)h->mesh.nCells;
    // the rounds' gradient store, lists and iteration counts (2-D Euler)
    const unsigned long long rounds = h->cfg.closure == 1 ? N * ( ( h->ldc + 2 + 3 ) / 4 * 4 * 8 + 4 * 4 ) : 0;
    return N * ( (unsigned long long)factor_stride( h ) * 4 + 4 ) + rounds;
}
// Allocates the store on first use; marks every stored factor invalid.
void reset_factor_store( uqc_solver* h ) {
    const size_t N = size_t( h->mesh.nCells );
    if( !h->d_factorStore ) {
        h->factorStride  = factor_stride( h );
        h->d_factorStore = dalloc<float>( N * h->factorStride );
        h->d_factorLevel = dalloc<int>( N );
    }
    if( h->v2Mode && !h->d_gStore ) {
        h->gStride      = int( ( h->ldc + 2 + 3 ) & ~size_t( 3 ) );
        h->d_gStore     = dalloc<double>( N * h->gStride );
        h->d_v2Lists    = dalloc<int>( 3 * N );
        h->d_chordIters = dalloc<int>( N );
    }
    CK( cudaMemsetAsync( h->d_factorLevel, 0xFF, N * sizeof( int ), h->stream ) );
}

// Round-to-nearest-even BF16 bits of a float.
unsigned short bf16_bits( float f ) {
    unsigned u;
    std::memcpy( &u, &f, 4 );
    if( ( u & 0x7F800000u ) == 0x7F800000u ) return (unsigned short)( u >> 16 );    // inf / nan
    u += 0x7FFFu + ( ( u >> 16 ) & 1u );
    return (unsigned short)( u >> 16 );
}
float bf16_value( unsigned short b ) {
    unsigned u = unsigned( b ) << 16;
    float f;
    std::memcpy( &f, &u, 4 );
    return f;
}

// Mixed form in rounds: eligibility, launch shapes, and the tensor-core
// table Q (pairs j <= i x nodes, Q = phi_kj phi_ki wt_k, high and low BF16
// parts in the K-major operand layout of k_hess_tc).
void plan_rounds( uqc_solver* h, int maxSmem ) {
    h->v2Mode = 0;
    const int cl = h->cfg.closure, nT = h->tab.nT, nQ = h->tab.nQ, nS = h->nS;
    if( h->roundsOpt == 0 ) {
        h->v2Why = "option mixed_hessian = 0";
        return;
    }
    if( cl != 1 || h->tab.nLevels != 1 || h->cfg.newtonMode == 2 || h->cfg.maxIterations < 2 || !h->chord ) {
        h->v2Why = "rounds serve the 2-D Euler closure with one refinement level, SolveClosure Newton, maxIterations > 1 and the chord form";
        return;
    }
    const int NP = closure_np( cl );
    // chord kernel: tables in shared memory when that leaves room for 8 cells
    const size_t tables = 2 * ( size_t( nQ ) * h->ld + 4 ) * sizeof( double );
    const size_t ws     = chord_ws_doubles( nS, nT, nQ ) * sizeof( double );
    h->chordTablesInSmem = tables <= 96 * 1024 && tables + 8 * ws <= size_t( maxSmem );
    const size_t avail   = size_t( maxSmem ) - ( h->chordTablesInSmem ? tables : 0 );
    const int warps      = int( std::min<size_t>( h->chordWarpsOpt ? h->chordWarpsOpt : 16, avail / ws ) );
    if( warps < 1 ) {
        h->v2Why = "chord workspace exceeds shared memory";
        return;
    }
    h->chordBlock = 32 * warps;
    h->chordSmem  = ( h->chordTablesInSmem ? tables : 0 ) + size_t( warps ) * ws;
    int occ       = 0;
    void* kc      = pick( cl, 32, KERNEL_CHORD );
    allow_dynamic_smem( kc );
    CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kc, h->chordBlock, h->chordSmem ) );
    h->chordGrid = std::max( 1, occ ) * h->numSMs;
    // tensor cores when the table fits one MMA's N (256) and shared memory
    const TcShape ts    = tc_shape( nS, NP, nT, nQ );
    const size_t hsmem  = hess_tc_smem( nS, NP, nT, nQ, h->ld );
    const bool tcFits   = ts.nPad <= 256 && ts.cellsPerTile >= 1 && hsmem <= size_t( maxSmem );
    int mode            = h->roundsOpt == 1 ? 1 : ( tcFits ? 2 : 1 );
    if( !tcFits && h->roundsOpt != 1 ) {
        // automatic: without the tensor-core Hessian the single kernel is faster
        // (measured on the three-uncertainty workload: 41 vs 50 ms per step)
        h->v2Why = "tensor-core Hessian: " + std::to_string( ts.pairs ) + " basis pairs or " + std::to_string( hsmem ) +
                   " B of shared memory exceed one MMA (256 pairs)";
        return;
    }
    // inverse kernel: by sweeps in registers (four warps per cell, four cells
    // per CTA) for n <= 84 after the tensor-core Hessian; else Cholesky and
    // triangular inverse, two warps per cell, as many cells (up to 4) as fit
    h->invSweep = mode == 2 && nS * nT <= 4 * SWEEP_RG && nS * nT <= 32 * SWEEP_CW;
    void* ki    = nullptr;
    if( h->invSweep ) {
        h->invBlock = 512;
        h->invSmem  = 4 * sweep_ws_floats( nT * ( nT + 1 ) / 2, NP ) * sizeof( float );
        ki          = pick( cl, 32, KERNEL_INVERT_SWEEP );
    }
    else {
        const size_t iws = invert_ws_bytes( nS * nT, nQ, NP, mode == 2 );
        const int groups = int( std::min<size_t>( 4, size_t( maxSmem ) / iws ) );
        if( groups < 1 ) {
            h->v2Why = "inverse workspace exceeds shared memory";
            return;
        }
        h->invBlock = 64 * groups;
        h->invSmem  = iws * groups;
        ki          = pick( cl, 32, mode == 2 ? KERNEL_INVERT_RAW : KERNEL_INVERT );
    }
    allow_dynamic_smem( ki );
    CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, ki, h->invBlock, h->invSmem ) );
    h->invGrid = std::max( 1, occ ) * h->numSMs;
    if( mode == 2 ) {
        h->hessSmem = hsmem;
        void* kh    = pick( cl, 32, KERNEL_HESS_TC );
        allow_dynamic_smem( kh );
        h->hessGrid = h->numSMs;
        if( !h->d_qTiles ) {
            std::vector<unsigned short> q( 2 * ts.qBytes / 2, 0 );
            for( int i = 0; i < nT; ++i )
                for( int j = 0; j <= i; ++j ) {
                    const int pr = i * ( i + 1 ) / 2 + j;
                    for( int k = 0; k < nQ; ++k ) {
                        const double v =
                            h->tab.phi[size_t( k ) * nT + j] * h->tab.phi[size_t( k ) * nT + i] * h->padWt[k];
                        const unsigned short hi = bf16_bits( float( v ) );
                        const unsigned short lo = bf16_bits( float( v - double( bf16_value( hi ) ) ) );
                        const size_t off        = umma_kmajor_offset( pr, k, ts.nPad ) / 2;
                        q[off]                  = hi;
                        q[ts.qBytes / 2 + off]  = lo;
                    }
                }
            h->d_qTiles = dupload( q );
        }
    }
    h->v2Mode = mode;
    h->v2Why.clear();
}

// Mixed-form closure: the FP32 Hessian halves the per-cell shared memory, so
// more cells share an SM: a warp per cell (n <= 32) or two warps per cell, up
// to 8 or 4 cells per CTA; the tables gain an FP32 copy of phi.
void plan_mixed( uqc_solver* h, int maxSmem ) {
    const int cl = h->cfg.closure, nT = h->tab.nT, nQ = h->tab.nQ, nS = h->nS;
    if( closure_linear( cl ) ) {
        h->mixedOk  = false;
        h->mixedWhy = "a linear closure (stochastic Galerkin or a filter) has no Newton system";
        return;
    }
    const size_t n       = size_t( nS ) * nT;
    const size_t tn      = size_t( nQ ) * h->ld + 4;
    const size_t tables  = 2 * tn * sizeof( double ) + ( tn + 1 ) / 2 * sizeof( double );
    const size_t ws0     = cell_ws_doubles( nS, nT, nQ, closure_np( cl ), 4 ) * sizeof( double );
    h->mixedTablesInSmem = h->closureTablesOpt != 0 && tables <= 112 * 1024 && tables + 2 * ws0 <= size_t( maxSmem );
    const size_t avail   = size_t( maxSmem ) - ( h->mixedTablesInSmem ? tables : 0 );
    const int fit0       = int( std::min<size_t>( 8, avail / ws0 ) );
    if( fit0 < 1 ) {
        h->mixedOk  = false;
        h->mixedWhy = "mixed-form closure workspace (" + std::to_string( ws0 ) + " B per cell) exceeds shared memory";
        return;
    }
    h->mixedGroup = n <= 32 ? 32 : 64;
    // chord directions from the packed inverse of the held factor (two
    // independent-output mat-vecs instead of two triangular solves), when its
    // shared memory costs no cell per CTA
    const int cap         = h->mixedGroup == 32 ? 8 : 4;
    const size_t wsX      = cell_ws_doubles( nS, nT, nQ, closure_np( cl ), 4, xpacked( int( n ) ) ) * sizeof( double );
    const int fitX        = int( std::min<size_t>( 8, avail / wsX ) );
    h->chordInverse       = h->chord && h->chordInverseOpt != 0 && std::min( cap, fitX ) >= std::min( cap, fit0 );
    const size_t wsCell   = h->chordInverse ? wsX : ws0;
    const int fit         = h->chordInverse ? fitX : fit0;
    h->mixedBlock = h->mixedGroup * std::min( cap, fit );
    h->mixedSmem  = wsCell * ( h->mixedBlock / h->mixedGroup ) + ( h->mixedTablesInSmem ? tables : 0 );
    void* k       = pick( cl, h->mixedGroup, 4 );
    allow_dynamic_smem( k );
    int occ = 0;
    CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, k, h->mixedBlock, h->mixedSmem ) );
    h->mixedGrid = std::max( 1, occ ) * h->numSMs;
    h->mixedOk   = true;
    h->mixedWhy.clear();
}

// Launch shape of the FP64 closure kernel k_closure for a handle's
// configuration: threads per cell (group), threads per CTA, dynamic shared
// memory and whether the basis tables are staged in it. Shared by the
// allocating entry points (plan_launches) and the no-alloc closure.
struct ClosureShape {
    int group = 32, block = 256;
    size_t smem       = 0;
    bool tablesInSmem = false;
};

ClosureShape fp64_closure_shape( const uqc_solver* h, int maxSmem ) {
    const int cl = h->cfg.closure, nT = h->tab.nT, nQ = h->tab.nQ, nS = h->nS;
    const size_t n      = size_t( nS ) * nT;
    const size_t tables = 2 * ( size_t( nQ ) * h->ld + 4 ) * sizeof( double );
    const size_t wsCell = cell_ws_doubles( nS, nT, nQ, closure_np( cl ) ) * sizeof( double );
    const bool canStage = tables <= 96 * 1024 && tables + wsCell <= size_t( maxSmem );
    ClosureShape s;
    {
        // automatic: read the tables through L1 when that lets more cells share a CTA
        const int cap     = n <= 32 ? 8 : 4;
        const int staged  = canStage ? int( std::min<size_t>( cap, ( size_t( maxSmem ) - tables ) / wsCell ) ) : 0;
        const int through = int( std::min<size_t>( cap, size_t( maxSmem ) / wsCell ) );
        s.tablesInSmem    = canStage && ( h->closureTablesOpt == 1 || ( h->closureTablesOpt == -1 && staged >= through ) );
    }
    const size_t avail = size_t( maxSmem ) - ( s.tablesInSmem ? tables : 0 );
    // small systems: a warp per cell, up to 8 per CTA; larger: two warps per
    // cell (named barriers), up to 4 per CTA; a whole CTA per cell otherwise
    const int fit = int( std::min<size_t>( 8, avail / wsCell ) );
    s.group       = h->closureGroupOverride ? h->closureGroupOverride : ( n <= 32 ? 32 : 64 );
    if( s.group == 32 && fit < 1 ) s.group = 256;
    if( s.group == 64 && fit < ( h->closureGroupOverride ? 1 : 2 ) ) s.group = 256;
    s.block                = s.group == 32 ? 32 * fit : ( s.group == 64 ? 64 * std::min( 4, fit ) : 256 );
    const int groupsPerCta = s.block / s.group;
    s.smem                 = wsCell * groupsPerCta + ( s.tablesInSmem ? tables : 0 );
    if( s.smem > size_t( maxSmem ) )
        throw ConfigError( "closure workspace (" + std::to_string( s.smem ) + " B) exceeds shared memory; reduce moments or nodes" );
    return s;
}

void plan_launches( uqc_solver* h ) {
    ++h->planGen;
    int dev;
    CK( cudaGetDevice( &dev ) );
    CK( cudaDeviceGetAttribute( &h->numSMs, cudaDevAttrMultiProcessorCount, dev ) );
    int maxSmem = 0;
    CK( cudaDeviceGetAttribute( &maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev ) );
    const int cl = h->cfg.closure, nT = h->tab.nT, nQ = h->tab.nQ, nS = h->nS;
    const size_t n = size_t( nS ) * nT;
    h->group = n <= 32 ? 32 : 256;    // thread group per cell of the update / init / mean-variance kernels
    // closure: a warp per cell (several per CTA) or a whole 256-thread CTA per cell
    const size_t tables  = 2 * ( size_t( nQ ) * h->ld + 4 ) * sizeof( double );
    const size_t wsCell  = cell_ws_doubles( nS, nT, nQ, closure_np( cl ) ) * sizeof( double );
    h->tablesInSmem = tables <= 96 * 1024 && tables + wsCell <= size_t( maxSmem );
    const ClosureShape cs  = fp64_closure_shape( h, maxSmem );
    h->closureTablesInSmem = cs.tablesInSmem;
    h->closureGroup        = cs.group;
    h->closureBlock        = cs.block;
    h->closureSmem         = cs.smem;
    void* kc = pick( cl, h->closureGroup, 0 );
    allow_dynamic_smem( kc );
    int occ = 0;
    CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kc, h->closureBlock, h->closureSmem ) );
    h->closureGrid = std::max( 1, occ ) * h->numSMs;
    // tiny systems (n <= TINY_N duals, <= 64 nodes): the register Newton, a warp per cell
    h->closureTiny = h->tinyOpt != 0 && h->closureGroup == 32 && n <= size_t( TINY_N ) && nQ <= 64 && !closure_linear( cl );
    if( h->closureTiny ) {
        void* kt = pick( cl, 32, KERNEL_CLOSURE_TINY );
        allow_dynamic_smem( kt );
        CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kt, h->closureBlock, h->closureSmem ) );
        h->tinyGrid = std::max( 1, occ ) * h->numSMs;
    }
    // update kernel: a warp per cell; phiWf + one node-flux buffer per warp
    {
        const size_t uTables = h->tablesInSmem ? ( ( size_t( nQ ) * h->ld + 4 + 3 ) & ~size_t( 3 ) ) * sizeof( double ) : 0;
        const size_t perWarp = update_warp_doubles( nS, nQ, h->mesh.nFaces ) * sizeof( double );
        void* kf             = pick( cl, h->group, update_kernel_id( h, true ) );
        void* kp             = pick( cl, h->group, update_kernel_id( h, false ) );
        void* ku             = update_test_on( h ) ? kf : kp;    // the variant the steps launch
        allow_dynamic_smem( kf );
        allow_dynamic_smem( kp );
        // warps per CTA: the option, else the count of 8, 4 or 2 that keeps the
        // most warps resident per SM (per-warp flux buffers of many nodes fill
        // shared memory before the registers run out; ties: the larger CTA)
        int warps = 0, bestResident = -1;
        for( int w : {8, 4, 2} ) {
            if( h->updateWarpsOpt && w != 8 ) break;
            const int cand = int( std::min<size_t>( h->updateWarpsOpt ? h->updateWarpsOpt : w, ( size_t( maxSmem ) - uTables ) / perWarp ) );
            if( cand < 1 ) continue;
            int o = 0;
            CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &o, ku, 32 * cand, uTables + size_t( cand ) * perWarp ) );
            if( o * cand > bestResident ) {
                bestResident = o * cand;
                warps        = cand;
            }
        }
        if( warps < 1 ) throw ConfigError( "update workspace exceeds shared memory" );
        h->updateBlock = 32 * warps;
        h->updateSmem  = uTables + size_t( warps ) * perWarp;
        // the grid fills the SMs for that variant (the two variants may differ
        // in registers, so in CTAs per SM)
        CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, ku, h->updateBlock, h->updateSmem ) );
        h->updateGrid = std::max( 1, occ ) * h->numSMs;
        h->updateGrid = std::min( h->updateGrid, std::max( 1, ( h->mesh.nCells + warps - 1 ) / warps ) );
        // one residual partial per CTA of k_update (grows with the grid; a
        // re-plan waits for the device in cudaFree before replacing it)
        if( h->updateGrid > h->blockPartialCap ) {
            if( h->d_blockPartial ) cudaFree( h->d_blockPartial );
            h->d_blockPartial  = dalloc<double>( size_t( h->updateGrid ) );
            h->blockPartialCap = h->updateGrid;
        }
    }
    const int ug = h->auxBlock / h->group;    // groups per CTA of the init / mean-variance kernels
    h->initSmem   = size_t( ug ) * ( size_t( nS ) * nQ + 8 ) * sizeof( double );
    h->mvSmem     = size_t( ug ) * ( 2 * size_t( nS ) * nQ + 8 ) * sizeof( double );
    for( int which : {2, 3} ) {
        size_t sm = which == 2 ? h->initSmem : h->mvSmem;
        if( sm > size_t( maxSmem ) ) throw ConfigError( "init/meanvar workspace exceeds shared memory" );
        allow_dynamic_smem( pick( cl, h->group, which ) );
    }
    h->auxGrid = std::min( 4 * h->numSMs, std::max( 1, ( h->mesh.nCells + ug - 1 ) / ug ) );
    // check kernel: a warp per cell, as many warps per CTA (up to 16) as shared memory allows
    {
        const size_t wsc = check_ws_doubles( nS, nT, nQ ) * sizeof( double );
        const size_t av  = size_t( maxSmem ) - ( h->tablesInSmem ? tables : 0 );
        const int warps  = int( std::min<size_t>( h->checkWarpsOpt ? h->checkWarpsOpt : 16, av / wsc ) );
        if( warps < 1 ) throw ConfigError( "check workspace exceeds shared memory" );
        h->checkBlock = 32 * warps;
        h->checkSmem  = wsc * warps + ( h->tablesInSmem ? tables : 0 );
        void* kk      = pick_check( cl );
        allow_dynamic_smem( kk );
        CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, kk, h->checkBlock, h->checkSmem ) );
        h->checkGrid = std::min( std::max( 1, occ ) * h->numSMs, std::max( 1, ( h->mesh.nCells + warps - 1 ) / warps ) );
    }
    plan_mixed( h, maxSmem );
    plan_rounds( h, maxSmem );
}

void reset_control( uqc_solver* h, double t ) {
    Control c{};
    c.t               = t;
    c.tEnd            = h->cfg.tEnd;
    c.minResidual     = h->cfg.minResidual;
    c.residual        = h->cfg.minResidual + 1.0;    // momentsolver.cpp:76
    if( h->sharded ) {
        // a shard's residual is its own cells' part: the stopping rule on the
        // summed residual is the caller's (after its all-reduce)
        c.minResidual = -1.0;
        c.residual    = 0.0;
    }
    c.dtBits          = 0x7FF0000000000000ull;
    c.dtBitsNext      = 0x7FF0000000000000ull;
    c.maxSteps        = h->cfg.maxSteps;
    c.active          = t < h->cfg.tEnd ? 1 : 0;
    c.levelCap        = h->cfg.retLevels.empty() ? ( 1 << 30 ) : h->cfg.retLevels[0];
    c.retIndex        = 0;
    *h->h_ctl         = c;
    h->lastIters      = 0;    // device counters restart from zero
    h->lastLs         = 0;
    h->lastFailed     = 0;
    h->lastFallback   = 0;
    CK( cudaMemcpyAsync( h->d_ctl, h->h_ctl, sizeof( Control ), cudaMemcpyHostToDevice, h->stream ) );
    CK( cudaStreamSynchronize( h->stream ) );
}

// Drops the next step's active-cell list that k_update built (after a change
// of the convergence test): the next k_check tests every cell again.
void invalidate_lists( uqc_solver* h ) {
    if( !h->deviceReady ) return;
    static const unsigned long long inf = 0x7FF0000000000000ull;
    CK( cudaMemsetAsync( &h->d_ctl->nActive[0], 0, 4 * sizeof( unsigned ) + sizeof( int ), h->stream ) );    // nActive, listReady, nCheck
    CK( cudaMemcpyAsync( &h->d_ctl->dtBits, &inf, sizeof( inf ), cudaMemcpyHostToDevice, h->stream ) );
    CK( cudaStreamSynchronize( h->stream ) );
}

void read_control( uqc_solver* h ) {
    CK( cudaMemcpyAsync( h->h_ctl, h->d_ctl, sizeof( Control ), cudaMemcpyDeviceToHost, h->stream ) );
    CK( cudaStreamSynchronize( h->stream ) );
}

void build( uqc_solver* h, const std::string& text, void* stream, const std::string& inputDir ) {
    h->cfgText      = text;
    h->cfg          = parse_config( text );
    h->cfg.inputDir = inputDir;
    h->tab = build_tables( h->cfg );
    h->nS  = closure_states( h->cfg.closure );
    h->ld  = ( h->tab.nT % 2 ) ? h->tab.nT : h->tab.nT + 1;    // odd row stride: conflict-free column reads
    h->ldc = size_t( h->nS ) * h->tab.nT;
    if( h->cfg.meshDim == 1 )
        h->mesh = build_mesh_1d( h->cfg.nCells1d, h->cfg.a, h->cfg.b );
    else if( h->cfg.meshKind == "su2" ) {
        const std::string& f = h->cfg.su2File;
        h->mesh              = read_su2_mesh( f[0] == '/' ? f : h->cfg.inputDir + "/" + f, h->cfg.su2BC );
    }
    else {
        int nn = ( h->cfg.nx + 1 ) * ( h->cfg.ny + 1 ), nt = 2 * h->cfg.nx * h->cfg.ny;
        std::vector<double> xy( 2 * size_t( nn ) );
        std::vector<int> bnd( nn ), tri( 3 * size_t( nt ) );
        tri_jitter_nodes( h->cfg.nx, h->cfg.ny, h->cfg.jitter, h->cfg.seed, xy.data(), bnd.data(), tri.data() );
        h->mesh = build_mesh_tri( nn, xy.data(), bnd.data(), nt, tri.data() );
    }
    h->area0     = h->mesh.area.empty() ? 0.0 : h->mesh.area[0];
    build_filters( h );
    h->precision = h->cfg.precision;
    h->userStream = (cudaStream_t)stream;
    // host copies of the tables in the device layout (row stride ld, 8 spare
    // doubles), used by uqc_closure_solve_device_noalloc
    h->padPhi.assign( size_t( h->tab.nQ ) * h->ld + 8, 0.0 );
    h->padPhiWf.assign( size_t( h->tab.nQ ) * h->ld + 8, 0.0 );
    // wt_k = w_k / 2^dimXi, so that phiWf(k, i) = phi(k, i) wt_k exactly
    h->padWt.resize( h->tab.nQ );
    for( int k = 0; k < h->tab.nQ; ++k ) h->padWt[k] = std::ldexp( h->tab.w[k], -h->tab.dimXi );
    for( int k = 0; k < h->tab.nQ; ++k )
        for( int i = 0; i < h->tab.nT; ++i ) {
            h->padPhi[size_t( k ) * h->ld + i]   = h->tab.phi[size_t( k ) * h->tab.nT + i];
            h->padPhiWf[size_t( k ) * h->ld + i] = h->tab.phiWf[size_t( k ) * h->tab.nT + i];
        }
}

// Factors of the linear closures as their constructors compute them, in the
// reference's operation order: L2Filter (l2filter.cpp:3-17; the loop over the
// states multiplies each factor in once per state), LassoFilter
// (lassofilter.cpp:3-22: p_i = prod_l index_l (index_l + 1), l1_i = sum_k
// |phiWf(k, i)|). index_l = digit l of i in base nMoments, the last level's
// degree (Settings::GetNMoments, settings.cpp:226). Stochastic Galerkin: 1.
void build_filters( uqc_solver* h ) {
    const int nT = h->tab.nT, nQ = h->tab.nQ, d = h->tab.dimXi, nS = h->nS;
    h->filterHost.assign( nT, 1.0 );
    h->lassoParamHost.assign( nT, 1.0 );
    h->lassoL1Host.assign( nT, 0.0 );
    if( !closure_linear( h->cfg.closure ) ) return;
    const unsigned nM = unsigned( h->cfg.degrees.back() );
    if( nM == 0 && h->cfg.filterKind != FILTER_SG ) throw ConfigError( "the moment filters need a degree of at least 1" );
    auto index = [&]( unsigned i, int l ) {
        const unsigned p = unsigned( std::pow( nM, l ) );
        return ( ( i - i % p ) / p ) % nM;
    };
    if( h->cfg.filterKind == FILTER_L2 ) {
        const double lam = 0.0000015;
        for( int s = 0; s < nS; ++s )
            for( int i = 0; i < nT; ++i )
                for( int l = 0; l < d; ++l ) {
                    const unsigned ix = index( unsigned( i ), l );
                    h->filterHost[i] *= 1.0 / ( 1.0 + lam * std::pow( ix, 2 ) * std::pow( ix + 1, 2 ) );
                }
    }
    else if( h->cfg.filterKind == FILTER_LASSO ) {
        for( int i = 0; i < nT; ++i )
            for( int k = 0; k < nQ; ++k ) h->lassoL1Host[i] += std::fabs( h->tab.phiWf[size_t( k ) * nT + i] );
        for( int i = 0; i < nT; ++i )
            for( int l = 0; l < d; ++l ) {
                const unsigned ix = index( unsigned( i ), l );
                h->lassoParamHost[i] *= ix * ( ix + 1 );
            }
    }
}

// Device side of a handle, set up on first use so that configuration, tables
// and mesh (host code) work without a GPU.
void ensure_device( uqc_solver* h ) {
    if( h->deviceReady ) return;
    if( h->userStream ) {
        h->stream = h->userStream;
    }
    else {
        CK( cudaStreamCreateWithFlags( &h->stream, cudaStreamNonBlocking ) );
        h->ownStream = true;
    }
    // tables with zero padding rows (row stride ld, 8 spare doubles)
    const int nQ = h->tab.nQ, nT = h->tab.nT;
    std::vector<double> phi( size_t( nQ ) * h->ld + 8, 0.0 ), phiWf( size_t( nQ ) * h->ld + 8, 0.0 );
    for( int k = 0; k < nQ; ++k )
        for( int i = 0; i < nT; ++i ) {
            phi[size_t( k ) * h->ld + i]   = h->tab.phi[size_t( k ) * nT + i];
            phiWf[size_t( k ) * h->ld + i] = h->tab.phiWf[size_t( k ) * nT + i];
        }
    h->d_phi   = dupload( phi );
    h->d_phiWf = dupload( phiWf );
    std::vector<float> phiF( phi.size() );
    for( size_t i = 0; i < phi.size(); ++i ) phiF[i] = float( phi[i] );
    h->d_phiF = dupload( phiF );
    h->d_xi    = dupload( h->tab.xi );
    h->d_filter     = dupload( h->filterHost );
    h->d_lassoParam = dupload( h->lassoParamHost );
    h->d_lassoL1    = dupload( h->lassoL1Host );
    h->d_wt    = dupload( h->padWt );
    const Mesh& m = h->mesh;
    std::vector<double> dx( m.nCells );
    for( int j = 0; j < m.nCells; ++j ) dx[j] = m.maxEdge[j] / m.area[j];    // momentsolver.cpp:130
    h->d_area     = dupload( m.area );
    h->d_dx       = dupload( dx );
    h->d_center   = dupload( m.center );
    h->d_unitN    = dupload( m.unitN );
    h->d_scaledN  = dupload( m.scaledN );
    h->d_nbr      = dupload( m.nbr );
    h->d_boundary = dupload( m.boundary );
    if( mesh_has_walls( m ) ) h->d_bndNormal = dupload( m.bndNormal );
    const size_t N = size_t( m.nCells );
    h->d_u         = dalloc<double>( N * h->ldc );
    h->d_lam       = dalloc<double>( N * h->ldc );
    h->d_uQ        = dalloc<double>( ( N + 1 ) * h->nS * nQ );    // +1: ghost cell (never read by Dirichlet runs)
    CK( cudaMemset( h->d_uQ, 0, ( N + 1 ) * h->nS * nQ * sizeof( double ) ) );
    h->d_uOld0  = dalloc<double>( N );
    h->d_level  = dalloc<unsigned>( N );
    h->d_status = dalloc<int>( N );
    h->d_iters  = dalloc<int>( N );
    h->d_activeList   = dalloc<int>( 2 * N );
    h->d_cellDt       = dalloc<double>( N );
    h->d_uRe          = dalloc<double>( N * h->ldc );
    h->d_checkList    = dalloc<int>( 2 * N );
    h->d_finFlag      = dalloc<unsigned char>( N );
    CK( cudaMemset( h->d_finFlag, 0, N ) );
    h->d_fallbackList = dalloc<int>( N );
    if( h->sharded && !h->shard.sendCells.empty() ) h->d_sendCells = dupload( h->shard.sendCells );
    h->d_ctl    = dalloc<Control>( 1 );
    CK( cudaMallocHost( &h->h_ctl, sizeof( Control ) ) );
    for( auto& e : h->ev ) CK( cudaEventCreate( &e ) );
    plan_launches( h );
    if( h->precision == UQC_MIXED && !h->mixedOk ) throw ConfigError( "mixed precision not available for this configuration: " + h->mixedWhy );
    if( h->precision == UQC_MIXED && h->chord ) reset_factor_store( h );
    h->deviceReady = true;
    reset_control( h, 0.0 );
}

void release( uqc_solver* h ) {
    for( auto& kv : h->graphs ) cudaGraphExecDestroy( kv.second.first );
    h->graphs.clear();
    for( void* p : {(void*)h->d_phi, (void*)h->d_phiWf, (void*)h->d_xi, (void*)h->d_wt, (void*)h->d_area, (void*)h->d_dx, (void*)h->d_center,
                    (void*)h->d_unitN, (void*)h->d_scaledN, (void*)h->d_nbr, (void*)h->d_boundary, (void*)h->d_u, (void*)h->d_lam,
                    (void*)h->d_bndNormal, (void*)h->d_uQ, (void*)h->d_uOld0, (void*)h->d_blockPartial, (void*)h->d_chunkPartial, (void*)h->d_level, (void*)h->d_status,
                    (void*)h->d_iters, (void*)h->d_ctl, (void*)h->d_xLam, (void*)h->d_xU, (void*)h->d_xNt, (void*)h->d_xStatus,
                    (void*)h->d_xIters, (void*)h->d_activeList, (void*)h->d_cellDt, (void*)h->d_uRe, (void*)h->d_checkList, (void*)h->d_finFlag, (void*)h->d_phiF, (void*)h->d_fallbackList,
                    (void*)h->d_factorStore, (void*)h->d_factorLevel, (void*)h->d_gStore, (void*)h->d_v2Lists,
                    (void*)h->d_chordIters, (void*)h->d_qTiles, (void*)h->d_sendCells, (void*)h->d_filter, (void*)h->d_lassoParam,
                    (void*)h->d_lassoL1} )
        if( p ) cudaFree( p );
    if( h->h_ctl ) cudaFreeHost( h->h_ctl );
    for( auto& e : h->ev )
        if( e ) cudaEventDestroy( e );
    if( h->asyncEv ) cudaEventDestroy( h->asyncEv );
    for( auto& e : h->stepEvents )
        if( e ) cudaEventDestroy( e );
    for( auto& e : h->hostEvents )
        if( e ) cudaEventDestroy( e );
    if( h->copyStream ) cudaStreamDestroy( h->copyStream );
    if( h->copyStreamOut ) cudaStreamDestroy( h->copyStreamOut );
    if( h->checkStream ) cudaStreamDestroy( h->checkStream );
    if( h->ownStream && h->stream ) cudaStreamDestroy( h->stream );
}

// Closure launch: the FP64 kernel; or the mixed-form kernel followed by the
// FP64 kernel over the cells the mixed form handed back (a launch that finds
// an empty list returns at once). The work counters and the fallback list
// length must be zero on entry (k_update resets them after every step).
void launch_closure( uqc_solver* h, KParams& P, int mode ) {
    if( h->closureTiny && h->cfg.newtonMode != 2 ) {
        // tiny systems: the FP64 register Newton in both precisions (the mixed
        // form's FP32 Hessian saves nothing at this size)
        KParams Q      = P;
        Q.tablesInSmem = h->closureTablesInSmem;
        void* args[]   = {&Q, &mode};
        launch( h, pick( h->cfg.closure, 32, KERNEL_CLOSURE_TINY ), h->tinyGrid, h->closureBlock, h->closureSmem, args );
        return;
    }
    if( mode == 1 && P.gStore ) {
        // the mixed form in rounds: k_chord, then per round the Hessians of
        // the listed cells (tensor cores or CUDA cores) and their inverses,
        // and k_chord again; then the FP64 pass over the fallback list
        const int cl = h->cfg.closure;
        KParams C    = P;
        C.tablesInSmem = h->chordTablesInSmem;
        if( h->mixedMaxIter > 1 && P.maxIter > 1 ) C.maxIter = std::min( P.maxIter, h->mixedMaxIter );
        for( int r = 0; r <= h->v2Rounds; ++r ) {
            if( r > 0 ) {
                int rr        = r - 1;
                void* hargs[] = {&C, &rr};
                if( h->v2Mode == 2 ) launch( h, pick( cl, 32, KERNEL_HESS_TC ), h->hessGrid, 256, h->hessSmem, hargs );
                const int ik = h->invSweep ? KERNEL_INVERT_SWEEP : ( h->v2Mode == 2 ? KERNEL_INVERT_RAW : KERNEL_INVERT );
                launch( h, pick( cl, 32, ik ), h->invGrid, h->invBlock, h->invSmem, hargs );
            }
            int rr       = r;
            void* args[] = {&C, &rr};
            launch( h, pick( cl, 32, KERNEL_CHORD ), h->chordGrid, h->chordBlock, h->chordSmem, args );
        }
        KParams F      = P;
        F.activeList   = h->d_fallbackList;
        F.activeCount  = &h->d_ctl->nFallback;
        F.listParity   = 0;
        F.workCounter  = &h->d_ctl->workCounter2;
        F.tablesInSmem = h->closureTablesInSmem;
        F.gStore       = nullptr;
        void* fargs[]  = {&F, &mode};
        launch( h, pick( cl, h->closureGroup, 0 ), h->closureGrid, h->closureBlock, h->closureSmem, fargs );
        return;
    }
    if( h->precision == UQC_MIXED && h->mixedOk ) {
        KParams M      = P;
        M.tablesInSmem = h->mixedTablesInSmem;
        if( h->mixedMaxIter > 1 && P.maxIter > 1 ) M.maxIter = std::min( P.maxIter, h->mixedMaxIter );
        void* margs[]  = {&M, &mode};
        launch( h, pick( h->cfg.closure, h->mixedGroup, 4 ), h->mixedGrid, h->mixedBlock, h->mixedSmem, margs );
        KParams F     = P;
        F.activeList  = h->d_fallbackList;
        F.activeCount = &h->d_ctl->nFallback;
        F.listParity  = 0;    // one fallback list
        F.workCounter  = &h->d_ctl->workCounter2;
        F.tablesInSmem = h->closureTablesInSmem;
        void* fargs[]  = {&F, &mode};
        launch( h, pick( h->cfg.closure, h->closureGroup, 0 ), h->closureGrid, h->closureBlock, h->closureSmem, fargs );
        return;
    }
    KParams Q      = P;
    Q.tablesInSmem = h->closureTablesInSmem;
    void* args[]   = {&Q, &mode};
    launch( h, pick( h->cfg.closure, h->closureGroup, 0 ), h->closureGrid, h->closureBlock, h->closureSmem, args );
}

// Zeroes the closure work counters and the fallback list length (three
// consecutive fields of Control) before a closure-only launch.
void reset_work( uqc_solver* h ) {
    CK( cudaMemsetAsync( &h->d_ctl->workCounter, 0, 3 * sizeof( unsigned ), h->stream ) );
}

// Closure half of a time step: k_check (warp per cell) finishes converged
// cells and lists the others, then k_closure runs Newton on the list. In
// SolveClosureSafe mode every cell takes a Newton step, so k_closure gets all.
// The two active-cell lists of step mode (see step_list): k_check fills the
// running step's list on the first step after a state change, k_update fills
// the next step's list from its own convergence test, so later k_check
// launches return at once (Control::listReady).
void step_lists( uqc_solver* h, KParams& P ) {
    if( h->sharded ) P.nWork = h->shard.nOwned;
    if( h->cfg.newtonMode == 2 ) return;
    P.activeList  = h->d_activeList;
    P.activeCount = h->d_ctl->nActive;
    P.listParity  = 1;
    P.checkList   = h->d_checkList;
    P.checkCount  = h->d_ctl->nCheck;
    P.finFlag     = h->d_finFlag;
}

void enqueue_closure_phase( uqc_solver* h, KParams P ) {
    step_lists( h, P );
    if( h->cfg.newtonMode != 2 ) {
        void* args[] = {&P};
        launch( h, pick_check( h->cfg.closure ), h->checkGrid, h->checkBlock, h->checkSmem, args );
    }
    launch_closure( h, P, 1 );
}

void enqueue_update( uqc_solver* h, KParams P ) {
    step_lists( h, P );
    P.finishInUpdate = update_test_on( h );
    void* args[]     = {&P};
    launch( h, pick( h->cfg.closure, h->group, update_kernel_id( h, P.finishInUpdate != 0 ) ), h->updateGrid, h->updateBlock, h->updateSmem,
            args );
}

void enqueue_step( uqc_solver* h, KParams& P ) {
    enqueue_closure_phase( h, P );
    enqueue_update( h, P );
}

// n time steps on the handle's stream: one launch of a cached CUDA graph of
// the n steps (captured on first use, re-captured after a change of launch
// plan, precision or Newton settings), or direct launches when graphs are
// off or the stream cannot be captured.
void launch_steps( uqc_solver* h, int n ) {
    if( h->useGraphs && h->graphGen != h->planGen ) {
        for( auto& kv : h->graphs ) CK( cudaGraphExecDestroy( kv.second.first ) );
        h->graphs.clear();
        h->graphGen = h->planGen;
    }
    if( h->useGraphs ) {
        auto it = h->graphs.find( n );
        if( it == h->graphs.end() ) {
            if( cudaStreamBeginCapture( h->stream, cudaStreamCaptureModeThreadLocal ) != cudaSuccess ) {
                cudaGetLastError();
                h->useGraphs = false;    // e.g. the legacy default stream
            }
            else {
                const int l0 = h->launches;
                KParams P    = make_params( h );
                for( int s = 0; s < n; ++s ) enqueue_step( h, P );
                cudaGraph_t g = nullptr;
                CK( cudaStreamEndCapture( h->stream, &g ) );
                cudaGraphExec_t ex = nullptr;
                const cudaError_t e = cudaGraphInstantiate( &ex, g, 0 );
                cudaGraphDestroy( g );
                CK( e );
                it          = h->graphs.emplace( n, std::make_pair( ex, h->launches - l0 ) ).first;
                h->launches = l0;
            }
        }
        if( h->useGraphs ) {
            CK( cudaGraphLaunch( it->second.first, h->stream ) );
            h->launches += it->second.second;
            return;
        }
    }
    KParams P = make_params( h );
    for( int s = 0; s < n; ++s ) enqueue_step( h, P );
}

// Reads the control block, fills info with this call's deltas, returns the
// number of cells that failed during the call; fill_info_host uses the host
// mirror of the control block as it stands.
int fill_info_host( uqc_solver* h, uqc_step_info* info, int stepsBefore ) {
    const Control& c = *h->h_ctl;
    const int failedNow = c.failedCells - h->lastFailed;
    if( info ) {
        info->t                  = c.t;
        info->dt                 = c.dt;
        info->residual           = c.residual;
        info->steps              = c.steps - stepsBefore;
        info->failed_cells       = c.failedCells - h->lastFailed;
        info->newton_iterations  = (long long)( c.newtonIters - h->lastIters );
        info->line_search_trials = (long long)( c.lineSearchTrials - h->lastLs );
        info->active_cells       = c.activeCellsLast;
        info->fallback_cells     = (long long)( c.fallbackCells - h->lastFallback );
        info->running            = c.active;
    }
    h->lastFallback = c.fallbackCells;
    h->lastIters  = c.newtonIters;
    h->lastLs     = c.lineSearchTrials;
    h->lastFailed = c.failedCells;
    return failedNow;
}

int fill_info( uqc_solver* h, uqc_step_info* info, int stepsBefore ) {
    read_control( h );
    if( h->h_ctl->v2Error ) throw CudaError( "k_hess_tc: the tensor cores did not complete a tile within the wait limit" );
    return fill_info_host( h, info, stepsBefore );
}

// Device memory of a handle once ensure_device has run (the allocations of
// ensure_device and plan_launches; closure-only scratch excluded).
unsigned long long factor_store_bytes( const uqc_solver* h );
unsigned long long device_bytes_of( const uqc_solver* h ) {
    const unsigned long long N = (unsigned long long)h->mesh.nCells, F = (unsigned long long)h->mesh.nFaces;
    const unsigned long long ldc = h->ldc, sq = (unsigned long long)h->nS * h->tab.nQ;
    const unsigned long long tab = ( (unsigned long long)h->tab.nQ * h->ld + 8 ) * ( 8 + 8 + 4 ) + h->tab.xi.size() * 8 + h->tab.nQ * 8;
    const unsigned long long d8  = N * ( 3 * ldc + 1 + 1 + 1 + 2 + 4 * F ) + ( N + 1 ) * sq;    // state (u, re-projected u, lambda), uQ, geometry, cell dt
    const unsigned long long d4  = N * ( F + 1 + 1 + 1 + 1 + 2 + 2 + 1 );                     // nbr, boundary, level, status, iters, lists
    return tab + 8 * d8 + 4 * d4 + N + ( mesh_has_walls( h->mesh ) ? 16 * N : 0 ) + sizeof( Control ) + 8 * 4096 + ( h->precision == UQC_MIXED && h->chord ? factor_store_bytes( h ) : 0 );
}

void to_layout( const uqc_solver* h, const double* src, double* dst, int layout, bool toDevice ) {
    // REF: (s, i) at i nS + s ; STATE_MAJOR: s nT + i
    const size_t N = size_t( h->mesh.nCells ), nT = size_t( h->tab.nT ), nS = size_t( h->nS );
    for( size_t j = 0; j < N; ++j )
        for( size_t s = 0; s < nS; ++s )
            for( size_t i = 0; i < nT; ++i ) {
                size_t sm = j * nS * nT + s * nT + i, rf = j * nS * nT + i * nS + s;
                if( toDevice )
                    dst[sm] = src[rf];
                else
                    dst[rf] = src[sm];
            }
    (void)layout;
}

}    // namespace

namespace {
// Files a config names (SU2MeshFile, restartFile) are relative to inputDir:
// the config file's directory (Settings::_inputDir, settings.cpp:30), or the
// working directory for a config given as text.
int create_impl( const char* toml_text, const std::string& inputDir, void* cuda_stream, uqc_solver** out, char* err, int err_len ) {
    *out           = nullptr;
    uqc_solver* h  = new uqc_solver();
    int rc         = guarded( h, [&] {
        build( h, toml_text, cuda_stream, inputDir );
        return UQC_OK;
    } );
    if( rc != UQC_OK ) {
        if( err && err_len > 0 ) {
            std::strncpy( err, h->err.c_str(), size_t( err_len - 1 ) );
            err[err_len - 1] = 0;
        }
        release( h );
        delete h;
        return rc;
    }
    *out = h;
    return UQC_OK;
}
}    // namespace

// ========================================================================== C ABI

extern "C" {


int uqc_create_from_string( const char* toml_text, void* cuda_stream, uqc_solver** out, char* err, int err_len ) {
    if( !out || !toml_text ) return UQC_ERR_ARGUMENT;
    return create_impl( toml_text, ".", cuda_stream, out, err, err_len );
}

void uqc_config_defaults( uqc_config* c ) {
    if( !c ) return;
    std::memset( c, 0, sizeof( *c ) );
    c->mesh_dimension = 1;
    c->dim_xi         = 1;
    c->min_residual   = -1.0;
    c->n_levels       = 1;
    c->max_iterations = 1000;    // settings.cpp: maxIterations default
    c->epsilon        = 5e-5;    // settings.cpp: epsilon default
    c->bounds[0]      = 3.0;
    c->bounds[1]      = 12.0;
}

int uqc_create_from_config( const uqc_config* cfg, void* cuda_stream, uqc_solver** out, char* err, int err_len ) {
    if( !cfg || !out ) return UQC_ERR_ARGUMENT;
    *out = nullptr;
    std::string text;
    try {
        text = config_struct_to_toml( cfg );
    } catch( const std::exception& e ) {
        if( err && err_len > 0 ) {
            std::strncpy( err, e.what(), size_t( err_len - 1 ) );
            err[err_len - 1] = 0;
        }
        return UQC_ERR_CONFIG;
    }
    return create_impl( text.c_str(), ".", cuda_stream, out, err, err_len );
}

int uqc_create_from_file( const char* toml_path, void* cuda_stream, uqc_solver** out, char* err, int err_len ) {
    if( !toml_path || !out ) return UQC_ERR_ARGUMENT;
    std::ifstream f( toml_path );
    if( !f ) {
        if( err && err_len > 0 ) std::snprintf( err, size_t( err_len ), "cannot open %s", toml_path );
        return UQC_ERR_CONFIG;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string path = toml_path;
    const size_t slash     = path.find_last_of( '/' );
    const int rc = create_impl( ss.str().c_str(), slash == std::string::npos ? "." : path.substr( 0, slash ), cuda_stream, out, err, err_len );
    if( rc == UQC_OK ) ( *out )->cfgName = path;
    return rc;
}

void uqc_destroy( uqc_solver* h ) {
    if( !h ) return;
    if( h->stream ) cudaStreamSynchronize( h->stream );
    release( h );
    delete h;
}

const char* uqc_last_error( const uqc_solver* h ) { return h ? h->err.c_str() : "null handle"; }

int uqc_get_info( const uqc_solver* h, uqc_info* o ) {
    if( !h || !o ) return UQC_ERR_ARGUMENT;
    std::memset( o, 0, sizeof( *o ) );
    o->n_cells  = h->mesh.nCells;
    o->n_states = h->nS;
    o->n_total  = h->tab.nT;
    o->n_quad   = h->tab.nQ;
    o->n_levels = h->tab.nLevels;
    o->dim_xi   = h->tab.dimXi;
    o->n_faces  = h->mesh.nFaces;
    o->mesh_dim = h->mesh.dim;
    for( int l = 0; l < h->tab.nLevels && l < 16; ++l ) o->n_total_level[l] = h->tab.nTLevel[l];
    o->precision   = h->precision;
    o->newton_mode = h->cfg.newtonMode;
    o->t           = h->h_ctl ? h->h_ctl->t : 0.0;
    o->steps       = h->h_ctl ? h->h_ctl->steps : 0;
    o->mixed_form  = h->deviceReady ? h->v2Mode : -1;
    o->mixed_rounds = h->v2Rounds;
    return UQC_OK;
}

int uqc_set_precision( uqc_solver* h, int precision ) {
    if( !h || ( precision != UQC_FP64 && precision != UQC_MIXED ) ) return UQC_ERR_ARGUMENT;
    int rc = guarded( h, [&] {
        ensure_device( h );
        return UQC_OK;
    } );
    if( rc != UQC_OK ) return rc;
    if( precision == UQC_MIXED && !h->mixedOk ) return fail( h, UQC_ERR_CONFIG, "mixed precision not available for this configuration: " + h->mixedWhy );
    if( precision == UQC_MIXED && h->chord ) {
        rc = guarded( h, [&] {
            reset_factor_store( h );
            return UQC_OK;
        } );
        if( rc != UQC_OK ) return rc;
    }
    const bool changed = h->precision != precision;
    h->precision       = precision;
    ++h->planGen;
    // the next step's list was built by the other form's update kernel (the
    // mixed form's rounds also need the listed cells' gradients): test every cell
    if( changed ) return guarded( h, [&] {
            invalidate_lists( h );
            return UQC_OK;
        } );
    return UQC_OK;
}

int uqc_set_option( uqc_solver* h, const char* key, double value ) {
    if( !h || !key ) return UQC_ERR_ARGUMENT;
    std::string k = key;
    if( k == "closure_group" ) {
        int v = int( value );
        if( v != 0 && v != 32 && v != 64 && v != 256 ) return fail( h, UQC_ERR_ARGUMENT, "closure_group must be 0, 32, 64 or 256" );
        h->closureGroupOverride = v;
        if( h->deviceReady ) return guarded( h, [&] {
                plan_launches( h );
                return UQC_OK;
            } );
        return UQC_OK;
    }
    if( k == "update_warps" || k == "check_warps" || k == "chord_warps" ) {
        int v = int( value );
        if( v < 0 || v > 16 ) return fail( h, UQC_ERR_ARGUMENT, k + " must be 0 (automatic) or 1..16" );
        ( k == "update_warps" ? h->updateWarpsOpt : k == "check_warps" ? h->checkWarpsOpt : h->chordWarpsOpt ) = v;
        if( h->deviceReady ) return guarded( h, [&] {
                plan_launches( h );
                return UQC_OK;
            } );
        return UQC_OK;
    }
    if( k == "closure_tiny" ) {
        int v = int( value );
        if( v < -1 || v > 1 ) return fail( h, UQC_ERR_ARGUMENT, "closure_tiny must be -1, 0 or 1" );
        h->tinyOpt = v;
        if( h->deviceReady ) return guarded( h, [&] {
                plan_launches( h );
                return UQC_OK;
            } );
        return UQC_OK;
    }
    if( k == "closure_tables_smem" ) {
        int v = int( value );
        if( v < -1 || v > 1 ) return fail( h, UQC_ERR_ARGUMENT, "closure_tables_smem must be -1, 0 or 1" );
        h->closureTablesOpt = v;
        if( h->deviceReady ) return guarded( h, [&] {
                plan_launches( h );
                return UQC_OK;
            } );
        return UQC_OK;
    }
    if( k == "mixed_max_iterations" ) {
        int v = int( value );
        if( v != 0 && v < 2 ) return fail( h, UQC_ERR_ARGUMENT, "mixed_max_iterations must be 0 or >= 2" );
        h->mixedMaxIter = v;
        ++h->planGen;
        return UQC_OK;
    }
    if( k == "mixed_chord" || k == "mixed_chord_inverse" ) {
        ( k == "mixed_chord" ? h->chord : h->chordInverseOpt ) = value != 0.0;
        if( h->deviceReady ) {
            int rc = guarded( h, [&] {
                plan_launches( h );    // the mixed workspace depends on the chord form
                if( h->chord && h->precision == UQC_MIXED ) reset_factor_store( h );
                return UQC_OK;
            } );
            if( rc != UQC_OK ) return rc;
        }
        ++h->planGen;
        return UQC_OK;
    }
    if( k == "mixed_hessian" || k == "mixed_rounds" ) {
        const int v = int( value );
        if( k == "mixed_hessian" && ( v < -1 || v > 2 ) ) return fail( h, UQC_ERR_ARGUMENT, "mixed_hessian must be -1, 0, 1 or 2" );
        if( k == "mixed_rounds" && ( v < 1 || v > 3 ) ) return fail( h, UQC_ERR_ARGUMENT, "mixed_rounds must be 1, 2 or 3" );
        ( k == "mixed_hessian" ? h->roundsOpt : h->v2Rounds ) = v;
        if( h->deviceReady ) {
            int rc = guarded( h, [&] {
                plan_launches( h );
                if( h->chord && h->precision == UQC_MIXED ) reset_factor_store( h );    // the store's format depends on the form
                invalidate_lists( h );    // the next step's list carries no stored gradients yet
                return UQC_OK;
            } );
            if( rc != UQC_OK ) return rc;
            if( k == "mixed_hessian" && v == 2 && h->v2Mode != 2 ) return fail( h, UQC_ERR_CONFIG, "tensor-core Hessian not available: " + h->v2Why );
        }
        ++h->planGen;
        return UQC_OK;
    }
    if( k == "mixed_chord_theta" ) {
        if( !( value > 0.0 && value < 1.0 ) ) return fail( h, UQC_ERR_ARGUMENT, "mixed_chord_theta must be in (0, 1)" );
        h->chordTheta = value;
        ++h->planGen;
        return UQC_OK;
    }
    if( k == "graphs" ) {
        h->useGraphs = value != 0.0;
        ++h->planGen;
        return UQC_OK;
    }
    if( k == "host_chunks" ) {
        if( value < 1.0 || value > 32.0 || value != double( int( value ) ) ) return fail( h, UQC_ERR_ARGUMENT, "host_chunks must be 1-32" );
        h->hostChunks = int( value );
        return UQC_OK;
    }
    if( k == "update_test" ) {
        if( value != 0.0 && value != 1.0 && value != -1.0 ) return fail( h, UQC_ERR_ARGUMENT, "update_test must be 1, 0 or -1" );
        h->finishInUpdateOpt = int( value );
        ++h->planGen;
        return guarded( h, [&] {
            if( h->deviceReady ) plan_launches( h );    // the update grid follows the variant
            invalidate_lists( h );
            return UQC_OK;
        } );
    }
    return fail( h, UQC_ERR_ARGUMENT, "unknown option '" + k + "'" );
}

int uqc_set_newton( uqc_solver* h, int max_iterations, double epsilon, int newton_mode ) {
    if( !h || max_iterations < 1 || !( epsilon > 0 ) || newton_mode < 0 || newton_mode > 2 ) return UQC_ERR_ARGUMENT;
    h->cfg.maxIterations = max_iterations;
    h->cfg.epsilon       = epsilon;
    h->cfg.newtonMode    = newton_mode;
    ++h->planGen;
    return guarded( h, [&] {
        invalidate_lists( h );    // the next step's list was built with the old test
        return UQC_OK;
    } );
}

int uqc_get_tables( const uqc_solver* h, double* phi, double* phi_wf, double* xi, double* w ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    if( phi ) std::memcpy( phi, h->tab.phi.data(), h->tab.phi.size() * sizeof( double ) );
    if( phi_wf ) std::memcpy( phi_wf, h->tab.phiWf.data(), h->tab.phiWf.size() * sizeof( double ) );
    if( xi ) std::memcpy( xi, h->tab.xi.data(), h->tab.xi.size() * sizeof( double ) );
    if( w ) std::memcpy( w, h->tab.w.data(), h->tab.w.size() * sizeof( double ) );
    return UQC_OK;
}

int uqc_get_geometry( const uqc_solver* h, double* area, double* max_edge, double* center, double* unit_normal, double* scaled_normal,
                      int* neighbor, int* boundary ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    const Mesh& m = h->mesh;
    if( area ) std::memcpy( area, m.area.data(), m.area.size() * sizeof( double ) );
    if( max_edge ) std::memcpy( max_edge, m.maxEdge.data(), m.maxEdge.size() * sizeof( double ) );
    if( center ) std::memcpy( center, m.center.data(), m.center.size() * sizeof( double ) );
    if( unit_normal ) std::memcpy( unit_normal, m.unitN.data(), m.unitN.size() * sizeof( double ) );
    if( scaled_normal ) std::memcpy( scaled_normal, m.scaledN.data(), m.scaledN.size() * sizeof( double ) );
    if( neighbor ) std::memcpy( neighbor, m.nbr.data(), m.nbr.size() * sizeof( int ) );
    if( boundary ) std::memcpy( boundary, m.boundary.data(), m.boundary.size() * sizeof( int ) );
    return UQC_OK;
}

// Reads one of the reference's state files (MomentSolver::Export,
// momentsolver.cpp:565-588): a line per cell, nS x nT values in state-major
// order, each followed by a comma (ImportPrevMoments/Duals, :614-650).
// The configuration a previous run echoed into its log file <restartFile>
// (main.cpp:160-180 writes it, MomentSolver::ImportPrevSettings reads it back,
// momentsolver.cpp:590-612): the lines after "Config file" (the fourth line
// after it is the first one kept) up to the next "====" line, each stripped
// up to and including the first '|'. Empty when the file has no echo.
static std::string read_config_echo( const std::string& path ) {
    std::ifstream f( path );
    if( !f ) return "";
    std::string line, out;
    bool section = false;
    while( std::getline( f, line ) ) {
        if( line.find( "Config file" ) != std::string::npos ) {
            section = true;
            for( int i = 0; i < 4; ++i ) std::getline( f, line );
        }
        else if( section && line.find( "==================================" ) != std::string::npos ) {
            break;
        }
        if( section ) {
            line.erase( 0, line.find_first_of( '|' ) + 1 );
            out += line + "\n";
        }
    }
    return out;
}

// The log a restart reads (main.cpp:160-180's PrintInit in spdlog's file
// pattern "%Y-%m-%d %H:%M:%S.%f | %v"): header, the input file's lines that do
// not start with '#', closing rule.
static void write_config_echo( const std::string& path, const std::string& cfgName, const std::string& text ) {
    std::ofstream f( path );
    if( !f ) throw ConfigError( "cannot write " + path );
    const auto now  = std::chrono::system_clock::now();
    const time_t tt = std::chrono::system_clock::to_time_t( now );
    const long us   = long( std::chrono::duration_cast<std::chrono::microseconds>( now.time_since_epoch() ).count() % 1000000 );
    char ts[64];
    std::strftime( ts, sizeof( ts ), "%Y-%m-%d %H:%M:%S", std::localtime( &tt ) );
    char stamp[80];
    std::snprintf( stamp, sizeof( stamp ), "%s.%06ld | ", ts, us );
    const std::string rule = "================================================================";
    f << stamp << "UQCreator\n" << stamp << rule << "\n" << stamp << "Git commit hash:\tuqcreator_b200\n";
    f << stamp << "Config file:\t" << cfgName << "\n" << stamp << "MPI Threads:\t1\n" << stamp << "OMP Threads:\t1\n";
    f << stamp << rule << "\n";
    std::istringstream in( text );
    std::string line;
    while( std::getline( in, line ) )
        if( line.empty() || line[0] != '#' ) f << stamp << " " << line << "\n";
    f << stamp << rule << "\n" << stamp << "\n";
    if( !f ) throw ConfigError( "cannot write " + path );
}

static void read_state_file( const std::string& path, size_t nCells, size_t perCell, std::vector<double>& out ) {
    std::ifstream f( path );
    if( !f ) throw ConfigError( "cannot open restart file " + path );
    out.assign( nCells * perCell, 0.0 );
    std::string line;
    for( size_t j = 0; j < nCells; ++j ) {
        if( !std::getline( f, line ) ) throw ConfigError( path + ": " + std::to_string( nCells ) + " cells expected, file ends at line " + std::to_string( j + 1 ) );
        std::stringstream ls( line );
        std::string cell;
        for( size_t k = 0; k < perCell; ++k ) {
            if( !std::getline( ls, cell, ',' ) || cell.empty() )
                throw ConfigError( path + " line " + std::to_string( j + 1 ) + ": " + std::to_string( perCell ) +
                                   " values expected (a restart with another number of moments is not supported)" );
            out[j * perCell + k] = std::stod( cell );
        }
    }
}

// FP64 closure of every resident cell in SolveClosureSafe mode with maxIter
// iterations (the initial duals of a restart, momentsolver.cpp:486-521).
static void safe_closure_all( uqc_solver* h, int maxIter ) {
    KParams P      = make_params( h );
    P.newtonMode   = 2;
    P.maxIter      = maxIter;
    P.tablesInSmem = h->closureTablesInSmem;
    int mode       = 0;
    reset_work( h );
    void* args[] = {&P, &mode};
    launch( h, pick( h->cfg.closure, h->closureGroup, 0 ), h->closureGrid, h->closureBlock, h->closureSmem, args );
    CK( cudaStreamSynchronize( h->stream ) );
    read_control( h );
    if( h->h_ctl->failedCells ) throw ConfigError( "restart: " + std::to_string( h->h_ctl->failedCells ) + " cells' initial duals did not converge" );
}

// Restart onto another number of moments (MomentSolver::DetermineMoments and
// SetDuals, momentsolver.cpp:418-435, 463-523): the previous run's moments
// (its own number nPrev), Dirichlet cells from the initial state of the new
// order; the previous duals (imported, or DS of the moments solved with the
// previous basis and quadrature, SolveClosureSafe, 10000 iterations); the
// solution U(Lambda) at the new quadrature nodes from the previous basis there,
// projected onto the new basis; the duals padded with zeros and solved again.
// DS and U of a closure kind on the host
static void host_closure_ds( int cl, const double* u, double* d, const PhysParams& pp ) {
    switch( cl ) {
        case 0: Closure<0>::DS( u, d, pp ); break;
        case 1: Closure<1>::DS( u, d, pp ); break;
        case 2: Closure<2>::DS( u, d, pp ); break;
        case 3: Closure<3>::DS( u, d, pp ); break;
        case 4: Closure<4>::DS( u, d, pp ); break;
        case 5: Closure<5>::DS( u, d, pp ); break;
        case 6: Closure<6>::DS( u, d, pp ); break;
        case 7: Closure<7>::DS( u, d, pp ); break;
        default: Closure<8>::DS( u, d, pp ); break;
    }
}
static void host_closure_u( int cl, const double* L, double* y, const PhysParams& pp ) {
    switch( cl ) {
        case 0: Closure<0>::U( L, y, false, pp ); break;
        case 1: Closure<1>::U( L, y, false, pp ); break;
        case 2: Closure<2>::U( L, y, false, pp ); break;
        case 3: Closure<3>::U( L, y, false, pp ); break;
        case 4: Closure<4>::U( L, y, false, pp ); break;
        case 5: Closure<5>::U( L, y, false, pp ); break;
        case 6: Closure<6>::U( L, y, false, pp ); break;
        case 7: Closure<7>::U( L, y, false, pp ); break;
        default: Closure<8>::U( L, y, false, pp ); break;
    }
}

static void restart_new_order( uqc_solver* h, const std::string& base, const std::string& echo, const Config& prev ) {
    const size_t N = size_t( h->mesh.nCells );
    const int nS = h->nS, nT = h->tab.nT, nQ = h->tab.nQ;
    const Tables pt = build_tables( prev );
    const int nP    = pt.nT;
    std::vector<double> u, lam;
    read_state_file( base + "_moments", N, size_t( nS ) * nP, u );
    // the new order's initial moments, for the Dirichlet cells
    {
        KParams P    = make_params( h );
        int keep     = 0;
        void* args[] = {&P, &keep};
        launch( h, pick( h->cfg.closure, h->group, 2 ), h->auxGrid, h->auxBlock, h->initSmem, args );
    }
    std::vector<double> uic( N * h->ldc );
    CK( cudaMemcpyAsync( uic.data(), h->d_u, uic.size() * sizeof( double ), cudaMemcpyDeviceToHost, h->stream ) );
    CK( cudaStreamSynchronize( h->stream ) );
    for( size_t j = 0; j < N; ++j )
        if( h->mesh.boundary[j] == BC_DIRICHLET )
            for( int s = 0; s < nS; ++s )
                for( int i = 0; i < nP; ++i ) u[( j * nS + s ) * nP + i] = uic[j * h->ldc + size_t( s ) * nT + i];
    // the previous order's duals
    if( h->cfg.importDualState ) {
        read_state_file( base + "_duals", N, size_t( nS ) * nP, lam );
    }
    else {
        uqc_solver* ph = nullptr;
        char err[512]  = {0};
        if( create_impl( echo.c_str(), h->cfg.inputDir, h->userStream, &ph, err, int( sizeof err ) ) != UQC_OK )
            throw ConfigError( std::string( "restart: the echoed configuration: " ) + err );
        ph->precision = UQC_FP64;
        std::vector<int> st( N );
        lam.assign( N * nS * nP, 0.0 );
        int rc = UQC_OK;
        try {
            // DS of the mean moments as the first guess (momentsolver.cpp:471-483), on the device
            ph->cfg.newtonMode    = 2;
            ph->cfg.maxIterations = 10000;
            std::vector<double> ds( nS );
            PhysParams pp = make_params( ph ).phys;
            for( size_t j = 0; j < N; ++j ) {
                double u0[4] = {0, 0, 0, 0}, d[4] = {0, 0, 0, 0};
                for( int s = 0; s < nS; ++s ) u0[s] = u[( j * nS + s ) * nP];
                host_closure_ds( h->cfg.closure, u0, d, pp );
                for( int s = 0; s < nS; ++s ) lam[( j * nS + s ) * nP] = d[s];
            }
            rc = uqc_closure_solve_host( ph, int( N ), lam.data(), u.data(), nullptr, UQC_LAYOUT_STATE_MAJOR, st.data() );
            if( rc != UQC_OK ) throw ConfigError( std::string( "restart: previous-order duals: " ) + uqc_last_error( ph ) );
        } catch( ... ) {
            uqc_destroy( ph );
            throw;
        }
        uqc_destroy( ph );
    }
    // U(Lambda) at the new nodes from the previous basis there, projected onto the new basis
    Config mid = prev;
    mid.nQuad  = h->cfg.nQuad;
    const Tables it = build_tables( mid );
    if( it.nQ != nQ ) throw ConfigError( "restart: quadrature mismatch" );
    const PhysParams pp = make_params( h ).phys;
    std::vector<double> un( N * h->ldc, 0.0 ), ln( N * h->ldc, 0.0 ), uq( size_t( nS ) * nQ );
    for( size_t j = 0; j < N; ++j ) {
        for( int k = 0; k < nQ; ++k ) {
            double L[4] = {0, 0, 0, 0}, y[4] = {0, 0, 0, 0};
            for( int s = 0; s < nS; ++s ) {
                double a = 0.0;
                for( int i = 0; i < nP; ++i ) a += lam[( j * nS + s ) * nP + i] * it.phi[size_t( k ) * nP + i];
                L[s] = a;
            }
            host_closure_u( h->cfg.closure, L, y, pp );
            for( int s = 0; s < nS; ++s ) uq[size_t( s ) * nQ + k] = y[s];
        }
        for( int s = 0; s < nS; ++s ) {
            for( int i = 0; i < nT; ++i ) {
                double a = 0.0;
                for( int k = 0; k < nQ; ++k ) a += uq[size_t( s ) * nQ + k] * h->tab.phiWf[size_t( k ) * nT + i];
                un[j * h->ldc + size_t( s ) * nT + i] = a;
            }
            for( int i = 0; i < nP && i < nT; ++i ) ln[j * h->ldc + size_t( s ) * nT + i] = lam[( j * nS + s ) * nP + i];
        }
    }
    CK( cudaMemcpyAsync( h->d_u, un.data(), un.size() * sizeof( double ), cudaMemcpyHostToDevice, h->stream ) );
    CK( cudaMemcpyAsync( h->d_lam, ln.data(), ln.size() * sizeof( double ), cudaMemcpyHostToDevice, h->stream ) );
    std::vector<unsigned> lv( N, unsigned( h->tab.nLevels - 1 ) );
    CK( cudaMemcpyAsync( h->d_level, lv.data(), N * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
    CK( cudaStreamSynchronize( h->stream ) );
    reset_control( h, 0.0 );
    safe_closure_all( h, h->cfg.maxIterations == 1 ? 10000 : h->cfg.maxIterations );
}

int uqc_init_state( uqc_solver* h ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    return guarded_dev( h, [&] {
        h->launches  = 0;
        KParams P    = make_params( h );
        int keep     = 0;
        double t0    = 0.0;
        bool oneShotSolve = false;
        if( !h->cfg.restartFile.empty() && h->sharded ) throw ConfigError( "a restart of a sharded handle is not supported" );
        if( !h->cfg.restartFile.empty() ) {
            // restart (MomentSolver::DetermineMoments / SetDuals, momentsolver.cpp:418-523)
            const std::string base = h->cfg.restartFile[0] == '/' ? h->cfg.restartFile : h->cfg.inputDir + "/" + h->cfg.restartFile;
            const size_t N = size_t( h->mesh.nCells );
            // the previous run's settings from its log (DeterminePreviousSettings, :437-450); the
            // time continues from their tEnd (momentsolver.cpp:47)
            const std::string echo = read_config_echo( base );
            Config prev            = h->cfg;
            if( !echo.empty() ) {
                prev = parse_config( echo );
                t0   = prev.tEnd;
            }
            const int nPrev = echo.empty() ? h->tab.nT : build_tables( prev ).nT;
            if( nPrev != h->tab.nT ) {
                restart_new_order( h, base, echo, prev );
                if( h->d_factorLevel ) reset_factor_store( h );
                reset_control( h, t0 );
                h->stateReady = true;
                return UQC_OK;
            }
            std::vector<double> u, lam;
            read_state_file( base + "_moments", N, h->ldc, u );
            CK( cudaMemcpyAsync( h->d_u, u.data(), u.size() * sizeof( double ), cudaMemcpyHostToDevice, h->stream ) );
            if( h->cfg.importDualState ) {
                read_state_file( base + "_duals", N, h->ldc, lam );
                CK( cudaMemcpyAsync( h->d_lam, lam.data(), lam.size() * sizeof( double ), cudaMemcpyHostToDevice, h->stream ) );
                std::vector<unsigned> lv( N, unsigned( h->tab.nLevels - 1 ) );
                CK( cudaMemcpyAsync( h->d_level, lv.data(), N * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
                CK( cudaStreamSynchronize( h->stream ) );
                keep = -1;
            }
            else {
                keep = 1;
            }
        }
        // One-Shot IPM (maxIterations 1): SetDuals converges the initial duals
        // (SolveClosureSafe, 10000 iterations, momentsolver.cpp:486-492) unless they are imported
        oneShotSolve = h->cfg.maxIterations == 1 && keep >= 0;
        if( keep >= 0 ) {
            void* args[] = {&P, &keep};
            launch( h, pick( h->cfg.closure, h->group, 2 ), h->auxGrid, h->auxBlock, h->initSmem, args );
        }
        CK( cudaGetLastError() );
        if( oneShotSolve ) {
            reset_control( h, t0 );
            safe_closure_all( h, 10000 );
        }
        if( h->d_factorLevel ) reset_factor_store( h );
        reset_control( h, t0 );
        h->stateReady = true;
        return UQC_OK;
    } );
}

// Legacy VTK unstructured grid of E and Var per cell, as Mesh1D::Export
// (mesh1d.cpp:90-220: cells as quads extruded to a tenth of the domain length,
// plus <file>ExpectedValue / <file>Variance text columns) and Mesh2D::Export
// (mesh2d.cpp:399-501: triangles) write it with VTK: the same arrays (names
// of the reference; momentum as a 3-component vector in 2-D), as cell data
// and averaged to the points (vtkCellDataToPointData with PassCellData).
int uqc_write_vtk( uqc_solver* h, const char* path ) {
    if( !h || !path ) return UQC_ERR_ARGUMENT;
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "VTK output of a sharded handle: gather the owned cells (uqc_download_state) instead" );
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    return guarded_dev( h, [&] {
        const Mesh& m = h->mesh;
        const int N = m.nCells, nS = h->nS;
        std::vector<double> mv( size_t( N ) * 2 * nS );
        if( uqc_mean_var( h, mv.data() ) != UQC_OK ) throw CudaError( h->err );
        // arrays: name, components, per-cell values (E and Var per state; 2-D Euler momentum as vectors)
        struct Arr {
            std::string name;
            int comps;
            std::vector<int> cols;    // columns of mv (-1: zero)
        };
        std::vector<Arr> arrs;
        const bool euler = h->nS == 4;
        const char* names1[] = {"u"};
        const char* namesSW[] = {"h", "hu"};
        const char* namesE1[] = {"rho", "rhoU", "rhoE"};
        for( int part = 0; part < 2; ++part ) {
            const std::string pre = part == 0 ? "E(" : "Var(";
            const int off         = part * nS;
            if( euler ) {
                arrs.push_back( {pre + "ρ)", 1, {off + 0}} );
                arrs.push_back( {pre + "ρU)", 3, {off + 1, off + 2, -1}} );
                arrs.push_back( {pre + "ρE)", 1, {off + 3}} );
            }
            else {
                for( int s2 = 0; s2 < nS; ++s2 )
                    arrs.push_back( {pre + ( nS == 1 ? names1[0] : ( nS == 3 ? namesE1[s2] : namesSW[s2] ) ) + ")", 1, {off + s2}} );
            }
        }
        const std::string file = ( std::string( path ).size() > 4 && std::string( path ).substr( std::string( path ).size() - 4 ) == ".vtk" ) ? path : std::string( path ) + ".vtk";
        FILE* f = std::fopen( file.c_str(), "w" );
        if( !f ) throw ConfigError( "cannot write " + file );
        // points and cells
        const int nNodes = int( m.nodeXY.size() / 2 );
        std::vector<std::vector<int>> cells( N );
        std::vector<double> pts;
        int cellType;
        if( m.dim == 1 ) {
            const double height = ( m.nodeXY[2 * ( nNodes - 1 )] - m.nodeXY[0] ) / 10;
            pts.resize( 3 * size_t( 2 * nNodes ), 0.0 );
            for( int i = 0; i < nNodes; ++i ) {
                pts[3 * i]                = m.nodeXY[2 * i];
                pts[3 * ( i + nNodes )]     = m.nodeXY[2 * i];
                pts[3 * ( i + nNodes ) + 1] = height;
            }
            for( int j = 0; j < N; ++j ) {
                const int a = m.cellNodes[2 * j], b = m.cellNodes[2 * j + 1];
                cells[j]    = {a, a + nNodes, b + nNodes, b};
            }
            cellType = 9;    // VTK_QUAD
        }
        else {
            pts.resize( 3 * size_t( nNodes ), 0.0 );
            for( int i = 0; i < nNodes; ++i ) {
                pts[3 * i]     = m.nodeXY[2 * i];
                pts[3 * i + 1] = m.nodeXY[2 * i + 1];
            }
            for( int j = 0; j < N; ++j ) cells[j] = {m.cellNodes[3 * j], m.cellNodes[3 * j + 1], m.cellNodes[3 * j + 2]};
            cellType = 5;    // VTK_TRIANGLE
        }
        const int nPts = int( pts.size() / 3 );
        std::fprintf( f, "# vtk DataFile Version 3.0\nUQCreator B200 mean and variance\nASCII\nDATASET UNSTRUCTURED_GRID\n" );
        std::fprintf( f, "POINTS %d double\n", nPts );
        for( int i = 0; i < nPts; ++i ) std::fprintf( f, "%.17g %.17g %.17g\n", pts[3 * i], pts[3 * i + 1], pts[3 * i + 2] );
        const int per = int( cells[0].size() );
        std::fprintf( f, "CELLS %d %d\n", N, N * ( per + 1 ) );
        for( int j = 0; j < N; ++j ) {
            std::fprintf( f, "%d", per );
            for( int v : cells[j] ) std::fprintf( f, " %d", v );
            std::fprintf( f, "\n" );
        }
        std::fprintf( f, "CELL_TYPES %d\n", N );
        for( int j = 0; j < N; ++j ) std::fprintf( f, "%d\n", cellType );
        auto value = [&]( int j, int col ) { return col < 0 ? 0.0 : mv[size_t( j ) * 2 * nS + col]; };
        // cell data
        std::fprintf( f, "CELL_DATA %d\nFIELD FieldData %d\n", N, int( arrs.size() ) );
        for( const Arr& a : arrs ) {
            std::fprintf( f, "%s %d %d double\n", a.name.c_str(), a.comps, N );
            for( int j = 0; j < N; ++j ) {
                for( int c = 0; c < a.comps; ++c ) std::fprintf( f, c ? " %.17g" : "%.17g", value( j, a.cols[c] ) );
                std::fprintf( f, "\n" );
            }
        }
        // point data: mean over the cells that share the point
        std::vector<int> count( nPts, 0 );
        for( int j = 0; j < N; ++j )
            for( int v : cells[j] ) ++count[v];
        std::fprintf( f, "POINT_DATA %d\nFIELD FieldData %d\n", nPts, int( arrs.size() ) );
        for( const Arr& a : arrs ) {
            std::vector<double> acc( size_t( nPts ) * a.comps, 0.0 );
            for( int j = 0; j < N; ++j )
                for( int v : cells[j] )
                    for( int c = 0; c < a.comps; ++c ) acc[size_t( v ) * a.comps + c] += value( j, a.cols[c] );
            std::fprintf( f, "%s %d %d double\n", a.name.c_str(), a.comps, nPts );
            for( int i = 0; i < nPts; ++i ) {
                for( int c = 0; c < a.comps; ++c )
                    std::fprintf( f, c ? " %.17g" : "%.17g", count[i] ? acc[size_t( i ) * a.comps + c] / count[i] : 0.0 );
                std::fprintf( f, "\n" );
            }
        }
        if( std::fclose( f ) != 0 ) throw ConfigError( "cannot write " + file );
        if( m.dim == 1 ) {
            // <file>ExpectedValue / <file>Variance: x, then the states (default stream format)
            const std::string stem = file.substr( 0, file.size() - 4 );
            for( int part = 0; part < 2; ++part ) {
                std::ofstream out( stem + ( part == 0 ? "ExpectedValue" : "Variance" ) );
                for( int j = 0; j < N; ++j ) {
                    out << m.center[2 * j];
                    for( int s2 = 0; s2 < nS; ++s2 ) out << " " << value( j, part * nS + s2 );
                    out << std::endl;
                }
                if( !out ) throw ConfigError( "cannot write " + stem );
            }
        }
        return UQC_OK;
    } );
}

int uqc_export_state( uqc_solver* h, const char* path_prefix ) {
    if( !h || !path_prefix ) return UQC_ERR_ARGUMENT;
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "export of a sharded handle: gather the owned cells (uqc_download_state) instead" );
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    return guarded_dev( h, [&] {
        const size_t N = size_t( h->mesh.nCells ), per = h->ldc;
        std::vector<double> u( N * per ), lam( N * per );
        CK( cudaMemcpyAsync( u.data(), h->d_u, u.size() * sizeof( double ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaMemcpyAsync( lam.data(), h->d_lam, lam.size() * sizeof( double ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaStreamSynchronize( h->stream ) );
        for( int which = 0; which < 2; ++which ) {
            const std::string path = std::string( path_prefix ) + ( which == 0 ? "_moments" : "_duals" );
            FILE* f                = std::fopen( path.c_str(), "w" );
            if( !f ) throw ConfigError( "cannot write " + path );
            const std::vector<double>& v = which == 0 ? u : lam;
            char buf[64];
            for( size_t j = 0; j < N; ++j ) {
                std::string line;
                line.reserve( per * 24 );
                for( size_t k = 0; k < per; ++k ) {
                    // std::setprecision(digits10 = 15) in the default float field: %.15g
                    std::snprintf( buf, sizeof( buf ), "%.15g,", v[j * per + k] );
                    line += buf;
                }
                line += '\n';
                std::fputs( line.c_str(), f );
            }
            if( std::fclose( f ) != 0 ) throw ConfigError( "cannot write " + path );
        }
        // the log a restart reads the previous settings from (main.cpp:160-180)
        write_config_echo( path_prefix, h->cfgName, h->cfgText );
        return UQC_OK;
    } );
}

int uqc_upload_state( uqc_solver* h, const double* u, const double* lambda, const unsigned* level, int layout, double t ) {
    if( !h || ( layout != UQC_LAYOUT_REF && layout != UQC_LAYOUT_STATE_MAJOR ) ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady && ( !u || !lambda ) ) return fail( h, UQC_ERR_STATE, "first upload needs both u and lambda" );
    return guarded_dev( h, [&] {
        const size_t N = size_t( h->mesh.nCells ), bytes = N * h->ldc * sizeof( double );
        std::vector<double> tmp;
        for( int which = 0; which < 2; ++which ) {
            const double* src = which == 0 ? u : lambda;
            double* dst       = which == 0 ? h->d_u : h->d_lam;
            if( !src ) continue;
            if( layout == UQC_LAYOUT_REF ) {
                tmp.resize( N * h->ldc );
                to_layout( h, src, tmp.data(), layout, true );
                src = tmp.data();
                CK( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyHostToDevice, h->stream ) );
                CK( cudaStreamSynchronize( h->stream ) );
            }
            else {
                CK( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyHostToDevice, h->stream ) );
            }
        }
        if( level ) {
            for( size_t j = 0; j < N; ++j )
                if( level[j] >= unsigned( h->tab.nLevels ) ) throw std::invalid_argument( "refinement level out of range" );
            CK( cudaMemcpyAsync( h->d_level, level, N * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
        }
        else if( !h->stateReady ) {
            std::vector<unsigned> lv( N, unsigned( h->tab.nLevels - 1 ) );
            CK( cudaMemcpyAsync( h->d_level, lv.data(), N * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
            CK( cudaStreamSynchronize( h->stream ) );
        }
        if( h->d_factorLevel ) reset_factor_store( h );
        reset_control( h, t );
        h->stateReady = true;
        return UQC_OK;
    } );
}

int uqc_download_state( uqc_solver* h, double* u, double* lambda, unsigned* level, int layout ) {
    if( !h || ( layout != UQC_LAYOUT_REF && layout != UQC_LAYOUT_STATE_MAJOR ) ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state (call uqc_init_state or uqc_upload_state)" );
    return guarded_dev( h, [&] {
        const size_t N = size_t( h->mesh.nCells ), bytes = N * h->ldc * sizeof( double );
        std::vector<double> tmp;
        for( int which = 0; which < 2; ++which ) {
            double* dst       = which == 0 ? u : lambda;
            const double* src = which == 0 ? h->d_u : h->d_lam;
            if( !dst ) continue;
            if( layout == UQC_LAYOUT_REF ) {
                tmp.resize( N * h->ldc );
                CK( cudaMemcpyAsync( tmp.data(), src, bytes, cudaMemcpyDeviceToHost, h->stream ) );
                CK( cudaStreamSynchronize( h->stream ) );
                to_layout( h, tmp.data(), dst, layout, false );
            }
            else {
                CK( cudaMemcpyAsync( dst, src, bytes, cudaMemcpyDeviceToHost, h->stream ) );
            }
        }
        if( level ) CK( cudaMemcpyAsync( level, h->d_level, N * sizeof( unsigned ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaStreamSynchronize( h->stream ) );
        return UQC_OK;
    } );
}

int uqc_solve_closure( uqc_solver* h, uqc_step_info* info ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    return guarded_dev( h, [&] {
        h->launches = 0;
        read_control( h );
        int stepsBefore = h->h_ctl->steps;
        reset_work( h );
        KParams P = make_params( h );
        launch_closure( h, P, 0 );
        CK( cudaGetLastError() );
        int failed = fill_info( h, info, stepsBefore );
        return failed ? fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" ) : UQC_OK;
    } );
}

void ensure_scratch( uqc_solver* h, size_t n );
int uqc_solve_closure_cells( uqc_solver* h, const unsigned* cells, int n_cells, double tol, int max_iter, uqc_step_info* info ) {
    if( !h || n_cells < 0 || ( cells && n_cells == 0 ) || tol < 0.0 || max_iter < 0 ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    if( cells )
        for( int i = 0; i < n_cells; ++i )
            if( cells[i] >= unsigned( h->mesh.nCells ) ) return fail( h, UQC_ERR_ARGUMENT, "cell id out of range" );
    return guarded_dev( h, [&] {
        h->launches = 0;
        read_control( h );
        int stepsBefore = h->h_ctl->steps;
        reset_work( h );
        KParams P = make_params( h );
        if( tol > 0.0 ) P.eps = tol;
        if( max_iter > 0 ) P.maxIter = max_iter;
        if( cells ) {
            // the subset as the kernel's work list (scratch: ids, then their count)
            ensure_scratch( h, size_t( n_cells ) + 1 );
            int* list      = reinterpret_cast<int*>( h->d_xStatus );
            unsigned* cnt  = reinterpret_cast<unsigned*>( h->d_xIters );
            const unsigned n = unsigned( n_cells );
            CK( cudaMemcpyAsync( list, cells, size_t( n_cells ) * sizeof( int ), cudaMemcpyHostToDevice, h->stream ) );
            CK( cudaMemcpyAsync( cnt, &n, sizeof( n ), cudaMemcpyHostToDevice, h->stream ) );
            CK( cudaStreamSynchronize( h->stream ) );    // n lives on this stack frame
            P.activeList  = list;
            P.activeCount = cnt;
            P.listParity  = 0;
        }
        launch_closure( h, P, 0 );
        CK( cudaGetLastError() );
        int failed = fill_info( h, info, stepsBefore );
        return failed ? fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" ) : UQC_OK;
    } );
}

int uqc_moments_mean_var( uqc_solver* h, double* out ) { return uqc_mean_var( h, out ); }

int uqc_cell_status( uqc_solver* h, int* status, int* iterations ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    return guarded_dev( h, [&] {
        size_t N = size_t( h->mesh.nCells );
        if( status ) CK( cudaMemcpyAsync( status, h->d_status, N * sizeof( int ), cudaMemcpyDeviceToHost, h->stream ) );
        if( iterations ) CK( cudaMemcpyAsync( iterations, h->d_iters, N * sizeof( int ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaStreamSynchronize( h->stream ) );
        return UQC_OK;
    } );
}

int uqc_step( uqc_solver* h, int n_steps, uqc_step_info* info ) {
    if( !h || n_steps < 0 ) return UQC_ERR_ARGUMENT;
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "a sharded handle steps through uqc_step_phase" );
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state (call uqc_init_state or uqc_upload_state)" );
    return guarded_dev( h, [&] {
        h->launches     = 0;
        int stepsBefore = h->h_ctl->steps;
        KParams P       = make_params( h );
        // CUDA events around every launch on the handle's stream: per-phase
        // device time summed over the steps of this call.
        if( h->stepEvents.size() < size_t( 3 * n_steps ) ) {
            size_t old = h->stepEvents.size();
            h->stepEvents.resize( 3 * size_t( n_steps ) );
            for( size_t i = old; i < h->stepEvents.size(); ++i ) CK( cudaEventCreate( &h->stepEvents[i] ) );
        }
        for( int s = 0; s < n_steps; ++s ) {
            CK( cudaEventRecord( h->stepEvents[3 * s], h->stream ) );
            enqueue_closure_phase( h, P );
            CK( cudaEventRecord( h->stepEvents[3 * s + 1], h->stream ) );
            enqueue_update( h, P );
            CK( cudaEventRecord( h->stepEvents[3 * s + 2], h->stream ) );
        }
        CK( cudaGetLastError() );
        int failed = fill_info( h, info, stepsBefore );
        h->lastMs[0] = h->lastMs[1] = h->lastMs[2] = 0.f;
        for( int s = 0; s < n_steps; ++s ) {
            float a = 0.f, b = 0.f;
            CK( cudaEventElapsedTime( &a, h->stepEvents[3 * s], h->stepEvents[3 * s + 1] ) );
            CK( cudaEventElapsedTime( &b, h->stepEvents[3 * s + 1], h->stepEvents[3 * s + 2] ) );
            h->lastMs[0] += a;
            h->lastMs[1] += b;
            h->lastMs[2] += a + b;
        }
        return failed ? fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" ) : UQC_OK;
    } );
}

int uqc_step_host( uqc_solver* h, const double* u_in, const double* lambda_in, const unsigned* level_in, double t, double* u_out,
                   double* lambda_out, unsigned* level_out, uqc_step_info* info ) {
    if( !h || !u_in || !lambda_in || !u_out || !lambda_out ) return UQC_ERR_ARGUMENT;
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "a sharded handle steps through uqc_step_phase" );
    if( h->asyncPending ) return fail( h, UQC_ERR_STATE, "a uqc_step_async is in flight" );
    return guarded_dev( h, [&] {
        const int N = h->mesh.nCells;
        if( level_in )
            for( int j = 0; j < N; ++j )
                if( level_in[j] >= unsigned( h->tab.nLevels ) ) throw std::invalid_argument( "refinement level out of range" );
        const int CHUNKS = h->hostChunks;
        if( !h->copyStream ) CK( cudaStreamCreateWithFlags( &h->copyStream, cudaStreamNonBlocking ) );
        if( !h->copyStreamOut ) CK( cudaStreamCreateWithFlags( &h->copyStreamOut, cudaStreamNonBlocking ) );
        if( !h->checkStream ) CK( cudaStreamCreateWithFlags( &h->checkStream, cudaStreamNonBlocking ) );
        if( h->hostEvents.size() < size_t( 3 * CHUNKS + 4 ) ) {
            const size_t old = h->hostEvents.size();
            h->hostEvents.resize( 3 * CHUNKS + 4 );
            for( size_t i = old; i < h->hostEvents.size(); ++i ) CK( cudaEventCreate( &h->hostEvents[i] ) );
        }
        // per chunk c: landed, closure done (later: update done), checked;
        // then start, closure phase end, update end, copies done
        cudaEvent_t* landed  = h->hostEvents.data();
        cudaEvent_t* solved  = landed + CHUNKS;
        cudaEvent_t* checked = solved + CHUNKS;
        cudaEvent_t* ev      = checked + CHUNKS;
        // the state the upload replaces (as uqc_upload_state): levels, no
        // held factors, a fresh control block (synchronous, so the earlier
        // work on the stream is done before the copies start)
        if( level_in )
            CK( cudaMemcpyAsync( h->d_level, level_in, size_t( N ) * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
        else if( !h->stateReady ) {
            std::vector<unsigned> lv( N, unsigned( h->tab.nLevels - 1 ) );
            CK( cudaMemcpyAsync( h->d_level, lv.data(), size_t( N ) * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
        }
        if( h->d_factorLevel ) reset_factor_store( h );
        reset_control( h, t );
        h->stateReady = true;
        h->launches   = 0;
        const int stepsBefore = h->h_ctl->steps;
        const int par         = h->h_ctl->steps & 1;    // the running step's active list
        KParams P             = make_params( h );
        step_lists( h, P );
        const size_t ldc = h->ldc;
        auto lo          = [&]( int c ) { return size_t( N ) * c / CHUNKS; };
        CK( cudaEventRecord( ev[0], h->stream ) );
        // moments and duals in chunks of cells on the upload stream
        for( int c = 0; c < CHUNKS; ++c ) {
            const size_t c0 = lo( c ), c1 = lo( c + 1 );
            if( c1 > c0 ) {
                CK( cudaMemcpyAsync( h->d_u + c0 * ldc, u_in + c0 * ldc, ( c1 - c0 ) * ldc * sizeof( double ), cudaMemcpyHostToDevice, h->copyStream ) );
                CK( cudaMemcpyAsync( h->d_lam + c0 * ldc, lambda_in + c0 * ldc, ( c1 - c0 ) * ldc * sizeof( double ), cudaMemcpyHostToDevice,
                                     h->copyStream ) );
            }
            CK( cudaEventRecord( landed[c], h->copyStream ) );
        }
        // the closure half of the step chunk by chunk as each lands: the
        // check of the chunk's cells, the Newton of those it lists (the work
        // counters and the list start again from zero for each chunk), then
        // the chunk's final duals go down on the download stream, beside the
        // later chunks' uploads. A cell's closure reads and writes only its
        // own state, so the chunks give the cells the unchunked results.
        auto download_duals = [&]( size_t c0, size_t c1, cudaEvent_t after ) {
            CK( cudaEventRecord( after, h->stream ) );
            CK( cudaStreamWaitEvent( h->copyStreamOut, after, 0 ) );
            if( c1 > c0 )
                CK( cudaMemcpyAsync( lambda_out + c0 * ldc, h->d_lam + c0 * ldc, ( c1 - c0 ) * ldc * sizeof( double ), cudaMemcpyDeviceToHost,
                                     h->copyStreamOut ) );
        };
        if( h->cfg.newtonMode != 2 ) {
            // the checks on a stream of their own, so that chunk c + 1's check
            // fills the SMs that chunk c's Newton leaves idle in its tail; the
            // chunks alternate between the two active lists (the next step's
            // list is not in use before the update), and a check waits until
            // the Newton two chunks back has consumed its list
            for( int c = 0; c < CHUNKS; ++c ) {
                const size_t c0 = lo( c ), c1 = lo( c + 1 );
                const int lp    = c & 1;
                KParams Q       = P;
                Q.activeList    = h->d_activeList + size_t( lp ) * N;
                Q.activeCount   = &h->d_ctl->nActive[lp];
                Q.listParity    = 0;
                CK( cudaStreamWaitEvent( h->checkStream, landed[c], 0 ) );
                if( c >= 2 ) CK( cudaStreamWaitEvent( h->checkStream, solved[c - 2], 0 ) );
                if( c1 > c0 ) {
                    if( c >= 2 ) CK( cudaMemsetAsync( &h->d_ctl->nActive[lp], 0, sizeof( unsigned ), h->checkStream ) );
                    KParams K    = Q;
                    K.cellBase   = int( c0 );
                    K.nWork      = int( c1 - c0 );
                    void* args[] = {&K};
                    CK( cudaLaunchKernel( pick_check( h->cfg.closure ), dim3( h->checkGrid ), dim3( h->checkBlock ), args, h->checkSmem,
                                          h->checkStream ) );
                    ++h->launches;
                }
                CK( cudaEventRecord( checked[c], h->checkStream ) );
                CK( cudaStreamWaitEvent( h->stream, checked[c], 0 ) );
                if( c1 > c0 ) {
                    if( c > 0 ) {
                        reset_work( h );
                        CK( cudaMemsetAsync( &h->d_ctl->v2Work[0], 0, sizeof( h->d_ctl->v2Work ) + sizeof( h->d_ctl->v2Count ), h->stream ) );
                    }
                    launch_closure( h, Q, 1 );
                }
                download_duals( c0, c1, solved[c] );
            }
            // the next step's list (k_update's, with its convergence test) starts empty
            CK( cudaMemsetAsync( &h->d_ctl->nActive[( par + 1 ) & 1], 0, sizeof( unsigned ), h->stream ) );
        }
        else {
            // safe mode: every cell takes Newton steps (no check), all at once
            CK( cudaStreamWaitEvent( h->stream, landed[CHUNKS - 1], 0 ) );
            launch_closure( h, P, 1 );
            download_duals( 0, size_t( N ), solved[0] );
        }
        CK( cudaEventRecord( ev[1], h->stream ) );
        // the update in chunks of cells too, each chunk's moments going down
        // as its launch ends (the residual sums the launches' CTA partials in
        // order: the same terms as one launch, in another order)
        const int need = h->updateGrid * CHUNKS;
        if( need > h->chunkPartialCap ) {
            if( h->d_chunkPartial ) {
                CK( cudaStreamSynchronize( h->stream ) );
                cudaFree( h->d_chunkPartial );
            }
            h->d_chunkPartial  = dalloc<double>( size_t( need ) );
            h->chunkPartialCap = need;
        }
        {
            KParams U = P;
            step_lists( h, U );
            U.finishInUpdate = update_test_on( h );
            U.blockPartial   = h->d_chunkPartial;
            U.updChunks      = CHUNKS;
            void* ku         = pick( h->cfg.closure, h->group, update_kernel_id( h, U.finishInUpdate != 0 ) );
            for( int c = 0; c < CHUNKS; ++c ) {
                const size_t c0 = lo( c ), c1 = lo( c + 1 );
                U.cellBase   = int( c0 );
                U.nWork      = int( c1 - c0 );
                U.updChunk   = c;
                void* args[] = {&U};
                launch( h, ku, h->updateGrid, h->updateBlock, h->updateSmem, args );
                CK( cudaEventRecord( solved[c], h->stream ) );
                CK( cudaStreamWaitEvent( h->copyStreamOut, solved[c], 0 ) );
                if( c1 > c0 )
                    CK( cudaMemcpyAsync( u_out + c0 * ldc, h->d_u + c0 * ldc, ( c1 - c0 ) * ldc * sizeof( double ), cudaMemcpyDeviceToHost,
                                         h->copyStreamOut ) );
            }
        }
        CK( cudaEventRecord( ev[2], h->stream ) );
        if( level_out ) CK( cudaMemcpyAsync( level_out, h->d_level, size_t( N ) * sizeof( unsigned ), cudaMemcpyDeviceToHost, h->copyStreamOut ) );
        CK( cudaEventRecord( ev[3], h->copyStreamOut ) );
        CK( cudaStreamWaitEvent( h->stream, ev[3], 0 ) );    // later work on the stream sees the copies done
        CK( cudaGetLastError() );
        CK( cudaStreamSynchronize( h->copyStreamOut ) );
        int failed = fill_info( h, info, stepsBefore );
        float a = 0.f, b = 0.f;
        CK( cudaEventElapsedTime( &a, ev[0], ev[1] ) );
        CK( cudaEventElapsedTime( &b, ev[1], ev[2] ) );
        h->lastMs[0] = a;    // closure phase, from the start of the first copy
        h->lastMs[1] = b;
        h->lastMs[2] = a + b;
        return failed ? fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" ) : UQC_OK;
    } );
}

int uqc_run( uqc_solver* h, double t_end, uqc_step_info* info ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "a sharded handle steps through uqc_step_phase" );
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    return guarded_dev( h, [&] {
        if( t_end > 0 ) {
            h->cfg.tEnd = t_end;
            read_control( h );
            h->h_ctl->tEnd   = t_end;
            h->h_ctl->active = ( h->h_ctl->t < t_end && h->h_ctl->residual > h->h_ctl->minResidual ) ? 1 : 0;
            CK( cudaMemcpyAsync( h->d_ctl, h->h_ctl, sizeof( Control ), cudaMemcpyHostToDevice, h->stream ) );
        }
        read_control( h );
        int stepsBefore = h->h_ctl->steps;
        unsigned long long it0 = h->lastIters, ls0 = h->lastLs;
        int f0 = h->lastFailed;
        while( h->h_ctl->active ) {
            launch_steps( h, 32 );    // kernels turn into no-ops once the loop condition fails
            read_control( h );
        }
        CK( cudaGetLastError() );
        h->lastIters  = it0;
        h->lastLs     = ls0;
        h->lastFailed = f0;
        int failed    = fill_info( h, info, stepsBefore );
        return failed ? fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" ) : UQC_OK;
    } );
}

int uqc_mean_var( uqc_solver* h, double* out ) {
    if( !h || !out ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    return guarded_dev( h, [&] {
        const size_t N = size_t( h->mesh.nCells ), cnt = N * 2 * h->nS;
        double* d_out  = dalloc<double>( cnt );
        KParams P      = make_params( h );
        void* args[]   = {&P, &d_out};
        launch( h, pick( h->cfg.closure, h->group, 3 ), h->auxGrid, h->auxBlock, h->mvSmem, args );
        CK( cudaMemcpyAsync( out, d_out, cnt * sizeof( double ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaStreamSynchronize( h->stream ) );
        cudaFree( d_out );
        return UQC_OK;
    } );
}

void ensure_scratch( uqc_solver* h, size_t n ) {
    if( n <= h->xCap ) return;
    for( void* p : {(void*)h->d_xLam, (void*)h->d_xU, (void*)h->d_xNt, (void*)h->d_xStatus, (void*)h->d_xIters} )
        if( p ) cudaFree( p );
    h->d_xLam    = dalloc<double>( n * h->ldc );
    h->d_xU      = dalloc<double>( n * h->ldc );
    h->d_xNt     = dalloc<unsigned>( n );
    h->d_xStatus = dalloc<int>( n );
    h->d_xIters  = dalloc<int>( n );
    h->xCap      = n;
}

static void closure_on( uqc_solver* h, int n, double* d_lam, const double* d_u, const unsigned* d_nt, int* d_status, int* d_iters ) {
    KParams P     = make_params( h );
    P.nCells      = n;
    P.nWork       = n;
    P.lam         = d_lam;
    P.u           = const_cast<double*>( d_u );
    P.level       = nullptr;
    P.nTotalCell  = d_nt;
    P.status      = d_status;
    P.iters       = d_iters;
    reset_work( h );
    launch_closure( h, P, 0 );
    CK( cudaGetLastError() );
}

int uqc_closure_solve_host( uqc_solver* h, int n, double* lambda, const double* u, const unsigned* n_total, int layout, int* status ) {
    if( !h || n < 0 || !lambda || !u || ( layout != UQC_LAYOUT_REF && layout != UQC_LAYOUT_STATE_MAJOR ) ) return UQC_ERR_ARGUMENT;
    if( n == 0 ) return UQC_OK;
    return guarded_dev( h, [&] {
        h->launches = 0;
        ensure_scratch( h, size_t( n ) );
        const size_t cnt = size_t( n ) * h->ldc, nT = size_t( h->tab.nT ), nS = size_t( h->nS );
        std::vector<double> L( cnt ), U( cnt );
        for( size_t j = 0; j < size_t( n ); ++j )
            for( size_t s = 0; s < nS; ++s )
                for( size_t i = 0; i < nT; ++i ) {
                    size_t sm = j * nS * nT + s * nT + i, src = layout == UQC_LAYOUT_REF ? j * nS * nT + i * nS + s : sm;
                    L[sm] = lambda[src];
                    U[sm] = u[src];
                }
        std::vector<unsigned> nt( n, unsigned( nT ) );
        if( n_total )
            for( int j = 0; j < n; ++j ) {
                if( std::find( h->tab.nTLevel.begin(), h->tab.nTLevel.end(), int( n_total[j] ) ) == h->tab.nTLevel.end() )
                    throw std::invalid_argument( "n_total[" + std::to_string( j ) + "] is not a refinement level size" );
                nt[j] = n_total[j];
            }
        CK( cudaMemcpyAsync( h->d_xLam, L.data(), cnt * sizeof( double ), cudaMemcpyHostToDevice, h->stream ) );
        CK( cudaMemcpyAsync( h->d_xU, U.data(), cnt * sizeof( double ), cudaMemcpyHostToDevice, h->stream ) );
        CK( cudaMemcpyAsync( h->d_xNt, nt.data(), n * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
        closure_on( h, n, h->d_xLam, h->d_xU, h->d_xNt, h->d_xStatus, h->d_xIters );
        std::vector<int> st( n );
        CK( cudaMemcpyAsync( L.data(), h->d_xLam, cnt * sizeof( double ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaMemcpyAsync( st.data(), h->d_xStatus, n * sizeof( int ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaStreamSynchronize( h->stream ) );
        for( size_t j = 0; j < size_t( n ); ++j )
            for( size_t s = 0; s < nS; ++s )
                for( size_t i = 0; i < nT; ++i ) {
                    size_t sm = j * nS * nT + s * nT + i, dst = layout == UQC_LAYOUT_REF ? j * nS * nT + i * nS + s : sm;
                    lambda[dst] = L[sm];
                }
        int bad = 0;
        for( int j = 0; j < n; ++j ) {
            if( status ) status[j] = st[j];
            bad += st[j] != 0;
        }
        return bad ? fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( bad ) + " cells did not converge" ) : UQC_OK;
    } );
}

int uqc_closure_solve_device( uqc_solver* h, int n, double* d_lambda, const double* d_u, const unsigned* d_n_total, int* d_status ) {
    if( !h || n < 0 || !d_lambda || !d_u ) return UQC_ERR_ARGUMENT;
    if( n == 0 ) return UQC_OK;
    return guarded_dev( h, [&] {
        h->launches = 0;
        ensure_scratch( h, size_t( n ) );
        unsigned* nt = const_cast<unsigned*>( d_n_total );
        if( !nt ) {
            std::vector<unsigned> v( n, unsigned( h->tab.nT ) );
            CK( cudaMemcpyAsync( h->d_xNt, v.data(), n * sizeof( unsigned ), cudaMemcpyHostToDevice, h->stream ) );
            CK( cudaStreamSynchronize( h->stream ) );
            nt = h->d_xNt;
        }
        closure_on( h, n, d_lambda, d_u, nt, d_status ? d_status : h->d_xStatus, h->d_xIters );
        return UQC_OK;
    } );
}

// ===================================================== asynchronous stepping

int uqc_step_async( uqc_solver* h, int n_steps ) {
    if( !h || n_steps < 0 ) return UQC_ERR_ARGUMENT;
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "a sharded handle steps through uqc_step_phase" );
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state (call uqc_init_state or uqc_upload_state)" );
    if( h->asyncPending ) return fail( h, UQC_ERR_STATE, "the previous uqc_step_async has not been queried to completion" );
    return guarded_dev( h, [&] {
        if( !h->asyncEv ) CK( cudaEventCreateWithFlags( &h->asyncEv, cudaEventDisableTiming ) );
        h->launches         = 0;
        h->asyncStepsBefore = h->h_ctl->steps;    // the mirror is current: no work is in flight
        launch_steps( h, n_steps );
        CK( cudaMemcpyAsync( h->h_ctl, h->d_ctl, sizeof( Control ), cudaMemcpyDeviceToHost, h->stream ) );
        CK( cudaEventRecord( h->asyncEv, h->stream ) );
        CK( cudaGetLastError() );
        h->asyncPending = true;
        return UQC_OK;
    } );
}

int uqc_step_query( uqc_solver* h, uqc_step_info* info ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    if( !h->asyncPending ) return fail( h, UQC_ERR_STATE, "no uqc_step_async in flight" );
    return guarded( h, [&] {
        cudaError_t e = cudaEventQuery( h->asyncEv );
        if( e == cudaErrorNotReady ) return 0;
        CK( e );
        h->asyncPending = false;
        const int failed = fill_info_host( h, info, h->asyncStepsBefore );
        if( failed ) return fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" );
        return 1;
    } );
}

int uqc_device_bytes( const uqc_solver* h, unsigned long long* bytes ) {
    if( !h || !bytes ) return UQC_ERR_ARGUMENT;
    *bytes = device_bytes_of( h );
    return UQC_OK;
}

// ===================================================== spatial sharding

int uqc_partition( uqc_solver* h, int rank, int n_ranks ) {
    if( !h || n_ranks < 1 || rank < 0 || rank >= n_ranks ) return UQC_ERR_ARGUMENT;
    if( h->deviceReady ) return fail( h, UQC_ERR_STATE, "uqc_partition must precede the first call that uses the device" );
    if( h->sharded ) return fail( h, UQC_ERR_STATE, "the handle is already sharded" );
    return guarded( h, [&] {
        if( n_ranks > h->mesh.nCells ) throw ConfigError( "more ranks than cells" );
        const std::vector<int> owner = partition_cells( h->mesh, n_ranks );
        h->mesh    = shard_mesh( h->mesh, owner, rank, n_ranks, h->shard );
        h->sharded = true;
        return UQC_OK;
    } );
}

int uqc_get_shard( const uqc_solver* h, uqc_shard_info* info, int* global_ids, int* peers, int* send_counts, int* recv_counts,
                   int* send_cells ) {
    if( !h || !info ) return UQC_ERR_ARGUMENT;
    const ShardPlan& s = h->shard;
    const bool on      = h->sharded;
    info->rank         = on ? s.rank : 0;
    info->n_ranks      = on ? s.nRanks : 1;
    info->n_global     = on ? s.nGlobal : h->mesh.nCells;
    info->n_owned      = on ? s.nOwned : h->mesh.nCells;
    info->n_halo       = h->mesh.nCells - info->n_owned;
    info->n_peers      = on ? int( s.peers.size() ) : 0;
    info->n_send       = on ? int( s.sendCells.size() ) : 0;
    info->row_doubles  = h->nS * h->tab.nQ;
    for( int i = 0; i < h->mesh.nCells && global_ids; ++i ) global_ids[i] = on ? s.globalId[i] : i;
    for( int p = 0; p < info->n_peers; ++p ) {
        if( peers ) peers[p] = s.peers[p];
        if( send_counts ) send_counts[p] = s.sendCount[p];
        if( recv_counts ) recv_counts[p] = s.recvCount[p];
    }
    for( int i = 0; i < info->n_send && send_cells; ++i ) send_cells[i] = s.sendCells[i];
    return UQC_OK;
}

int uqc_shard_buffers( uqc_solver* h, double** d_halo_rows, unsigned long long** d_dt_bits, double** d_residual ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    return guarded_dev( h, [&] {
        const size_t row = size_t( h->nS ) * h->tab.nQ;
        const size_t own = size_t( h->sharded ? h->shard.nOwned : h->mesh.nCells );
        if( d_halo_rows ) *d_halo_rows = h->d_uQ + own * row;
        if( d_dt_bits ) *d_dt_bits = &h->d_ctl->dtBits;
        if( d_residual ) *d_residual = &h->d_ctl->residual;
        return UQC_OK;
    } );
}

__global__ void k_halo_pack( const double* __restrict__ uQ, const int* __restrict__ cells, int n, int row, double* __restrict__ out ) {
    for( int r = blockIdx.x; r < n; r += gridDim.x ) {
        const double* src = uQ + size_t( cells[r] ) * row;
        double* dst       = out + size_t( r ) * row;
        for( int i = threadIdx.x; i < row; i += blockDim.x ) dst[i] = src[i];
    }
}

int uqc_halo_pack( uqc_solver* h, double* d_send ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    const int n = h->sharded ? int( h->shard.sendCells.size() ) : 0;
    if( n == 0 ) return UQC_OK;
    if( !d_send ) return UQC_ERR_ARGUMENT;
    return guarded_dev( h, [&] {
        const int row = h->nS * h->tab.nQ, grid = std::min( n, 4 * h->numSMs );
        k_halo_pack<<<grid, 128, 0, h->stream>>>( h->d_uQ, h->d_sendCells, n, row, d_send );
        ++h->launches;
        CK( cudaGetLastError() );
        return UQC_OK;
    } );
}

int uqc_step_phase( uqc_solver* h, int phase, uqc_step_info* info ) {
    if( !h || phase < 0 || phase > 1 ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state (call uqc_init_state or uqc_upload_state)" );
    if( h->asyncPending ) return fail( h, UQC_ERR_STATE, "a uqc_step_async is in flight" );
    return guarded_dev( h, [&] {
        if( phase == 0 ) h->launches = 0;
        const int stepsBefore = h->h_ctl->steps;
        KParams P             = make_params( h );
        if( phase == 0 )
            enqueue_closure_phase( h, P );
        else
            enqueue_update( h, P );
        CK( cudaGetLastError() );
        if( phase == 1 && info ) {
            const int failed = fill_info( h, info, stepsBefore );
            if( failed ) return fail( h, UQC_ERR_NOT_CONVERGED, std::to_string( failed ) + " cells did not converge" );
        }
        return int( UQC_OK );
    } );
}

// ===================================================== request server

struct uqc_request {
    long long id       = 0;
    uqc_solver* h      = nullptr;
    int state          = UQC_REQ_QUEUED;
    int status         = UQC_OK;
    int precision      = UQC_FP64;
    int nCells = 0, nStates = 0, steps = 0;
    double t           = 0.0;
    long long iters    = 0;
    unsigned long long bytes = 0;
    bool admitted            = false;    // its bytes count against the budget
    bool stepping            = false;    // a slice of steps is in flight
    double submitMs = 0, admitMs = 0, doneMs = 0;
    double workPerStep = 0;    // estimated device work of one time step (cells x duals x nodes)
    int horizon        = 0;    // time steps to the end, when known ([uqc] steps), else 0
    std::vector<double> meanVar;
    std::string err;
};

struct uqc_server {
    unsigned long long budget = 0, used = 0;
    int maxActive = 1, slice = 1;
    int policy      = 0;        // 0: every running request steps (round robin); 1: shortest remaining time first
    int maxStepping = 0;        // policy 1: requests with a slice in flight at a time (0: no limit)
    double aging    = 1.0;      // policy 1: ms of remaining service time that one ms of waiting offsets
    double workDone = 0.0;      // work of the finished slices (units of uqc_request::workPerStep)
    double busyMs   = 0.0;      // time with requests running (between progress calls)
    double lastPassMs = -1.0;
    long long nextId = 1;
    std::map<long long, uqc_request> reqs;
    std::deque<long long> queue;      // waiting, in submission order
    std::vector<long long> running;
    int done = 0;
    std::chrono::steady_clock::time_point t0;
    std::string err;
    // submissions may come from another thread than progress(): the server's
    // state is changed under this lock (a submission takes it only to enqueue,
    // after building its solver)
    mutable std::recursive_mutex mu;
    double now() const { return std::chrono::duration<double, std::milli>( std::chrono::steady_clock::now() - t0 ).count(); }
};

namespace {
int sfail( uqc_server* s, int code, const std::string& m ) {
    s->err = m;
    return code;
}
void retire( uqc_server* s, uqc_request& r, int status, const std::string& err ) {
    r.status = status;
    r.err    = err;
    r.state  = status == UQC_OK ? UQC_REQ_DONE : UQC_REQ_FAILED;
    r.doneMs = s->now();
    if( r.h ) {
        uqc_destroy( r.h );    // frees the request's device memory
        r.h = nullptr;
    }
    if( r.admitted ) {
        s->used -= r.bytes;
        r.admitted = false;
    }
    ++s->done;
}
}    // namespace

int uqc_server_create( unsigned long long device_budget_bytes, int max_active, int steps_per_slice, uqc_server** out ) {
    if( !out || device_budget_bytes == 0 || max_active < 1 || steps_per_slice < 1 ) return UQC_ERR_ARGUMENT;
    uqc_server* s = new( std::nothrow ) uqc_server();
    if( !s ) return UQC_ERR_MEMORY;
    s->budget    = device_budget_bytes;
    s->maxActive = max_active;
    s->slice     = steps_per_slice;
    s->t0        = std::chrono::steady_clock::now();
    *out         = s;
    return UQC_OK;
}

void uqc_server_destroy( uqc_server* s ) {
    if( !s ) return;
    for( auto& kv : s->reqs )
        if( kv.second.h ) uqc_destroy( kv.second.h );
    delete s;
}

const char* uqc_server_last_error( const uqc_server* s ) { return s ? s->err.c_str() : "null server"; }

int uqc_server_submit( uqc_server* s, const char* toml_text, int precision, long long* id ) {
    if( !s || !toml_text || !id || ( precision != UQC_FP64 && precision != UQC_MIXED ) ) return UQC_ERR_ARGUMENT;
    uqc_request r;
    char err[512] = {0};
    int rc = uqc_create_from_string( toml_text, nullptr, &r.h, err, sizeof( err ) );    // host side only
    std::lock_guard<std::recursive_mutex> lock( s->mu );
    if( rc != UQC_OK ) return sfail( s, rc, err );
    r.id        = s->nextId++;
    r.precision = precision;
    r.nCells    = r.h->mesh.nCells;
    r.nStates   = r.h->nS;
    r.bytes     = device_bytes_of( r.h ) + ( precision == UQC_MIXED && r.h->chord ? factor_store_bytes( r.h ) : 0 );
    r.submitMs  = s->now();
    r.workPerStep = double( r.nCells ) * double( r.h->ldc ) * double( r.h->tab.nQ );
    r.horizon     = r.h->cfg.maxSteps;
    *id         = r.id;
    s->queue.push_back( r.id );
    s->reqs.emplace( r.id, std::move( r ) );
    return UQC_OK;
}

namespace {
// Priority of a request under the shortest-remaining-time policy (smaller
// first), in ms: its remaining work over the server's measured rate (work of
// finished slices per ms with requests running), minus its waiting time
// times the aging factor, so that a request that has waited as long as its
// remaining service time ranks with one that is about to finish.
double priority( const uqc_server* s, const uqc_request& r, double now ) {
    const int left    = r.horizon > 0 ? std::max( 0, r.horizon - r.steps ) : 1000;
    const double rate = s->busyMs > 0.0 && s->workDone > 0.0 ? s->workDone / s->busyMs : 1e6;
    return r.workPerStep * double( left ) / rate - s->aging * ( now - r.submitMs );
}

// Queues the next slice of steps of idle running requests: all of them
// (policy 0), or in priority order while fewer than maxStepping have a slice
// in flight (policy 1). A request whose slice cannot be queued is retired.
void launch_slices( uqc_server* s ) {
    const double now = s->now();
    int inFlight     = 0;
    std::vector<std::pair<double, long long>> idle;
    for( long long id : s->running ) {
        const uqc_request& r = s->reqs[id];
        if( r.stepping )
            ++inFlight;
        else
            idle.emplace_back( s->policy == 1 ? priority( s, r, now ) : 0.0, id );
    }
    if( s->policy == 1 ) std::stable_sort( idle.begin(), idle.end() );
    for( auto& pr : idle ) {
        if( s->policy == 1 && s->maxStepping > 0 && inFlight >= s->maxStepping ) break;
        uqc_request& r = s->reqs[pr.second];
        const int rc   = uqc_step_async( r.h, s->slice );
        if( rc != UQC_OK ) {
            retire( s, r, rc, uqc_last_error( r.h ) );
            s->running.erase( std::find( s->running.begin(), s->running.end(), pr.second ) );
            continue;
        }
        r.stepping = true;
        ++inFlight;
    }
}
}    // namespace

int uqc_server_progress( uqc_server* s, int* n_queued, int* n_running, int* n_done ) {
    if( !s ) return UQC_ERR_ARGUMENT;
    std::lock_guard<std::recursive_mutex> lock( s->mu );
    const double pass = s->now();
    if( s->lastPassMs >= 0.0 && !s->running.empty() ) s->busyMs += pass - s->lastPassMs;
    s->lastPassMs = pass;
    // running requests: collect finished slices, retire finished solves
    for( size_t k = 0; k < s->running.size(); ) {
        uqc_request& r = s->reqs[s->running[k]];
        bool finished  = false;
        if( r.stepping ) {
            uqc_step_info info{};
            const int q = uqc_step_query( r.h, &info );
            if( q == 0 ) {
                ++k;
                continue;
            }
            r.stepping = false;
            if( q < 0 ) {
                retire( s, r, q, uqc_last_error( r.h ) );
                finished = true;
            }
            else {
                r.steps += info.steps;
                s->workDone += r.workPerStep * double( info.steps );
                r.iters += info.newton_iterations;
                r.t = info.t;
                if( !info.running ) {
                    r.meanVar.assign( size_t( r.nCells ) * 2 * r.nStates, 0.0 );
                    const int rc = uqc_mean_var( r.h, r.meanVar.data() );
                    retire( s, r, rc, rc == UQC_OK ? "" : uqc_last_error( r.h ) );
                    finished = true;
                }
            }
        }
        if( finished )
            s->running.erase( s->running.begin() + long( k ) );
        else
            ++k;
    }
    // next slices: every idle running request (round robin), or the idle ones
    // with the least remaining work while fewer than maxStepping are in flight
    launch_slices( s );
    // admission, first fit: in submission order (round robin) or by priority
    if( s->policy == 1 && s->queue.size() > 1 ) {
        const double now = s->now();
        std::stable_sort( s->queue.begin(), s->queue.end(), [&]( long long a, long long b ) {
            return priority( s, s->reqs[a], now ) < priority( s, s->reqs[b], now );
        } );
    }
    for( auto it = s->queue.begin(); it != s->queue.end() && int( s->running.size() ) < s->maxActive; ) {
        uqc_request& r = s->reqs[*it];
        if( r.bytes > s->budget ) {
            retire( s, r, UQC_ERR_CAPACITY,
                    "request needs " + std::to_string( r.bytes ) + " device bytes, the server budget is " + std::to_string( s->budget ) );
            it = s->queue.erase( it );
            continue;
        }
        if( s->used + r.bytes > s->budget ) {
            ++it;
            continue;
        }
        s->used += r.bytes;
        r.admitted = true;
        r.state    = UQC_REQ_RUNNING;
        r.admitMs = s->now();
        int rc    = uqc_init_state( r.h );
        if( rc == UQC_OK && r.precision == UQC_MIXED ) rc = uqc_set_precision( r.h, UQC_MIXED );
        if( rc != UQC_OK )
            retire( s, r, rc, uqc_last_error( r.h ) );
        else
            s->running.push_back( r.id );    // its first slice goes out with the next pass's slices
        it = s->queue.erase( it );
    }
    // first slices of the requests admitted in this pass
    launch_slices( s );
    if( n_queued ) *n_queued = int( s->queue.size() );
    if( n_running ) *n_running = int( s->running.size() );
    if( n_done ) *n_done = s->done;
    return UQC_OK;
}

int uqc_server_set_option( uqc_server* s, const char* key, double value ) {
    if( !s || !key ) return UQC_ERR_ARGUMENT;
    std::lock_guard<std::recursive_mutex> lock( s->mu );
    const std::string k = key;
    if( k == "policy" ) {
        if( value != 0.0 && value != 1.0 ) return sfail( s, UQC_ERR_ARGUMENT, "policy must be 0 or 1" );
        s->policy = int( value );
        return UQC_OK;
    }
    if( k == "max_stepping" ) {
        if( value < 0 ) return sfail( s, UQC_ERR_ARGUMENT, "max_stepping must be >= 0" );
        s->maxStepping = int( value );
        return UQC_OK;
    }
    if( k == "aging" ) {
        if( !( value >= 0 ) ) return sfail( s, UQC_ERR_ARGUMENT, "aging must be >= 0" );
        s->aging = value;
        return UQC_OK;
    }
    return sfail( s, UQC_ERR_ARGUMENT, "unknown server option '" + k + "'" );
}

int uqc_server_request( const uqc_server* s, long long id, uqc_request_info* info, double* mean_var ) {
    if( !s || !info ) return UQC_ERR_ARGUMENT;
    std::lock_guard<std::recursive_mutex> lock( s->mu );
    auto it = s->reqs.find( id );
    if( it == s->reqs.end() ) return UQC_ERR_ARGUMENT;
    const uqc_request& r    = it->second;
    info->id                = r.id;
    info->state             = r.state;
    info->status            = r.status;
    info->n_cells           = r.nCells;
    info->n_states          = r.nStates;
    info->steps             = r.steps;
    info->t                 = r.t;
    info->newton_iterations = r.iters;
    info->device_bytes      = r.bytes;
    info->submit_ms         = r.submitMs;
    info->admit_ms          = r.admitMs;
    info->done_ms           = r.doneMs;
    if( mean_var && r.state == UQC_REQ_DONE ) std::memcpy( mean_var, r.meanVar.data(), r.meanVar.size() * sizeof( double ) );
    return UQC_OK;
}

const char* uqc_server_request_error( const uqc_server* s, long long id ) {
    if( !s ) return "null server";
    std::lock_guard<std::recursive_mutex> lock( s->mu );
    auto it = s->reqs.find( id );
    return it == s->reqs.end() ? "unknown request" : it->second.err.c_str();
}

int uqc_server_release( uqc_server* s, long long id ) {
    if( !s ) return UQC_ERR_ARGUMENT;
    std::lock_guard<std::recursive_mutex> lock( s->mu );
    auto it = s->reqs.find( id );
    if( it == s->reqs.end() || ( it->second.state != UQC_REQ_DONE && it->second.state != UQC_REQ_FAILED ) )
        return sfail( s, UQC_ERR_STATE, "request " + std::to_string( id ) + " is not finished" );
    s->reqs.erase( it );
    return UQC_OK;
}

int uqc_last_timing( uqc_solver* h, float* ms3 ) {
    if( !h || !ms3 ) return UQC_ERR_ARGUMENT;
    for( int i = 0; i < 3; ++i ) ms3[i] = h->lastMs[i];
    return UQC_OK;
}

int uqc_device_state( uqc_solver* h, double** d_u, double** d_lambda ) {
    if( !h ) return UQC_ERR_ARGUMENT;
    int rc = guarded( h, [&] {
        ensure_device( h );
        invalidate_lists( h );    // the caller may write the state: the next step tests every cell
        return UQC_OK;
    } );
    if( rc != UQC_OK ) return rc;
    if( d_u ) *d_u = h->d_u;
    if( d_lambda ) *d_lambda = h->d_lam;
    return UQC_OK;
}

int uqc_last_launch_count( uqc_solver* h ) { return h ? h->launches : 0; }

int uqc_debug_mixed_inverse( uqc_solver* h, int n, const int* cells, int form, float* out ) {
    if( !h || n < 1 || !cells || !out || ( form != 1 && form != 2 ) ) return UQC_ERR_ARGUMENT;
    if( !h->stateReady ) return fail( h, UQC_ERR_STATE, "no state" );
    for( int i = 0; i < n; ++i )
        if( cells[i] < 0 || cells[i] >= h->mesh.nCells ) return fail( h, UQC_ERR_ARGUMENT, "cell id out of range" );
    return guarded_dev( h, [&] {
        if( !h->v2Mode ) throw ConfigError( "the mixed form's rounds are not available: " + h->v2Why );
        if( form == 2 && h->v2Mode != 2 ) throw ConfigError( "tensor-core Hessian not available: " + h->v2Why );
        if( n > h->mesh.nCells ) throw ConfigError( "too many cells" );
        if( !h->d_gStore ) {
            const int v = h->v2Mode;
            reset_factor_store( h );
            h->v2Mode = v;
        }
        read_control( h );
        const Control saved = *h->h_ctl;
        Control c           = saved;
        c.active            = 1;
        c.v2Error           = 0;
        for( int r = 0; r < 16; ++r ) c.v2Work[r] = 0;
        for( int r = 0; r < 4; ++r ) c.v2Count[r] = 0;
        c.v2Count[0] = unsigned( n );
        *h->h_ctl    = c;
        CK( cudaMemcpyAsync( h->d_ctl, h->h_ctl, sizeof( Control ), cudaMemcpyHostToDevice, h->stream ) );
        CK( cudaMemcpyAsync( h->d_v2Lists, cells, size_t( n ) * sizeof( int ), cudaMemcpyHostToDevice, h->stream ) );
        KParams P          = make_params( h );
        P.factorStore      = h->d_factorStore;
        P.factorLevel      = h->d_factorLevel;
        P.factorStride     = h->factorStride;
        P.v2Lists          = h->d_v2Lists;
        P.fallbackList     = h->d_fallbackList;
        int r0             = 0;
        void* args[]       = {&P, &r0};
        const int cl       = h->cfg.closure;
        int dev = 0, maxSmem = 0, occ = 0;
        CK( cudaGetDevice( &dev ) );
        CK( cudaDeviceGetAttribute( &maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev ) );
        if( form == 2 ) launch( h, pick( cl, 32, KERNEL_HESS_TC ), h->hessGrid, 256, h->hessSmem, args );
        if( form == 2 && h->invSweep ) {
            launch( h, pick( cl, 32, KERNEL_INVERT_SWEEP ), h->invGrid, h->invBlock, h->invSmem, args );
        }
        else {
            const size_t iws = invert_ws_bytes( h->nS * h->tab.nT, h->tab.nQ, closure_np( cl ), form == 2 );
            const int groups = int( std::min<size_t>( 4, size_t( maxSmem ) / iws ) );
            void* ki         = pick( cl, 32, form == 2 ? KERNEL_INVERT_RAW : KERNEL_INVERT );
            allow_dynamic_smem( ki );
            CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, ki, 64 * groups, iws * groups ) );
            launch( h, ki, std::max( 1, occ ) * h->numSMs, 64 * groups, iws * groups, args );
        }
        const size_t nn = size_t( h->nS ) * h->tab.nT * h->nS * h->tab.nT;
        for( int i = 0; i < n; ++i )
            CK( cudaMemcpyAsync( out + i * nn, h->d_factorStore + size_t( cells[i] ) * h->factorStride, nn * sizeof( float ),
                                 cudaMemcpyDeviceToHost, h->stream ) );
        read_control( h );
        const int err = h->h_ctl->v2Error;
        *h->h_ctl     = saved;
        CK( cudaMemcpyAsync( h->d_ctl, h->h_ctl, sizeof( Control ), cudaMemcpyHostToDevice, h->stream ) );
        CK( cudaMemsetAsync( h->d_factorLevel, 0xFF, size_t( h->mesh.nCells ) * sizeof( int ), h->stream ) );
        CK( cudaStreamSynchronize( h->stream ) );
        if( err ) throw CudaError( "k_hess_tc: the tensor cores did not complete a tile within the wait limit" );
        return UQC_OK;
    } );
}

void* uqc_stream( uqc_solver* h ) {
    if( !h || guarded( h, [&] {
            ensure_device( h );
            return UQC_OK;
        } ) != UQC_OK )
        return nullptr;
    return (void*)h->stream;
}

int uqc_mesh_tri_jitter( int nx, int ny, double jitter, unsigned long long seed, double* xy, int* node_boundary, int* tri ) {
    if( nx < 1 || ny < 1 || !xy || !node_boundary || !tri ) return UQC_ERR_ARGUMENT;
    tri_jitter_nodes( nx, ny, jitter, seed, xy, node_boundary, tri );
    return UQC_OK;
}

}    // extern "C"

#ifdef UQC_PHASE_TIMERS
// Diagnostic builds only: the per-phase cycle counters of k_closure (summed
// over CTAs since the last call), then reset.
extern "C" int uqc_debug_phase_cycles( double* out32 ) {
    for( int i = 0; i < 32; ++i ) out32[i] = 0.0;
    for( int cl = 0; cl < 3; ++cl ) {    // one counter array per kernel translation unit
        void* addr = nullptr;
        try {
            addr = pick( cl, 32, KERNEL_PHASE_COUNTERS );
        } catch( ... ) {
            return UQC_ERR_CUDA;
        }
        unsigned long long v[32];
        if( cudaMemcpy( v, addr, sizeof( v ), cudaMemcpyDeviceToHost ) != cudaSuccess ) return UQC_ERR_CUDA;
        for( int i = 0; i < 32; ++i ) out32[i] += double( v[i] );
        std::memset( v, 0, sizeof( v ) );
        if( cudaMemcpy( addr, v, sizeof( v ), cudaMemcpyHostToDevice ) != cudaSuccess ) return UQC_ERR_CUDA;
    }
    return UQC_OK;
}
#endif

// ===================================================== closure without allocation
//
// Statically allocated scratch of uqc_closure_solve_device_noalloc (layout:
// Control block in the first 256 bytes, then the per-cell iteration counts,
// then the two padded basis tables). In host code the name below is only a
// host-side stand-in for the array: kernels get the device address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__( 256 ) unsigned char g_noallocScratch[UQC_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noallocMutex;
unsigned char* g_noallocAddr[kMaxDevices] = {};    // device address per device id, set once

unsigned char* noalloc_scratch_address() {
    int dev = 0;
    CK( cudaGetDevice( &dev ) );
    if( dev < 0 || dev >= kMaxDevices ) throw std::invalid_argument( "device id beyond the no-alloc table" );
    std::lock_guard<std::mutex> lock( g_noallocMutex );
    if( !g_noallocAddr[dev] ) {
        void* p = nullptr;
        CK( cudaGetSymbolAddress( &p, g_noallocScratch ) );
        g_noallocAddr[dev] = static_cast<unsigned char*>( p );
    }
    return g_noallocAddr[dev];
}
}    // namespace

extern "C" int uqc_closure_solve_device_noalloc( uqc_solver* h, int n, double* d_lambda, const double* d_u, const unsigned* d_n_total,
                                                 int* d_status, void* cuda_stream ) {
    if( !h || n < 0 || ( n > 0 && ( !d_lambda || !d_u || !d_status ) ) ) return UQC_ERR_ARGUMENT;
    if( n > UQC_NOALLOC_MAX_CELLS )
        return fail( h, UQC_ERR_CAPACITY,
                     "uqc_closure_solve_device_noalloc: " + std::to_string( n ) + " cells exceed UQC_NOALLOC_MAX_CELLS = " +
                         std::to_string( UQC_NOALLOC_MAX_CELLS ) + "; split the batch" );
    const size_t tableLen = size_t( h->tab.nQ ) * h->ld + 8;
    if( tableLen + size_t( h->tab.nQ ) > size_t( UQC_NOALLOC_MAX_TABLE ) )
        return fail( h, UQC_ERR_CAPACITY,
                     "uqc_closure_solve_device_noalloc: basis tables of " + std::to_string( tableLen + h->tab.nQ ) +
                         " doubles exceed UQC_NOALLOC_MAX_TABLE = " +
                         std::to_string( UQC_NOALLOC_MAX_TABLE ) + "; use uqc_closure_solve_device" );
    if( n == 0 ) return UQC_OK;
    return guarded( h, [&] {
        cudaStream_t st      = (cudaStream_t)cuda_stream;
        unsigned char* base  = noalloc_scratch_address();
        Control* ctl         = reinterpret_cast<Control*>( base );
        int* iters           = reinterpret_cast<int*>( base + 256 );
        double* tPhi         = reinterpret_cast<double*>( base + 256 + 4 * size_t( UQC_NOALLOC_MAX_CELLS ) );
        double* tPhiWf       = tPhi + UQC_NOALLOC_MAX_TABLE;
        // the array keeps the previous call's contents: the control block must start at zero
        CK( cudaMemsetAsync( ctl, 0, sizeof( Control ), st ) );
        CK( cudaMemcpyAsync( tPhi, h->padPhi.data(), tableLen * sizeof( double ), cudaMemcpyHostToDevice, st ) );
        CK( cudaMemcpyAsync( tPhiWf, h->padPhiWf.data(), tableLen * sizeof( double ), cudaMemcpyHostToDevice, st ) );
        double* tWt = tPhiWf + tableLen;    // node weights after the second table
        CK( cudaMemcpyAsync( tWt, h->padWt.data(), h->padWt.size() * sizeof( double ), cudaMemcpyHostToDevice, st ) );
        KParams P      = make_params( h );
        P.wt           = tWt;
        P.nCells       = n;
        P.nWork        = n;
        P.phi          = tPhi;
        P.phiWf        = tPhiWf;
        P.lam          = d_lambda;
        P.u            = const_cast<double*>( d_u );
        P.level        = nullptr;
        P.nTotalCell   = d_n_total;
        P.status       = d_status;
        P.iters        = iters;
        P.ctl          = ctl;
        P.workCounter  = &ctl->workCounter;
        P.activeList   = nullptr;
        P.fallbackList = nullptr;
        // the FP64 kernel in the launch shape that the allocating entry point uses
        int dev = 0, maxSmem = 0, sms = 0, occ = 0;
        CK( cudaGetDevice( &dev ) );
        CK( cudaDeviceGetAttribute( &maxSmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev ) );
        CK( cudaDeviceGetAttribute( &sms, cudaDevAttrMultiProcessorCount, dev ) );
        const ClosureShape cs = fp64_closure_shape( h, maxSmem );
        P.tablesInSmem        = cs.tablesInSmem;
        void* fn              = pick( h->cfg.closure, cs.group, 0 );
        allow_dynamic_smem( fn );
        CK( cudaOccupancyMaxActiveBlocksPerMultiprocessor( &occ, fn, cs.block, cs.smem ) );
        int mode     = 0;
        void* args[] = {&P, &mode};
        CK( cudaLaunchKernel( fn, dim3( std::max( 1, occ ) * sms ), dim3( cs.block ), args, cs.smem, st ) );
        return UQC_OK;
    } );
}
