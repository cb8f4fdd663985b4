// FP64 kernels of the IPM time step.
//
//   k_closure  persistent, work-stealing: one thread group (a warp for small
//              systems, a whole CTA for n = nS nT > 32) per cell. Runs the
//              damped Newton of Closure::SolveClosure (closure.cpp:133-193) with
//              the basis tables staged in shared memory, the Hessian kept in
//              packed upper-triangular form in shared memory and a right-looking
//              Cholesky; then, in step mode, the fused epilogue of
//              MomentSolver::Solve phases [C]-[F] (momentsolver.cpp:99-133):
//              nodal reconstruction uQ, refinement level, moment
//              re-projection and the CFL time step (grid-wide min).
//   k_update   kinetic flux at the quadrature nodes of every face, projected
//              onto the basis and applied as the explicit Euler update
//              (expliciteuler.cpp:17-74), plus the residual of
//              momentsolver.cpp:149-152 and the time/loop control, finished
//              by the last CTA.
//   k_init     initial moments and duals (momentsolver.cpp:463-563).
//   k_meanvar  mean and variance per cell (momentsolver.cpp:302-328).
#pragma once
#include <cuda_runtime.h>

#include "linalg.cuh"
#include "physics.cuh"
#include "uqc.h"

namespace uqc {

constexpr int MAXLEV = 16;

// Phase counters (slots 0-7 of g_phaseCycles, diagnostic builds; rank 0 of
// each thread group accumulates clock64 deltas): 0 newton, 1 initial
// gradient, 2 Hessian, 3 Cholesky, 4 back substitution, 5 trial gradients,
// 6 epilogue, 7 load; chord Newton of the mixed form: 21 solves with the
// held factor, 22 initial gradient, 23 whole cell, and counts 25 held-factor
// directions, 26 refreshed factors, 27 trial gradients.
#ifdef UQC_PHASE_TIMERS
#define PT_BEGIN( v ) long long v = clock64();
#define PT_END( v, id ) \
    if( g.r == 0 ) atomicAdd( &g_phaseCycles[id], (unsigned long long)( clock64() - v ) );
#define PT_COUNT( id ) \
    if( g.r == 0 ) atomicAdd( &g_phaseCycles[id], 1ull );
#else
#define PT_BEGIN( v )
#define PT_END( v, id )
#define PT_COUNT( id )
#endif

// Grid-wide loop state kept on the device so a step needs no host round trip.
struct Control {
    double t, tEnd, minResidual, residual, dt;
    int maxSteps;                  // 0: no limit on the number of steps
    unsigned long long dtBits;     // atomicMin of the positive dt as integer bits
    unsigned int workCounter;      // closure work stealing
    unsigned int workCounter2;     // ... of the FP64 pass over the mixed form's fallback cells
    unsigned int nFallback;        // length of that fallback list
    unsigned int doneBlocks;       // last-block detection in k_update
    int active;                    // the loop condition of momentsolver.cpp:79
    int steps;
    int failedCells;
    int activeCells;      // cells with Newton iterations in the running step
    int activeCellsLast;  // ... in the last finished step
    unsigned int nActive[2];      // lengths of the two active-cell lists (step parity)
    int listReady;                // k_update built the running step's lists: k_check runs only the check list
    unsigned int nCheck[2];       // lengths of the two check lists (cells whose level changes)
    unsigned long long dtBitsNext;    // min dt of the cells k_update finished for the next step
    unsigned long long newtonIters, lineSearchTrials;
    unsigned long long fallbackCells;    // mixed form: cells handed to the FP64 form
    // mixed form in rounds (chord.cuh): work-stealing counters (0-3 k_chord
    // rounds, 4-7 k_hess_tc, 8-11 k_invert), re-factor list lengths, and an
    // error flag (tensor-core wait timed out)
    unsigned int v2Work[16];
    unsigned int v2Count[4];
    int v2Error;
    // refinement retardation: the highest level the level rule may reach, and
    // how many of the residual thresholds the residual has fallen below
    int levelCap;
    int retIndex;
};

struct KParams {
    int nS, nT, nQ, ld;       // ld: row stride of the tables (odd, >= nT)
    int nLevels;
    int nTLevel[MAXLEV];
    // level rule: indicator (0 sum of |u(0, i)| over the level's own moments,
    // 1 the share of their energy S_l), bounds, retardation schedule
    int refIndicator;
    double refDown, refUp;
    int nRet;                 // residual thresholds of the retardation schedule (0: none)
    double retRes[8];
    int retLev[9];
    // linear closures (kinds 3-5): 0 stochastic Galerkin (factors 1 in filter),
    // 1 L2 filter (factors in filter), 2 Lasso filter
    int filterKind;
    const double* filter;        // nT factors
    const double* lassoParam;    // nT: prod_l index_l (index_l + 1)
    const double* lassoL1;       // nT: sum_k |phiWf(k, i)|
    int nCells, nFaces, dimXi;
    int nWork;                // cells a time step works on: the first nWork (a shard's owned cells), else nCells
    int cellBase;             // k_check without a list: cells cellBase .. cellBase + nWork - 1 (0 but for uqc_step_host's chunks)
    double eps;
    int maxIter, newtonMode;
    PhysParams phys;
    // tables
    const double* phi;       // nQ x ld
    const double* phiWf;     // nQ x ld
    const double* xi;        // nQ x dimXi
    const double* wt;        // nQ: w_k / 2^dimXi (phiWf = phi wt)
    const float* phiF;       // nQ x ld: phi rounded to FP32 (mixed form)
    bool tablesInSmem;
    // geometry
    const double *area, *dx, *center, *unitN, *scaledN;
    const int *nbr, *boundary;    // boundary: 0 interior, 1 Dirichlet, 2 no-slip wall, 3 shallow-water wall
    const double* bndNormal;      // unit normal of each wall cell's ghost face (null without walls)
    // state
    double *u, *lam, *uQ, *uOld0;
    double* uRe;              // step mode: the moments re-projected by the closure epilogue (k_update's input)
    unsigned* level;
    const unsigned* nTotalCell;  // closure-only calls: moments per cell (else from level)
    int *status, *iters;
    double* blockPartial;     // one per CTA of k_update (and launch, for a chunked update)
    int updChunk, updChunks;  // k_update over cells cellBase .. cellBase + nWork - 1 as launch updChunk of updChunks (else 0 of 1)
    int* activeList;          // step mode: cells that need Newton (filled by k_check / k_update), or null
    unsigned* activeCount;
    int listParity;           // step mode: two lists of nCells, the running step's is (ctl->steps & 1)
    int finishInUpdate;       // k_update tests the next step's convergence and fills the other lists
    int* checkList;           // step mode: converged cells whose level changes (k_check's epilogue), two lists
    unsigned* checkCount;
    unsigned char* finFlag;   // per cell: finished by k_update for the next step (no closure there)
    double* cellDt;           // per cell: the CFL step of its nodal states (written by the epilogue)
    unsigned* workCounter;    // work-stealing counter of k_closure (in ctl)
    float* factorStore;       // mixed form, step mode: each cell's last FP32 factor (or null)
    int* factorLevel;         // ... nTj it was formed for, -1 none
    int factorStride;         // floats per cell in factorStore
    int chordInverse;         // the store and the workspace hold the packed inverse X = U^-1 (else the factor)
    double chordTheta;        // re-factor after a held-factor step that reduced ||g|| by less than 1/chordTheta
    int* fallbackList;        // mixed form: cells handed to the FP64 form (non-PD FP32 factor, ...)
    unsigned* fallbackCount;
    // mixed form in rounds (chord.cuh)
    double* gStore;           // per cell: gradient at the accepted duals (compact) and its norm at [nS nT]; or null
    int gStride;              // doubles per cell in gStore
    int* v2Lists;             // re-factor lists, one of nCells per round
    int v2Rounds;             // re-factor rounds per step
    int* chordIters;          // per cell: Newton iterations of the step so far
    const unsigned short* qTiles;    // tensor-core Hessian: the BF16 high and low parts of Q in the operand layout
    Control* ctl;
};


// ------------------------------------------------------------------ workspace

// Shared-memory workspace of one cell (doubles), sizes for the finest level.
struct CellWs {
    double *lam, *lamN, *uh, *g, *gN, *d;   // n each
    double *LA, *LB, *uk;                   // nS nQ each
    double* du;                             // NP nQ
    double* H;                              // block-packed upper triangle + right-hand side (hess_doubles(n))
    double *D, *I;                          // Cholesky pivots and their inverses (n each)
    double* red;                            // reduction scratch (16) + broadcast (16)
    float* X;                               // mixed chord form: packed inverse of the factor (or null)
};

// Layout: [lam uh g LA D I red] then a region shared by the trial data
// [LB uk gN d lamN] and the nodal DU of the Hessian: whenever the Hessian is
// assembled, the trial buffers are dead (the next trial is formed after the
// solve), so DU aliases them. Then the block-packed Hessian. Every buffer
// starts on a 32-byte boundary; D and I are padded to whole tiles.
struct WsLayout {
    size_t lam, uh, g, LA, D, I, red, LB, uk, gN, d, lamN, du, H, X, total;    // offsets in doubles
};

// hElem: bytes of a Hessian element (8 FP64 form, 4 mixed form); xFloats:
// floats of the packed factor inverse (mixed chord form) or 0
__host__ __device__ inline WsLayout ws_layout( int nS, int nT, int nQ, int NP, int hElem, int xFloats = 0 ) {
    auto a4          = []( size_t x ) { return ( x + 3 ) & ~size_t( 3 ); };
    const size_t n   = size_t( nS ) * nT, n8 = size_t( hnb( int( n ) ) ) * 8, sq = size_t( nS ) * nQ;
    const size_t npp = size_t( ( NP + 1 ) & ~1 );
    WsLayout L;
    size_t o = 0;
    L.lam    = o, o += a4( n );
    L.uh     = o, o += a4( n );
    L.g      = o, o += a4( n );
    L.LA     = o, o += a4( sq );
    L.D      = o, o += a4( n8 );
    L.I      = o, o += a4( n8 );
    L.red    = o, o += 32;
    const size_t t = o;
    L.du           = t;
    L.LB           = t;
    L.uk           = L.LB + a4( sq );
    L.gN           = L.uk + a4( sq );
    L.d            = L.gN + a4( n );
    L.lamN         = L.d + a4( n );
    const size_t trialEnd = L.lamN + a4( n ), duEnd = t + a4( size_t( nQ ) * npp );
    o       = trialEnd > duEnd ? trialEnd : duEnd;
    L.H     = o;
    o += a4( ( hess_doubles( int( n ) ) * size_t( hElem ) + 7 ) / 8 );
    L.X = o;
    o += a4( ( size_t( xFloats ) * 4 + 7 ) / 8 );
    L.total = o;
    return L;
}

__host__ __device__ inline size_t cell_ws_doubles( int nS, int nT, int nQ, int NP, int hElem = 8, int xFloats = 0 ) {
    return ws_layout( nS, nT, nQ, NP, hElem, xFloats ).total;
}

__device__ inline CellWs carve( double* p, int nS, int nT, int nQ, int NP, int hElem, int xFloats = 0 ) {
    const WsLayout L = ws_layout( nS, nT, nQ, NP, hElem, xFloats );
    CellWs w;
    w.lam  = p + L.lam;
    w.uh   = p + L.uh;
    w.g    = p + L.g;
    w.LA   = p + L.LA;
    w.D    = p + L.D;
    w.I    = p + L.I;
    w.red  = p + L.red;
    w.LB   = p + L.LB;
    w.uk   = p + L.uk;
    w.gN   = p + L.gN;
    w.d    = p + L.d;
    w.lamN = p + L.lamN;
    w.du   = p + L.du;    // aliases the trial buffers while the Hessian is assembled
    w.H    = p + L.H;
    w.X    = xFloats ? reinterpret_cast<float*>( p + L.X ) : nullptr;
    return w;
}

// ------------------------------------------------------------------ building blocks

// sum_k u[k] tab(k, i) over nQ nodes (table row stride ld). Long sums (256
// nodes and more) use four partial sums (nodes k = 0, 1, 2, 3 mod 4): a
// quarter of the dependent FMA chain; short ones one chain, which issues
// fewer instructions (measured faster at 100 nodes, slower at 512).
__device__ __forceinline__ double node_dot( const double* u, const double* tab, int ld, int i, int nQ ) {
    if( nQ < 256 ) {
        double a = 0.0;
        for( int k = 0; k < nQ; ++k ) a = fma( u[k], tab[size_t( k ) * ld + i], a );
        return a;
    }
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const double* t = tab + i;
    int k           = 0;
    for( ; k + 3 < nQ; k += 4, t += 4 * size_t( ld ) ) {
        a0 = fma( u[k], t[0], a0 );
        a1 = fma( u[k + 1], t[ld], a1 );
        a2 = fma( u[k + 2], t[2 * ld], a2 );
        a3 = fma( u[k + 3], t[3 * ld], a3 );
    }
    for( ; k < nQ; ++k, t += ld ) a0 = fma( u[k], t[0], a0 );
    return ( a0 + a1 ) + ( a2 + a3 );
}

// Lambda_k[s] = sum_{i < nTj} lam[s nT + i] phi(k, i)   (closure.cpp:205-213).
// Warp groups: one node per thread, the NS states as independent chains
// sharing the row. CTA groups: one (state, node) per thread.
template <int NS, int GROUP>
__device__ __forceinline__ void eval_lambda_body( const Grp<GROUP>& g, const KParams& P, const double* phi, const double* lam, int nTj, double* L ) {
    if constexpr( GROUP >= 256 ) {
        for( int idx = g.r; idx < NS * P.nQ; idx += GROUP ) {
            const int s       = idx / P.nQ, k = idx - s * P.nQ;
            const double* row = phi + size_t( k ) * P.ld;
            const double* ls  = lam + s * P.nT;
            double a          = 0.0;
            for( int i = 0; i < nTj; ++i ) a = fma( ls[i], row[i], a );
            L[s * P.nQ + k] = a;
        }
        return;
    }
    for( int k = g.r; k < P.nQ; k += GROUP ) {
        const double* row = phi + size_t( k ) * P.ld;
        double a[NS];
#pragma unroll
        for( int s = 0; s < NS; ++s ) a[s] = 0.0;
        for( int i = 0; i < nTj; ++i ) {
            const double r = row[i];
#pragma unroll
            for( int s = 0; s < NS; ++s ) a[s] = fma( lam[s * P.nT + i], r, a[s] );
        }
#pragma unroll
        for( int s = 0; s < NS; ++s ) L[s * P.nQ + k] = a[s];
    }
}

// U at every node from Lambda (node-major loop, one node per thread).
template <int CL, int GROUP>
__device__ void eval_u( const Grp<GROUP>& g, const KParams& P, const double* L, double* uk, bool vecForm ) {
    constexpr int NS = Closure<CL>::NS;
    for( int k = g.r; k < P.nQ; k += GROUP ) {
        double Lk[NS], y[NS];
#pragma unroll
        for( int s = 0; s < NS; ++s ) Lk[s] = L[s * P.nQ + k];
        Closure<CL>::U( Lk, y, vecForm, P.phys );
#pragma unroll
        for( int s = 0; s < NS; ++s ) uk[s * P.nQ + k] = y[s];
    }
}

// Gradient (closure.cpp:234-253) at the duals whose Lambda is in L:
// gout[s nTj + i] = sum_k U_s(k) phiWf(k, i) - uh[s nT + i]; returns ||gout||_2.
// Vectors of the Newton system use the level's compact stride nTj.
// The sums m(s, i) = sum_k uk(s, k) phiWf(k, i) of the gradient, and
// sum_(s,i) (m - uh)^2 of this thread. Warp groups: a thread per basis
// function i, its NS sums as independent chains sharing each table value (one
// table load per NS FMAs, one chain of nQ per sum, in node order as
// node_dot's single chain; a single warp with nTj <= 16 also splits the nodes
// over lane groups); CTA groups: a thread per (s, i) with node_dot.
// gout (compact stride nTj) and ms (stride nT) may be null.
template <int NS, int GROUP>
__device__ __forceinline__ double gradient_sums( const Grp<GROUP>& g, const KParams& P, const double* phiWf, const double* uk, const double* uh,
                                                 int nTj, double* gout, double* ms ) {
    double sq = 0.0;
    if constexpr( GROUP == 32 ) {
        if( nTj <= 16 ) {
            // few basis functions: the warp splits the nodes as well, lane =
            // i + w part (w = nTj rounded up to a power of two), each part
            // summing the nodes k = part (mod 32 / w), then a butterfly over
            // the parts (a fixed order, so the sums are reproducible)
            int w = 1;
            while( w < nTj ) w <<= 1;
            const int i = g.r & ( w - 1 ), part = g.r / w, parts = 32 / w;
            double a[NS];
#pragma unroll
            for( int st = 0; st < NS; ++st ) a[st] = 0.0;
            if( i < nTj ) {
                const double* t = phiWf + size_t( part ) * P.ld + i;
                for( int k = part; k < P.nQ; k += parts, t += size_t( parts ) * P.ld ) {
                    const double wk = *t;
#pragma unroll
                    for( int st = 0; st < NS; ++st ) a[st] = fma( uk[st * P.nQ + k], wk, a[st] );
                }
            }
#pragma unroll
            for( int st = 0; st < NS; ++st )
                for( int o = w; o < 32; o <<= 1 ) a[st] += __shfl_xor_sync( 0xffffffffu, a[st], o );
            if( part == 0 && i < nTj ) {
#pragma unroll
                for( int st = 0; st < NS; ++st ) {
                    if( ms ) ms[st * P.nT + i] = a[st];
                    const double d = a[st] - uh[st * P.nT + i];
                    if( gout ) gout[st * nTj + i] = d;
                    sq += d * d;
                }
            }
            return sq;
        }
    }
    if constexpr( GROUP <= 64 ) {
        for( int i = g.r; i < nTj; i += GROUP ) {
            double a[NS];
#pragma unroll
            for( int s = 0; s < NS; ++s ) a[s] = 0.0;
            const double* t = phiWf + i;
            for( int k = 0; k < P.nQ; ++k, t += P.ld ) {
                const double w = *t;
#pragma unroll
                for( int s = 0; s < NS; ++s ) a[s] = fma( uk[s * P.nQ + k], w, a[s] );
            }
#pragma unroll
            for( int s = 0; s < NS; ++s ) {
                if( ms ) ms[s * P.nT + i] = a[s];
                const double d = a[s] - uh[s * P.nT + i];
                if( gout ) gout[s * nTj + i] = d;
                sq += d * d;
            }
        }
    }
    else {
        for( int idx = g.r; idx < NS * nTj; idx += GROUP ) {
            const int s    = idx / nTj, i = idx - s * nTj;
            const double m = node_dot( uk + s * P.nQ, phiWf, P.ld, i, P.nQ );
            if( ms ) ms[s * P.nT + i] = m;
            const double d = m - uh[s * P.nT + i];
            if( gout ) gout[idx] = d;
            sq += d * d;
        }
    }
    return sq;
}

template <int CL, int GROUP>
__device__ __forceinline__ double gradient_body( const Grp<GROUP>& g, const KParams& P, const double* phiWf, const double* L, const double* uh,
                                                 int nTj, double* uk, double* gout, double* red ) {
    constexpr int NS = Closure<CL>::NS;
    eval_u<CL, GROUP>( g, P, L, uk, true );
    g.sync();
    const double sq = gradient_sums<NS, GROUP>( g, P, phiWf, uk, uh, nTj, gout, nullptr );
    return sqrt( group_sum<GROUP>( g, sq, red ) );
}

// Out-of-line copies for the CTA-per-cell closure kernel: its Newton loop
// calls these at several sites, and one copy of each (instead of one per
// call site) measured faster there (512-node cells); the warp-group kernels
// inline them.
template <int NS, int GROUP>
__device__ __noinline__ void eval_lambda_ool( const Grp<GROUP>& g, const KParams& P, const double* phi, const double* lam, int nTj, double* L ) {
    eval_lambda_body<NS, GROUP>( g, P, phi, lam, nTj, L );
}
template <int CL, int GROUP>
__device__ __noinline__ double gradient_ool( const Grp<GROUP>& g, const KParams& P, const double* phiWf, const double* L, const double* uh, int nTj,
                                             double* uk, double* gout, double* red ) {
    return gradient_body<CL, GROUP>( g, P, phiWf, L, uh, nTj, uk, gout, red );
}
template <int NS, int GROUP>
__device__ __forceinline__ void eval_lambda( const Grp<GROUP>& g, const KParams& P, const double* phi, const double* lam, int nTj, double* L ) {
    if constexpr( GROUP >= 256 )
        eval_lambda_ool<NS, GROUP>( g, P, phi, lam, nTj, L );
    else
        eval_lambda_body<NS, GROUP>( g, P, phi, lam, nTj, L );
}
template <int CL, int GROUP>
__device__ __forceinline__ double gradient( const Grp<GROUP>& g, const KParams& P, const double* phiWf, const double* L, const double* uh, int nTj,
                                            double* uk, double* gout, double* red ) {
    if constexpr( GROUP >= 256 )
        return gradient_ool<CL, GROUP>( g, P, phiWf, L, uh, nTj, uk, gout, red );
    else
        return gradient_body<CL, GROUP>( g, P, phiWf, L, uh, nTj, uk, gout, red );
}

// Newton direction d = H(lambda)^-1 g (closure.cpp:145-150 / 162-168): Hessian
// at the duals whose Lambda is in LA, then posv. Returns 0 or UQC_CELL_NOT_PD.
// HT = double: the FP64 form. HT = float (mixed form): Hessian, factor and
// triangular solves in FP32 from phiH = phi in FP32, the gradient g and the
// direction d in FP64; the FP64 gradient test of the caller decides
// convergence, so an FP32 direction costs at most extra iterations.
template <int CL, int GROUP, class HT>
__device__ int newton_direction( const Grp<GROUP>& g, const KParams& P, const double* phi, const HT* phiH, CellWs& w, int nTj,
                                 const double* LA ) {
    constexpr int NS = Closure<CL>::NS, NP = Closure<CL>::NP;
    const int n = NS * nTj, rhs = hrhs( hnb( n ) );
    HT* H = reinterpret_cast<HT*>( w.H );
    HT* D = reinterpret_cast<HT*>( w.D );
    HT* I = reinterpret_cast<HT*>( w.I );
    PT_BEGIN( t0 );
    hessian_sym<NS, NP, GROUP, HT>( g, P.nQ, P.ld, phiH, P.wt, LA, nTj, reinterpret_cast<HT*>( w.du ), H,
                                    [&]( const double* L, double* y ) { Closure<CL>::DU( L, y, P.phys ); } );
    for( int r = g.r; r < n; r += GROUP ) H[rhs + r] = HT( w.g[r] );
    g.sync();
    PT_END( t0, 2 );
    PT_BEGIN( t1 );
    if( cholesky_la<GROUP, HT>( g, H, n, D, I, reinterpret_cast<int*>( w.red + 24 ) ) ) return UQC_CELL_NOT_PD;
    PT_END( t1, 3 );
    PT_BEGIN( t2 );
    back_solve_warp<GROUP, HT>( g, H, n, I, w.d );
    PT_END( t2, 4 );
    return 0;
}

// lamOut[s nT + i] = lamIn[s nT + i] + c d[s nTj + i], i < nTj (closure.cpp:273-279)
template <int GROUP> __device__ void add_step( const Grp<GROUP>& g, const KParams& P, int nTj, const double* lamIn, double c, const double* d, double* lamOut ) {
    for( int idx = g.r; idx < P.nS * nTj; idx += GROUP ) {
        int s = idx / nTj, i = idx - s * nTj;
        lamOut[s * P.nT + i] = lamIn[s * P.nT + i] + c * d[idx];
    }
}

// Damped Newton on one cell in shared memory. On return w.lam holds the duals
// and w.LA the Lambda of w.lam at all nodes (laValid). Returns a uqc_cell_code.
template <int CL, int GROUP, class HT>
__device__ int newton_cell( const Grp<GROUP>& g, const KParams& P, const double* phi, const double* phiWf, const HT* phiH, CellWs& w, int nTj,
                            int& iters, int& lsTrials ) {
    const int n      = P.nS * nTj;
    const double eps = P.eps;
    const bool guard = P.newtonMode != 0;
    iters            = 0;
    lsTrials         = 0;
    double* LA = w.LA;
    double* LB = w.LB;
    // lam <- lamN and LA <- LB by copy: LA must stay outside the region that
    // the Hessian's DU buffer aliases
    auto accept = [&]() {
        for( int idx = g.r; idx < P.nS * P.nT; idx += GROUP ) w.lam[idx] = w.lamN[idx];
        for( int idx = g.r; idx < Closure<CL>::NS * P.nQ; idx += GROUP ) LA[idx] = LB[idx];
    };
    int rc = UQC_CELL_MAX_ITER;
    eval_lambda<Closure<CL>::NS, GROUP>( g, P, phi, w.lam, nTj, LA );
    g.sync();
    if( P.newtonMode == 2 ) {
        // Closure::SolveClosureSafe (closure.cpp:297-339)
        for( int l = 0; l < P.maxIter; ++l ) {
            double stepSize = 1.0;
            double gn       = gradient<CL, GROUP>( g, P, phiWf, LA, w.uh, nTj, w.uk, w.g, w.red );
            if( newton_direction<CL, GROUP, HT>( g, P, phi, phiH, w, nTj, LA ) ) {
                rc = UQC_CELL_NOT_PD;
                goto out;
            }
            ++iters;
            for( int idx = g.r; idx < P.nS * P.nT; idx += GROUP ) w.lamN[idx] = w.lam[idx];
            add_step<GROUP>( g, P, nTj, w.lam, -stepSize, w.d, w.lamN );
            g.sync();
            eval_lambda<Closure<CL>::NS, GROUP>( g, P, phi, w.lamN, nTj, LB );
            g.sync();
            double gnN = gradient<CL, GROUP>( g, P, phiWf, LB, w.uh, nTj, w.uk, w.gN, w.red );
            int refine = 0;
            while( gn < gnN || !isfinite( gnN ) ) {
                stepSize *= 0.5;
                ++lsTrials;
                add_step<GROUP>( g, P, nTj, w.lam, -stepSize, w.d, w.lamN );
                g.sync();
                eval_lambda<Closure<CL>::NS, GROUP>( g, P, phi, w.lamN, nTj, LB );
                g.sync();
                gnN = gradient<CL, GROUP>( g, P, phiWf, LB, w.uh, nTj, w.uk, w.gN, w.red );
                if( gnN < eps ) {
                    accept();
                    rc = UQC_CELL_CONVERGED;
                    goto out;
                }
                if( ++refine > 1000 ) {
                    rc = UQC_CELL_LINE_SEARCH;
                    goto out;
                }
            }
            accept();
            g.sync();
            if( gnN < eps ) {
                rc = UQC_CELL_CONVERGED;
                goto out;
            }
        }
        goto out;
    }
    {
        // Closure::SolveClosure (closure.cpp:133-193); guard = the finiteness test of :318
        PT_BEGIN( tg );
        double gn = gradient<CL, GROUP>( g, P, phiWf, LA, w.uh, nTj, w.uk, w.g, w.red );
        PT_END( tg, 1 );
        if( gn < eps ) {
            rc = UQC_CELL_CONVERGED;
            goto out;
        }
        double gnN = 0.0;
        for( int l = 0; l < P.maxIter; ++l ) {
            double stepSize = 1.0;
            if( l != 0 ) {
                // the gradient at lam is the accepted trial gradient (same duals, same arithmetic)
                for( int idx = g.r; idx < n; idx += GROUP ) w.g[idx] = w.gN[idx];
                gn = gnN;
            }
            if( newton_direction<CL, GROUP, HT>( g, P, phi, phiH, w, nTj, LA ) ) {
                rc = UQC_CELL_NOT_PD;
                goto out;
            }
            ++iters;
            if( P.maxIter == 1 ) {
                // One-Shot IPM: lam -= alpha H^-1 g, no line search (closure.cpp:151-154)
                add_step<GROUP>( g, P, nTj, w.lam, -1.0, w.d, w.lam );
                g.sync();
                eval_lambda<Closure<CL>::NS, GROUP>( g, P, phi, w.lam, nTj, LA );
                g.sync();
                eval_u<CL, GROUP>( g, P, LA, w.uk, true );    // keep uk = U(lam) for the epilogue
                rc = UQC_CELL_CONVERGED;
                goto out;
            }
            PT_BEGIN( tt );
            for( int idx = g.r; idx < P.nS * P.nT; idx += GROUP ) w.lamN[idx] = w.lam[idx];
            add_step<GROUP>( g, P, nTj, w.lam, -stepSize, w.d, w.lamN );
            g.sync();
            eval_lambda<Closure<CL>::NS, GROUP>( g, P, phi, w.lamN, nTj, LB );
            g.sync();
            gnN        = gradient<CL, GROUP>( g, P, phiWf, LB, w.uh, nTj, w.uk, w.gN, w.red );
            PT_END( tt, 5 );
            int refine = 0;
            while( gn < gnN || ( guard && !isfinite( gnN ) ) ) {
                stepSize *= 0.5;
                ++lsTrials;
                add_step<GROUP>( g, P, nTj, w.lam, -stepSize, w.d, w.lamN );
                g.sync();
                eval_lambda<Closure<CL>::NS, GROUP>( g, P, phi, w.lamN, nTj, LB );
                g.sync();
                gnN = gradient<CL, GROUP>( g, P, phiWf, LB, w.uh, nTj, w.uk, w.gN, w.red );
                if( gnN < eps ) {
                    accept();
                    rc = UQC_CELL_CONVERGED;
                    goto out;
                }
                if( ++refine > 1000 ) {
                    rc = UQC_CELL_LINE_SEARCH;
                    goto out;
                }
            }
            accept();
            g.sync();
            if( gnN < eps ) {
                rc = UQC_CELL_CONVERGED;
                goto out;
            }
        }
    }
out:
    g.sync();
    w.LA = LA;
    w.LB = LB;
    return rc;
}

// Closure of a cell with at most TINY_N duals (n = NS nTj) and at most 64
// nodes on one warp, all in registers: lane l holds nodes l and l + 32, sums
// over nodes are butterfly reductions (every lane ends with the full sums),
// and every lane factors and solves the n x n system itself, so an iteration
// has no shared-memory round trip and no warp barrier. The iteration is
// newton_cell's SolveClosure path (closure.cpp:133-193: Newton direction by
// posv, step halving while the gradient norm grows, convergence on ||g|| <
// eps), with the finiteness guard of newtonMode 1 and the One-Shot step of
// maxIter == 1; SolveClosureSafe (newtonMode 2) runs newton_cell. On return
// w.lam holds the duals and, for a converged cell, w.uk holds U at them
// (state-major), as newton_cell leaves them.
constexpr int TINY_N = 6;
template <int NS> __device__ __forceinline__ constexpr int du_index( int m, int l ) {
    // DU's packed order of the state pair (m, l), m <= l: rows m' < m first
    int p = 0;
    for( int a = 0; a < m; ++a ) p += NS - a;
    return p + ( l - m );
}
template <int CL>
__device__ int newton_cell_tiny( const KParams& P, const double* phi, const double* phiWf, CellWs& w, int nTj, int& iters, int& lsTrials ) {
    constexpr int NS = Closure<CL>::NS, NP = Closure<CL>::NP, TN = TINY_N, TT = TINY_N / NS, TH = TINY_N * ( TINY_N + 1 ) / 2;
    const int lane = threadIdx.x & 31;
    const int n    = NS * nTj;
    const bool guard = P.newtonMode != 0;
    iters    = 0;
    lsTrials = 0;
    // the lane's nodes: basis values and weights (phiWf(k, i) = phi(k, i) wt_k
    // exactly: wt_k = w_k / 2^dimXi)
    double ph[2][TT], wk[2];
    bool valid[2];
    (void)phiWf;
#pragma unroll
    for( int q = 0; q < 2; ++q ) {
        const int k = lane + 32 * q;
        valid[q]    = k < P.nQ;
        wk[q]       = valid[q] ? P.wt[k] : 0.0;
#pragma unroll
        for( int i = 0; i < TT; ++i ) ph[q][i] = valid[q] && i < nTj ? phi[size_t( k ) * P.ld + i] : 0.0;
    }
    double lam[TN], uh[TN], g[TN], d[TN], lamN[TN], gN[TN];
#pragma unroll
    for( int r = 0; r < TN; ++r ) {
        const int s = r / TT, i = r - s * TT;    // compact index r = s TT + i (TT columns per state)
        const bool on = i < nTj;
        lam[r] = on ? w.lam[s * P.nT + i] : 0.0;
        uh[r]  = on ? w.uh[s * P.nT + i] : 0.0;
        g[r] = d[r] = lamN[r] = gN[r] = 0.0;
    }
    // Lambda and U at the lane's nodes for the duals x; gradient into gout; returns ||g||
    double LamA[2][NS], UA[2][NS];    // at the accepted duals
    double LamT[2][NS], UT[2][NS];    // at the last trial
    auto gradient_at = [&]( const double( &x )[TN], double( &Lam )[2][NS], double( &U )[2][NS], double( &gout )[TN] ) {
        double acc[TN];
#pragma unroll
        for( int r = 0; r < TN; ++r ) acc[r] = 0.0;
#pragma unroll
        for( int q = 0; q < 2; ++q ) {
#pragma unroll
            for( int st = 0; st < NS; ++st ) {
                double a = 0.0;
#pragma unroll
                for( int i = 0; i < TT; ++i )
                    if( i < nTj ) a = fma( x[st * TT + i], ph[q][i], a );
                Lam[q][st] = a;
            }
            if( valid[q] ) Closure<CL>::U( Lam[q], U[q], true, P.phys );
            else {
#pragma unroll
                for( int st = 0; st < NS; ++st ) U[q][st] = 0.0;
            }
#pragma unroll
            for( int r = 0; r < TN; ++r ) {
                const int st = r / TT, i = r - st * TT;
                acc[r] = fma( U[q][st], ph[q][i] * wk[q], acc[r] );
            }
        }
        double sq = 0.0;
#pragma unroll
        for( int r = 0; r < TN; ++r ) {
            double v = acc[r];
#pragma unroll
            for( int o = 16; o > 0; o >>= 1 ) v += __shfl_xor_sync( 0xffffffffu, v, o );
            const int i = r - ( r / TT ) * TT;
            gout[r]     = i < nTj ? v - uh[r] : 0.0;
            sq          = fma( gout[r], gout[r], sq );
        }
        return sqrt( sq );
    };
    // Newton direction d = H^-1 g at the accepted duals (LamA); false: not positive definite
    auto direction = [&]() {
        double h[TH];
#pragma unroll
        for( int e = 0; e < TH; ++e ) h[e] = 0.0;
#pragma unroll
        for( int q = 0; q < 2; ++q ) {
            double y[NP];
            if( valid[q] ) Closure<CL>::DU( LamA[q], y, P.phys );
            else {
#pragma unroll
                for( int e = 0; e < NP; ++e ) y[e] = 0.0;
            }
#pragma unroll
            for( int a = 0; a < TN; ++a ) {
                const int sa = a / TT, ia = a - sa * TT;
#pragma unroll
                for( int b = 0; b <= a; ++b ) {
                    const int sb = b / TT, ib = b - sb * TT;
                    const double du = y[du_index<NS>( sb < sa ? sb : sa, sb < sa ? sa : sb )];
                    h[a * ( a + 1 ) / 2 + b] = fma( ph[q][ia] * ph[q][ib] * wk[q], du, h[a * ( a + 1 ) / 2 + b] );
                }
            }
        }
#pragma unroll
        for( int e = 0; e < TH; ++e ) {
#pragma unroll
            for( int o = 16; o > 0; o >>= 1 ) h[e] += __shfl_xor_sync( 0xffffffffu, h[e], o );
        }
        // Cholesky H = L L^T in place (rows and columns of the unused states'
        // padding are skipped), then L y = g, L^T d = y
        bool pd = true;
#pragma unroll
        for( int j = 0; j < TN; ++j ) {
            if( j - ( j / TT ) * TT >= nTj ) continue;
            double dj = h[j * ( j + 1 ) / 2 + j];
#pragma unroll
            for( int k = 0; k < j; ++k )
                if( k - ( k / TT ) * TT < nTj ) dj -= h[j * ( j + 1 ) / 2 + k] * h[j * ( j + 1 ) / 2 + k];
            pd = pd && dj > 0.0;
            const double ljj = sqrt( dj );
            h[j * ( j + 1 ) / 2 + j] = ljj;
#pragma unroll
            for( int i = j + 1; i < TN; ++i ) {
                if( i - ( i / TT ) * TT >= nTj ) continue;
                double v = h[i * ( i + 1 ) / 2 + j];
#pragma unroll
                for( int k = 0; k < j; ++k )
                    if( k - ( k / TT ) * TT < nTj ) v -= h[i * ( i + 1 ) / 2 + k] * h[j * ( j + 1 ) / 2 + k];
                h[i * ( i + 1 ) / 2 + j] = v / ljj;
            }
        }
        double y[TN];
#pragma unroll
        for( int i = 0; i < TN; ++i ) {
            double v = g[i];
#pragma unroll
            for( int k = 0; k < i; ++k )
                if( k - ( k / TT ) * TT < nTj ) v -= h[i * ( i + 1 ) / 2 + k] * y[k];
            y[i] = i - ( i / TT ) * TT < nTj ? v / h[i * ( i + 1 ) / 2 + i] : 0.0;
        }
#pragma unroll
        for( int i = TN - 1; i >= 0; --i ) {
            double v = y[i];
#pragma unroll
            for( int k = i + 1; k < TN; ++k )
                if( k - ( k / TT ) * TT < nTj ) v -= h[k * ( k + 1 ) / 2 + i] * d[k];
            d[i] = i - ( i / TT ) * TT < nTj ? v / h[i * ( i + 1 ) / 2 + i] : 0.0;
        }
        return pd;
    };
    auto trial = [&]( double step ) {
#pragma unroll
        for( int r = 0; r < TN; ++r ) lamN[r] = lam[r] + -step * d[r];
        return gradient_at( lamN, LamT, UT, gN );
    };
    auto accept = [&]() {
#pragma unroll
        for( int r = 0; r < TN; ++r ) {
            lam[r] = lamN[r];
            g[r]   = gN[r];
        }
#pragma unroll
        for( int q = 0; q < 2; ++q )
#pragma unroll
            for( int st = 0; st < NS; ++st ) {
                LamA[q][st] = LamT[q][st];
                UA[q][st]   = UT[q][st];
            }
    };
    int rc    = UQC_CELL_MAX_ITER;
    double gn = gradient_at( lam, LamA, UA, g );
    double gnN = 0.0;
    if( gn < P.eps ) {
        rc = UQC_CELL_CONVERGED;
        goto out;
    }
    for( int l = 0; l < P.maxIter; ++l ) {
        if( l != 0 ) gn = gnN;
        if( !direction() ) {
            rc = UQC_CELL_NOT_PD;
            goto out;
        }
        ++iters;
        if( P.maxIter == 1 ) {
            // One-Shot IPM: lam -= H^-1 g, no line search (closure.cpp:151-154)
            trial( 1.0 );
            accept();
            rc = UQC_CELL_CONVERGED;
            goto out;
        }
        double stepSize = 1.0;
        gnN             = trial( stepSize );
        int refine      = 0;
        while( gn < gnN || ( guard && !isfinite( gnN ) ) ) {
            stepSize *= 0.5;
            ++lsTrials;
            gnN = trial( stepSize );
            if( gnN < P.eps ) {
                accept();
                rc = UQC_CELL_CONVERGED;
                goto out;
            }
            if( ++refine > 1000 ) {
                rc = UQC_CELL_LINE_SEARCH;
                goto out;
            }
        }
        accept();
        if( gnN < P.eps ) {
            rc = UQC_CELL_CONVERGED;
            goto out;
        }
    }
out:
#pragma unroll
    for( int r = 0; r < TN; ++r ) {
        const int st = r / TT, i = r - st * TT;
        if( i < nTj && lane == r ) w.lam[st * P.nT + i] = lam[r];
    }
    if( rc == UQC_CELL_CONVERGED ) {
#pragma unroll
        for( int q = 0; q < 2; ++q )
            if( valid[q] )
#pragma unroll
                for( int st = 0; st < NS; ++st ) w.uk[st * P.nQ + lane + 32 * q] = UA[q][st];
    }
    __syncwarp();
    return rc;
}

// Mixed form, step mode: inexact (chord) Newton with a reused FP32 factor.
// Same loop as newton_cell's SolveClosure path (FP64 gradient, line search,
// convergence test), but the direction H0^-1 g comes from the factor the cell
// holds (loaded from the store, formed at an earlier iteration or time step)
// while it contracts well; the Hessian is re-assembled and factored when there
// is no factor, when a step with the held factor does not reduce ||g|| at all
// (the direction is then recomputed, not line-searched), and after a step
// that reduced ||g|| by less than the factor 1/P.chordTheta. `fresh` reports whether w.H
// ends with a factor formed in this solve (to store).
template <int CL, int GROUP>
__device__ int newton_cell_chord( const Grp<GROUP>& g, const KParams& P, const double* phi, const double* phiWf, const float* phiH, CellWs& w,
                                  int nTj, bool have, int& iters, int& lsTrials, bool& fresh ) {
    constexpr int NS = Closure<CL>::NS;
    const int n      = NS * nTj;
    const double eps = P.eps;
    const bool guard = P.newtonMode != 0;
    iters            = 0;
    lsTrials         = 0;
    fresh            = false;
    double* LA       = w.LA;
    double* LB       = w.LB;
    float* H         = reinterpret_cast<float*>( w.H );
    float* I         = reinterpret_cast<float*>( w.I );
    auto accept      = [&]() {
        for( int idx = g.r; idx < P.nS * P.nT; idx += GROUP ) w.lam[idx] = w.lamN[idx];
        for( int idx = g.r; idx < NS * P.nQ; idx += GROUP ) LA[idx] = LB[idx];
    };
    auto trial = [&]( double step ) {
        PT_BEGIN( tt );
        PT_COUNT( 27 );
        add_step<GROUP>( g, P, nTj, w.lam, -step, w.d, w.lamN );
        g.sync();
        eval_lambda<NS, GROUP>( g, P, phi, w.lamN, nTj, LB );
        g.sync();
        const double r = gradient<CL, GROUP>( g, P, phiWf, LB, w.uh, nTj, w.uk, w.gN, w.red );
        PT_END( tt, 5 );
        return r;
    };
    int rc = UQC_CELL_MAX_ITER;
    PT_BEGIN( tc );
    PT_BEGIN( t0 );
    eval_lambda<NS, GROUP>( g, P, phi, w.lam, nTj, LA );
    g.sync();
    double gn = gradient<CL, GROUP>( g, P, phiWf, LA, w.uh, nTj, w.uk, w.g, w.red );
    PT_END( t0, 22 );
    if( gn < eps ) return UQC_CELL_CONVERGED;
    bool refresh = !have;
    double gnN   = 0.0;
    for( int l = 0; l < P.maxIter; ++l ) {
        if( l != 0 ) {
            for( int idx = g.r; idx < n; idx += GROUP ) w.g[idx] = w.gN[idx];
            gn = gnN;
        }
        for( int idx = g.r; idx < P.nS * P.nT; idx += GROUP ) w.lamN[idx] = w.lam[idx];
        bool chord = false;
        for( int attempt = 0; attempt < 2; ++attempt ) {
            if( refresh ) {
                PT_COUNT( 26 );
                if( newton_direction<CL, GROUP, float>( g, P, phi, phiH, w, nTj, LA ) ) return UQC_CELL_NOT_PD;
                if( P.chordInverse ) tri_inverse_packed<GROUP, float>( g, H, I, n, w.X );
                fresh   = true;
                refresh = false;
                chord   = false;
            }
            else {
                PT_BEGIN( ts );
                PT_COUNT( 25 );
                g.sync();    // w.g complete (copied by the whole group)
                if( P.chordInverse )
                    chord_direction_packed<GROUP, float>( g, w.X, n, w.g, reinterpret_cast<float*>( w.D ), I, w.d );
                else {
                    forward_solve_warp<GROUP, float>( g, H, n, I, w.g );
                    back_solve_warp<GROUP, float>( g, H, n, I, w.d );
                }
                PT_END( ts, 21 );
                chord = true;
            }
            ++iters;
            gnN = trial( 1.0 );
            if( chord && !( gnN < gn ) ) {
                refresh = true;    // no decrease with the held factor: form the true Newton direction
                continue;
            }
            break;
        }
        double stepSize = 1.0;
        int refine      = 0;
        while( gn < gnN || ( guard && !isfinite( gnN ) ) ) {
            stepSize *= 0.5;
            ++lsTrials;
            gnN = trial( stepSize );
            if( gnN < eps ) {
                accept();
                rc = UQC_CELL_CONVERGED;
                goto out;
            }
            if( ++refine > 1000 ) {
                rc = UQC_CELL_LINE_SEARCH;
                goto out;
            }
        }
        accept();
        g.sync();
        if( gnN < eps ) {
            rc = UQC_CELL_CONVERGED;
            goto out;
        }
        if( chord && gnN > P.chordTheta * gn ) refresh = true;
    }
out:
    g.sync();
    PT_END( tc, 23 );
    w.LA = LA;
    w.LB = LB;
    return rc;
}

// ------------------------------------------------------------------ kernels

// Duals of a linear closure from the moments (state-major, finest stride nT):
// lambda(s, i) = f_i u(s, i) for stochastic Galerkin (f = 1) and the L2
// filter (l2filter.cpp:29-35); the Lasso filter (lassofilter.cpp:36-47) scales by
// 1 - strength_s p_i l1_i / |u(s, i)|, cut to 0 below 0 or for |u(s, i)| <
// 1e-7, strength_s = |u(s, nT-1)| / (p_{nT-1} l1_{nT-1}), in the reference's
// operation order. Every moment of the finest level, as the reference loops
// over GetNTotal() whatever the cell's level.
template <int NS, int GROUP> __device__ void linear_duals( const Grp<GROUP>& g, const KParams& P, const double* uh, double* lam ) {
    const int nT = P.nT;
    for( int idx = g.r; idx < NS * nT; idx += GROUP ) {
        const int s = idx / nT, i = idx - s * nT;
        if( P.filterKind == 2 ) {
            const int nMax         = nT - 1;
            const double strength  = fabs( uh[s * nT + nMax] ) / ( P.lassoParam[nMax] * P.lassoL1[nMax] );
            double sc              = 1.0 - strength * P.lassoParam[i] * P.lassoL1[i] / fabs( uh[idx] );
            if( sc < 0 || fabs( uh[idx] ) < 1e-7 ) sc = 0.0;
            lam[idx] = sc * uh[idx];
        }
        else
            lam[idx] = P.filter[i] * uh[idx];
    }
}

// Refinement indicator of a cell at level lev (nTj moments) from its first
// state's moments at(i): the sum of |u(0, i)| over the moments the level adds
// (the last two in one uncertain dimension) of MomentSolver::ComputeRefIndicator
// (momentsolver.cpp:271-289), or S_l = <(u_l - u_{l-1})^2> / <u_l^2> of
// Paper1/adaptivity.tex:12-14, which for the orthonormal basis tables is the
// sum of the added moments' squares over the sum of all squares (level 0
// measures against the mean alone, as the code's indicator does).
template <class AT> __device__ __forceinline__ double level_indicator( const KParams& P, AT at, int lev, int nTj ) {
    double ind = 0.0;
    if( P.refIndicator == 1 ) {
        const int prev = lev == 0 ? 1 : P.nTLevel[lev - 1];
        double num = 0.0, den = 0.0;
        for( int i = 0; i < nTj; ++i ) {
            const double v = at( i );
            den += v * v;
            if( i >= prev ) num += v * v;
        }
        return den > 0.0 ? num / den : 0.0;
    }
    if( P.dimXi == 1 )
        ind = fabs( at( nTj - 1 ) ) + fabs( at( nTj - 2 ) );
    else {
        const int prev = lev == 0 ? 1 : P.nTLevel[lev - 1];
        for( int i = prev; i < nTj; ++i ) ind += fabs( at( i ) );
    }
    return ind;
}

// The level rule of momentsolver.cpp:104-112 with configurable bounds, capped
// by the retardation schedule (a level above the cap drops to it).
__device__ __forceinline__ int level_rule( const KParams& P, double ind, int lev ) {
    const int cap = min( P.nLevels - 1, P.ctl->levelCap );
    if( lev > cap ) return cap;
    if( ind > P.refUp && lev < cap ) return lev + 1;
    if( ind < P.refDown && lev > 0 ) return lev - 1;
    return lev;
}

// Epilogue of a cell whose closure is done, phases [C]-[F] of
// MomentSolver::Solve (momentsolver.cpp:99-133): uk holds U(Lambda(lam)) at
// the nodes, uh the moments before re-projection. Writes uQ, the new
// refinement level (indicator of :271-289, thresholds of :104-112) and the
// re-projected moments, and returns the cell's CFL time step.
// NM: uk node-major (uk[k NS + s]) instead of state-major (uk[s nQ + k]).
template <int CL, int GROUP, bool NM = false>
__device__ double cell_epilogue( const Grp<GROUP>& g, const KParams& P, const double* phiWf, const double* uh, const double* uk, int cell,
                                 int lev, int nTj, double* red,
                                 const double* ugs = nullptr ) {
    constexpr int NS = Closure<CL>::NS;
    auto ukAt = [&]( int s, int k ) { return NM ? uk[k * NS + s] : uk[s * P.nQ + k]; };
    const size_t ldc = size_t( NS ) * P.nT;
    int newLev       = lev;
    if( P.nLevels > 1 ) newLev = level_rule( P, level_indicator( P, [&]( int i ) { return uh[i]; }, lev, nTj ), lev );
    const int nTn = P.nTLevel[newLev];
    if( g.r == 0 ) {
        P.uOld0[cell] = uh[0];
        P.level[cell] = unsigned( newLev );
    }
    double* uq = P.uQ + size_t( cell ) * NS * P.nQ;
    for( int idx = g.r; idx < NS * P.nQ; idx += GROUP ) {
        const int s = idx / P.nQ, k = idx - s * P.nQ;
        uq[idx]     = ukAt( s, k );
    }
    // [E] u(s, i) = sum_k uQ(s, k) phiWf(k, i) for i < nT(new level), 0 beyond
    for( int idx = g.r; idx < int( ldc ); idx += GROUP ) {
        int s = idx / P.nT, i = idx - s * P.nT;
        // ugs: the same sums kept from the gradient test (i < nTj), when the caller has them
        double m = 0.0;
        if( i < nTn ) {
            if( ugs && i < nTj )
                m = ugs[idx];
            else if( !NM )
                m = node_dot( uk + s * P.nQ, phiWf, P.ld, i, P.nQ );
            else
                for( int k = 0; k < P.nQ; ++k ) m = fma( uk[k * NS + s], phiWf[size_t( k ) * P.ld + i], m );
        }
        P.uRe[cell * ldc + idx] = m;
        if( i >= nTn ) P.u[cell * ldc + idx] = 0.0;    // the update writes u below the level only
    }
    // [F] the cell's time step (min over its nodes)
    double dloc = 1e300;
    for( int k = g.r; k < P.nQ; k += GROUP ) {
        double uqk[NS];
#pragma unroll
        for( int s = 0; s < NS; ++s ) uqk[s] = ukAt( s, k );
        double d = Problem<CL>::dt( uqk, P.dx[cell], P.phys );
        dloc     = d < dloc ? d : dloc;
    }
    dloc = group_min<GROUP>( g, dloc, red );
    if( g.r == 0 && P.cellDt ) P.cellDt[cell] = dloc;
    return dloc;
}

// The active-cell list of the running step (step mode: one of two, by step
// parity; k_update fills the other one for the next step).
__device__ __forceinline__ void step_list( const KParams& P, int ahead, int*& list, unsigned*& count ) {
    list  = P.activeList;
    count = P.activeCount;
    if( P.listParity && list ) {
        const int par = ( P.ctl->steps + ahead ) & 1;
        list += size_t( par ) * P.nCells;
        count += par;
    }
}

__device__ __forceinline__ void atomic_min_pos_double( unsigned long long* addr, double v ) {
    if( v >= 0.0 ) atomicMin( addr, (unsigned long long)__double_as_longlong( v ) );
}

// Threads per CTA of k_closure: up to 8 warp groups or 4 two-warp groups
// (256 threads: up to 255 registers per thread).
template <int GROUP> constexpr int closure_max_block() { return GROUP <= 64 ? 256 : GROUP; }

// Persistent closure kernel. mode 0: closure only; mode 1: closure + fused
// epilogue of a time step. Tables are staged in shared memory when they fit.
// HT = float is the mixed form: cells whose FP32 Newton does not converge
// (FP32 factor not positive definite, line search or iteration limit) are
// appended to P.fallbackList, with their last accepted duals written back,
// for a pass of the FP64 form; they get no status or epilogue here.
// TINY (GROUP 32, HT double): every cell's Newton runs in registers
// (newton_cell_tiny; n <= TINY_N duals, <= 64 nodes, not SolveClosureSafe).
template <int CL, int GROUP, class HT, bool TINY = false>
__global__ void __launch_bounds__( closure_max_block<GROUP>(), 1 ) k_closure( KParams P, int mode ) {
    constexpr int NS = Closure<CL>::NS, NP = Closure<CL>::NP;
    constexpr bool MIXED = sizeof( HT ) == 4;
    extern __shared__ __align__( 16 ) double smem[];
    if( mode == 1 && !P.ctl->active ) return;
    const int gid = threadIdx.x / GROUP;
    Grp<GROUP> g{int( threadIdx.x % GROUP ), 1 + gid};
    const double *phi = P.phi, *phiWf = P.phiWf;
    const HT* phiH;
    if constexpr( MIXED )
        phiH = P.phiF;
    else
        phiH = P.phi;
    double* base = smem;
    if( P.tablesInSmem ) {
        const size_t tn = size_t( P.nQ ) * P.ld + 4;
        for( size_t i = threadIdx.x; i < tn; i += blockDim.x ) {
            base[i]      = i < size_t( P.nQ ) * P.ld ? P.phi[i] : 0.0;
            base[tn + i] = i < size_t( P.nQ ) * P.ld ? P.phiWf[i] : 0.0;
        }
        phi   = base;
        phiWf = base + tn;
        base += 2 * tn;
        if constexpr( MIXED ) {
            float* f = reinterpret_cast<float*>( base );
            for( size_t i = threadIdx.x; i < tn; i += blockDim.x ) f[i] = i < size_t( P.nQ ) * P.ld ? P.phiF[i] : 0.0f;
            phiH = f;
            base += ( tn + 1 ) / 2;
        }
        else {
            phiH = phi;
        }
        __syncthreads();
    }
    const int xf = MIXED && P.chordInverse ? xpacked( NS * P.nT ) : 0;
    CellWs w     = carve( base + gid * cell_ws_doubles( NS, P.nT, P.nQ, NP, sizeof( HT ), xf ), NS, P.nT, P.nQ, NP, sizeof( HT ), xf );
    const size_t ldc = size_t( NS ) * P.nT;
    double* bc       = w.red + 16;    // broadcast slot
    unsigned long long itSum = 0, lsSum = 0;
    int failSum = 0, activeSum = 0, fbSum = 0;
    double dtMin = 1e300;
    // work items: all cells, or the cells k_check / k_update found unconverged
    int* alist;
    unsigned* acount;
    step_list( P, 0, alist, acount );
    const int nWork = alist ? int( *acount ) : P.nWork;
    for( ;; ) {
        int item;
        if( g.r == 0 ) bc[0] = double( atomicAdd( P.workCounter, 1u ) );
        g.sync();
        item = int( bc[0] );
        g.sync();
        if( item >= nWork ) break;
        const int cell = alist ? alist[item] : item;
        const int lev = P.level ? int( P.level[cell] ) : P.nLevels - 1;
        const int nTj = P.nTotalCell ? int( P.nTotalCell[cell] ) : P.nTLevel[lev];
        // load duals and moments (state-major, finest stride), checking finiteness on the way
        bool bad = false;
        for( int idx = g.r; idx < int( ldc ); idx += GROUP ) {
            double a = P.lam[cell * ldc + idx], b = P.u[cell * ldc + idx];
            w.lam[idx] = a;
            w.uh[idx]  = b;
            bad        = bad || !isfinite( a ) || !isfinite( b );
        }
        const bool anyBad = group_any<GROUP>( g, bad, w.red );
        g.sync();
        int iters = 0, ls = 0, rc;
        if( anyBad )
            rc = UQC_CELL_NONFINITE;
        else
        {
            PT_BEGIN( tn );
            if constexpr( Closure<CL>::LINEAR ) {
                linear_duals<NS, GROUP>( g, P, w.uh, w.lam );
                g.sync();
                rc = UQC_CELL_CONVERGED;
            }
            else if constexpr( TINY ) {
                rc = newton_cell_tiny<CL>( P, phi, phiWf, w, nTj, iters, ls );
            }
            else if constexpr( MIXED ) {
                if( mode == 1 && P.factorStore && P.newtonMode != 2 && P.maxIter > 1 ) {
                    // reuse the cell's stored FP32 factor when it was formed for this level
                    const int nH    = int( ( hess_doubles( NS * nTj ) + 1 ) & ~size_t( 1 ) );    // floats of the tiles
                    const int n8    = hnb( NS * nTj ) * 8;
                    float* st       = P.factorStore + size_t( cell ) * P.factorStride;
                    float* H        = reinterpret_cast<float*>( w.H );
                    float* Iv       = reinterpret_cast<float*>( w.I );
                    const bool have = P.factorLevel[cell] == nTj;
                    const int nX    = xpacked( NS * nTj );
                    if( have ) {
                        if( P.chordInverse )
                            for( int i = g.r; i < nX; i += GROUP ) w.X[i] = st[i];
                        else {
                            for( int i = g.r; i < nH; i += GROUP ) H[i] = st[i];
                            for( int i = g.r; i < n8; i += GROUP ) Iv[i] = st[nH + i];
                        }
                    }
                    g.sync();
                    bool fresh = false;
                    rc         = newton_cell_chord<CL, GROUP>( g, P, phi, phiWf, phiH, w, nTj, have, iters, ls, fresh );
                    if( rc == UQC_CELL_CONVERGED && fresh ) {
                        if( P.chordInverse )
                            for( int i = g.r; i < nX; i += GROUP ) st[i] = w.X[i];
                        else {
                            for( int i = g.r; i < nH; i += GROUP ) st[i] = H[i];
                            for( int i = g.r; i < n8; i += GROUP ) st[nH + i] = Iv[i];
                        }
                    }
                    if( g.r == 0 ) P.factorLevel[cell] = rc == UQC_CELL_CONVERGED ? ( fresh || have ? nTj : -1 ) : -1;
                }
                else {
                    rc = newton_cell<CL, GROUP, HT>( g, P, phi, phiWf, phiH, w, nTj, iters, ls );
                }
            }
            else {
                rc = newton_cell<CL, GROUP, HT>( g, P, phi, phiWf, phiH, w, nTj, iters, ls );
            }
            PT_END( tn, 0 );
        }
        if( MIXED && rc != UQC_CELL_CONVERGED && rc != UQC_CELL_NONFINITE ) {
            for( int idx = g.r; idx < int( ldc ); idx += GROUP ) P.lam[cell * ldc + idx] = w.lam[idx];
            if( g.r == 0 ) {
                P.fallbackList[atomicAdd( P.fallbackCount, 1u )] = cell;
                ++fbSum;
                itSum += iters;
                lsSum += ls;
            }
            g.sync();
            continue;
        }
        if( g.r == 0 ) {
            P.status[cell] = rc;
            P.iters[cell]  = iters;
            itSum += iters;
            lsSum += ls;
            failSum += rc != 0;
            activeSum += iters > 0;
        }
        for( int idx = g.r; idx < int( ldc ); idx += GROUP ) P.lam[cell * ldc + idx] = w.lam[idx];
        PT_BEGIN( te );
        if( mode == 1 ) {
            // [C] uQ = U(Lambda(lam)). A converged cell's last gradient evaluation
            // was at the accepted duals, so w.uk already holds U there (the
            // U(Vector&) form; the reference reconstructs with U(const Matrix&),
            // which for the Euler closure differs in the last bits only).
            if( rc != 0 || Closure<CL>::LINEAR ) {
                eval_lambda<NS, GROUP>( g, P, phi, w.lam, nTj, w.LA );
                g.sync();
                eval_u<CL, GROUP>( g, P, w.LA, w.uk, true );
            }
            g.sync();
            const double dloc = cell_epilogue<CL, GROUP>( g, P, phiWf, w.uh, w.uk, cell, lev, nTj, w.red );
            dtMin             = dloc < dtMin ? dloc : dtMin;
        }
        PT_END( te, 6 );
        g.sync();
    }
    if( g.r == 0 ) {
        if( itSum ) atomicAdd( &P.ctl->newtonIters, itSum );
        if( lsSum ) atomicAdd( &P.ctl->lineSearchTrials, lsSum );
        if( failSum ) atomicAdd( &P.ctl->failedCells, failSum );
        if( activeSum ) atomicAdd( &P.ctl->activeCells, activeSum );
        if( fbSum ) atomicAdd( &P.ctl->fallbackCells, (unsigned long long)fbSum );
        if( mode == 1 && dtMin < 1e300 ) atomic_min_pos_double( &P.ctl->dtBits, dtMin );
    }
}

__host__ __device__ inline size_t check_ws_doubles( int nS, int nT, int nQ ) {
    size_t ldc = size_t( nS ) * nT;
    return ( ( 3 * ldc + size_t( nS ) * nQ + 32 ) + 3 ) & ~size_t( 3 );
}

// Step mode, first half of the closure: one warp per cell evaluates the
// gradient at the current duals (the initial test of closure.cpp:139-142).
// Converged cells are finished here (epilogue [C]-[F]); the others are
// appended to P.activeList for k_closure. Lambda is formed node by node in
// registers and U(Lambda) stored (no nodal Lambda buffer), so up to 16 warps
// share a CTA and the latency of this per-cell work is hidden.
template <int CL> __global__ void __launch_bounds__( 512, 2 ) k_check( KParams P ) {
    constexpr int NS = Closure<CL>::NS;
    extern __shared__ __align__( 16 ) double smem[];
    if( !P.ctl->active ) return;
    // after a state change every cell; otherwise only the check list that
    // k_update filled (converged cells whose refinement level changes)
    const bool listMode = P.ctl->listReady != 0;
    const int par       = P.ctl->steps & 1;
    const int nItems    = listMode ? int( P.checkCount[par] ) : P.nWork;
    if( nItems == 0 ) return;
    int* alist;
    unsigned* acount;
    step_list( P, 0, alist, acount );
    Grp<32> g{int( threadIdx.x & 31 ), 0};
    const int warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    const double *phi = P.phi, *phiWf = P.phiWf;
    double* base = smem;
    if( P.tablesInSmem ) {
        size_t tn = size_t( P.nQ ) * P.ld + 4;
        for( size_t i = threadIdx.x; i < tn; i += blockDim.x ) {
            base[i]      = i < size_t( P.nQ ) * P.ld ? P.phi[i] : 0.0;
            base[tn + i] = i < size_t( P.nQ ) * P.ld ? P.phiWf[i] : 0.0;
        }
        phi   = base;
        phiWf = base + tn;
        base += 2 * tn;
        __syncthreads();
    }
    const size_t ldc = size_t( NS ) * P.nT;
    double* lam      = base + warp * check_ws_doubles( NS, P.nT, P.nQ );
    double* uh       = lam + ldc;
    double* ugs      = uh + ldc;    // sum_k U_s(k) phiWf(k, i), kept for the re-projection
    double* uk       = ugs + ldc;
    double* red      = uk + size_t( NS ) * P.nQ;
    double dtMin     = 1e300;
    for( int item = blockIdx.x * nWarps + warp; item < nItems; item += gridDim.x * nWarps ) {
        const int cell = listMode ? P.checkList[size_t( par ) * P.nCells + item] : P.cellBase + item;
        if( !listMode && P.finFlag && g.r == 0 ) P.finFlag[cell] = 0;
        CT_BEGIN( tcell );
        CT_BEGIN( tload );
        const int lev = int( P.level[cell] ), nTj = P.nTLevel[lev];
        bool bad = false;
        // the duals node-major (lam[i NS + s]: a basis function's NS duals in
        // 16-byte loads for the nodal sums), state-major for the linear closures
        for( int idx = g.r; idx < int( ldc ); idx += 32 ) {
            double a = P.lam[cell * ldc + idx], b = P.u[cell * ldc + idx];
            if constexpr( Closure<CL>::LINEAR )
                lam[idx] = a;
            else {
                const int s = idx / P.nT, i = idx - s * P.nT;
                lam[i * NS + s] = a;
            }
            uh[idx]  = b;
            bad      = bad || !isfinite( a ) || !isfinite( b );
        }
        bad = __any_sync( 0xffffffffu, bad );
        __syncwarp();
        CT_END( tload, 16, g.r == 0 );
        bool converged = false;
        if constexpr( Closure<CL>::LINEAR ) {
            // the duals come from the moments: no test, every cell finishes here
            if( !bad ) {
                linear_duals<NS, 32>( g, P, uh, lam );
                __syncwarp();
                for( int idx = g.r; idx < int( ldc ); idx += 32 ) P.lam[cell * ldc + idx] = lam[idx];
                converged = true;
            }
        }
        if( !bad ) {
            CT_BEGIN( tlu );
            // U(Lambda_k) at every node, Lambda_k in registers (closure.cpp:205-213, 234-253)
            for( int k = g.r; k < P.nQ; k += 32 ) {
                const double* row = phi + size_t( k ) * P.ld;
                double Lk[NS], y[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) Lk[s] = 0.0;
                for( int i = 0; i < nTj; ++i ) {
                    const double r = row[i];
                    double li[NS];
                    if constexpr( Closure<CL>::LINEAR ) {
#pragma unroll
                        for( int s = 0; s < NS; ++s ) li[s] = lam[s * P.nT + i];
                    }
                    else if constexpr( NS % 2 == 0 ) {
#pragma unroll
                        for( int s = 0; s < NS; s += 2 ) {
                            const double2 t = *reinterpret_cast<const double2*>( lam + i * NS + s );
                            li[s]           = t.x;
                            li[s + 1]       = t.y;
                        }
                    }
                    else {
#pragma unroll
                        for( int s = 0; s < NS; ++s ) li[s] = lam[i * NS + s];
                    }
#pragma unroll
                    for( int s = 0; s < NS; ++s ) Lk[s] = fma( li[s], r, Lk[s] );
                }
                Closure<CL>::U( Lk, y, true, P.phys );
#pragma unroll
                for( int s = 0; s < NS; ++s ) uk[s * P.nQ + k] = y[s];
            }
            __syncwarp();
            CT_END( tlu, 17, g.r == 0 );
            CT_BEGIN( tgr );
            if constexpr( !Closure<CL>::LINEAR ) {
            const double sq = gradient_sums<NS, 32>( g, P, phiWf, uk, uh, nTj, nullptr, ugs );
            const double gn = sqrt( group_sum<32>( g, sq, red ) );
            converged       = gn < P.eps;
            if( !converged && P.gStore ) {
                // the gradient the mixed form's Newton starts from: g = sum_k U phiWf - u
                double* gs = P.gStore + size_t( cell ) * P.gStride;
                for( int idx = g.r; idx < NS * nTj; idx += 32 ) {
                    const int s = idx / nTj, i = idx - s * nTj;
                    gs[idx]     = ugs[s * P.nT + i] - uh[s * P.nT + i];
                }
                if( g.r == 0 ) gs[ldc] = gn;
            }
            }
            CT_END( tgr, 18, g.r == 0 );
        }
        if( converged ) {
            if( g.r == 0 ) {
                P.status[cell] = UQC_CELL_CONVERGED;
                P.iters[cell]  = 0;
            }
            __syncwarp();
            CT_BEGIN( tep );
            const double d = cell_epilogue<CL, 32>( g, P, phiWf, uh, uk, cell, lev, nTj, red, Closure<CL>::LINEAR ? nullptr : ugs );
            dtMin          = d < dtMin ? d : dtMin;
            CT_END( tep, 19, g.r == 0 );
        }
        else if( g.r == 0 ) {
            alist[atomicAdd( acount, 1u )] = cell;
        }
        __syncwarp();
        CT_END( tcell, 20, g.r == 0 );
    }
    if( g.r == 0 && dtMin < 1e300 ) atomic_min_pos_double( &P.ctl->dtBits, dtMin );
}

// Ghost state of a wall cell at one node (expliciteuler.cpp:24-58): the
// velocity v = (u1, u2) / u0 loses its component along the boundary normal n,
// Vb = v - (n.v) n; momentum becomes u0 Vb, and on a no-slip wall the energy
// changes by u0 (|Vb|^2 - |v|^2) / 2. Euler 2-D states only.
template <int CL> __device__ __forceinline__ void wall_ghost( const double* a, const double* n, bool noslip, double* gh ) {
    constexpr int NS = Closure<CL>::NS;
#pragma unroll
    for( int s = 0; s < NS; ++s ) gh[s] = a[s];
    if constexpr( NS >= 4 ) {
        const double v0 = a[1] / a[0], v1 = a[2] / a[0];
        const double vn = n[0] * v0 + n[1] * v1;
        const double b0 = -( vn * n[0] ) + v0, b1 = -( vn * n[1] ) + v1;
        const double rho = a[0];
        gh[1]            = rho * b0;
        gh[2]            = rho * b1;
        if( noslip ) gh[3] += rho * 0.5 * ( ( b0 * b0 + b1 * b1 ) - ( v0 * v0 + v1 * v1 ) );
    }
}

// rhs(s, i) = sum_k Gs(s, k) phiWf(k, i) for one i (t = phiWf + i), the NS
// states as independent chains sharing each table value; SPLIT: over the nodes
// k = k0, k0 + dk, ... only (a separate instance: the contiguous loop's
// constant strides keep its addressing cheap).
// Gs is node-major (Gs[k NS + s]), so a node's NS values come in 16-byte
// shared-memory loads.
template <int NS, bool SPLIT = false>
__device__ __forceinline__ void project_lane( const double* Gs, const double* t, int ld, int nQ, double* r, int k0 = 0, int dk = 1 ) {
#pragma unroll
    for( int s = 0; s < NS; ++s ) r[s] = 0.0;
    if constexpr( !SPLIT ) {
        k0 = 0;
        dk = 1;
    }
    t += size_t( k0 ) * ld;
    const size_t tStep = size_t( dk ) * ld;
    for( int k = k0; k < nQ; k += dk, t += tStep ) {
        const double w = *t;
        double g[NS];
        if constexpr( NS % 2 == 0 ) {
#pragma unroll
            for( int s = 0; s < NS; s += 2 ) {
                const double2 v = *reinterpret_cast<const double2*>( Gs + k * NS + s );
                g[s]            = v.x;
                g[s + 1]        = v.y;
            }
        }
        else {
#pragma unroll
            for( int s = 0; s < NS; ++s ) g[s] = Gs[k * NS + s];
        }
#pragma unroll
        for( int s = 0; s < NS; ++s ) r[s] = fma( g[s], w, r[s] );
    }
}

// doubles per warp of k_update's shared memory: the nodal flux sums, 16 of
// face data, and the face fluxes of the nodes after the last full 64-node block
__host__ __device__ inline size_t update_warp_doubles( int nS, int nQ, int nFaces ) {
    return ( ( size_t( nS ) * nQ + 3 ) & ~size_t( 3 ) ) + 16 + ( ( size_t( nFaces ) * ( nQ & 63 ) * nS + 3 ) & ~size_t( 3 ) );
}

// Warp-buffered append to a device list (warp-uniform call): lane `cnt` keeps
// the entry; 32 entries take one atomicAdd on the list length.
struct WarpListBuf {
    int cell = 0, cnt = 0;
    __device__ __forceinline__ void push( int lane, int c, int* list, unsigned* count ) {
        if( lane == cnt ) cell = c;
        if( ++cnt == 32 ) flush( lane, list, count );
    }
    __device__ __forceinline__ void flush( int lane, int* list, unsigned* count ) {
        if( cnt == 0 ) return;
        unsigned base = 0;
        if( lane == 0 ) base = atomicAdd( count, unsigned( cnt ) );
        base = __shfl_sync( 0xffffffffu, base, 0 );
        if( lane < cnt ) list[base + lane] = cell;
        cnt = 0;
    }
};

// A cell whose next closure test k_update found passed: it keeps its duals,
// nodal states, moments and level; the next step sees it converged with no
// iterations, its residual reference is u_new(0, 0) and its dt the stored one.
// Its closure status of that step (converged, 0 iterations) is written by the
// k_update of that step, so that between steps the status arrays describe the
// last closure, as without this shortcut.
__device__ __forceinline__ void finish_cell( const KParams& P, int cell, double u00, double& dtNext ) {
    P.uOld0[cell]  = u00;
    P.finFlag[cell] = 1;    // its status is written by the next k_update (after the step it skips)
    const double d = P.cellDt[cell];
    dtNext         = d < dtNext ? d : dtNext;
}

// Flux + explicit Euler update (expliciteuler.cpp:17-74), one warp per cell
// (grid-stride over cells, many warps per SM), and the residual / time
// control finished by the last CTA. Per node the kinetic fluxes of the cell's
// faces are summed first (sum_f G_f), then projected once onto the basis:
// rhs(s, i) = sum_k Gsum(s, k) phiWf(k, i). The reference accumulates the
// projection face by face (momentsolver.cpp:413-416); the sums agree up to
// reassociation. Each lane carries two outputs with two partial sums each.
// FIN: with the next step's convergence test (P.finishInUpdate); the plain
// instance (adaptive configurations, test off) carries none of its code.
// WALL: the mesh has wall cells (ghost states at their boundary faces); the
// instance without walls evaluates two nodes per lane at a time (independent
// flux chains for the scheduler) with no ghost-state code.
// SPLIT: a level's last block of m <= 16 basis functions also splits the nodes
// over lane groups in the projection (an instance of its own: the second copy
// of the projection loop measured 1.7 % slower on 2-D Euler with 21 functions,
// which never takes it; 10 % faster on 35 functions and 512 nodes).
// CTAs per SM the register budget is cut for: 2 with three or four states, 4
// with one or two (3 for two states with the next-step test, which would spill
// more at 64 registers). The small systems are latency-bound on the loads of
// the neighbours' nodal states; more resident warps hide it (measured, 1M-cell
// shallow water: 2.33 / 1.78 / 1.61 ms at 2 / 3 / 4 CTAs per SM).
template <int CL, bool FIN> constexpr int update_min_ctas() {
    return Closure<CL>::NS >= 3 ? 2 : ( Closure<CL>::NS == 2 && FIN ? 3 : 4 );
}

template <int CL, bool FIN, bool WALL, bool SPLIT>
__global__ void __launch_bounds__( 256, ( update_min_ctas<CL, FIN>() ) ) k_update( KParams P ) {
    const bool finish = FIN && P.finishInUpdate;
    constexpr int NS = Closure<CL>::NS;
    extern __shared__ __align__( 16 ) double smem[];
    __shared__ double blockRes[32];
    __shared__ int isLast;
    if( !P.ctl->active ) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nWarps = blockDim.x >> 5;
    const double* phiWf = P.phiWf;
    double* base        = smem;
    if( P.tablesInSmem ) {
        size_t tn = size_t( P.nQ ) * P.ld;
        for( size_t i = threadIdx.x; i < tn; i += blockDim.x ) base[i] = P.phiWf[i];
        phiWf = base;
        base += ( tn + 4 ) & ~size_t( 3 );
        __syncthreads();
    }
    // per warp: the summed nodal fluxes (NS x nQ, node-major), then the cell's
    // face data: unit normal (2), scaled normal (2) and length of each face
    double* Gs       = base + size_t( warp ) * update_warp_doubles( NS, P.nQ, P.nFaces );
    double* fd       = Gs + ( ( size_t( NS ) * P.nQ + 3 ) & ~size_t( 3 ) );
    const double dt  = __longlong_as_double( (long long)P.ctl->dtBits );
    const size_t ldc = size_t( NS ) * P.nT;
    double res       = 0.0;
    double dtNext    = 1e300;    // lane 0: min dt of the cells finished for the next step
    int* nlist       = nullptr;
    unsigned* ncount = nullptr;
    if( finish ) step_list( P, 1, nlist, ncount );
    int* clist        = nullptr;
    unsigned* ccount  = nullptr;
    if( finish ) {
        clist  = P.checkList + size_t( ( P.ctl->steps + 1 ) & 1 ) * P.nCells;
        ccount = P.checkCount + ( ( P.ctl->steps + 1 ) & 1 );
    }
    WarpListBuf nbuf, cbuf;    // next step's active list and check list
    for( int cell = P.cellBase + blockIdx.x * nWarps + warp; cell < P.cellBase + P.nWork; cell += gridDim.x * nWarps ) {
        const int bc = P.boundary[cell];
        if( finish && lane == 0 && P.finFlag[cell] ) {
            // finished by the previous update: this step's closure status
            P.status[cell]  = UQC_CELL_CONVERGED;
            P.iters[cell]   = 0;
            P.finFlag[cell] = 0;
        }
        if( bc == 1 ) {
            // Dirichlet cell: uNew = u (expliciteuler.cpp:21-23)
            for( int idx = lane; idx < int( ldc ); idx += 32 ) P.u[cell * ldc + idx] = P.uRe[cell * ldc + idx];
            if( lane == 0 ) {
                const double u0 = P.uRe[cell * ldc];
                res += fabs( u0 - P.uOld0[cell] ) * P.area[cell];
                // its moments are the re-projected ones: the next closure test passes
                if( finish && P.nLevels == 1 ) finish_cell( P, cell, u0, dtNext );
            }
            // with refinement levels k_check's epilogue applies the level rule
            if( finish && P.nLevels > 1 ) cbuf.push( lane, cell, clist, ccount );
            continue;
        }
        const int nTj    = P.nTLevel[P.level[cell]];
        const double* ua = P.uQ + size_t( cell ) * NS * P.nQ;
        // the faces' neighbours and normals, once per cell (nFaces <= 3)
        const double* ub[3];
        bool ghost[3];
        // wall cells (Euler 2-D): faces without a neighbour see the cell's own
        // states reflected at the boundary normal (expliciteuler.cpp:24-70)
        const bool wall = WALL && NS == 4 && bc >= 2;
        double bn[2]    = {0.0, 0.0};
        if( wall ) {
            bn[0] = P.bndNormal[2 * cell];
            bn[1] = P.bndNormal[2 * cell + 1];
        }
#pragma unroll
        for( int f = 0; f < 3; ++f ) {
            ghost[f] = false;
            ub[f]    = ua;
            if( f < P.nFaces ) {
                const int nb = P.nbr[cell * P.nFaces + f];
                ghost[f]     = wall && nb == P.nCells;
                ub[f]        = P.uQ + size_t( nb ) * NS * P.nQ;
            }
        }
        __syncwarp();    // the previous cell's face data is read
        if( lane < P.nFaces ) {
            const int f    = lane;
            const double a = P.scaledN[( cell * P.nFaces + f ) * 2], b = P.scaledN[( cell * P.nFaces + f ) * 2 + 1];
            fd[5 * f]      = P.unitN[( cell * P.nFaces + f ) * 2];
            fd[5 * f + 1]  = P.unitN[( cell * P.nFaces + f ) * 2 + 1];
            fd[5 * f + 2]  = a;
            fd[5 * f + 3]  = b;
            fd[5 * f + 4]  = sqrt( a * a + b * b );    // |n| of euler2d.cpp:84, once per face
        }
        __syncwarp();
        if constexpr( WALL ) {
            for( int k = lane; k < P.nQ; k += 32 ) {
                double a[NS], gsum[NS], gh[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) {
                    a[s]    = ua[s * P.nQ + k];
                    gsum[s] = 0.0;
                }
                if( wall ) wall_ghost<CL>( a, bn, bc == 2, gh );
#pragma unroll
                for( int f = 0; f < 3; ++f ) {
                    if( f < P.nFaces ) {
                        double b[NS], y[NS];
                        if( ghost[f] )
                            Problem<CL>::flux( gh, gh, fd + 5 * f, fd + 5 * f + 2, fd[5 * f + 4], y, P.phys );
                        else {
#pragma unroll
                            for( int s = 0; s < NS; ++s ) b[s] = ub[f][s * P.nQ + k];
                            Problem<CL>::flux( a, b, fd + 5 * f, fd + 5 * f + 2, fd[5 * f + 4], y, P.phys );
                        }
#pragma unroll
                        for( int s = 0; s < NS; ++s ) gsum[s] += y[s];
                    }
                }
#pragma unroll
                for( int s = 0; s < NS; ++s ) Gs[k * NS + s] = gsum[s];
            }
        }
        else {
            // nodes k and k + 32 together over the full 64-node blocks
            const int kPair = P.nQ & ~63;
            for( int k0 = lane; k0 < kPair; k0 += 64 ) {
                const bool two = true;
                const int k1   = k0 + 32;
                double a0[NS], a1[NS], g0[NS], g1[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) {
                    a0[s] = ua[s * P.nQ + k0];
                    a1[s] = ua[s * P.nQ + k1];
                    g0[s] = g1[s] = 0.0;
                }
#pragma unroll
                for( int f = 0; f < 3; ++f ) {
                    if( f < P.nFaces ) {
                        double b0[NS], b1[NS], y0[NS], y1[NS];
#pragma unroll
                        for( int s = 0; s < NS; ++s ) {
                            b0[s] = ub[f][s * P.nQ + k0];
                            b1[s] = ub[f][s * P.nQ + k1];
                        }
                        Problem<CL>::flux( a0, b0, fd + 5 * f, fd + 5 * f + 2, fd[5 * f + 4], y0, P.phys );
                        Problem<CL>::flux( a1, b1, fd + 5 * f, fd + 5 * f + 2, fd[5 * f + 4], y1, P.phys );
#pragma unroll
                        for( int s = 0; s < NS; ++s ) {
                            g0[s] += y0[s];
                            g1[s] += y1[s];
                        }
                    }
                }
#pragma unroll
                for( int s = 0; s < NS; ++s ) Gs[k0 * NS + s] = g0[s];
                if( two ) {
#pragma unroll
                    for( int s = 0; s < NS; ++s ) Gs[k1 * NS + s] = g1[s];
                }
            }
            // the remaining R = nQ mod 64 nodes: a slot per (face, node), two
            // slots per lane at a time (a lane without a second slot repeats its
            // first), so that no lane idles for a whole face; the fluxes go to
            // the scratch, then each node's are summed in face order as above
            const int R = P.nQ - kPair;
            if( R > 0 ) {
                double* Yt  = fd + 16;
                const int S = P.nFaces * R;
                for( int j0 = lane; j0 < S; j0 += 64 ) {
                    const bool two = j0 + 32 < S;
                    const int j1   = two ? j0 + 32 : j0;
                    const int f0 = j0 / R, k0 = kPair + j0 - f0 * R;
                    const int f1 = j1 / R, k1 = kPair + j1 - f1 * R;
                    const double* n0 = f0 == 0 ? ub[0] : ( f0 == 1 ? ub[1] : ub[2] );
                    const double* n1 = f1 == 0 ? ub[0] : ( f1 == 1 ? ub[1] : ub[2] );
                    double a0[NS], a1[NS], b0[NS], b1[NS], y0[NS], y1[NS];
#pragma unroll
                    for( int s = 0; s < NS; ++s ) {
                        a0[s] = ua[s * P.nQ + k0];
                        a1[s] = ua[s * P.nQ + k1];
                        b0[s] = n0[s * P.nQ + k0];
                        b1[s] = n1[s * P.nQ + k1];
                    }
                    Problem<CL>::flux( a0, b0, fd + 5 * f0, fd + 5 * f0 + 2, fd[5 * f0 + 4], y0, P.phys );
                    Problem<CL>::flux( a1, b1, fd + 5 * f1, fd + 5 * f1 + 2, fd[5 * f1 + 4], y1, P.phys );
#pragma unroll
                    for( int s = 0; s < NS; ++s ) Yt[j0 * NS + s] = y0[s];
                    if( two ) {
#pragma unroll
                        for( int s = 0; s < NS; ++s ) Yt[j1 * NS + s] = y1[s];
                    }
                }
                __syncwarp();
                for( int t = lane; t < R; t += 32 ) {
                    double gsum[NS];
#pragma unroll
                    for( int s = 0; s < NS; ++s ) gsum[s] = 0.0;
                    for( int f = 0; f < P.nFaces; ++f ) {
#pragma unroll
                        for( int s = 0; s < NS; ++s ) gsum[s] += Yt[( f * R + t ) * NS + s];
                    }
#pragma unroll
                    for( int s = 0; s < NS; ++s ) Gs[( kPair + t ) * NS + s] = gsum[s];
                }
            }
        }
        __syncwarp();
        // projection and update: a lane per basis function i, the NS states as
        // independent chains sharing each table value
        const double c = dt / P.area[cell];
        double sq      = 0.0;
        double v0a = 0.0, v0b = 0.0;    // u_new(0, lane) and u_new(0, lane + 32), for the level rule
        auto apply     = [&]( int i, const double* old, const double* r ) {
#pragma unroll
            for( int s = 0; s < NS; ++s ) {
                const double v   = old[s] - r[s] * c;
                const double gi  = old[s] - v;
                P.u[cell * ldc + s * P.nT + i] = v;
                sq                             = fma( gi, gi, sq );
                if( s == 0 && i < 32 ) v0a = v;
                if( s == 0 && i >= 32 && i < 64 ) v0b = v;
                if( s == 0 && i == 0 ) res += fabs( v - P.uOld0[cell] ) * P.area[cell];
            }
        };
        if constexpr( !SPLIT ) {
            for( int i = lane; i < nTj; i += 32 ) {    // beyond the level u stays zero (epilogue)
                // the re-projected moments first: their loads overlap the
                // projection (uRe and u may alias, so a load after a store to u
                // could not be moved ahead of it)
                double old[NS], r[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) old[s] = P.uRe[cell * ldc + s * P.nT + i];
                project_lane<NS>( Gs, phiWf + i, P.ld, P.nQ, r );
                apply( i, old, r );
            }
        }
        else {
            // blocks of 32 functions; a block of m <= 16 (the last) splits the
            // nodes over 32 / w lane groups too (w = m rounded up to a power
            // of two), each group summing the nodes k = part (mod 32 / w),
            // then a butterfly over the groups
            for( int i0 = 0; i0 < nTj; i0 += 32 ) {
                const int m = min( 32, nTj - i0 );
                int w       = 1;
                while( w < m ) w <<= 1;
                const int part = lane / w, i = i0 + ( lane & ( w - 1 ) );
                const bool in  = i < i0 + m;
                double old[NS], r[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) {
                    old[s] = ( in && part == 0 ) ? P.uRe[cell * ldc + s * P.nT + i] : 0.0;
                    r[s]   = 0.0;
                }
                if( in ) {
                    if( w == 32 )
                        project_lane<NS>( Gs, phiWf + i, P.ld, P.nQ, r );
                    else
                        project_lane<NS, true>( Gs, phiWf + i, P.ld, P.nQ, r, part, 32 / w );
                }
#pragma unroll
                for( int s = 0; s < NS; ++s )
                    for( int o = w; o < 32; o <<= 1 ) r[s] += __shfl_xor_sync( 0xffffffffu, r[s], o );
                if( in && part == 0 ) apply( i, old, r );
            }
        }
        if( finish ) {
            // The next step's closure test, here: its gradient is
            // sum_k U(Lambda_k) phiWf(k, i) - u_new = uRe - u_new, because uRe was
            // re-projected from the same duals' nodal states (which this kernel
            // just used). A cell that passes (and keeps its level) would only
            // be re-projected onto uRe again: it skips the closure and keeps
            // uRe; the others go to the next step's list.
            for( int o = 16; o > 0; o >>= 1 ) sq += __shfl_xor_sync( 0xffffffffu, sq, o );
            sq              = __shfl_sync( 0xffffffffu, sq, 0 );    // one decision for the warp
            const bool pass = sqrt( sq ) < P.eps;
            bool fin        = pass;
            if( fin && P.nLevels > 1 ) {
                // the level rule of the epilogue, on u_new(0, .) in the same order
                // (values from the lanes' registers; beyond 64 moments from memory)
                __syncwarp();
                const int lev = int( P.level[cell] );
                auto at       = [&]( int i ) {
                    const double r = __shfl_sync( 0xffffffffu, ( i >> 5 ) ? v0b : v0a, i & 31 );
                    return i < 64 ? r : P.u[cell * ldc + i];
                };
                if( level_rule( P, level_indicator( P, at, lev, nTj ), lev ) != lev ) fin = false;
            }
            if( fin ) {
                if( lane == 0 ) finish_cell( P, cell, v0a, dtNext );
            }
            else if( pass )
                cbuf.push( lane, cell, clist, ccount );    // converged, new level: k_check's epilogue
            else {
                if( P.gStore ) {
                    // the gradient the mixed form's Newton starts from: uRe - u_new,
                    // the same differences as gi above (from the values just stored)
                    __syncwarp();
                    double* gs = P.gStore + size_t( cell ) * P.gStride;
                    for( int idx = lane; idx < NS * nTj; idx += 32 ) {
                        const int s = idx / nTj, i = idx - s * nTj;
                        gs[idx]     = P.uRe[cell * ldc + s * P.nT + i] - P.u[cell * ldc + s * P.nT + i];
                    }
                    if( lane == 0 ) gs[ldc] = sqrt( sq );
                }
                nbuf.push( lane, cell, nlist, ncount );
            }
        }
        __syncwarp();
    }
    if( finish ) {
        nbuf.flush( lane, nlist, ncount );
        cbuf.flush( lane, clist, ccount );
    }
    if( lane == 0 && dtNext < 1e300 ) atomic_min_pos_double( &P.ctl->dtBitsNext, dtNext );
    // deterministic residual: per-thread partials -> CTA sum -> per-CTA slot -> last CTA sums in order
    for( int o = 16; o > 0; o >>= 1 ) res += __shfl_xor_sync( 0xffffffffu, res, o );
    if( ( threadIdx.x & 31 ) == 0 ) blockRes[threadIdx.x >> 5] = res;
    __syncthreads();
    if( threadIdx.x == 0 ) {
        double s = 0.0;
        for( int w = 0; w < int( blockDim.x >> 5 ); ++w ) s += blockRes[w];
        P.blockPartial[size_t( P.updChunk ) * gridDim.x + blockIdx.x] = s;
        __threadfence();
        unsigned done = atomicAdd( &P.ctl->doneBlocks, 1u );
        // the launches of a chunked update run one after another on the
        // stream: the last CTA of the last launch finishes the step
        isLast = done == gridDim.x * unsigned( P.updChunks ) - 1;
    }
    __syncthreads();
    double total = 0.0;
    if( isLast && threadIdx.x < 32 ) {
        __threadfence();
        // the CTA partials in launch and CTA order: the warp loads 32 at a
        // time, lane 0 adds them in sequence from the shuffles
        const unsigned nb = gridDim.x * unsigned( P.updChunks );
        for( unsigned b0 = 0; b0 < nb; b0 += 32 ) {
            const unsigned b = b0 + threadIdx.x;
            const double v   = b < nb ? ( (volatile double*)P.blockPartial )[b] : 0.0;
            const unsigned m = min( 32u, nb - b0 );
            for( unsigned j = 0; j < m; ++j ) total += __shfl_sync( 0xffffffffu, v, int( j ) );
        }
    }
    if( isLast && threadIdx.x == 0 ) {
        Control* C    = P.ctl;
        C->nActive[C->steps & 1] = 0;    // this step's lists are consumed (before steps advances)
        C->nCheck[C->steps & 1]  = 0;
        C->residual   = total;
        C->dt         = dt;
        C->t          = C->t + dt;
        C->steps      = C->steps + 1;
        C->active     = ( C->t < C->tEnd && C->residual > C->minResidual && ( C->maxSteps == 0 || C->steps < C->maxSteps ) ) ? 1 : 0;
        C->activeCellsLast = C->activeCells;
        C->activeCells     = 0;
        // retardation: raise the level cap as the residual falls below the thresholds
        if( P.nRet > 0 ) {
            int k = C->retIndex;
            while( k < P.nRet && total < P.retRes[k] ) ++k;
            C->retIndex = k;
            C->levelCap = P.retLev[k];
        }
        // the next step's min starts from the cells finished here (+inf if none)
        C->dtBits     = finish ? ( (volatile unsigned long long*)&C->dtBitsNext )[0] : 0x7FF0000000000000ull;
        C->dtBitsNext = 0x7FF0000000000000ull;
        C->listReady = finish ? 1 : 0;
        C->workCounter  = 0;
        C->workCounter2 = 0;
        C->nFallback    = 0;
        for( int r = 0; r < 16; ++r ) C->v2Work[r] = 0;
        for( int r = 0; r < 4; ++r ) C->v2Count[r] = 0;
        C->doneBlocks  = 0;
    }
}

// Initial moments u_j = U_IC(x_j, xi_k) phiWf and duals lambda_j(:,0) = DS(u_j(:,0)).
// keepMoments: the moments are already in place (restart without duals,
// momentsolver.cpp:463-485); only the duals are set.
template <int CL, int GROUP> __global__ void __launch_bounds__( GROUP == 32 ? 256 : GROUP ) k_init( KParams P, int keepMoments ) {
    constexpr int NS = Closure<CL>::NS;
    extern __shared__ __align__( 16 ) double smem[];
    const int groups = blockDim.x / GROUP;
    Grp<GROUP> g{int( threadIdx.x % GROUP ), 1 + int( threadIdx.x / GROUP )};
    const int gid   = threadIdx.x / GROUP;
    double* uic     = smem + size_t( gid ) * ( size_t( NS ) * P.nQ + 8 );
    const size_t ldc = size_t( NS ) * P.nT;
    for( int cell = blockIdx.x * groups + gid; cell < P.nCells; cell += gridDim.x * groups ) {
        for( int k = g.r; k < P.nQ && !keepMoments; k += GROUP ) {
            double y[NS];
            Problem<CL>::ic( P.center + 2 * cell, P.xi + size_t( k ) * P.dimXi, y, P.phys );
#pragma unroll
            for( int s = 0; s < NS; ++s ) uic[s * P.nQ + k] = y[s];
        }
        g.sync();
        for( int idx = g.r; idx < int( ldc ); idx += GROUP ) {
            int s = idx / P.nT, i = idx - s * P.nT;
            if( !keepMoments ) {
                double a = 0.0;
                for( int k = 0; k < P.nQ; ++k ) a = fma( uic[s * P.nQ + k], P.phiWf[size_t( k ) * P.ld + i], a );
                P.u[cell * ldc + idx] = a;
            }
            P.lam[cell * ldc + idx] = 0.0;
        }
        g.sync();
        if( g.r == 0 ) {
            double u0[NS], ds[NS];
#pragma unroll
            for( int s = 0; s < NS; ++s ) u0[s] = P.u[cell * ldc + s * P.nT];
            Closure<CL>::DS( u0, ds, P.phys );
#pragma unroll
            for( int s = 0; s < NS; ++s ) P.lam[cell * ldc + s * P.nT] = ds[s];
            P.level[cell] = unsigned( P.nLevels - 1 );
        }
        g.sync();
    }
}

// Mean and variance (vector-form ansatz), out[cell 2 NS + r].
template <int CL, int GROUP> __global__ void __launch_bounds__( GROUP == 32 ? 256 : GROUP ) k_meanvar( KParams P, double* out ) {
    constexpr int NS = Closure<CL>::NS;
    extern __shared__ __align__( 16 ) double smem[];
    const int groups = blockDim.x / GROUP;
    Grp<GROUP> g{int( threadIdx.x % GROUP ), 1 + int( threadIdx.x / GROUP )};
    const int gid    = threadIdx.x / GROUP;
    double* L        = smem + size_t( gid ) * ( 2 * size_t( NS ) * P.nQ + 8 );
    double* uk       = L + size_t( NS ) * P.nQ;
    const size_t ldc = size_t( NS ) * P.nT;
    for( int cell = blockIdx.x * groups + gid; cell < P.nCells; cell += gridDim.x * groups ) {
        const int nTj = P.nTLevel[P.level[cell]];
        eval_lambda<NS, GROUP>( g, P, P.phi, P.lam + cell * ldc, nTj, L );
        g.sync();
        eval_u<CL, GROUP>( g, P, L, uk, true );
        g.sync();
        for( int s = g.r; s < NS; s += GROUP ) {
            double e = 0.0, v = 0.0;
            for( int k = 0; k < P.nQ; ++k ) e = fma( uk[s * P.nQ + k], P.phiWf[size_t( k ) * P.ld], e );
            for( int k = 0; k < P.nQ; ++k ) {
                double dv = uk[s * P.nQ + k] - e;
                v         = fma( dv * dv, P.phiWf[size_t( k ) * P.ld], v );
            }
            out[cell * 2 * NS + s]      = e;
            out[cell * 2 * NS + NS + s] = v;
        }
        g.sync();
    }
}

}    // namespace uqc
