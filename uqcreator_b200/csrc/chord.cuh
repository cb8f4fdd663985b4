// Mixed-form closure of the time step, split by what bounds each part.
//
// The damped Newton of Closure::SolveClosure (closure.cpp:133-193) spends
// most of its iterations on directions and line-search trials; the Hessian
// and its factorisation are needed only when a cell's held inverse stops
// contracting (an inexact, chord Newton). The three kernels below split the
// work accordingly, and a time step runs them in rounds:
//
//   k_chord   a warp per cell, about 8 KB of shared memory per cell (duals,
//             moments, gradients and nodal states; no Hessian), so that many
//             cells share an SM and hide each other's FP64 latency. Newton
//             directions d = H0^-1 g from the cell's held inverse (FP32, read
//             from HBM/L2 as one coalesced mat-vec), FP64 trial gradients,
//             line search and convergence test, then the epilogue of a
//             converged cell. A cell without a usable inverse is appended to
//             the round's re-factor list and leaves.
//   k_hess_tc the Hessians of the listed cells on the tensor cores: every
//             block (l, m) of a cell's Hessian is sum_k phi_kj phi_ki wt_k
//             DU_lm(Lambda_k) (closure.cpp:255-271, the pair-product table
//             _hPartial of :69-72), i.e. the product of a constant table Q
//             (pairs j <= i x nodes) with the cell's nodal DU (nodes x blocks).
//             Twelve cells' DU rows form the A operand (M = 128) and Q the B
//             operand (N = pairs), both BF16 split into a high and a low part
//             (three products: FP32-level accuracy), accumulated in FP32 in
//             tensor memory by tcgen05.mma and written out per cell.
//   k_invert  per cell (two warps): the Hessian (from k_hess_tc, or assembled
//             on CUDA cores), Cholesky factor (FP32), inverse H^-1 = U^-1
//             U^-T written to the cell's store slot for the next k_chord round.
//
// The gradient, the line-search and convergence tests, the duals and the
// moments stay FP64, so a converged cell meets the FP64 tolerance. Cells that
// the mixed form cannot finish (iteration or refinement limit, FP32 factor
// not positive definite, more re-factorisations than rounds) go to the FP64
// kernel's fallback list with their last accepted duals.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "ipm_kernels.cuh"

namespace uqc {

// ---------------------------------------------------------------- chord kernel

// Per-warp workspace of k_chord (doubles): duals and moments at the finest
// stride nT (state-major, as in HBM); trial duals basis-major (lamI[i NS + s],
// so a basis function's NS values are 16-byte loads); the trial's moment sums
// m(s, i) = sum_k U phiWf (kept for the epilogue's re-projection); gradient,
// trial gradient and direction (compact, n = NS nTj); nodal states uk
// node-major (uk[k NS + s]); reduction scratch; the gradient in FP32.
struct ChordWs {
    double *lam, *lamI, *uh, *m, *g, *gN, *d, *uk, *red;
    float* gf;
};

__host__ __device__ inline size_t chord_ws_doubles( int nS, int nT, int nQ ) {
    auto a4          = []( size_t x ) { return ( x + 3 ) & ~size_t( 3 ); };
    const size_t ldc = size_t( nS ) * nT;
    return 7 * a4( ldc ) + a4( size_t( nS ) * nQ ) + 32 + a4( ( ldc + 1 ) / 2 );
}

__device__ inline ChordWs chord_carve( double* p, int nS, int nT, int nQ ) {
    auto a4          = []( size_t x ) { return ( x + 3 ) & ~size_t( 3 ); };
    const size_t ldc = a4( size_t( nS ) * nT );
    ChordWs w;
    w.lam  = p;
    w.lamI = p + ldc;
    w.uh   = p + 2 * ldc;
    w.m    = p + 3 * ldc;
    w.g    = p + 4 * ldc;
    w.gN   = p + 5 * ldc;
    w.d    = p + 6 * ldc;
    w.uk   = p + 7 * ldc;
    w.red  = w.uk + a4( size_t( nS ) * nQ );
    w.gf   = reinterpret_cast<float*>( w.red + 32 );
    return w;
}

// Lists of the mixed form's rounds: round r's re-factor list is the input of
// k_hess_tc / k_invert round r and of k_chord round r + 1.
__device__ __forceinline__ int* refactor_list( const KParams& P, int r ) { return P.v2Lists + size_t( r ) * P.nCells; }

// gStore slot of a cell: the gradient at its accepted duals (compact, n values)
// and its norm at index ldc.
__device__ __forceinline__ double* gslot( const KParams& P, int cell ) { return P.gStore + size_t( cell ) * P.gStride; }

// d = H0^-1 g with the cell's held inverse (FP32, n x n, symmetric, row-major):
// lane o sums column o, d_o = sum_j Hinv(j, o) g_j; each step j reads a row of
// the inverse with consecutive lanes on consecutive addresses. The rows are
// loaded in batches of CHORD_JB before their FMAs, so that a batch's loads
// are in flight together (the inverse comes from L2 or HBM).
constexpr int CHORD_JB = 14;
__device__ __forceinline__ void chord_direction( const float* __restrict__ Hinv, int n, const float* gf, double* d, int lane ) {
    const int o0 = lane, o1 = lane + 32, o2 = lane + 64;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f;
    if( n % CHORD_JB == 0 && n > 64 && n <= 96 ) {
        // whole batches, two full column blocks: only the third needs a bound
        const bool in2 = o2 < n;
        for( int j0 = 0; j0 < n; j0 += CHORD_JB ) {
            float h0[CHORD_JB], h1[CHORD_JB], h2[CHORD_JB];
            const float* rj = Hinv + size_t( j0 ) * n;
#pragma unroll
            for( int t = 0; t < CHORD_JB; ++t ) {
                h0[t] = __ldg( rj + t * n + o0 );
                h1[t] = __ldg( rj + t * n + o1 );
                h2[t] = in2 ? __ldg( rj + t * n + o2 ) : 0.f;
            }
#pragma unroll
            for( int t = 0; t < CHORD_JB; ++t ) {
                const float gj = gf[j0 + t];
                a0             = fmaf( h0[t], gj, a0 );
                a1             = fmaf( h1[t], gj, a1 );
                a2             = fmaf( h2[t], gj, a2 );
            }
        }
        d[o0] = double( a0 );
        d[o1] = double( a1 );
        if( in2 ) d[o2] = double( a2 );
        return;
    }
    for( int j0 = 0; j0 < n; j0 += CHORD_JB ) {
        float h0[CHORD_JB], h1[CHORD_JB], h2[CHORD_JB];
#pragma unroll
        for( int t = 0; t < CHORD_JB; ++t ) {
            const int j     = j0 + t;
            const float* rj = Hinv + size_t( j ) * n;
            h0[t]           = ( j < n && o0 < n ) ? __ldg( rj + o0 ) : 0.f;
            h1[t]           = ( j < n && o1 < n ) ? __ldg( rj + o1 ) : 0.f;
            h2[t]           = ( j < n && o2 < n ) ? __ldg( rj + o2 ) : 0.f;
        }
#pragma unroll
        for( int t = 0; t < CHORD_JB; ++t ) {
            const float gj = j0 + t < n ? gf[j0 + t] : 0.f;
            a0             = fmaf( h0[t], gj, a0 );
            a1             = fmaf( h1[t], gj, a1 );
            a2             = fmaf( h2[t], gj, a2 );
        }
    }
    if( o0 < n ) d[o0] = double( a0 );
    if( o1 < n ) d[o1] = double( a1 );
    if( o2 < n ) d[o2] = double( a2 );
    for( int o = lane + 96; o < n; o += 32 ) {    // systems beyond 96 duals
        float a = 0.f;
        for( int j = 0; j < n; ++j ) a = fmaf( __ldg( Hinv + size_t( j ) * n + o ), gf[j], a );
        d[o] = double( a );
    }
}

// NS values of node k of a node-major array (16-byte loads for even NS).
template <int NS> __device__ __forceinline__ void load_node( const double* a, int k, double* v ) {
    if constexpr( NS % 2 == 0 ) {
#pragma unroll
        for( int s = 0; s < NS; s += 2 ) {
            const double2 t = *reinterpret_cast<const double2*>( a + k * NS + s );
            v[s]            = t.x;
            v[s + 1]        = t.y;
        }
    }
    else {
#pragma unroll
        for( int s = 0; s < NS; ++s ) v[s] = a[k * NS + s];
    }
}

// The trial gradient for nTj <= 64 / PARTS basis functions: the warp's lanes
// take (part, i) slots in two rounds (slot j = part nTj + i, round j / 32,
// lane j mod 32), each summing the nodes k = part (mod PARTS), so that no lane
// idles over all nodes; lane i then gathers its PARTS partial sums by
// shuffles and adds them in part order. Outputs as chord_gradient's.
template <int NS, int PARTS>
__device__ __forceinline__ double chord_gradient_split( const KParams& P, const double* phiWf, const double* uk, const double* uh, int nTj,
                                                        double* gout, double* ms, int lane ) {
    const int slots = PARTS * nTj;
    double v[2][NS];
#pragma unroll
    for( int r = 0; r < 2; ++r ) {
#pragma unroll
        for( int s = 0; s < NS; ++s ) v[r][s] = 0.0;
        const int j = lane + 32 * r;
        if( j < slots ) {
            const int p = j / nTj, i = j - p * nTj;
            const double* t = phiWf + size_t( p ) * P.ld + i;
            const int tStep = PARTS * P.ld;
            for( int k = p; k < P.nQ; k += PARTS, t += tStep ) {
                const double w = *t;
                double x[NS];
                load_node<NS>( uk, k, x );
#pragma unroll
                for( int s = 0; s < NS; ++s ) v[r][s] = fma( x[s], w, v[r][s] );
            }
        }
    }
    double m[NS];
#pragma unroll
    for( int p = 0; p < PARTS; ++p ) {
        const int j = p * nTj + lane, src = j & 31;
        const bool second = j >= 32;
#pragma unroll
        for( int s = 0; s < NS; ++s ) {
            const double a0 = __shfl_sync( 0xffffffffu, v[0][s], src );
            const double a1 = __shfl_sync( 0xffffffffu, v[1][s], src );
            const double x  = second ? a1 : a0;
            m[s]            = p == 0 ? x : m[s] + x;
        }
    }
    double sq = 0.0;
    if( lane < nTj ) {
#pragma unroll
        for( int s = 0; s < NS; ++s ) {
            const double d       = m[s] - uh[s * P.nT + lane];
            ms[s * P.nT + lane]  = m[s];
            gout[s * nTj + lane] = d;
            sq += d * d;
        }
    }
    return sq;
}

// Trial gradient of the chord kernel (closure.cpp:234-253): lane i sums
// m(s, i) = sum_k uk(s, k) phiWf(k, i) over even and odd nodes as separate
// chains (half the dependent FMA chain of one sum), uk node-major;
// gout[s nTj + i] = m - uh, ms[s nT + i] = m; returns this lane's share of ||gout||^2.
template <int NS>
__device__ __forceinline__ double chord_gradient( const KParams& P, const double* phiWf, const double* uk, const double* uh, int nTj,
                                                  double* gout, double* ms, int lane ) {
    double sq = 0.0;
    for( int i = lane; i < nTj; i += 32 ) {
        double a0[NS], a1[NS];
#pragma unroll
        for( int s = 0; s < NS; ++s ) a0[s] = a1[s] = 0.0;
        const double* t = phiWf + i;
        int k           = 0;
        for( ; k + 1 < P.nQ; k += 2, t += 2 * P.ld ) {
            const double w0 = t[0], w1 = t[P.ld];
            double v0[NS], v1[NS];
            load_node<NS>( uk, k, v0 );
            load_node<NS>( uk, k + 1, v1 );
#pragma unroll
            for( int s = 0; s < NS; ++s ) {
                a0[s] = fma( v0[s], w0, a0[s] );
                a1[s] = fma( v1[s], w1, a1[s] );
            }
        }
        if( k < P.nQ ) {
            const double w0 = t[0];
            double v0[NS];
            load_node<NS>( uk, k, v0 );
#pragma unroll
            for( int s = 0; s < NS; ++s ) a0[s] = fma( v0[s], w0, a0[s] );
        }
#pragma unroll
        for( int s = 0; s < NS; ++s ) {
            const double mm   = a0[s] + a1[s];
            const double d    = mm - uh[s * P.nT + i];
            ms[s * P.nT + i]  = mm;
            gout[s * nTj + i] = d;
            sq += d * d;
        }
    }
    return sq;
}

// Chord Newton rounds of the mixed form, step mode. round 0 takes the step's
// active list (cells k_check or the previous k_update found unconverged);
// round r > 0 takes the cells re-factored in round r - 1. A cell whose held
// inverse is missing or stops contracting goes to the re-factor list of this
// round (the last round: to the FP64 fallback list).
template <int CL> __global__ void __launch_bounds__( 512, 1 ) k_chord( KParams P, int round ) {
    constexpr int NS = Closure<CL>::NS;
    extern __shared__ __align__( 16 ) double smem[];
    if( !P.ctl->active ) return;
    const int* inList;
    int nIn;
    if( round == 0 ) {
        int* al;
        unsigned* ac;
        step_list( P, 0, al, ac );
        inList = al;
        nIn    = int( *ac );
    }
    else {
        inList = refactor_list( P, round - 1 );
        nIn    = int( P.ctl->v2Count[round - 1] );
    }
    if( nIn == 0 ) return;
    const bool last = round >= P.v2Rounds;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Grp<32> g{lane, 0};
    const double *phi = P.phi, *phiWf = P.phiWf;
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
        __syncthreads();
    }
    ChordWs w        = chord_carve( base + warp * chord_ws_doubles( NS, P.nT, P.nQ ), NS, P.nT, P.nQ );
    const size_t ldc = size_t( NS ) * P.nT;
    const double eps = P.eps;
    const bool guard = P.newtonMode != 0;
    unsigned long long itSum = 0, lsSum = 0;
    int activeSum = 0, fbSum = 0;
    double dtMin = 1e300;
    int* outList      = last ? P.fallbackList : refactor_list( P, round );
    unsigned* outCnt  = last ? P.fallbackCount : &P.ctl->v2Count[round];
    unsigned* counter = &P.ctl->v2Work[round];
    for( ;; ) {
        int item = 0;
        if( lane == 0 ) item = int( atomicAdd( counter, 1u ) );
        item = __shfl_sync( 0xffffffffu, item, 0 );
        if( item >= nIn ) break;
        const int cell = inList[item];
        if( round > 0 && P.factorLevel[cell] == -2 ) continue;    // not positive definite: in the FP64 list already
        const int lev = int( P.level[cell] ), nTj = P.nTLevel[lev], n = NS * nTj;
        bool bad = false;
        for( int idx = lane; idx < int( ldc ); idx += 32 ) {
            const double a = P.lam[cell * ldc + idx], b = P.u[cell * ldc + idx];
            w.lam[idx] = a;
            w.uh[idx]  = b;
            bad         = bad || !isfinite( a ) || !isfinite( b );
        }
        const double* gs = gslot( P, cell );
        for( int idx = lane; idx < n; idx += 32 ) w.g[idx] = gs[idx];
        double gn = gs[ldc];
        bad       = __any_sync( 0xffffffffu, bad );
        int iters = round == 0 ? 0 : P.chordIters[cell];
        const int iters0 = iters;    // iterations of earlier rounds of this step
        int ls = 0, rc = -1;         // rc: uqc_cell_code once decided
        bool refactor = !bad && P.factorLevel[cell] != nTj;
        bool fresh    = round > 0;    // the inverse was formed at the current duals
        const float* Hinv = P.factorStore + size_t( cell ) * P.factorStride;
        __syncwarp();
        // lamN <- lam + c d (closure.cpp:273-279), Lambda and U at the nodes,
        // the trial gradient (closure.cpp:234-253) and its norm
        auto trial = [&]( double c ) {
#pragma unroll
            for( int s = 0; s < NS; ++s )
                for( int i = lane; i < nTj; i += 32 ) w.lamI[i * NS + s] = w.lam[s * P.nT + i] + c * w.d[s * nTj + i];
            __syncwarp();
            // nodes k0 and k0 + 32 together (a basis function's duals loaded once
            // for both); a lane without a second node repeats its first
            for( int k0 = lane; k0 < P.nQ; k0 += 64 ) {
                const bool two     = k0 + 32 < P.nQ;
                const int k1       = two ? k0 + 32 : k0;
                const double* row0 = phi + size_t( k0 ) * P.ld;
                const double* row1 = phi + size_t( k1 ) * P.ld;
                double L0[NS], L1[NS], y0[NS], y1[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) L0[s] = L1[s] = 0.0;
                for( int i = 0; i < nTj; ++i ) {
                    const double r0 = row0[i], r1 = row1[i];
                    double li[NS];
                    load_node<NS>( w.lamI, i, li );
#pragma unroll
                    for( int s = 0; s < NS; ++s ) {
                        L0[s] = fma( li[s], r0, L0[s] );
                        L1[s] = fma( li[s], r1, L1[s] );
                    }
                }
                Closure<CL>::U( L0, y0, true, P.phys );
                Closure<CL>::U( L1, y1, true, P.phys );
#pragma unroll
                for( int s = 0; s < NS; ++s ) w.uk[k0 * NS + s] = y0[s];
                if( two ) {
#pragma unroll
                    for( int s = 0; s < NS; ++s ) w.uk[k1 * NS + s] = y1[s];
                }
            }
            __syncwarp();
            const double sq = nTj <= 16 ? chord_gradient_split<NS, 4>( P, phiWf, w.uk, w.uh, nTj, w.gN, w.m, lane )
                              : nTj <= 21 ? chord_gradient_split<NS, 3>( P, phiWf, w.uk, w.uh, nTj, w.gN, w.m, lane )
                                          : chord_gradient<NS>( P, phiWf, w.uk, w.uh, nTj, w.gN, w.m, lane );
            return sqrt( group_sum<32>( g, sq, w.red ) );
        };
        if( bad ) {
            rc = UQC_CELL_NONFINITE;    // the FP64 form reports it
        }
        else {
            while( !refactor && rc < 0 ) {
                if( iters >= P.maxIter ) {
                    rc = UQC_CELL_MAX_ITER;
                    break;
                }
                for( int j = lane; j < n; j += 32 ) w.gf[j] = float( w.g[j] );
                __syncwarp();
                chord_direction( Hinv, n, w.gf, w.d, lane );
                __syncwarp();
                ++iters;
                double gnN = trial( -1.0 );
                if( !fresh && !( gnN < gn ) ) {    // no decrease with a held inverse: a new one, same duals
                    refactor = true;
                    break;
                }
                double step = 1.0;
                int refine  = 0;
                bool done   = false;
                while( gn < gnN || ( guard && !isfinite( gnN ) ) ) {
                    step *= 0.5;
                    ++ls;
                    gnN = trial( -step );
                    if( gnN < eps ) {
                        done = true;
                        break;
                    }
                    if( ++refine > 1000 ) {
                        rc = UQC_CELL_LINE_SEARCH;
                        break;
                    }
                }
                if( rc >= 0 ) break;
                // accept: lam <- the trial duals, g <- gN (the gradient at the accepted duals)
#pragma unroll
                for( int s = 0; s < NS; ++s )
                    for( int i = lane; i < nTj; i += 32 ) w.lam[s * P.nT + i] = w.lamI[i * NS + s];
                for( int idx = lane; idx < n; idx += 32 ) w.g[idx] = w.gN[idx];
                __syncwarp();
                if( done || gnN < eps ) {
                    rc = UQC_CELL_CONVERGED;
                    break;
                }
                const bool held = !fresh;
                const double gPrev = gn;
                gn    = gnN;
                fresh = false;
                if( held && gnN > P.chordTheta * gPrev ) refactor = true;    // contracts too slowly: re-factor
            }
        }
        for( int idx = lane; idx < int( ldc ); idx += 32 ) P.lam[cell * ldc + idx] = w.lam[idx];
        if( rc == UQC_CELL_CONVERGED ) {
            if( lane == 0 ) {
                P.status[cell] = rc;
                P.iters[cell]  = iters;
                ++activeSum;
            }
            itSum += iters - iters0;
            lsSum += ls;
            // uk holds U at the accepted duals (the last trial evaluated) and w.m
            // its moment sums, the re-projected moments of momentsolver.cpp:120-124
            const double dloc = cell_epilogue<CL, 32, true>( g, P, phiWf, w.uh, w.uk, cell, lev, nTj, w.red, w.m );
            dtMin             = dloc < dtMin ? dloc : dtMin;
        }
        else if( refactor && !last ) {
            double* gsw = gslot( P, cell );
            for( int idx = lane; idx < n; idx += 32 ) gsw[idx] = w.g[idx];
            if( lane == 0 ) {
                gsw[ldc]              = gn;
                P.chordIters[cell]    = iters;
                outList[atomicAdd( outCnt, 1u )] = cell;
            }
            itSum += iters - iters0;
            lsSum += ls;
        }
        else {
            // the FP64 form continues from the last accepted duals
            if( lane == 0 ) {
                P.fallbackList[atomicAdd( P.fallbackCount, 1u )] = cell;
                ++fbSum;
            }
            itSum += iters - iters0;
            lsSum += ls;
        }
        __syncwarp();
    }
    if( lane == 0 ) {
        if( itSum ) atomicAdd( &P.ctl->newtonIters, itSum );
        if( lsSum ) atomicAdd( &P.ctl->lineSearchTrials, lsSum );
        if( activeSum ) atomicAdd( &P.ctl->activeCells, activeSum );
        if( fbSum ) atomicAdd( &P.ctl->fallbackCells, (unsigned long long)fbSum );
        if( dtMin < 1e300 ) atomic_min_pos_double( &P.ctl->dtBits, dtMin );
    }
}

// ---------------------------------------------------------------- tcgen05 helpers

__device__ __forceinline__ unsigned smem_u32( const void* p ) { return unsigned( __cvta_generic_to_shared( p ) ); }

// Shared-memory matrix descriptor of tcgen05.mma, K-major operand without
// swizzle: core matrices of 8 rows x 16 bytes stored contiguously; lbo = byte
// distance of core matrices adjacent along K, sbo = along M/N; version 1
// (bits 46-47) as the sm_100 format requires.
__device__ __forceinline__ unsigned long long umma_desc( unsigned addr, unsigned lbo, unsigned sbo ) {
    unsigned long long d = 0;
    d |= (unsigned long long)( ( addr >> 4 ) & 0x3FFF );
    d |= (unsigned long long)( ( lbo >> 4 ) & 0x3FFF ) << 16;
    d |= (unsigned long long)( ( sbo >> 4 ) & 0x3FFF ) << 32;
    d |= 1ull << 46;
    return d;
}

// Instruction descriptor, kind::f16: BF16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr unsigned umma_idesc_bf16( int M, int N ) {
    return ( 1u << 4 ) | ( 1u << 7 ) | ( 1u << 10 ) | ( unsigned( N >> 3 ) << 17 ) | ( unsigned( M >> 4 ) << 24 );
}

__device__ __forceinline__ void umma_bf16( unsigned tmem_d, unsigned long long da, unsigned long long db, unsigned idesc, int accumulate ) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"( tmem_d ),
        "l"( da ), "l"( db ), "r"( idesc ), "r"( accumulate ) );
}

__device__ __forceinline__ void umma_commit( unsigned long long* bar ) {
    asm volatile( "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"( smem_u32( bar ) ) : "memory" );
}

__device__ __forceinline__ void mbar_init( unsigned long long* bar, unsigned count ) {
    asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"( smem_u32( bar ) ), "r"( count ) : "memory" );
}

// Waits until the barrier's phase `parity` has completed; gives up after about
// `limitCycles` SM cycles and returns false.
__device__ __forceinline__ bool mbar_wait( unsigned long long* bar, unsigned parity, long long limitCycles ) {
    const unsigned a  = smem_u32( bar );
    const long long t0 = clock64();
    for( ;; ) {
        unsigned ok = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"( ok )
            : "r"( a ), "r"( parity )
            : "memory" );
        if( ok ) return true;
        if( clock64() - t0 > limitCycles ) return false;
    }
}

__device__ __forceinline__ void tc_fence_before() { asm volatile( "tcgen05.fence::before_thread_sync;" ::: "memory" ); }
__device__ __forceinline__ void tc_fence_after() { asm volatile( "tcgen05.fence::after_thread_sync;" ::: "memory" ); }
__device__ __forceinline__ void fence_async_smem() { asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" ); }

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w reads lanes
// 32 (w % 4) .. + 31 at taddr's column).
__device__ __forceinline__ void tmem_ld16( unsigned taddr, float* v ) {
    unsigned r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"( r[0] ), "=r"( r[1] ), "=r"( r[2] ), "=r"( r[3] ), "=r"( r[4] ), "=r"( r[5] ), "=r"( r[6] ), "=r"( r[7] ), "=r"( r[8] ),
          "=r"( r[9] ), "=r"( r[10] ), "=r"( r[11] ), "=r"( r[12] ), "=r"( r[13] ), "=r"( r[14] ), "=r"( r[15] )
        : "r"( taddr ) );
    asm volatile( "tcgen05.wait::ld.sync.aligned;" ::: "memory" );
#pragma unroll
    for( int i = 0; i < 16; ++i ) v[i] = __uint_as_float( r[i] );
}

// Byte offset of element (row, k) of a K-major operand tile without swizzle,
// stored as [K/8 core columns][rows/8 core rows][8 rows][8 BF16 values].
__host__ __device__ inline unsigned umma_kmajor_offset( int row, int k, int rows ) {
    return unsigned( ( ( k >> 3 ) * ( rows >> 3 ) + ( row >> 3 ) ) * 128 + ( row & 7 ) * 16 + ( k & 7 ) * 2 );
}

// ---------------------------------------------------------------- Hessians on the tensor cores

// Shape of the tensor-core Hessian for a configuration (host and device).
struct TcShape {
    int pairs, nPad, kPad, cellsPerTile, tmemCols;
    size_t qBytes, aBytes;    // one BF16 part (high or low) of B = Q and of A = DU
};
__host__ __device__ inline TcShape tc_shape( int nS, int NP, int nT, int nQ ) {
    TcShape s;
    s.pairs        = nT * ( nT + 1 ) / 2;
    s.nPad         = ( s.pairs + 15 ) & ~15;
    s.kPad         = ( nQ + 15 ) & ~15;
    s.cellsPerTile = 128 / NP;
    s.tmemCols     = 32;
    while( s.tmemCols < s.nPad ) s.tmemCols <<= 1;
    s.qBytes = size_t( s.nPad ) * s.kPad * 2;
    s.aBytes = size_t( 128 ) * s.kPad * 2;
    (void)nS;
    return s;
}

// Bytes of dynamic shared memory of k_hess_tc.
__host__ __device__ inline size_t hess_tc_smem( int nS, int NP, int nT, int nQ, int ld ) {
    const TcShape s = tc_shape( nS, NP, nT, nQ );
    return 1024 + 2 * s.qBytes + 2 * s.aBytes + size_t( nQ ) * ld * 8 + size_t( s.cellsPerTile ) * nS * nT * 8 + 64;
}

// Hessians of the cells of re-factor list `round` on the tensor cores:
// persistent CTAs of 256 threads, tiles of cellsPerTile cells. Per tile the
// threads evaluate Lambda and DU at every node of every cell (FP64) and store
// DU in BF16 high and low parts as A rows (cell, block); one thread issues
// Dh Qh + Dh Ql + Dl Qh (three tcgen05.mma per K step of 16 nodes) into the
// FP32 accumulator in tensor memory; the eight warps read it back (warp w:
// lanes 32 (w % 4).., column half w / 4) and write each cell's values as
// raw[p NP + b] (pair p, block b) at the start of the cell's store slot.
// Q (P.qTiles): the two BF16 parts of the constant table in the operand layout.
template <int CL> __global__ void __launch_bounds__( 256, 1 ) k_hess_tc( KParams P, int round ) {
    constexpr int NS = Closure<CL>::NS, NP = Closure<CL>::NP;
    extern __shared__ __align__( 1024 ) unsigned char sm[];
    if( !P.ctl->active ) return;
    const int nIn = int( P.ctl->v2Count[round] );
    if( nIn == 0 ) return;
    const TcShape S  = tc_shape( NS, NP, P.nT, P.nQ );
    unsigned char* b = reinterpret_cast<unsigned char*>( ( reinterpret_cast<size_t>( sm ) + 1023 ) & ~size_t( 1023 ) );
    unsigned char* qh = b;
    unsigned char* ql = qh + S.qBytes;
    unsigned char* ah = ql + S.qBytes;
    unsigned char* al = ah + S.aBytes;
    double* phiS      = reinterpret_cast<double*>( al + S.aBytes );
    double* lamS      = phiS + size_t( P.nQ ) * P.ld;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>( lamS + size_t( S.cellsPerTile ) * NS * P.nT );
    unsigned* tmemBase      = reinterpret_cast<unsigned*>( bar + 1 );
    int* tileInfo           = reinterpret_cast<int*>( tmemBase + 1 );    // [0] tile index, [1] error
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // stage Q (both parts) and phi; zero the A operand (its padding rows and
    // K columns stay zero)
    {
        const uint4* src = reinterpret_cast<const uint4*>( P.qTiles );
        uint4* dst       = reinterpret_cast<uint4*>( qh );
        for( size_t i = threadIdx.x; i < 2 * S.qBytes / 16; i += blockDim.x ) dst[i] = src[i];
        uint4* a = reinterpret_cast<uint4*>( ah );
        for( size_t i = threadIdx.x; i < 2 * S.aBytes / 16; i += blockDim.x ) a[i] = make_uint4( 0, 0, 0, 0 );
        for( size_t i = threadIdx.x; i < size_t( P.nQ ) * P.ld; i += blockDim.x ) phiS[i] = P.phi[i];
    }
    if( threadIdx.x == 0 ) {
        mbar_init( bar, 1 );
        asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
    }
    if( warp == 0 ) {
        asm volatile( "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"( smem_u32( tmemBase ) ), "r"( S.tmemCols ) );
        asm volatile( "tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" );
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem  = *tmemBase;
    const unsigned idesc = umma_idesc_bf16( 128, S.nPad );
    const unsigned lboA = 16 * 128, lboB = unsigned( S.nPad / 8 ) * 128;
    const int kSteps    = S.kPad / 16;
    const size_t ldc    = size_t( NS ) * P.nT;
    const int nTiles    = ( nIn + S.cellsPerTile - 1 ) / S.cellsPerTile;
    const int* list     = refactor_list( P, round );
    unsigned phase      = 0;
    for( ;; ) {
        if( threadIdx.x == 0 ) tileInfo[0] = int( atomicAdd( &P.ctl->v2Work[4 + round], 1u ) );
        __syncthreads();
        const int tile = tileInfo[0];
        if( tile >= nTiles ) break;
        const int c0 = tile * S.cellsPerTile, nc = min( S.cellsPerTile, nIn - c0 );
        for( int idx = threadIdx.x; idx < nc * int( ldc ); idx += blockDim.x ) {
            const int c = idx / int( ldc ), e = idx - c * int( ldc );
            lamS[idx]   = P.lam[size_t( list[c0 + c] ) * ldc + e];
        }
        __syncthreads();
        // A rows (cell c, block b) = DU_b(Lambda_k) at node k, as high + low BF16
        for( int it = threadIdx.x; it < S.cellsPerTile * P.nQ; it += blockDim.x ) {
            const int c = it / P.nQ, k = it - c * P.nQ;
            double y[NP];
            if( c < nc ) {
                const double* lam = lamS + size_t( c ) * ldc;
                const double* row = phiS + size_t( k ) * P.ld;
                double Lk[NS];
#pragma unroll
                for( int s = 0; s < NS; ++s ) Lk[s] = 0.0;
                for( int i = 0; i < P.nT; ++i ) {
                    const double r = row[i];
#pragma unroll
                    for( int s = 0; s < NS; ++s ) Lk[s] = fma( lam[s * P.nT + i], r, Lk[s] );
                }
                Closure<CL>::DU( Lk, y, P.phys );
            }
            else {
#pragma unroll
                for( int p = 0; p < NP; ++p ) y[p] = 0.0;
            }
#pragma unroll
            for( int p = 0; p < NP; ++p ) {
                const __nv_bfloat16 hi = __double2bfloat16( y[p] );
                const __nv_bfloat16 lo = __double2bfloat16( y[p] - double( __bfloat162float( hi ) ) );
                const unsigned off     = umma_kmajor_offset( c * NP + p, k, 128 );
                *reinterpret_cast<__nv_bfloat16*>( ah + off ) = hi;
                *reinterpret_cast<__nv_bfloat16*>( al + off ) = lo;
            }
        }
        fence_async_smem();
        __syncthreads();
        if( threadIdx.x == 0 ) {
            tc_fence_after();
            const unsigned aH = smem_u32( ah ), aL = smem_u32( al ), bH = smem_u32( qh ), bL = smem_u32( ql );
            for( int ks = 0; ks < kSteps; ++ks ) {
                const unsigned oa = unsigned( ks ) * 2 * lboA, ob = unsigned( ks ) * 2 * lboB;
                umma_bf16( tmem, umma_desc( aH + oa, lboA, 128 ), umma_desc( bH + ob, lboB, 128 ), idesc, ks > 0 );
                umma_bf16( tmem, umma_desc( aH + oa, lboA, 128 ), umma_desc( bL + ob, lboB, 128 ), idesc, 1 );
                umma_bf16( tmem, umma_desc( aL + oa, lboA, 128 ), umma_desc( bH + ob, lboB, 128 ), idesc, 1 );
            }
            umma_commit( bar );
        }
        __syncwarp();
        // about a second at the SM clock: far beyond the microseconds a tile takes
        const bool ok = mbar_wait( bar, phase, 2000000000ll );
        phase ^= 1u;
        if( __syncthreads_or( !ok ) ) {
            // the tensor cores did not finish in time: flag the error, give the
            // MMAs in flight another bounded wait, then free tensor memory
            if( threadIdx.x == 0 ) {
                P.ctl->v2Error = 1;
                mbar_wait( bar, phase ^ 1u, 2000000000ll );
            }
            __syncthreads();
            break;
        }
        tc_fence_after();
        // read the accumulator back: thread row m = 32 (warp % 4) + lane = (cell, block)
        const int q = warp & 3, half = warp >> 2;
        const int m = 32 * q + lane, c = m / NP, bk = m - c * NP;
        const int cell = c < nc ? list[c0 + c] : -1;
        float* raw     = cell >= 0 ? P.factorStore + size_t( cell ) * P.factorStride : nullptr;
        const int colBeg = half * ( S.nPad / 2 ) & ~15, colEnd = half ? S.nPad : ( ( S.nPad / 2 ) & ~15 );
        for( int col = colBeg; col < colEnd; col += 16 ) {
            float v[16];
            tmem_ld16( tmem + ( unsigned( 32 * q ) << 16 ) + unsigned( col ), v );
            if( raw ) {
#pragma unroll
                for( int t = 0; t < 16; ++t )
                    if( col + t < S.pairs ) raw[size_t( col + t ) * NP + bk] = v[t];
            }
        }
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if( warp == 0 ) asm volatile( "tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"( tmem ), "r"( S.tmemCols ) );
}

// ---------------------------------------------------------------- inverse of each listed cell's Hessian

__host__ __device__ inline size_t invert_ws_bytes( int n, int nQ, int NP, bool raw ) {
    auto a16       = []( size_t x ) { return ( x + 15 ) & ~size_t( 15 ); };
    const size_t n8 = size_t( hnb( n ) ) * 8;
    size_t b       = a16( hess_doubles( n ) * 4 ) + 2 * a16( n8 * 4 ) + a16( size_t( xpacked( n ) ) * 4 ) + 64;
    if( !raw ) b += a16( size_t( ( NP + 1 ) & ~1 ) * nQ * 4 ) + a16( size_t( 4 ) * nQ * 8 );
    return b;
}

// Per cell (two warps): the Hessian in FP32 block-packed tiles, either from
// the raw pair values k_hess_tc left in the store slot (RAW) or assembled on
// the CUDA cores (hessian_sym, FP32); Cholesky (cholesky_la); the packed
// inverse X = U^-1 (tri_inverse_packed); H^-1 = X X^T written over the slot
// (n x n, row-major, symmetric). A factor that is not positive definite sends
// the cell to the FP64 fallback list (factorLevel -2).
template <int CL, bool RAW> __global__ void __launch_bounds__( 256, 1 ) k_invert( KParams P, int round ) {
    constexpr int NS = Closure<CL>::NS, NP = Closure<CL>::NP;
    extern __shared__ __align__( 16 ) double smem[];
    if( !P.ctl->active ) return;
    const int nIn = int( P.ctl->v2Count[round] );
    if( nIn == 0 ) return;
    const int gid = threadIdx.x >> 6, groups = blockDim.x >> 6;
    Grp<64> g{int( threadIdx.x & 63 ), 1 + gid};
    const int* list  = refactor_list( P, round );
    const size_t ldc = size_t( NS ) * P.nT;
    const int nMax   = NS * P.nT;
    unsigned char* ws = reinterpret_cast<unsigned char*>( smem ) + size_t( gid ) * invert_ws_bytes( nMax, P.nQ, NP, RAW );
    auto a16          = []( size_t x ) { return ( x + 15 ) & ~size_t( 15 ); };
    float* H          = reinterpret_cast<float*>( ws );
    float* D          = reinterpret_cast<float*>( ws + a16( hess_doubles( nMax ) * 4 ) );
    float* Iv         = D + a16( size_t( hnb( nMax ) ) * 8 * 4 ) / 4;
    float* X          = Iv + a16( size_t( hnb( nMax ) ) * 8 * 4 ) / 4;
    int* flag         = reinterpret_cast<int*>( X + a16( size_t( xpacked( nMax ) ) * 4 ) / 4 );
    int* itemS        = flag + 1;
    float* du         = reinterpret_cast<float*>( flag + 16 );
    double* LA        = reinterpret_cast<double*>( reinterpret_cast<unsigned char*>( du ) + a16( size_t( ( NP + 1 ) & ~1 ) * P.nQ * 4 ) );
    for( ;; ) {
        if( g.r == 0 ) *itemS = int( atomicAdd( &P.ctl->v2Work[8 + round], 1u ) );
        g.sync();
        const int item = *itemS;
        g.sync();
        if( item >= nIn ) break;
        const int cell = list[item];
        const int nTj = P.nTLevel[P.level[cell]], n = NS * nTj, nb = hnb( n );
        float* slot   = P.factorStore + size_t( cell ) * P.factorStride;
        if constexpr( RAW ) {
            const int pairs = nTj * ( nTj + 1 ) / 2;
            for( int e = g.r; e < pairs * NP; e += 64 ) {
                const int p = e / NP, bk = e - p * NP;
                int j, i;
                unpack_pair( p, j, i );
                int m = 0, l = 0, q = bk;    // block bk -> (m, l), m <= l, in DU's packed order
                while( q >= NS - m ) {
                    q -= NS - m;
                    ++m;
                }
                l             = m + q;
                const float a = slot[e];
                H[hblk( m * nTj + j, l * nTj + i )] = a;
                if( m < l && j != i ) H[hblk( m * nTj + i, l * nTj + j )] = a;
            }
            if( n & 7 ) {
                const int C = nb - 1;
                for( int e = g.r; e < nb * 64; e += 64 ) {
                    const int R = e >> 6, col = C * 8 + ( ( e >> 3 ) & 7 ), row = R * 8 + ( e & 7 );
                    if( col >= n && row <= col ) H[hblk( row, col )] = row == col ? 1.f : 0.f;
                }
            }
        }
        else {
            for( int idx = g.r; idx < NS * P.nQ; idx += 64 ) {
                const int s = idx / P.nQ, k = idx - s * P.nQ;
                const double* row = P.phi + size_t( k ) * P.ld;
                double a          = 0.0;
                for( int i = 0; i < nTj; ++i ) a = fma( P.lam[cell * ldc + s * P.nT + i], row[i], a );
                LA[idx] = a;
            }
            g.sync();
            hessian_sym<NS, NP, 64, float>( g, P.nQ, P.ld, P.phiF, P.wt, LA, nTj, du, H,
                                           [&]( const double* L, double* y ) { Closure<CL>::DU( L, y, P.phys ); } );
        }
        for( int r = g.r; r < nb * 8; r += 64 ) H[hrhs( nb ) + r] = 0.f;
        g.sync();
        if( cholesky_la<64, float>( g, H, n, D, Iv, flag ) ) {
            if( g.r == 0 ) {
                P.factorLevel[cell] = -2;
                P.fallbackList[atomicAdd( P.fallbackCount, 1u )] = cell;
                atomicAdd( &P.ctl->fallbackCells, 1ull );
            }
            g.sync();
            continue;
        }
        tri_inverse_packed<64, float>( g, H, Iv, n, X );
        // H^-1 (a, b) = sum_{k >= max(a, b)} X(a, k) X(b, k), full rows
        for( int a = 0; a < n; ++a ) {
            const float* xa = X + xrow( a, n ) - a;
            for( int bcol = g.r; bcol < n; bcol += 64 ) {
                const float* xb = X + xrow( bcol, n ) - bcol;
                float s0 = 0.f, s1 = 0.f;
                int k    = a > bcol ? a : bcol;
                for( ; k + 1 < n; k += 2 ) {
                    s0 = fmaf( xa[k], xb[k], s0 );
                    s1 = fmaf( xa[k + 1], xb[k + 1], s1 );
                }
                if( k < n ) s0 = fmaf( xa[k], xb[k], s0 );
                slot[size_t( a ) * n + bcol] = s0 + s1;
            }
        }
        if( g.r == 0 ) P.factorLevel[cell] = nTj;
        g.sync();
    }
}

// ---------------------------------------------------------------- inverse by symmetric sweeps

// Rows of a cell's matrix per warp and columns per lane of k_invert_sweep:
// four warps per cell hold the n x n matrix (n <= 4 SWEEP_RG) in registers,
// warp g rows [SWEEP_RG g, SWEEP_RG (g + 1)), lane l columns l, l + 32, l + 64.
constexpr int SWEEP_RG = 21, SWEEP_CW = 3;

// floats per cell of k_invert_sweep's shared memory: the raw values (rounded
// up to 16 bytes), two pivot-row buffers, two ints; a multiple of 4 floats
__host__ __device__ inline size_t sweep_raw_floats( int pairs, int NP ) { return ( size_t( pairs ) * NP + 3 ) & ~size_t( 3 ); }
// a pivot-row buffer: 32 SWEEP_CW columns (those beyond the matrix hold
// zeros) and the pivot itself at index 32 SWEEP_CW
constexpr int SWEEP_PR = 32 * SWEEP_CW + 4;
// a pivot-column buffer: the same values by row group, SWEEP_PG floats per
// group (SWEEP_RG rounded up to 4), so that a warp reads its rows' column
// values in 16-byte loads
constexpr int SWEEP_PG = ( SWEEP_RG + 3 ) & ~3, SWEEP_PC = 4 * SWEEP_PG;
__host__ __device__ inline size_t sweep_ws_floats( int pairs, int NP ) {
    return sweep_raw_floats( pairs, NP ) + 2 * SWEEP_PR + 2 * SWEEP_PC + 8;
}

// H^-1 of the cells of re-factor list `round` from the raw values k_hess_tc
// left in their store slots, by the sweep operator (Gauss-Jordan on a
// symmetric matrix: sweeping pivot k maps a_kk -> -1/a_kk, a_ik -> a_ik / a_kk,
// a_ij -> a_ij - a_ik a_kj / a_kk; after all n pivots the matrix is -H^-1).
// The matrix stays symmetric, so column k is row k: one warp publishes the
// pivot row in shared memory, one named barrier per pivot, and every thread
// updates its 21 x 3 register block with one FMA per element. No pivoting:
// H is symmetric positive definite, and a pivot that is not positive (FP32
// factor not positive definite) sends the cell to the FP64 fallback list.
template <int CL> __global__ void __launch_bounds__( 512, 1 ) k_invert_sweep( KParams P, int round ) {
    constexpr int NS = Closure<CL>::NS, NP = Closure<CL>::NP;
    constexpr int RG = SWEEP_RG, CW = SWEEP_CW;
    extern __shared__ __align__( 16 ) float fsm[];
    if( !P.ctl->active ) return;
    const int nIn = int( P.ctl->v2Count[round] );
    if( nIn == 0 ) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int cg = warp >> 2, g = warp & 3;    // cell group of the CTA, row group of the warp
    const int nT = P.nT, n = NS * nT, pairs = nT * ( nT + 1 ) / 2;
    float* raw  = fsm + size_t( cg ) * sweep_ws_floats( pairs, NP );
    float* prow = raw + sweep_raw_floats( pairs, NP );    // two pivot-row buffers of SWEEP_PR floats
    float* pcol = prow + 2 * SWEEP_PR;                     // two pivot-column buffers of SWEEP_PC floats
    int* misc   = reinterpret_cast<int*>( pcol + 2 * SWEEP_PC );    // [0] item, [1] not positive definite
    const int bar = 1 + cg, tid = threadIdx.x & 127;
    auto sync = [&]() { asm volatile( "bar.sync %0, 128;" ::"r"( bar ) : "memory" ); };
    const int* list = refactor_list( P, round );
    // decomposition of this thread's columns: c = l nT + i
    int cm[CW], ci[CW];
#pragma unroll
    for( int q = 0; q < CW; ++q ) {
        const int c = lane + 32 * q;
        cm[q]       = c / nT;
        ci[q]       = c - cm[q] * nT;
    }
    for( ;; ) {
        if( tid == 0 ) misc[0] = int( atomicAdd( &P.ctl->v2Work[8 + round], 1u ) );
        sync();
        const int item = misc[0];
        if( item >= nIn ) break;
        const int cell = list[item];
        float* slot    = P.factorStore + size_t( cell ) * P.factorStride;
        for( int e = tid; e < pairs * NP; e += 128 ) raw[e] = slot[e];
        if( tid == 0 ) misc[1] = 0;
        sync();
        // gather: element (r, c), r = m nT + j, c = l nT + i, is block (min, max)
        // of (m, l) at pair (min, max) of (j, i); identity beyond n
        float a[RG][CW];
#pragma unroll
        for( int rr = 0; rr < RG; ++rr ) {
            const int r = RG * g + rr, rm = r / nT, rj = r - rm * nT;
#pragma unroll
            for( int q = 0; q < CW; ++q ) {
                const int c = lane + 32 * q;
                float v     = r == c ? 1.f : 0.f;
                if( r < n && c < n ) {
                    const int lo = min( rm, cm[q] ), hi = max( rm, cm[q] );
                    const int b  = lo * NS - ( lo * ( lo - 1 ) ) / 2 + ( hi - lo );
                    const int pl = min( rj, ci[q] ), ph = max( rj, ci[q] );
                    v            = raw[( ( ph * ( ph + 1 ) ) / 2 + pl ) * NP + b];
                }
                a[rr][q] = v;
            }
        }
        bool bad = false;
        for( int gg = 0; gg < 4; ++gg ) {
#pragma unroll
            for( int rr = 0; rr < RG; ++rr ) {
                const int k = RG * gg + rr;
                if( k >= n ) break;
                float* pr = prow + ( k & 1 ) * SWEEP_PR;
                float* pc = pcol + ( k & 1 ) * SWEEP_PC;
                const int kl = k & 31, kq = k >> 5;
                if( g == gg ) {
                    // the pivot row; at the pivot p - 1 (so that pr[k] / p = 1 - 1/p,
                    // the factor that turns column k into a_ik / p), p itself at the end;
                    // the same values by row group in the column buffer
#pragma unroll
                    for( int q = 0; q < CW; ++q ) {
                        float v = a[rr][q];
                        if( lane == kl && q == kq ) {
                            pr[32 * CW] = v;
                            v -= 1.f;
                        }
                        const int c       = lane + 32 * q;
                        pr[c]             = v;
                        const int cg2     = c / RG;
                        if( cg2 < 4 ) pc[cg2 * SWEEP_PG + ( c - cg2 * RG )] = v;
                    }
                }
                sync();
                const float p    = pr[32 * CW];
                bad              = bad || !( p > 0.f );
                const float pinv = __frcp_rn( p );
                // a_ij -= a_ik a_kj / p (column k: a_ik / p)
                float sv[CW];
#pragma unroll
                for( int q = 0; q < CW; ++q ) sv[q] = pr[lane + 32 * q] * pinv;
                // a_ik of this warp's rows (column k = row k), 16 bytes at a time
                float f[SWEEP_PG];
                const float4* pc4 = reinterpret_cast<const float4*>( pc + g * SWEEP_PG );
#pragma unroll
                for( int v4 = 0; v4 < SWEEP_PG / 4; ++v4 ) {
                    const float4 x = pc4[v4];
                    f[4 * v4]      = x.x;
                    f[4 * v4 + 1]  = x.y;
                    f[4 * v4 + 2]  = x.z;
                    f[4 * v4 + 3]  = x.w;
                }
#pragma unroll
                for( int rr2 = 0; rr2 < RG; ++rr2 ) {
#pragma unroll
                    for( int q = 0; q < CW; ++q ) a[rr2][q] = fmaf( -f[rr2], sv[q], a[rr2][q] );
                }
                if( g == gg ) {    // the pivot row: a_kj / p, and -1/p at the pivot
#pragma unroll
                    for( int q = 0; q < CW; ++q ) a[rr][q] = ( lane == kl && q == kq ) ? sv[q] - 1.f : sv[q];
                }
            }
        }
        if( bad ) misc[1] = 1;
        sync();
        if( misc[1] ) {
            if( tid == 0 ) {
                P.factorLevel[cell] = -2;
                P.fallbackList[atomicAdd( P.fallbackCount, 1u )] = cell;
                atomicAdd( &P.ctl->fallbackCells, 1ull );
            }
        }
        else {
            // H^-1 = -(the swept matrix), row-major n x n
#pragma unroll
            for( int rr = 0; rr < RG; ++rr ) {
                const int r = RG * g + rr;
                if( r < n ) {
#pragma unroll
                    for( int q = 0; q < CW; ++q ) {
                        const int c = lane + 32 * q;
                        if( c < n ) slot[size_t( r ) * n + c] = -a[rr][q];
                    }
                }
            }
            if( tid == 0 ) P.factorLevel[cell] = nT;
        }
        sync();
    }
}

}    // namespace uqc
