// Per-cell dense linear algebra of the Newton step, for one thread group
// (a warp, or a whole CTA) working on one cell in shared memory.
//
//   hessian_sym   H = sum_k DU(Lambda_k) (x) phi_k phiWf_k^T, upper triangle
//   cholesky_blk  H = U^T U of [H | g] (g appended as column n), blocked
//   back_solve    x = U^-1 y (y = column n after cholesky_blk)
//
// Together they compute posv(H, g) of the reference (vectorspace.cpp:152-171,
// LAPACK dposv with uplo 'U'): a Cholesky factorisation and two triangular
// solves, the forward one fused into the factorisation.
#pragma once
#include <cuda_runtime.h>

namespace uqc {

template <int GROUP> struct Grp {
    int r;
    __device__ __forceinline__ void sync() const {
        if constexpr( GROUP == 32 )
            __syncwarp();
        else
            __syncthreads();
    }
};

// Sum over the group, same value returned to every member. scratch: >= GROUP/32 doubles.
template <int GROUP> __device__ double group_sum( const Grp<GROUP>& g, double v, double* scratch ) {
    for( int o = 16; o > 0; o >>= 1 ) v += __shfl_xor_sync( 0xffffffffu, v, o );
    if constexpr( GROUP == 32 ) {
        return v;
    }
    else {
        if( ( g.r & 31 ) == 0 ) scratch[g.r >> 5] = v;
        g.sync();
        double s = 0.0;
        for( int w = 0; w < GROUP / 32; ++w ) s += scratch[w];
        g.sync();
        return s;
    }
}

template <int GROUP> __device__ double group_min( const Grp<GROUP>& g, double v, double* scratch ) {
    for( int o = 16; o > 0; o >>= 1 ) v = fmin( v, __shfl_xor_sync( 0xffffffffu, v, o ) );
    if constexpr( GROUP == 32 ) {
        return v;
    }
    else {
        if( ( g.r & 31 ) == 0 ) scratch[g.r >> 5] = v;
        g.sync();
        double s = scratch[0];
        for( int w = 1; w < GROUP / 32; ++w ) s = fmin( s, scratch[w] );
        g.sync();
        return s;
    }
}

// Row stride of the full Hessian storage for n unknowns plus one right-hand
// side: odd, so that a warp reading a row of the column-major matrix hits 32
// different banks.
__host__ __device__ inline int hess_ld( int n ) { return ( ( n + 1 ) & 1 ) ? n + 1 : n + 2; }
__host__ __device__ inline size_t hess_doubles( int n ) { return size_t( hess_ld( n ) ) * ( n + 1 ); }

// Upper-triangular pair index e -> (j, i), j <= i, column-major packed order.
__device__ __forceinline__ void unpack_pair( int e, int& j, int& i ) {
    int c = int( ( sqrtf( 8.0f * float( e ) + 1.0f ) - 1.0f ) * 0.5f );
    while( c * ( c + 1 ) / 2 > e ) --c;
    while( ( c + 1 ) * ( c + 2 ) / 2 <= e ) ++c;
    i = c;
    j = e - c * ( c + 1 ) / 2;
}

// Hessian of the dual problem (closure.cpp:255-271): block (m, l) of H is
// sum_k phi(k, .) phiWf(k, .)^T DU(l, m)(Lambda_k). With phiWf(k, i) =
// phi(k, i) wt_k (wt_k = w_k / 2^dimXi, an exact identity in binary floating
// point) every block is phi^T diag(wt DU_lm) phi: symmetric, and the product
// phi(k,j) phi(k,i) is shared by all NS(NS+1)/2 blocks. One thread owns a pair
// j <= i and accumulates it for every block; off-diagonal blocks are mirrored.
// du (NP x nQ) receives wt_k DU(Lambda_k). Writes the upper triangle of H
// (column-major, row stride ldH); the lower triangle is never read.
template <int NS, int NP, int GROUP, class DUF>
__device__ void hessian_sym( const Grp<GROUP>& g, int nQ, int ld, const double* phi, const double* wt, const double* L, int nTj, double* du,
                             double* H, int ldH, DUF&& duf ) {
    for( int k = g.r; k < nQ; k += GROUP ) {
        double Lk[NS], y[NP];
#pragma unroll
        for( int s = 0; s < NS; ++s ) Lk[s] = L[s * nQ + k];
        duf( Lk, y );
        const double w = wt[k];
#pragma unroll
        for( int p = 0; p < NP; ++p ) du[p * nQ + k] = w * y[p];
    }
    g.sync();
    const int pairs = nTj * ( nTj + 1 ) / 2;
    for( int e = g.r; e < pairs; e += GROUP ) {
        int j, i;
        unpack_pair( e, j, i );
        double acc[NP];
#pragma unroll
        for( int p = 0; p < NP; ++p ) acc[p] = 0.0;
        const double* pj = phi + j;
        const double* pi = phi + i;
        for( int k = 0; k < nQ; ++k ) {
            const double prod = pj[size_t( k ) * ld] * pi[size_t( k ) * ld];
#pragma unroll
            for( int p = 0; p < NP; ++p ) acc[p] = fma( prod, du[p * nQ + k], acc[p] );
        }
        int p = 0;
#pragma unroll
        for( int m = 0; m < NS; ++m )
#pragma unroll
            for( int l = m; l < NS; ++l, ++p ) {
                const int row = m * nTj + j, col = l * nTj + i;
                H[size_t( col ) * ldH + row] = acc[p];
                if( m < l && j != i ) H[size_t( l * nTj + j ) * ldH + ( m * nTj + i )] = acc[p];
            }
    }
}

// Blocked right-looking Cholesky of the n x n upper-stored matrix with the
// right-hand side in column n: on return the upper triangle holds U (U^T U =
// H), column n holds y = U^-T b, D[j] = U(j,j), I[j] = 1/U(j,j). Per panel of
// B columns: (1) one warp factors the diagonal block, (2) the panel rows are
// solved column by column (one thread per column, right-hand side included),
// (3) the trailing upper triangle (and right-hand side) is updated with 2 x 2
// register tiles. Three group barriers per panel. Returns 0, or j + 1 for the
// first pivot that is not positive (posv's info > 0). flag: one int in shared
// memory.
template <int GROUP, class T>
__device__ int cholesky_blk( const Grp<GROUP>& g, T* H, int ldH, int n, T* D, T* I, int* flag ) {
    constexpr int B = 8;
    if( g.r == 0 ) *flag = 0;
    g.sync();
    for( int j0 = 0; j0 < n; j0 += B ) {
        const int jb = n - j0 < B ? n - j0 : B;
        // (1) diagonal block, warp 0
        if( g.r < 32 ) {
            const int lane = g.r;
            for( int jj = 0; jj < jb; ++jj ) {
                const int j = j0 + jj;
                const T a   = H[size_t( j ) * ldH + j];
                if( !( a > T( 0 ) ) ) {
                    if( lane == 0 ) *flag = j + 1;
                    break;
                }
                const T d = sqrt( a ), inv = T( 1 ) / d;
                const int c = j + 1 + lane;
                if( c < j0 + jb ) H[size_t( c ) * ldH + j] *= inv;
                if( lane == 0 ) {
                    H[size_t( j ) * ldH + j] = d;
                    D[j]                     = d;
                    I[j]                     = inv;
                }
                __syncwarp();
                // rank-1 update of the rest of the diagonal block: (r, c), j < r <= c < j0 + jb
                const int m = j0 + jb - j - 1, cnt = m * ( m + 1 ) / 2;
                for( int e = lane; e < cnt; e += 32 ) {
                    int rr, cc;
                    unpack_pair( e, rr, cc );
                    const int r = j + 1 + rr, c2 = j + 1 + cc;
                    H[size_t( c2 ) * ldH + r] -= H[size_t( r ) * ldH + j] * H[size_t( c2 ) * ldH + j];
                }
                __syncwarp();
            }
        }
        g.sync();
        if( *flag ) return *flag;
        // (2) panel rows: U(J, c) = U_JJ^-T A(J, c) for c in [j0 + jb, n]
        const int s = j0 + jb;
        for( int c = s + g.r; c <= n; c += GROUP ) {
            T x[B];
#pragma unroll
            for( int jj = 0; jj < B; ++jj ) {
                if( jj < jb ) {
                    const int j = j0 + jj;
                    T v         = H[size_t( c ) * ldH + j];
#pragma unroll
                    for( int kk = 0; kk < B; ++kk )
                        if( kk < jj ) v -= H[size_t( j ) * ldH + j0 + kk] * x[kk];
                    x[jj]                    = v * I[j];
                    H[size_t( c ) * ldH + j] = x[jj];
                }
            }
        }
        g.sync();
        // (3) trailing update: A(r, c) -= sum_{k in J} U(k, r) U(k, c), s <= r <= c, r < n, c <= n
        const int m = n - s;    // trailing rows
        if( m > 0 ) {
            const int mt = ( m + 2 ) / 2;    // column tiles over m + 1 columns
            const int tiles = mt * ( mt + 1 ) / 2;
            for( int t = g.r; t < tiles; t += GROUP ) {
                int tr, tc;
                unpack_pair( t, tr, tc );
                const int r0 = s + 2 * tr, c0 = s + 2 * tc;
                if( r0 >= n ) continue;
                const int r1 = r0 + 1 < n ? r0 + 1 : r0, c1 = c0 + 1 <= n ? c0 + 1 : c0;
                T a00 = 0, a01 = 0, a10 = 0, a11 = 0;
#pragma unroll
                for( int kk = 0; kk < B; ++kk ) {
                    if( kk < jb ) {
                        const int k = j0 + kk;
                        const T u0 = H[size_t( r0 ) * ldH + k], u1 = H[size_t( r1 ) * ldH + k];
                        const T v0 = H[size_t( c0 ) * ldH + k], v1 = H[size_t( c1 ) * ldH + k];
                        a00 += u0 * v0;
                        a01 += u0 * v1;
                        a10 += u1 * v0;
                        a11 += u1 * v1;
                    }
                }
                H[size_t( c0 ) * ldH + r0] -= a00;
                if( c1 != c0 ) H[size_t( c1 ) * ldH + r0] -= a01;
                if( r1 != r0 && r1 <= c0 ) H[size_t( c0 ) * ldH + r1] -= a10;
                if( r1 != r0 && c1 != c0 ) H[size_t( c1 ) * ldH + r1] -= a11;
            }
        }
        g.sync();
    }
    return 0;
}

// Back substitution U x = y by one warp (y in column n of H, LAPACK dtrsm
// 'Left','Upper','No transpose' order), x written to out[0..n).
template <int GROUP, class T> __device__ void back_solve( const Grp<GROUP>& g, const T* H, int ldH, int n, const T* I, double* out ) {
    if( g.r >= 32 ) return;
    const int lane     = g.r;
    constexpr int MAXR = 8;    // rows per lane: n <= 256
    T y[MAXR];
#pragma unroll
    for( int q = 0; q < MAXR; ++q ) y[q] = ( lane + 32 * q < n ) ? H[size_t( n ) * ldH + lane + 32 * q] : T( 0 );
    for( int k = n - 1; k >= 0; --k ) {
        T xk     = 0;
        const int own = k & 31, q0 = k >> 5;
#pragma unroll
        for( int q = 0; q < MAXR; ++q )
            if( q == q0 && lane == own ) {
                if( y[q] != T( 0 ) ) y[q] = y[q] * I[k];
                xk = y[q];
            }
        xk = __shfl_sync( 0xffffffffu, xk, own );
        if( xk != T( 0 ) ) {
            const T* col = H + size_t( k ) * ldH;
#pragma unroll
            for( int q = 0; q < MAXR; ++q ) {
                const int r = lane + 32 * q;
                if( r < k ) y[q] = y[q] - xk * col[r];
            }
        }
    }
#pragma unroll
    for( int q = 0; q < MAXR; ++q )
        if( lane + 32 * q < n ) out[lane + 32 * q] = double( y[q] );
}

}    // namespace uqc
