// Per-cell dense linear algebra of the Newton step, for one thread group
// (a warp, two warps, or a whole CTA) working on one cell in shared memory.
//
//   hessian_sym       H = sum_k DU(Lambda_k) (x) phi_k phiWf_k^T, upper triangle
//   cholesky_la       H = U^T U, right-hand side appended, by 8 x 8 tiles with
//                     look-ahead (one group barrier per tile column)
//   back_solve_warp   x = U^-1 y
//
// Together they compute posv(H, g) of the reference (vectorspace.cpp:152-171,
// LAPACK dposv with uplo 'U'): a Cholesky factorisation and two triangular
// solves, the forward one fused into the factorisation.
//
// Storage ("block-packed upper"): the n x n matrix is padded to nb = ceil(n/8)
// tiles of 8 x 8, the padding being the identity, so every tile is full. Only
// tiles (R, C) with R <= C are stored, in column-major tile order; inside a
// tile, element (k, c) sits at 8 c + (k ^ c): column-major with the row index
// XOR-swizzled by the column, so that both a tile column and a tile row read
// by eight lanes fall in distinct shared-memory banks. The right-hand side
// follows as nb segments of 8.
#pragma once
#include <cuda_runtime.h>

namespace uqc {

// Optional cycle counters of the closure kernel (diagnostic builds compiled
// with -DUQC_PHASE_TIMERS): slots 0-7 are phases of the Newton step, 8-15
// parts of the factorisation (8 critical warp, 9 trailing warp, 10 barrier
// wait of the critical warp, 11 barrier wait of a trailing warp, 12 tile
// factor, 13 tile inverse, 14 tile-row update, 15 panel solve), 16-20 parts
// of the check kernel (load, Lambda and U, gradient sums, epilogue, cell).
#ifdef UQC_PHASE_TIMERS
__device__ unsigned long long g_phaseCycles[32];
#define CT_BEGIN( v ) long long v = clock64();
#define CT_END( v, id, cond ) \
    if( cond ) atomicAdd( &g_phaseCycles[id], (unsigned long long)( clock64() - v ) );
#else
#define CT_BEGIN( v )
#define CT_END( v, id, cond )
#endif

// A thread group working on one cell: GROUP = 32 (a warp), 64 (two warps,
// several groups per CTA, synchronised by named barrier `bar`) or the CTA.
template <int GROUP> struct Grp {
    int r;      // rank in the group
    int bar;    // named barrier id (GROUP == 64)
    __device__ __forceinline__ void sync() const {
        if constexpr( GROUP == 32 )
            __syncwarp();
        else if constexpr( GROUP == 64 )
            asm volatile( "bar.sync %0, 64;" ::"r"( bar ) : "memory" );
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

template <int GROUP> __device__ bool group_any( const Grp<GROUP>& g, bool v, double* scratch ) {
    bool w = __any_sync( 0xffffffffu, v );
    if constexpr( GROUP == 32 ) {
        return w;
    }
    else {
        if( ( g.r & 31 ) == 0 ) scratch[g.r >> 5] = w ? 1.0 : 0.0;
        g.sync();
        bool any = false;
        for( int i = 0; i < GROUP / 32; ++i ) any = any || scratch[i] != 0.0;
        g.sync();
        return any;
    }
}

// 1/sqrt(a) for a > 0 on the Cholesky critical path: the single-precision
// hardware estimate (relative error below 2^-22) refined by one Newton-Raphson
// step for f(y) = 1/y^2 - a, y <- y (3 - a y^2) / 2, which squares the relative
// error (below 2^-43, about 1e-13: the pivots, and through them the Newton
// direction, are exact to far below the closure tolerance; convergence is
// decided by the FP64 gradient). Arguments beyond single-precision range use
// rsqrt().
__device__ __forceinline__ double rsqrt_nr( double a ) {
    if( !( a > 1e-30 && a < 1e30 ) ) return rsqrt( a );
    const double y = double( rsqrtf( float( a ) ) );
    return y * fma( -0.5 * a * y, y, 1.5 );
}
__device__ __forceinline__ float rsqrt_nr( float a ) { return rsqrtf( a ); }

// ---- block-packed storage
__host__ __device__ inline int hnb( int n ) { return ( n + 7 ) >> 3; }
__host__ __device__ inline size_t hess_doubles( int n ) {
    const size_t nb = size_t( hnb( n ) );
    return nb * ( nb + 1 ) / 2 * 64 + nb * 8;
}
// in-tile offset of element (row k, column c)
__device__ __forceinline__ int tix( int k, int c ) { return ( c << 3 ) | ( k ^ c ); }
__device__ __forceinline__ int htile( int R, int C ) { return ( ( ( C * ( C + 1 ) ) >> 1 ) + R ) * 64; }
// offset of element (r, c), tile row r/8 <= tile column c/8
__device__ __forceinline__ int hblk( int r, int c ) { return htile( r >> 3, c >> 3 ) + tix( r & 7, c & 7 ); }
__device__ __forceinline__ int hrhs( int nb ) { return ( ( nb * ( nb + 1 ) ) >> 1 ) * 64; }

// Upper-triangular pair index e -> (j, i), j <= i, column-major packed order.
__device__ __forceinline__ void unpack_pair( int e, int& j, int& i ) {
    int c = int( ( sqrtf( 8.0f * float( e ) + 1.0f ) - 1.0f ) * 0.5f );
    while( c * ( c + 1 ) / 2 > e ) --c;
    while( ( c + 1 ) * ( c + 2 ) / 2 <= e ) ++c;
    i = c;
    j = e - c * ( c + 1 ) / 2;
}

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Hessian of the dual problem (closure.cpp:255-271): block (m, l) of H is
// sum_k phi(k, .) phiWf(k, .)^T DU(l, m)(Lambda_k). With phiWf(k, i) =
// phi(k, i) wt_k (wt_k = w_k / 2^dimXi, an exact identity in binary floating
// point) every block is phi^T diag(wt DU_lm) phi: symmetric, and the product
// phi(k,j) phi(k,i) is shared by all NS(NS+1)/2 blocks. A thread owns the two
// pairs (j, i0) and (j, i0 + 1), i0 even, j <= i0 + 1, and accumulates them for
// every block; off-diagonal blocks are mirrored. du (nQ x np_pad(NP), node-
// major) receives wt_k DU(Lambda_k). Writes the upper triangle of H and the
// identity padding (the right-hand side is written by the caller). T = double
// (FP64 form) or float (mixed form: DU evaluated in FP64 and rounded, products
// and sums in FP32, phi the FP32 copy of the table).
template <int NS, int NP, int GROUP, class T, class DUF>
__device__ void hessian_sym( const Grp<GROUP>& g, int nQ, int ld, const T* phi, const double* wt, const double* L, int nTj, T* du, T* H,
                             DUF&& duf ) {
    constexpr int NPP = ( NP + 1 ) & ~1;    // node-major DU rows padded to pairs
    using V2          = typename Vec2<T>::type;
    const int n = NS * nTj, nb = hnb( n );
    for( int k = g.r; k < nQ; k += GROUP ) {
        double Lk[NS], y[NP];
#pragma unroll
        for( int s = 0; s < NS; ++s ) Lk[s] = L[s * nQ + k];
        duf( Lk, y );
        const double w = wt[k];
#pragma unroll
        for( int p = 0; p < NPP; ++p ) du[k * NPP + p] = p < NP ? T( w * y[p] ) : T( 0 );
    }
    // identity padding of the last tile column (rows and columns >= n) and of the right-hand side
    if( n & 7 ) {
        const int C = nb - 1;
        for( int e = g.r; e < nb * 64; e += GROUP ) {
            const int R = e >> 6, col = C * 8 + ( ( e >> 3 ) & 7 ), row = R * 8 + ( e & 7 );
            if( col >= n && row <= col ) H[hblk( row, col )] = row == col ? T( 1 ) : T( 0 );
        }
        for( int r = n + g.r; r < nb * 8; r += GROUP ) H[hrhs( nb ) + r] = T( 0 );
    }
    g.sync();
    // pair blocks: i-pair q (i0 = 2q) has min(2q + 2, nTj) values of j
    const int nq = ( nTj + 1 ) >> 1, last = nq - 1;
    const int blocks = last * ( last + 1 ) + ( 2 * last + 2 < nTj ? 2 * last + 2 : nTj );
    for( int b = g.r; b < blocks; b += GROUP ) {
        int q = int( ( sqrtf( 4.0f * float( b ) + 1.0f ) - 1.0f ) * 0.5f );
        while( q * ( q + 1 ) > b ) --q;
        while( ( q + 1 ) * ( q + 2 ) <= b ) ++q;
        const int j = b - q * ( q + 1 ), i0 = 2 * q;
        T acc0[NPP], acc1[NPP];
#pragma unroll
        for( int p = 0; p < NPP; ++p ) acc0[p] = acc1[p] = T( 0 );
        const T* rowp = phi;
        for( int k = 0; k < nQ; ++k, rowp += ld ) {
            const T pj = rowp[j], prod0 = pj * rowp[i0], prod1 = pj * rowp[i0 + 1];
            const V2* d2 = reinterpret_cast<const V2*>( du + k * NPP );
#pragma unroll
            for( int p = 0; p < NPP / 2; ++p ) {
                const V2 v      = d2[p];
                acc0[2 * p]     = fma( prod0, v.x, acc0[2 * p] );
                acc0[2 * p + 1] = fma( prod0, v.y, acc0[2 * p + 1] );
                acc1[2 * p]     = fma( prod1, v.x, acc1[2 * p] );
                acc1[2 * p + 1] = fma( prod1, v.y, acc1[2 * p + 1] );
            }
        }
#pragma unroll
        for( int h = 0; h < 2; ++h ) {
            const int i = i0 + h;
            if( j > i || i >= nTj ) continue;
            int p = 0;
#pragma unroll
            for( int m = 0; m < NS; ++m )
#pragma unroll
                for( int l = m; l < NS; ++l, ++p ) {
                    const T a = h ? acc1[p] : acc0[p];
                    H[hblk( m * nTj + j, l * nTj + i )] = a;
                    if( m < l && j != i ) H[hblk( m * nTj + i, l * nTj + j )] = a;
                }
        }
    }
}

// ---- tile kernels of the factorisation; `lane` of one warp

// One thread: Cholesky of the (updated) diagonal tile in registers. Writes
// U_JJ over its upper triangle, D = diag(U), I = 1/diag(U); sets *flag to
// j0 + jj + 1 at the first pivot that is not positive.
template <class T> __device__ void tile_factor( T* DT, T* D, T* I, int j0, int* flag ) {
    double a[8][8];
#pragma unroll
    for( int r = 0; r < 8; ++r )
#pragma unroll
        for( int c = r; c < 8; ++c ) a[r][c] = DT[tix( r, c )];
    int bad = 0;
#pragma unroll
    for( int jj = 0; jj < 8; ++jj ) {
        if( !bad ) {
            const double ajj = a[jj][jj];
            if( !( ajj > 0.0 ) ) {
                bad = j0 + jj + 1;
            }
            else {
                const double inv = rsqrt_nr( ajj ), d = ajj * inv;
                a[jj][jj]        = d;
                D[j0 + jj]       = T( d );
                I[j0 + jj]       = T( inv );
#pragma unroll
                for( int c = jj + 1; c < 8; ++c ) a[jj][c] *= inv;
#pragma unroll
                for( int r = jj + 1; r < 8; ++r )
#pragma unroll
                    for( int c = r; c < 8; ++c ) a[r][c] -= a[jj][r] * a[jj][c];
            }
        }
    }
    if( bad ) *flag = bad;
#pragma unroll
    for( int r = 0; r < 8; ++r )
#pragma unroll
        for( int c = r; c < 8; ++c ) DT[tix( r, c )] = T( a[r][c] );
}

// Lanes 0..7: row i of X = U_JJ^-1 (upper triangular) into the strictly lower
// half of the diagonal tile, X(i, c) at element (c, i):
// X(i,i) = I[i], X(i,c) = -I[c] sum_{k=i}^{c-1} X(i,k) U(k,c). The strictly
// upper part of U and I are read into registers first (the stores go to the
// lower half), so the chain is FMA latency only.
template <class T> __device__ void tile_inverse( T* DT, const T* I, int j0, int lane ) {
    if( lane >= 8 ) return;
    const int i = lane;
    T u[8][8], iv[8];
#pragma unroll
    for( int c = 1; c < 8; ++c )
#pragma unroll
        for( int k = 0; k < c; ++k ) u[k][c] = DT[tix( k, c )];
#pragma unroll
    for( int c = 0; c < 8; ++c ) iv[c] = I[j0 + c];
    T x[8];
#pragma unroll
    for( int c = 0; c < 8; ++c ) x[c] = c == i ? iv[c] : T( 0 );
#pragma unroll
    for( int c = 1; c < 8; ++c ) {
        T s = 0;
#pragma unroll
        for( int k = 0; k < c; ++k ) s = fma( x[k], u[k][c], s );    // x[k] = 0 for k < i
        if( c > i ) x[c] = -s * iv[c];
    }
#pragma unroll
    for( int c = 1; c < 8; ++c )
        if( c > i ) DT[tix( c, i )] = x[c];
}

// D = A B + C on the FP64 tensor cores, one 8 x 8 x 4 product per warp
// (mma.sync m8n8k4, A row-major 8 x 4, B column-major 4 x 8). Lane 4 g + t
// holds a = A(g, t), b = B(t, g), c0 = C(g, 2t), c1 = C(g, 2t + 1).
__device__ __forceinline__ void dmma_8x8x4( double& c0, double& c1, double a, double b ) {
    asm( "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n" : "+d"( c0 ), "+d"( c1 ) : "d"( a ), "d"( b ) );
}

// Tile (R, C) -= U(J, R)^T U(J, C) on the FP64 tensor cores: two mma k-steps
// with A(g, t) = -U(J, R)(t, g), B(t, g) = U(J, C)(t, g), C = the tile; one
// shared-memory value per lane and operand per k-step. T = double, or float
// (mixed form: FP32 storage, FP64 products).
template <class T> __device__ __forceinline__ void tile_update_mma( T* H, int J, int R, int C, int lane ) {
    const int g = lane >> 2, t = lane & 3;
    const T* A      = H + htile( J, R );
    const T* B      = H + htile( J, C );
    T* O            = H + htile( R, C );
    const double a0 = -double( A[tix( t, g )] ), a1 = -double( A[tix( t + 4, g )] );
    const double b0 = B[tix( t, g )], b1 = B[tix( t + 4, g )];
    double c0 = O[tix( g, 2 * t )], c1 = O[tix( g, 2 * t + 1 )];
    dmma_8x8x4( c0, c1, a0, b0 );
    dmma_8x8x4( c0, c1, a1, b1 );
    O[tix( g, 2 * t )]     = T( c0 );
    O[tix( g, 2 * t + 1 )] = T( c1 );
}

// Panel of tile row J on the FP64 tensor cores: U(J, C) = X^T A(J, C) with
// A(g, t) = X(t, g) (the stored inverse; X^T is lower triangular), B(t, g) =
// A(J, C)(t, g). The right-hand side segment by lanes 0..7.
template <class T> __device__ void tile_row_solve_mma( T* H, int J, int nb, const T* I, int lane ) {
    const int g = lane >> 2, t = lane & 3;
    const T* DT = H + htile( J, J );
    auto xt     = [&]( int k ) { return k < g ? double( DT[tix( g, k )] ) : ( k == g ? double( I[J * 8 + g] ) : 0.0 ); };    // X(k, g)
    const double a0 = xt( t ), a1 = xt( t + 4 );
    for( int C = J + 1; C < nb; ++C ) {
        T* A            = H + htile( J, C );
        const double b0 = A[tix( t, g )], b1 = A[tix( t + 4, g )];
        double c0 = 0.0, c1 = 0.0;
        dmma_8x8x4( c0, c1, a0, b0 );
        dmma_8x8x4( c0, c1, a1, b1 );
        A[tix( g, 2 * t )]     = T( c0 );
        A[tix( g, 2 * t + 1 )] = T( c1 );
    }
    T* b     = H + hrhs( nb ) + J * 8;
    double y = 0.0;
    if( lane < 8 ) {
#pragma unroll
        for( int k = 0; k < 8; ++k )
            y += ( k < lane ? double( DT[tix( lane, k )] ) : ( k == lane ? double( I[J * 8 + lane] ) : 0.0 ) ) * double( b[k] );
    }
    __syncwarp();
    if( lane < 8 ) b[lane] = T( y );
}

// Right-hand side segment R -= U(J, R)^T y_J (lanes 0..7).
template <class T> __device__ __forceinline__ void rhs_update( T* H, int J, int R, int nb, int lane ) {
    if( lane >= 8 ) return;
    const T* A  = H + htile( J, R );
    const T* yJ = H + hrhs( nb ) + J * 8;
    T s         = 0;
#pragma unroll
    for( int k = 0; k < 8; ++k ) s += A[tix( k, lane )] * yJ[k];
    H[hrhs( nb ) + R * 8 + lane] -= s;
}

// Blocked right-looking Cholesky H = U^T U with look-ahead, right-hand side b
// appended (y = U^-T b in its place). Per tile column J one warp (warp 0)
// carries the critical path: it applies row J's update to tile row J + 1,
// factors and inverts the diagonal tile J + 1 and solves tile row J + 1 (the
// panel); meanwhile the other warps (all of the group's warps but warp 0, or
// warp 0 itself afterwards when the group is one warp) apply row J's update
// to the trailing tiles (R, C), J + 2 <= R <= C, and right-hand side segments.
// One group barrier per tile column. On return the upper tiles hold U, D[j] =
// U(j,j), I[j] = 1/U(j,j) (padded to 8 nb entries), and the strictly lower
// half of each diagonal tile holds the transposed inverse of its U block.
// Returns 0, or j + 1 for the first pivot that is not positive (posv's
// info > 0). flag: one int in shared memory.
template <int GROUP, class T>
__device__ int cholesky_la( const Grp<GROUP>& g, T* H, int n, T* D, T* I, int* flag ) {
    constexpr int W = GROUP / 32;
    const int nb = hnb( n ), warp = g.r >> 5, lane = g.r & 31;
    if( warp == 0 ) {
        if( lane == 0 ) {
            *flag = 0;
            tile_factor<T>( H, D, I, 0, flag );
        }
        __syncwarp();
        tile_inverse<T>( H, I, 0, lane );
        __syncwarp();
        if( !*flag ) tile_row_solve_mma<T>( H, 0, nb, I, lane );
    }
    g.sync();
    if( *flag ) return *flag;
    for( int J = 0; J + 1 < nb; ++J ) {
        const int K = J + 1;
        CT_BEGIN( tc );
        if( warp == 0 ) {
            CT_BEGIN( t0 );
            for( int C = K; C < nb; ++C ) tile_update_mma<T>( H, J, K, C, lane );
            rhs_update<T>( H, J, K, nb, lane );
            __syncwarp();
            CT_END( t0, 14, g.r == 0 );
            CT_BEGIN( t1 );
            if( lane == 0 ) tile_factor<T>( H + htile( K, K ), D, I, K * 8, flag );
            __syncwarp();
            CT_END( t1, 12, g.r == 0 );
            CT_BEGIN( t2 );
            tile_inverse<T>( H + htile( K, K ), I, K * 8, lane );
            __syncwarp();
            CT_END( t2, 13, g.r == 0 );
            CT_BEGIN( t3 );
            if( !*flag ) tile_row_solve_mma<T>( H, K, nb, I, lane );
            CT_END( t3, 15, g.r == 0 );
        }
        CT_END( tc, 8, g.r == 0 );
        CT_BEGIN( tw );
        if( W == 1 || warp > 0 ) {
            const int worker = W == 1 ? 0 : warp - 1, workers = W == 1 ? 1 : W - 1;
            if( W == 1 ) __syncwarp();
            // items: tiles (R, C), J + 2 <= R <= C, then rhs segments
            for( int R = J + 2, e = 0; R < nb; ++R ) {
                for( int C = R; C < nb; ++C, ++e )
                    if( e % workers == worker ) tile_update_mma<T>( H, J, R, C, lane );
            }
            for( int R = J + 2 + worker; R < nb; R += workers ) rhs_update<T>( H, J, R, nb, lane );
        }
        CT_END( tw, 9, g.r == 32 );
        CT_BEGIN( tb );
        g.sync();
        CT_END( tb, 10, g.r == 0 );
        CT_END( tb, 11, g.r == 32 );
        if( *flag ) return *flag;
    }
    return 0;
}

// Forward substitution U^T y = b by warp 0 with a factor that cholesky_la left
// (tiles, tile inverses, I): y_J = X_J^T (b_J - sum_{K < J} U(K, J)^T y_K),
// tile rows first to last; y goes to the right-hand side tiles, where
// back_solve_warp reads it. b: n values (the padding rows are zero).
template <int GROUP, class T>
__device__ void forward_solve_warp( const Grp<GROUP>& g, T* H, int n, const T* I, const double* b ) {
    const int nb = hnb( n ), warp = g.r >> 5, lane = g.r & 31;
    if( warp == 0 ) {
        const int r = lane & 7, q = lane >> 3;
        T* y        = H + hrhs( nb );
        for( int J = 0; J < nb; ++J ) {
            T acc = 0;
            for( int K = 0; K < J; ++K ) {
                const T* A = H + htile( K, J );
#pragma unroll
                for( int kk = q; kk < 8; kk += 4 ) acc += A[tix( kk, r )] * y[K * 8 + kk];
            }
            acc += __shfl_xor_sync( 0xffffffffu, acc, 8 );
            acc += __shfl_xor_sync( 0xffffffffu, acc, 16 );
            const int row = J * 8 + r;
            const T rr    = ( row < n ? T( b[row] ) : T( 0 ) ) - acc;
            const T* DT   = H + htile( J, J );
            T v           = I[J * 8 + r] * rr;
#pragma unroll
            for( int k = 0; k < 7; ++k ) {
                const T rk = __shfl_sync( 0xffffffffu, rr, k );
                if( k < r ) v += DT[tix( r, k )] * rk;
            }
            __syncwarp();
            if( q == 0 ) y[J * 8 + r] = v;
            __syncwarp();
        }
    }
    g.sync();
}

// Back substitution U x = y by warp 0, tile rows last first: r_J = y_J -
// sum_{C > J} U(J, C) x_C (lane (r, q) sums columns q, q + 4 of each tile,
// then two shuffles), x_J = X_J r_J with the stored tile inverse. Only x[0..n)
// is written; the group synchronises at the end.
template <int GROUP, class T>
__device__ void back_solve_warp( const Grp<GROUP>& g, const T* H, int n, const T* I, double* x ) {
    const int nb = hnb( n ), warp = g.r >> 5, lane = g.r & 31;
    if( warp == 0 ) {
        const int r = lane & 7, q = lane >> 3;
        const T* y = H + hrhs( nb );
        for( int J = nb - 1; J >= 0; --J ) {
            T acc = 0;
            for( int C = J + 1; C < nb; ++C ) {
                const T* A = H + htile( J, C );
#pragma unroll
                for( int cc = q; cc < 8; cc += 4 ) {
                    const int c = C * 8 + cc;
                    if( c < n ) acc += A[tix( r, cc )] * T( x[c] );
                }
            }
            acc += __shfl_xor_sync( 0xffffffffu, acc, 8 );
            acc += __shfl_xor_sync( 0xffffffffu, acc, 16 );
            const T rr  = y[J * 8 + r] - acc;
            const T* DT = H + htile( J, J );
            T v         = I[J * 8 + r] * rr;
#pragma unroll
            for( int k = 1; k < 8; ++k ) {
                const T rk = __shfl_sync( 0xffffffffu, rr, k );
                if( k > r ) v += DT[tix( k, r )] * rk;
            }
            if( q == 0 && J * 8 + r < n ) x[J * 8 + r] = double( v );
            __syncwarp();
        }
    }
    g.sync();
}

// ---- explicit inverse of the factor (chord Newton of the mixed form)
//
// X = U^-1 in packed upper-triangular storage, row-major: X(i, j), i <= j,
// at xrow(i, n) + j - i. With it a held-factor direction H^-1 g = X (X^T g)
// is two mat-vecs with independent outputs instead of two triangular solves
// with a dependent chain per tile row.
__device__ __forceinline__ int xrow( int i, int n ) { return i * n - ( ( i * ( i - 1 ) ) >> 1 ); }
__host__ __device__ inline int xpacked( int n ) { return ( n * ( n + 1 ) ) >> 1; }

// X from a factor that cholesky_la left: off-diagonal tiles hold U(I, K);
// a diagonal tile holds U in its upper part and its inverse X_JJ in the lower
// part (X_JJ(r, c) at tix(c, r)), with the inverse pivots in Iv. A thread per
// column j (columns are independent): the column's own tile from X_JJ, then
// tile rows I = J-1 .. 0 by blocks, x_I = -X_II sum_{K > I} U(I, K) x_K. The
// warp's lanes step through (I, K) together, so the U elements they read are
// broadcasts.
template <int GROUP, class T>
__device__ void tri_inverse_packed( const Grp<GROUP>& g, const T* H, const T* Iv, int n, T* X ) {
    const int nb = hnb( n );
    for( int j0 = 0; j0 < n; j0 += GROUP ) {
        if( j0 + ( g.r & ~31 ) >= n ) continue;    // the warp has no column in this round
        const int j = j0 + g.r;
        // the warp's largest tile column (lanes step through the tiles together)
        const int Jw = min( j0 + ( g.r & ~31 ) + 31, n - 1 ) >> 3;
        const bool act = j < n;
        const int J = act ? j >> 3 : -1, c = j & 7;
        if( act ) {
            const T* DJ = H + htile( J, J );
            for( int r = 0; r <= c; ++r ) X[xrow( 8 * J + r, n ) + j - 8 * J - r] = r == c ? Iv[8 * J + c] : DJ[tix( c, r )];
        }
        for( int I = Jw - 1; I >= 0; --I ) {
            T s[8];
#pragma unroll
            for( int r = 0; r < 8; ++r ) s[r] = T( 0 );
            for( int K = I + 1; K <= Jw; ++K ) {
                const T* A = H + htile( I, K );
#pragma unroll
                for( int kk = 0; kk < 8; ++kk ) {
                    const int k = 8 * K + kk;
                    if( act && I < J && k <= j ) {
                        const T xk = X[xrow( k, n ) + j - k];
#pragma unroll
                        for( int r = 0; r < 8; ++r ) s[r] = fma( A[tix( r, kk )], xk, s[r] );
                    }
                }
            }
            if( act && I < J ) {
                const T* DI = H + htile( I, I );
#pragma unroll
                for( int r = 0; r < 8; ++r ) {
                    T v = Iv[8 * I + r] * s[r];
#pragma unroll
                    for( int q = r + 1; q < 8; ++q ) v = fma( DI[tix( q, r )], s[q], v );
                    X[xrow( 8 * I + r, n ) + j - 8 * I - r] = -v;
                }
            }
        }
    }
    g.sync();
}

// d = X (X^T b) = H^-1 b with the packed inverse; gf, tf: n floats of scratch.
template <int GROUP, class T>
__device__ void chord_direction_packed( const Grp<GROUP>& g, const T* X, int n, const double* b, T* gf, T* tf, double* d ) {
    for( int i = g.r; i < n; i += GROUP ) gf[i] = T( b[i] );
    g.sync();
    for( int o = g.r; o < n; o += GROUP ) {    // t = X^T b: column o, rows 0..o
        T a0 = 0, a1 = 0;
        int i = 0;
        for( ; i + 1 <= o; i += 2 ) {
            a0 = fma( X[xrow( i, n ) + o - i], gf[i], a0 );
            a1 = fma( X[xrow( i + 1, n ) + o - i - 1], gf[i + 1], a1 );
        }
        if( i <= o ) a0 = fma( X[xrow( i, n ) + o - i], gf[i], a0 );
        tf[o] = a0 + a1;
    }
    g.sync();
    for( int o = g.r; o < n; o += GROUP ) {    // d = X t: row o, columns o..n-1
        const T* row = X + xrow( o, n ) - o;
        T a0 = 0, a1 = 0;
        int j = o;
        for( ; j + 1 < n; j += 2 ) {
            a0 = fma( row[j], tf[j], a0 );
            a1 = fma( row[j + 1], tf[j + 1], a1 );
        }
        if( j < n ) a0 = fma( row[j], tf[j], a0 );
        d[o] = double( a0 + a1 );
    }
    g.sync();
}

}    // namespace uqc
