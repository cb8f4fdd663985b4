/* Test-infrastructure shim: LAPACK dposv_/dgesv_ for the oracle harness.
 *
 * The reference links a system LAPACK (third-party; which implementation and
 * version is not pinned anywhere in the reference) and calls dposv_ with
 * uplo='U' from posv() (vectorspace.cpp:152-171) to solve the Newton system
 * H x = g, and dgesv_ from gesv() (vectorspace.cpp:132-150, unused on the hot
 * path). This file restates the published Netlib reference algorithms:
 *   dposv = dpotrf (here the unblocked dpotf2, upper) + dpotrs
 *   dpotrs = dtrsm(L,U,T,N) then dtrsm(L,U,N,N)
 * in plain C with the same loop and summation order as the Netlib Fortran.
 * Results differ from an optimised LAPACK only by floating-point rounding.
 * info > 0 reports the first non-positive pivot, as LAPACK does.
 */
#include <math.h>

#define A_(i, j) a[(long)(j) * lda + (i)]

void dposv_( const char* uplo, const int* n_, const int* nrhs_, double* a, const int* lda_, double* b, const int* ldb_, int* info ) {
    const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
    (void)uplo; /* the reference always passes 'U' */
    *info = 0;
    if( n == 0 ) return;
    /* dpotf2, upper: A = U^T U, column by column */
    for( int j = 0; j < n; ++j ) {
        double dot = 0.0;
        for( int k = 0; k < j; ++k ) dot += A_( k, j ) * A_( k, j );
        double ajj = A_( j, j ) - dot;
        if( ajj <= 0.0 || isnan( ajj ) ) {
            A_( j, j ) = ajj;
            *info      = j + 1;
            return;
        }
        ajj        = sqrt( ajj );
        A_( j, j ) = ajj;
        /* dgemv('T'): A(j, j+1:n) -= A(0:j-1, j+1:n)^T A(0:j-1, j) */
        for( int c = j + 1; c < n; ++c ) {
            double t = 0.0;
            for( int k = 0; k < j; ++k ) t += A_( k, c ) * A_( k, j );
            A_( j, c ) = A_( j, c ) + ( -1.0 ) * t;
        }
        /* dscal by 1/ajj */
        const double r = 1.0 / ajj;
        for( int c = j + 1; c < n; ++c ) A_( j, c ) *= r;
    }
    /* dpotrs: U^T y = b, then U x = y */
    for( int r = 0; r < nrhs; ++r ) {
        double* x = b + (long)r * ldb;
        for( int i = 0; i < n; ++i ) {
            double t = x[i];
            for( int k = 0; k < i; ++k ) t = t - A_( k, i ) * x[k];
            x[i] = t / A_( i, i );
        }
        for( int k = n - 1; k >= 0; --k ) {
            if( x[k] != 0.0 ) {
                x[k] = x[k] / A_( k, k );
                for( int i = 0; i < k; ++i ) x[i] = x[i] - x[k] * A_( i, k );
            }
        }
    }
}

void dgesv_( const int* n_, const int* nrhs_, double* a, const int* lda_, int* ipiv, double* b, const int* ldb_, int* info ) {
    const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
    *info = 0;
    /* LU with partial pivoting (dgetf2), then forward/back substitution */
    for( int j = 0; j < n; ++j ) {
        int p     = j;
        double mx = fabs( A_( j, j ) );
        for( int i = j + 1; i < n; ++i )
            if( fabs( A_( i, j ) ) > mx ) {
                mx = fabs( A_( i, j ) );
                p  = i;
            }
        ipiv[j] = p + 1;
        if( A_( p, j ) == 0.0 ) {
            if( *info == 0 ) *info = j + 1;
            continue;
        }
        if( p != j )
            for( int c = 0; c < n; ++c ) {
                double t   = A_( j, c );
                A_( j, c ) = A_( p, c );
                A_( p, c ) = t;
            }
        const double r = 1.0 / A_( j, j );
        for( int i = j + 1; i < n; ++i ) A_( i, j ) *= r;
        for( int c = j + 1; c < n; ++c )
            for( int i = j + 1; i < n; ++i ) A_( i, c ) -= A_( i, j ) * A_( j, c );
    }
    if( *info ) return;
    for( int r = 0; r < nrhs; ++r ) {
        double* x = b + (long)r * ldb;
        for( int j = 0; j < n; ++j )
            if( ipiv[j] - 1 != j ) {
                double t         = x[j];
                x[j]             = x[ipiv[j] - 1];
                x[ipiv[j] - 1] = t;
            }
        for( int j = 0; j < n; ++j )
            for( int i = j + 1; i < n; ++i ) x[i] -= A_( i, j ) * x[j];
        for( int j = n - 1; j >= 0; --j ) {
            x[j] /= A_( j, j );
            for( int i = 0; i < j; ++i ) x[i] -= A_( i, j ) * x[j];
        }
    }
}
