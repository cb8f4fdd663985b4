/* FP64 CPU restatement of UQCreator's IPM hot path (the oracle).
 *
 * TEST INFRASTRUCTURE ONLY (see uqc_oracle.h). Every function cites the
 * reference file:line it restates (paths relative to UQCreator's code/src).
 * Operation order follows the reference so that, built with
 * -ffp-contract=off against the same libm, results are bit-identical to the
 * reference's own code (checked by tests/test_oracle_pin.py).
 */
#include "uqc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXS 4

struct uqco {
    uqco_config cfg;
    int nS, nT, nQ, nCells, nFaces, nLevels, dimXi;
    int nTLevel[16];
    int* idx;          /* nT x dimXi polynomial degrees */
    double *phi, *phiWf, *xi, *w;
    /* geometry */
    double *area, *maxEdge, *center, *unitN, *scaledN;
    int *nbr, *bnd; /* bnd: 0 interior, 1 Dirichlet, 2 no-slip wall, 3 shallow-water wall */
    double* bndN;   /* unit normal of each cell's ghost face (Cell::UpdateBoundaryNormal) */
    double dtFixed; /* TimeSolver dt = area(0) CFL / 12 (timesolver.cpp:4-9) */
    /* state */
    double *u, *lam, *uQ, *uNew, *uOld;
    unsigned* level;
    double t;
    int levelCap, retIndex; /* retardation: highest level allowed, thresholds passed */
};

static void reset_retardation( uqco* h );

/* ------------------------------------------------------------------ tables */

/* MathTools::Pythag (mathtools.cpp:3-7). */
static double pythag( double a, double b ) {
    double absa = fabs( a ), absb = fabs( b );
    return absa > absb ? absa * sqrt( 1.0 + pow( absb / absa, 2 ) ) : ( absb == 0.0 ? 0.0 : absb * sqrt( 1.0 + pow( absa / absb, 2 ) ) );
}

/* Implicit QL on a symmetric tridiagonal matrix: eigenvalues d and
 * eigenvector matrix z (row major z[r * n + c]); restates
 * MathTools::ComputeEigenValTriDiagMatrix (mathtools.cpp:41-104). */
static void tridiag_ql( int n, double* d, double* e, double* z ) {
    const double eps = 2.220446049250313e-16;
    int m, l, iter, i, k;
    double s, r, p, g, f, dd, c, b;
    for( i = 1; i < n; i++ ) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for( l = 0; l < n; l++ ) {
        iter = 0;
        do {
            for( m = l; m < n - 1; m++ ) {
                dd = fabs( d[m] ) + fabs( d[m + 1] );
                if( fabs( e[m] ) <= eps * dd ) break;
            }
            if( m != l ) {
                if( iter++ == 30 ) return;
                g = ( d[l + 1] - d[l] ) / ( 2.0 * e[l] );
                r = pythag( g, 1.0 );
                g = d[m] - d[l] + e[l] / ( g + copysign( r, g ) );
                s = c = 1.0;
                p     = 0.0;
                for( i = m - 1; i >= l; i-- ) {
                    f        = s * e[i];
                    b        = c * e[i];
                    e[i + 1] = ( r = pythag( f, g ) );
                    if( r == 0.0 ) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s        = f / r;
                    c        = g / r;
                    g        = d[i + 1] - p;
                    r        = ( d[i] - g ) * s + 2.0 * c * b;
                    d[i + 1] = g + ( p = s * r );
                    g        = c * r - b;
                    for( k = 0; k < n; k++ ) {
                        f                = z[k * n + i + 1];
                        z[k * n + i + 1] = s * z[k * n + i] + c * f;
                        z[k * n + i]     = c * z[k * n + i] - s * f;
                    }
                }
                if( r == 0.0 && i >= l ) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while( m != l );
    }
}

/* Gauss-Legendre nodes and weights by Golub-Welsch, sorted ascending;
 * restates Legendre::Compute (legendre.cpp:9-28) and Polynomial::Sort
 * (polynomial.cpp:7-16). */
static void gauss_legendre( int n, double* x, double* w ) {
    double* d = calloc( n, sizeof( double ) );
    double* e = calloc( n, sizeof( double ) );
    double* z = calloc( (size_t)n * n, sizeof( double ) );
    double* sub = calloc( n, sizeof( double ) );
    for( int i = 0; i < n - 1; ++i ) sub[i + 1] = sqrt( 1 / ( 4 - 1 / pow( (double)( i + 1 ), 2 ) ) );
    for( int i = 0; i < n; ++i ) {
        d[i]         = 0.0;
        z[i * n + i] = 1.0;
        e[i]         = i == 0 ? 0.0 : sub[i];
    }
    tridiag_ql( n, d, e, z );
    double* xs = malloc( n * sizeof( double ) );
    double* ws = malloc( n * sizeof( double ) );
    for( int i = 0; i < n; ++i ) {
        xs[i] = fabs( d[i] ) < 1e-15 ? 0 : d[i];
        ws[i] = 2 * pow( z[0 * n + i], 2 );
    }
    /* selection by rank: nodes are distinct, so a stable ascending order */
    for( int i = 0; i < n; ++i ) {
        int rank = 0;
        for( int j = 0; j < n; ++j )
            if( xs[j] < xs[i] ) ++rank;
        x[rank] = xs[i];
        w[rank] = ws[i];
    }
    free( d ); free( e ); free( z ); free( sub ); free( xs ); free( ws );
}

/* P_m(x) by the three-term recurrence (the published algorithm of
 * boost::math::legendre_p, called at legendre.cpp:30). */
static double legendre_p( int l, double x ) {
    double p0 = 1.0, p1 = x;
    if( l == 0 ) return p0;
    unsigned n = 1;
    while( n < (unsigned)l ) {
        double t = p0;
        p0       = p1;
        p1       = t;
        p1       = ( ( 2.0 * n + 1.0 ) * x * p0 - (double)n * p1 ) / (double)( n + 1 );
        ++n;
    }
    return p1;
}

static unsigned upow( unsigned b, unsigned e ) { return (unsigned)pow( b, e ); }

/* Polynomial index set with level ordering: restates settings.cpp:241-265. */
static int index_set( const uqco_config* c, int* idx, int maxOut, int* nTLevel ) {
    int count = 0, previousDegree = -1;
    unsigned nMoments = (unsigned)c->degree[c->n_levels - 1];
    int test[8];
    for( int level = 0; level < c->n_levels; ++level ) {
        for( unsigned i = 0; i < pow( nMoments + 1, c->dim_xi ); ++i ) {
            int totalDegree = 0;
            for( int l = 0; l < c->dim_xi; ++l ) {
                test[l] = (int)( ( ( i - i % upow( nMoments + 1, l ) ) / upow( nMoments + 1, l ) ) % ( nMoments + 1 ) );
                totalDegree += test[l];
            }
            if( ( (unsigned)totalDegree <= (unsigned)c->degree[level] && totalDegree > previousDegree ) || c->max_degree ) {
                if( count < maxOut )
                    for( int l = 0; l < c->dim_xi; ++l ) idx[count * c->dim_xi + l] = test[l];
                ++count;
            }
        }
        nTLevel[level] = count;
        if( c->max_degree ) break;
        previousDegree = c->degree[level];
    }
    return count;
}

/* Tensor grid (tensorizedquadrature.cpp:27-74) and the scaled basis tables
 * phiTilde, phiTildeWf (closure.cpp:49-64; Legendre L2Norm sqrt(1/(2i+1)),
 * fXi = 1/2, legendre.cpp:36-38). */
static void build_tables( uqco* h ) {
    const uqco_config* c = &h->cfg;
    int nq1 = c->n_quad, d = c->dim_xi;
    double* x1 = malloc( nq1 * sizeof( double ) );
    double* w1 = malloc( nq1 * sizeof( double ) );
    gauss_legendre( nq1, x1, w1 );
    h->nQ = (int)(unsigned)pow( nq1, d );
    h->xi = malloc( (size_t)h->nQ * d * sizeof( double ) );
    h->w  = malloc( h->nQ * sizeof( double ) );
    for( int k = 0; k < h->nQ; ++k ) {
        h->w[k] = 1.0;
        for( int l = 0; l < d; ++l ) {
            unsigned q            = (unsigned)( ( k - k % upow( nq1, l ) ) / upow( nq1, l ) ) % nq1;
            h->xi[k * d + l]      = x1[q];
            h->w[k] *= w1[q];
        }
    }
    h->phi   = malloc( (size_t)h->nQ * h->nT * sizeof( double ) );
    h->phiWf = malloc( (size_t)h->nQ * h->nT * sizeof( double ) );
    for( int k = 0; k < h->nQ; ++k )
        for( int i = 0; i < h->nT; ++i ) {
            double p = 1.0, pw = 1.0;
            for( int l = 0; l < d; ++l ) {
                int m       = h->idx[i * d + l];
                double xk   = h->xi[k * d + l];
                double norm = sqrt( 1.0 / ( 2.0 * m + 1.0 ) );
                p *= legendre_p( m, xk ) / norm;
                pw *= legendre_p( m, xk ) / norm * 0.5;
            }
            pw *= h->w[k];
            h->phi[k * h->nT + i]   = p;
            h->phiWf[k * h->nT + i] = pw;
        }
    free( x1 ); free( w1 );
}

/* ---------------------------------------------------------------- ansatz */

/* BoundedBarrier::U (boundedbarrier.cpp:19-31). */
static double bb_u( double L, double um, double up ) {
    double ePos = exp( L ), eNeg = 1.0 / ePos;
    if( L > 0.0 ) return up / ( eNeg + 1.0 ) + um * eNeg / ( 1.0 + eNeg );
    return um / ( ePos + 1.0 ) + up * ePos / ( 1.0 + ePos );
}
/* BoundedBarrier::DU (boundedbarrier.cpp:67-80). */
static double bb_du( double L, double um, double up ) {
    double ePos = exp( L ), eNeg = 1 / ePos;
    if( L > 0 ) return eNeg * ( up - um ) / ( exp( -2.0 * L ) + 2.0 * eNeg + 1.0 );
    return ePos * ( up - um ) / ( 1.0 + 2.0 * ePos + exp( 2.0 * L ) );
}

/* U(Lambda) at one node. vec_form selects the formula of U(Vector&, ...)
 * used by Gradient and WriteMeanAndVar; otherwise the U(const Matrix&) formula
 * used to reconstruct uQ (momentsolver.cpp:99-101). They differ only for the
 * Euler closure (eulerclosure2d.cpp:7-18 vs :27-32). */
static void ansatz_u( const uqco* h, const double* L, double* out, int vec_form ) {
    const uqco_config* c = &h->cfg;
    if( c->closure == UQCO_BOUNDED_BARRIER ) {
        for( int l = 0; l < h->nS; ++l ) out[l] = bb_u( L[l], c->bb_minus, c->bb_plus );
    }
    else if( c->closure == UQCO_EULER2D ) {
        double g = -c->gamma; /* EulerClosure2D stores -gamma (eulerclosure2d.cpp:3) */
        double v1 = L[0], v2 = L[1], v3 = L[2], v4 = L[3];
        double expTerm;
        if( vec_form )
            expTerm = exp( 1.0 / ( 1.0 + g ) * ( ( pow( v2, 2 ) + pow( v3, 2 ) - 2.0 * v1 * v4 - 2.0 * v4 * g ) / ( 2.0 * v4 ) ) ) * pow( -v4, 1.0 / ( 1.0 + g ) );
        else
            expTerm = pow( -exp( ( ( pow( v2, 2 ) + pow( v3, 2 ) - 2.0 * v1 * v4 - 2.0 * v4 * g ) / ( 2.0 * v4 ) ) ) * v4, 1.0 / ( 1.0 + g ) );
        out[0] = expTerm;
        out[1] = -( ( v2 * expTerm ) / v4 );
        out[2] = -( ( v3 * expTerm ) / v4 );
        out[3] = -( ( expTerm * ( -pow( v2, 2 ) - pow( v3, 2 ) + 2.0 * v4 ) ) / ( 2.0 * pow( v4, 2 ) ) );
    }
    else {
        /* ShallowWaterClosure::U (shallowwaterclosure.cpp:10-13), g = 9.81 */
        const double gr = 9.81;
        out[0] = ( 0.5 * ( 2 * L[0] + pow( L[1], 2 ) ) ) / ( gr );
        out[1] = ( 0.5 * ( 2 * L[0] * L[1] + pow( L[1], 3 ) ) ) / gr;
    }
}

/* DU(Lambda) at one node, y[l * nS + m] = y(l, m). */
static void ansatz_du( const uqco* h, const double* L, double* y ) {
    const uqco_config* c = &h->cfg;
    int nS               = h->nS;
    if( c->closure == UQCO_BOUNDED_BARRIER ) {
        for( int l = 0; l < nS; ++l )
            for( int m = 0; m < nS; ++m ) y[l * nS + m] = bb_du( L[l], c->bb_minus, c->bb_plus );
    }
    else if( c->closure == UQCO_EULER2D ) {
        /* EulerClosure2D::DU (eulerclosure2d.cpp:54-88) */
        double g = -c->gamma;
        double v1 = L[0], v2 = L[1], v3 = L[2], v4 = L[3];
        double v4pow3 = pow( v4, 3 ), v4pow2 = pow( v4, 2 ), v4pow2Inv = 1.0 / v4pow2;
        double v3pow2 = pow( v3, 2 ), v2pow2 = pow( v2, 2 );
        double expTerm = exp( 1.0 / ( 1.0 + g ) * ( ( pow( v2, 2 ) + pow( v3, 2 ) - 2.0 * v1 * v4 - 2.0 * v4 * g ) / ( 2.0 * v4 ) ) ) * pow( -v4, 1.0 / ( 1.0 + g ) ) /
                         ( 1.0 + g );
        double vTerm = expTerm * ( v2pow2 + v3pow2 + 2.0 * v4 * g ) / ( 2 * v4pow3 );
        y[0 * 4 + 0] = -( expTerm );
        y[0 * 4 + 1] = ( v2 * expTerm ) / ( v4 );
        y[0 * 4 + 2] = ( v3 * expTerm ) / ( v4 );
        y[0 * 4 + 3] = -( 0.5 * ( ( v2pow2 + v3pow2 - 2.0 * v4 ) * expTerm ) * v4pow2Inv );
        y[1 * 4 + 0] = y[0 * 4 + 1];
        y[1 * 4 + 1] = -( ( expTerm * ( v2pow2 + ( g + 1.0 ) * v4 ) ) * v4pow2Inv );
        y[1 * 4 + 2] = -( ( v2 * v3 * expTerm ) * v4pow2Inv );
        y[1 * 4 + 3] = v2 * vTerm;
        y[2 * 4 + 0] = y[0 * 4 + 2];
        y[2 * 4 + 1] = y[1 * 4 + 2];
        y[2 * 4 + 2] = -( ( expTerm * ( v3pow2 + ( g + 1.0 ) * v4 ) ) * v4pow2Inv );
        y[2 * 4 + 3] = v3 * vTerm;
        y[3 * 4 + 0] = y[0 * 4 + 3];
        y[3 * 4 + 1] = y[1 * 4 + 3];
        y[3 * 4 + 2] = y[2 * 4 + 3];
        y[3 * 4 + 3] = -( expTerm * ( pow( v2, 4 ) + pow( v3, 4 ) + 4.0 * v3pow2 * v4 * g - 4.0 * v4pow2 * g + 2.0 * v2pow2 * ( v3pow2 + 2.0 * v4 * g ) ) ) /
                       ( 4.0 * pow( v4, 4 ) );
    }
    else {
        /* ShallowWaterClosure::DU (shallowwaterclosure.cpp:32-37) */
        const double gr = 9.81;
        y[0] = 1.0 / gr;
        y[1] = L[1] / gr;
        y[2] = L[1] / gr;
        y[3] = ( L[0] + 1.5 * pow( L[1], 2 ) ) / gr;
    }
}

/* Closure::DS: initial dual guess from the mean state; Euler
 * (eulerclosure2d.cpp:90-106), shallow water (shallowwaterclosure.cpp:39-42);
 * the base class leaves ds unchanged (closure.cpp:289). */
static void entropy_grad( const uqco* h, const double* u, double* ds ) {
    const uqco_config* c = &h->cfg;
    if( c->closure == UQCO_EULER2D ) {
        double gamma = -c->gamma;
        double rho = u[0], rhoU = u[1], rhoV = u[2], rhoE = u[3];
        double rhoV2 = pow( rhoV, 2 ), rhoU2 = pow( rhoU, 2 );
        ds[0] = ( rhoU2 + rhoV2 + gamma * ( 2 * rho * rhoE - rhoU2 - rhoV2 ) ) / ( -2 * rho * rhoE + rhoU2 + rhoV2 ) -
                log( pow( rho, gamma ) * ( rhoE - ( rhoU2 + rhoV2 ) / ( 2 * rho ) ) );
        ds[1] = -( ( 2 * rho * rhoU ) / ( -2 * rho * rhoE + rhoU2 + rhoV2 ) );
        ds[2] = -( ( 2 * rho * rhoV ) / ( -2 * rho * rhoE + rhoU2 + rhoV2 ) );
        ds[3] = -( rho / ( rhoE - ( rhoU2 + rhoV2 ) / ( 2 * rho ) ) );
    }
    else if( c->closure == UQCO_SHALLOW_WATER ) {
        const double gr = 9.81;
        ds[0] = ( gr * pow( u[0], 3 ) - 0.5 * pow( u[1], 2 ) ) / pow( u[0], 2 );
        ds[1] = u[1] / u[0];
    }
}

/* --------------------------------------------------------------- closure */

/* Lambda_k[s] = sum_i lambda(s,i) phiTilde(k,i), i < nT (closure.cpp:205-213). */
static void eval_lambda( const uqco* h, const double* lam, int k, int nT, double* out ) {
    for( int s = 0; s < h->nS; ++s ) {
        double a = 0.0;
        for( int i = 0; i < nT; ++i ) a += lam[s * h->nT + i] * h->phi[k * h->nT + i];
        out[s] = a;
    }
}

/* Closure::Gradient (closure.cpp:234-253): g[l nT + i] = sum_k U_l phiWf(k,i) - u(l,i). */
static void gradient( const uqco* h, double* g, const double* lam, const double* u, int nT ) {
    double L[MAXS], uk[MAXS];
    int nS = h->nS;
    for( int r = 0; r < nS * nT; ++r ) g[r] = 0.0;
    for( int k = 0; k < h->nQ; ++k ) {
        eval_lambda( h, lam, k, nT, L );
        ansatz_u( h, L, uk, 1 );
        for( int i = 0; i < nT; ++i )
            for( int l = 0; l < nS; ++l ) g[l * nT + i] += uk[l] * h->phiWf[k * h->nT + i];
    }
    for( int l = 0; l < nS; ++l )
        for( int j = 0; j < nT; ++j ) g[l * nT + j] = g[l * nT + j] - u[l * h->nT + j];
}

/* Closure::Hessian (closure.cpp:255-271): H column-major n x n,
 * H(m nT + j, l nT + i) += phi(k,j) phiWf(k,i) DU(l,m). */
static void hessian( const uqco* h, double* H, const double* lam, int nT ) {
    int nS = h->nS, n = nS * nT;
    double L[MAXS], du[MAXS * MAXS];
    memset( H, 0, sizeof( double ) * n * n );
    for( int k = 0; k < h->nQ; ++k ) {
        eval_lambda( h, lam, k, nT, L );
        ansatz_du( h, L, du );
        for( int l = 0; l < nS; ++l )
            for( int m = 0; m < nS; ++m )
                for( int j = 0; j < nT; ++j )
                    for( int i = 0; i < nT; ++i ) {
                        double hp = h->phi[k * h->nT + j] * h->phiWf[k * h->nT + i];
                        H[(long)( l * nT + i ) * n + ( m * nT + j )] += hp * du[l * nS + m];
                    }
    }
}

/* Cholesky solve H x = b (LAPACK dposv, uplo 'U', unblocked dpotf2 + dpotrs
 * as published by Netlib), called through posv (vectorspace.cpp:152-171).
 * Returns 0 or the 1-based index of the first non-positive pivot. */
static int posv( double* a, int n, double* x ) {
    for( int j = 0; j < n; ++j ) {
        double dot = 0.0;
        for( int k = 0; k < j; ++k ) dot += a[(long)j * n + k] * a[(long)j * n + k];
        double ajj = a[(long)j * n + j] - dot;
        if( ajj <= 0.0 || isnan( ajj ) ) {
            a[(long)j * n + j] = ajj;
            return j + 1;
        }
        ajj                = sqrt( ajj );
        a[(long)j * n + j] = ajj;
        for( int c = j + 1; c < n; ++c ) {
            double t = 0.0;
            for( int k = 0; k < j; ++k ) t += a[(long)c * n + k] * a[(long)j * n + k];
            a[(long)c * n + j] = a[(long)c * n + j] + ( -1.0 ) * t;
        }
        const double r = 1.0 / ajj;
        for( int c = j + 1; c < n; ++c ) a[(long)c * n + j] *= r;
    }
    for( int i = 0; i < n; ++i ) {
        double t = x[i];
        for( int k = 0; k < i; ++k ) t = t - a[(long)i * n + k] * x[k];
        x[i] = t / a[(long)i * n + i];
    }
    for( int k = n - 1; k >= 0; --k ) {
        if( x[k] != 0.0 ) {
            x[k] = x[k] / a[(long)k * n + k];
            for( int i = 0; i < k; ++i ) x[i] = x[i] - x[k] * a[(long)k * n + i];
        }
    }
    return 0;
}

/* Closure::CalcNorm (closure.cpp:195-203). */
static double calc_norm( const double* v, int n ) {
    double out = 0.0;
    for( int r = 0; r < n; ++r ) out += pow( v[r], 2 );
    return sqrt( out );
}

/* y(l,j) = A(l,j) + s * d[l nT + j] for j < nT (closure.cpp:273-279, with the
 * scalar product -stepSize * alpha * g of :156,167,174). */
static void add_step( const uqco* h, const double* A, double s, const double* d, double* y, int nT ) {
    for( int l = 0; l < h->nS; ++l )
        for( int j = 0; j < nT; ++j ) y[l * h->nT + j] = A[l * h->nT + j] + s * d[l * nT + j];
}

/* Closure::SolveClosure (closure.cpp:133-193), alpha = 1 for every closure
 * here. Returns 0 converged, 1 max iterations, 2 line search > 1000 halvings,
 * 3 Hessian not positive definite. lam is updated in place (first nT columns). */
static int solve_closure( const uqco* h, double* lam, const double* u, int nT, int* itersOut ) {
    const double eps = h->cfg.epsilon, alpha = 1.0;
    const int maxIt = h->cfg.max_iterations, n = h->nS * nT;
    int rc = 1, iters = 0;
    double* g    = calloc( n, sizeof( double ) );
    double* dl   = calloc( n, sizeof( double ) );
    double* dln  = calloc( n, sizeof( double ) );
    double* H    = calloc( (size_t)n * n, sizeof( double ) );
    double* lamN = calloc( (size_t)h->nS * h->nT, sizeof( double ) );
    const int guard = h->cfg.newton_mode != 0;
    if( h->cfg.newton_mode == 2 ) {
        /* Closure::SolveClosureSafe (closure.cpp:297-339): no initial check,
         * every iteration recomputes the gradient, non-finite trial norms are
         * rejected by the line search (:318). */
        for( int l = 0; l < maxIt; ++l ) {
            double stepSize = 1.0;
            gradient( h, g, lam, u, nT );
            for( int r = 0; r < n; ++r ) dl[r] = -g[r];
            hessian( h, H, lam, nT );
            if( posv( H, n, g ) ) {
                rc = 3;
                goto done;
            }
            ++iters;
            memcpy( lamN, lam, sizeof( double ) * h->nS * h->nT );
            add_step( h, lam, -stepSize * alpha, g, lamN, nT );
            gradient( h, dln, lamN, u, nT );
            int refinementCounter = 0;
            while( calc_norm( dl, n ) < calc_norm( dln, n ) || !isfinite( calc_norm( dln, n ) ) ) {
                stepSize *= 0.5;
                add_step( h, lam, -stepSize * alpha, g, lamN, nT );
                gradient( h, dln, lamN, u, nT );
                if( calc_norm( dln, n ) < eps ) {
                    for( int s = 0; s < h->nS; ++s ) memcpy( lam + s * h->nT, lamN + s * h->nT, nT * sizeof( double ) );
                    rc = 0;
                    goto done;
                }
                else if( ++refinementCounter > 1000 ) {
                    rc = 2;
                    goto done;
                }
            }
            for( int s = 0; s < h->nS; ++s ) memcpy( lam + s * h->nT, lamN + s * h->nT, nT * sizeof( double ) );
            if( calc_norm( dln, n ) < eps ) {
                rc = 0;
                goto done;
            }
        }
        goto done;
    }
    gradient( h, g, lam, u, nT );
    if( calc_norm( g, n ) < eps ) {
        rc = 0;
        goto done;
    }
    for( int r = 0; r < n; ++r ) dl[r] = -g[r];
    hessian( h, H, lam, nT );
    if( posv( H, n, g ) ) {
        rc = 3;
        goto done;
    }
    iters = 1;
    if( maxIt == 1 ) {
        add_step( h, lam, -alpha, g, lam, nT );
        rc = 0;
        goto done;
    }
    memcpy( lamN, lam, sizeof( double ) * h->nS * h->nT );
    add_step( h, lam, -alpha, g, lamN, nT );
    gradient( h, dln, lamN, u, nT );
    for( int l = 0; l < maxIt; ++l ) {
        double stepSize = 1.0;
        if( l != 0 ) {
            gradient( h, g, lam, u, nT );
            for( int r = 0; r < n; ++r ) dl[r] = -g[r];
            hessian( h, H, lam, nT );
            if( posv( H, n, g ) ) {
                rc = 3;
                goto done;
            }
            ++iters;
            add_step( h, lam, -stepSize * alpha, g, lamN, nT );
            gradient( h, dln, lamN, u, nT );
        }
        int refinementCounter = 0;
        while( calc_norm( dl, n ) < calc_norm( dln, n ) || ( guard && !isfinite( calc_norm( dln, n ) ) ) ) {
            stepSize *= 0.5;
            add_step( h, lam, -stepSize * alpha, g, lamN, nT );
            gradient( h, dln, lamN, u, nT );
            if( calc_norm( dln, n ) < eps ) {
                for( int s = 0; s < h->nS; ++s ) memcpy( lam + s * h->nT, lamN + s * h->nT, nT * sizeof( double ) );
                rc = 0;
                goto done;
            }
            else if( ++refinementCounter > 1000 ) {
                rc = 2;
                goto done;
            }
        }
        for( int s = 0; s < h->nS; ++s ) memcpy( lam + s * h->nT, lamN + s * h->nT, nT * sizeof( double ) );
        if( calc_norm( dln, n ) < eps ) {
            rc = 0;
            goto done;
        }
    }
done:
    if( itersOut ) *itersOut = iters;
    free( g ); free( dl ); free( dln ); free( H ); free( lamN );
    return rc;
}

/* ------------------------------------------------------------- problems */

/* Initial states of the harness problems (oracle/ref/harness.cpp), which
 * keep the reference's forms: Burgers ramp (burgers.cpp:48-68), Sod-type Euler
 * interface, dam break. */
static void initial_state( const uqco* h, const double* x, const double* xi, double* y ) {
    const uqco_config* c = &h->cfg;
    if( c->problem == UQCO_BURGERS ) {
        double uL = c->ic[0], uR = c->ic[1], x0 = c->ic[2], x1 = c->ic[3], sg = c->sigma[0];
        if( x[0] < x0 + sg * xi[0] )
            y[0] = uL;
        else if( x[0] < x1 + sg * xi[0] )
            y[0] = uL + ( uR - uL ) * ( x0 + sg * xi[0] - x[0] ) / ( x0 - x1 );
        else
            y[0] = uR;
    }
    else if( c->problem == UQCO_EULER ) {
        double xs = c->ic[0], rhoL = c->ic[1], pL = c->ic[2], rhoR = c->ic[3], pR = c->ic[4], rho, p;
        int d = c->dim_xi;
        if( x[0] < xs + c->sigma[0] * xi[0] ) {
            rho = rhoL * ( 1.0 + ( d > 1 ? c->sigma[1] * xi[1] : 0.0 ) );
            p   = pL * ( 1.0 + ( d > 2 ? c->sigma[2] * xi[2] : 0.0 ) );
        }
        else {
            rho = rhoR;
            p   = pR;
        }
        y[0] = rho;
        y[1] = 0.0;
        y[2] = 0.0;
        y[3] = p / ( c->gamma - 1.0 );
    }
    else {
        y[0] = x[0] < c->ic[0] ? c->ic[1] * ( 1.0 + c->sigma[0] * xi[0] ) : c->ic[2];
        y[1] = 0.0;
    }
}

/* Euler2D::F (euler2d.cpp:89-106) times n: (F(u) n)[i] = F(i,0) n0 + F(i,1) n1. */
static void euler_fn( double gm, const double* u, const double* n, double* out ) {
    double rhoInv = 1.0 / u[0], v1 = u[1] * rhoInv, v2 = u[2] * rhoInv;
    double p = ( gm - 1.0 ) * ( u[3] - 0.5 * u[0] * ( pow( v1, 2 ) + pow( v2, 2 ) ) );
    double F0[4] = {u[1], u[1] * v1 + p, u[1] * v2, ( u[3] + p ) * v1};
    double F1[4] = {u[2], u[2] * v1, u[2] * v2 + p, ( u[3] + p ) * v2};
    for( int i = 0; i < 4; ++i ) out[i] = ( 0.0 + F0[i] * n[0] ) + F1[i] * n[1];
}

/* Numerical flux g(u, v) at one node for a face with unit normal nu and
 * scaled normal n. Burgers: local Lax-Friedrichs of the Julia prototype
 * (julia/Tensorization/IPMSolver.jl:38-42); Euler: HLL (euler2d.cpp:52-87);
 * shallow water: Lax-Friedrichs with dx/dt = 12/CFL (shallowwater.cpp:21-35). */
static void num_flux( const uqco* h, const double* u, const double* v, const double* nu, const double* n, double* y ) {
    const uqco_config* c = &h->cfg;
    if( c->problem == UQCO_BURGERS ) {
        double beta = fabs( u[0] ) < fabs( v[0] ) ? fabs( v[0] ) : fabs( u[0] ); /* std::max */
        y[0] = 0.5 * ( 0.5 * u[0] * u[0] + 0.5 * v[0] * v[0] ) * n[0] - 0.5 * beta * ( v[0] - u[0] ) * fabs( n[0] );
    }
    else if( c->problem == UQCO_EULER ) {
        double gm = c->gamma;
        double rhoInv = 1.0 / u[0], uU = u[1] * rhoInv, vU = u[2] * rhoInv;
        double p  = ( gm - 1.0 ) * ( u[3] - 0.5 * u[0] * ( pow( uU, 2 ) + pow( vU, 2 ) ) );
        double aU = sqrt( gm * p * rhoInv );
        rhoInv    = 1.0 / v[0];
        double uV = v[1] * rhoInv, vV = v[2] * rhoInv;
        p         = ( gm - 1.0 ) * ( v[3] - 0.5 * v[0] * ( pow( uV, 2 ) + pow( vV, 2 ) ) );
        double aV = sqrt( gm * p * rhoInv );
        double lambdaMin = ( nu[0] * uU + nu[1] * vU ) - aU;
        double lambdaMax = ( nu[0] * uV + nu[1] * vV ) + aV;
        if( lambdaMin >= 0 )
            euler_fn( gm, u, n, y );
        else if( lambdaMax <= 0 )
            euler_fn( gm, v, n, y );
        else {
            /* (1/(lmax-lmin)) ((lmax F(u) - lmin F(v)) n + lmax lmin (v - u) |n|) */
            double rhoIu = 1.0 / u[0], a1 = u[1] * rhoIu, a2 = u[2] * rhoIu;
            double pu = ( gm - 1.0 ) * ( u[3] - 0.5 * u[0] * ( pow( a1, 2 ) + pow( a2, 2 ) ) );
            double rhoIv = 1.0 / v[0], b1 = v[1] * rhoIv, b2 = v[2] * rhoIv;
            double pv = ( gm - 1.0 ) * ( v[3] - 0.5 * v[0] * ( pow( b1, 2 ) + pow( b2, 2 ) ) );
            double Fu0[4] = {u[1], u[1] * a1 + pu, u[1] * a2, ( u[3] + pu ) * a1};
            double Fu1[4] = {u[2], u[2] * a1, u[2] * a2 + pu, ( u[3] + pu ) * a2};
            double Fv0[4] = {v[1], v[1] * b1 + pv, v[1] * b2, ( v[3] + pv ) * b1};
            double Fv1[4] = {v[2], v[2] * b1, v[2] * b2 + pv, ( v[3] + pv ) * b2};
            double nn = sqrt( ( 0.0 + fabs( n[0] ) * fabs( n[0] ) ) + fabs( n[1] ) * fabs( n[1] ) );
            double ll = lambdaMax * lambdaMin, inv = 1.0 / ( lambdaMax - lambdaMin );
            for( int i = 0; i < 4; ++i ) {
                double m0 = Fu0[i] * lambdaMax - Fv0[i] * lambdaMin;
                double m1 = Fu1[i] * lambdaMax - Fv1[i] * lambdaMin;
                double a  = ( 0.0 + m0 * n[0] ) + m1 * n[1];
                double b  = ( ll * ( v[i] - u[i] ) ) * nn;
                y[i]      = inv * ( a + b );
            }
        }
    }
    else {
        const double gr = 9.81;
        double dtdx     = c->cfl / 12.0;
        double Fl0 = u[1], Fl1 = pow( u[1], 2 ) / u[0] + 0.5 * gr * pow( u[0], 2 );
        double Fr0 = v[1], Fr1 = pow( v[1], 2 ) / v[0] + 0.5 * gr * pow( v[0], 2 );
        double a0 = ( 0.0 + Fl0 * n[0] ) + ( 0.0 + Fr0 * n[0] );
        double a1 = ( 0.0 + Fl1 * n[0] ) + ( 0.0 + Fr1 * n[0] );
        double s  = 0.5 / dtdx;
        y[0]      = 0.5 * a0 - s * ( v[0] - u[0] );
        y[1]      = 0.5 * a1 - s * ( v[1] - u[1] );
    }
}

/* Problem::ComputeDt for one cell's nodal states (burgers.cpp:114-122,
 * euler2d.cpp:114-134; shallow water: Settings::GetDT, problem.cpp:44). */
static double compute_dt( const uqco* h, const double* uq, double dx ) {
    const uqco_config* c = &h->cfg;
    double dtMinTotal    = 1e10;
    if( c->problem == UQCO_BURGERS ) {
        for( int k = 0; k < h->nQ; ++k ) {
            double d = c->cfl * dx / ( fabs( uq[k] ) );
            dtMinTotal = ( dtMinTotal < d ) ? dtMinTotal : d;
        }
    }
    else if( c->problem == UQCO_EULER ) {
        double gm = c->gamma;
        for( int k = 0; k < h->nQ; ++k ) {
            double rhoInv = 1.0 / uq[0 * h->nQ + k];
            double uU     = uq[1 * h->nQ + k] * rhoInv, vU = uq[2 * h->nQ + k] * rhoInv;
            double p      = ( gm - 1.0 ) * ( uq[3 * h->nQ + k] - 0.5 * uq[0 * h->nQ + k] * ( pow( uU, 2 ) + pow( vU, 2 ) ) );
            double a      = sqrt( gm * p * rhoInv );
            /* std::min(a, b) = b < a ? b : a */
            double t0 = fabs( 1.0 / ( vU - a ) ), t1 = fabs( 1.0 / ( vU + a ) );
            double m1 = ( t1 < t0 ) ? t1 : t0;
            double t2 = fabs( 1.0 / ( uU + a ) ), t3 = fabs( 1.0 / ( uU - a ) );
            double m2 = ( t3 < t2 ) ? t3 : t2;
            double mm = ( m2 < m1 ) ? m2 : m1;
            double d  = ( c->cfl / dx ) * mm;
            dtMinTotal = ( dtMinTotal < d ) ? dtMinTotal : d;
        }
    }
    else {
        dtMinTotal = h->dtFixed;
    }
    return dtMinTotal;
}

/* -------------------------------------------------------------- geometry */

/* Triangle geometry: area, centre, edges (A,B) = (n0,n1), (n1,n2), (n2,n0),
 * outward unit normals and lengths; restates triangle.cpp:3-70. */
static void triangle_geometry( const double* X, const double* Y, double* area, double* cen, double* un, double* sn, double* maxEdge ) {
    *area  = fabs( ( X[0] * ( Y[1] - Y[2] ) + X[1] * ( Y[2] - Y[0] ) + X[2] * ( Y[0] - Y[1] ) ) / 2 );
    cen[0] = ( X[0] + X[1] + X[2] ) / 3;
    cen[1] = ( Y[0] + Y[1] + Y[2] ) / 3;
    double mx = -1e10;
    for( int e = 0; e < 3; ++e ) {
        int A = e, B = ( e + 1 ) % 3;
        double length = sqrt( pow( X[A] - X[B], 2 ) + pow( Y[A] - Y[B], 2 ) );
        double dx = X[A] - X[B], dy = Y[A] - Y[B];
        double n0 = -dy, n1 = dx;
        double q0 = cen[0] - X[A], q1 = cen[1] - Y[A];
        if( ( 0.0 + n0 * q0 ) + n1 * q1 > 0 ) {
            n0 *= -1.0;
            n1 *= -1.0;
        }
        double nn = sqrt( ( 0.0 + fabs( n0 ) * fabs( n0 ) ) + fabs( n1 ) * fabs( n1 ) );
        n0 /= nn;
        n1 /= nn;
        nn = sqrt( ( 0.0 + fabs( n0 ) * fabs( n0 ) ) + fabs( n1 ) * fabs( n1 ) );
        n0 /= nn;
        n1 /= nn;
        un[2 * e]     = n0;
        un[2 * e + 1] = n1;
        sn[2 * e]     = length * n0;
        sn[2 * e + 1] = length * n1;
        if( mx < length ) mx = length;
    }
    *maxEdge = mx;
}

/* ------------------------------------------------------------------ API */

static int cmp_pair( const void* a, const void* b ) {
    const long* x = a;
    const long* y = b;
    if( x[0] != y[0] ) return x[0] < y[0] ? -1 : 1;
    return x[1] < y[1] ? -1 : ( x[1] > y[1] );
}

int uqco_create( const uqco_config* cfg, int n_nodes, const double* xy, const int* node_boundary, int n_tri, const int* tri, uqco** out ) {
    uqco* h = calloc( 1, sizeof( uqco ) );
    h->cfg  = *cfg;
    h->nS   = cfg->closure == UQCO_BOUNDED_BARRIER ? 1 : ( cfg->closure == UQCO_EULER2D ? 4 : 2 );
    h->dimXi   = cfg->dim_xi;
    h->nLevels = cfg->max_degree ? 1 : cfg->n_levels;
    h->nT      = index_set( cfg, NULL, 0, h->nTLevel );
    h->idx     = malloc( (size_t)h->nT * cfg->dim_xi * sizeof( int ) );
    index_set( cfg, h->idx, h->nT, h->nTLevel );
    build_tables( h );
    if( cfg->mesh_dim == 1 ) {
        int N      = cfg->n_cells_1d;
        h->nCells  = N;
        h->nFaces  = 2;
        h->area    = calloc( N, sizeof( double ) );
        h->maxEdge = calloc( N, sizeof( double ) );
        h->center  = calloc( 2 * N, sizeof( double ) );
        h->unitN   = calloc( 4 * N, sizeof( double ) );
        h->scaledN = calloc( 4 * N, sizeof( double ) );
        h->nbr     = calloc( 2 * N, sizeof( int ) );
        h->bnd     = calloc( N, sizeof( int ) );
        /* Mesh1D (mesh1d.cpp:5-67) with Line cells (line.cpp:3-44): centre is
         * the left node, maxEdge = dx^2, normals -1 / +1 of length 1. */
        for( int j = 0; j < N; ++j ) {
            double x0 = cfg->a + j * ( cfg->b - cfg->a ) / ( N );
            double x1 = cfg->a + ( j + 1 ) * ( cfg->b - cfg->a ) / ( N );
            h->area[j]         = fabs( x1 - x0 );
            h->maxEdge[j]      = pow( h->area[j], 2 );
            h->center[2 * j]   = ( x0 + x0 ) / 2;
            h->unitN[4 * j]    = -1.0;
            h->unitN[4 * j + 2] = 1.0;
            h->scaledN[4 * j]   = -1.0;
            h->scaledN[4 * j + 2] = 1.0;
            h->bnd[j]          = ( j == 0 || j == N - 1 );
            h->nbr[2 * j]      = h->bnd[j] ? N : j - 1;
            h->nbr[2 * j + 1]  = h->bnd[j] ? N : j + 1;
        }
    }
    else {
        int N      = n_tri;
        h->nCells  = N;
        h->nFaces  = 3;
        h->area    = calloc( N, sizeof( double ) );
        h->maxEdge = calloc( N, sizeof( double ) );
        h->center  = calloc( 2 * N, sizeof( double ) );
        h->unitN   = calloc( 6 * N, sizeof( double ) );
        h->scaledN = calloc( 6 * N, sizeof( double ) );
        h->nbr     = malloc( 3 * N * sizeof( int ) );
        h->bnd     = calloc( N, sizeof( int ) );
        for( int c = 0; c < N; ++c ) {
            double X[3], Y[3];
            int nb = 0;
            for( int v = 0; v < 3; ++v ) {
                X[v] = xy[2 * tri[3 * c + v]];
                Y[v] = xy[2 * tri[3 * c + v] + 1];
                nb += node_boundary[tri[3 * c + v]] != 0;
            }
            triangle_geometry( X, Y, &h->area[c], &h->center[2 * c], &h->unitN[6 * c], &h->scaledN[6 * c], &h->maxEdge[c] );
            h->bnd[c] = nb == 2;
        }
        /* neighbour across edge l = (node l, node l+1 mod 3); ghost id N */
        for( int r = 0; r < 3 * N; ++r ) h->nbr[r] = N;
        /* edge matching: sort (edge key, face) pairs, equal keys are neighbours */
        long ne   = 3L * N;
        long* key = malloc( ne * 2 * sizeof( long ) );
        for( int c = 0; c < N; ++c )
            for( int l = 0; l < 3; ++l ) {
                long a = tri[3 * c + l], b = tri[3 * c + ( l + 1 ) % 3];
                long lo = a < b ? a : b, hi = a < b ? b : a;
                key[2 * ( 3L * c + l )]     = lo * ( n_nodes + 1L ) + hi;
                key[2 * ( 3L * c + l ) + 1] = 3L * c + l;
            }
        qsort( key, ne, 2 * sizeof( long ), cmp_pair );
        for( long i = 0; i + 1 < ne; ++i )
            if( key[2 * i] == key[2 * ( i + 1 )] ) {
                long f0 = key[2 * i + 1], f1 = key[2 * i + 3];
                h->nbr[f0] = (int)( f1 / 3 );
                h->nbr[f1] = (int)( f0 / 3 );
                ++i;
            }
        free( key );
    }
    h->dtFixed = h->area[0] * cfg->cfl / 12.0;
    size_t n   = (size_t)h->nS * h->nT;
    h->u       = calloc( h->nCells * n, sizeof( double ) );
    h->lam     = calloc( h->nCells * n, sizeof( double ) );
    h->uNew    = calloc( h->nCells * n, sizeof( double ) );
    h->uOld    = calloc( h->nCells * n, sizeof( double ) );
    /* + the ghost row uQ[N], zero as in momentsolver.cpp:50 */
    h->uQ      = calloc( (size_t)( h->nCells + 1 ) * h->nS * h->nQ, sizeof( double ) );
    h->level   = calloc( h->nCells, sizeof( unsigned ) );
    /* Cell::UpdateBoundaryNormal (cell.cpp:57-68): the unit normal of the face
       with the largest neighbour id, the first such face on ties */
    h->bndN = calloc( 2 * (size_t)h->nCells, sizeof( double ) );
    for( int c = 0; c < h->nCells; ++c ) {
        int id = 0;
        for( int f = 1; f < h->nFaces; ++f )
            if( h->nbr[c * h->nFaces + f] > h->nbr[c * h->nFaces + id] ) id = f;
        h->bndN[2 * c]     = h->unitN[( c * h->nFaces + id ) * 2];
        h->bndN[2 * c + 1] = h->unitN[( c * h->nFaces + id ) * 2 + 1];
    }
    *out       = h;
    return 0;
}

void uqco_destroy( uqco* h ) {
    if( !h ) return;
    free( h->idx ); free( h->phi ); free( h->phiWf ); free( h->xi ); free( h->w );
    free( h->area ); free( h->maxEdge ); free( h->center ); free( h->unitN ); free( h->scaledN );
    free( h->nbr ); free( h->bnd ); free( h->bndN );
    free( h->u ); free( h->lam ); free( h->uNew ); free( h->uOld ); free( h->uQ ); free( h->level );
    free( h );
}

/* Boundary types of an SU2 mesh (Mesh2D::LoadSU2MeshFromFile,
   mesh2d.cpp:197-214): codes[c] (1 Dirichlet, 2 no-slip, 3 shallow-water
   wall) replaces the Dirichlet default of each boundary cell. */
void uqco_set_cell_bc( uqco* h, const int* codes ) {
    for( int c = 0; c < h->nCells; ++c )
        if( h->bnd[c] && codes[c] >= 1 && codes[c] <= 3 ) h->bnd[c] = codes[c];
}

void uqco_sizes( const uqco* h, int* out ) {
    out[0] = h->nCells;
    out[1] = h->nS;
    out[2] = h->nT;
    out[3] = h->nQ;
    out[4] = h->nLevels;
    out[5] = h->dimXi;
    out[6] = h->nFaces;
    for( int l = 0; l < h->nLevels; ++l ) out[7 + l] = h->nTLevel[l];
}

void uqco_tables( const uqco* h, double* phi, double* phiWf, double* xi, double* w ) {
    memcpy( phi, h->phi, sizeof( double ) * h->nQ * h->nT );
    memcpy( phiWf, h->phiWf, sizeof( double ) * h->nQ * h->nT );
    memcpy( xi, h->xi, sizeof( double ) * h->nQ * h->dimXi );
    memcpy( w, h->w, sizeof( double ) * h->nQ );
}

void uqco_geometry( const uqco* h, double* area, double* max_edge, double* center, double* unit_n, double* scaled_n, int* nbr, int* boundary ) {
    int N = h->nCells, F = h->nFaces;
    memcpy( area, h->area, sizeof( double ) * N );
    memcpy( max_edge, h->maxEdge, sizeof( double ) * N );
    memcpy( center, h->center, sizeof( double ) * 2 * N );
    memcpy( unit_n, h->unitN, sizeof( double ) * 2 * F * N );
    memcpy( scaled_n, h->scaledN, sizeof( double ) * 2 * F * N );
    memcpy( nbr, h->nbr, sizeof( int ) * F * N );
    memcpy( boundary, h->bnd, sizeof( int ) * N );
}

/* MomentSolver::SetupIC (momentsolver.cpp:535-563) and SetDuals without
 * restart (:463-485). */
void uqco_init_state( uqco* h ) {
    int nS = h->nS, nT = h->nT, nQ = h->nQ, d = h->dimXi;
    reset_retardation( h );
    double* uIC = malloc( sizeof( double ) * nS * nQ );
    double ds[MAXS] = {0, 0, 0, 0}, u0[MAXS];
    for( int j = 0; j < h->nCells; ++j ) {
        double x[2] = {h->center[2 * j], h->center[2 * j + 1]};
        for( int k = 0; k < nQ; ++k ) {
            double y[MAXS];
            initial_state( h, x, h->xi + k * d, y );
            for( int s = 0; s < nS; ++s ) uIC[s * nQ + k] = y[s];
        }
        double* u = h->u + (size_t)j * nS * nT;
        for( int s = 0; s < nS; ++s )
            for( int i = 0; i < nT; ++i ) {
                double a = 0.0;
                for( int k = 0; k < nQ; ++k ) a += uIC[s * nQ + k] * h->phiWf[k * nT + i];
                u[s * nT + i] = a;
            }
        double* lam = h->lam + (size_t)j * nS * nT;
        memset( lam, 0, sizeof( double ) * nS * nT );
        for( int s = 0; s < nS; ++s ) u0[s] = u[s * nT];
        entropy_grad( h, u0, ds );
        for( int s = 0; s < nS; ++s ) lam[s * nT] = ds[s];
        h->level[j] = (unsigned)( h->nLevels - 1 );
    }
    free( uIC );
    h->t = 0.0;
}

void uqco_get_state( const uqco* h, double* u, double* lambda, unsigned* level ) {
    size_t n = (size_t)h->nCells * h->nS * h->nT;
    if( u ) memcpy( u, h->u, n * sizeof( double ) );
    if( lambda ) memcpy( lambda, h->lam, n * sizeof( double ) );
    if( level ) memcpy( level, h->level, h->nCells * sizeof( unsigned ) );
}

void uqco_set_state( uqco* h, const double* u, const double* lambda, const unsigned* level, double t ) {
    size_t n = (size_t)h->nCells * h->nS * h->nT;
    if( u ) memcpy( h->u, u, n * sizeof( double ) );
    if( lambda ) memcpy( h->lam, lambda, n * sizeof( double ) );
    if( level ) memcpy( h->level, level, h->nCells * sizeof( unsigned ) );
    h->t = t;
    reset_retardation( h );
}

int uqco_solve_closure( const uqco* h, int n, double* lambda, const double* u, const unsigned* n_total_cell, int* status, int* iters ) {
    size_t m  = (size_t)h->nS * h->nT;
    int nFail = 0;
    for( int j = 0; j < n; ++j ) {
        int it = 0;
        int rc = solve_closure( h, lambda + j * m, u + j * m, n_total_cell ? (int)n_total_cell[j] : h->nT, &it );
        if( status ) status[j] = rc;
        if( iters ) iters[j] = it;
        nFail += rc != 0;
    }
    return nFail;
}

/* The retardation schedule from its start (no threshold passed). */
static void reset_retardation( uqco* h ) {
    h->levelCap = h->cfg.n_ret_levels > 0 ? h->cfg.ret_lev[0] : 1 << 30;
    h->retIndex = 0;
}

/* Refinement indicator (momentsolver.cpp:271-289), or the paper's
 * S_l = <(u_l - u_{l-1})^2> / <u_l^2> (Paper1/adaptivity.tex:12-14) of the first
 * state, written with the coefficients (the basis is orthonormal under the
 * quadrature): the added moments' squares over all squares, level 0 against
 * the mean alone. */
static double ref_indicator( const uqco* h, const double* u, unsigned lev ) {
    double ind = 0.0;
    if( h->cfg.ref_indicator == 1 ) {
        int prev = lev == 0 ? 1 : h->nTLevel[lev - 1];
        double num = 0.0, den = 0.0;
        for( int i = 0; i < h->nTLevel[lev]; ++i ) {
            den += u[i] * u[i];
            if( i >= prev ) num += u[i] * u[i];
        }
        return den > 0.0 ? num / den : 0.0;
    }
    if( h->dimXi == 1 ) {
        ind += fabs( u[h->nTLevel[lev] - 1] ) + fabs( u[h->nTLevel[lev] - 2] );
    }
    else {
        int prev = lev == 0 ? 1 : h->nTLevel[lev - 1];
        for( int i = prev; i < h->nTLevel[lev]; ++i ) ind += fabs( u[i] );
    }
    return ind;
}

/* One time step = body of MomentSolver::Solve (momentsolver.cpp:79-152) with
 * ExplicitEuler::Advance (expliciteuler.cpp:8-75), Dirichlet boundaries only. */
int uqco_step( uqco* h, int n_steps, double* out ) {
    int nS = h->nS, nT = h->nT, nQ = h->nQ, N = h->nCells, F = h->nFaces;
    size_t m  = (size_t)nS * nT;
    int fails = 0;
    double dt = 0.0, residual = 0.0;
    double* G = malloc( sizeof( double ) * nS * nQ );
    double* rhs = malloc( sizeof( double ) * m );
    for( int step = 0; step < n_steps; ++step ) {
        residual = 0.0;
        for( int j = 0; j < N; ++j ) fails += solve_closure( h, h->lam + j * m, h->u + j * m, h->nTLevel[h->level[j]], NULL ) != 0;
        memcpy( h->uOld, h->u, sizeof( double ) * N * m );
        for( int j = 0; j < N; ++j ) {
            double L[MAXS], y[MAXS];
            for( int k = 0; k < nQ; ++k ) {
                eval_lambda( h, h->lam + j * m, k, h->nTLevel[h->level[j]], L );
                ansatz_u( h, L, y, 0 );
                for( int s = 0; s < nS; ++s ) h->uQ[( (size_t)j * nS + s ) * nQ + k] = y[s];
            }
        }
        if( h->nLevels > 1 )
            for( int j = 0; j < N; ++j ) {
                double ind = ref_indicator( h, h->u + j * m, h->level[j] );
                int cap    = h->levelCap < h->nLevels - 1 ? h->levelCap : h->nLevels - 1;
                if( (int)h->level[j] > cap )
                    h->level[j] = (unsigned)cap;
                else if( ind > h->cfg.ref_up && (int)h->level[j] < cap )
                    h->level[j] += 1;
                else if( ind < h->cfg.ref_down && h->level[j] > 0 )
                    h->level[j] -= 1;
            }
        for( int j = 0; j < N; ++j ) {
            double* u = h->u + j * m;
            int nTj   = h->nTLevel[h->level[j]];
            memset( u, 0, sizeof( double ) * m );
            for( int s = 0; s < nS; ++s )
                for( int i = 0; i < nTj; ++i ) {
                    double a = 0.0;
                    for( int k = 0; k < nQ; ++k ) a += h->uQ[( (size_t)j * nS + s ) * nQ + k] * h->phiWf[k * nT + i];
                    u[s * nT + i] = a;
                }
        }
        double dtMin = 1e10;
        for( int j = 0; j < N; ++j ) {
            double d = compute_dt( h, h->uQ + (size_t)j * nS * nQ, h->maxEdge[j] / h->area[j] );
            if( d < dtMin ) dtMin = d;
        }
        dt = dtMin;
        h->t += dt;
        for( int j = 0; j < N; ++j ) {
            double* un      = h->uNew + j * m;
            const double* u = h->u + j * m;
            if( h->bnd[j] == 1 ) {
                memcpy( un, u, sizeof( double ) * m );
                continue;
            }
            /* wall cells: ghost states at each node (expliciteuler.cpp:24-58) */
            const int wall = h->bnd[j] >= 2 && nS == 4;
            int nTj = h->nTLevel[h->level[j]];
            memset( rhs, 0, sizeof( double ) * m );
            for( int f = 0; f < F; ++f ) {
                int nb           = h->nbr[j * F + f];
                const double* ua = h->uQ + (size_t)j * nS * nQ;
                const double* ub = h->uQ + (size_t)nb * nS * nQ;
                for( int k = 0; k < nQ; ++k ) {
                    double a[MAXS], b[MAXS], y[MAXS];
                    for( int s = 0; s < nS; ++s ) {
                        a[s] = ua[s * nQ + k];
                        b[s] = ub[s * nQ + k];
                    }
                    if( wall && nb == N ) {
                        /* flux G(ghost, ghost) on the cell's ghost faces (:62-66) */
                        const double* n = h->bndN + 2 * j;
                        double v0 = a[1] / a[0], v1 = a[2] / a[0];
                        double vn = n[0] * v0 + n[1] * v1;
                        double b0 = -( vn * n[0] ) + v0, b1 = -( vn * n[1] ) + v1;
                        double rho = a[0];
                        a[1]       = rho * b0;
                        a[2]       = rho * b1;
                        if( h->bnd[j] == 2 ) a[3] += rho * 0.5 * ( ( b0 * b0 + b1 * b1 ) - ( v0 * v0 + v1 * v1 ) );
                        for( int s = 0; s < nS; ++s ) b[s] = a[s];
                    }
                    num_flux( h, a, b, h->unitN + ( j * F + f ) * 2, h->scaledN + ( j * F + f ) * 2, y );
                    for( int s = 0; s < nS; ++s ) G[s * nQ + k] = y[s];
                }
                for( int s = 0; s < nS; ++s )
                    for( int i = 0; i < nTj; ++i )
                        for( int k = 0; k < nQ; ++k ) rhs[s * nT + i] += G[s * nQ + k] * h->phiWf[k * nT + i];
            }
            double c = dt / h->area[j];
            for( size_t r = 0; r < m; ++r ) un[r] = u[r] - rhs[r] * c;
        }
        memcpy( h->u, h->uNew, sizeof( double ) * N * m );
        for( int j = 0; j < N; ++j ) residual += fabs( h->u[j * m] - h->uOld[j * m] ) * h->area[j];
        if( h->cfg.n_ret_levels > 0 ) {
            while( h->retIndex < h->cfg.n_ret_levels - 1 && residual < h->cfg.ret_res[h->retIndex] ) ++h->retIndex;
            h->levelCap = h->cfg.ret_lev[h->retIndex];
        }
    }
    free( G );
    free( rhs );
    out[0] = h->t;
    out[1] = dt;
    out[2] = residual;
    out[3] = fails;
    return fails;
}

/* MomentSolver::WriteMeanAndVar (momentsolver.cpp:302-328). */
void uqco_mean_var( const uqco* h, double* out ) {
    int nS = h->nS, nT = h->nT;
    size_t m = (size_t)nS * nT;
    double L[MAXS], y[MAXS];
    for( int j = 0; j < h->nCells; ++j ) {
        double* mv = out + (size_t)j * 2 * nS;
        int nTj    = h->nTLevel[h->level[j]];
        for( int r = 0; r < 2 * nS; ++r ) mv[r] = 0.0;
        for( int k = 0; k < h->nQ; ++k ) {
            eval_lambda( h, h->lam + j * m, k, nTj, L );
            ansatz_u( h, L, y, 1 );
            for( int i = 0; i < nS; ++i ) mv[i] += y[i] * h->phiWf[k * nT + 0];
        }
        for( int k = 0; k < h->nQ; ++k ) {
            eval_lambda( h, h->lam + j * m, k, nTj, L );
            ansatz_u( h, L, y, 1 );
            for( int i = 0; i < nS; ++i ) mv[i + nS] += pow( y[i] - mv[i], 2 ) * h->phiWf[k * nT + 0];
        }
    }
}

void uqco_ansatz( const uqco* h, const double* Lambda, double* u, double* du, int matrix_form ) {
    if( u ) ansatz_u( h, Lambda, u, !matrix_form );
    if( du ) ansatz_du( h, Lambda, du );
}

void uqco_entropy_grad( const uqco* h, const double* u, double* ds ) { entropy_grad( h, u, ds ); }
