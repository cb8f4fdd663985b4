// Basis and quadrature tables of the IPM closure, computed on the host once
// per solver and uploaded to HBM. Built with -ffp-contract=off so the tables
// are bit-identical to the reference's (checked by tests/test_host_core.py).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "host.h"

namespace uqc {
namespace {

// hypot without overflow, the form of MathTools::Pythag (mathtools.cpp:3-7).
double pythag( double a, double b ) {
    double absa = std::fabs( a ), absb = std::fabs( b );
    if( absa > absb ) return absa * std::sqrt( 1.0 + std::pow( absb / absa, 2 ) );
    return absb == 0.0 ? 0.0 : absb * std::sqrt( 1.0 + std::pow( absa / absb, 2 ) );
}

// Eigen-decomposition of the symmetric tridiagonal Jacobi matrix by implicit
// QL iterations (the algorithm of MathTools::ComputeEigenValTriDiagMatrix,
// mathtools.cpp:41-104). d: diagonal -> eigenvalues, e: sub-diagonal (e[0]
// unused), z: row-major eigenvectors (columns).
void jacobi_eigen( int n, std::vector<double>& d, std::vector<double>& e, std::vector<double>& z ) {
    const double eps = 2.220446049250313e-16;
    for( int i = 1; i < n; ++i ) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    for( int l = 0; l < n; ++l ) {
        int iter = 0, m;
        do {
            for( m = l; m < n - 1; ++m ) {
                double dd = std::fabs( d[m] ) + std::fabs( d[m + 1] );
                if( std::fabs( e[m] ) <= eps * dd ) break;
            }
            if( m == l ) break;
            if( iter++ == 30 ) throw ConfigError( "Gauss-Legendre eigenvalue iteration did not converge" );
            double g = ( d[l + 1] - d[l] ) / ( 2.0 * e[l] );
            double r = pythag( g, 1.0 );
            g        = d[m] - d[l] + e[l] / ( g + std::copysign( r, g ) );
            double s = 1.0, c = 1.0, p = 0.0;
            int i;
            for( i = m - 1; i >= l; --i ) {
                double f = s * e[i], b = c * e[i];
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
                for( int k = 0; k < n; ++k ) {
                    double fk        = z[k * n + i + 1];
                    z[k * n + i + 1] = s * z[k * n + i] + c * fk;
                    z[k * n + i]     = c * z[k * n + i] - s * fk;
                }
            }
            if( r == 0.0 && i >= l ) continue;
            d[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        } while( m != l );
    }
}

// Legendre polynomial by the three-term recurrence.
double legendre( int m, double x ) {
    double p0 = 1.0, p1 = x;
    if( m == 0 ) return p0;
    for( unsigned n = 1; n < unsigned( m ); ++n ) {
        double next = ( ( 2.0 * n + 1.0 ) * x * p1 - double( n ) * p0 ) / double( n + 1 );
        p0          = p1;
        p1          = next;
    }
    return p1;
}

unsigned ipow( unsigned b, unsigned e ) { return unsigned( std::pow( b, e ) ); }

}    // namespace

// Golub-Welsch: nodes = eigenvalues of the Jacobi matrix with off-diagonal
// sqrt(1 / (4 - 1/i^2)), weights = 2 v_0^2, sorted by node (legendre.cpp:9-28).
void gauss_legendre( int n, std::vector<double>& x, std::vector<double>& w ) {
    std::vector<double> d( n, 0.0 ), e( n, 0.0 ), z( size_t( n ) * n, 0.0 );
    for( int i = 0; i < n; ++i ) {
        z[size_t( i ) * n + i] = 1.0;
        if( i > 0 ) e[i] = std::sqrt( 1 / ( 4 - 1 / std::pow( double( i ), 2 ) ) );
    }
    jacobi_eigen( n, d, e, z );
    std::vector<double> xs( n ), ws( n );
    for( int i = 0; i < n; ++i ) {
        xs[i] = std::fabs( d[i] ) < 1e-15 ? 0 : d[i];
        ws[i] = 2 * std::pow( z[i], 2 );
    }
    std::vector<int> order( n );
    std::iota( order.begin(), order.end(), 0 );
    std::sort( order.begin(), order.end(), [&]( int a, int b ) { return xs[a] < xs[b]; } );
    x.resize( n );
    w.resize( n );
    for( int i = 0; i < n; ++i ) {
        x[i] = xs[order[i]];
        w[i] = ws[order[i]];
    }
}

Tables build_tables( const Config& c ) {
    Tables t;
    t.dimXi = c.dimXi;
    // Index set: degrees of every basis function, ordered by refinement level
    // so that level l uses the first nTLevel[l] functions (settings.cpp:241-265).
    const unsigned nMom = unsigned( c.degrees.back() );
    int previous        = -1;
    for( size_t level = 0; level < c.degrees.size(); ++level ) {
        for( unsigned i = 0; i < std::pow( nMom + 1, c.dimXi ); ++i ) {
            int total = 0;
            int deg[4];
            for( int l = 0; l < c.dimXi; ++l ) {
                deg[l] = int( ( ( i - i % ipow( nMom + 1, l ) ) / ipow( nMom + 1, l ) ) % ( nMom + 1 ) );
                total += deg[l];
            }
            if( ( unsigned( total ) <= unsigned( c.degrees[level] ) && total > previous ) || c.maxDegree )
                for( int l = 0; l < c.dimXi; ++l ) t.index.push_back( deg[l] );
        }
        t.nTLevel.push_back( int( t.index.size() ) / c.dimXi );
        if( c.maxDegree ) break;
        previous = c.degrees[level];
    }
    t.nLevels = int( t.nTLevel.size() );
    t.nT      = t.nTLevel.back();
    // Tensor Gauss grid: node k has 1-D index (k / n^l) mod n in dimension l
    // (tensorizedquadrature.cpp:27-74).
    std::vector<double> x1, w1;
    gauss_legendre( c.nQuad, x1, w1 );
    t.nQ = int( unsigned( std::pow( c.nQuad, c.dimXi ) ) );
    t.xi.assign( size_t( t.nQ ) * c.dimXi, 0.0 );
    t.w.assign( t.nQ, 1.0 );
    for( int k = 0; k < t.nQ; ++k )
        for( int l = 0; l < c.dimXi; ++l ) {
            unsigned q               = unsigned( ( k - k % ipow( c.nQuad, l ) ) / ipow( c.nQuad, l ) ) % unsigned( c.nQuad );
            t.xi[size_t( k ) * c.dimXi + l] = x1[q];
            t.w[k] *= w1[q];
        }
    // phiTilde(k, i) = prod_l P_{deg}(xi_kl) / ||P_deg||, ||P_m|| = sqrt(1/(2m+1));
    // phiTildeWf = prod_l (P/||P|| * f_Xi) * w_k with f_Xi = 1/2 (closure.cpp:49-64).
    t.phi.assign( size_t( t.nQ ) * t.nT, 1.0 );
    t.phiWf.assign( size_t( t.nQ ) * t.nT, 1.0 );
    for( int k = 0; k < t.nQ; ++k )
        for( int i = 0; i < t.nT; ++i ) {
            double p = 1.0, pw = 1.0;
            for( int l = 0; l < c.dimXi; ++l ) {
                int m       = t.index[size_t( i ) * c.dimXi + l];
                double v    = legendre( m, t.xi[size_t( k ) * c.dimXi + l] );
                double norm = std::sqrt( 1.0 / ( 2.0 * m + 1.0 ) );
                p *= v / norm;
                pw *= v / norm * 0.5;
            }
            t.phi[size_t( k ) * t.nT + i]   = p;
            t.phiWf[size_t( k ) * t.nT + i] = pw * t.w[k];
        }
    return t;
}

}    // namespace uqc
