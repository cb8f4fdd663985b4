// Test-infrastructure shim for boost::math::legendre_p (Boost is a third-party
// dependency of the reference, version unpinned: no manifest in the reference).
// Called at legendre.cpp:30 to tabulate the basis at the quadrature nodes.
// Restates Boost's published algorithm: the Bonnet three-term recurrence
//   P_0 = 1, P_1 = x, P_{n+1} = ((2n+1) x P_n - n P_{n-1}) / (n+1),
// evaluated upward from n = 1 exactly as boost::math::legendre_next does.
#pragma once
#include <utility>

namespace boost {
namespace math {
inline double legendre_p( int l, double x ) {
    if( l < 0 ) l = -l - 1;
    double p0 = 1.0, p1 = x;
    if( l == 0 ) return p0;
    unsigned n = 1;
    while( n < unsigned( l ) ) {
        std::swap( p0, p1 );
        p1 = ( ( 2.0 * n + 1.0 ) * x * p0 - double( n ) * p1 ) / double( n + 1 );
        ++n;
    }
    return p1;
}
}    // namespace math
}    // namespace boost
