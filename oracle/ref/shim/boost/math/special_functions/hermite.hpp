// Test-infrastructure shim for boost::math::hermite (third-party, unpinned).
// Only needed so hermite.cpp compiles; no hot-path configuration uses a
// Hermite basis. Physicists' recurrence H_{n+1} = 2x H_n - 2n H_{n-1}.
#pragma once
#include <utility>

namespace boost {
namespace math {
inline double hermite( unsigned n, double x ) {
    double h0 = 1.0, h1 = 2.0 * x;
    if( n == 0 ) return h0;
    for( unsigned k = 1; k < n; ++k ) {
        std::swap( h0, h1 );
        h1 = 2.0 * x * h0 - 2.0 * double( k ) * h1;
    }
    return h1;
}
}    // namespace math
}    // namespace boost
