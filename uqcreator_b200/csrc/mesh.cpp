// Meshes of the hot-path workloads: the reference's uniform 1-D grid and the
// seeded jittered triangle mesh, with cell geometry computed as the
// reference's Line / Triangle classes compute it. Built with
// -ffp-contract=off so the geometry is bit-identical to the reference's.
#include <algorithm>
#include <cmath>

#include "host.h"

namespace uqc {

// Mesh1D + Line (mesh1d.cpp:5-67, line.cpp:3-44): N cells on [a, b], nodes
// a + i (b - a) / N; the "centre" is the left node; maxEdge = dx^2 so that
// maxEdge / area = dx; faces (j-1, -1) and (j+1, +1) of length 1; the two end
// cells are Dirichlet with ghost neighbours.
Mesh build_mesh_1d( int N, double a, double b ) {
    Mesh m;
    m.dim = 1;
    m.nCells = N;
    m.nFaces = 2;
    m.area.resize( N );
    m.maxEdge.resize( N );
    m.center.assign( 2 * size_t( N ), 0.0 );
    m.unitN.assign( 4 * size_t( N ), 0.0 );
    m.scaledN.assign( 4 * size_t( N ), 0.0 );
    m.nbr.resize( 2 * size_t( N ) );
    m.boundary.resize( N );
    for( int j = 0; j < N; ++j ) {
        double x0 = a + j * ( b - a ) / ( N ), x1 = a + ( j + 1 ) * ( b - a ) / ( N );
        m.area[j]           = std::fabs( x1 - x0 );
        m.maxEdge[j]        = std::pow( m.area[j], 2 );
        m.center[2 * j]     = ( x0 + x0 ) / 2;
        m.unitN[4 * j]      = -1.0;
        m.unitN[4 * j + 2]  = 1.0;
        m.scaledN[4 * j]    = -1.0;
        m.scaledN[4 * j + 2] = 1.0;
        m.boundary[j]       = ( j == 0 || j == N - 1 ) ? 1 : 0;
        m.nbr[2 * j]        = m.boundary[j] ? N : j - 1;
        m.nbr[2 * j + 1]    = m.boundary[j] ? N : j + 1;
    }
    m.nodeXY.assign( 2 * size_t( N + 1 ), 0.0 );
    for( int j = 0; j <= N; ++j ) m.nodeXY[2 * j] = a + j * ( b - a ) / ( N );
    m.cellNodes.resize( 2 * size_t( N ) );
    for( int j = 0; j < N; ++j ) {
        m.cellNodes[2 * j]     = j;
        m.cellNodes[2 * j + 1] = j + 1;
    }
    return m;
}

namespace {
uint64_t splitmix64( uint64_t x ) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z          = ( z ^ ( z >> 30 ) ) * 0xBF58476D1CE4E5B9ull;
    z          = ( z ^ ( z >> 27 ) ) * 0x94D049BB133111EBull;
    return z ^ ( z >> 31 );
}
double unit( uint64_t key ) { return double( splitmix64( key ) >> 11 ) * 0x1.0p-53; }
}    // namespace

// Nodes (i, j), id j (nx+1) + i: interior nodes at ((i + a rx)/nx, (j + a ry)/ny),
// r = 2 U - 1 with U = SplitMix64(seed 2^32 + 2 id + c) / 2^64; boundary nodes
// on the grid. Rectangle (i, j) = corners a, b = a+1, c = a+nx+2, d = a+nx+1
// splits into (a,b,c),(a,c,d), except the top-left and bottom-right corner
// rectangles, which split into (a,b,d),(b,c,d) so that no triangle has three
// boundary nodes. Triangle id 2 (j nx + i) + t.
void tri_jitter_nodes( int nx, int ny, double jitter, uint64_t seed, double* xy, int* bnd, int* tri ) {
    for( int j = 0; j <= ny; ++j )
        for( int i = 0; i <= nx; ++i ) {
            long id  = long( j ) * ( nx + 1 ) + i;
            bool b   = i == 0 || i == nx || j == 0 || j == ny;
            bnd[id]  = b ? 1 : 0;
            uint64_t key = seed * ( uint64_t( 1 ) << 32 ) + 2 * uint64_t( id );
            double fx = double( i ), fy = double( j );
            xy[2 * id]     = b ? fx / nx : ( fx + jitter * ( 2.0 * unit( key ) - 1.0 ) ) / nx;
            xy[2 * id + 1] = b ? fy / ny : ( fy + jitter * ( 2.0 * unit( key + 1 ) - 1.0 ) ) / ny;
        }
    for( int j = 0; j < ny; ++j )
        for( int i = 0; i < nx; ++i ) {
            long r  = long( j ) * nx + i;
            int a   = j * ( nx + 1 ) + i, b = a + 1, c = a + nx + 2, d = a + nx + 1;
            bool fl = ( i == 0 && j == ny - 1 ) || ( i == nx - 1 && j == 0 );
            int* t  = tri + 6 * r;
            if( fl ) {
                t[0] = a; t[1] = b; t[2] = d;
                t[3] = b; t[4] = c; t[5] = d;
            }
            else {
                t[0] = a; t[1] = b; t[2] = c;
                t[3] = a; t[4] = c; t[5] = d;
            }
        }
}

// Triangle geometry (triangle.cpp:3-70): area |x0(y1-y2)+x1(y2-y0)+x2(y0-y1)|/2,
// centroid, edges (n0,n1),(n1,n2),(n2,n0), outward unit normal of each edge
// (normalised twice, as the reference does), scaled normal = length * unit,
// maxEdge = longest edge. Neighbour across edge l = the other triangle sharing
// its two nodes (Mesh2D::DetermineNeighbors/AddNeighbor, mesh2d.cpp:282-346),
// found here by sorting edge keys. A triangle with exactly two boundary nodes
// is a (Dirichlet) boundary cell.
Mesh build_mesh_tri( int nNodes, const double* xy, const int* bnd, int N, const int* tri ) {
    Mesh m;
    m.dim    = 2;
    m.nCells = N;
    m.nFaces = 3;
    m.area.resize( N );
    m.maxEdge.resize( N );
    m.center.resize( 2 * size_t( N ) );
    m.unitN.resize( 6 * size_t( N ) );
    m.scaledN.resize( 6 * size_t( N ) );
    m.nbr.assign( 3 * size_t( N ), N );
    m.boundary.resize( N );
    for( int c = 0; c < N; ++c ) {
        double X[3], Y[3];
        int nb = 0;
        for( int v = 0; v < 3; ++v ) {
            X[v] = xy[2 * tri[3 * c + v]];
            Y[v] = xy[2 * tri[3 * c + v] + 1];
            nb += bnd[tri[3 * c + v]] != 0;
        }
        m.boundary[c] = nb == 2;
        m.area[c]     = std::fabs( ( X[0] * ( Y[1] - Y[2] ) + X[1] * ( Y[2] - Y[0] ) + X[2] * ( Y[0] - Y[1] ) ) / 2 );
        double cx = ( X[0] + X[1] + X[2] ) / 3, cy = ( Y[0] + Y[1] + Y[2] ) / 3;
        m.center[2 * c]     = cx;
        m.center[2 * c + 1] = cy;
        double mx           = -1e10;
        for( int e = 0; e < 3; ++e ) {
            int A = e, B = ( e + 1 ) % 3;
            double len = std::sqrt( std::pow( X[A] - X[B], 2 ) + std::pow( Y[A] - Y[B], 2 ) );
            double n0 = -( Y[A] - Y[B] ), n1 = X[A] - X[B];
            if( ( 0.0 + n0 * ( cx - X[A] ) ) + n1 * ( cy - Y[A] ) > 0 ) {
                n0 *= -1.0;
                n1 *= -1.0;
            }
            for( int rep = 0; rep < 2; ++rep ) {
                double nn = std::sqrt( ( 0.0 + std::fabs( n0 ) * std::fabs( n0 ) ) + std::fabs( n1 ) * std::fabs( n1 ) );
                n0 /= nn;
                n1 /= nn;
            }
            m.unitN[6 * c + 2 * e]       = n0;
            m.unitN[6 * c + 2 * e + 1]   = n1;
            m.scaledN[6 * c + 2 * e]     = len * n0;
            m.scaledN[6 * c + 2 * e + 1] = len * n1;
            if( mx < len ) mx = len;
        }
        m.maxEdge[c] = mx;
    }
    std::vector<std::pair<long long, long long>> keys( 3 * size_t( N ) );
    for( int c = 0; c < N; ++c )
        for( int l = 0; l < 3; ++l ) {
            long long a = tri[3 * c + l], b = tri[3 * c + ( l + 1 ) % 3];
            keys[3 * size_t( c ) + l] = {std::min( a, b ) * ( nNodes + 1LL ) + std::max( a, b ), 3LL * c + l};
        }
    std::sort( keys.begin(), keys.end() );
    for( size_t i = 0; i + 1 < keys.size(); ++i )
        if( keys[i].first == keys[i + 1].first ) {
            m.nbr[keys[i].second]     = int( keys[i + 1].second / 3 );
            m.nbr[keys[i + 1].second] = int( keys[i].second / 3 );
            ++i;
        }
    m.nodeXY.assign( xy, xy + 2 * size_t( nNodes ) );
    m.cellNodes.assign( tri, tri + 3 * size_t( N ) );
    return m;
}

}    // namespace uqc
