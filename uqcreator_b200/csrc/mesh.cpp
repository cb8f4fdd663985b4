// Meshes of the hot-path workloads: the reference's uniform 1-D grid and the
// seeded jittered triangle mesh, with cell geometry computed as the
// reference's Line / Triangle classes compute it. Built with
// -ffp-contract=off so the geometry is bit-identical to the reference's.
#include <algorithm>
#include <cmath>

#include "host.h"

#include <cctype>
#include <fstream>
#include <map>
#include <sstream>

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

// Cell::UpdateBoundaryNormal (cell.cpp:57-68): the unit normal of the face
// with the largest neighbour id (the ghost face), first such face on ties.
void set_boundary_normals( Mesh& m ) {
    m.bndNormal.assign( 2 * size_t( m.nCells ), 0.0 );
    for( int c = 0; c < m.nCells; ++c ) {
        int id = 0;
        for( int f = 1; f < m.nFaces; ++f )
            if( m.nbr[size_t( c ) * m.nFaces + f] > m.nbr[size_t( c ) * m.nFaces + id] ) id = f;
        m.bndNormal[2 * c]     = m.unitN[( size_t( c ) * m.nFaces + id ) * 2];
        m.bndNormal[2 * c + 1] = m.unitN[( size_t( c ) * m.nFaces + id ) * 2 + 1];
    }
}

namespace {
// Mesh2D::GetTrailingNumber (mesh2d.cpp:261-263): the number from the first digit on.
unsigned trailing_number( const std::string& line ) {
    const size_t p = line.find_first_of( "0123456789" );
    if( p == std::string::npos ) throw ConfigError( "[mesh2d] no number in '" + line + "'" );
    return unsigned( std::stoul( line.substr( p ) ) );
}
}    // namespace

// The reader follows mesh2d.cpp:68-259: NPOIN lines "x y id" (nodes sorted by
// id), NMARK markers (MARKER_TAG, MARKER_ELEMS with line elements "3 a b";
// their nodes are boundary nodes), NELEM lines "5 a b c id" (triangles;
// quadrangles are refused). A triangle with two boundary nodes is a boundary
// cell; its code is that of the last marker (in file order) holding one of
// its nodes as the first or second node of an element, scanning the cell's
// nodes in order (:197-211). Neighbours come from sorted edge keys
// (O(N log N), instead of the reference's O(N^2) pair search).
Mesh read_su2_mesh( const std::string& path, const std::vector<std::pair<std::string, int>>& bcs ) {
    std::ifstream f( path );
    if( !f ) throw ConfigError( "[mesh2d] File not found: " + path );
    std::vector<std::string> lines;
    for( std::string l; std::getline( f, l ); ) {
        if( !l.empty() && l.back() == '\r' ) l.pop_back();
        lines.push_back( l );
    }
    auto find = [&]( const char* key ) -> size_t {
        for( size_t i = 0; i < lines.size(); ++i )
            if( lines[i].find( key ) != std::string::npos ) return i;
        throw ConfigError( std::string( "[mesh2d] " ) + key + " not found in " + path );
    };
    if( trailing_number( lines[find( "NDIME" )] ) != 2 ) throw ConfigError( "[mesh2d] NDIME must be 2" );
    // nodes
    size_t at           = find( "NPOIN" );
    const unsigned nPts = trailing_number( lines[at] );
    std::vector<std::pair<unsigned, std::pair<double, double>>> pts( nPts );
    for( unsigned i = 0; i < nPts; ++i ) {
        if( at + 1 + i >= lines.size() ) throw ConfigError( "[mesh2d] truncated NPOIN section" );
        std::stringstream ss( lines[at + 1 + i] );
        double x = 0, y = 0;
        unsigned id = i;
        ss >> x >> y;
        if( !( ss >> id ) ) id = i;
        pts[i] = {id, {x, y}};
    }
    std::sort( pts.begin(), pts.end(), []( const auto& a, const auto& b ) { return a.first < b.first; } );
    std::map<unsigned, int> index;
    std::vector<double> xy( 2 * size_t( nPts ) );
    for( unsigned i = 0; i < nPts; ++i ) {
        index[pts[i].first] = int( i );
        xy[2 * i]           = pts[i].second.first;
        xy[2 * i + 1]       = pts[i].second.second;
    }
    auto node = [&]( unsigned id ) {
        auto it = index.find( id );
        if( it == index.end() ) throw ConfigError( "[mesh2d] unknown node id " + std::to_string( id ) );
        return it->second;
    };
    // markers
    std::vector<int> bnd( nPts, 0 );
    struct Marker {
        int code;
        std::vector<std::pair<int, int>> elems;
    };
    std::vector<Marker> markers;
    at                  = find( "NMARK" );
    const unsigned nMrk = trailing_number( lines[at] );
    size_t k            = at + 1;
    for( unsigned m = 0; m < nMrk; ++m ) {
        std::string tag;
        Marker mk{0, {}};
        for( int part = 0; part < 2; ++part, ++k ) {
            if( k >= lines.size() ) throw ConfigError( "[mesh2d] truncated NMARK section" );
            const std::string& l = lines[k];
            if( l.find( "MARKER_TAG" ) != std::string::npos ) {
                tag = l.substr( l.find( '=' ) + 1 );
                tag.erase( std::remove_if( tag.begin(), tag.end(), ::isspace ), tag.end() );
            }
            else if( l.find( "MARKER_ELEMS" ) != std::string::npos ) {
                const unsigned ne = trailing_number( l );
                for( unsigned e = 0; e < ne; ++e ) {
                    std::stringstream ss( lines.at( k + 1 + e ) );
                    unsigned type = 0, a = 0, b = 0;
                    ss >> type >> a >> b;
                    const int ia = node( a ), ib = node( b );
                    bnd[ia] = bnd[ib] = 1;
                    mk.elems.emplace_back( ia, ib );
                }
                k += ne;
            }
            else {
                throw ConfigError( "[mesh2d] expected MARKER_TAG / MARKER_ELEMS at line " + std::to_string( k + 1 ) );
            }
        }
        for( const auto& b : bcs )
            if( b.first == tag ) mk.code = b.second;
        if( mk.code == 0 ) throw ConfigError( "[mesh2d] no SU2BC entry for marker '" + tag + "'" );
        markers.push_back( std::move( mk ) );
    }
    // cells
    at                  = find( "NELEM" );
    const unsigned nEl  = trailing_number( lines[at] );
    std::vector<int> tri( 3 * size_t( nEl ) );
    for( unsigned c = 0; c < nEl; ++c ) {
        std::stringstream ss( lines.at( at + 1 + c ) );
        unsigned type = 0, a = 0, b = 0, d = 0;
        ss >> type;
        if( type != 5 ) throw ConfigError( "[mesh2d] element type " + std::to_string( type ) + " is not supported (triangles only)" );
        ss >> a >> b >> d;
        unsigned id = c;
        if( ( ss >> id ) && id != c ) throw ConfigError( "[mesh2d] element " + std::to_string( c ) + " carries id " + std::to_string( id ) + "; ids must follow file order" );
        tri[3 * c]     = node( a );
        tri[3 * c + 1] = node( b );
        tri[3 * c + 2] = node( d );
    }
    Mesh m = build_mesh_tri( int( nPts ), xy.data(), bnd.data(), int( nEl ), tri.data() );
    for( int c = 0; c < m.nCells; ++c ) {
        if( !m.boundary[c] ) continue;
        int code = BC_DIRICHLET;
        for( int v = 0; v < 3; ++v ) {
            const int nid = tri[3 * c + v];
            for( const Marker& mk : markers )
                for( const auto& e : mk.elems )
                    if( e.first == nid || e.second == nid ) code = mk.code;
        }
        m.boundary[c] = code;
    }
    set_boundary_normals( m );
    return m;
}

namespace {
void bisect( const Mesh& m, std::vector<int>& cells, size_t lo, size_t hi, int r0, int r1, std::vector<int>& owner ) {
    if( r1 - r0 <= 1 ) {
        for( size_t i = lo; i < hi; ++i ) owner[cells[i]] = r0;
        return;
    }
    double ext[2];
    for( int d = 0; d < 2; ++d ) {
        double a = 1e300, b = -1e300;
        for( size_t i = lo; i < hi; ++i ) {
            const double x = m.center[2 * size_t( cells[i] ) + d];
            a              = std::min( a, x );
            b              = std::max( b, x );
        }
        ext[d] = hi > lo ? b - a : 0.0;
    }
    const int d = ext[1] > ext[0] ? 1 : 0;
    std::sort( cells.begin() + lo, cells.begin() + hi, [&]( int p, int q ) {
        const double a = m.center[2 * size_t( p ) + d], b = m.center[2 * size_t( q ) + d];
        return a < b || ( a == b && p < q );
    } );
    const int nl     = ( r1 - r0 ) / 2;
    const size_t mid = lo + size_t( ( (long long)( hi - lo ) * nl ) / ( r1 - r0 ) );
    bisect( m, cells, lo, mid, r0, r0 + nl, owner );
    bisect( m, cells, mid, hi, r0 + nl, r1, owner );
}
}    // namespace

std::vector<int> partition_cells( const Mesh& m, int nRanks ) {
    std::vector<int> owner( m.nCells, 0 ), cells( m.nCells );
    for( int c = 0; c < m.nCells; ++c ) cells[c] = c;
    bisect( m, cells, 0, cells.size(), 0, std::max( nRanks, 1 ), owner );
    return owner;
}

Mesh shard_mesh( const Mesh& g, const std::vector<int>& owner, int rank, int nRanks, ShardPlan& plan ) {
    const int N = g.nCells, F = g.nFaces;
    plan           = ShardPlan{};
    plan.rank      = rank;
    plan.nRanks    = nRanks;
    plan.nGlobal   = N;
    std::vector<int>& gid = plan.globalId;
    for( int c = 0; c < N; ++c )
        if( owner[c] == rank ) gid.push_back( c );
    plan.nOwned = int( gid.size() );
    // halo: neighbours of owned cells owned elsewhere, by (owner, global id)
    std::vector<std::pair<int, int>> halo;
    for( int i = 0; i < plan.nOwned; ++i )
        for( int f = 0; f < F; ++f ) {
            const int nb = g.nbr[size_t( gid[i] ) * F + f];
            if( nb < N && owner[nb] != rank ) halo.push_back( {owner[nb], nb} );
        }
    std::sort( halo.begin(), halo.end() );
    halo.erase( std::unique( halo.begin(), halo.end() ), halo.end() );
    for( const auto& h : halo ) gid.push_back( h.second );
    const int L = int( gid.size() );
    std::vector<int> local( N, -1 );
    for( int i = 0; i < L; ++i ) local[gid[i]] = i;
    // sends: owned cells that neighbour a cell of peer p, in global order
    std::map<int, std::vector<int>> send;
    for( int c = 0; c < N; ++c ) {
        const int p = owner[c];
        if( p == rank ) continue;
        for( int f = 0; f < F; ++f ) {
            const int nb = g.nbr[size_t( c ) * F + f];
            if( nb < N && owner[nb] == rank ) send[p].push_back( nb );
        }
    }
    std::map<int, int> recv;
    for( const auto& h : halo ) ++recv[h.first];
    std::vector<int> peers;
    for( const auto& kv : send ) peers.push_back( kv.first );
    for( const auto& kv : recv ) peers.push_back( kv.first );
    std::sort( peers.begin(), peers.end() );
    peers.erase( std::unique( peers.begin(), peers.end() ), peers.end() );
    for( int p : peers ) {
        std::vector<int>& s = send[p];
        std::sort( s.begin(), s.end() );
        s.erase( std::unique( s.begin(), s.end() ), s.end() );
        plan.peers.push_back( p );
        plan.sendCount.push_back( int( s.size() ) );
        plan.recvCount.push_back( recv.count( p ) ? recv[p] : 0 );
        for( int c : s ) plan.sendCells.push_back( local[c] );
    }
    // the local mesh: per-cell data copied, neighbours renumbered
    Mesh m;
    m.dim    = g.dim;
    m.nCells = L;
    m.nFaces = F;
    m.area.resize( L );
    m.maxEdge.resize( L );
    m.center.resize( 2 * size_t( L ) );
    m.unitN.resize( 2 * size_t( L ) * F );
    m.scaledN.resize( 2 * size_t( L ) * F );
    m.nbr.resize( size_t( L ) * F );
    m.boundary.resize( L );
    if( !g.bndNormal.empty() ) m.bndNormal.resize( 2 * size_t( L ) );
    for( int i = 0; i < L; ++i ) {
        const size_t c = size_t( gid[i] );
        m.area[i]         = g.area[c];
        m.maxEdge[i]      = g.maxEdge[c];
        m.center[2 * i]   = g.center[2 * c];
        m.center[2 * i + 1] = g.center[2 * c + 1];
        m.boundary[i]     = g.boundary[c];
        for( int f = 0; f < F; ++f ) {
            const size_t a = size_t( i ) * F + f, b = c * F + f;
            const int nb   = g.nbr[b];
            m.nbr[a]       = nb < N && local[nb] >= 0 ? local[nb] : L;
            for( int k = 0; k < 2; ++k ) {
                m.unitN[2 * a + k]   = g.unitN[2 * b + k];
                m.scaledN[2 * a + k] = g.scaledN[2 * b + k];
            }
        }
        if( !g.bndNormal.empty() ) {
            m.bndNormal[2 * i]     = g.bndNormal[2 * c];
            m.bndNormal[2 * i + 1] = g.bndNormal[2 * c + 1];
        }
    }
    return m;
}

}    // namespace uqc
