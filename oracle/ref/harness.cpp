// Oracle harness around the reference's OWN sources (test infrastructure).
//
// Built by oracle/ref/Makefile from UQCreator's code/src files where they lie,
// against the project-written shims in oracle/ref/shim (spdlog, cpptoml, boost
// Legendre/Hermite, single-rank MPI, LAPACK dposv_). The files that cannot be
// compiled here (mesh.cpp/mesh1d.cpp/mesh2d.cpp need VTK, boundedbarrier.cpp
// hard-codes its bounds, main.cpp needs spdlog sinks) are replaced by the
// definitions below, each citing what it restates.
//
// Exposes a C API (uqcref_*) that tests, the golden-vector script and the
// CPU-baseline leg of bench.py call through ctypes. Nothing in the product
// links or calls this file.
#include <cmath>
#include <fstream>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "boundedbarrier.h"
#include "burgers.h"
#include "closure.h"
#include "euler.h"
#include "euler2d.h"
#include "eulerclosure.h"
#include "eulerclosure2d.h"
#include "line.h"
#include "mesh.h"
#include "momentsolver.h"
#include "problem.h"
#include "settings.h"
#include "shallowwater.h"
#include "shallowwaterclosure.h"
#include "timesolver.h"
#include "triangle.h"

// ---------------------------------------------------------------------------
// Harness-wide parameters (bounded-barrier bounds are hard-coded in the
// reference, boundedbarrier.cpp:7-14; configurations need other bounds).
static double g_bbMinus = 3.0, g_bbPlus = 12.0;

// ---------------------------------------------------------------------------
// Mesh base-class members: restate mesh.cpp:5-81 (that file includes the VTK
// based Mesh1D/Mesh2D headers and cannot compile here).
Mesh::Mesh( Settings* settings, unsigned dimension ) : _settings( settings ), _dimension( dimension ), _nBoundaries( 2 ) {
    _log        = spdlog::get( "event" );
    _outputFile = _settings->GetOutputFile();
}
Mesh::~Mesh() {
    for( auto& c : _cells ) delete c;
    for( auto& n : _nodes ) delete n;
}
Mesh* Mesh::Create( Settings* ) { return nullptr; }
unsigned Mesh::GetNumCells() const { return _numCells; }
unsigned Mesh::GetDimension() const { return _dimension; }
std::vector<Cell*>& Mesh::GetGrid() { return _cells; }
std::vector<Cell*> Mesh::GetGrid() const { return _cells; }
double Mesh::GetArea( unsigned i ) const { return _cells[i]->GetArea(); }
double Mesh::GetMinEdge( unsigned i ) const { return _cells[i]->GetMinEdge(); }
double Mesh::GetMaxEdge( unsigned i ) const { return _cells[i]->GetMaxEdge(); }
std::vector<Cell*> Mesh::GetNeighbors( unsigned i ) const { return _cells[i]->GetNeighbors(); }
Vector Mesh::GetNormals( unsigned i, unsigned l ) const { return _cells[i]->GetEdges()[l]->scaledNormal; }
Vector Mesh::GetUnitNormals( unsigned i, unsigned l ) const { return _cells[i]->GetEdges()[l]->unitNormal; }
Vector Mesh::GetCenterPos( unsigned i ) const { return _cells[i]->GetCenter(); }
unsigned Mesh::GetNBoundaries() const { return _nBoundaries; }
VectorU Mesh::GetNeighborIDs( unsigned i ) const { return _neighborIDs[i]; }
BoundaryType Mesh::GetBoundaryType( unsigned i ) const { return _boundaryType[i]; }
void Mesh::PlotInXi( const Matrix&, unsigned ) const {}
double Mesh::GetDomainArea() const {
    double area = 0;
    for( unsigned j = 0; j < _cells.size(); ++j ) area += this->GetArea( j );
    return area;
}

// Captures what MomentSolver::Solve exports (momentsolver.cpp:157-158,224):
// the mean/variance matrix arrives here at full precision.
struct HarnessMeshBase : public Mesh {
    HarnessMeshBase( Settings* s, unsigned d ) : Mesh( s, d ) {}
    mutable std::map<std::string, Matrix> exported;
    std::vector<Vector> Import() const override { return {}; }
    // Boundary types of an SU2 mesh, as Mesh2D::LoadSU2MeshFromFile sets them
    // (mesh2d.cpp:197-214): each boundary cell takes its given type, and its
    // boundary normal comes from the reference's Cell::UpdateBoundaryNormal
    // (mesh2d.cpp:342-344).
    void SetCellTypes( const int* codes ) {
        static const BoundaryType types[4] = {BoundaryType::NONE, BoundaryType::DIRICHLET, BoundaryType::NOSLIP, BoundaryType::SWWALL};
        for( unsigned c = 0; c < _cells.size(); ++c ) {
            if( !_cells[c]->IsBoundaryCell() || codes[c] < 1 || codes[c] > 3 ) continue;
            _boundaryType[c] = types[codes[c]];
            _cells[c]->SetBoundaryType( types[codes[c]] );
            _cells[c]->UpdateBoundaryNormal();
        }
    }
    void Export( const Matrix& results, std::string append ) const override { exported[append] = results; }
    Vector GetNodePositionsX() const override {
        Vector x( unsigned( _nodes.size() ) );
        for( unsigned i = 0; i < _nodes.size(); ++i ) x[i] = _nodes[i]->coords[0];
        return x;
    }
};

// 1-D uniform grid: restates Mesh1D's constructor and CreateGrid
// (mesh1d.cpp:5-48,52-67): nodes a + i(b-a)/N, Line cells, neighbours
// (j-1, j+1), both end cells Dirichlet with ghost id N.
struct HarnessMesh1D : public HarnessMeshBase {
    HarnessMesh1D( Settings* s, unsigned numCells, double a, double b ) : HarnessMeshBase( s, 1 ) {
        _numCells = numCells;
        _settings->SetNumCells( _numCells );
        _cells.resize( _numCells );
        _nodes.resize( _numCells + 1 );
        for( unsigned i = 0; i < _numCells + 1; ++i )
            _nodes[i] = new Node{i, i == 0 || i == _numCells, std::vector<double>( _dimension, a + i * ( b - a ) / ( _numCells ) )};
        for( unsigned i = 0; i < _numCells; ++i ) _cells[i] = new Line( i, std::vector<Node*>{_nodes[i], _nodes[i + 1]} );
        _cells[0]->AddNeighbor( _cells[1], 1 );
        for( unsigned i = 1; i < _numCells - 1; ++i ) {
            _cells[i]->AddNeighbor( _cells[i - 1], 0 );
            _cells[i]->AddNeighbor( _cells[i + 1], 1 );
        }
        _cells[_numCells - 1]->AddNeighbor( _cells[_numCells - 2], 0 );
        _neighborIDs.resize( _numCells );
        _boundaryType.resize( _numCells );
        for( unsigned i = 1; i < _numCells - 1; ++i ) {
            _neighborIDs[i].resize( 2 );
            _neighborIDs[i][0] = i - 1;
            _neighborIDs[i][1] = i + 1;
            _boundaryType[i]   = BoundaryType::NONE;
        }
        for( unsigned e : {0u, _numCells - 1} ) {
            _neighborIDs[e].resize( 2 );
            _neighborIDs[e][0] = _numCells;
            _neighborIDs[e][1] = _numCells;
            _boundaryType[e]   = BoundaryType::DIRICHLET;
            _cells[e]->SetBoundaryType( BoundaryType::DIRICHLET );
        }
    }
};

// 2-D triangle mesh given as arrays (the reference reads SU2 files,
// mesh2d.cpp:68-259). Cells are the reference's own Triangle objects
// (triangle.cpp), so area, centre, edge lengths and outward normals are the
// reference's. Neighbour l is the cell across edge (node l, node l+1 mod 3),
// the mapping of Mesh2D::AddNeighbor (mesh2d.cpp:282-313); faces without a
// neighbour keep the ghost id N (Cell::SetDefaultCellId). Every boundary cell
// (two boundary nodes, triangle.cpp:10-16) is Dirichlet.
struct HarnessMesh2D : public HarnessMeshBase {
    HarnessMesh2D( Settings* s, unsigned nNodes, const double* xy, const int* bnd, unsigned nCells, const int* tri ) : HarnessMeshBase( s, 2 ) {
        _numCells = nCells;
        _nodes.resize( nNodes );
        for( unsigned i = 0; i < nNodes; ++i ) _nodes[i] = new Node{i, bnd[i] != 0, std::vector<double>{xy[2 * i], xy[2 * i + 1]}};
        _cells.resize( nCells );
        for( unsigned c = 0; c < nCells; ++c ) {
            _cells[c] = new Triangle( c, std::vector<Node*>{_nodes[tri[3 * c]], _nodes[tri[3 * c + 1]], _nodes[tri[3 * c + 2]]} );
            _cells[c]->SetDefaultCellId( nCells );
        }
        std::map<std::pair<int, int>, std::pair<unsigned, unsigned>> edge;    // key -> (cell, local edge)
        for( unsigned c = 0; c < nCells; ++c )
            for( unsigned l = 0; l < 3; ++l ) {
                int a = tri[3 * c + l], b = tri[3 * c + ( l + 1 ) % 3];
                auto key = std::make_pair( std::min( a, b ), std::max( a, b ) );
                auto it  = edge.find( key );
                if( it == edge.end() )
                    edge[key] = std::make_pair( c, l );
                else {
                    _cells[c]->AddNeighborId( it->second.first, l );
                    _cells[it->second.first]->AddNeighborId( c, it->second.second );
                }
            }
        _neighborIDs.resize( nCells );
        _boundaryType.resize( nCells );
        for( unsigned c = 0; c < nCells; ++c ) {
            _neighborIDs[c]  = _cells[c]->GetNeighborIDs();
            _boundaryType[c] = _cells[c]->IsBoundaryCell() ? BoundaryType::DIRICHLET : BoundaryType::NONE;
            _cells[c]->SetBoundaryType( _boundaryType[c] );
        }
        _settings->SetNumCells( _numCells );
    }
};

// ---------------------------------------------------------------------------
// BoundedBarrier with configurable bounds: restates boundedbarrier.cpp:3-80
// (the four formulas for U and DU are the reference's; only the bounds of
// :7-14 come from the harness).
BoundedBarrier::BoundedBarrier( Settings* settings ) : Closure( settings ) {
    _alpha  = 1.0;
    _uMinus = g_bbMinus;
    _uPlus  = g_bbPlus;
}
BoundedBarrier::~BoundedBarrier() {}
void BoundedBarrier::U( Vector& out, const Vector& Lambda ) {
    double ePos, eNeg;
    for( unsigned l = 0; l < _nStates; ++l ) {
        ePos = exp( Lambda[l] );
        eNeg = 1.0 / ePos;
        if( Lambda[l] > 0.0 )
            out[l] = _uPlus / ( eNeg + 1.0 ) + _uMinus * eNeg / ( 1.0 + eNeg );
        else
            out[l] = _uMinus / ( ePos + 1.0 ) + _uPlus * ePos / ( 1.0 + ePos );
    }
}
void BoundedBarrier::U( Matrix& out, const Matrix& Lambda ) {
    for( unsigned l = 0; l < _nStates; ++l )
        for( unsigned k = 0; k < Lambda.columns(); ++k ) {
            double ePos = exp( Lambda( l, k ) ), eNeg = 1.0 / ePos;
            if( Lambda( l, k ) > 0 )
                out( l, k ) = _uPlus / ( eNeg + 1.0 ) + _uMinus * eNeg / ( 1.0 + eNeg );
            else
                out( l, k ) = _uMinus / ( ePos + 1.0 ) + _uPlus * ePos / ( 1.0 + ePos );
        }
}
Matrix BoundedBarrier::U( const Matrix& Lambda ) {
    Matrix y( _nStates, Lambda.columns(), 0.0 );
    U( y, Lambda );
    return y;
}
void BoundedBarrier::DU( Matrix& y, const Vector& Lambda ) {
    for( unsigned l = 0; l < _nStates; ++l )
        for( unsigned m = 0; m < _nStates; ++m ) {
            double ePos = exp( Lambda[l] );
            double eNeg = 1 / ePos;
            if( Lambda[l] > 0 )
                y( l, m ) = eNeg * ( _uPlus - _uMinus ) / ( exp( -2.0 * Lambda[l] ) + 2.0 * eNeg + 1.0 );
            else
                y( l, m ) = ePos * ( _uPlus - _uMinus ) / ( 1.0 + 2.0 * ePos + exp( 2.0 * Lambda[l] ) );
        }
}

// ---------------------------------------------------------------------------
// Harness problems: the reference's physics with the workloads' initial data.

// 1-D Burgers with the local Lax-Friedrichs (Rusanov) flux of the Julia
// prototype (julia/Tensorization/IPMSolver.jl:38-42), written for a face
// normal n: 0.5 (f(u) + f(v)) n - 0.5 max(|u|,|v|) (v - u) |n|.
// Initial state: the reference's ramp form (burgers.cpp:48-68) with
// configurable x0, x1, uL, uR; sigma from the config.
struct HarnessBurgers : public Burgers {
    double uL, uR, x0, x1;
    HarnessBurgers( Settings* s, const double* p ) : Burgers( s ), uL( p[0] ), uR( p[1] ), x0( p[2] ), x1( p[3] ) {
        _settings->SetExactSolution( false );
    }
    Matrix G( const Matrix& u, const Matrix& v, const Vector& nUnit, const Vector& n ) override {
        (void)nUnit;
        Matrix y( u.rows(), u.columns() );
        for( unsigned k = 0; k < u.columns(); ++k ) {
            double a = u( 0, k ), b = v( 0, k );
            double beta = std::max( std::fabs( a ), std::fabs( b ) );
            y( 0, k )   = 0.5 * ( 0.5 * a * a + 0.5 * b * b ) * n[0] - 0.5 * beta * ( b - a ) * std::fabs( n[0] );
        }
        return y;
    }
    Vector IC( const Vector& x, const Vector& xi ) override {
        Vector y( 1 );
        double sigma = _settings->GetSigma( 0 );
        if( x[0] < x0 + sigma * xi[0] )
            y[0] = uL;
        else if( x[0] < x1 + sigma * xi[0] )
            y[0] = uL + ( uR - uL ) * ( x0 + sigma * xi[0] - x[0] ) / ( x0 - x1 );
        else
            y[0] = uR;
        return y;
    }
};

// 2-D Euler, the reference's HLL flux and CFL rule (euler2d.cpp:52-134) with a
// Sod-type interface: rho, p jump at x = xs + sigma_0 xi_0; left density
// rhoL (1 + sigma_1 xi_1), left pressure pL (1 + sigma_2 xi_2) when a third
// uncertainty is configured; u = v = 0.
struct HarnessEuler2D : public Euler2D {
    double xs, rhoL, pL, rhoR, pR, gam;
    HarnessEuler2D( Settings* s, const double* p ) : Euler2D( s ), xs( p[0] ), rhoL( p[1] ), pL( p[2] ), rhoR( p[3] ), pR( p[4] ), gam( s->GetGamma() ) {}
    Vector IC( const Vector& x, const Vector& xi ) override {
        Vector y( 4 );
        unsigned d = unsigned( xi.size() );
        double rho, p;
        if( x[0] < xs + _settings->GetSigma( 0 ) * xi[0] ) {
            rho = rhoL * ( 1.0 + ( d > 1 ? _settings->GetSigma( 1 ) * xi[1] : 0.0 ) );
            p   = pL * ( 1.0 + ( d > 2 ? _settings->GetSigma( 2 ) * xi[2] : 0.0 ) );
        }
        else {
            rho = rhoR;
            p   = pR;
        }
        y[0] = rho;
        y[1] = 0.0;
        y[2] = 0.0;
        y[3] = p / ( gam - 1.0 );
        return y;
    }
};

// 1-D shallow water, the reference's Lax-Friedrichs flux (shallowwater.cpp:21-55),
// dam break h = hL (1 + sigma xi) for x < xd else hR, hu = 0. The reference's
// ComputeDt is not implemented (shallowwater.cpp:69-72); the step used is the
// base-class rule Problem::ComputeDt = Settings::GetDT (problem.cpp:44), i.e.
// TimeSolver's dx CFL / 12 (timesolver.cpp:4-9), which matches the flux's
// fixed dx/dt = 12 / CFL.
struct HarnessShallowWater : public ShallowWater {
    double xd, hL, hR;
    HarnessShallowWater( Settings* s, const double* p ) : ShallowWater( s ), xd( p[0] ), hL( p[1] ), hR( p[2] ) {}
    double ComputeDt( const Matrix&, double ) const override { return _settings->GetDT(); }
    Vector IC( const Vector& x, const Vector& xi ) override {
        Vector y( 2 );
        y[0] = x[0] < xd ? hL * ( 1.0 + _settings->GetSigma( 0 ) * xi[0] ) : hR;
        y[1] = 0.0;
        return y;
    }
};

// ---------------------------------------------------------------------------
// "Guarded" Newton: Closure::SolveClosure (closure.cpp:133-193) with one change,
// the line search also halves while the trial residual norm is not finite,
// the test SolveClosureSafe applies (closure.cpp:318). The reference's own
// SolveClosure accepts such a step (:172) and then stops at the next posv.
template <class B> struct Guarded : public B {
    explicit Guarded( Settings* s ) : B( s ) {}
    void SolveClosure( Matrix& lambda, const Matrix& u, unsigned nTotal, unsigned nQTotal ) override {
        int maxRefinements = 1000;
        unsigned nS        = this->_nStates;
        double eps         = this->_settings->GetEpsilon();
        Vector g( nS * nTotal );
        this->Gradient( g, lambda, u, nTotal, nQTotal );
        if( this->CalcNorm( g, nTotal ) < eps ) return;
        Matrix H( nS * nTotal, nS * nTotal );
        Vector dlambdaNew( nS * nTotal );
        Vector dlambda = -g;
        this->Hessian( H, lambda, nTotal, nQTotal );
        posv( H, g );
        if( this->_maxIterations == 1 ) {
            this->AddMatrixVectorToMatrix( lambda, -this->_alpha * g, lambda, nTotal );
            return;
        }
        Matrix lambdaNew( nS, nTotal );
        this->AddMatrixVectorToMatrix( lambda, -this->_alpha * g, lambdaNew, nTotal );
        this->Gradient( dlambdaNew, lambdaNew, u, nTotal, nQTotal );
        for( unsigned l = 0; l < this->_maxIterations; ++l ) {
            double stepSize = 1.0;
            if( l != 0 ) {
                this->Gradient( g, lambda, u, nTotal, nQTotal );
                dlambda = -g;
                this->Hessian( H, lambda, nTotal, nQTotal );
                posv( H, g );
                this->AddMatrixVectorToMatrix( lambda, -stepSize * this->_alpha * g, lambdaNew, nTotal );
                this->Gradient( dlambdaNew, lambdaNew, u, nTotal, nQTotal );
            }
            int refinementCounter = 0;
            while( this->CalcNorm( dlambda, nTotal ) < this->CalcNorm( dlambdaNew, nTotal ) || !std::isfinite( this->CalcNorm( dlambdaNew, nTotal ) ) ) {
                stepSize *= 0.5;
                this->AddMatrixVectorToMatrix( lambda, -stepSize * this->_alpha * g, lambdaNew, nTotal );
                this->Gradient( dlambdaNew, lambdaNew, u, nTotal, nQTotal );
                if( this->CalcNorm( dlambdaNew, nTotal ) < eps ) {
                    lambda = lambdaNew;
                    return;
                }
                else if( ++refinementCounter > maxRefinements ) {
                    this->_log->error( "[closure] Newton needed too many refinement steps!" );
                }
            }
            lambda = lambdaNew;
            if( this->CalcNorm( dlambdaNew, nTotal ) < eps ) return;
        }
        this->_log->error( "[closure] Newton did not converge!" );
    }
};

static Closure* make_closure( Settings* s, int newtonMode ) {
    if( newtonMode != 1 ) return Closure::Create( s );
    switch( s->GetClosureType() ) {
        case ClosureType::C_BOUNDEDBARRIER: return new Guarded<BoundedBarrier>( s );
        case ClosureType::C_EULER_2D: return new Guarded<EulerClosure2D>( s );
        case ClosureType::C_EULER_1D: return new Guarded<EulerClosure>( s );
        case ClosureType::C_SHALLOWWATER_1D: return new Guarded<ShallowWaterClosure>( s );
        default: return Closure::Create( s );
    }
}

static void solve_one( Closure* cl, int newtonMode, Matrix& lambda, const Matrix& u, unsigned nTotal, unsigned nQTotal ) {
    if( newtonMode == 2 )
        cl->SolveClosureSafe( lambda, u, nTotal, nQTotal );
    else
        cl->SolveClosure( lambda, u, nTotal, nQTotal );
}

// ---------------------------------------------------------------------------
struct uqcref {
    std::unique_ptr<Settings> settings;
    std::unique_ptr<HarnessMeshBase> mesh;
    std::unique_ptr<Problem> problem;
    std::unique_ptr<Closure> closure;
    std::unique_ptr<TimeSolver> time;
    MatVec u, lambda, uQ, uNew, uOld;
    std::vector<unsigned> level;
    VectorU nTotalForRef;
    unsigned nCells = 0, nStates = 0, nTotal = 0, nQTotal = 0;
    int newtonMode  = 0; // 0 SolveClosure, 1 guarded, 2 SolveClosureSafe
    double t = 0.0;
    std::string err;
};

static void set_err( char* err, int errlen, const std::string& m ) {
    if( err && errlen > 0 ) {
        std::strncpy( err, m.c_str(), size_t( errlen - 1 ) );
        err[errlen - 1] = 0;
    }
}

static int full_solve_files( uqcref* h, const char* prefix, double* meanVar, char* err, int errlen, bool gpu );

extern "C" {

// Builds settings (the reference's own Settings parser, settings.cpp:22-323),
// a harness problem (kind 1 Burgers, 2 Euler2D, 3 shallow water, 4 the reference's
// own Euler1D), the mesh and
// the reference's Closure (closure.cpp:16-84) and ExplicitEuler.
// 1-D meshes come from the [mesh] table; 2-D meshes from the arrays.
int uqcref_create( const char* toml,
                   int kind,
                   int newtonMode,
                   const double* params,
                   double bbMinus,
                   double bbPlus,
                   int nNodes,
                   const double* xy,
                   const int* nodeBoundary,
                   int nCells2d,
                   const int* tri,
                   uqcref** out,
                   char* err,
                   int errlen ) {
    try {
        g_bbMinus = bbMinus;
        g_bbPlus  = bbPlus;
        auto h    = std::make_unique<uqcref>();
        h->settings.reset( new Settings( std::string( toml ) ) );
        Settings* s = h->settings.get();
        if( kind == 1 )
            h->problem.reset( new HarnessBurgers( s, params ) );
        else if( kind == 2 )
            h->problem.reset( new HarnessEuler2D( s, params ) );
        else if( kind == 3 )
            h->problem.reset( new HarnessShallowWater( s, params ) );
        else if( kind == 4 )
            h->problem.reset( new Euler( s ) );    // the reference's own 1-D Euler problem (Sod state fixed in euler.cpp:95-128)
        else
            throw uqc_ref_error( "unknown problem kind" );
        if( s->GetMeshDimension() == 1 ) {
            auto file  = cpptoml::parse_file( std::string( toml ) );
            auto table = file->get_table( "mesh" );
            h->mesh.reset( new HarnessMesh1D( s,
                                              *table->get_as<unsigned>( "numberOfCells" ),
                                              table->get_as<double>( "a" ).value_or( 0.0 ),
                                              table->get_as<double>( "b" ).value_or( 0.0 ) ) );
        }
        else {
            h->mesh.reset( new HarnessMesh2D( s, unsigned( nNodes ), xy, nodeBoundary, unsigned( nCells2d ), tri ) );
        }
        // MomentSolver's constructor order (momentsolver.cpp:4-30).
        h->newtonMode = newtonMode;
        h->closure.reset( make_closure( s, newtonMode ) );
        s->SetNQTotal( h->closure->GetQuadratureGrid()->GetNodeCount() );
        h->time.reset( TimeSolver::Create( s, h->mesh.get() ) );
        s->SetDT( h->time->GetTimeStepSize() );
        h->nCells       = s->GetNumCells();
        h->nStates      = s->GetNStates();
        h->nTotal       = s->GetNTotal();
        h->nQTotal      = s->GetNQTotal();
        h->nTotalForRef = s->GetNTotalRefinementLevel();
        h->level.assign( h->nCells, s->GetNRefinementLevels() - 1 );
        *out = h.release();
        return 0;
    } catch( const std::exception& e ) {
        set_err( err, errlen, e.what() );
        return -1;
    }
}

void uqcref_destroy( uqcref* h ) { delete h; }

// Per-cell boundary types of an SU2 mesh (1 Dirichlet, 2 no-slip, 3 shallow-water wall).
void uqcref_set_cell_bc( uqcref* h, const int* codes ) { h->mesh->SetCellTypes( codes ); }

// Boundary unit normal of each boundary cell (Cell::GetBoundaryUnitNormal), zero elsewhere.
void uqcref_boundary_normals( uqcref* h, double* out ) {
    for( unsigned j = 0; j < h->nCells; ++j ) {
        Cell* c = h->mesh->GetGrid()[j];
        Vector n( 2, 0.0 );
        if( c->IsBoundaryCell() && c->GetBoundaryType() != BoundaryType::NONE ) n = c->GetBoundaryUnitNormal();
        out[2 * j]     = n[0];
        out[2 * j + 1] = n[1];
    }
}

void uqcref_sizes( uqcref* h, int* out ) {
    out[0] = int( h->nCells );
    out[1] = int( h->nStates );
    out[2] = int( h->nTotal );
    out[3] = int( h->nQTotal );
    out[4] = int( h->settings->GetNRefinementLevels() );
    out[5] = int( h->settings->GetNDimXi() );
    for( unsigned l = 0; l < h->settings->GetNRefinementLevels() && l < 16; ++l ) out[6 + l] = int( h->nTotalForRef[l] );
}

// Tables of closure.cpp:49-64: phiTilde and phiTildeWf (nQ x nT, column-major)
// plus the tensor grid nodes (nQ x dimXi) and weights.
void uqcref_tables( uqcref* h, double* phi, double* phiWf, double* xi, double* w ) {
    const Matrix& P  = h->closure->GetPhiTilde();
    const Matrix& PW = h->closure->GetPhiTildeWf();
    for( unsigned i = 0; i < h->nTotal; ++i )
        for( unsigned k = 0; k < h->nQTotal; ++k ) {
            phi[i * h->nQTotal + k]   = P( k, i );
            phiWf[i * h->nQTotal + k] = PW( k, i );
        }
    auto grid  = h->closure->GetQuadratureGrid();
    auto nodes = grid->GetNodes();
    auto wts   = grid->GetWeights();
    unsigned d = h->settings->GetNDimXi();
    for( unsigned k = 0; k < h->nQTotal; ++k ) {
        for( unsigned l = 0; l < d; ++l ) xi[k * d + l] = nodes[k][l];
        w[k] = wts[k];
    }
}

// Mesh geometry as the reference computes it: per cell area, maxEdge,
// centre (2), and per face unit normal (2), scaled normal (2), neighbour id.
void uqcref_geometry( uqcref* h, double* area, double* maxEdge, double* center, double* unitN, double* scaledN, int* nbr, int* boundary ) {
    unsigned nf = h->mesh->GetDimension() == 1 ? 2 : 3;
    for( unsigned j = 0; j < h->nCells; ++j ) {
        Cell* c    = h->mesh->GetGrid()[j];
        area[j]    = c->GetArea();
        maxEdge[j] = c->GetMaxEdge();
        Vector cc  = c->GetCenter();
        center[2 * j]     = cc[0];
        center[2 * j + 1] = cc.size() > 1 ? cc[1] : 0.0;
        boundary[j]       = c->IsBoundaryCell() ? 1 : 0;
        VectorU nb        = c->GetNeighborIDs();
        for( unsigned l = 0; l < nf; ++l ) {
            Vector un = c->GetUnitNormal( l ), sn = c->GetNormal( l );
            unitN[( j * nf + l ) * 2]       = un[0];
            unitN[( j * nf + l ) * 2 + 1]   = un.size() > 1 ? un[1] : 0.0;
            scaledN[( j * nf + l ) * 2]     = sn[0];
            scaledN[( j * nf + l ) * 2 + 1] = sn.size() > 1 ? sn[1] : 0.0;
            nbr[j * nf + l]                 = int( nb[l] );
        }
    }
}

// Initial moments and duals: restates MomentSolver::SetupIC (momentsolver.cpp:535-563)
// and the no-restart branch of SetDuals (:463-485): u_j = U_IC(x_j, xi_k) * phiTildeWf,
// lambda_j(:,0) = DS(u_j(:,0)).
void uqcref_init_state( uqcref* h ) {
    Settings* s = h->settings.get();
    h->u        = MatVec( h->nCells, Matrix( h->nStates, h->nTotal ) );
    Vector xiEta( s->GetNDimXi() );
    Matrix uIC( h->nStates, h->nQTotal );
    Matrix phiTildeWf = h->closure->GetPhiTildeWf();
    auto xiQuad       = h->closure->GetQuadratureGrid()->GetNodes();
    for( unsigned j = 0; j < h->nCells; ++j ) {
        for( unsigned k = 0; k < h->nQTotal; ++k ) {
            for( unsigned l = 0; l < s->GetNDimXi(); ++l ) xiEta[l] = xiQuad[k][l];
            column( uIC, k ) = h->problem->IC( h->mesh->GetCenterPos( j ), xiEta );
        }
        h->u[j] = uIC * phiTildeWf;
    }
    h->lambda = MatVec( h->nCells, Matrix( h->nStates, h->nTotal, 0.0 ) );
    Vector ds( h->nStates );
    Vector u0( h->nStates );
    for( unsigned j = 0; j < h->nCells; ++j ) {
        for( unsigned l = 0; l < h->nStates; ++l ) u0[l] = h->u[j]( l, 0 );
        h->closure->DS( ds, u0 );
        for( unsigned l = 0; l < h->nStates; ++l ) h->lambda[j]( l, 0 ) = ds[l];
    }
    h->level.assign( h->nCells, s->GetNRefinementLevels() - 1 );
    h->uQ   = MatVec( h->nCells + 1, Matrix( h->nStates, s->GetNqPE() ) );
    h->uNew = h->u;
    h->uOld = h->u;
    h->t    = 0.0;
}

// State in the reference layout: per cell an nStates x nTotal column-major matrix.
void uqcref_get_state( uqcref* h, double* u, double* lambda, unsigned* level ) {
    size_t n = size_t( h->nStates ) * h->nTotal;
    for( unsigned j = 0; j < h->nCells; ++j ) {
        if( u ) std::memcpy( u + j * n, h->u[j].GetPointer(), n * sizeof( double ) );
        if( lambda ) std::memcpy( lambda + j * n, h->lambda[j].GetPointer(), n * sizeof( double ) );
        if( level ) level[j] = h->level[j];
    }
}
void uqcref_set_state( uqcref* h, const double* u, const double* lambda, const unsigned* level, double t ) {
    size_t n = size_t( h->nStates ) * h->nTotal;
    if( h->u.size() != h->nCells ) uqcref_init_state( h );
    for( unsigned j = 0; j < h->nCells; ++j ) {
        if( u ) std::memcpy( h->u[j].GetPointer(), u + j * n, n * sizeof( double ) );
        if( lambda ) std::memcpy( h->lambda[j].GetPointer(), lambda + j * n, n * sizeof( double ) );
        if( level ) h->level[j] = level[j];
    }
    h->t = t;
}

// Batched Closure::SolveClosure (closure.cpp:133-193) on caller-owned cells in
// the reference layout; status[j] = 0 converged, 1 the closure raised an error.
int uqcref_solve_closure( uqcref* h, int nCells, double* lambda, const double* u, const unsigned* nTotalCell, int* status ) {
    size_t n  = size_t( h->nStates ) * h->nTotal;
    int nFail = 0;
#pragma omp parallel for schedule( dynamic, 10 ) reduction( + : nFail )
    for( int j = 0; j < nCells; ++j ) {
        Matrix lam( h->nStates, h->nTotal ), uu( h->nStates, h->nTotal );
        std::memcpy( lam.GetPointer(), lambda + j * n, n * sizeof( double ) );
        std::memcpy( uu.GetPointer(), u + j * n, n * sizeof( double ) );
        int st = 0;
        try {
            solve_one( h->closure.get(), h->newtonMode, lam, uu, nTotalCell ? nTotalCell[j] : h->nTotal, h->nQTotal );
        } catch( const std::exception& ) {
            st = 1;
        }
        std::memcpy( lambda + j * n, lam.GetPointer(), n * sizeof( double ) );
        if( status ) status[j] = st;
        nFail += st;
    }
    return nFail;
}

// One refinement indicator: restates MomentSolver::ComputeRefIndicator
// (momentsolver.cpp:271-289).
static double ref_indicator( uqcref* h, const Matrix& u, unsigned refLevel ) {
    double indicator = 0;
    if( h->settings->GetNDimXi() == 1 ) {
        indicator += std::fabs( u( 0, h->nTotalForRef[refLevel] - 1 ) ) + std::fabs( u( 0, h->nTotalForRef[refLevel] - 2 ) );
    }
    else {
        unsigned prev = refLevel == 0 ? 1 : h->nTotalForRef[refLevel - 1];
        for( unsigned i = prev; i < h->nTotalForRef[refLevel]; ++i ) indicator += std::fabs( u( 0, i ) );
    }
    return indicator;
}

// Time steps: restates the body of MomentSolver::Solve (momentsolver.cpp:79-152)
// for one rank, calling the reference's closure, ansatz, projection, problem
// and ExplicitEuler::Advance. out = {t, dt of the last step, residual of the
// last step, number of closure failures}.
int uqcref_step( uqcref* h, int nSteps, double* out ) {
    Settings* s = h->settings.get();
    Closure* cl = h->closure.get();
    Problem* pr = h->problem.get();
    auto numFlux = [cl, pr, s]( Matrix& o, const Matrix& u1, const Matrix& u2, const Vector& nUnit, const Vector& n, unsigned nTotal ) {
        multOnPENoReset( pr->G( u1, u2, nUnit, n ), cl->GetPhiTildeWf(), o, s->GetKStart(), s->GetKEnd(), nTotal );
    };
    double dt = 0.0, residual = 0.0;
    int nFail = 0;
    VectorU refLevel( h->nCells );
    for( int step = 0; step < nSteps; ++step ) {
        residual = 0.0;
        int fails = 0;
#pragma omp parallel for schedule( dynamic, 10 ) reduction( + : fails )
        for( unsigned j = 0; j < h->nCells; ++j ) {
            try {
                solve_one( cl, h->newtonMode, h->lambda[j], h->u[j], h->nTotalForRef[h->level[j]], h->nQTotal );
            } catch( const std::exception& ) {
                fails += 1;
            }
        }
        nFail += fails;
        for( unsigned j = 0; j < h->nCells; ++j ) h->uOld[j] = h->u[j];
#pragma omp parallel for
        for( unsigned j = 0; j < h->nCells; ++j ) h->uQ[j] = cl->U( cl->EvaluateLambdaOnPE( h->lambda[j], h->nTotalForRef[h->level[j]] ) );
        for( unsigned j = 0; j < h->nCells; ++j ) {
            double indicator = ref_indicator( h, h->u[j], h->level[j] );
            if( indicator > 0.02 && h->level[j] < s->GetNRefinementLevels() - 1 )
                h->level[j] += 1;
            else if( indicator < 0.004 && h->level[j] > 0 )
                h->level[j] -= 1;
        }
#pragma omp parallel for
        for( unsigned j = 0; j < h->nCells; ++j ) {
            h->u[j].reset();
            multOnPENoReset( h->uQ[j], cl->GetPhiTildeWf(), h->u[j], s->GetKStart(), s->GetKEnd(), h->nTotalForRef[h->level[j]] );
        }
        double dtMin = 1e10;
        for( unsigned j = 0; j < h->nCells; ++j ) {
            double d = pr->ComputeDt( h->uQ[j], h->mesh->GetMaxEdge( j ) / h->mesh->GetArea( j ) );
            if( d < dtMin ) dtMin = d;
        }
        dt = dtMin;
        h->t += dt;
        for( unsigned j = 0; j < h->nCells; ++j ) refLevel[j] = h->level[j];
        h->time->Advance( numFlux, h->uNew, h->u, h->uQ, dt, refLevel );
        size_t n = size_t( h->nStates ) * h->nTotal;
        for( unsigned j = 0; j < h->nCells; ++j ) std::memcpy( h->u[j].GetPointer(), h->uNew[j].GetPointer(), n * sizeof( double ) );
        for( unsigned j = 0; j < h->nCells; ++j ) residual += std::abs( h->u[j]( 0, 0 ) - h->uOld[j]( 0, 0 ) ) * h->mesh->GetArea( j );
    }
    out[0] = h->t;
    out[1] = dt;
    out[2] = residual;
    out[3] = double( nFail );
    return nFail;
}

// Mean and variance per cell: restates MomentSolver::WriteMeanAndVar
// (momentsolver.cpp:302-328). out[j * 2 nS + r], rows 0..nS-1 = E, nS..2nS-1 = Var.
void uqcref_mean_var( uqcref* h, double* out ) {
    Matrix phiTildeWf = h->closure->GetPhiTildeWf();
    unsigned nS       = h->nStates;
    Vector tmp( nS, 0.0 );
    for( unsigned j = 0; j < h->nCells; ++j ) {
        double* mv = out + size_t( j ) * 2 * nS;
        for( unsigned r = 0; r < 2 * nS; ++r ) mv[r] = 0.0;
        for( unsigned k = 0; k < h->nQTotal; ++k ) {
            h->closure->U( tmp, h->closure->EvaluateLambda( h->lambda[j], k, h->nTotalForRef[h->level[j]] ) );
            for( unsigned i = 0; i < nS; ++i ) mv[i] += tmp[i] * phiTildeWf( k, 0 );
        }
        for( unsigned k = 0; k < h->nQTotal; ++k ) {
            h->closure->U( tmp, h->closure->EvaluateLambda( h->lambda[j], k, h->nTotalForRef[h->level[j]] ) );
            for( unsigned i = 0; i < nS; ++i ) mv[i + nS] += pow( tmp[i] - mv[i], 2 ) * phiTildeWf( k, 0 );
        }
    }
}

// The reference's own MomentSolver::Solve() end to end (momentsolver.cpp:37-269)
// on this handle's settings, mesh and problem. Returns the final mean/variance
// matrix that Solve exports (2 nS rows per cell, full precision) and the final
// duals as written by MomentSolver::Export (15 significant digits).
int uqcref_full_solve( uqcref* h, double* meanVar, double* lambda15, char* err, int errlen ) {
    try {
        auto dualLog             = spdlog::get( "duals" );
        dualLog->capture_enabled = true;
        dualLog->lines.clear();
        h->mesh->exported.clear();
        {
            MomentSolver solver( h->settings.get(), h->mesh.get(), h->problem.get() );
            solver.Solve();
        }
        dualLog->capture_enabled = false;
        auto it = h->mesh->exported.find( "" );
        if( it == h->mesh->exported.end() ) throw uqc_ref_error( "Solve exported no mean/variance" );
        const Matrix& mv = it->second;
        unsigned nS      = h->nStates;
        for( unsigned j = 0; j < h->nCells; ++j )
            for( unsigned r = 0; r < 2 * nS; ++r ) meanVar[size_t( j ) * 2 * nS + r] = mv( r, j );
        size_t n = size_t( nS ) * h->nTotal;
        for( unsigned j = 0; j < h->nCells && j < dualLog->lines.size(); ++j ) {
            std::stringstream ls( dualLog->lines[j] );
            std::string cell;
            for( unsigned s = 0; s < nS; ++s )
                for( unsigned i = 0; i < h->nTotal; ++i ) {
                    std::getline( ls, cell, ',' );
                    lambda15[j * n + i * nS + s] = std::stod( cell );
                }
        }
        return 0;
    } catch( const std::exception& e ) {
        set_err( err, errlen, e.what() );
        return -1;
    }
}

// MomentSolver::Solve() as full_solve, also writing what a run of the
// reference leaves for a restart: <prefix>_moments and <prefix>_duals (the
// lines MomentSolver::Export writes to its "moments"/"duals" loggers,
// momentsolver.cpp:565-588, whose file sinks use the pattern "%v"), and the log
// <prefix> with the configuration echo of main.cpp's PrintInit (:160-180) in
// the file sink's pattern "%Y-%m-%d %H:%M:%S.%f | %v" (restated here: main.cpp
// is not compiled into the harness).
int uqcref_full_solve_export( uqcref* h, const char* prefix, double* meanVar, char* err, int errlen ) {
    return full_solve_files( h, prefix, meanVar, err, errlen, false );
}

// The same with GpuMomentSolver (oracle/ref/gpumomentsolver.cpp, linked into
// the GPU variant of the harness only) in place of MomentSolver.
int uqcref_full_solve_gpu( uqcref* h, const char* prefix, double* meanVar, char* err, int errlen ) {
    return full_solve_files( h, prefix, meanVar, err, errlen, true );
}

}    // extern "C"

// GpuMomentSolver(settings, mesh, problem).Solve(), defined by the GPU variant.
extern "C" __attribute__( ( weak ) ) int uqcref_gpu_moment_solver_run( Settings*, Mesh*, Problem*, char*, int );

static int full_solve_files( uqcref* h, const char* prefix, double* meanVar, char* err, int errlen, bool gpu ) {
    try {
        auto momentLog = spdlog::get( "moments" );
        auto dualLog   = spdlog::get( "duals" );
        momentLog->capture_enabled = dualLog->capture_enabled = true;
        momentLog->lines.clear();
        dualLog->lines.clear();
        h->mesh->exported.clear();
        if( gpu ) {
            if( !uqcref_gpu_moment_solver_run ) throw uqc_ref_error( "this harness variant has no GpuMomentSolver" );
            char e[512] = {0};
            if( uqcref_gpu_moment_solver_run( h->settings.get(), h->mesh.get(), h->problem.get(), e, int( sizeof e ) ) != 0 )
                throw uqc_ref_error( e );
        }
        else {
            MomentSolver solver( h->settings.get(), h->mesh.get(), h->problem.get() );
            solver.Solve();
        }
        momentLog->capture_enabled = dualLog->capture_enabled = false;
        auto it = h->mesh->exported.find( "" );
        if( it == h->mesh->exported.end() ) throw uqc_ref_error( "Solve exported no mean/variance" );
        const Matrix& mv = it->second;
        for( unsigned j = 0; j < h->nCells; ++j )
            for( unsigned r = 0; r < 2 * h->nStates; ++r ) meanVar[size_t( j ) * 2 * h->nStates + r] = mv( r, j );
        const std::string base = prefix;
        for( int which = 0; which < 2; ++which ) {
            std::ofstream f( base + ( which == 0 ? "_moments" : "_duals" ) );
            for( const auto& line : ( which == 0 ? momentLog : dualLog )->lines ) f << line << "\n";
            if( !f ) throw uqc_ref_error( "cannot write " + base );
        }
        std::ofstream log( base );
        const std::string stamp = "2000-01-01 00:00:00.000000 | ", rule = "================================================================";
        log << stamp << "UQCreator\n" << stamp << rule << "\n" << stamp << "Git commit hash:\tharness\n";
        log << stamp << "Config file:\t" << h->settings->GetInputFile() << "\n";
        log << stamp << "MPI Threads:\t1\n" << stamp << "OMP Threads:\t1\n" << stamp << rule << "\n";
        std::ifstream ifs( h->settings->GetInputFile() );
        std::string line;
        while( !ifs.eof() ) {
            std::getline( ifs, line );
            if( line[0] != '#' ) log << stamp << " " << line << "\n";
        }
        log << stamp << rule << "\n" << stamp << "\n";
        if( !log ) throw uqc_ref_error( "cannot write " + base );
        return 0;
    } catch( const std::exception& e ) {
        set_err( err, errlen, e.what() );
        return -1;
    }
}
