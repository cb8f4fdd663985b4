// Host-side core of the B200 IPM solver: configuration (the reference's TOML
// schema), basis/quadrature tables and meshes. Device code lives in *.cu.
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace uqc {

struct ConfigError : public std::runtime_error {
    explicit ConfigError( const std::string& m ) : std::runtime_error( m ) {}
};

// Kernel closure kinds. 3-5: the linear closures (stochastic Galerkin and the
// moment filters, Config::filterKind) with the states of Burgers, 2-D Euler and
// shallow water; 6: the 1-D Euler entropy closure; 7: the linear closures with
// its three states; 8: LogSin (one state).
enum ClosureKind {
    CL_BOUNDED_BARRIER = 0,
    CL_EULER2D         = 1,
    CL_SHALLOW_WATER   = 2,
    CL_LINEAR_BURGERS  = 3,
    CL_LINEAR_EULER2D  = 4,
    CL_LINEAR_SW       = 5,
    CL_EULER1D         = 6,    // EulerClosure, three states
    CL_LINEAR_EULER1D  = 7,
    CL_LOGSIN          = 8     // LogSin, one state (Burgers)
};
enum FilterKind { FILTER_SG = 0, FILTER_L2 = 1, FILTER_LASSO = 2 };
inline int closure_states( int cl ) {
    return ( cl == 0 || cl == 3 || cl == 8 ) ? 1 : ( ( cl == 1 || cl == 4 ) ? 4 : ( ( cl == 6 || cl == 7 ) ? 3 : 2 ) );
}
inline bool closure_linear( int cl ) { return ( cl >= CL_LINEAR_BURGERS && cl <= CL_LINEAR_SW ) || cl == CL_LINEAR_EULER1D; }
enum ProblemKind { PR_BURGERS = 0, PR_EULER2D = 1, PR_SHALLOW_WATER = 2, PR_EULER1D = 3 };

// Everything the hot path reads from the input file. Keys and defaults follow
// Settings::Init (settings.cpp:22-323); the [uqc] table carries what the
// reference hard-codes in its problem classes (initial data, barrier bounds)
// and this implementation's own options.
struct Config {
    // [general]
    std::string problemName;
    ProblemKind problem = PR_BURGERS;
    // [mesh]
    int meshDim = 1;
    int nCells1d = 0;
    double a = 0.0, b = 0.0;
    // [problem]
    int dimXi = 1;
    std::vector<double> sigma;
    double cfl = 0.0, tEnd = 0.0, minResidual = -1.0, gamma = 1.4;
    // [moment_system]
    ClosureKind closure = CL_BOUNDED_BARRIER;
    int filterKind      = FILTER_SG;    // linear closures: which one (closure names of settings.cpp:176-205)
    bool maxDegree = false;
    std::vector<int> degrees;    // per refinement level
    int nQuad = 0;               // Gauss nodes per dimension (last level)
    int maxIterations = 1000;
    double epsilon = 5e-5;
    // [uqc]
    std::vector<double> ic;
    double bbMinus = 3.0, bbPlus = 12.0;
    std::string meshKind = "uniform1d";
    std::string su2File;                                  // [mesh] format = "SU2": SU2MeshFile (mesh2d.cpp:5-59)
    std::vector<std::pair<std::string, int>> su2BC;       // [mesh] SU2BC: marker -> BC code (1 dirichlet, 2 noslip, 3 swwall)
    int nx = 0, ny = 0;
    double jitter = 0.0;
    uint64_t seed = 0;
    int precision = 0;     // uqc_precision
    int newtonMode = 0;    // 0 reference, 1 guarded, 2 safe
    int maxSteps   = 0;    // [uqc] steps: stop after this many time steps (0: no limit)
    // refinement levels: indicator and bounds of the level rule, retardation
    int refIndicator = 0;              // 0: sum of |u(0, i)| (momentsolver.cpp:271-289); 1: S_l (Paper1/adaptivity.tex:12-14)
    double refDown = 0.004, refUp = 0.02;    // level - 1 below refDown, + 1 above refUp (momentsolver.cpp:104-112)
    std::vector<int> retLevels;        // highest level allowed, raised as the residual falls below ...
    std::vector<double> retResiduals;  // ... each of these (one fewer than retLevels)
    std::string restartFile;       // [general] restartFile (settings.cpp:74-79), relative to the input file's directory
    bool importDualState = false;  // [general] importDualState: duals from <restartFile>_duals too
    std::string inputDir = ".";    // directory of the input file (uqc_create_from_file), else "."
};

Config parse_config( const std::string& tomlText );

// The input file equivalent to a uqc_config struct (include/uqc.h).
std::string config_struct_to_toml( const void* uqcConfig );

// Basis and quadrature: tensor Gauss-Legendre grid and scaled Legendre basis
// tables phiTilde / phiTildeWf of Closure::Closure (closure.cpp:16-84).
struct Tables {
    int nT = 0, nQ = 0, dimXi = 0, nLevels = 0;
    std::vector<int> nTLevel;       // moments per refinement level
    std::vector<int> index;         // nT x dimXi polynomial degrees (settings.cpp:241-265)
    std::vector<double> xi, w;      // nodes (nQ x dimXi), weights
    std::vector<double> phi, phiWf; // nQ x nT, row k contiguous
};

Tables build_tables( const Config& c );
void gauss_legendre( int n, std::vector<double>& x, std::vector<double>& w );

// Cell geometry in structure-of-arrays form, faces per cell = 2 (1-D) or 3.
struct Mesh {
    int nCells = 0, nFaces = 0, dim = 1;
    std::vector<double> area, maxEdge, center;       // center: 2 per cell
    std::vector<double> unitN, scaledN;              // 2 per face
    std::vector<int> nbr;                            // per face; ghost = nCells
    std::vector<int> boundary;                       // Dirichlet cell flag
    std::vector<double> nodeXY;                      // node coordinates (x, y), for output
    std::vector<int> cellNodes;                      // nodes per cell (2 in 1-D, 3 for triangles)
    std::vector<double> bndNormal;                   // per cell: unit normal of its ghost face (Cell::UpdateBoundaryNormal)
};

// Boundary codes of Mesh::boundary: 0 interior, 1 Dirichlet (frozen cell),
// 2 no-slip wall, 3 shallow-water wall (reflecting ghost states,
// expliciteuler.cpp:25-58).
enum BoundaryCode { BC_NONE = 0, BC_DIRICHLET = 1, BC_NOSLIP = 2, BC_SWWALL = 3 };

// SU2 mesh (Mesh2D::LoadSU2MeshFromFile, mesh2d.cpp:68-259): triangles only.
// Builds the mesh and sets each boundary cell's code from the markers.
Mesh read_su2_mesh( const std::string& path, const std::vector<std::pair<std::string, int>>& bcs );

Mesh build_mesh_1d( int nCells, double a, double b );
void tri_jitter_nodes( int nx, int ny, double jitter, uint64_t seed, double* xy, int* bnd, int* tri );
void set_boundary_normals( Mesh& m );
inline bool mesh_has_walls( const Mesh& m ) {
    for( int b : m.boundary )
        if( b >= BC_NOSLIP ) return true;
    return false;
}
Mesh build_mesh_tri( int nNodes, const double* xy, const int* bnd, int nTri, const int* tri );

// Spatial sharding: one rank's part of a mesh. The reference splits the dual
// solves round-robin over MPI ranks and replicates every cell's duals and
// moments on every rank (PEforCell, _cellIndexPE; momentsolver.cpp:83-146).
// Here a rank owns a compact block of cells and keeps only those plus a
// one-ring halo: local cells 0..nOwned-1 are the owned ones in global order,
// then the halo cells grouped by owning rank (ascending), each group in global
// order. A rank sends to each peer the nodal states of its cells that lie in
// the peer's halo, in global order, which is the order the peer stores them in.
struct ShardPlan {
    int rank = 0, nRanks = 1, nGlobal = 0, nOwned = 0;
    std::vector<int> globalId;     // per local cell
    std::vector<int> peers;        // ranks exchanged with, ascending
    std::vector<int> sendCount;    // per peer
    std::vector<int> recvCount;    // per peer: halo cells it owns (contiguous, in peer order)
    std::vector<int> sendCells;    // local ids, grouped by peer
};

// Owner rank of every cell: recursive coordinate bisection of the cell
// centres (split across the wider extent, cells ordered by coordinate then id,
// rank counts split as evenly as possible, cell counts in proportion).
std::vector<int> partition_cells( const Mesh& m, int nRanks );

// The rank's local mesh (owned cells, then the halo) and its exchange plan.
// Neighbours outside the local cells, and the global mesh's ghost index, map
// to the local ghost index (the local cell count).
Mesh shard_mesh( const Mesh& g, const std::vector<int>& owner, int rank, int nRanks, ShardPlan& plan );

}    // namespace uqc
