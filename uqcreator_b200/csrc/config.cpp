// Reader for UQCreator's TOML input files (the subset they use: [tables],
// key = string | integer | float | boolean | nested arrays, # comments) and
// the mapping of its keys onto uqc::Config, following Settings::Init
// (settings.cpp:22-323) for key names, accepted values and defaults.
#include <cmath>
#include <sstream>

#include "host.h"
#include "uqc.h"

#include <cstdio>

namespace uqc {
namespace {

struct Value {
    enum Kind { STR, INT, FLT, BOOL, ARR } kind = STR;
    std::string s;
    long long i = 0;
    double f    = 0.0;
    bool b      = false;
    std::vector<Value> items;
    double num() const {
        if( kind == INT ) return double( i );
        if( kind == FLT ) return f;
        throw ConfigError( "expected a number" );
    }
};

using Table = std::map<std::string, Value>;
using Doc   = std::map<std::string, Table>;

struct Parser {
    const char* p;
    int line;
    void ws() {
        while( *p == ' ' || *p == '\t' || *p == '\r' ) ++p;
    }
    [[noreturn]] void fail( const std::string& m ) { throw ConfigError( "TOML line " + std::to_string( line ) + ": " + m ); }
    Value value() {
        ws();
        Value v;
        if( *p == '"' ) {
            ++p;
            v.kind = Value::STR;
            while( *p && *p != '"' ) v.s += *p++;
            if( *p != '"' ) fail( "unterminated string" );
            ++p;
        }
        else if( *p == '[' ) {
            ++p;
            v.kind = Value::ARR;
            ws();
            while( *p && *p != ']' ) {
                v.items.push_back( value() );
                ws();
                if( *p == ',' ) ++p;
                ws();
            }
            if( *p != ']' ) fail( "unterminated array" );
            ++p;
        }
        else if( std::string( p, 4 ) == "true" ) {
            v.kind = Value::BOOL;
            v.b    = true;
            p += 4;
        }
        else if( std::string( p, 5 ) == "false" ) {
            v.kind = Value::BOOL;
            p += 5;
        }
        else {
            std::string tok;
            while( *p && *p != ',' && *p != ']' && *p != '#' && *p != ' ' && *p != '\t' && *p != '\r' ) tok += *p++;
            if( tok.empty() ) fail( "missing value" );
            try {
                if( tok.find_first_of( ".eEn" ) != std::string::npos ) {
                    v.kind = Value::FLT;
                    v.f    = std::stod( tok );
                }
                else {
                    v.kind = Value::INT;
                    v.i    = std::stoll( tok );
                }
            } catch( const std::exception& ) {
                fail( "bad number '" + tok + "'" );
            }
        }
        return v;
    }
};

std::string trim( const std::string& s ) {
    size_t a = s.find_first_not_of( " \t\r" ), b = s.find_last_not_of( " \t\r" );
    return a == std::string::npos ? std::string() : s.substr( a, b - a + 1 );
}

Doc parse_doc( const std::string& text ) {
    Doc doc;
    std::istringstream in( text );
    std::string ln, section;
    Parser ps{nullptr, 0};
    while( std::getline( in, ln ) ) {
        ++ps.line;
        ps.p = ln.c_str();
        ps.ws();
        if( *ps.p == 0 || *ps.p == '#' ) continue;
        if( *ps.p == '[' ) {
            size_t e = ln.find( ']' );
            if( e == std::string::npos ) ps.fail( "bad table header" );
            section = trim( ln.substr( ln.find( '[' ) + 1, e - ln.find( '[' ) - 1 ) );
            doc[section];
            continue;
        }
        size_t eq = ln.find( '=' );
        if( eq == std::string::npos ) ps.fail( "expected key = value" );
        std::string key = trim( ln.substr( 0, eq ) );
        ps.p            = ln.c_str() + eq + 1;
        doc[section][key] = ps.value();
    }
    return doc;
}

const Value* find( const Doc& d, const std::string& t, const std::string& k ) {
    auto it = d.find( t );
    if( it == d.end() ) return nullptr;
    auto jt = it->second.find( k );
    return jt == it->second.end() ? nullptr : &jt->second;
}

const Value& need( const Doc& d, const std::string& t, const std::string& k ) {
    const Value* v = find( d, t, k );
    if( !v ) throw ConfigError( "[" + t + "] '" + k + "' not set!" );
    return *v;
}

std::string str( const Value& v, const std::string& what ) {
    if( v.kind != Value::STR ) throw ConfigError( what + " must be a string" );
    return v.s;
}

}    // namespace

Config parse_config( const std::string& text ) {
    Doc d = parse_doc( text );
    Config c;
    // [general] problem (settings.cpp:34-63)
    c.problemName = str( need( d, "general", "problem" ), "[general] problem" );
    if( c.problemName == "Burgers1D" )
        c.problem = PR_BURGERS;
    else if( c.problemName == "Euler2D" )
        c.problem = PR_EULER2D;
    else if( c.problemName == "ShallowWater1D" )
        c.problem = PR_SHALLOW_WATER;
    else if( c.problemName == "Euler1D" )
        c.problem = PR_EULER1D;
    else if( c.problemName == "PNEquations2D" )
        // momentsolver.cpp:403-411: the source of every cell is accumulated into
        // one matrix shared by the threads of an OpenMP loop and never reset,
        // so the reference's result depends on thread scheduling
        throw ConfigError( "[general] 'problem' = 'PNEquations2D': the reference's source term is accumulated across cells by racing threads" );
    else if( c.problemName == "ShallowWater2D" )
        // shallowwater2d.cpp:87-90: ComputeDt is not implemented and returns 0,
        // so the reference's time loop never advances
        throw ConfigError( "[general] 'problem' = 'ShallowWater2D': the reference's time step for it is not implemented (always 0)" );
    else
        throw ConfigError( "[general] 'problem' = '" + c.problemName + "' is not on this hot path (Burgers1D, Euler1D, Euler2D, ShallowWater1D)" );
    // [mesh] (settings.cpp:95-111, mesh1d.cpp:6-17)
    c.meshDim = int( need( d, "mesh", "dimension" ).num() );
    if( const Value* v = find( d, "mesh", "numberOfCells" ) ) c.nCells1d = int( v->num() );
    if( const Value* v = find( d, "mesh", "a" ) ) c.a = v->num();
    if( const Value* v = find( d, "mesh", "b" ) ) c.b = v->num();
    // [problem] (settings.cpp:114-170, euler2d.cpp:10)
    std::string ts = str( need( d, "problem", "timestepping" ), "[problem] timestepping" );
    if( ts != "explicitEuler" ) throw ConfigError( "[problem] 'timestepping' is invalid! Please set one of the following types: explicitEuler" );
    const Value& dist = need( d, "problem", "distribution" );
    if( dist.kind != Value::ARR || dist.items.size() != 2 || dist.items[0].kind != Value::ARR )
        throw ConfigError( "[problem] 'distribution' must be [[types],[sigmas]]" );
    c.dimXi = int( dist.items[0].items.size() );
    for( size_t l = 0; l < dist.items[0].items.size(); ++l ) {
        if( str( dist.items[0].items[l], "distribution type" ) != "Legendre" )
            throw ConfigError( "[problem] 'distribution': only Legendre is on this hot path" );
        c.sigma.push_back( dist.items[1].items.at( l ).num() );
    }
    if( c.dimXi < 1 || c.dimXi > 3 ) throw ConfigError( "[problem] 'distribution': 1 to 3 uncertain dimensions supported" );
    c.cfl  = need( d, "problem", "CFL" ).num();
    c.tEnd = need( d, "problem", "tEnd" ).num();
    if( const Value* v = find( d, "problem", "residual" ) ) c.minResidual = v->num();
    if( const Value* v = find( d, "problem", "gamma" ) ) c.gamma = v->num();
    // [moment_system] (settings.cpp:173-314)
    std::string cl = str( need( d, "moment_system", "closure" ), "[moment_system] closure" );
    if( cl == "BoundedBarrier" )
        c.closure = CL_BOUNDED_BARRIER;
    else if( cl == "Euler2D" )
        c.closure = CL_EULER2D;
    else if( cl == "ShallowWater" )
        c.closure = CL_SHALLOW_WATER;
    else if( cl == "Euler" )
        c.closure = CL_EULER1D;
    else if( cl == "LogSin" )
        c.closure = CL_LOGSIN;
    else if( cl == "StochasticGalerkin" || cl == "L2Filter" || cl == "LassoFilter" ) {
        // the linear closures take the states of the problem
        c.closure    = c.problem == PR_BURGERS ? CL_LINEAR_BURGERS
                       : c.problem == PR_EULER2D  ? CL_LINEAR_EULER2D
                       : c.problem == PR_EULER1D  ? CL_LINEAR_EULER1D
                                                  : CL_LINEAR_SW;
        c.filterKind = cl == "StochasticGalerkin" ? FILTER_SG : ( cl == "L2Filter" ? FILTER_L2 : FILTER_LASSO );
    }
    else if( cl == "ExponentialFilter" )
        // exponentialfilter.cpp:4-20 reads the filter order (never set) and the
        // time step (set only after the closure is built, momentsolver.cpp:18-24):
        // its factors are undefined, so there is nothing to reproduce
        throw ConfigError( "[moment_system] 'closure' = 'ExponentialFilter': the reference's filter reads an uninitialised order and time step" );
    else
        throw ConfigError( "[moment_system] 'closure' = '" + cl +
                           "' is not on this hot path (BoundedBarrier, LogSin, Euler, Euler2D, ShallowWater, StochasticGalerkin, L2Filter, LassoFilter)" );
    const Value& mom = need( d, "moment_system", "moments" );
    if( mom.kind != Value::ARR || mom.items.size() != 2 ) throw ConfigError( "[moment_system] 'moments' must be [[type],[degrees]]" );
    std::string degType = str( mom.items[0].items.at( 0 ), "moments type" );
    if( degType == "maxDegree" )
        c.maxDegree = true;
    else if( degType != "totalDegree" )
        throw ConfigError( "[moment_system] 'moments' is invalid! Please set one of the following types: totalDegree, maxDegree" );
    for( auto& v : mom.items[1].items ) c.degrees.push_back( int( v.num() ) );
    if( c.degrees.empty() || c.degrees.size() > 16 ) throw ConfigError( "[moment_system] 'moments': 1 to 16 refinement levels" );
    const Value& qp = need( d, "moment_system", "quadPoints" );
    if( qp.kind != Value::ARR || qp.items.size() != 2 ) throw ConfigError( "[moment_system] 'quadPoints' must be [[type],[n per level]]" );
    if( str( qp.items[0].items.at( 0 ), "quadPoints type" ) == "sparseGrid" )
        throw ConfigError( "[moment_system] 'quadPoints': sparse grids are not on this hot path" );
    c.nQuad = int( qp.items[1].items.back().num() );
    if( const Value* v = find( d, "moment_system", "maxIterations" ) ) c.maxIterations = int( v->num() );
    if( const Value* v = find( d, "moment_system", "epsilon" ) ) c.epsilon = v->num();
    // closure / problem consistency (the reference pairs them in Problem::Create)
    int nS = closure_states( c.closure );
    int nSp = c.problem == PR_BURGERS ? 1 : ( c.problem == PR_EULER2D ? 4 : ( c.problem == PR_EULER1D ? 3 : 2 ) );
    if( nS != nSp ) throw ConfigError( "closure '" + cl + "' does not match problem '" + c.problemName + "'" );
    // [uqc]
    if( const Value* v = find( d, "uqc", "ic" ) )
        for( auto& x : v->items ) c.ic.push_back( x.num() );
    if( const Value* v = find( d, "uqc", "bounds" ) ) {
        c.bbMinus = v->items.at( 0 ).num();
        c.bbPlus  = v->items.at( 1 ).num();
    }
    if( const Value* v = find( d, "uqc", "mesh" ) ) c.meshKind = str( *v, "[uqc] mesh" );
    if( const Value* v = find( d, "mesh", "format" ) ) {
        if( str( *v, "[mesh] format" ) != "SU2" ) throw ConfigError( "[mesh2d] Unsupported mesh format! Please set one of the following formats: SU2" );
        const Value* f = find( d, "mesh", "SU2MeshFile" );
        if( !f ) throw ConfigError( "[mesh2d] 'SU2MeshFile' not set!" );
        c.meshKind = "su2";
        c.su2File  = str( *f, "[mesh] SU2MeshFile" );
        const Value* b = find( d, "mesh", "SU2BC" );
        if( !b || b->kind != Value::ARR ) throw ConfigError( "[mesh2d] 'SU2BC' Not set!" );
        for( const Value& pair : b->items ) {
            if( pair.kind != Value::ARR || pair.items.size() != 2 ) throw ConfigError( "[mesh] SU2BC entries are [marker, type]" );
            const std::string tag = str( pair.items[0], "[mesh] SU2BC marker" ), type = str( pair.items[1], "[mesh] SU2BC type" );
            int code;
            if( type == "dirichlet" )
                code = 1;
            else if( type == "noslip" )
                code = 2;
            else if( type == "swwall" )
                code = 3;
            else if( type == "neumann" || type == "periodic" )
                throw ConfigError( "[mesh2d] boundary condition '" + type + "' on '" + tag + "' is not supported on the hot path" );
            else
                throw ConfigError( "[mesh2d] Invalid boundary condition on boundary '" + tag + "'!" );
            c.su2BC.emplace_back( tag, code );
        }
    }
    if( const Value* v = find( d, "uqc", "mesh_params" ) ) {
        c.nx     = int( v->items.at( 0 ).num() );
        c.ny     = int( v->items.at( 1 ).num() );
        c.jitter = v->items.at( 2 ).num();
        c.seed   = uint64_t( v->items.at( 3 ).num() );
    }
    if( const Value* v = find( d, "uqc", "precision" ) ) {
        std::string p = str( *v, "[uqc] precision" );
        if( p == "fp64" )
            c.precision = 0;
        else if( p == "mixed" )
            c.precision = 1;
        else
            throw ConfigError( "[uqc] 'precision' must be fp64 or mixed" );
    }
    if( const Value* v = find( d, "uqc", "newton" ) ) {
        std::string p = str( *v, "[uqc] newton" );
        if( p == "reference" )
            c.newtonMode = 0;
        else if( p == "guarded" )
            c.newtonMode = 1;
        else if( p == "safe" )
            c.newtonMode = 2;
        else
            throw ConfigError( "[uqc] 'newton' must be reference, guarded or safe" );
    }
    if( const Value* v = find( d, "general", "restartFile" ) ) c.restartFile = str( *v, "[general] restartFile" );
    if( const Value* v = find( d, "general", "importDualState" ) ) {
        if( v->kind != Value::BOOL ) throw ConfigError( "[general] 'importDualState' must be true or false" );
        c.importDualState = v->b;
    }
    if( const Value* v = find( d, "uqc", "steps" ) ) {
        c.maxSteps = int( v->num() );
        if( c.maxSteps < 0 ) throw ConfigError( "[uqc] 'steps' must be >= 0" );
    }
    if( const Value* v = find( d, "uqc", "refinementIndicator" ) ) {
        const std::string p = str( *v, "[uqc] refinementIndicator" );
        if( p == "moments" )
            c.refIndicator = 0;
        else if( p == "energy" )
            c.refIndicator = 1;
        else
            throw ConfigError( "[uqc] 'refinementIndicator' must be moments or energy" );
    }
    if( const Value* v = find( d, "uqc", "refinementBounds" ) ) {
        if( v->kind != Value::ARR || v->items.size() != 2 ) throw ConfigError( "[uqc] 'refinementBounds' must be [lower, upper]" );
        c.refDown = v->items[0].num();
        c.refUp   = v->items[1].num();
        if( !( c.refDown < c.refUp ) ) throw ConfigError( "[uqc] 'refinementBounds' needs lower < upper" );
    }
    if( const Value* v = find( d, "uqc", "retardationLevels" ) ) {
        for( auto& x : v->items ) c.retLevels.push_back( int( x.num() ) );
        if( const Value* r = find( d, "uqc", "retardationResiduals" ) )
            for( auto& x : r->items ) c.retResiduals.push_back( x.num() );
        if( c.retLevels.empty() || c.retLevels.size() > 9 || c.retResiduals.size() + 1 != c.retLevels.size() )
            throw ConfigError( "[uqc] retardation: 1 to 9 'retardationLevels' and one fewer 'retardationResiduals'" );
        for( size_t k = 0; k < c.retLevels.size(); ++k ) {
            if( c.retLevels[k] < 0 || ( k && c.retLevels[k] < c.retLevels[k - 1] ) )
                throw ConfigError( "[uqc] 'retardationLevels' must be non-negative and non-decreasing" );
            if( k && k < c.retResiduals.size() && !( c.retResiduals[k] < c.retResiduals[k - 1] ) )
                throw ConfigError( "[uqc] 'retardationResiduals' must be decreasing" );
        }
    }
    // Euler1D: the reference's initial state is fixed in the problem (euler.cpp:95-128);
    // [uqc] ic = [x0, rhoL, pL, rhoR, pR] may replace it
    size_t needIc = c.problem == PR_BURGERS ? 4 : ( c.problem == PR_EULER2D ? 5 : ( c.problem == PR_EULER1D ? 0 : 3 ) );
    if( c.problem == PR_EULER1D && !c.ic.empty() && c.ic.size() < 5 ) throw ConfigError( "[uqc] 'ic' needs 5 values for Euler1D (or none)" );
    if( c.ic.size() < needIc ) throw ConfigError( "[uqc] 'ic' needs " + std::to_string( needIc ) + " values for " + c.problemName );
    if( c.meshDim == 1 ) {
        if( c.nCells1d < 3 || ( std::fabs( c.a ) <= 2.2e-16 && std::fabs( c.b ) <= 2.2e-16 ) )
            throw ConfigError( "[mesh1d] Invalid mesh parameters!" );
    }
    else if( c.meshDim == 2 ) {
        if( c.meshKind != "su2" && ( c.meshKind != "tri_jitter" || c.nx < 2 || c.ny < 2 ) )
            throw ConfigError( "[uqc] 2-D runs need [mesh] format = \"SU2\" or mesh = \"tri_jitter\" with mesh_params = [nx, ny, jitter, seed], nx, ny >= 2" );
    }
    else
        throw ConfigError( "[mesh] 'dimension' must be 1 or 2" );
    if( c.problem == PR_EULER2D && c.meshDim != 2 ) throw ConfigError( "Euler2D needs a 2-D mesh" );
    if( c.problem != PR_EULER2D && c.meshDim != 1 ) throw ConfigError( c.problemName + " needs a 1-D mesh" );
    return c;
}

namespace {
std::string toml_str( const char* v ) {
    std::string out = "\"";
    for( const char* p = v; *p; ++p ) {
        if( *p == '"' || *p == '\\' ) out += '\\';
        out += *p;
    }
    return out + "\"";
}
std::string toml_num( double v ) {
    char b[40];
    std::snprintf( b, sizeof b, "%.17g", v );
    std::string s = b;
    if( s.find_first_of( ".eEn" ) == std::string::npos ) s += ".0";    // a float, not an integer
    return s;
}
}    // namespace

std::string config_struct_to_toml( const void* p ) {
    const uqc_config& c = *static_cast<const uqc_config*>( p );
    if( !c.problem || !c.closure ) throw ConfigError( "uqc_config: problem and closure are required" );
    if( c.n_levels < 1 || c.n_levels > 16 ) throw ConfigError( "uqc_config: n_levels must be 1..16" );
    if( c.dim_xi < 1 || c.dim_xi > 3 ) throw ConfigError( "uqc_config: dim_xi must be 1..3" );
    if( c.n_ic < 0 || c.n_ic > 8 ) throw ConfigError( "uqc_config: n_ic must be 0..8" );
    std::string t;
    t += "[general]\nproblem = " + toml_str( c.problem ) + "\n";
    if( c.restart_file ) {
        t += "restartFile = " + toml_str( c.restart_file ) + "\n";
        t += std::string( "importDualState = " ) + ( c.import_dual_state ? "true" : "false" ) + "\n";
    }
    t += "\n[mesh]\ndimension = " + std::to_string( c.mesh_dimension ) + "\n";
    if( c.mesh_dimension == 1 ) t += "numberOfCells = " + std::to_string( c.n_cells ) + "\na = " + toml_num( c.a ) + "\nb = " + toml_num( c.b ) + "\n";
    if( c.su2_file ) {
        t += "format = \"SU2\"\nSU2MeshFile = " + toml_str( c.su2_file ) + "\nSU2BC = [";
        for( int i = 0; i < c.n_su2_bc; ++i ) {
            if( !c.su2_bc_marker || !c.su2_bc_type || !c.su2_bc_marker[i] || !c.su2_bc_type[i] ) throw ConfigError( "uqc_config: SU2 marker or type missing" );
            t += std::string( i ? ", " : "" ) + "[" + toml_str( c.su2_bc_marker[i] ) + ", " + toml_str( c.su2_bc_type[i] ) + "]";
        }
        t += "]\n";
    }
    t += "\n[problem]\ntimestepping = \"explicitEuler\"\ndistribution = [[";
    for( int l = 0; l < c.dim_xi; ++l ) t += std::string( l ? ", " : "" ) + "\"Legendre\"";
    t += "], [";
    for( int l = 0; l < c.dim_xi; ++l ) t += std::string( l ? ", " : "" ) + toml_num( c.sigma[l] );
    t += "]]\nCFL = " + toml_num( c.cfl ) + "\ntEnd = " + toml_num( c.t_end ) + "\n";
    if( c.min_residual >= 0.0 ) t += "residual = " + toml_num( c.min_residual ) + "\n";
    if( c.gamma > 0.0 ) t += "gamma = " + toml_num( c.gamma ) + "\n";
    t += "\n[moment_system]\nclosure = " + toml_str( c.closure ) + "\nmoments = [[" + std::string( c.max_degree ? "\"maxDegree\"" : "\"totalDegree\"" ) + "], [";
    for( int l = 0; l < c.n_levels; ++l ) t += std::string( l ? ", " : "" ) + std::to_string( c.degree[l] );
    t += "]]\nquadPoints = [[\"tensorizedGrid\"], [";
    for( int l = 0; l < c.n_levels; ++l ) t += std::string( l ? ", " : "" ) + std::to_string( c.quad_points[l] );
    t += "]]\nmaxIterations = " + std::to_string( c.max_iterations ) + "\nepsilon = " + toml_num( c.epsilon ) + "\n";
    t += "\n[uqc]\nic = [";
    for( int i = 0; i < c.n_ic; ++i ) t += std::string( i ? ", " : "" ) + toml_num( c.ic[i] );
    t += "]\nbounds = [" + toml_num( c.bounds[0] ) + ", " + toml_num( c.bounds[1] ) + "]\n";
    if( c.nx > 0 )
        t += "mesh = \"tri_jitter\"\nmesh_params = [" + std::to_string( c.nx ) + ", " + std::to_string( c.ny ) + ", " + toml_num( c.jitter ) + ", " +
             std::to_string( c.seed ) + "]\n";
    t += std::string( "precision = " ) + ( c.precision == 1 ? "\"mixed\"" : "\"fp64\"" ) + "\n";
    if( c.newton_mode < 0 || c.newton_mode > 2 ) throw ConfigError( "uqc_config: newton_mode must be 0, 1 or 2" );
    static const char* modes[] = {"reference", "guarded", "safe"};
    t += std::string( "newton = \"" ) + modes[c.newton_mode] + "\"\nsteps = " + std::to_string( c.steps ) + "\n";
    return t;
}

}    // namespace uqc
