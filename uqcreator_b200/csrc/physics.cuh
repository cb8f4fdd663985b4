// Device physics of the hot path: entropy ansatz U, its Jacobian DU and the
// entropy gradient DS of each closure, numerical fluxes, time-step rules and
// initial states. Formulas and their evaluation order follow the reference
// files cited per function; CUDA's exp/pow/log/sqrt are called as is.
#pragma once
#include <cuda_runtime.h>

namespace uqc {

struct PhysParams {
    double bbMinus, bbPlus;   // bounded barrier bounds
    double gamma;             // Euler
    double eulerA;            // Euler: 1 / (1 - gamma), the exponent of the entropy ansatz
    double cfl;
    double ic[8];
    int nIc;                  // initial-state parameters given ([uqc] ic)
    double sigma[4];
    int dimXi;
    double dtFixed;           // shallow water: TimeSolver's dx CFL / 12
};

template <int CL> struct Closure;

// ---------------------------------------------------------------- bounded barrier
// U and DU of BoundedBarrier (boundedbarrier.cpp:19-31, 67-80), one state.
template <> struct Closure<0> {
    static constexpr int NS = 1, NP = 1;
    static constexpr bool LINEAR = false;
    __host__ __device__ static void U( const double* L, double* u, bool, const PhysParams& p ) {
        double ePos = exp( L[0] ), eNeg = 1.0 / ePos;
        if( L[0] > 0.0 )
            u[0] = p.bbPlus / ( eNeg + 1.0 ) + p.bbMinus * eNeg / ( 1.0 + eNeg );
        else
            u[0] = p.bbMinus / ( ePos + 1.0 ) + p.bbPlus * ePos / ( 1.0 + ePos );
    }
    // packed symmetric DU: du[0] = DU(0,0)
    __host__ __device__ static void DU( const double* L, double* du, const PhysParams& p ) {
        double ePos = exp( L[0] ), eNeg = 1 / ePos;
        if( L[0] > 0 )
            du[0] = eNeg * ( p.bbPlus - p.bbMinus ) / ( exp( -2.0 * L[0] ) + 2.0 * eNeg + 1.0 );
        else
            du[0] = ePos * ( p.bbPlus - p.bbMinus ) / ( 1.0 + 2.0 * ePos + exp( 2.0 * L[0] ) );
    }
    // Closure::DS of the base class leaves the guess unchanged (zero)
    __host__ __device__ static void DS( const double*, double* ds, const PhysParams& ) { ds[0] = 0.0; }
};

// ---------------------------------------------------------------- Euler 2-D
// EulerClosure2D (eulerclosure2d.cpp); the class stores g = -gamma (:3).
template <> struct Closure<1> {
    static constexpr int NS = 4, NP = 10;
    static constexpr bool LINEAR = false;
    // The reference has two forms, U(Vector&) of :7-18 (gradient, mean/variance):
    // rho = exp(A q) (-v4)^A, and U(const Matrix&) of :27-32 (reconstruction):
    // rho = (-exp(q) v4)^A, with A = 1/(1 + g), g = -gamma. Both equal
    // exp(A (q + log(-v4))), which is evaluated here with one exponential and
    // one logarithm instead of exp and pow, and one division (1/v4); the
    // results agree with the reference's to a few ulps of the exponent.
    // vecForm is kept for the interface.
    __host__ __device__ static void U( const double* L, double* u, bool /*vecForm*/, const PhysParams& p ) {
        const double g = -p.gamma;
        const double v1 = L[0], v2 = L[1], v3 = L[2], v4 = L[3];
        const double i4 = 1.0 / v4;
        const double q  = ( v2 * v2 + v3 * v3 - 2.0 * v1 * v4 - 2.0 * v4 * g ) * ( 0.5 * i4 );
        const double e  = exp( p.eulerA * ( q + log( -v4 ) ) );
        const double ei = e * i4;
        u[0]            = e;
        u[1]            = -( v2 * ei );
        u[2]            = -( v3 * ei );
        u[3]            = -( ( -( v2 * v2 ) - v3 * v3 + 2.0 * v4 ) * ( 0.5 * ei * i4 ) );
    }
    // packed upper DU (:54-88): order (0,0)(0,1)(0,2)(0,3)(1,1)(1,2)(1,3)(2,2)(2,3)(3,3)
    // Same rewriting as U: rho' = A exp(A (q + log(-v4))), powers of 1/v4 from one division.
    __host__ __device__ static void DU( const double* L, double* y, const PhysParams& p ) {
        const double g = -p.gamma;
        double v1 = L[0], v2 = L[1], v3 = L[2], v4 = L[3];
        double i4 = 1.0 / v4, v4i2 = i4 * i4, v3p2 = v3 * v3, v2p2 = v2 * v2, v4p2 = v4 * v4;
        double q     = ( v2p2 + v3p2 - 2.0 * v1 * v4 - 2.0 * v4 * g ) * ( 0.5 * i4 );
        double e     = p.eulerA * exp( p.eulerA * ( q + log( -v4 ) ) );
        double vTerm = e * ( v2p2 + v3p2 + 2.0 * v4 * g ) * ( 0.5 * v4i2 * i4 );
        y[0] = -( e );
        y[1] = ( v2 * e ) * i4;
        y[2] = ( v3 * e ) * i4;
        y[3] = -( 0.5 * ( ( v2p2 + v3p2 - 2.0 * v4 ) * e ) * v4i2 );
        y[4] = -( ( e * ( v2p2 + ( g + 1.0 ) * v4 ) ) * v4i2 );
        y[5] = -( ( v2 * v3 * e ) * v4i2 );
        y[6] = v2 * vTerm;
        y[7] = -( ( e * ( v3p2 + ( g + 1.0 ) * v4 ) ) * v4i2 );
        y[8] = v3 * vTerm;
        y[9] = -( e * ( v2p2 * v2p2 + v3p2 * v3p2 + 4.0 * v3p2 * v4 * g - 4.0 * v4p2 * g + 2.0 * v2p2 * ( v3p2 + 2.0 * v4 * g ) ) ) * ( 0.25 * v4i2 * v4i2 );
    }
    // EulerClosure2D::DS (:90-106)
    __host__ __device__ static void DS( const double* u, double* ds, const PhysParams& p ) {
        const double gamma = -p.gamma;
        double rho = u[0], rhoU = u[1], rhoV = u[2], rhoE = u[3];
        double rhoV2 = rhoV * rhoV, rhoU2 = rhoU * rhoU;
        ds[0] = ( rhoU2 + rhoV2 + gamma * ( 2 * rho * rhoE - rhoU2 - rhoV2 ) ) / ( -2 * rho * rhoE + rhoU2 + rhoV2 ) -
                log( pow( rho, gamma ) * ( rhoE - ( rhoU2 + rhoV2 ) / ( 2 * rho ) ) );
        ds[1] = -( ( 2 * rho * rhoU ) / ( -2 * rho * rhoE + rhoU2 + rhoV2 ) );
        ds[2] = -( ( 2 * rho * rhoV ) / ( -2 * rho * rhoE + rhoU2 + rhoV2 ) );
        ds[3] = -( rho / ( rhoE - ( rhoU2 + rhoV2 ) / ( 2 * rho ) ) );
    }
};

// ---------------------------------------------------------------- shallow water 1-D
// ShallowWaterClosure (shallowwaterclosure.cpp:10-42), g = 9.81.
template <> struct Closure<2> {
    static constexpr int NS = 2, NP = 3;
    static constexpr bool LINEAR = false;
    __host__ __device__ static void U( const double* L, double* u, bool, const PhysParams& ) {
        const double gr = 9.81;
        u[0] = ( 0.5 * ( 2 * L[0] + L[1] * L[1] ) ) / gr;
        u[1] = ( 0.5 * ( 2 * L[0] * L[1] + L[1] * L[1] * L[1] ) ) / gr;
    }
    __host__ __device__ static void DU( const double* L, double* y, const PhysParams& ) {
        const double gr = 9.81;
        y[0] = 1.0 / gr;
        y[1] = L[1] / gr;
        y[2] = ( L[0] + 1.5 * ( L[1] * L[1] ) ) / gr;
    }
    __host__ __device__ static void DS( const double* u, double* ds, const PhysParams& ) {
        const double gr = 9.81;
        ds[0] = ( gr * ( u[0] * u[0] * u[0] ) - 0.5 * ( u[1] * u[1] ) ) / ( u[0] * u[0] );
        ds[1] = u[1] / u[0];
    }
};

// ---------------------------------------------------------------- linear closures
// Stochastic Galerkin and the filtered forms (stochasticgalerkin.cpp:7-17,
// l2filter.cpp:29-43, lassofilter.cpp:36-60): the
// ansatz is the polynomial itself, U(Lambda) = Lambda, DU = identity, and the
// duals come from the moments without a Newton solve (linear_duals in
// ipm_kernels.cuh). Kinds 3, 4, 5 carry the states of Burgers, 2-D Euler and
// shallow water; DS of the base class (zero) is the initial guess.
template <int NSV> struct LinearClosure {
    static constexpr int NS = NSV, NP = NSV * ( NSV + 1 ) / 2;
    static constexpr bool LINEAR = true;
    __host__ __device__ static void U( const double* L, double* u, bool, const PhysParams& ) {
        for( int s = 0; s < NS; ++s ) u[s] = L[s];
    }
    __host__ __device__ static void DU( const double*, double* du, const PhysParams& ) {
        int p = 0;
        for( int a = 0; a < NS; ++a )
            for( int b = a; b < NS; ++b ) du[p++] = a == b ? 1.0 : 0.0;
    }
    __host__ __device__ static void DS( const double*, double* ds, const PhysParams& ) {
        for( int s = 0; s < NS; ++s ) ds[s] = 0.0;
    }
};
template <> struct Closure<3> : LinearClosure<1> {};
template <> struct Closure<4> : LinearClosure<4> {};
template <> struct Closure<5> : LinearClosure<2> {};
template <> struct Closure<7> : LinearClosure<3> {};

// ---------------------------------------------------------------- LogSin
// LogSin (logsin.cpp:3-50): one state, U = ((u+ - u-) / PI) (PI / 2 + atan
// Lambda) + u-, DU = ((u+ - u-) / PI) / (Lambda^2 + 1), with the reference's
// PI = 3.14159265359 (mathtools.h:8) and its fixed bounds: u- = 1 - 0.1,
// u+ = 12 + 0.1 + 0.2 with two uncertain dimensions, else u- = 3 - 0.1,
// u+ = 12 + 0.1. DS of the base class (zero).
template <> struct Closure<8> {
    static constexpr int NS = 1, NP = 1;
    static constexpr bool LINEAR = false;
    __host__ __device__ static void bounds( const PhysParams& p, double& lo, double& hi ) {
        const double du = 0.1;
        lo              = p.dimXi == 2 ? 1.0 - du : 3.0 - du;
        hi              = p.dimXi == 2 ? 12.0 + du + 0.2 : 12.0 + du;
    }
    __host__ __device__ static void U( const double* L, double* u, bool, const PhysParams& p ) {
        const double pi = 3.14159265359;
        double lo, hi;
        bounds( p, lo, hi );
        u[0] = ( ( hi - lo ) / pi ) * ( pi / 2 + atan( L[0] ) ) + lo;
    }
    __host__ __device__ static void DU( const double* L, double* du, const PhysParams& p ) {
        const double pi = 3.14159265359;
        double lo, hi;
        bounds( p, lo, hi );
        du[0] = ( ( hi - lo ) / pi ) / ( L[0] * L[0] + 1.0 );
    }
    __host__ __device__ static void DS( const double*, double* ds, const PhysParams& ) { ds[0] = 0.0; }
};

// ---------------------------------------------------------------- Euler 1-D
// EulerClosure (eulerclosure.cpp:7-80): three states (rho, rho u, rho E), the
// gamma of [problem] gamma. DU is packed as the entries the reference's Newton
// reads: the Hessian block (m, l), m <= l, takes DU(l, m) (closure.cpp:255-270)
// and posv reads the upper triangle (uplo 'U', vectorspace.cpp:152-171), so the
// pair (m, l) holds the reference's y(l, m) (its lower triangle and diagonal,
// with y(2, 2) as written there).
template <> struct Closure<6> {
    static constexpr int NS = 3, NP = 6;
    static constexpr bool LINEAR = false;
    __host__ __device__ static double E( const double* L, const PhysParams& p ) {
        const double g = p.gamma;
        return exp( ( 2.0 * L[0] * L[2] - 2.0 * L[2] * log( -L[2] ) - 2.0 * L[2] * g - L[1] * L[1] ) / ( 2.0 * L[2] * ( g - 1.0 ) ) );
    }
    __host__ __device__ static void U( const double* L, double* u, bool, const PhysParams& p ) {
        u[0] = E( L, p );
        u[1] = -( L[1] / L[2] ) * u[0];
        u[2] = ( ( L[1] * L[1] - 2.0 * L[2] ) / ( 2.0 * ( L[2] * L[2] ) ) ) * u[0];
    }
    __host__ __device__ static void DU( const double* L, double* y, const PhysParams& p ) {
        const double g = p.gamma, e = E( L, p ), l2sq = L[2] * L[2];
        const double d1 = ( 1.0 / ( g - 1.0 ) ) * e;
        const double d2 = -( L[1] / ( L[2] * ( g - 1.0 ) ) ) * e;
        const double d3 = ( ( -2.0 * g + 2.0 * L[0] - 2.0 * log( -L[2] ) - 2.0 ) / ( 2.0 * ( g - 1.0 ) * L[2] ) -
                            ( -2.0 * g * L[2] + 2.0 * L[0] * L[2] - L[1] * L[1] - 2.0 * L[2] * log( -L[2] ) ) / ( 2.0 * ( g - 1.0 ) * l2sq ) ) *
                          e;
        const double c = ( L[1] * L[1] - 2.0 * L[2] ) / ( 2.0 * l2sq );
        y[0] = d1;                                                                        // (0, 0)
        y[1] = -( L[1] / L[2] ) * d1;                                                     // y(1, 0)
        y[2] = c * d1;                                                                    // y(2, 0)
        y[3] = -( 1.0 / L[2] ) * e - ( L[1] / L[2] ) * d2;                                // y(1, 1)
        y[4] = c * d2 + ( 2.0 * L[1] / ( 2.0 * l2sq ) ) * e;                              // y(2, 1)
        y[5] = ( L[1] * L[1] / pow( L[2], -3.0 ) + pow( L[2], -2.0 ) ) * e + c * d3;    // y(2, 2)
    }
    __host__ __device__ static void DS( const double* u, double* ds, const PhysParams& p ) {
        const double gamma = -p.gamma, rho = u[0], rhoU = u[1], rhoU2 = rhoU * rhoU, rhoE = u[2];
        ds[0] = ( rhoU2 + gamma * ( 2 * rho * rhoE - rhoU2 ) ) / ( -2 * rho * rhoE + rhoU2 ) - log( pow( rho, gamma ) * ( rhoE - ( rhoU2 ) / ( 2 * rho ) ) );
        ds[1] = -( ( 2 * rho * rhoU ) / ( -2 * rho * rhoE + rhoU2 ) );
        ds[2] = -( rho / ( rhoE - ( rhoU2 ) / ( 2 * rho ) ) );
    }
};

// packed index of the symmetric pair (a, b)
template <int NS> __device__ __forceinline__ int pair_index( int a, int b ) {
    int lo = a < b ? a : b, hi = a < b ? b : a;
    return lo * NS - ( lo * ( lo - 1 ) ) / 2 + ( hi - lo );
}

// ---------------------------------------------------------------- problems
// Numerical flux g(u, v) for face unit normal nu, scaled normal n and face
// length nn = |n| (computed once per face by the caller).
template <int CL> struct Problem;

// Burgers with the local Lax-Friedrichs flux (julia/Tensorization/IPMSolver.jl:38-42)
// and CFL rule of burgers.cpp:114-122; ramp initial state (burgers.cpp:48-68).
template <> struct Problem<0> {
    __device__ static void flux( const double* u, const double* v, const double*, const double* n, double, double* y, const PhysParams& ) {
        double beta = fabs( u[0] ) < fabs( v[0] ) ? fabs( v[0] ) : fabs( u[0] );
        y[0]        = 0.5 * ( 0.5 * u[0] * u[0] + 0.5 * v[0] * v[0] ) * n[0] - 0.5 * beta * ( v[0] - u[0] ) * fabs( n[0] );
    }
    __device__ static double dt( const double* uq, double dx, const PhysParams& p ) { return p.cfl * dx / fabs( uq[0] ); }
    __device__ static void ic( const double* x, const double* xi, double* y, const PhysParams& p ) {
        double uL = p.ic[0], uR = p.ic[1], x0 = p.ic[2], x1 = p.ic[3], s = p.sigma[0];
        if( x[0] < x0 + s * xi[0] )
            y[0] = uL;
        else if( x[0] < x1 + s * xi[0] )
            y[0] = uL + ( uR - uL ) * ( x0 + s * xi[0] - x[0] ) / ( x0 - x1 );
        else
            y[0] = uR;
    }
};

// Euler 2-D: HLL flux (euler2d.cpp:52-87), physical flux F (:89-106), CFL rule
// (:114-134); Sod-type initial state with uncertain interface, density, pressure.
template <> struct Problem<1> {
    __device__ static void Fn( double gm, const double* u, const double* n, double* out ) {
        double rhoInv = 1.0 / u[0], v1 = u[1] * rhoInv, v2 = u[2] * rhoInv;
        double p = ( gm - 1.0 ) * ( u[3] - 0.5 * u[0] * ( v1 * v1 + v2 * v2 ) );
        out[0]   = u[1] * n[0] + u[2] * n[1];
        out[1]   = ( u[1] * v1 + p ) * n[0] + ( u[2] * v1 ) * n[1];
        out[2]   = ( u[1] * v2 ) * n[0] + ( u[2] * v2 + p ) * n[1];
        out[3]   = ( ( u[3] + p ) * v1 ) * n[0] + ( ( u[3] + p ) * v2 ) * n[1];
    }
    __device__ static void flux( const double* u, const double* v, const double* nu, const double* n, double nn, double* y,
                                 const PhysParams& P ) {
        const double gm = P.gamma;
        double rhoInv = 1.0 / u[0], uU = u[1] * rhoInv, vU = u[2] * rhoInv;
        double p  = ( gm - 1.0 ) * ( u[3] - 0.5 * u[0] * ( uU * uU + vU * vU ) );
        double aU = sqrt( gm * p * rhoInv );
        rhoInv    = 1.0 / v[0];
        double uV = v[1] * rhoInv, vV = v[2] * rhoInv;
        p         = ( gm - 1.0 ) * ( v[3] - 0.5 * v[0] * ( uV * uV + vV * vV ) );
        double aV = sqrt( gm * p * rhoInv );
        double lmin = ( nu[0] * uU + nu[1] * vU ) - aU;
        double lmax = ( nu[0] * uV + nu[1] * vV ) + aV;
        if( lmin >= 0 )
            Fn( gm, u, n, y );
        else if( lmax <= 0 )
            Fn( gm, v, n, y );
        else {
            double fu[4], fv[4];
            Fn( gm, u, n, fu );
            Fn( gm, v, n, fv );
            double ll = lmax * lmin, inv = 1.0 / ( lmax - lmin );
            for( int i = 0; i < 4; ++i ) y[i] = inv * ( ( lmax * fu[i] - lmin * fv[i] ) + ll * ( v[i] - u[i] ) * nn );
        }
    }
    __device__ static double dt( const double* uq, double dx, const PhysParams& P ) {
        const double gm = P.gamma;
        double rhoInv = 1.0 / uq[0], uU = uq[1] * rhoInv, vU = uq[2] * rhoInv;
        double p = ( gm - 1.0 ) * ( uq[3] - 0.5 * uq[0] * ( uU * uU + vU * vU ) );
        double a = sqrt( gm * p * rhoInv );
        // the minimum of |1 / (v -+ a)| and |1 / (u +- a)| (euler2d.cpp:114-134)
        // is 1 / the maximum of the four |.|: the rounded reciprocal is
        // monotone, so both give the same double
        const double w = fmax( fmax( fabs( vU - a ), fabs( vU + a ) ), fmax( fabs( uU + a ), fabs( uU - a ) ) );
        return ( P.cfl / dx ) * ( 1.0 / w );
    }
    __device__ static void ic( const double* x, const double* xi, double* y, const PhysParams& P ) {
        double rho, pr;
        if( x[0] < P.ic[0] + P.sigma[0] * xi[0] ) {
            rho = P.ic[1] * ( 1.0 + ( P.dimXi > 1 ? P.sigma[1] * xi[1] : 0.0 ) );
            pr  = P.ic[2] * ( 1.0 + ( P.dimXi > 2 ? P.sigma[2] * xi[2] : 0.0 ) );
        }
        else {
            rho = P.ic[3];
            pr  = P.ic[4];
        }
        y[0] = rho;
        y[1] = 0.0;
        y[2] = 0.0;
        y[3] = pr / ( P.gamma - 1.0 );
    }
};

// Shallow water 1-D: Lax-Friedrichs with dx/dt = 12 / CFL (shallowwater.cpp:21-35);
// time step Settings::GetDT (problem.cpp:44); dam-break initial state.
template <> struct Problem<2> {
    __device__ static void flux( const double* u, const double* v, const double*, const double* n, double, double* y,
                                 const PhysParams& P ) {
        const double gr = 9.81;
        double s        = 0.5 / ( P.cfl / 12.0 );
        double fl1 = ( u[1] * u[1] ) / u[0] + 0.5 * gr * ( u[0] * u[0] );
        double fr1 = ( v[1] * v[1] ) / v[0] + 0.5 * gr * ( v[0] * v[0] );
        y[0]       = 0.5 * ( u[1] * n[0] + v[1] * n[0] ) - s * ( v[0] - u[0] );
        y[1]       = 0.5 * ( fl1 * n[0] + fr1 * n[0] ) - s * ( v[1] - u[1] );
    }
    __device__ static double dt( const double*, double, const PhysParams& P ) { return P.dtFixed; }
    __device__ static void ic( const double* x, const double* xi, double* y, const PhysParams& P ) {
        y[0] = x[0] < P.ic[0] ? P.ic[1] * ( 1.0 + P.sigma[0] * xi[0] ) : P.ic[2];
        y[1] = 0.0;
    }
};

// the linear closures' problems are those of the kinds with the same states
template <> struct Problem<3> : Problem<0> {};
template <> struct Problem<4> : Problem<1> {};
template <> struct Problem<5> : Problem<2> {};

// Euler 1-D (euler.cpp:23-128): HLL flux with the projected velocities, CFL
// rule min over nodes of cfl dx min(|1 / (v - a)|, |1 / (v + a)|), Sod initial
// state x0 = 0.3 + s0 xi0, left (1, 0, 1), right (0.3 + s1 xi1, 0, 0.3 + s2
// xi2) with gamma 1.4 in the initial state (the reference's fixed values;
// [uqc] ic = [x0, rhoL, pL, rhoR, pR] replaces them).
template <> struct Problem<6> {
    __device__ static void F( double gm, const double* u, double n, double* f ) {
        const double rhoInv = 1.0 / u[0], v = u[1] * rhoInv;
        const double p      = ( gm - 1.0 ) * ( u[2] - 0.5 * u[0] * ( v * v ) );
        f[0]                = u[1] * n;
        f[1]                = ( u[1] * v + p ) * n;
        f[2]                = ( ( u[2] + p ) * v ) * n;
    }
    __device__ static void flux( const double* u, const double* v, const double* nu, const double* n, double nn, double* y,
                                 const PhysParams& P ) {
        const double gm = P.gamma;
        double rhoInv   = 1.0 / u[0];
        double vU       = u[1] * rhoInv;
        double p        = ( gm - 1.0 ) * ( u[2] - 0.5 * u[0] * ( vU * vU ) );
        double aU       = sqrt( gm * p * rhoInv );
        rhoInv          = 1.0 / v[0];
        double vV       = v[1] * rhoInv;
        p               = ( gm - 1.0 ) * ( v[2] - 0.5 * v[0] * ( vV * vV ) );
        double aV       = sqrt( gm * p * rhoInv );
        double lmin = nu[0] * vU - aU, lmax = nu[0] * vV + aV;
        if( lmin >= 0 )
            F( gm, u, n[0], y );
        else if( lmax <= 0 )
            F( gm, v, n[0], y );
        else {
            // (lmax F(u) n - lmin F(v) n + lmax lmin (v - u) |n|) / (lmax - lmin), in that order
            const double rU = 1.0 / u[0], wU = u[1] * rU, pU = ( gm - 1.0 ) * ( u[2] - 0.5 * u[0] * ( wU * wU ) );
            const double rV = 1.0 / v[0], wV = v[1] * rV, pV = ( gm - 1.0 ) * ( v[2] - 0.5 * v[0] * ( wV * wV ) );
            const double fu[3] = {u[1], u[1] * wU + pU, ( u[2] + pU ) * wU};
            const double fv[3] = {v[1], v[1] * wV + pV, ( v[2] + pV ) * wV};
            const double inv = 1.0 / ( lmax - lmin ), ll = lmax * lmin;
            for( int i = 0; i < 3; ++i ) y[i] = inv * ( ( ( lmax * fu[i] ) * n[0] - ( lmin * fv[i] ) * n[0] ) + ( ll * ( v[i] - u[i] ) ) * nn );
        }
    }
    __device__ static double dt( const double* uq, double dx, const PhysParams& P ) {
        const double gm = P.gamma, rhoInv = 1.0 / uq[0], v = uq[1] * rhoInv;
        const double p = ( gm - 1.0 ) * ( uq[2] - 0.5 * uq[0] * ( v * v ) ), a = sqrt( gm * p * rhoInv );
        return ( P.cfl * dx ) * fmin( fabs( 1.0 / ( v - a ) ), fabs( 1.0 / ( v + a ) ) );
    }
    __device__ static void ic( const double* x, const double* xi, double* y, const PhysParams& P ) {
        const double gic = 1.4;
        const bool own   = P.nIc >= 5;
        const double x0 = own ? P.ic[0] : 0.3, rhoL = own ? P.ic[1] : 1.0, pL = own ? P.ic[2] : 1.0;
        const double rhoR = own ? P.ic[3] : 0.3;
        double pR         = own ? P.ic[4] : 0.3;
        if( x[0] < x0 + P.sigma[0] * xi[0] ) {
            y[0] = rhoL;
            y[1] = rhoL * 0.0;
            y[2] = 0.5 * rhoL * ( 0.0 * 0.0 ) + ( pL / ( rhoL * ( gic - 1 ) ) ) * rhoL;
        }
        else {
            y[0] = rhoR;
            if( P.dimXi > 1 ) y[0] += P.sigma[1] * xi[1];
            if( P.dimXi > 2 ) pR += P.sigma[2] * xi[2];
            y[1] = rhoR * 0.0;
            y[2] = 0.5 * rhoR * ( 0.0 * 0.0 ) + ( pR / ( rhoR * ( gic - 1 ) ) ) * rhoR;
        }
    }
};
template <> struct Problem<7> : Problem<6> {};
template <> struct Problem<8> : Problem<0> {};    // LogSin with Burgers

}    // namespace uqc
