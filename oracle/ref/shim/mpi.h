// Test-infrastructure shim: single-rank MPI so the reference's sources compile
// and run in one process. Only the calls made on the hot path exist
// (momentsolver.cpp:92-95,115-117,133,144-146,152; settings.cpp:27-28).
// With one rank a reduction is a copy of the send buffer into the receive
// buffer, and a broadcast is a no-op.
#pragma once
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_UNSIGNED 2
#define MPI_INT 3
#define MPI_SUM 10
#define MPI_MIN 11
#define MPI_MAX 12

inline int uqc_shim_mpi_size( MPI_Datatype t ) { return t == MPI_DOUBLE ? 8 : 4; }
inline int MPI_Init( int*, char*** ) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank( MPI_Comm, int* r ) { *r = 0; return 0; }
inline int MPI_Comm_size( MPI_Comm, int* s ) { *s = 1; return 0; }
inline int MPI_Bcast( void*, int, MPI_Datatype, int, MPI_Comm ) { return 0; }
inline int MPI_Reduce( const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm ) {
    if( s != r ) std::memcpy( r, s, size_t( n ) * uqc_shim_mpi_size( t ) );
    return 0;
}
inline int MPI_Allreduce( const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm ) {
    if( s != r ) std::memcpy( r, s, size_t( n ) * uqc_shim_mpi_size( t ) );
    return 0;
}
