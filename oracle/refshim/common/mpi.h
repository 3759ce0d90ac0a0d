/* one-rank stand-in for <mpi.h>; the MPI calls themselves are macros in snac_shim_core.h */
#ifndef SNAC_SHIM_MPI_H
#define SNAC_SHIM_MPI_H
typedef int MPI_Comm;
typedef struct { int dummy; } MPI_Status;
#define MPI_DOUBLE 0
#define MPI_MAX 0
#define MPI_MIN 1
#endif
