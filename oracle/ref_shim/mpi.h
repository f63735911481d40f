/* Minimal MPI declarations so the reference's single-rank tau00 path compiles
 * without an MPI installation.  Test infrastructure only (oracle build). */
#pragma once
typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Status;
typedef int MPI_Op;
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_CHAR 3
#define MPI_MAX 1
#define MPI_SUM 2
#define MPI_COMM_WORLD 0
static inline int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
double MPI_Wtime();
