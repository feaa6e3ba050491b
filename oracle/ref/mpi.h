/* Minimal single-rank stand-in for <mpi.h>, used only to compile the reference
 * cuPF sources into the parity harness (test infrastructure).  Every call is a
 * no-op for rank 0 of a world of size 1. */
#pragma once
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_FLOAT 1
#define MPI_INT 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
