// MPIsetting.h — for callers written against the reference's headers
// (3DgrainMPI/MPIsetting.h): the driver's single-process MPI setting under the
// reference's names, and, unless CUPF_USE_MPI is defined (then <mpi.h> is
// used), a single-process stand-in for the MPI calls of the reference's
// main.cpp (MPI_Init, MPI_Comm_rank, MPI_Comm_size, MPI_Finalize): one process
// drives the whole domain on one GPU.
#pragma once
#ifdef CUPF_USE_MPI
#include <mpi.h>
#else
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return 0; }
#endif
#include "../phase_field.h"
using cupf_host::MPIsetting;
using cupf_host::MPIsetting1D;
using cupf_host::MPIsetting2D;
