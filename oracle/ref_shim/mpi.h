// Stand-in for mpi.h: the compiled CPU kernels never call MPI.
#ifndef RTM_SHIM_MPI_H
#define RTM_SHIM_MPI_H
#endif
