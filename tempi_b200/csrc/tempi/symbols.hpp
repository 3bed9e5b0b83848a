// The underlying MPI library, reached with dlsym(RTLD_NEXT) so that this
// library's own MPI_* definitions (the interposed entry points) can forward
// to it.  Same role as the reference's MpiFunc table
// (include/symbols.hpp:180-212, src/internal/symbols.cpp:22-90).
//
// Differences: every MPI call made inside TEMPI goes through this table
// (so the library has no undefined MPI symbols and loads without an MPI
// already present), resolution happens on first use rather than in MPI_Init,
// and when RTLD_NEXT finds nothing the library opens $TEMPI_LIBMPI, then
// libmpi.so, then libminimpi.so (searched next to this library).
#pragma once

#include <mpi.h>

namespace tempi {

struct LibMPI {
  int (*Init)(int *, char ***);
  int (*Init_thread)(int *, char ***, int, int *);
  int (*Finalize)(void);
  int (*Comm_rank)(MPI_Comm, int *);
  int (*Comm_size)(MPI_Comm, int *);
  int (*Type_commit)(MPI_Datatype *);
  int (*Type_free)(MPI_Datatype *);
  int (*Type_size)(MPI_Datatype, int *);
  int (*Type_get_extent)(MPI_Datatype, MPI_Aint *, MPI_Aint *);
  int (*Type_get_envelope)(MPI_Datatype, int *, int *, int *, int *);
  int (*Type_get_contents)(MPI_Datatype, int, int, int, int[], MPI_Aint[],
                           MPI_Datatype[]);
  int (*Pack)(const void *, int, MPI_Datatype, void *, int, int *, MPI_Comm);
  int (*Unpack)(const void *, int, int *, void *, int, MPI_Datatype, MPI_Comm);
  int (*Pack_size)(int, MPI_Datatype, MPI_Comm, int *);
  int (*Send)(const void *, int, MPI_Datatype, int, int, MPI_Comm);
  int (*Recv)(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *);
  int (*Isend)(const void *, int, MPI_Datatype, int, int, MPI_Comm,
               MPI_Request *);
  int (*Irecv)(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *);
  int (*Send_init)(const void *, int, MPI_Datatype, int, int, MPI_Comm,
                   MPI_Request *);
  int (*Start)(MPI_Request *);
  int (*Test)(MPI_Request *, int *, MPI_Status *);
  int (*Wait)(MPI_Request *, MPI_Status *);
  int (*Request_free)(MPI_Request *);
  int (*Type_contiguous)(int, MPI_Datatype, MPI_Datatype *);
  int (*Type_create_hvector)(int, int, MPI_Aint, MPI_Datatype, MPI_Datatype *);
  int (*Type_create_resized)(MPI_Datatype, MPI_Aint, MPI_Aint, MPI_Datatype *);
  int (*Dist_graph_neighbors_count)(MPI_Comm, int *, int *, int *);
  int (*Dist_graph_neighbors)(MPI_Comm, int, int[], int[], int, int[], int[]);
  int (*Neighbor_alltoallw)(const void *, const int[], const MPI_Aint[],
                            const MPI_Datatype[], void *, const int[],
                            const MPI_Aint[], const MPI_Datatype[], MPI_Comm);
  int (*Alltoallv)(const void *, const int[], const int[], MPI_Datatype,
                   void *, const int[], const int[], MPI_Datatype, MPI_Comm);
};

// Resolve the table once; returns false (and logs) if any symbol is missing.
bool resolve_symbols();
extern LibMPI libmpi;

} // namespace tempi
