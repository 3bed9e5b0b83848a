#pragma once

#include "runtime.hpp"

namespace tempi {

int send_strided(TypeRecord &r, Method m, const void *buf, int count, int dest,
                 int tag, MPI_Comm comm);
int recv_strided(TypeRecord &r, Method m, void *buf, int count, int source,
                 int tag, MPI_Comm comm, MPI_Status *status);
int send_contiguous_staged(const void *buf, int count, MPI_Datatype dt,
                           int64_t bytes, int dest, int tag, MPI_Comm comm);
int recv_contiguous_staged(void *buf, int count, MPI_Datatype dt,
                           int64_t bytes, int source, int tag, MPI_Comm comm,
                           MPI_Status *status);

int start_isend(TypeRecord &r, Method m, const void *buf, int count, int dest,
                int tag, MPI_Comm comm, MPI_Request *request);
int start_irecv(TypeRecord &r, Method m, void *buf, int count, int source,
                int tag, MPI_Comm comm, MPI_Request *request);
int try_progress();
// start every managed send whose pack has finished, waiting (bounded) for
// packs still in flight
int progress_sends();
bool is_managed(MPI_Request r);
int wait_managed(MPI_Request *request, MPI_Status *status);
void async_finalize();

} // namespace tempi
