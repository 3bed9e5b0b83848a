/* mpi.h -- header of libminimpi, a self-only MPI library (world size 1).

   No MPI implementation is installed on the machines this project runs on, so
   libminimpi plays the part of "the underlying MPI library" that the
   interposer (libtempi_b200.so) forwards to with dlsym(RTLD_NEXT).  It follows
   the MPI-3.1 C bindings for the calls it provides, with MPICH-style integer
   handles.  Communication is between rank 0 and itself only: sends are
   buffered eagerly and matched against posted receives in MPI order.
   Buffers may be host memory or CUDA device memory (copies use
   cudaMemcpyDefault), as in a CUDA-aware MPI.

   Only the constants and functions below exist.  A real MPI that provides the
   same symbols can replace libminimpi without rebuilding the interposer.
*/
#ifndef MINIMPI_MPI_H
#define MINIMPI_MPI_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Op;
typedef int MPI_Info;
typedef intptr_t MPI_Aint;
typedef long long MPI_Count;

typedef struct MPI_Status {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  int reserved_;
  long long bytes_; /* received byte count, read by MPI_Get_count */
} MPI_Status;

#define MPI_VERSION 3
#define MPI_SUBVERSION 1

/* error classes */
#define MPI_SUCCESS 0
#define MPI_ERR_BUFFER 1
#define MPI_ERR_COUNT 2
#define MPI_ERR_TYPE 3
#define MPI_ERR_TAG 4
#define MPI_ERR_COMM 5
#define MPI_ERR_RANK 6
#define MPI_ERR_REQUEST 7
#define MPI_ERR_TRUNCATE 15
#define MPI_ERR_ARG 12
#define MPI_ERR_OTHER 16
#define MPI_ERR_INTERN 17
#define MPI_ERR_PENDING 18
#define MPI_ERR_UNKNOWN 13
#define MPI_ERR_NO_MEM 34
#define MPI_ERR_LASTCODE 0x3fffffff

/* communicators */
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2

/* named datatypes */
#define MPI_DATATYPE_NULL 0
#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_UNSIGNED_CHAR 3
#define MPI_SHORT 4
#define MPI_INT 5
#define MPI_UNSIGNED 6
#define MPI_LONG 7
#define MPI_LONG_LONG 8
#define MPI_FLOAT 9
#define MPI_DOUBLE 10
#define MPI_PACKED 11
#define MPI_INT64_T 12
#define MPI_UINT64_T 13
#define MPI_LONG_LONG_INT MPI_LONG_LONG

/* type constructors, as reported by MPI_Type_get_envelope */
#define MPI_COMBINER_NAMED 1
#define MPI_COMBINER_DUP 2
#define MPI_COMBINER_CONTIGUOUS 3
#define MPI_COMBINER_VECTOR 4
#define MPI_COMBINER_HVECTOR 6
#define MPI_COMBINER_INDEXED 7
#define MPI_COMBINER_HINDEXED 9
#define MPI_COMBINER_INDEXED_BLOCK 10
#define MPI_COMBINER_HINDEXED_BLOCK 11
#define MPI_COMBINER_STRUCT 13
#define MPI_COMBINER_SUBARRAY 14
#define MPI_COMBINER_DARRAY 15
#define MPI_COMBINER_RESIZED 18

#define MPI_ORDER_C 56
#define MPI_ORDER_FORTRAN 57

#define MPI_REQUEST_NULL 0
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-1)
#define MPI_UNDEFINED (-32766)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define MPI_MAX_LIBRARY_VERSION_STRING 256

/* distributed graph topologies */
#define MPI_INFO_NULL 0
#define MPI_UNWEIGHTED ((int *)1)
#define MPI_WEIGHTS_EMPTY ((int *)2)

/* environment */
int MPI_Init(int *argc, char ***argv);
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Finalize(void);
int MPI_Initialized(int *flag);
int MPI_Finalized(int *flag);
int MPI_Abort(MPI_Comm comm, int errorcode);
double MPI_Wtime(void);
int MPI_Get_library_version(char *version, int *resultlen);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Barrier(MPI_Comm comm);
int MPI_Alltoallv(const void *sendbuf, const int sendcounts[], const int sdispls[],
                  MPI_Datatype sendtype, void *recvbuf, const int recvcounts[],
                  const int rdispls[], MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Error_string(int errorcode, char *string, int *resultlen);

/* datatypes */
int MPI_Type_contiguous(int count, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_vector(int count, int blocklength, int stride,
                    MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_hvector(int count, int blocklength, MPI_Aint stride,
                            MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_indexed(int count, const int array_of_blocklengths[],
                     const int array_of_displacements[], MPI_Datatype oldtype,
                     MPI_Datatype *newtype);
int MPI_Type_create_hindexed(int count, const int array_of_blocklengths[],
                             const MPI_Aint array_of_displacements[],
                             MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_indexed_block(int count, int blocklength,
                                  const int array_of_displacements[],
                                  MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_hindexed_block(int count, int blocklength,
                                   const MPI_Aint array_of_displacements[],
                                   MPI_Datatype oldtype,
                                   MPI_Datatype *newtype);
int MPI_Type_create_struct(int count, const int array_of_blocklengths[],
                           const MPI_Aint array_of_displacements[],
                           const MPI_Datatype array_of_types[],
                           MPI_Datatype *newtype);
int MPI_Type_create_subarray(int ndims, const int array_of_sizes[],
                             const int array_of_subsizes[],
                             const int array_of_starts[], int order,
                             MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_resized(MPI_Datatype oldtype, MPI_Aint lb, MPI_Aint extent,
                            MPI_Datatype *newtype);
int MPI_Type_dup(MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *datatype);
int MPI_Type_free(MPI_Datatype *datatype);
int MPI_Type_size(MPI_Datatype datatype, int *size);
int MPI_Type_get_extent(MPI_Datatype datatype, MPI_Aint *lb, MPI_Aint *extent);
int MPI_Type_get_true_extent(MPI_Datatype datatype, MPI_Aint *true_lb,
                             MPI_Aint *true_extent);
int MPI_Type_get_envelope(MPI_Datatype datatype, int *num_integers,
                          int *num_addresses, int *num_datatypes,
                          int *combiner);
int MPI_Type_get_contents(MPI_Datatype datatype, int max_integers,
                          int max_addresses, int max_datatypes,
                          int array_of_integers[],
                          MPI_Aint array_of_addresses[],
                          MPI_Datatype array_of_datatypes[]);

/* packing */
int MPI_Pack(const void *inbuf, int incount, MPI_Datatype datatype,
             void *outbuf, int outsize, int *position, MPI_Comm comm);
int MPI_Unpack(const void *inbuf, int insize, int *position, void *outbuf,
               int outcount, MPI_Datatype datatype, MPI_Comm comm);
int MPI_Pack_size(int incount, MPI_Datatype datatype, MPI_Comm comm,
                  int *size);

/* point to point (self only) */
int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest,
             int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status);
int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest,
              int tag, MPI_Comm comm, MPI_Request *request);
int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
              MPI_Comm comm, MPI_Request *request);
int MPI_Send_init(const void *buf, int count, MPI_Datatype datatype, int dest,
                  int tag, MPI_Comm comm, MPI_Request *request);
int MPI_Recv_init(void *buf, int count, MPI_Datatype datatype, int source,
                  int tag, MPI_Comm comm, MPI_Request *request);
int MPI_Start(MPI_Request *request);
int MPI_Test(MPI_Request *request, int *flag, MPI_Status *status);
int MPI_Wait(MPI_Request *request, MPI_Status *status);
int MPI_Waitall(int count, MPI_Request array_of_requests[],
                MPI_Status array_of_statuses[]);
int MPI_Request_free(MPI_Request *request);
int MPI_Get_count(const MPI_Status *status, MPI_Datatype datatype, int *count);

/* distributed graph communicators (MPI-3.1 7.5.4) and neighbourhood
   collectives (7.6).  In a world of one rank every neighbour is rank 0;
   the k-th edge to a neighbour is matched with the k-th edge from it, in
   the order the neighbour lists give. */
int MPI_Dist_graph_create_adjacent(MPI_Comm comm_old, int indegree,
                                   const int sources[],
                                   const int sourceweights[], int outdegree,
                                   const int destinations[],
                                   const int destweights[], MPI_Info info,
                                   int reorder, MPI_Comm *comm_dist_graph);
int MPI_Dist_graph_neighbors_count(MPI_Comm comm, int *indegree,
                                   int *outdegree, int *weighted);
int MPI_Dist_graph_neighbors(MPI_Comm comm, int maxindegree, int sources[],
                             int sourceweights[], int maxoutdegree,
                             int destinations[], int destweights[]);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Neighbor_alltoallv(const void *sendbuf, const int sendcounts[],
                           const int sdispls[], MPI_Datatype sendtype,
                           void *recvbuf, const int recvcounts[],
                           const int rdispls[], MPI_Datatype recvtype,
                           MPI_Comm comm);
int MPI_Neighbor_alltoallw(const void *sendbuf, const int sendcounts[],
                           const MPI_Aint sdispls[],
                           const MPI_Datatype sendtypes[], void *recvbuf,
                           const int recvcounts[], const MPI_Aint rdispls[],
                           const MPI_Datatype recvtypes[], MPI_Comm comm);

#ifdef __cplusplus
}
#endif

#endif /* MINIMPI_MPI_H */
