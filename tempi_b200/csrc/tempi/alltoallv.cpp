// Interposed MPI_Alltoallv on device buffers (reference src/alltoallv.cpp:
// 14-66 and the methods of src/internal/alltoallv_impl.cpp:21-258).
//
// Same decision order as the reference: the library takes the call when
// TEMPI is disabled or TEMPI_NO_ALLTOALLV is set, when either buffer is
// memory the GPU cannot reach, and when the communicator is not
// MPI_COMM_WORLD; otherwise one of four methods runs (TEMPI_ALLTOALLV_*,
// default STAGED as the reference's AUTO):
//
//   STAGED              the send blocks to pinned host memory, the library's
//                       MPI_Alltoallv between host buffers, the received
//                       blocks back to the device
//   REMOTE_FIRST        an MPI_Isend per destination (ranks on other nodes
//                       first), an MPI_Irecv per source, then waits
//   ISIR_STAGED         STAGED's copies around REMOTE_FIRST's Isend/Irecv
//   ISIR_REMOTE_STAGED  only blocks to and from ranks on other nodes go
//                       through host memory; blocks between ranks that share
//                       a node stay on the device
//
// Differences, each deliberate:
//  * displacements count extents of the datatype, as MPI defines them (the
//    reference adds them to the buffer as bytes, right only for MPI_BYTE);
//  * the staging buffers are the pinned slabs of the senders, and the copies
//    run on TEMPI's link stream;
//  * only the received blocks are copied back to the device, so bytes of
//    the receive buffer between blocks are never written (the reference
//    copies the whole receive span back, over them);
//  * types whose elements are not dense (size != extent, or lb != 0) go to
//    the library, which handles them;
//  * ranks share a node unless TEMPI_RANKS_PER_NODE=k says ranks r and s
//    share one only when r/k == s/k (the reference learns node names with an
//    MPI exchange at init, src/internal/topology.cpp; topology is outside
//    this library's scope).
//  * errors are returned as MPI codes; nothing exits.

#include "internal.hpp"
#include "runtime.hpp"
#include "sender.hpp"
#include "symbols.hpp"

#include <mpi.h>

#include <algorithm>
#include <vector>

namespace tempi {
namespace {

struct Args {
  const void *sendbuf;
  const int *sendcounts, *sdispls;
  MPI_Datatype sendtype;
  void *recvbuf;
  const int *recvcounts, *rdispls;
  MPI_Datatype recvtype;
  MPI_Comm comm;
  int size = 0, rank = 0;
  int64_t sext = 0, rext = 0; // extents (= sizes) of the two types
};

// bytes from the buffer start to the end of the last block
int64_t span(const int *counts, const int *displs, int n, int64_t ext) {
  int64_t hi = 0;
  for (int i = 0; i < n; ++i)
    if (counts[i] > 0)
      hi = std::max(hi, (int64_t(displs[i]) + counts[i]) * ext);
  return hi;
}

bool colocated(int a, int b) {
  const int k = env().ranks_per_node;
  return k <= 0 || a / k == b / k;
}

// whether a type's elements are dense (size == extent, lb == 0); *ext = its
// extent
bool dense_type(MPI_Datatype t, int64_t *ext) {
  int size = 0;
  MPI_Aint lb = 0, extent = 0;
  if (libmpi.Type_size(t, &size) != MPI_SUCCESS ||
      libmpi.Type_get_extent(t, &lb, &extent) != MPI_SUCCESS)
    return false;
  *ext = extent;
  return lb == 0 && int64_t(size) == int64_t(extent);
}

int copy(void *dst, const void *src, int64_t n, cudaStream_t s) {
  if (n <= 0)
    return TEMPI_OK;
  cudaError_t e = cudaMemcpyAsync(dst, src, size_t(n), cudaMemcpyDefault, s);
  return e == cudaSuccess ? TEMPI_OK : cuda_error(e, "alltoallv staging copy");
}

int sync(cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? TEMPI_OK : cuda_error(e, "alltoallv staging");
}

int to_mpi(int e) {
  return e == TEMPI_OK ? MPI_SUCCESS
         : e == TEMPI_ERR_NO_MEM ? MPI_ERR_NO_MEM
                                 : MPI_ERR_OTHER;
}

// Host staging of the blocks with `pick(rank)` true: the send blocks (or, with
// the whole span, every send byte) out of the device, and later the received
// blocks back in.
struct Staging {
  char *hs = nullptr, *hr = nullptr;
  int64_t ns = 0, nr = 0;
  ~Staging() {
    slab_free(Space::HOST_MAPPED, hs);
    slab_free(Space::HOST_MAPPED, hr);
  }
  int alloc(const Args &a) {
    ns = span(a.sendcounts, a.sdispls, a.size, a.sext);
    nr = span(a.recvcounts, a.rdispls, a.size, a.rext);
    if (ns > 0 && !(hs = static_cast<char *>(slab_alloc(Space::HOST_MAPPED, size_t(ns)))))
      return TEMPI_ERR_NO_MEM;
    if (nr > 0 && !(hr = static_cast<char *>(slab_alloc(Space::HOST_MAPPED, size_t(nr)))))
      return TEMPI_ERR_NO_MEM;
    return TEMPI_OK;
  }
  template <typename Pick> int out(const Args &a, Pick pick, cudaStream_t s) {
    for (int j = 0; j < a.size; ++j) {
      if (!pick(j) || a.sendcounts[j] <= 0)
        continue;
      const int64_t off = int64_t(a.sdispls[j]) * a.sext;
      if (int e = copy(hs + off, static_cast<const char *>(a.sendbuf) + off,
                       int64_t(a.sendcounts[j]) * a.sext, s))
        return e;
    }
    return sync(s);
  }
  template <typename Pick> int in(const Args &a, Pick pick, cudaStream_t s) {
    for (int i = 0; i < a.size; ++i) {
      if (!pick(i) || a.recvcounts[i] <= 0)
        continue;
      const int64_t off = int64_t(a.rdispls[i]) * a.rext;
      if (int e = copy(static_cast<char *>(a.recvbuf) + off, hr + off,
                       int64_t(a.recvcounts[i]) * a.rext, s))
        return e;
    }
    return sync(s);
  }
};

int staged(const Args &a) {
  counters().alltoallv_staged++;
  cudaStream_t s = link_stream();
  Staging st;
  int e = st.alloc(a);
  auto all = [](int) { return true; };
  if (!e)
    e = st.out(a, all, s);
  if (e)
    return to_mpi(e);
  int m = libmpi.Alltoallv(st.hs, a.sendcounts, a.sdispls, a.sendtype, st.hr,
                           a.recvcounts, a.rdispls, a.recvtype, a.comm);
  if (m)
    return m;
  return to_mpi(st.in(a, all, s));
}

// a tag of its own, so these blocks never match a user's messages (the
// reference uses tag 0)
constexpr int kTag = 0x7ee2;

// Isend of every block, `first` ranks' before the others, then an Irecv per
// source, then waits for all; send_at / recv_at: where block j of each side
// is (the device buffers, or host staging)
template <typename First, typename SendAt, typename RecvAt>
int isir(const Args &a, First first, SendAt send_at, RecvAt recv_at) {
  std::vector<MPI_Request> reqs;
  int err = MPI_SUCCESS;
  for (int pass = 0; pass < 2 && !err; ++pass)
    for (int j = 0; j < a.size && !err; ++j) {
      if (first(j) != (pass == 0))
        continue;
      MPI_Request q = MPI_REQUEST_NULL;
      err = MPI_Isend(send_at(j), a.sendcounts[j], a.sendtype, j, kTag, a.comm, &q);
      reqs.push_back(q);
    }
  for (int i = 0; i < a.size && !err; ++i) {
    MPI_Request q = MPI_REQUEST_NULL;
    err = MPI_Irecv(recv_at(i), a.recvcounts[i], a.recvtype, i, kTag, a.comm, &q);
    reqs.push_back(q);
  }
  for (MPI_Request &q : reqs) { // every posted request is completed
    const int e = q == MPI_REQUEST_NULL ? MPI_SUCCESS : MPI_Wait(&q, MPI_STATUS_IGNORE);
    err = err ? err : e;
  }
  return err;
}

int remote_first(const Args &a) {
  counters().alltoallv_remote_first++;
  return isir(
      a, [&](int j) { return !colocated(a.rank, j); },
      [&](int j) {
        return static_cast<const char *>(a.sendbuf) + int64_t(a.sdispls[j]) * a.sext;
      },
      [&](int i) {
        return static_cast<char *>(a.recvbuf) + int64_t(a.rdispls[i]) * a.rext;
      });
}

int isir_staged(const Args &a, bool remote_only) {
  (remote_only ? counters().alltoallv_isir_remote_staged
               : counters().alltoallv_isir_staged)++;
  cudaStream_t s = link_stream();
  auto via_host = [&](int j) { return !remote_only || !colocated(a.rank, j); };
  bool any = false;
  for (int j = 0; j < a.size; ++j)
    any = any || via_host(j);
  Staging st;
  int e = any ? st.alloc(a) : TEMPI_OK;
  if (!e && any)
    e = st.out(a, via_host, s);
  if (e)
    return to_mpi(e);
  int m = isir(
      a, [&](int j) { return !colocated(a.rank, j); },
      [&](int j) -> const void * {
        const int64_t off = int64_t(a.sdispls[j]) * a.sext;
        return via_host(j) ? st.hs + off : static_cast<const char *>(a.sendbuf) + off;
      },
      [&](int i) -> void * {
        const int64_t off = int64_t(a.rdispls[i]) * a.rext;
        return via_host(i) ? st.hr + off : static_cast<char *>(a.recvbuf) + off;
      });
  if (m)
    return m;
  return any ? to_mpi(st.in(a, via_host, s)) : MPI_SUCCESS;
}

} // namespace
} // namespace tempi

using namespace tempi;

extern "C" int MPI_Alltoallv(const void *sendbuf, const int sendcounts[],
                             const int sdispls[], MPI_Datatype sendtype,
                             void *recvbuf, const int recvcounts[],
                             const int rdispls[], MPI_Datatype recvtype,
                             MPI_Comm comm) {
  TraceRange trace("MPI_Alltoallv");
  if (!resolve_symbols())
    return MPI_ERR_OTHER;
  auto library = [&] {
    counters().alltoallv_lib++;
    return libmpi.Alltoallv(sendbuf, sendcounts, sdispls, sendtype, recvbuf,
                            recvcounts, rdispls, recvtype, comm);
  };
  if (env().disable || env().alltoallv == Alltoallv::NONE)
    return library();
  // memory the GPU cannot reach goes to the library (a null buffer, which
  // only empty blocks may use, counts as reachable, as in the reference)
  if ((sendbuf && !classify(sendbuf).device_accessible) ||
      (recvbuf && !classify(recvbuf).device_accessible))
    return library();
  if (comm != MPI_COMM_WORLD)
    return library();
  Args a{sendbuf, sendcounts, sdispls, sendtype, recvbuf, recvcounts, rdispls, recvtype, comm};
  if (libmpi.Comm_size(comm, &a.size) != MPI_SUCCESS ||
      libmpi.Comm_rank(comm, &a.rank) != MPI_SUCCESS || a.size <= 0)
    return library();
  if (!dense_type(sendtype, &a.sext) || !dense_type(recvtype, &a.rext))
    return library();
  try_progress();
  switch (env().alltoallv) {
  case Alltoallv::REMOTE_FIRST: return remote_first(a);
  case Alltoallv::ISIR_STAGED: return isir_staged(a, false);
  case Alltoallv::ISIR_REMOTE_STAGED: return isir_staged(a, true);
  default: return staged(a); // AUTO and STAGED, as the reference's AUTO
  }
}
