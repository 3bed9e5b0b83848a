// The interposed MPI entry points.  Each follows the reference's decision
// order (src/pack.cpp, src/unpack.cpp, src/type_commit.cpp,
// src/type_free.cpp, src/internal/send.cpp, src/recv.cpp,
// src/internal/isend.cpp, src/internal/irecv.cpp, src/wait.cpp) with these
// changes:
//  * errors come back as MPI error codes; nothing calls exit();
//  * MPI_Pack/MPI_Unpack check outsize/insize (MPI_ERR_TRUNCATE, nothing
//    written), which the reference does not;
//  * a committed type that TEMPI cannot describe goes to the library instead
//    of dereferencing a null packer;
//  * once TEMPI has taken a call onto the GPU path it never falls back to a
//    CPU copy: a CUDA failure is returned as MPI_ERR_OTHER;
//  * a contiguous run of at least 8 MiB between two pinned host buffers goes
//    through the copy engines (hostlink.cpp), strided ones through the
//    kernels.

#include "dispatch.hpp"
#include "runtime.hpp"
#include "sender.hpp"

#include <vector>

namespace tempi {
namespace {

bool ready() { return resolve_symbols(); }

int to_mpi(int e) {
  switch (e) {
  case TEMPI_OK: return MPI_SUCCESS;
  case TEMPI_ERR_TRUNCATE: return MPI_ERR_TRUNCATE;
  case TEMPI_ERR_ARG: return MPI_ERR_ARG;
  case TEMPI_ERR_NO_MEM: return MPI_ERR_NO_MEM;
  default: return MPI_ERR_OTHER;
  }
}

// Both buffers pinned host memory and enough bytes: the copy engines move
// the objects across the host link (hostlink.cpp) when they are one
// contiguous run (RUN) or, for an unpack, rows of one strided dimension
// (ROWS, shape in *rows); anything else stays on the kernels (NONE).  The
// rows path is for unpacks only: measured host to host, it unpacks 256-B
// rows at 22 GB/s against 20 by the kernels and 1-KiB rows at 30 against
// 28, but packs them at 30 against 32-33.
enum class HostLink { NONE, RUN, ROWS };
HostLink use_host_link(const PtrInfo &a, const PtrInfo &b, const tempi_desc &d,
                       int64_t count, bool unpack, HostRows *rows) {
  if (!env().host_link_dma || !a.is_host || !b.is_host)
    return HostLink::NONE;
  if (int64_t(count) * d.size < kHostLinkMinBytes)
    return HostLink::NONE;
  if (contiguous_run(d, count) == int64_t(count) * d.size)
    return HostLink::RUN;
  return unpack && host_rows(d, count, rows) ? HostLink::ROWS : HostLink::NONE;
}

// A contiguous device buffer goes through host staging under
// TEMPI_CONTIGUOUS_STAGED always, under TEMPI_CONTIGUOUS_AUTO when the
// measured tables say staging is faster (reference types_init and
// type_commit.cpp:37-58 choose SendRecv1DStaged / SendRecv1D the same way);
// otherwise the library sends it as it is.
bool contiguous_staged(const TypeRecord *r, const PtrInfo &p, int count) {
  if (!r || !r->packable || r->desc.ndims != 0 || count <= 0 || !p.is_device)
    return false;
  if (env().contiguous == Contiguous::STAGED)
    return true;
  return env().contiguous == Contiguous::AUTO &&
         contiguous_staged_faster(int64_t(count) * r->desc.size);
}

void on_init() {
  read_env();
  dispatch_init();
  // the staged kernels' failure word, allocated here rather than at a first
  // launch that might come while another thread captures a stream
  if (!env().disable)
    staged_channel(nullptr);
  // the named types a contiguous send uses are known from the start, as in
  // the reference's types_init (src/internal/types.cpp:723-755, called from
  // src/init.cpp:63 unless TEMPI is disabled)
  if (!env().disable)
    for (MPI_Datatype t : {MPI_BYTE, MPI_FLOAT, MPI_DOUBLE})
      commit_type(t);
}

void on_finalize() {
  async_finalize();
  slab_release_all();
  events_release_all();
}

} // namespace
} // namespace tempi

using namespace tempi;

extern "C" {

int MPI_Init(int *argc, char ***argv) {
  if (!ready())
    return MPI_ERR_OTHER;
  int err = libmpi.Init(argc, argv);
  if (err == MPI_SUCCESS)
    on_init();
  return err;
}

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
  if (!ready())
    return MPI_ERR_OTHER;
  int err = libmpi.Init_thread(argc, argv, required, provided);
  if (err == MPI_SUCCESS)
    on_init();
  return err;
}

int MPI_Finalize(void) {
  if (!ready())
    return MPI_ERR_OTHER;
  if (!env().disable)
    on_finalize();
  return libmpi.Finalize();
}

int MPI_Type_commit(MPI_Datatype *datatype) {
  TraceRange trace("MPI_Type_commit");
  if (!ready())
    return MPI_ERR_OTHER;
  int err = libmpi.Type_commit(datatype);
  if (err != MPI_SUCCESS || env().disable || env().no_type_commit)
    return err;
  on_commit(*commit_type(*datatype));
  return err;
}

int MPI_Type_free(MPI_Datatype *datatype) {
  if (!ready())
    return MPI_ERR_OTHER;
  if (!env().disable && !env().no_type_commit && datatype)
    release_type(*datatype); // before the library may reuse the handle
  return libmpi.Type_free(datatype);
}

int MPI_Pack(const void *inbuf, int incount, MPI_Datatype datatype,
             void *outbuf, int outsize, int *position, MPI_Comm comm) {
  TraceRange trace("MPI_Pack");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable || env().no_pack)
    return libmpi.Pack(inbuf, incount, datatype, outbuf, outsize, position,
                       comm);
  TypeRecord *r = find_type(datatype);
  if (!r || !r->packable) {
    counters().lib_pack++;
    return libmpi.Pack(inbuf, incount, datatype, outbuf, outsize, position,
                       comm);
  }
  PtrInfo in = classify(inbuf), out = classify(outbuf);
  if (!in.device_accessible || !out.device_accessible) {
    counters().lib_pack++;
    return libmpi.Pack(inbuf, incount, datatype, outbuf, outsize, position,
                       comm);
  }
  if (!position || incount < 0)
    return MPI_ERR_ARG;
  const int64_t bytes = int64_t(incount) * r->desc.size;
  if (*position < 0 || *position + bytes > int64_t(outsize))
    return MPI_ERR_TRUNCATE;
  cudaStream_t s = pack_stream();
  int e;
  HostRows hr{};
  if (use_host_link(in, out, r->desc, incount, false, &hr) == HostLink::RUN) {
    e = host_link_copy(static_cast<char *>(outbuf) + *position,
                       static_cast<const char *>(inbuf) + r->desc.start,
                       size_t(bytes), s);
  } else {
    tempi_config cfg =
        choose_config(*r, incount, in.is_host, out.is_host, false);
    e = pack_known(&r->desc, in.device_ptr, incount,
                   static_cast<char *>(out.device_ptr) + *position, &cfg, s,
                   in.is_device && out.is_device ? 1 : 0);
  }
  if (!e) {
    cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess)
      e = cuda_error(ce, "MPI_Pack synchronize");
    else
      e = tempi_staged_check();
  }
  if (e)
    return to_mpi(e);
  *position += int(bytes);
  return MPI_SUCCESS;
}

int MPI_Unpack(const void *inbuf, int insize, int *position, void *outbuf,
               int outcount, MPI_Datatype datatype, MPI_Comm comm) {
  TraceRange trace("MPI_Unpack");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable || env().no_pack)
    return libmpi.Unpack(inbuf, insize, position, outbuf, outcount, datatype,
                         comm);
  TypeRecord *r = find_type(datatype);
  if (!r || !r->packable) {
    counters().lib_unpack++;
    return libmpi.Unpack(inbuf, insize, position, outbuf, outcount, datatype,
                         comm);
  }
  PtrInfo in = classify(inbuf), out = classify(outbuf);
  if (!in.device_accessible || !out.device_accessible) {
    counters().lib_unpack++;
    return libmpi.Unpack(inbuf, insize, position, outbuf, outcount, datatype,
                         comm);
  }
  if (!position || outcount < 0)
    return MPI_ERR_ARG;
  const int64_t bytes = int64_t(outcount) * r->desc.size;
  if (*position < 0 || *position + bytes > int64_t(insize))
    return MPI_ERR_TRUNCATE;
  cudaStream_t s = pack_stream();
  int e;
  HostRows hr{};
  const HostLink link = use_host_link(in, out, r->desc, outcount, true, &hr);
  if (link == HostLink::RUN) {
    e = host_link_copy(static_cast<char *>(outbuf) + r->desc.start,
                       static_cast<const char *>(inbuf) + *position,
                       size_t(bytes), s);
  } else if (link == HostLink::ROWS) {
    e = host_link_rows(static_cast<char *>(outbuf) + r->desc.start, hr.pitch,
                       static_cast<const char *>(inbuf) + *position, hr.width,
                       hr.width, hr.rows, s);
  } else {
    tempi_config cfg =
        choose_config(*r, outcount, out.is_host, in.is_host, true);
    e = unpack_known(&r->desc,
                     static_cast<const char *>(in.device_ptr) + *position,
                     outcount, out.device_ptr, &cfg, s,
                     in.is_device && out.is_device ? 1 : 0);
  }
  if (!e) {
    cudaError_t ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess)
      e = cuda_error(ce, "MPI_Unpack synchronize");
    else
      e = tempi_staged_check();
  }
  if (e)
    return to_mpi(e);
  *position += int(bytes);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest,
             int tag, MPI_Comm comm) {
  TraceRange trace("MPI_Send");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable)
    return libmpi.Send(buf, count, datatype, dest, tag, comm);
  // earlier non-blocking sends reach the library first (non-overtaking)
  if (int e = progress_sends())
    return e;
  PtrInfo p = classify(buf);
  TypeRecord *r = p.device_accessible ? find_type(datatype) : nullptr;
  if (r && r->packable && r->desc.ndims >= 1 && count > 0) {
    Method m = choose_method(*r, count);
    return send_strided(*r, m, p.device_ptr, count, dest, tag, comm);
  }
  if (contiguous_staged(r, p, count)) {
    return send_contiguous_staged(buf, count, datatype,
                                  int64_t(count) * r->desc.size, dest, tag,
                                  comm);
  }
  counters().send_lib++;
  return libmpi.Send(buf, count, datatype, dest, tag, comm);
}

int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status) {
  TraceRange trace("MPI_Recv");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable)
    return libmpi.Recv(buf, count, datatype, source, tag, comm, status);
  PtrInfo p = classify(buf);
  TypeRecord *r = p.device_accessible ? find_type(datatype) : nullptr;
  if (r && r->packable && r->desc.ndims >= 1 && count > 0) {
    Method m = choose_method(*r, count);
    return recv_strided(*r, m, p.device_ptr, count, source, tag, comm, status);
  }
  if (contiguous_staged(r, p, count)) {
    return recv_contiguous_staged(buf, count, datatype,
                                  int64_t(count) * r->desc.size, source, tag,
                                  comm, status);
  }
  counters().recv_lib++;
  return libmpi.Recv(buf, count, datatype, source, tag, comm, status);
}

int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest,
              int tag, MPI_Comm comm, MPI_Request *request) {
  TraceRange trace("MPI_Isend");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable)
    return libmpi.Isend(buf, count, datatype, dest, tag, comm, request);
  PtrInfo p = classify(buf);
  TypeRecord *r = p.device_accessible ? find_type(datatype) : nullptr;
  int err;
  if (r && r->packable && r->desc.ndims >= 1 && count > 0) {
    Method m = choose_method(*r, count);
    err = start_isend(*r, m, p.device_ptr, count, dest, tag, comm, request);
  } else {
    // earlier managed sends reach the library first (non-overtaking)
    err = progress_sends();
    if (!err)
      err = libmpi.Isend(buf, count, datatype, dest, tag, comm, request);
  }
  try_progress();
  return err;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
              MPI_Comm comm, MPI_Request *request) {
  TraceRange trace("MPI_Irecv");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable)
    return libmpi.Irecv(buf, count, datatype, source, tag, comm, request);
  PtrInfo p = classify(buf);
  TypeRecord *r = p.device_accessible ? find_type(datatype) : nullptr;
  int err;
  if (r && r->packable && r->desc.ndims >= 1 && count > 0) {
    Method m = choose_method(*r, count);
    err = start_irecv(*r, m, p.device_ptr, count, source, tag, comm, request);
  } else {
    err = libmpi.Irecv(buf, count, datatype, source, tag, comm, request);
  }
  try_progress();
  return err;
}

// Neighbourhood all-to-all with a datatype per edge (reference
// src/neighbor_alltoallw.cpp:11-17 -> neighbor_alltoallw::isir,
// src/internal/neighbor_alltoallw.cpp:19-85: an MPI_Isend per out-edge and
// an MPI_Irecv per in-edge, then waits).  When every edge is an edge to this
// rank and every region is a committed strided type in device-accessible
// memory, the k-th out-edge's region is copied straight into the k-th
// in-edge's region by one fused kernel (copy_batch_run): pack, transfer and
// unpack in one launch, no packed buffer.  Otherwise the reference's
// Isend/Irecv sequence runs through TEMPI's own senders, and calls with no
// region TEMPI can describe go to the library.
int MPI_Neighbor_alltoallw(const void *sendbuf, const int sendcounts[],
                           const MPI_Aint sdispls[],
                           const MPI_Datatype sendtypes[], void *recvbuf,
                           const int recvcounts[], const MPI_Aint rdispls[],
                           const MPI_Datatype recvtypes[], MPI_Comm comm) {
  TraceRange trace("MPI_Neighbor_alltoallw");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable)
    return libmpi.Neighbor_alltoallw(sendbuf, sendcounts, sdispls, sendtypes,
                                     recvbuf, recvcounts, rdispls, recvtypes,
                                     comm);
  int indeg = 0, outdeg = 0, weighted = 0, me = 0;
  int err = libmpi.Dist_graph_neighbors_count(comm, &indeg, &outdeg, &weighted);
  if (err)
    return err;
  std::vector<int> sources(size_t(indeg) + 1), sw(size_t(indeg) + 1);
  std::vector<int> dests(size_t(outdeg) + 1), dw(size_t(outdeg) + 1);
  err = libmpi.Dist_graph_neighbors(comm, indeg, sources.data(), sw.data(),
                                    outdeg, dests.data(), dw.data());
  if (!err)
    err = libmpi.Comm_rank(comm, &me);
  if (err)
    return err;
  const PtrInfo ps = classify(sendbuf), pr = classify(recvbuf);
  bool any_described = false, fusable = indeg == outdeg && ps.device_accessible &&
                                        pr.device_accessible;
  std::vector<tempi_copy_region> regs;
  for (int k = 0; k < outdeg; ++k) {
    const TypeRecord *ts = find_type(sendtypes[k]);
    const TypeRecord *tr = k < indeg ? find_type(recvtypes[k]) : nullptr;
    const bool ds = ts && ts->packable, dr = tr && tr->packable;
    any_described = any_described || ds || dr;
    if (!fusable)
      continue;
    if (dests[k] != me || sources[k] != me || !ds || !dr ||
        sendcounts[k] < 0 || recvcounts[k] < 0 ||
        int64_t(sendcounts[k]) * ts->desc.size !=
            int64_t(recvcounts[k]) * tr->desc.size) {
      fusable = false;
      continue;
    }
    tempi_copy_region c{};
    c.src_origin = static_cast<const char *>(ps.device_ptr) + sdispls[k];
    c.dst_origin = static_cast<char *>(pr.device_ptr) + rdispls[k];
    c.src_desc = ts->desc;
    c.dst_desc = tr->desc;
    c.src_count = sendcounts[k];
    c.dst_count = recvcounts[k];
    regs.push_back(c);
  }
  if (fusable) {
    cudaStream_t s = pack_stream();
    int e = copy_batch_run(regs.data(), int32_t(regs.size()), s);
    if (!e) {
      cudaError_t ce = cudaStreamSynchronize(s);
      if (ce != cudaSuccess)
        e = cuda_error(ce, "MPI_Neighbor_alltoallw synchronize");
    }
    counters().neighbor_fused++;
    return to_mpi(e);
  }
  if (!any_described) {
    counters().neighbor_lib++;
    return libmpi.Neighbor_alltoallw(sendbuf, sendcounts, sdispls, sendtypes,
                                     recvbuf, recvcounts, rdispls, recvtypes,
                                     comm);
  }
  counters().neighbor_isir++;
  const int tag = 0x7ee1; // reserved for this collective
  std::vector<MPI_Request> sreqs, rreqs;
  for (int i = 0; i < outdeg && !err; ++i) {
    MPI_Request q = MPI_REQUEST_NULL;
    err = MPI_Isend(static_cast<const char *>(sendbuf) + sdispls[i],
                    sendcounts[i], sendtypes[i], dests[i], tag, comm, &q);
    sreqs.push_back(q);
  }
  for (int j = 0; j < indeg && !err; ++j) {
    MPI_Request q = MPI_REQUEST_NULL;
    err = MPI_Irecv(static_cast<char *>(recvbuf) + rdispls[j], recvcounts[j],
                    recvtypes[j], sources[j], tag, comm, &q);
    rreqs.push_back(q);
  }
  for (MPI_Request &q : sreqs) {
    const int e = q == MPI_REQUEST_NULL ? MPI_SUCCESS : MPI_Wait(&q, MPI_STATUS_IGNORE);
    err = err ? err : e;
  }
  for (MPI_Request &q : rreqs) {
    const int e = q == MPI_REQUEST_NULL ? MPI_SUCCESS : MPI_Wait(&q, MPI_STATUS_IGNORE);
    err = err ? err : e;
  }
  return err;
}

int MPI_Wait(MPI_Request *request, MPI_Status *status) {
  TraceRange trace("MPI_Wait");
  if (!ready())
    return MPI_ERR_OTHER;
  if (env().disable || !request || !is_managed(*request)) {
    // an unmanaged receive may match a managed send whose pack is in flight
    int e = progress_sends();
    if (e)
      return e;
    return libmpi.Wait(request, status);
  }
  return wait_managed(request, status);
}

} // extern "C"
