// Blocking and non-blocking transfers of strided objects that live in device
// memory, by one of three methods (reference include/sender.hpp,
// src/internal/sender.cpp:88-328, src/internal/async_operation.cpp):
//
//   DEVICE   pack into a device slab, hand the slab to MPI as MPI_PACKED
//   ONE_SHOT pack straight into mapped pinned host memory (the kernel's
//            stores cross the host link), hand that to MPI
//   STAGED   pack into a device slab, copy it to a pinned host slab, hand
//            that to MPI (the reference sends the staged bytes with the
//            original datatype, sender.cpp:218; this sends MPI_PACKED)
//
// Receives mirror each method.  Non-blocking operations are two-state
// machines driven by MPI_Wait and by progress calls from every TEMPI entry
// point; unlike the reference, waiting progresses every active operation
// (needed for self-sends, where the receive can only complete once the
// matching send has been started) and gives up after TEMPI_WAIT_TIMEOUT_S.

#include "sender.hpp"

#include "dispatch.hpp"

#include <algorithm>
#include <chrono>
#include <map>
#include <memory>

namespace tempi {

namespace {

int to_mpi(int tempi_err) {
  switch (tempi_err) {
  case TEMPI_OK: return MPI_SUCCESS;
  case TEMPI_ERR_NO_MEM: return MPI_ERR_NO_MEM;
  case TEMPI_ERR_TRUNCATE: return MPI_ERR_TRUNCATE;
  case TEMPI_ERR_ARG: return MPI_ERR_ARG;
  default: return MPI_ERR_OTHER;
  }
}

int sync(cudaStream_t s) {
  cudaError_t e = cudaStreamSynchronize(s);
  return e == cudaSuccess ? tempi_staged_check()
                          : cuda_error(e, "stream synchronize");
}

void *host_dev_ptr(void *h) {
  void *d = nullptr;
  if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
    cudaGetLastError();
    return h;
  }
  return d;
}

} // namespace

int send_strided(TypeRecord &r, Method m, const void *buf, int count, int dest,
                 int tag, MPI_Comm comm) {
  const int64_t bytes = int64_t(count) * r.desc.size;
  cudaStream_t s = pack_stream();
  tempi_config cfg = choose_config(r, count, false, m == Method::ONESHOT,
                                   false);
  int err = TEMPI_OK;
  switch (m) {
  case Method::ONESHOT: {
    counters().send_oneshot++;
    void *h = slab_alloc(Space::HOST_MAPPED, bytes);
    if (!h)
      return MPI_ERR_NO_MEM;
    err = tempi_pack(&r.desc, buf, count, host_dev_ptr(h), &cfg, s);
    if (!err)
      err = sync(s);
    int merr = err ? to_mpi(err)
                   : libmpi.Send(h, int(bytes), MPI_PACKED, dest, tag, comm);
    slab_free(Space::HOST_MAPPED, h);
    return merr;
  }
  case Method::STAGED: {
    counters().send_staged++;
    void *d = slab_alloc(Space::DEVICE, bytes);
    void *h = slab_alloc(Space::HOST_MAPPED, bytes);
    if (!d || !h) {
      slab_free(Space::DEVICE, d);
      slab_free(Space::HOST_MAPPED, h);
      return MPI_ERR_NO_MEM;
    }
    err = tempi_pack(&r.desc, buf, count, d, &cfg, s);
    if (!err) {
      cudaError_t e = cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s);
      err = e == cudaSuccess ? sync(s) : cuda_error(e, "staged copy");
    }
    int merr = err ? to_mpi(err)
                   : libmpi.Send(h, int(bytes), MPI_PACKED, dest, tag, comm);
    slab_free(Space::DEVICE, d);
    slab_free(Space::HOST_MAPPED, h);
    return merr;
  }
  default: {
    counters().send_device++;
    void *d = slab_alloc(Space::DEVICE, bytes);
    if (!d)
      return MPI_ERR_NO_MEM;
    err = tempi_pack(&r.desc, buf, count, d, &cfg, s);
    if (!err)
      err = sync(s);
    int merr = err ? to_mpi(err)
                   : libmpi.Send(d, int(bytes), MPI_PACKED, dest, tag, comm);
    slab_free(Space::DEVICE, d);
    return merr;
  }
  }
}

int recv_strided(TypeRecord &r, Method m, void *buf, int count, int source,
                 int tag, MPI_Comm comm, MPI_Status *status) {
  const int64_t bytes = int64_t(count) * r.desc.size;
  cudaStream_t s = pack_stream();
  tempi_config cfg = choose_config(r, count, false, m == Method::ONESHOT,
                                   true);
  int err = TEMPI_OK;
  switch (m) {
  case Method::ONESHOT: {
    counters().recv_oneshot++;
    void *h = slab_alloc(Space::HOST_MAPPED, bytes);
    if (!h)
      return MPI_ERR_NO_MEM;
    int merr =
        libmpi.Recv(h, int(bytes), MPI_PACKED, source, tag, comm, status);
    if (merr == MPI_SUCCESS) {
      err = tempi_unpack(&r.desc, host_dev_ptr(h), count, buf, &cfg, s);
      if (!err)
        err = sync(s);
      merr = to_mpi(err);
    }
    slab_free(Space::HOST_MAPPED, h);
    return merr;
  }
  case Method::STAGED: {
    counters().recv_staged++;
    void *d = slab_alloc(Space::DEVICE, bytes);
    void *h = slab_alloc(Space::HOST_MAPPED, bytes);
    if (!d || !h) {
      slab_free(Space::DEVICE, d);
      slab_free(Space::HOST_MAPPED, h);
      return MPI_ERR_NO_MEM;
    }
    int merr =
        libmpi.Recv(h, int(bytes), MPI_PACKED, source, tag, comm, status);
    if (merr == MPI_SUCCESS) {
      cudaError_t e = cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
      err = e == cudaSuccess ? tempi_unpack(&r.desc, d, count, buf, &cfg, s)
                             : cuda_error(e, "staged copy");
      if (!err)
        err = sync(s);
      merr = to_mpi(err);
    }
    slab_free(Space::DEVICE, d);
    slab_free(Space::HOST_MAPPED, h);
    return merr;
  }
  default: {
    counters().recv_device++;
    void *d = slab_alloc(Space::DEVICE, bytes);
    if (!d)
      return MPI_ERR_NO_MEM;
    int merr =
        libmpi.Recv(d, int(bytes), MPI_PACKED, source, tag, comm, status);
    if (merr == MPI_SUCCESS) {
      err = tempi_unpack(&r.desc, d, count, buf, &cfg, s);
      if (!err)
        err = sync(s);
      merr = to_mpi(err);
    }
    slab_free(Space::DEVICE, d);
    return merr;
  }
  }
}

// ---- contiguous staged transfers (reference SendRecv1DStaged,
//      sender.cpp:34-61) -------------------------------------------------------

int send_contiguous_staged(const void *buf, int count, MPI_Datatype dt,
                           int64_t bytes, int dest, int tag, MPI_Comm comm) {
  void *h = slab_alloc(Space::HOST_MAPPED, bytes);
  if (!h)
    return MPI_ERR_NO_MEM;
  cudaError_t e = cudaMemcpy(h, buf, bytes, cudaMemcpyDefault);
  int merr = e == cudaSuccess ? libmpi.Send(h, count, dt, dest, tag, comm)
                              : to_mpi(cuda_error(e, "staged copy"));
  slab_free(Space::HOST_MAPPED, h);
  counters().send_contig_staged++;
  return merr;
}

int recv_contiguous_staged(void *buf, int count, MPI_Datatype dt,
                           int64_t bytes, int source, int tag, MPI_Comm comm,
                           MPI_Status *status) {
  void *h = slab_alloc(Space::HOST_MAPPED, bytes);
  if (!h)
    return MPI_ERR_NO_MEM;
  int merr = libmpi.Recv(h, count, dt, source, tag, comm, status);
  if (merr == MPI_SUCCESS) {
    cudaError_t e = cudaMemcpy(buf, h, bytes, cudaMemcpyDefault);
    if (e != cudaSuccess)
      merr = to_mpi(cuda_error(e, "staged copy"));
  }
  slab_free(Space::HOST_MAPPED, h);
  counters().recv_contig_staged++;
  return merr;
}

// ---- non-blocking ----------------------------------------------------------

namespace {

class AsyncOp {
public:
  uint64_t seq = 0; // creation order among managed operations
  virtual ~AsyncOp() {}
  virtual int wake() = 0;       // advance if possible
  virtual bool waiting() = 0;   // still needs wake() to reach its last state
  virtual int finish(MPI_Status *status) = 0; // after !waiting()
  virtual bool is_send() const = 0;
};

class IsendOp : public AsyncOp {
  Method m_;
  void *dev_ = nullptr, *host_ = nullptr;
  MPI_Request req_ = MPI_REQUEST_NULL;
  cudaEvent_t ev_ = nullptr;
  bool started_ = false;

public:
  int err = MPI_SUCCESS;
  IsendOp(TypeRecord &r, Method m, const void *buf, int count, int dest,
          int tag, MPI_Comm comm)
      : m_(m) {
    const int64_t bytes = int64_t(count) * r.desc.size;
    cudaStream_t s = pack_stream();
    tempi_config cfg = choose_config(r, count, false, m == Method::ONESHOT,
                                   false);
    ev_ = event_acquire();
    void *packed = nullptr;
    int terr = TEMPI_OK;
    (m == Method::ONESHOT  ? counters().send_oneshot
     : m == Method::STAGED ? counters().send_staged
                           : counters().send_device)++;
    if (m == Method::ONESHOT) {
      host_ = slab_alloc(Space::HOST_MAPPED, bytes);
      packed = host_;
      if (host_)
        terr = tempi_pack(&r.desc, buf, count, host_dev_ptr(host_), &cfg, s);
    } else {
      dev_ = slab_alloc(Space::DEVICE, bytes);
      packed = dev_;
      if (dev_)
        terr = tempi_pack(&r.desc, buf, count, dev_, &cfg, s);
      if (m == Method::STAGED && dev_ && !terr) {
        host_ = slab_alloc(Space::HOST_MAPPED, bytes);
        packed = host_;
        cudaError_t e = host_ ? cudaMemcpyAsync(host_, dev_, bytes,
                                                cudaMemcpyDeviceToHost, s)
                              : cudaSuccess;
        if (e != cudaSuccess)
          terr = cuda_error(e, "staged copy");
      }
    }
    if (!packed || !ev_) {
      err = MPI_ERR_NO_MEM;
      return;
    }
    if (terr) {
      err = to_mpi(terr);
      return;
    }
    cudaEventRecord(ev_, s);
    err = libmpi.Send_init(packed, int(bytes), MPI_PACKED, dest, tag, comm,
                           &req_);
  }
  ~IsendOp() override {
    if (req_ != MPI_REQUEST_NULL)
      libmpi.Request_free(&req_);
    slab_free(Space::DEVICE, dev_);
    slab_free(Space::HOST_MAPPED, host_);
    event_release(ev_);
  }
  int wake() override {
    if (started_ || err)
      return err;
    cudaError_t e = cudaEventQuery(ev_);
    if (e == cudaErrorNotReady)
      return MPI_SUCCESS;
    if (e != cudaSuccess) {
      err = to_mpi(cuda_error(e, "isend pack"));
      return err;
    }
    if (int c = tempi_staged_check()) {
      err = to_mpi(c);
      return err;
    }
    started_ = true;
    err = libmpi.Start(&req_);
    return err;
  }
  bool waiting() override { return !started_ && !err; }
  bool is_send() const override { return true; }
  int finish(MPI_Status *status) override {
    if (err)
      return err;
    return libmpi.Wait(&req_, status);
  }
};

class IrecvOp : public AsyncOp {
  TypeRecord &r_;
  Method m_;
  void *buf_;
  int count_;
  void *dev_ = nullptr, *host_ = nullptr;
  MPI_Request req_ = MPI_REQUEST_NULL;
  cudaEvent_t ev_ = nullptr;
  bool unpacking_ = false;
  MPI_Status st_{};

public:
  int err = MPI_SUCCESS;
  IrecvOp(TypeRecord &r, Method m, void *buf, int count, int source, int tag,
          MPI_Comm comm)
      : r_(r), m_(m), buf_(buf), count_(count) {
    const int64_t bytes = int64_t(count) * r.desc.size;
    ev_ = event_acquire();
    void *packed = nullptr;
    if (m == Method::ONESHOT || m == Method::STAGED) {
      host_ = slab_alloc(Space::HOST_MAPPED, bytes);
      packed = host_;
    }
    if (m != Method::ONESHOT) {
      dev_ = slab_alloc(Space::DEVICE, bytes);
      if (m == Method::DEVICE)
        packed = dev_;
    }
    if (!packed || !ev_ || (m == Method::STAGED && !dev_)) {
      err = MPI_ERR_NO_MEM;
      return;
    }
    err = libmpi.Irecv(packed, int(bytes), MPI_PACKED, source, tag, comm,
                       &req_);
  }
  ~IrecvOp() override {
    if (req_ != MPI_REQUEST_NULL) // never matched: withdraw it from the library
      libmpi.Request_free(&req_);
    slab_free(Space::DEVICE, dev_);
    slab_free(Space::HOST_MAPPED, host_);
    event_release(ev_);
  }
  int wake() override {
    if (unpacking_ || err)
      return err;
    int flag = 0;
    err = libmpi.Test(&req_, &flag, &st_);
    if (err || !flag)
      return err;
    const int64_t bytes = int64_t(count_) * r_.desc.size;
    cudaStream_t s = pack_stream();
    tempi_config cfg = choose_config(r_, count_, false, m_ == Method::ONESHOT,
                                   true);
    int terr = TEMPI_OK;
    if (m_ == Method::ONESHOT) {
      terr = tempi_unpack(&r_.desc, host_dev_ptr(host_), count_, buf_, &cfg, s);
    } else {
      if (m_ == Method::STAGED) {
        cudaError_t e =
            cudaMemcpyAsync(dev_, host_, bytes, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess)
          terr = cuda_error(e, "staged copy");
      }
      if (!terr)
        terr = tempi_unpack(&r_.desc, dev_, count_, buf_, &cfg, s);
    }
    if (!terr && cudaEventRecord(ev_, s) != cudaSuccess)
      terr = cuda_error(cudaGetLastError(), "event record");
    unpacking_ = true;
    err = to_mpi(terr);
    return err;
  }
  bool waiting() override { return !unpacking_ && !err; }
  bool is_send() const override { return false; }
  int finish(MPI_Status *status) override {
    if (err)
      return err;
    cudaError_t e = cudaEventSynchronize(ev_);
    if (e != cudaSuccess)
      return to_mpi(cuda_error(e, "irecv unpack"));
    if (int c = tempi_staged_check())
      return to_mpi(c);
    if (status)
      *status = st_;
    return MPI_SUCCESS;
  }
};

std::mutex g_async_mu;
std::map<MPI_Request, std::unique_ptr<AsyncOp>> g_active;
uint32_t g_next = 0;
uint64_t g_seq = 0;

// Start the library sends of managed operations in creation order, each once
// its pack has finished, stopping at the first whose pack has not: a send
// never reaches the library ahead of an earlier one, which MPI's
// non-overtaking rule needs (messages to one destination with one tag
// arrive in the order sent).  Packs all run on one stream and so finish in
// order, but a scan could otherwise see a later event complete that an
// earlier query found pending.  Caller holds g_async_mu.  *pending: a send
// is still waiting for its pack.
int start_sends_in_order(bool *pending) {
  std::vector<AsyncOp *> sends;
  for (auto &kv : g_active)
    if (kv.second->is_send() && kv.second->waiting())
      sends.push_back(kv.second.get());
  std::sort(sends.begin(), sends.end(),
            [](const AsyncOp *a, const AsyncOp *b) { return a->seq < b->seq; });
  *pending = false;
  for (AsyncOp *op : sends) {
    const int e = op->wake();
    if (e)
      return e;
    if (op->waiting()) {
      *pending = true;
      break;
    }
  }
  return MPI_SUCCESS;
}

MPI_Request make_request() {
  // minimpi keeps its own handles below 2^30; these sit above it
  return MPI_Request(0x40000000u | (g_next++ & 0x3fffffffu));
}

} // namespace

int start_isend(TypeRecord &r, Method m, const void *buf, int count, int dest,
                int tag, MPI_Comm comm, MPI_Request *request) {
  auto op = std::make_unique<IsendOp>(r, m, buf, count, dest, tag, comm);
  if (op->err)
    return op->err;
  std::lock_guard<std::mutex> l(g_async_mu);
  *request = make_request();
  op->seq = g_seq++;
  g_active[*request] = std::move(op);
  counters().isend_managed++;
  return MPI_SUCCESS;
}

int start_irecv(TypeRecord &r, Method m, void *buf, int count, int source,
                int tag, MPI_Comm comm, MPI_Request *request) {
  auto op = std::make_unique<IrecvOp>(r, m, buf, count, source, tag, comm);
  if (op->err)
    return op->err;
  std::lock_guard<std::mutex> l(g_async_mu);
  *request = make_request();
  op->seq = g_seq++;
  g_active[*request] = std::move(op);
  counters().irecv_managed++;
  return MPI_SUCCESS;
}

int try_progress() {
  std::lock_guard<std::mutex> l(g_async_mu);
  bool pending = false;
  int first = start_sends_in_order(&pending);
  for (auto &kv : g_active) {
    if (!kv.second->is_send() && kv.second->waiting()) {
      int e = kv.second->wake();
      if (e && !first)
        first = e;
    }
  }
  return first;
}

int progress_sends() {
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    bool pending = false;
    {
      std::lock_guard<std::mutex> l(g_async_mu);
      int e = start_sends_in_order(&pending);
      if (e)
        return e;
    }
    if (!pending)
      return MPI_SUCCESS;
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() -
                                              t0)
                    .count();
    if (dt > env().wait_timeout_s)
      return set_error(TEMPI_ERR_TIMEOUT, "send progress gave up"),
             MPI_ERR_OTHER;
  }
}

bool is_managed(MPI_Request r) {
  std::lock_guard<std::mutex> l(g_async_mu);
  return g_active.count(r) != 0;
}

int wait_managed(MPI_Request *request, MPI_Status *status) {
  AsyncOp *op = nullptr;
  {
    std::lock_guard<std::mutex> l(g_async_mu);
    auto it = g_active.find(*request);
    if (it == g_active.end())
      return MPI_ERR_REQUEST;
    op = it->second.get();
  }
  const auto t0 = std::chrono::steady_clock::now();
  const double limit = env().wait_timeout_s;
  int err = MPI_SUCCESS;
  while (op->waiting()) {
    if (op->is_send()) { // in order: the earlier sends go first
      bool pending = false;
      std::lock_guard<std::mutex> l(g_async_mu);
      err = start_sends_in_order(&pending);
    } else {
      err = op->wake();
    }
    if (err)
      break;
    if (!op->waiting())
      break;
    try_progress(); // the matching send may be another active operation
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() -
                                              t0)
                    .count();
    if (dt > limit) {
      set_error(TEMPI_ERR_TIMEOUT, "MPI_Wait gave up after %.1f s", dt);
      err = MPI_ERR_OTHER;
      break;
    }
  }
  if (!err)
    err = op->finish(status);
  std::lock_guard<std::mutex> l(g_async_mu);
  g_active.erase(*request);
  *request = MPI_REQUEST_NULL;
  return err;
}

void async_finalize() {
  std::lock_guard<std::mutex> l(g_async_mu);
  if (!g_active.empty())
    LOG_WARN("%zu managed async operations were never waited on",
             g_active.size());
  g_active.clear();
}

} // namespace tempi
