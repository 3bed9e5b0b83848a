// libminimpi: a small MPI library that stands in for the system MPI, which
// does not exist on the machines this project runs on.  One process is world
// size 1; several processes on one host form a larger world when each is
// started with MINIMPI_SIZE, MINIMPI_RANK and a shared MINIMPI_DIR: the ranks
// then connect by Unix-domain stream sockets in that directory, one per pair.
//
// Datatypes follow the MPI-3.1 type-map definitions (section 4.1): each
// constructor describes a sequence of (displacement, basic type) entries in a
// fixed order, and MPI_Pack copies the described bytes in exactly that order.
// The walker below visits that order, merging byte runs that are adjacent in
// the source so that each merged run is one memcpy.
//
// Point-to-point calls match in MPI order: a send goes to the earliest posted
// receive that matches it, else it is buffered (eagerly, always) as an
// unexpected message; a receive takes the earliest matching unexpected message.
// A send to another rank is packed into host bytes and written to that rank's
// socket; a stream per pair keeps messages between two ranks in order, as
// MPI's non-overtaking rule needs.  Messages are read from the sockets
// whenever a call makes progress (tests, waits, and a send blocked on a full
// socket, so two ranks sending to each other never deadlock).  With one
// rank, a blocking receive that has nothing to match can never complete, so
// it returns MPI_ERR_OTHER instead of hanging; with several, it waits for at
// most MINIMPI_TIMEOUT_S seconds (default 60) before it does the same.

#include "mpi.h"

#include <cuda_runtime.h>

#include <fcntl.h>
#include <poll.h>
#include <sys/socket.h>
#include <sys/stat.h>
#include <sys/un.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <ctime>
#include <deque>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace {

struct TypeRec {
  int combiner = MPI_COMBINER_NAMED;
  std::vector<int> ints;
  std::vector<MPI_Aint> addrs;
  std::vector<MPI_Datatype> types;
  int64_t size = 0;
  int64_t lb = 0, ub = 0;           // extent = ub - lb
  int64_t true_lb = 0, true_ub = 0; // bounds of the bytes actually described
  bool dense = false; // type map is one ascending contiguous run, lb==true_lb
  bool committed = false;
  bool freed = false;
  int64_t extent() const { return ub - lb; }
};

std::recursive_mutex g_mu;
std::vector<TypeRec> g_types;
bool g_initialized = false, g_finalized = false;

void init_named() {
  if (!g_types.empty())
    return;
  g_types.resize(MPI_UINT64_T + 1);
  const int sizes[] = {0, 1, 1, 1, 2, 4, 4, 8, 8, 4, 8, 1, 8, 8};
  for (int h = 1; h <= MPI_UINT64_T; ++h) {
    TypeRec &t = g_types[h];
    t.combiner = MPI_COMBINER_NAMED;
    t.size = sizes[h];
    t.lb = t.true_lb = 0;
    t.ub = t.true_ub = sizes[h];
    t.dense = true;
    t.committed = true;
  }
}

TypeRec *get(MPI_Datatype h) {
  init_named();
  if (h <= 0 || h >= (int)g_types.size() || g_types[h].freed)
    return nullptr;
  return &g_types[h];
}

MPI_Datatype add(TypeRec &&t) {
  init_named();
  g_types.push_back(std::move(t));
  return (MPI_Datatype)(g_types.size() - 1);
}

// Bounds of a set of copies of child `c` placed at displacements in
// [dmin, dmax] (both attained); `n` copies in total.
void set_bounds(TypeRec &t, const TypeRec &c, int64_t dmin, int64_t dmax,
                int64_t n) {
  if (n <= 0 || (c.size == 0 && c.extent() == 0)) {
    t.lb = t.ub = t.true_lb = t.true_ub = 0;
    return;
  }
  t.lb = dmin + c.lb;
  t.ub = dmax + c.ub;
  t.true_lb = dmin + c.true_lb;
  t.true_ub = dmax + c.true_ub;
}

// Range of j*step for 0 <= j < count.
void term_range(int64_t count, int64_t step, int64_t &lo, int64_t &hi) {
  int64_t last = (count - 1) * step;
  lo = std::min<int64_t>(0, last);
  hi = std::max<int64_t>(0, last);
}

// ---- type-map walk ---------------------------------------------------------

struct Runs {
  int64_t off = 0, len = 0;
  template <class Flush> void emit(int64_t o, int64_t l, Flush &flush) {
    if (l <= 0)
      return;
    if (len > 0 && o == off + len) {
      len += l;
      return;
    }
    if (len > 0)
      flush(off, len);
    off = o;
    len = l;
  }
  template <class Flush> void finish(Flush &flush) {
    if (len > 0)
      flush(off, len);
    len = 0;
  }
};

template <class Flush>
void walk(const TypeRec &t, int64_t base, Runs &r, Flush &flush);

// `count` copies of child c, copy k at base + k*step
template <class Flush>
void walk_run(const TypeRec &c, int64_t base, int64_t count, int64_t step,
              Runs &r, Flush &flush) {
  if (c.dense && step == c.size) {
    r.emit(base + c.lb, count * c.size, flush);
    return;
  }
  for (int64_t k = 0; k < count; ++k)
    walk(c, base + k * step, r, flush);
}

template <class Flush>
void walk(const TypeRec &t, int64_t base, Runs &r, Flush &flush) {
  if (t.dense) {
    r.emit(base + t.true_lb, t.size, flush);
    return;
  }
  switch (t.combiner) {
  case MPI_COMBINER_DUP:
  case MPI_COMBINER_RESIZED:
    walk(g_types[t.types[0]], base, r, flush);
    return;
  case MPI_COMBINER_CONTIGUOUS: {
    const TypeRec &c = g_types[t.types[0]];
    walk_run(c, base, t.ints[0], c.extent(), r, flush);
    return;
  }
  case MPI_COMBINER_VECTOR:
  case MPI_COMBINER_HVECTOR: {
    const TypeRec &c = g_types[t.types[0]];
    const int64_t count = t.ints[0], bl = t.ints[1];
    const int64_t stride = t.combiner == MPI_COMBINER_VECTOR
                               ? int64_t(t.ints[2]) * c.extent()
                               : int64_t(t.addrs[0]);
    for (int64_t j = 0; j < count; ++j)
      walk_run(c, base + j * stride, bl, c.extent(), r, flush);
    return;
  }
  case MPI_COMBINER_INDEXED:
  case MPI_COMBINER_HINDEXED: {
    const TypeRec &c = g_types[t.types[0]];
    const int n = t.ints[0];
    for (int i = 0; i < n; ++i) {
      int64_t d = t.combiner == MPI_COMBINER_INDEXED
                      ? int64_t(t.ints[1 + n + i]) * c.extent()
                      : int64_t(t.addrs[i]);
      walk_run(c, base + d, t.ints[1 + i], c.extent(), r, flush);
    }
    return;
  }
  case MPI_COMBINER_INDEXED_BLOCK:
  case MPI_COMBINER_HINDEXED_BLOCK: {
    const TypeRec &c = g_types[t.types[0]];
    const int n = t.ints[0], bl = t.ints[1];
    for (int i = 0; i < n; ++i) {
      int64_t d = t.combiner == MPI_COMBINER_INDEXED_BLOCK
                      ? int64_t(t.ints[2 + i]) * c.extent()
                      : int64_t(t.addrs[i]);
      walk_run(c, base + d, bl, c.extent(), r, flush);
    }
    return;
  }
  case MPI_COMBINER_STRUCT: {
    const int n = t.ints[0];
    for (int i = 0; i < n; ++i) {
      const TypeRec &c = g_types[t.types[i]];
      walk_run(c, base + t.addrs[i], t.ints[1 + i], c.extent(), r, flush);
    }
    return;
  }
  case MPI_COMBINER_SUBARRAY: {
    const TypeRec &c = g_types[t.types[0]];
    const int nd = t.ints[0];
    const int *sizes = &t.ints[1], *subs = &t.ints[1 + nd],
              *starts = &t.ints[1 + 2 * nd];
    const bool corder = t.ints[1 + 3 * nd] == MPI_ORDER_C;
    // dims listed slowest-varying first
    std::vector<int64_t> cnt(nd), str(nd);
    int64_t off = 0;
    for (int k = 0; k < nd; ++k) {
      int d = corder ? k : nd - 1 - k;
      int64_t s = c.extent();
      if (corder)
        for (int j = d + 1; j < nd; ++j)
          s *= sizes[j];
      else
        for (int j = 0; j < d; ++j)
          s *= sizes[j];
      cnt[k] = subs[d];
      str[k] = s;
      off += int64_t(starts[d]) * s;
    }
    for (int k = 0; k < nd; ++k)
      if (cnt[k] == 0)
        return;
    std::vector<int64_t> idx(nd, 0);
    const int inner = nd - 1;
    while (true) {
      int64_t o = base + off;
      for (int k = 0; k < inner; ++k)
        o += idx[k] * str[k];
      walk_run(c, o, cnt[inner], str[inner], r, flush);
      int k = inner - 1;
      while (k >= 0 && ++idx[k] == cnt[k]) {
        idx[k] = 0;
        --k;
      }
      if (k < 0)
        break;
    }
    return;
  }
  default:
    return;
  }
}

// ---- device awareness ------------------------------------------------------

bool is_device(const void *p) {
  if (!p)
    return false;
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice;
}

// Every copy that touches GPU memory runs on the library's own stream and is
// waited for before the call returns, so a completed send or receive has its
// bytes in place for any later work on any stream.  (A device-to-device
// cudaMemcpy returns before the copy is done, and the legacy stream it runs
// on does not order work on non-blocking streams, such as the one a caller
// unpacks a received buffer on.)
int cuda_copy(void *dst, const void *src, size_t n) {
  static cudaStream_t stream = nullptr;
  if (n == 0)
    return MPI_SUCCESS;
  if (!stream && cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    return MPI_ERR_OTHER;
  }
  if (cudaMemcpyAsync(dst, src, n, cudaMemcpyDefault, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess) {
    cudaGetLastError();
    return MPI_ERR_OTHER;
  }
  return MPI_SUCCESS;
}

// whether p is host memory (pageable or pinned)
bool host_memory(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeUnregistered || a.type == cudaMemoryTypeHost;
}

// One contiguous copy of a self-message, as a library's shared-memory path
// would make it: host to host by memcpy (split over threads above 16 MiB,
// as an optimised copy loop would run), anything touching device or managed
// memory by cuda_copy.
int copy_bytes(void *dst, const void *src, int64_t n) {
  if (n <= 0)
    return MPI_SUCCESS;
  if (host_memory(src) && host_memory(dst)) {
    constexpr int64_t kSplit = int64_t(16) << 20;
    const int nt = n < kSplit ? 1 : int(std::min<int64_t>(8, n / kSplit));
    if (nt == 1) {
      std::memcpy(dst, src, size_t(n));
      return MPI_SUCCESS;
    }
    std::vector<std::thread> ts;
    const int64_t per = (n + nt - 1) / nt;
    for (int i = 0; i < nt; ++i) {
      const int64_t a = i * per, b = std::min(n, a + per);
      if (a < b)
        ts.emplace_back([=] {
          std::memcpy(static_cast<char *>(dst) + a,
                      static_cast<const char *>(src) + a, size_t(b - a));
        });
    }
    for (auto &t : ts)
      t.join();
    return MPI_SUCCESS;
  }
  return cuda_copy(dst, src, size_t(n));
}

// byte span [lo, hi) touched by `count` objects of type t
void span(const TypeRec &t, int64_t count, int64_t &lo, int64_t &hi) {
  if (count <= 0 || t.size == 0) {
    lo = hi = 0;
    return;
  }
  int64_t a = 0, b = (count - 1) * t.extent();
  lo = std::min(a, b) + t.true_lb;
  hi = std::max(a, b) + t.true_ub;
}

// pack `count` objects at `in` (host memory) into `out` (host memory)
int64_t pack_host(const TypeRec &t, const char *in, int64_t count, char *out) {
  int64_t pos = 0;
  auto flush = [&](int64_t o, int64_t l) {
    std::memcpy(out + pos, in + o, l);
    pos += l;
  };
  Runs r;
  for (int64_t i = 0; i < count; ++i)
    walk(t, i * t.extent(), r, flush);
  r.finish(flush);
  return pos;
}

int64_t unpack_host(const TypeRec &t, const char *in, int64_t count,
                    char *out) {
  int64_t pos = 0;
  auto flush = [&](int64_t o, int64_t l) {
    std::memcpy(out + o, in + pos, l);
    pos += l;
  };
  Runs r;
  for (int64_t i = 0; i < count; ++i)
    walk(t, i * t.extent(), r, flush);
  r.finish(flush);
  return pos;
}

// pack from any memory into a host vector
int pack_any(const TypeRec &t, const void *buf, int64_t count,
             std::vector<char> &out) {
  out.resize(size_t(count * t.size));
  if (out.empty())
    return MPI_SUCCESS;
  if (!is_device(buf)) {
    pack_host(t, (const char *)buf, count, out.data());
    return MPI_SUCCESS;
  }
  int64_t lo, hi;
  span(t, count, lo, hi);
  std::vector<char> stage(size_t(hi - lo));
  if (cuda_copy(stage.data(), (const char *)buf + lo, size_t(hi - lo)))
    return MPI_ERR_OTHER;
  pack_host(t, stage.data() - lo, count, out.data());
  return MPI_SUCCESS;
}

// unpack `n` packed bytes into any memory
int unpack_any(const TypeRec &t, const char *packed, int64_t count, void *buf) {
  if (count <= 0 || t.size == 0)
    return MPI_SUCCESS;
  if (!is_device(buf)) {
    unpack_host(t, packed, count, (char *)buf);
    return MPI_SUCCESS;
  }
  int64_t lo, hi;
  span(t, count, lo, hi);
  std::vector<char> stage(size_t(hi - lo));
  char *dev = (char *)buf + lo;
  if (cuda_copy(stage.data(), dev, size_t(hi - lo)))
    return MPI_ERR_OTHER;
  unpack_host(t, packed, count, stage.data() - lo);
  if (cuda_copy(dev, stage.data(), size_t(hi - lo)))
    return MPI_ERR_OTHER;
  return MPI_SUCCESS;
}

// ---- point to point ----------------------------------------------------------

// A buffered message.  Contiguous payloads sent from device memory stay in
// device memory (a CUDA-aware MPI moves them device to device); everything
// else is packed into host memory.
struct Message {
  int tag;
  MPI_Comm comm;
  std::vector<char> data; // host payload
  void *dev = nullptr;    // device payload, if any
  int64_t bytes = 0;
  int source = 0; // sending rank
};

std::unordered_map<int64_t, std::vector<void *>> g_dev_pool;

void *dev_get(int64_t n) {
  auto &v = g_dev_pool[n];
  if (!v.empty()) {
    void *p = v.back();
    v.pop_back();
    return p;
  }
  void *p = nullptr;
  if (cudaMalloc(&p, n) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void dev_put(void *p, int64_t n) {
  if (p)
    g_dev_pool[n].push_back(p);
}

struct Req {
  bool send = false, persistent = false, active = false, complete = false;
  const void *sbuf = nullptr;
  void *rbuf = nullptr;
  int count = 0;
  MPI_Datatype type = MPI_DATATYPE_NULL;
  int peer = 0, tag = 0;
  MPI_Comm comm = MPI_COMM_WORLD;
  MPI_Status st{};
};

std::deque<Message> g_unexpected;
std::deque<int> g_posted; // active receive requests, in posting order
std::unordered_map<int, Req> g_reqs;
int g_next_req = 1;

// Distributed graph communicators.  Point-to-point traffic of a
// neighbourhood collective travels on the communicator's collective context
// (the handle with kCollBit set), so it never matches user messages.
struct Graph {
  std::vector<int> sources, sweights, dests, dweights;
  bool weighted = false;
};
std::unordered_map<MPI_Comm, Graph> g_graphs;
MPI_Comm g_next_comm = 16;
constexpr MPI_Comm kCollBit = 0x40000000;
// tags of the library's own collectives (on collective contexts only)
constexpr int kBarrierTag = 0x7ffffff0, kAlltoallvTag = 0x7ffffff1;

bool valid_comm(MPI_Comm c) {
  c &= ~kCollBit;
  return c == MPI_COMM_WORLD || c == MPI_COMM_SELF || g_graphs.count(c) > 0;
}

bool tag_match(int want, int have) { return want == MPI_ANY_TAG || want == have; }

// deliver message bytes into a receive request
int deliver(Req &r, const Message &m) {
  const TypeRec *t = get(r.type);
  if (!t)
    return MPI_ERR_TYPE;
  int64_t cap = int64_t(r.count) * t->size;
  int64_t n = m.bytes;
  int err = MPI_SUCCESS;
  if (n > cap) {
    err = MPI_ERR_TRUNCATE;
    n = cap;
  }
  int64_t whole = t->size ? n / t->size : 0;
  int e2 = MPI_SUCCESS;
  if (t->dense && n > 0) {
    // contiguous receive: one copy, whatever memory either side is in
    char *dst = (char *)r.rbuf + t->lb;
    const void *src = m.dev ? m.dev : (const void *)m.data.data();
    e2 = copy_bytes(dst, src, n);
  } else if (m.dev) {
    std::vector<char> host(size_t(m.bytes));
    if (cuda_copy(host.data(), m.dev, size_t(m.bytes)))
      e2 = MPI_ERR_OTHER;
    else
      e2 = unpack_any(*t, host.data(), whole, r.rbuf);
  } else {
    e2 = unpack_any(*t, m.data.data(), whole, r.rbuf);
  }
  if (e2 != MPI_SUCCESS)
    err = e2;
  r.st.MPI_SOURCE = m.source;
  r.st.MPI_TAG = m.tag;
  r.st.MPI_ERROR = err;
  r.st.bytes_ = n;
  r.complete = true;
  return err;
}

// ---- ranks on one host -------------------------------------------------------

int g_rank = 0, g_size = 1;
double g_timeout_s = 60;
std::string g_sock_path; // this rank's listening socket, removed at finalize

struct Peer {
  int fd = -1;
  std::vector<char> in; // bytes read, not yet parsed into messages
  size_t head = 0;      // first unparsed byte of `in`
};
std::vector<Peer> g_peers; // by rank; g_peers[g_rank] unused

struct WireHeader {
  uint32_t magic;
  int32_t source, tag, comm;
  int64_t bytes;
};
constexpr uint32_t kWireMagic = 0x314d504du;

void arrive(Message &&m);

// read what the sockets hold and hand every complete message to the matcher
int progress_locked() {
  if (g_size <= 1)
    return MPI_SUCCESS;
  static std::vector<char> tmp(size_t(1) << 20);
  int err = MPI_SUCCESS;
  for (int p = 0; p < g_size; ++p) {
    Peer &pe = g_peers[p];
    if (pe.fd < 0)
      continue;
    while (true) {
      const ssize_t got = ::recv(pe.fd, tmp.data(), tmp.size(), 0);
      if (got > 0) {
        pe.in.insert(pe.in.end(), tmp.data(), tmp.data() + got);
        continue;
      }
      if (got < 0 && errno == EINTR)
        continue;
      if (got < 0 && (errno == EAGAIN || errno == EWOULDBLOCK))
        break;
      // 0: the peer closed its end (it finalised); < 0: a real error
      if (got < 0)
        err = MPI_ERR_OTHER;
      ::close(pe.fd);
      pe.fd = -1;
      break;
    }
    while (pe.in.size() - pe.head >= sizeof(WireHeader)) {
      WireHeader h;
      std::memcpy(&h, pe.in.data() + pe.head, sizeof(h));
      if (h.magic != kWireMagic || h.bytes < 0) {
        std::fprintf(stderr, "minimpi: corrupt message from rank %d\n", p);
        return MPI_ERR_INTERN;
      }
      const size_t need = sizeof(h) + size_t(h.bytes);
      if (pe.in.size() - pe.head < need)
        break;
      Message m{h.tag, MPI_Comm(h.comm), {}, nullptr, h.bytes, h.source};
      const char *payload = pe.in.data() + pe.head + sizeof(h);
      m.data.assign(payload, payload + h.bytes);
      pe.head += need;
      arrive(std::move(m));
    }
    if (pe.head > 0 && (pe.head == pe.in.size() || pe.head > (size_t(16) << 20))) {
      pe.in.erase(pe.in.begin(), pe.in.begin() + ptrdiff_t(pe.head));
      pe.head = 0;
    }
  }
  return err;
}

// wait (up to ms milliseconds) until a socket has something to read, or
// (want_write) until `write_fd` can take more
void wait_io(int ms, int write_fd = -1) {
  std::vector<pollfd> fds;
  for (const Peer &pe : g_peers)
    if (pe.fd >= 0)
      fds.push_back({pe.fd, short(pe.fd == write_fd ? POLLIN | POLLOUT : POLLIN), 0});
  if (!fds.empty())
    ::poll(fds.data(), fds.size(), ms);
}

// write all of [p, p + n) to `fd`, reading incoming messages whenever the
// socket is full, so that two ranks writing to each other both progress
int write_all(int fd, const char *p, size_t n) {
  const auto t0 = std::chrono::steady_clock::now();
  while (n > 0) {
    const ssize_t put = ::send(fd, p, n, MSG_NOSIGNAL);
    if (put > 0) {
      p += put;
      n -= size_t(put);
      continue;
    }
    if (put < 0 && errno == EINTR)
      continue;
    if (put < 0 && errno != EAGAIN && errno != EWOULDBLOCK)
      return MPI_ERR_OTHER;
    progress_locked();
    wait_io(1, fd);
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0)
            .count() > g_timeout_s)
      return MPI_ERR_OTHER;
  }
  return MPI_SUCCESS;
}

// an eager send to another rank: the described bytes in MPI order
int send_remote(const void *buf, int count, const TypeRec &t, int dest,
                int tag, MPI_Comm comm) {
  Peer &pe = g_peers[dest];
  if (pe.fd < 0)
    return MPI_ERR_OTHER;
  std::vector<char> data;
  int err = pack_any(t, buf, count, data);
  if (err)
    return err;
  const WireHeader h{kWireMagic, g_rank, tag, int32_t(comm), int64_t(data.size())};
  err = write_all(pe.fd, reinterpret_cast<const char *>(&h), sizeof(h));
  if (!err)
    err = write_all(pe.fd, data.data(), data.size());
  return err;
}

// Join the world named by MINIMPI_SIZE / MINIMPI_RANK / MINIMPI_DIR: listen
// on <dir>/r<rank>.sock, connect to every lower rank (sending our rank), and
// accept every higher one.
int world_init() {
  const char *sz = std::getenv("MINIMPI_SIZE");
  const char *rk = std::getenv("MINIMPI_RANK");
  const char *dir = std::getenv("MINIMPI_DIR");
  if (const char *t = std::getenv("MINIMPI_TIMEOUT_S"))
    g_timeout_s = std::max(1.0, std::atof(t));
  g_size = sz ? std::max(1, std::atoi(sz)) : 1;
  g_rank = rk ? std::atoi(rk) : 0;
  if (g_size <= 1) {
    g_size = 1;
    g_rank = 0;
    return MPI_SUCCESS;
  }
  if (g_rank < 0 || g_rank >= g_size || !dir) {
    std::fprintf(stderr, "minimpi: MINIMPI_SIZE=%d needs MINIMPI_RANK in range "
                         "and MINIMPI_DIR\n", g_size);
    return MPI_ERR_OTHER;
  }
  ::mkdir(dir, 0700);
  g_peers.assign(size_t(g_size), Peer{});
  auto path_of = [&](int r) { return std::string(dir) + "/r" + std::to_string(r) + ".sock"; };
  const int lfd = ::socket(AF_UNIX, SOCK_STREAM, 0);
  sockaddr_un a{};
  a.sun_family = AF_UNIX;
  g_sock_path = path_of(g_rank);
  if (lfd < 0 || g_sock_path.size() >= sizeof(a.sun_path))
    return MPI_ERR_OTHER;
  std::strcpy(a.sun_path, g_sock_path.c_str());
  ::unlink(a.sun_path);
  if (::bind(lfd, reinterpret_cast<sockaddr *>(&a), sizeof(a)) != 0 ||
      ::listen(lfd, g_size) != 0) {
    ::close(lfd);
    return MPI_ERR_OTHER;
  }
  const auto t0 = std::chrono::steady_clock::now();
  auto late = [&] {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0)
               .count() > g_timeout_s;
  };
  for (int p = 0; p < g_rank; ++p) { // connect to the lower ranks
    sockaddr_un b{};
    b.sun_family = AF_UNIX;
    std::strcpy(b.sun_path, path_of(p).c_str());
    int fd = -1;
    while (true) {
      fd = ::socket(AF_UNIX, SOCK_STREAM, 0);
      if (fd >= 0 && ::connect(fd, reinterpret_cast<sockaddr *>(&b), sizeof(b)) == 0)
        break;
      if (fd >= 0)
        ::close(fd);
      fd = -1;
      if (late()) {
        ::close(lfd);
        return MPI_ERR_OTHER;
      }
      ::usleep(2000);
    }
    const int32_t me = g_rank;
    if (::send(fd, &me, sizeof(me), MSG_NOSIGNAL) != ssize_t(sizeof(me))) {
      ::close(fd);
      ::close(lfd);
      return MPI_ERR_OTHER;
    }
    g_peers[p].fd = fd;
  }
  for (int k = g_rank + 1; k < g_size; ++k) { // accept the higher ranks
    pollfd pf{lfd, POLLIN, 0};
    while (::poll(&pf, 1, 10) == 0)
      if (late()) {
        ::close(lfd);
        return MPI_ERR_OTHER;
      }
    const int fd = ::accept(lfd, nullptr, nullptr);
    int32_t who = -1;
    if (fd < 0 || ::recv(fd, &who, sizeof(who), MSG_WAITALL) != ssize_t(sizeof(who)) ||
        who <= g_rank || who >= g_size || g_peers[who].fd >= 0) {
      if (fd >= 0)
        ::close(fd);
      ::close(lfd);
      return MPI_ERR_OTHER;
    }
    g_peers[who].fd = fd;
  }
  ::close(lfd);
  for (Peer &pe : g_peers)
    if (pe.fd >= 0)
      ::fcntl(pe.fd, F_SETFL, ::fcntl(pe.fd, F_GETFL) | O_NONBLOCK);
  return MPI_SUCCESS;
}

void world_finalize() {
  for (Peer &pe : g_peers)
    if (pe.fd >= 0) {
      ::close(pe.fd);
      pe.fd = -1;
    }
  if (!g_sock_path.empty())
    ::unlink(g_sock_path.c_str());
  g_sock_path.clear();
}

int do_send(const void *buf, int count, MPI_Datatype type, int dest, int tag,
            MPI_Comm comm) {
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  if (dest == MPI_PROC_NULL)
    return MPI_SUCCESS;
  if (dest < 0 || dest >= g_size)
    return MPI_ERR_RANK;
  if (count < 0)
    return MPI_ERR_COUNT;
  const TypeRec *t = get(type);
  if (!t)
    return MPI_ERR_TYPE;
  if (dest != g_rank)
    return send_remote(buf, count, *t, dest, tag, comm);
  // rendezvous: a matching receive is already posted and both sides are
  // contiguous, so the bytes go straight from buffer to buffer in one copy
  for (auto it = g_posted.begin(); it != g_posted.end(); ++it) {
    Req &r = g_reqs[*it];
    if (r.comm != comm || !(r.peer == g_rank || r.peer == MPI_ANY_SOURCE) ||
        !tag_match(r.tag, tag))
      continue;
    const TypeRec *rt = get(r.type);
    if (!rt || !t->dense || !rt->dense)
      break; // the buffered path below delivers to this same receive
    g_posted.erase(it);
    int64_t n = int64_t(count) * t->size;
    const int64_t cap = int64_t(r.count) * rt->size;
    int err = MPI_SUCCESS;
    if (n > cap) {
      err = MPI_ERR_TRUNCATE;
      n = cap;
    }
    const char *src = (const char *)buf + t->lb;
    char *dst = (char *)r.rbuf + rt->lb;
    if (int e = copy_bytes(dst, src, n))
      err = e;
    r.st.MPI_SOURCE = g_rank;
    r.st.MPI_TAG = tag;
    r.st.MPI_ERROR = err;
    r.st.bytes_ = n;
    r.complete = true;
    return MPI_SUCCESS;
  }
  Message m{tag, comm, {}, nullptr, int64_t(count) * t->size, g_rank};
  if (t->dense && m.bytes > 0 && is_device(buf)) {
    m.dev = dev_get(m.bytes);
    if (!m.dev || cuda_copy(m.dev, (const char *)buf + t->lb, size_t(m.bytes)))
      return MPI_ERR_OTHER;
  } else {
    int err = pack_any(*t, buf, count, m.data);
    if (err)
      return err;
  }
  arrive(std::move(m));
  return MPI_SUCCESS;
}

// a message from any rank: to the earliest matching posted receive, else
// into the unexpected queue
void arrive(Message &&m) {
  for (auto it = g_posted.begin(); it != g_posted.end(); ++it) {
    Req &r = g_reqs[*it];
    if (r.comm == m.comm && (r.peer == m.source || r.peer == MPI_ANY_SOURCE) &&
        tag_match(r.tag, m.tag)) {
      g_posted.erase(it);
      deliver(r, m);
      dev_put(m.dev, m.bytes);
      return;
    }
  }
  g_unexpected.push_back(std::move(m));
}

// try to satisfy an active receive from the unexpected queue
bool try_match(Req &r) {
  for (auto it = g_unexpected.begin(); it != g_unexpected.end(); ++it) {
    if (it->comm == r.comm && tag_match(r.tag, it->tag) &&
        (r.peer == MPI_ANY_SOURCE || r.peer == it->source)) {
      Message m = std::move(*it);
      g_unexpected.erase(it);
      deliver(r, m);
      dev_put(m.dev, m.bytes);
      return true;
    }
  }
  return false;
}

int start_req(int id) {
  Req &r = g_reqs[id];
  r.active = true;
  r.complete = false;
  r.st = MPI_Status{};
  if (r.send) {
    int err = do_send(r.sbuf, r.count, r.type, r.peer, r.tag, r.comm);
    r.complete = true;
    r.st.MPI_ERROR = err;
    return err;
  }
  if (r.peer == MPI_PROC_NULL) {
    r.complete = true;
    r.st.MPI_SOURCE = MPI_PROC_NULL;
    r.st.MPI_TAG = MPI_ANY_TAG;
    return MPI_SUCCESS;
  }
  if (r.peer != MPI_ANY_SOURCE && (r.peer < 0 || r.peer >= g_size))
    return MPI_ERR_RANK;
  progress_locked();
  if (!try_match(r))
    g_posted.push_back(id);
  return MPI_SUCCESS;
}

int new_req(Req &&r) {
  int id = g_next_req++;
  if (g_next_req >= 0x40000000)
    g_next_req = 1; // stay clear of the high bit range
  g_reqs[id] = std::move(r);
  return id;
}

void finish_req(MPI_Request *request, MPI_Status *status) {
  Req &r = g_reqs[*request];
  if (status)
    *status = r.st;
  if (r.persistent) {
    r.active = false;
  } else {
    g_reqs.erase(*request);
    *request = MPI_REQUEST_NULL;
  }
}

// Test hook (minimpi_fail_nth): the n-th call of one entry point from then
// on returns MPI_ERR_OTHER and does nothing, so the error paths of the
// library's callers can be exercised on the host.  Caller holds g_mu.
std::string g_fail_call;
int g_fail_left = 0;
bool injected_failure(const char *name) {
  if (g_fail_left <= 0 || g_fail_call != name)
    return false;
  return --g_fail_left == 0;
}

int new_type(TypeRec &&t, MPI_Datatype *newtype) {
  if (!newtype)
    return MPI_ERR_ARG;
  *newtype = add(std::move(t));
  return MPI_SUCCESS;
}

} // namespace

extern "C" {

// Arms the failure of the n-th later call of `call` ("MPI_Send", "MPI_Recv",
// "MPI_Irecv", "MPI_Send_init", "MPI_Start" or "MPI_Test"; calls the library
// makes to itself count too); n <= 0 disarms it.  Not part of MPI: a test
// hook of this stand-in library.
int minimpi_fail_nth(const char *call, int n) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  g_fail_call = call ? call : "";
  g_fail_left = n > 0 ? n : 0;
  return MPI_SUCCESS;
}

int MPI_Init(int *, char ***) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  init_named();
  if (!g_initialized) {
    int err = world_init();
    if (err)
      return err;
  }
  g_initialized = true;
  return MPI_SUCCESS;
}
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
  (void)required;
  if (provided)
    *provided = MPI_THREAD_SERIALIZED;
  return MPI_Init(argc, argv);
}
int MPI_Finalize(void) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (g_finalized)
    return MPI_SUCCESS;
  int err = g_size > 1 ? MPI_Barrier(MPI_COMM_WORLD) : MPI_SUCCESS;
  world_finalize();
  g_finalized = true;
  return err;
}
int MPI_Initialized(int *flag) {
  *flag = g_initialized;
  return MPI_SUCCESS;
}
int MPI_Finalized(int *flag) {
  *flag = g_finalized;
  return MPI_SUCCESS;
}
int MPI_Abort(MPI_Comm, int errorcode) {
  std::fprintf(stderr, "minimpi: MPI_Abort(%d)\n", errorcode);
  std::exit(errorcode);
}
double MPI_Wtime(void) {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
int MPI_Get_library_version(char *version, int *resultlen) {
  const char *s = "minimpi 1.0 (self-only MPI stand-in)";
  std::strncpy(version, s, MPI_MAX_LIBRARY_VERSION_STRING - 1);
  version[MPI_MAX_LIBRARY_VERSION_STRING - 1] = 0;
  *resultlen = (int)std::strlen(version);
  return MPI_SUCCESS;
}
int MPI_Comm_rank(MPI_Comm comm, int *rank) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  *rank = comm == MPI_COMM_SELF ? 0 : g_rank;
  return MPI_SUCCESS;
}
int MPI_Comm_size(MPI_Comm comm, int *size) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  *size = comm == MPI_COMM_SELF ? 1 : g_size;
  return MPI_SUCCESS;
}
// Every rank sends an empty message to every other rank on the world's
// collective context and waits for all of theirs.
int MPI_Barrier(MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  if (g_size <= 1 || comm == MPI_COMM_SELF)
    return MPI_SUCCESS;
  const MPI_Comm cc = MPI_COMM_WORLD | kCollBit;
  std::vector<MPI_Request> reqs;
  char none = 0;
  int err = MPI_SUCCESS;
  for (int p = 0; p < g_size && !err; ++p) {
    if (p == g_rank)
      continue;
    MPI_Request r;
    err = MPI_Irecv(&none, 0, MPI_BYTE, p, kBarrierTag, cc, &r);
    if (!err)
      reqs.push_back(r);
  }
  for (int p = 0; p < g_size && !err; ++p) {
    if (p == g_rank)
      continue;
    MPI_Request r;
    err = MPI_Isend(&none, 0, MPI_BYTE, p, kBarrierTag, cc, &r);
    if (!err)
      reqs.push_back(r);
  }
  const int werr = MPI_Waitall(int(reqs.size()), reqs.data(), MPI_STATUSES_IGNORE);
  return err ? err : werr;
}
int MPI_Error_string(int errorcode, char *string, int *resultlen) {
  std::snprintf(string, 64, "MPI error %d", errorcode);
  *resultlen = (int)std::strlen(string);
  return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype oldtype,
                        MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (count < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = MPI_COMBINER_CONTIGUOUS;
  t.ints = {count};
  t.types = {oldtype};
  t.size = count * c->size;
  int64_t lo, hi;
  term_range(count, c->extent(), lo, hi);
  set_bounds(t, *c, lo, hi, count);
  t.dense = c->dense && count > 0;
  return new_type(std::move(t), newtype);
}

static int make_vector(int combiner, int count, int bl, int64_t stride_bytes,
                       const std::vector<int> &ints,
                       const std::vector<MPI_Aint> &addrs, MPI_Datatype oldtype,
                       MPI_Datatype *newtype) {
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (count < 0 || bl < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = combiner;
  t.ints = ints;
  t.addrs = addrs;
  t.types = {oldtype};
  t.size = int64_t(count) * bl * c->size;
  int64_t a0, a1, b0, b1;
  term_range(count, stride_bytes, a0, a1);
  term_range(bl, c->extent(), b0, b1);
  set_bounds(t, *c, a0 + b0, a1 + b1, int64_t(count) * bl);
  t.dense = c->dense && count > 0 && bl > 0 &&
            (count == 1 || stride_bytes == bl * c->extent());
  return new_type(std::move(t), newtype);
}

int MPI_Type_vector(int count, int blocklength, int stride,
                    MPI_Datatype oldtype, MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  return make_vector(MPI_COMBINER_VECTOR, count, blocklength,
                     int64_t(stride) * c->extent(),
                     {count, blocklength, stride}, {}, oldtype, newtype);
}

int MPI_Type_create_hvector(int count, int blocklength, MPI_Aint stride,
                            MPI_Datatype oldtype, MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  return make_vector(MPI_COMBINER_HVECTOR, count, blocklength, stride,
                     {count, blocklength}, {stride}, oldtype, newtype);
}

// blocks of bls[i] copies of c at byte displacements d[i]
static void bounds_blocks(TypeRec &t, const TypeRec &c,
                          const std::vector<int64_t> &bl,
                          const std::vector<int64_t> &d) {
  bool any = false;
  int64_t lb = 0, ub = 0, tlb = 0, tub = 0;
  for (size_t i = 0; i < bl.size(); ++i) {
    if (bl[i] <= 0)
      continue;
    int64_t lo, hi;
    term_range(bl[i], c.extent(), lo, hi);
    int64_t l0 = d[i] + lo + c.lb, u0 = d[i] + hi + c.ub;
    int64_t tl = d[i] + lo + c.true_lb, tu = d[i] + hi + c.true_ub;
    if (!any) {
      lb = l0, ub = u0, tlb = tl, tub = tu, any = true;
    } else {
      lb = std::min(lb, l0), ub = std::max(ub, u0);
      tlb = std::min(tlb, tl), tub = std::max(tub, tu);
    }
  }
  t.lb = lb, t.ub = ub, t.true_lb = tlb, t.true_ub = tub;
}

int MPI_Type_indexed(int count, const int bls[], const int displs[],
                     MPI_Datatype oldtype, MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (count < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = MPI_COMBINER_INDEXED;
  t.ints.push_back(count);
  std::vector<int64_t> bl, d;
  for (int i = 0; i < count; ++i)
    t.ints.push_back(bls[i]), bl.push_back(bls[i]), t.size += bls[i] * c->size;
  for (int i = 0; i < count; ++i)
    t.ints.push_back(displs[i]), d.push_back(int64_t(displs[i]) * c->extent());
  t.types = {oldtype};
  bounds_blocks(t, *c, bl, d);
  return new_type(std::move(t), newtype);
}

int MPI_Type_create_hindexed(int count, const int bls[], const MPI_Aint displs[],
                             MPI_Datatype oldtype, MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (count < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = MPI_COMBINER_HINDEXED;
  t.ints.push_back(count);
  std::vector<int64_t> bl, d;
  for (int i = 0; i < count; ++i) {
    t.ints.push_back(bls[i]);
    t.addrs.push_back(displs[i]);
    bl.push_back(bls[i]);
    d.push_back(displs[i]);
    t.size += bls[i] * c->size;
  }
  t.types = {oldtype};
  bounds_blocks(t, *c, bl, d);
  return new_type(std::move(t), newtype);
}

int MPI_Type_create_indexed_block(int count, int blocklength,
                                  const int displs[], MPI_Datatype oldtype,
                                  MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (count < 0 || blocklength < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = MPI_COMBINER_INDEXED_BLOCK;
  t.ints = {count, blocklength};
  std::vector<int64_t> bl(count, blocklength), d;
  for (int i = 0; i < count; ++i)
    t.ints.push_back(displs[i]), d.push_back(int64_t(displs[i]) * c->extent());
  t.types = {oldtype};
  t.size = int64_t(count) * blocklength * c->size;
  bounds_blocks(t, *c, bl, d);
  return new_type(std::move(t), newtype);
}

int MPI_Type_create_hindexed_block(int count, int blocklength,
                                   const MPI_Aint displs[],
                                   MPI_Datatype oldtype,
                                   MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (count < 0 || blocklength < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = MPI_COMBINER_HINDEXED_BLOCK;
  t.ints = {count, blocklength};
  std::vector<int64_t> bl(count, blocklength), d;
  for (int i = 0; i < count; ++i)
    t.addrs.push_back(displs[i]), d.push_back(displs[i]);
  t.types = {oldtype};
  t.size = int64_t(count) * blocklength * c->size;
  bounds_blocks(t, *c, bl, d);
  return new_type(std::move(t), newtype);
}

int MPI_Type_create_struct(int count, const int bls[], const MPI_Aint displs[],
                           const MPI_Datatype types[], MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (count < 0)
    return MPI_ERR_COUNT;
  TypeRec t;
  t.combiner = MPI_COMBINER_STRUCT;
  t.ints.push_back(count);
  bool any = false;
  for (int i = 0; i < count; ++i) {
    const TypeRec *c = get(types[i]);
    if (!c)
      return MPI_ERR_TYPE;
    t.ints.push_back(bls[i]);
    t.addrs.push_back(displs[i]);
    t.types.push_back(types[i]);
    t.size += bls[i] * c->size;
    if (bls[i] <= 0)
      continue;
    TypeRec one;
    bounds_blocks(one, *c, {bls[i]}, {displs[i]});
    if (!any) {
      t.lb = one.lb, t.ub = one.ub, t.true_lb = one.true_lb,
      t.true_ub = one.true_ub, any = true;
    } else {
      t.lb = std::min(t.lb, one.lb), t.ub = std::max(t.ub, one.ub);
      t.true_lb = std::min(t.true_lb, one.true_lb);
      t.true_ub = std::max(t.true_ub, one.true_ub);
    }
  }
  return new_type(std::move(t), newtype);
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[],
                             const int starts[], int order,
                             MPI_Datatype oldtype, MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  if (ndims <= 0 || (order != MPI_ORDER_C && order != MPI_ORDER_FORTRAN))
    return MPI_ERR_ARG;
  for (int d = 0; d < ndims; ++d)
    if (sizes[d] <= 0 || subsizes[d] < 0 || starts[d] < 0 ||
        starts[d] + subsizes[d] > sizes[d])
      return MPI_ERR_ARG;
  TypeRec t;
  t.combiner = MPI_COMBINER_SUBARRAY;
  t.ints.push_back(ndims);
  for (int d = 0; d < ndims; ++d)
    t.ints.push_back(sizes[d]);
  for (int d = 0; d < ndims; ++d)
    t.ints.push_back(subsizes[d]);
  for (int d = 0; d < ndims; ++d)
    t.ints.push_back(starts[d]);
  t.ints.push_back(order);
  t.types = {oldtype};
  int64_t n = 1, full = 1;
  bool whole = true;
  int64_t tlo = 0, thi = 0;
  for (int d = 0; d < ndims; ++d) {
    n *= subsizes[d];
    full *= sizes[d];
    whole = whole && subsizes[d] == sizes[d];
  }
  // true bounds: first and last described element
  int64_t first = 0, last = 0;
  for (int d = 0; d < ndims; ++d) {
    int64_t s = c->extent();
    if (order == MPI_ORDER_C)
      for (int j = d + 1; j < ndims; ++j)
        s *= sizes[j];
    else
      for (int j = 0; j < d; ++j)
        s *= sizes[j];
    first += int64_t(starts[d]) * s;
    last += int64_t(starts[d] + subsizes[d] - 1) * s;
  }
  tlo = first + c->true_lb;
  thi = last + c->true_ub;
  t.size = n * c->size;
  // the subarray type spans the whole array: lb = 0, extent = prod(sizes)*ext
  t.lb = 0;
  t.ub = full * c->extent();
  if (n > 0) {
    t.true_lb = tlo;
    t.true_ub = thi;
  }
  t.dense = c->dense && whole;
  return new_type(std::move(t), newtype);
}

int MPI_Type_create_resized(MPI_Datatype oldtype, MPI_Aint lb, MPI_Aint extent,
                            MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  TypeRec t;
  t.combiner = MPI_COMBINER_RESIZED;
  t.addrs = {lb, extent};
  t.types = {oldtype};
  t.size = c->size;
  t.lb = lb;
  t.ub = lb + extent;
  t.true_lb = c->true_lb;
  t.true_ub = c->true_ub;
  t.dense = c->dense && lb == c->lb && extent == c->extent();
  return new_type(std::move(t), newtype);
}

int MPI_Type_dup(MPI_Datatype oldtype, MPI_Datatype *newtype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *c = get(oldtype);
  if (!c)
    return MPI_ERR_TYPE;
  TypeRec t = *c;
  t.combiner = MPI_COMBINER_DUP;
  t.ints.clear();
  t.addrs.clear();
  t.types = {oldtype};
  t.committed = false;
  return new_type(std::move(t), newtype);
}

int MPI_Type_commit(MPI_Datatype *datatype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  TypeRec *t = get(datatype ? *datatype : 0);
  if (!t)
    return MPI_ERR_TYPE;
  t->committed = true;
  return MPI_SUCCESS;
}

int MPI_Type_free(MPI_Datatype *datatype) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  TypeRec *t = get(datatype ? *datatype : 0);
  if (!t || t->combiner == MPI_COMBINER_NAMED)
    return MPI_ERR_TYPE;
  // handles are never reused, so types built on this one stay valid
  t->freed = true;
  *datatype = MPI_DATATYPE_NULL;
  return MPI_SUCCESS;
}

int MPI_Type_size(MPI_Datatype datatype, int *size) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  *size = (int)t->size;
  return MPI_SUCCESS;
}

int MPI_Type_get_extent(MPI_Datatype datatype, MPI_Aint *lb, MPI_Aint *extent) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  *lb = t->lb;
  *extent = t->extent();
  return MPI_SUCCESS;
}

int MPI_Type_get_true_extent(MPI_Datatype datatype, MPI_Aint *true_lb,
                             MPI_Aint *true_extent) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  *true_lb = t->true_lb;
  *true_extent = t->true_ub - t->true_lb;
  return MPI_SUCCESS;
}

int MPI_Type_get_envelope(MPI_Datatype datatype, int *ni, int *na, int *nd,
                          int *combiner) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  *combiner = t->combiner;
  if (t->combiner == MPI_COMBINER_NAMED) {
    *ni = *na = *nd = 0;
  } else {
    *ni = (int)t->ints.size();
    *na = (int)t->addrs.size();
    *nd = (int)t->types.size();
  }
  return MPI_SUCCESS;
}

int MPI_Type_get_contents(MPI_Datatype datatype, int max_integers,
                          int max_addresses, int max_datatypes, int ints[],
                          MPI_Aint addrs[], MPI_Datatype types[]) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *t = get(datatype);
  if (!t || t->combiner == MPI_COMBINER_NAMED)
    return MPI_ERR_TYPE;
  if (max_integers < (int)t->ints.size() ||
      max_addresses < (int)t->addrs.size() ||
      max_datatypes < (int)t->types.size())
    return MPI_ERR_ARG;
  std::copy(t->ints.begin(), t->ints.end(), ints);
  std::copy(t->addrs.begin(), t->addrs.end(), addrs);
  std::copy(t->types.begin(), t->types.end(), types);
  return MPI_SUCCESS;
}

int MPI_Pack(const void *inbuf, int incount, MPI_Datatype datatype,
             void *outbuf, int outsize, int *position, MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  if (incount < 0 || !position || *position < 0)
    return MPI_ERR_ARG;
  int64_t need = int64_t(incount) * t->size;
  if (*position + need > outsize)
    return MPI_ERR_TRUNCATE;
  std::vector<char> packed;
  int err = pack_any(*t, inbuf, incount, packed);
  if (err)
    return err;
  char *dst = (char *)outbuf + *position;
  if (is_device(outbuf)) {
    if (need && cuda_copy(dst, packed.data(), size_t(need)))
      return MPI_ERR_OTHER;
  } else if (need) {
    std::memcpy(dst, packed.data(), need);
  }
  *position += (int)need;
  return MPI_SUCCESS;
}

int MPI_Unpack(const void *inbuf, int insize, int *position, void *outbuf,
               int outcount, MPI_Datatype datatype, MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  if (outcount < 0 || !position || *position < 0)
    return MPI_ERR_ARG;
  int64_t need = int64_t(outcount) * t->size;
  if (*position + need > insize)
    return MPI_ERR_TRUNCATE;
  std::vector<char> packed((size_t)need);
  const char *src = (const char *)inbuf + *position;
  if (need) {
    if (is_device(inbuf)) {
      if (cuda_copy(packed.data(), src, size_t(need)))
        return MPI_ERR_OTHER;
    } else {
      std::memcpy(packed.data(), src, need);
    }
  }
  int err = unpack_any(*t, packed.data(), outcount, outbuf);
  if (err)
    return err;
  *position += (int)need;
  return MPI_SUCCESS;
}

int MPI_Pack_size(int incount, MPI_Datatype datatype, MPI_Comm comm,
                  int *size) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  const TypeRec *t = get(datatype);
  if (!t)
    return MPI_ERR_TYPE;
  *size = (int)(int64_t(incount) * t->size);
  return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype datatype, int dest,
             int tag, MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (injected_failure("MPI_Send"))
    return MPI_ERR_OTHER;
  return do_send(buf, count, datatype, dest, tag, comm);
}

int MPI_Recv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
             MPI_Comm comm, MPI_Status *status) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (injected_failure("MPI_Recv"))
    return MPI_ERR_OTHER;
  MPI_Request req;
  int err = MPI_Irecv(buf, count, datatype, source, tag, comm, &req);
  if (err)
    return err;
  err = MPI_Wait(&req, status);
  if (err && req != MPI_REQUEST_NULL)
    MPI_Request_free(&req);
  return err;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype datatype, int dest,
              int tag, MPI_Comm comm, MPI_Request *request) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  int err = MPI_Send_init(buf, count, datatype, dest, tag, comm, request);
  if (err)
    return err;
  g_reqs[*request].persistent = false;
  return start_req(*request);
}

int MPI_Irecv(void *buf, int count, MPI_Datatype datatype, int source, int tag,
              MPI_Comm comm, MPI_Request *request) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (injected_failure("MPI_Irecv"))
    return MPI_ERR_OTHER;
  int err = MPI_Recv_init(buf, count, datatype, source, tag, comm, request);
  if (err)
    return err;
  g_reqs[*request].persistent = false;
  return start_req(*request);
}

int MPI_Send_init(const void *buf, int count, MPI_Datatype datatype, int dest,
                  int tag, MPI_Comm comm, MPI_Request *request) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (injected_failure("MPI_Send_init"))
    return MPI_ERR_OTHER;
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  if (!get(datatype))
    return MPI_ERR_TYPE;
  Req r;
  r.send = true;
  r.persistent = true;
  r.sbuf = buf;
  r.count = count;
  r.type = datatype;
  r.peer = dest;
  r.tag = tag;
  r.comm = comm;
  *request = new_req(std::move(r));
  return MPI_SUCCESS;
}

int MPI_Recv_init(void *buf, int count, MPI_Datatype datatype, int source,
                  int tag, MPI_Comm comm, MPI_Request *request) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm))
    return MPI_ERR_COMM;
  if (!get(datatype))
    return MPI_ERR_TYPE;
  Req r;
  r.send = false;
  r.persistent = true;
  r.rbuf = buf;
  r.count = count;
  r.type = datatype;
  r.peer = source;
  r.tag = tag;
  r.comm = comm;
  *request = new_req(std::move(r));
  return MPI_SUCCESS;
}

int MPI_Start(MPI_Request *request) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (injected_failure("MPI_Start"))
    return MPI_ERR_OTHER;
  if (!request || !g_reqs.count(*request))
    return MPI_ERR_REQUEST;
  Req &r = g_reqs[*request];
  if (!r.persistent || r.active)
    return MPI_ERR_REQUEST;
  return start_req(*request);
}

int MPI_Test(MPI_Request *request, int *flag, MPI_Status *status) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (injected_failure("MPI_Test"))
    return MPI_ERR_OTHER;
  progress_locked();
  if (!request)
    return MPI_ERR_REQUEST;
  if (*request == MPI_REQUEST_NULL) {
    *flag = 1;
    return MPI_SUCCESS;
  }
  auto it = g_reqs.find(*request);
  if (it == g_reqs.end())
    return MPI_ERR_REQUEST;
  Req &r = it->second;
  if (r.persistent && !r.active) {
    *flag = 1;
    return MPI_SUCCESS;
  }
  *flag = r.complete;
  if (!r.complete)
    return MPI_SUCCESS;
  int err = r.st.MPI_ERROR;
  finish_req(request, status);
  return err;
}

int MPI_Wait(MPI_Request *request, MPI_Status *status) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  int flag = 0;
  int err = MPI_Test(request, &flag, status);
  if (err)
    return err;
  if (flag)
    return MPI_SUCCESS;
  if (g_size <= 1) {
    // one rank, one thread: no send can arrive while we block
    std::fprintf(stderr,
                 "minimpi: MPI_Wait on a receive with no matching send "
                 "(would deadlock at world size 1)\n");
    return MPI_ERR_OTHER;
  }
  const auto t0 = std::chrono::steady_clock::now();
  while (true) {
    wait_io(1);
    err = MPI_Test(request, &flag, status);
    if (err || flag)
      return err;
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0)
            .count() > g_timeout_s) {
      std::fprintf(stderr, "minimpi: rank %d gave up waiting after %.0f s\n",
                   g_rank, g_timeout_s);
      return MPI_ERR_OTHER;
    }
  }
}

int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status stats[]) {
  int err = MPI_SUCCESS;
  for (int i = 0; i < count; ++i) {
    int e = MPI_Wait(&reqs[i], stats ? &stats[i] : MPI_STATUS_IGNORE);
    if (e && !err)
      err = e;
  }
  return err;
}

// ---- distributed graph topologies ---------------------------------------------

int MPI_Dist_graph_create_adjacent(MPI_Comm comm_old, int indegree,
                                   const int sources[],
                                   const int sourceweights[], int outdegree,
                                   const int destinations[],
                                   const int destweights[], MPI_Info info,
                                   int reorder, MPI_Comm *comm_dist_graph) {
  (void)info;
  (void)reorder; // ranks keep their numbers
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm_old) || (comm_old & kCollBit))
    return MPI_ERR_COMM;
  if (indegree < 0 || outdegree < 0 || !comm_dist_graph ||
      (indegree > 0 && !sources) || (outdegree > 0 && !destinations))
    return MPI_ERR_ARG;
  Graph g;
  g.weighted = sourceweights != MPI_UNWEIGHTED && destweights != MPI_UNWEIGHTED;
  for (int i = 0; i < indegree; ++i) {
    if (sources[i] < 0 || sources[i] >= g_size)
      return MPI_ERR_RANK;
    g.sources.push_back(sources[i]);
    g.sweights.push_back(g.weighted && sourceweights != MPI_WEIGHTS_EMPTY
                             ? sourceweights[i]
                             : 1);
  }
  for (int i = 0; i < outdegree; ++i) {
    if (destinations[i] < 0 || destinations[i] >= g_size)
      return MPI_ERR_RANK;
    g.dests.push_back(destinations[i]);
    g.dweights.push_back(g.weighted && destweights != MPI_WEIGHTS_EMPTY
                             ? destweights[i]
                             : 1);
  }
  const MPI_Comm c = g_next_comm++;
  g_graphs[c] = std::move(g);
  *comm_dist_graph = c;
  return MPI_SUCCESS;
}

int MPI_Dist_graph_neighbors_count(MPI_Comm comm, int *indegree,
                                   int *outdegree, int *weighted) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  auto it = g_graphs.find(comm);
  if (it == g_graphs.end())
    return MPI_ERR_COMM;
  if (indegree)
    *indegree = int(it->second.sources.size());
  if (outdegree)
    *outdegree = int(it->second.dests.size());
  if (weighted)
    *weighted = it->second.weighted ? 1 : 0;
  return MPI_SUCCESS;
}

int MPI_Dist_graph_neighbors(MPI_Comm comm, int maxindegree, int sources[],
                             int sourceweights[], int maxoutdegree,
                             int destinations[], int destweights[]) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  auto it = g_graphs.find(comm);
  if (it == g_graphs.end())
    return MPI_ERR_COMM;
  const Graph &g = it->second;
  for (int i = 0; i < maxindegree && i < int(g.sources.size()); ++i) {
    sources[i] = g.sources[i];
    if (g.weighted && sourceweights && sourceweights != MPI_UNWEIGHTED)
      sourceweights[i] = g.sweights[i];
  }
  for (int i = 0; i < maxoutdegree && i < int(g.dests.size()); ++i) {
    destinations[i] = g.dests[i];
    if (g.weighted && destweights && destweights != MPI_UNWEIGHTED)
      destweights[i] = g.dweights[i];
  }
  return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!comm || !g_graphs.count(*comm))
    return MPI_ERR_COMM;
  g_graphs.erase(*comm);
  *comm = MPI_COMM_NULL;
  return MPI_SUCCESS;
}

extern "C++" {
namespace {

// Post every receive, then every send, on the collective context, and wait
// for all: with FIFO matching per (source, tag) the k-th edge to rank 0 meets
// the k-th edge from it, as MPI-3.1 7.6 requires for repeated edges.
template <typename SendAt, typename RecvAt>
int neighbor_exchange(MPI_Comm comm, SendAt send_at, RecvAt recv_at) {
  auto it = g_graphs.find(comm);
  if (it == g_graphs.end())
    return MPI_ERR_COMM;
  const Graph &g = it->second;
  const MPI_Comm cc = comm | kCollBit;
  std::vector<MPI_Request> reqs;
  int err = MPI_SUCCESS;
  for (size_t j = 0; j < g.sources.size() && !err; ++j) {
    void *buf;
    int count;
    MPI_Datatype t;
    recv_at(j, &buf, &count, &t);
    MPI_Request r;
    err = MPI_Irecv(buf, count, t, g.sources[j], 0, cc, &r);
    if (!err)
      reqs.push_back(r);
  }
  for (size_t i = 0; i < g.dests.size() && !err; ++i) {
    const void *buf;
    int count;
    MPI_Datatype t;
    send_at(i, &buf, &count, &t);
    MPI_Request r;
    err = MPI_Isend(buf, count, t, g.dests[i], 0, cc, &r);
    if (!err)
      reqs.push_back(r);
  }
  const int werr = MPI_Waitall(int(reqs.size()), reqs.data(), MPI_STATUSES_IGNORE);
  return err ? err : werr;
}

} // namespace
} // extern "C++"

int MPI_Neighbor_alltoallv(const void *sendbuf, const int sendcounts[],
                           const int sdispls[], MPI_Datatype sendtype,
                           void *recvbuf, const int recvcounts[],
                           const int rdispls[], MPI_Datatype recvtype,
                           MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *st = get(sendtype), *rt = get(recvtype);
  if (!st || !rt)
    return MPI_ERR_TYPE;
  const int64_t se = st->extent(), re = rt->extent();
  return neighbor_exchange(
      comm,
      [&](size_t i, const void **b, int *n, MPI_Datatype *t) {
        *b = (const char *)sendbuf + int64_t(sdispls[i]) * se;
        *n = sendcounts[i];
        *t = sendtype;
      },
      [&](size_t j, void **b, int *n, MPI_Datatype *t) {
        *b = (char *)recvbuf + int64_t(rdispls[j]) * re;
        *n = recvcounts[j];
        *t = recvtype;
      });
}

int MPI_Neighbor_alltoallw(const void *sendbuf, const int sendcounts[],
                           const MPI_Aint sdispls[],
                           const MPI_Datatype sendtypes[], void *recvbuf,
                           const int recvcounts[], const MPI_Aint rdispls[],
                           const MPI_Datatype recvtypes[], MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  return neighbor_exchange(
      comm,
      [&](size_t i, const void **b, int *n, MPI_Datatype *t) {
        *b = (const char *)sendbuf + sdispls[i];
        *n = sendcounts[i];
        *t = sendtypes[i];
      },
      [&](size_t j, void **b, int *n, MPI_Datatype *t) {
        *b = (char *)recvbuf + rdispls[j];
        *n = recvcounts[j];
        *t = recvtypes[j];
      });
}

// Every rank's block to every rank: one receive per source and one send per
// destination on the communicator's collective context, then wait for all.
int MPI_Alltoallv(const void *sendbuf, const int sendcounts[],
                  const int sdispls[], MPI_Datatype sendtype, void *recvbuf,
                  const int recvcounts[], const int rdispls[],
                  MPI_Datatype recvtype, MPI_Comm comm) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!valid_comm(comm) || (comm & kCollBit))
    return MPI_ERR_COMM;
  const TypeRec *st = get(sendtype), *rt = get(recvtype);
  if (!st || !rt)
    return MPI_ERR_TYPE;
  const int n = comm == MPI_COMM_SELF ? 1 : g_size;
  const int me = comm == MPI_COMM_SELF ? 0 : g_rank;
  const MPI_Comm cc = comm | kCollBit;
  std::vector<MPI_Request> reqs;
  int err = MPI_SUCCESS;
  for (int i = 0; i < n && !err; ++i) {
    MPI_Request r;
    err = MPI_Irecv((char *)recvbuf + int64_t(rdispls[i]) * rt->extent(),
                    recvcounts[i], recvtype, comm == MPI_COMM_SELF ? me : i,
                    kAlltoallvTag, cc, &r);
    if (!err)
      reqs.push_back(r);
  }
  for (int j = 0; j < n && !err; ++j) {
    MPI_Request r;
    err = MPI_Isend((const char *)sendbuf + int64_t(sdispls[j]) * st->extent(),
                    sendcounts[j], sendtype, comm == MPI_COMM_SELF ? me : j,
                    kAlltoallvTag, cc, &r);
    if (!err)
      reqs.push_back(r);
  }
  const int werr = MPI_Waitall(int(reqs.size()), reqs.data(), MPI_STATUSES_IGNORE);
  return err ? err : werr;
}

int MPI_Request_free(MPI_Request *request) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  if (!request || !g_reqs.count(*request))
    return MPI_ERR_REQUEST;
  g_posted.erase(std::remove(g_posted.begin(), g_posted.end(), *request),
                 g_posted.end());
  g_reqs.erase(*request);
  *request = MPI_REQUEST_NULL;
  return MPI_SUCCESS;
}

int MPI_Get_count(const MPI_Status *status, MPI_Datatype datatype,
                  int *count) {
  std::lock_guard<std::recursive_mutex> l(g_mu);
  const TypeRec *t = get(datatype);
  if (!t || !status)
    return MPI_ERR_ARG;
  if (t->size == 0) {
    *count = 0;
  } else if (status->bytes_ % t->size) {
    *count = MPI_UNDEFINED;
  } else {
    *count = (int)(status->bytes_ / t->size);
  }
  return MPI_SUCCESS;
}

} // extern "C"
