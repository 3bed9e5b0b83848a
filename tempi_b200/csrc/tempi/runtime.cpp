// Environment, device stream, pointer classification, slab allocators and
// the event pool.

#include "runtime.hpp"

#include <nvtx3/nvToolsExtCudaRt.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>

namespace tempi {

// ---- environment ----------------------------------------------------------

static Env g_env;
static bool g_env_read = false;

static bool has(const char *name) { return std::getenv(name) != nullptr; }

void read_env() {
  Env e;
  // any value, even empty, counts as set (reference env.cpp:31-83)
  e.disable = has("TEMPI_DISABLE");
  e.no_pack = has("TEMPI_NO_PACK");
  e.no_type_commit = has("TEMPI_NO_TYPE_COMMIT");
  if (has("TEMPI_DATATYPE_ONESHOT"))
    e.datatype = Method::ONESHOT;
  if (has("TEMPI_DATATYPE_DEVICE"))
    e.datatype = Method::DEVICE;
  if (has("TEMPI_DATATYPE_STAGED"))
    e.datatype = Method::STAGED;
  if (has("TEMPI_DATATYPE_AUTO"))
    e.datatype = Method::AUTO;
  if (has("TEMPI_CONTIGUOUS_STAGED"))
    e.contiguous = Contiguous::STAGED;
  if (has("TEMPI_CONTIGUOUS_AUTO"))
    e.contiguous = Contiguous::AUTO;
  if (const char *s = std::getenv("TEMPI_DISPATCH")) {
    std::string v(s);
    if (v == "table")
      e.dispatch = Dispatch::TABLE;
    else if (v == "exhaustive")
      e.dispatch = Dispatch::EXHAUSTIVE;
    else if (v == "heuristic")
      e.dispatch = Dispatch::HEURISTIC;
    else
      e.dispatch = Dispatch::LEARNED;
  }
  if (const char *s = std::getenv("TEMPI_WAIT_TIMEOUT_S"))
    e.wait_timeout_s = std::atof(s);
  if (const char *s = std::getenv("TEMPI_HOST_LINK"))
    e.host_link_dma = std::string(s) != "kernel";
  if (const char *s = std::getenv("TEMPI_HOST_LINK_CHUNK_KB"))
    e.host_link_chunk_kb =
        std::max(0L, std::min(65536L, std::atol(s))) / 256 * 256;
  if (const char *s = std::getenv("TEMPI_TEST_STAGED_SHORTFALL"))
    e.staged_shortfall = std::max(0, std::min(4096, std::atoi(s))) & ~15;
  if (has("TEMPI_ALLTOALLV_REMOTE_FIRST"))
    e.alltoallv = Alltoallv::REMOTE_FIRST;
  if (has("TEMPI_ALLTOALLV_STAGED"))
    e.alltoallv = Alltoallv::STAGED;
  if (has("TEMPI_ALLTOALLV_ISIR_STAGED"))
    e.alltoallv = Alltoallv::ISIR_STAGED;
  if (has("TEMPI_ALLTOALLV_ISIR_REMOTE_STAGED"))
    e.alltoallv = Alltoallv::ISIR_REMOTE_STAGED;
  if (has("TEMPI_NO_ALLTOALLV"))
    e.alltoallv = Alltoallv::NONE;
  if (const char *s = std::getenv("TEMPI_RANKS_PER_NODE"))
    e.ranks_per_node = std::max(0, std::atoi(s));
  if (const char *s = std::getenv("TEMPI_SLAB_CACHE_MB"))
    e.slab_cache_mb = std::max(0L, std::atol(s));
  // test-only: the n-th slab allocation from here on fails
  slab_test_fail_after(std::getenv("TEMPI_TEST_FAIL_SLAB")
                           ? std::atoll(std::getenv("TEMPI_TEST_FAIL_SLAB"))
                           : 0);
  if (const char *cd = std::getenv("TEMPI_CACHE_DIR")) {
    e.cache_dir = cd;
  } else if (const char *x = std::getenv("XDG_CACHE_HOME")) {
    e.cache_dir = std::string(x) + "/tempi";
  } else if (const char *h = std::getenv("HOME")) {
    e.cache_dir = std::string(h) + "/.tempi";
  } else {
    e.cache_dir = "/var/tmp";
  }
  g_env = e;
  g_env_read = true;
}

const Env &env() {
  if (!g_env_read)
    read_env();
  return g_env;
}

// ---- device state ---------------------------------------------------------

static std::mutex g_dev_mu;
static cudaStream_t g_stream = nullptr;
static int g_cuda_ok = -1;

bool cuda_available() {
  if (g_cuda_ok < 0) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess)
      cudaGetLastError();
    g_cuda_ok = (e == cudaSuccess && n > 0) ? 1 : 0;
  }
  return g_cuda_ok == 1;
}

cudaStream_t pack_stream() {
  std::lock_guard<std::mutex> l(g_dev_mu);
  if (!g_stream) {
    if (cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking) !=
        cudaSuccess) {
      cudaGetLastError();
      g_stream = nullptr;
    } else {
      nvtxNameCudaStreamA(g_stream, "TEMPI_pack");
    }
  }
  return g_stream;
}

cudaStream_t link_stream() {
  static cudaStream_t h = nullptr;
  std::lock_guard<std::mutex> l(g_dev_mu);
  if (!h) {
    if (cudaStreamCreateWithFlags(&h, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      h = nullptr;
    } else {
      nvtxNameCudaStreamA(h, "TEMPI_link");
    }
  }
  return h;
}

PtrInfo classify(const void *p) {
  PtrInfo info;
  if (!p || !cuda_available())
    return info;
  cudaPointerAttributes a{};
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return info;
  }
  info.device_accessible = a.devicePointer != nullptr;
  info.is_device = a.type == cudaMemoryTypeDevice;
  info.is_host = a.type == cudaMemoryTypeHost;
  info.device_ptr = a.devicePointer;
  return info;
}

// ---- slab allocators --------------------------------------------------------
//
// Intermediate packed buffers of the senders (reference allocator_slab.hpp:
// power-of-two slabs kept for reuse).  Requests up to 64 MiB round up to a
// power of two and come back through per-class free lists; larger ones round
// up to a multiple of 2 MiB, so a 1 GiB + 1 B message takes 1 GiB + 2 MiB,
// not 2 GiB.  Freed blocks are kept for reuse only while the bytes kept stay
// within TEMPI_SLAB_CACHE_MB (default 4 GiB) per memory space; beyond that
// a freed block goes straight back to CUDA.

namespace {
constexpr int kMaxClass = 26; // 64 MiB
constexpr size_t kLargeGrain = size_t(2) << 20;
struct Slab {
  std::vector<void *> free_[kMaxClass + 1];
  std::vector<std::pair<size_t, void *>> large; // cached blocks above 64 MiB
  std::unordered_map<void *, size_t> size_of;   // every block this space owns
  size_t cached = 0, live = 0;
};
std::mutex g_slab_mu;
Slab g_slabs[2];
std::atomic<int64_t> g_fail_countdown{0};

int size_class(size_t bytes) {
  int c = 8; // 256 B minimum
  while ((size_t(1) << c) < bytes)
    ++c;
  return c;
}

size_t block_size(size_t bytes) {
  const int c = size_class(bytes);
  if (c <= kMaxClass)
    return size_t(1) << c;
  return (bytes + kLargeGrain - 1) / kLargeGrain * kLargeGrain;
}

void release_block(Space s, void *p) {
  cudaError_t e = s == Space::DEVICE ? cudaFree(p) : cudaFreeHost(p);
  if (e != cudaSuccess)
    cuda_error(e, "slab release");
}

void update_gauges() {
  counters().slab_live_bytes =
      int64_t(g_slabs[0].live + g_slabs[1].live);
  counters().slab_cached_bytes =
      int64_t(g_slabs[0].cached + g_slabs[1].cached);
}
} // namespace

void slab_test_fail_after(int64_t n) { g_fail_countdown = n > 0 ? n : 0; }

void *slab_alloc(Space s, size_t bytes) {
  // the test-only failure countdown (TEMPI_TEST_FAIL_SLAB): the n-th
  // allocation from when the knob was read fails as if CUDA had refused it
  int64_t left = g_fail_countdown.load();
  while (left > 0 && !g_fail_countdown.compare_exchange_weak(left, left - 1)) {
  }
  if (left == 1) {
    set_error(TEMPI_ERR_NO_MEM, "slab allocation failed (injected by TEMPI_TEST_FAIL_SLAB)");
    return nullptr;
  }
  const size_t n = block_size(bytes);
  std::lock_guard<std::mutex> l(g_slab_mu);
  Slab &sl = g_slabs[int(s)];
  void *p = nullptr;
  if (n <= (size_t(1) << kMaxClass)) {
    auto &fl = sl.free_[size_class(n)];
    if (!fl.empty()) {
      p = fl.back();
      fl.pop_back();
    }
  } else {
    // the smallest cached large block that fits with at most 1/4 to spare
    size_t best = 0;
    for (size_t i = 0; i < sl.large.size(); ++i)
      if (sl.large[i].first >= n && sl.large[i].first <= n + n / 4 &&
          (!p || sl.large[i].first < sl.large[best].first)) {
        best = i;
        p = sl.large[i].second;
      }
    if (p)
      sl.large.erase(sl.large.begin() + best);
  }
  if (p) {
    const size_t have = sl.size_of[p];
    sl.cached -= have;
    sl.live += have;
    counters().slab_hits++;
    update_gauges();
    return p;
  }
  cudaError_t e = s == Space::DEVICE
                      ? cudaMalloc(&p, n)
                      : cudaHostAlloc(&p, n, cudaHostAllocMapped |
                                                 cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cuda_error(e, "slab allocation");
    return nullptr;
  }
  sl.size_of[p] = n;
  sl.live += n;
  counters().slab_misses++;
  counters().slab_bytes += int64_t(n);
  update_gauges();
  return p;
}

void slab_free(Space s, void *p) {
  if (!p)
    return;
  std::lock_guard<std::mutex> l(g_slab_mu);
  Slab &sl = g_slabs[int(s)];
  auto it = sl.size_of.find(p);
  if (it == sl.size_of.end()) {
    LOG_ERROR("slab_free of a pointer this allocator does not own");
    return;
  }
  const size_t n = it->second;
  sl.live -= n;
  const size_t cap = size_t(env().slab_cache_mb) << 20;
  if (sl.cached + n > cap) { // over the cap: back to CUDA
    sl.size_of.erase(it);
    counters().slab_bytes -= int64_t(n);
    release_block(s, p);
  } else {
    sl.cached += n;
    if (n <= (size_t(1) << kMaxClass))
      sl.free_[size_class(n)].push_back(p);
    else
      sl.large.push_back({n, p});
  }
  update_gauges();
}

void slab_release_all() {
  std::lock_guard<std::mutex> l(g_slab_mu);
  for (int s = 0; s < 2; ++s) {
    for (auto &kv : g_slabs[s].size_of)
      release_block(Space(s), kv.first);
    g_slabs[s].size_of.clear();
    for (auto &f : g_slabs[s].free_)
      f.clear();
    g_slabs[s].large.clear();
    g_slabs[s].cached = g_slabs[s].live = 0;
  }
  counters().slab_bytes = 0;
  update_gauges();
}

// ---- events ---------------------------------------------------------------

static std::mutex g_ev_mu;
static std::vector<cudaEvent_t> g_ev_free;
static int g_ev_used = 0;

cudaEvent_t event_acquire() {
  std::lock_guard<std::mutex> l(g_ev_mu);
  cudaEvent_t e = nullptr;
  if (!g_ev_free.empty()) {
    e = g_ev_free.back();
    g_ev_free.pop_back();
  } else if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) !=
             cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  ++g_ev_used;
  return e;
}

void event_release(cudaEvent_t e) {
  if (!e)
    return;
  std::lock_guard<std::mutex> l(g_ev_mu);
  g_ev_free.push_back(e);
  --g_ev_used;
}

void events_release_all() {
  std::lock_guard<std::mutex> l(g_ev_mu);
  if (g_ev_used)
    LOG_WARN("%d events were never released", g_ev_used);
  for (cudaEvent_t e : g_ev_free)
    cudaEventDestroy(e);
  g_ev_free.clear();
}

} // namespace tempi

extern "C" void *tempi_stream(void) { return tempi::pack_stream(); }

extern "C" int tempi_reload_env(void) {
  tempi::read_env();
  return TEMPI_OK;
}
