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
  if (const char *s = std::getenv("TEMPI_TEST_STAGED_SHORTFALL"))
    e.staged_shortfall = std::max(0, std::min(4096, std::atoi(s))) & ~15;
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

namespace {
struct Slab {
  std::vector<void *> free_[64];
  std::unordered_map<void *, int> cls;
};
std::mutex g_slab_mu;
Slab g_slabs[2];

int size_class(size_t bytes) {
  int c = 8; // 256 B minimum
  while ((size_t(1) << c) < bytes)
    ++c;
  return c;
}
} // namespace

void *slab_alloc(Space s, size_t bytes) {
  const int c = size_class(bytes);
  std::lock_guard<std::mutex> l(g_slab_mu);
  Slab &sl = g_slabs[int(s)];
  if (!sl.free_[c].empty()) {
    void *p = sl.free_[c].back();
    sl.free_[c].pop_back();
    counters().slab_hits++;
    return p;
  }
  void *p = nullptr;
  const size_t n = size_t(1) << c;
  cudaError_t e = s == Space::DEVICE
                      ? cudaMalloc(&p, n)
                      : cudaHostAlloc(&p, n, cudaHostAllocMapped |
                                                 cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cuda_error(e, "slab allocation");
    return nullptr;
  }
  sl.cls[p] = c;
  counters().slab_misses++;
  counters().slab_bytes += int64_t(n);
  return p;
}

void slab_free(Space s, void *p) {
  if (!p)
    return;
  std::lock_guard<std::mutex> l(g_slab_mu);
  Slab &sl = g_slabs[int(s)];
  auto it = sl.cls.find(p);
  if (it == sl.cls.end()) {
    LOG_ERROR("slab_free of a pointer this allocator does not own");
    return;
  }
  sl.free_[it->second].push_back(p);
}

void slab_release_all() {
  std::lock_guard<std::mutex> l(g_slab_mu);
  for (int s = 0; s < 2; ++s) {
    for (auto &kv : g_slabs[s].cls) {
      if (s == int(Space::DEVICE))
        cudaFree(kv.first);
      else
        cudaFreeHost(kv.first);
    }
    g_slabs[s].cls.clear();
    for (auto &f : g_slabs[s].free_)
      f.clear();
  }
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
