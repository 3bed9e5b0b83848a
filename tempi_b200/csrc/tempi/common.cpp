// Logging, error reporting and counters (reference include/logging.hpp,
// include/counters.hpp, src/internal/counters.cpp).  Unlike the reference,
// errors are returned to the caller and never end the process.

#include "internal.hpp"

#include <cstdarg>
#include <mutex>

namespace tempi {

int log_level() {
  static int level = [] {
    const char *s = std::getenv("TEMPI_LOG_LEVEL");
    return s ? std::atoi(s) : 0;
  }();
  return level;
}

static thread_local char g_err[512];
static thread_local const char *g_last_kernel = "none";

int set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  LOG_ERROR("%s", g_err);
  return code;
}

int cuda_error(cudaError_t e, const char *what) {
  cudaGetLastError();
  return set_error(TEMPI_ERR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e),
                   cudaGetErrorString(e));
}

cudaError_t copy_complete(void *dst, const void *src, size_t n) {
  static std::mutex mu;
  static cudaStream_t stream = nullptr;
  if (n == 0)
    return cudaSuccess;
  std::lock_guard<std::mutex> l(mu);
  cudaError_t e = cudaSuccess;
  if (!stream)
    e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dst, src, n, cudaMemcpyDefault, stream);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(stream);
  return e;
}

Counters &counters() {
  static Counters c;
  return c;
}

void set_last_kernel(const char *name) { g_last_kernel = name; }

} // namespace tempi

extern "C" const char *tempi_last_error(void) { return tempi::g_err; }

extern "C" int64_t tempi_kernel_launches(void) {
  return tempi::counters().kernel_launches.load();
}

extern "C" const char *tempi_last_kernel(void) { return tempi::g_last_kernel; }

extern "C" int64_t tempi_counter(const char *name) {
  if (!name)
    return -1;
  if (std::string(name) == "staged_timeouts")
    return tempi::staged_timeouts();
  auto &c = tempi::counters();
  const std::string n(name);
#define C(x)                                                                   \
  if (n == #x)                                                                 \
    return c.x.load();
  C(kernel_launches) C(packs) C(unpacks) C(pack_bytes) C(unpack_bytes)
  C(lib_pack) C(lib_unpack) C(cached_types) C(send_device) C(send_oneshot)
  C(send_staged) C(send_lib) C(recv_device) C(recv_oneshot) C(recv_staged)
  C(recv_lib) C(isend_managed) C(irecv_managed) C(dispatch_hit)
  C(dispatch_miss) C(dispatch_measured) C(slab_hits) C(slab_misses) C(slab_bytes) C(slab_live_bytes) C(slab_cached_bytes) C(host_link_copies)
  C(send_contig_staged) C(recv_contig_staged) C(neighbor_fused)
  C(neighbor_isir) C(neighbor_lib) C(alltoallv_staged) C(alltoallv_remote_first)
  C(alltoallv_isir_staged) C(alltoallv_isir_remote_staged) C(alltoallv_lib)
#undef C
  return -1;
}
