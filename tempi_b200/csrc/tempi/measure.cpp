// Measurement harness: times every candidate the dispatcher chooses among,
// on scratch buffers shaped like the object.  Used three ways: as the
// exhaustive fallback when the cost model's ensemble disagrees, as the
// TEMPI_DISPATCH=exhaustive policy, and to produce the model's training data
// (the reference measures its tables with bin/measure_system.cpp and
// src/internal/measure_system.cu:381-610; these are measurements of this
// library's own kernels and transfers on this machine).

#include "dispatch.hpp"

#include <mpi.h>

#include <chrono>
#include <cmath>
#include <mutex>

namespace tempi {

namespace {

struct Buf {
  void *p = nullptr;
  size_t n = 0;
  bool host = false;
};

std::mutex g_mu;
// one scratch buffer per role and memory kind, grown (never shrunk) so that
// alternating device and host layouts do not reallocate
Buf g_typed[2], g_typed2, g_packed[2];
cudaStream_t g_stream = nullptr;

void *get(Buf &b, size_t n, bool host) {
  if (b.p && b.n >= n)
    return b.p;
  if (b.p)
    b.host ? cudaFreeHost(b.p) : cudaFree(b.p);
  b.p = nullptr;
  b.n = 0;
  n = std::max(n, size_t(1) << 24); // round small requests up to 16 MiB
  cudaError_t e = host ? cudaHostAlloc(&b.p, n, cudaHostAllocMapped |
                                                    cudaHostAllocPortable)
                       : cudaMalloc(&b.p, n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    b.p = nullptr;
    return nullptr;
  }
  b.n = n;
  b.host = host;
  return b.p;
}

void *dev_view(void *p, bool host) {
  if (!host)
    return p;
  void *d = nullptr;
  if (cudaHostGetDevicePointer(&d, p, 0) != cudaSuccess) {
    cudaGetLastError();
    return p;
  }
  return d;
}

// bytes spanned by `incount` objects (non-negative strides only)
int64_t span_of(const tempi_desc &d, int64_t incount) {
  int64_t hi = d.start + d.block;
  for (int k = 0; k < d.ndims; ++k)
    hi += (d.counts[k] - 1) * d.strides[k];
  hi += (incount - 1) * d.extent;
  return hi;
}

// an MPI datatype with d's layout relative to origin + start
int build_type(const tempi_desc &d, MPI_Datatype *out) {
  MPI_Datatype t;
  if (libmpi.Type_contiguous(int(d.block), MPI_BYTE, &t) != MPI_SUCCESS)
    return TEMPI_ERR_ARG;
  for (int k = 0; k < d.ndims; ++k) {
    MPI_Datatype n;
    if (libmpi.Type_create_hvector(int(d.counts[k]), 1, d.strides[k], t, &n) !=
        MPI_SUCCESS)
      return TEMPI_ERR_ARG;
    t = n;
  }
  MPI_Datatype r;
  if (libmpi.Type_create_resized(t, 0, d.extent, &r) != MPI_SUCCESS)
    return TEMPI_ERR_ARG;
  if (MPI_Type_commit(&r) != MPI_SUCCESS) // through TEMPI: canonicalised
    return TEMPI_ERR_ARG;
  *out = r;
  return TEMPI_OK;
}

} // namespace

void measure_release() {
  std::lock_guard<std::mutex> l(g_mu);
  for (Buf *b : {&g_typed[0], &g_typed[1], &g_typed2, &g_packed[0], &g_packed[1]}) {
    if (b->p)
      b->host ? cudaFreeHost(b->p) : cudaFree(b->p);
    *b = Buf{};
  }
}

int measure_candidates(const tempi_desc &d, int64_t incount, bool src_host,
                       bool dst_host, int what, int reps, float *times) {
  for (int j = 0; j < kMeasured; ++j)
    times[j] = NAN;
  if (d.size <= 0 || incount <= 0 || d.start < 0 || d.extent < 0)
    return set_error(TEMPI_ERR_ARG, "measure: empty or negative layout");
  for (int k = 0; k < d.ndims; ++k)
    if (d.strides[k] < 0)
      return set_error(TEMPI_ERR_ARG, "measure: negative stride");
  const int64_t span = span_of(d, incount), packed = d.size * incount;
  if (span > (int64_t(8) << 30) || packed > INT32_MAX)
    return set_error(TEMPI_ERR_ARG, "measure: object too large");
  reps = std::max(1, reps);
  std::lock_guard<std::mutex> l(g_mu);
  struct Guard {
    Guard() { set_measuring(true); }
    ~Guard() { set_measuring(false); }
  } guard;
  if (!g_stream &&
      cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking) != cudaSuccess)
    return cuda_error(cudaGetLastError(), "measure stream");
  void *typed = get(g_typed[src_host], size_t(span), src_host);
  void *pk = get(g_packed[dst_host], size_t(packed), dst_host);
  if (!typed || !pk)
    return set_error(TEMPI_ERR_NO_MEM, "measure: scratch allocation failed");
  char *t_dev = static_cast<char *>(dev_view(typed, src_host));
  char *p_dev = static_cast<char *>(dev_view(pk, dst_host));
  if (what & 1) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    // the fixed rules first, then every eligible candidate, packs and
    // unpacks timed apart.  The first timed pass doubles as the warm-up; a
    // candidate more than 3x slower than the best so far is not repeated
    // `reps` times but timed once more, keeping the faster of its two
    // passes (a first pass can carry one-off costs, such as the first
    // launch of a kernel variant).
    float best[2] = {INFINITY, INFINITY};
    auto pass = [&](const tempi_config *cfg, bool unpack, int n) -> float {
      cudaEventRecord(a, g_stream);
      for (int r = 0; r < n; ++r) {
        if (unpack)
          tempi_unpack(&d, p_dev, incount, t_dev, cfg, g_stream);
        else
          tempi_pack(&d, t_dev, incount, p_dev, cfg, g_stream);
      }
      cudaEventRecord(b, g_stream);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      return 1e3f * ms / n;
    };
    for (int i = 0; i <= kNumConfigs; ++i) {
      const int k = i == 0 ? -1 : i - 1; // -1: the fixed rules
      if (k >= 0 && !eligible(d, incount, k))
        continue;
      const tempi_config *cfg = k < 0 ? nullptr : &kCandidates[k];
      for (int u = 0; u < 2; ++u) {
        float t = pass(cfg, u == 1, 1);
        if (t <= 3 * best[u])
          t = pass(cfg, u == 1, reps);
        else
          t = std::min(t, pass(cfg, u == 1, 1));
        times[k < 0 ? (u ? kFixedUnpack : kFixedPack)
                    : (u ? kUnpackOut : kPackOut) + k] = t;
        best[u] = std::min(best[u], t);
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      return cuda_error(e, "measure configurations");
    if (staged_failed())
      return set_error(TEMPI_ERR_TIMEOUT,
                       "measure: a staged kernel gave up on its bulk copies");
  }
  if ((what & 2) && !src_host && incount <= INT32_MAX) {
    void *typed2 = get(g_typed2, size_t(span), false);
    if (!typed2)
      return set_error(TEMPI_ERR_NO_MEM, "measure: scratch allocation failed");
    MPI_Datatype t;
    int err = build_type(d, &t);
    if (err)
      return set_error(err, "measure: could not build the datatype");
    char *src = static_cast<char *>(typed) + d.start;
    char *dst = static_cast<char *>(typed2) + d.start;
    for (int m = 1; m <= kNumMethods && !err; ++m) {
      force_method(m);
      const int tag = 0x7e3a;
      for (int r = 0; r <= reps && !err; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        err = MPI_Send(src, int(incount), t, 0, tag, MPI_COMM_WORLD) ||
              MPI_Recv(dst, int(incount), t, 0, tag, MPI_COMM_WORLD,
                       MPI_STATUS_IGNORE);
        const double us = std::chrono::duration<double, std::micro>(
                              std::chrono::steady_clock::now() - t0)
                              .count();
        if (r == 1)
          times[kMethodOut + m - 1] = 0;
        if (r >= 1) // r == 0 is the warm-up
          times[kMethodOut + m - 1] += float(us / reps);
      }
    }
    force_method(-1);
    MPI_Type_free(&t);
    if (err)
      return set_error(TEMPI_ERR_ARG, "measure: self-send failed");
  }
  return TEMPI_OK;
}

} // namespace tempi

extern "C" int tempi_measure(const tempi_desc *d, int64_t incount, int src_host,
                             int dst_host, int what, int reps,
                             float *times_us) {
  if (!d || !times_us)
    return tempi::set_error(TEMPI_ERR_ARG, "null argument");
  return tempi::measure_candidates(*d, incount, src_host != 0, dst_host != 0,
                                   what, reps, times_us);
}
