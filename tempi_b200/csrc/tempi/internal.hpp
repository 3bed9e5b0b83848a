// Internal declarations shared by the host and device sources of
// libtempi_b200.so.  Nothing here is part of the public ABI.
#pragma once

#include "tempi_b200.h"

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>

namespace tempi {

// ---- logging ------------------------------------------------------------
// TEMPI_LOG_LEVEL: 0 silent (default), 1 errors, 2 warnings, 3 info, 4 debug
int log_level();
#define TEMPI_LOG(lvl, tag, ...)                                               \
  do {                                                                         \
    if (::tempi::log_level() >= (lvl)) {                                       \
      std::fprintf(stderr, "[tempi " tag "] " __VA_ARGS__);                    \
      std::fputc('\n', stderr);                                                \
    }                                                                          \
  } while (0)
#define LOG_ERROR(...) TEMPI_LOG(1, "error", __VA_ARGS__)
#define LOG_WARN(...) TEMPI_LOG(2, "warn", __VA_ARGS__)
#define LOG_INFO(...) TEMPI_LOG(3, "info", __VA_ARGS__)
#define LOG_DEBUG(...) TEMPI_LOG(4, "debug", __VA_ARGS__)

// record a message for tempi_last_error() and return `code`
int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);

// Copy n bytes and return only once they have landed.  A plain cudaMemcpy
// from pageable host memory (or between device buffers) can return before
// the copy is done, and work the caller then issues on a non-blocking stream
// is not ordered after it; this runs the copy on a private stream and waits.
cudaError_t copy_complete(void *dst, const void *src, size_t n);

// ---- counters (reference include/counters.hpp:14-115) ----------------------
struct Counters {
  std::atomic<int64_t> kernel_launches{0};
  std::atomic<int64_t> packs{0}, unpacks{0};
  std::atomic<int64_t> pack_bytes{0}, unpack_bytes{0};
  std::atomic<int64_t> lib_pack{0}, lib_unpack{0};
  std::atomic<int64_t> send_device{0}, send_oneshot{0}, send_staged{0},
      send_lib{0};
  std::atomic<int64_t> recv_device{0}, recv_oneshot{0}, recv_staged{0},
      recv_lib{0};
  std::atomic<int64_t> isend_managed{0}, irecv_managed{0};
  std::atomic<int64_t> dispatch_hit{0}, dispatch_miss{0}, dispatch_measured{0};
  std::atomic<int64_t> slab_hits{0}, slab_misses{0};
  // bytes held from CUDA (live + cached), handed out, kept for reuse
  std::atomic<int64_t> slab_bytes{0}, slab_live_bytes{0}, slab_cached_bytes{0};
  std::atomic<int64_t> cached_types{0};
  std::atomic<int64_t> host_link_copies{0};
  std::atomic<int64_t> send_contig_staged{0}, recv_contig_staged{0};
  std::atomic<int64_t> neighbor_fused{0}, neighbor_isir{0}, neighbor_lib{0};
  std::atomic<int64_t> alltoallv_staged{0}, alltoallv_remote_first{0},
      alltoallv_isir_staged{0}, alltoallv_isir_remote_staged{0}, alltoallv_lib{0};
};
Counters &counters();

// last kernel variant name, for tests and profiling
void set_last_kernel(const char *name);

// An NVTX range over a scope, as the reference marks its interposed calls
// (src/pack.cpp:37,66): visible in Nsight Systems, free when no tool is
// attached (NVTX3 is header-only and resolves its hooks lazily).
struct TraceRange {
  explicit TraceRange(const char *name) { nvtxRangePushA(name); }
  ~TraceRange() { nvtxRangePop(); }
  TraceRange(const TraceRange &) = delete;
  TraceRange &operator=(const TraceRange &) = delete;
};

// ---- launch geometry ------------------------------------------------------

constexpr int KDIMS = TEMPI_MAX_DIMS + 1; // strided dims plus the object count

// Exact division of n < 2^31 by an invariant d < 2^31 with one multiply-high
// and a shift: the round-up method of Granlund and Montgomery, "Division by
// invariant integers using multiplication" (PLDI 1994).  With
// l = ceil(log2 d) and m = ceil(2^(31+l) / d) < 2^32, floor(n/d) =
// floor(n*m / 2^(31+l)) for all n < 2^31, i.e. umulhi(n, m) >> (l-1).
struct FastDiv {
  uint32_t d, m, s;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f{d, 0, 0};
  if (d <= 1)
    return f;
  uint32_t l = 32 - __builtin_clz(d - 1);
  uint64_t m = ((uint64_t(1) << (31 + l)) + d - 1) / d;
  f.m = (uint32_t)m;
  f.s = l - 1;
  return f;
}

// A normalised launch: rows of `block` bytes; row r splits into digits over
// counts (fastest first); the strided side of row r starts at
// base + sum digit_k * strides[k]; the packed side at packed + r*block.
struct Geometry {
  int64_t strides[KDIMS];
  FastDiv cdiv[KDIMS];
  uint32_t nd;    // strided dims in use (0..KDIMS)
  uint32_t width; // bytes per vector word
  uint32_t wpr;   // words per row
  FastDiv wdiv;   // divides by wpr
  uint32_t rows;
  uint32_t total_words; // rows * wpr, < 2^31
  int64_t block;
};

// Build a normalised geometry for `incount` objects of `d` with the given
// base pointers.  Folds unit dims, merges dims that are contiguous with each
// other and proves the widest vector width.  Returns TEMPI_OK, or an error;
// sets *empty when there is nothing to copy.
int make_geometry(const tempi_desc *d, int64_t incount, uintptr_t strided_base,
                  uintptr_t packed_base, int max_width, Geometry *g,
                  bool *empty);

// Launch one pack (unpack=false) or unpack on `stream`.  both_device: 1 when
// the caller knows both buffers are device memory proper, 0 when it knows
// they are not, -1 to ask the runtime (only the staged kernels need it).
int launch_geometry(const Geometry &g, const char *strided_base, char *packed,
                    bool unpack, const tempi_config *cfg, cudaStream_t stream,
                    int both_device = -1);
// tempi_pack / tempi_unpack with the buffers' kind already known (see
// launch_geometry's both_device).
int pack_known(const tempi_desc *d, const void *origin, int64_t incount,
               void *packed, const tempi_config *cfg, cudaStream_t stream,
               int both_device);
int unpack_known(const tempi_desc *d, const void *packed, int64_t incount,
                 void *origin, const tempi_config *cfg, cudaStream_t stream,
                 int both_device);

int num_sms();
// Staged launches (kernel 4) that gave up waiting on a bulk copy, counted
// once the host has seen their failure word (0 unless something failed).
int64_t staged_timeouts();
// Allocate the staged kernels' failure word now (MPI_Init calls this with
// stream 0), unless `stream` is being captured; whether it exists.
bool staged_channel(cudaStream_t stream);
// After synchronising the stream of a staged launch: whether a staged kernel
// gave up since the last call (its output is then incomplete).  Clears the
// failure word.
bool staged_failed();

// The copy batch's kernel (tempi_batch_create_copy) for one call, with its
// pair table in a grow-only device buffer; launches on `s`, which the caller
// synchronises before calling again.
int copy_batch_run(const tempi_copy_region *regions, int32_t n,
                   cudaStream_t s);

} // namespace tempi
