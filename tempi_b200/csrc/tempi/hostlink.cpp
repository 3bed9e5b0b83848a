// Copy-engine path for a contiguous run between two pinned host buffers.
//
// When the typed and the packed buffer of an MPI_Pack / MPI_Unpack are both
// pinned host memory and the described bytes form one contiguous run, the
// pack is a host-to-host copy that must cross the host link twice.  A kernel
// that reads and writes host memory itself moves about 40 GB/s each way on a
// B200 behind PCIe 5.0 x16; the two copy engines, kept busy in opposite
// directions at once, move about 46 GB/s each way.  So the run is cut into
// chunks that go host -> device staging on the caller's stream and staging
// -> host on link_stream(), kStages chunks in flight.  The reference sends
// contiguous types to cudaMemcpyAsync the same way (Packer1D,
// src/internal/packer_1d.cu:16-50); strided runs stay on the kernels.
#include "runtime.hpp"

#include <algorithm>

namespace tempi {

namespace {
constexpr int kStages = 4;
constexpr size_t kMaxChunk = size_t(8) << 20;
constexpr size_t kMinChunk = size_t(1) << 20;
} // namespace

int64_t contiguous_run(const tempi_desc &d, int64_t incount) {
  Geometry g;
  bool empty = false;
  if (make_geometry(&d, incount, 0, 0, 16, &g, &empty) != TEMPI_OK)
    return -1; // the kernel path reports the descriptor's error
  if (empty)
    return 0;
  return g.nd == 0 ? g.block : -1;
}

int host_link_copy(void *dst, const void *src, size_t n, cudaStream_t s) {
  if (n == 0)
    return TEMPI_OK;
  cudaStream_t h = link_stream();
  if (!h)
    return set_error(TEMPI_ERR_CUDA, "host link: no helper stream");
  // at least 2 * kStages chunks so both directions overlap for most of it;
  // whole MiB, so every staging slot and chunk offset stays aligned
  const size_t want = (n / (2 * kStages) + kMinChunk - 1) / kMinChunk * kMinChunk;
  const size_t chunk = std::min(kMaxChunk, std::max(kMinChunk, want));
  char *stage = static_cast<char *>(slab_alloc(Space::DEVICE, kStages * chunk));
  if (!stage)
    return set_error(TEMPI_ERR_NO_MEM, "host link: staging allocation failed");
  cudaEvent_t start = event_acquire(), done = event_acquire();
  cudaEvent_t in[kStages], out[kStages];
  for (int k = 0; k < kStages; ++k) {
    in[k] = event_acquire();
    out[k] = event_acquire();
  }
  bool have_events = start && done;
  for (int k = 0; k < kStages; ++k)
    have_events = have_events && in[k] && out[k];
  const char *sp = static_cast<const char *>(src);
  char *dp = static_cast<char *>(dst);
  cudaError_t e = have_events ? cudaEventRecord(start, s)
                              : cudaErrorMemoryAllocation;
  if (e == cudaSuccess)
    e = cudaStreamWaitEvent(h, start, 0);
  const size_t nchunks = (n + chunk - 1) / chunk;
  for (size_t i = 0; i < nchunks && e == cudaSuccess; ++i) {
    const int k = int(i % kStages);
    const size_t off = i * chunk, len = std::min(chunk, n - off);
    char *slot = stage + size_t(k) * chunk;
    // slot k is free once its previous chunk has left for the host
    if (i >= size_t(kStages))
      e = cudaStreamWaitEvent(s, out[k], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(slot, sp + off, len, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaEventRecord(in[k], s);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(h, in[k], 0);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(dp + off, slot, len, cudaMemcpyDeviceToHost, h);
    if (e == cudaSuccess)
      e = cudaEventRecord(out[k], h);
  }
  if (e == cudaSuccess)
    e = cudaEventRecord(done, h);
  if (e == cudaSuccess)
    e = cudaStreamWaitEvent(s, done, 0);
  // whatever was enqueued must finish before the staging and events return
  // to their pools
  const cudaError_t es = cudaStreamSynchronize(s);
  const cudaError_t eh = cudaStreamSynchronize(h);
  if (e == cudaSuccess)
    e = es != cudaSuccess ? es : eh;
  for (int k = 0; k < kStages; ++k) {
    if (in[k])
      event_release(in[k]);
    if (out[k])
      event_release(out[k]);
  }
  if (start)
    event_release(start);
  if (done)
    event_release(done);
  slab_free(Space::DEVICE, stage);
  if (e != cudaSuccess)
    return cuda_error(e, "host link copy");
  counters().host_link_copies++;
  return TEMPI_OK;
}

} // namespace tempi
