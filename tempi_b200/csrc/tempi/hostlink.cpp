// Copy-engine paths between two pinned host buffers.
//
// When the typed and the packed buffer of an MPI_Pack / MPI_Unpack are both
// pinned host memory, every described byte must cross the host link twice.
// A kernel that reads and writes host memory itself moves about 40 GB/s each
// way on a B200 behind PCIe 5.0 x16 for long runs, and far less for short
// rows: its reads of host memory go out per instruction, and a 64-B row at
// an odd offset costs several requests (about 13 GB/s measured).  The two
// copy engines, kept busy in opposite directions at once, move about 46 GB/s
// each way for long runs, and a lone 2-D copy moves rows of 64 B and more at
// 24-55 GB/s (one request per row: 2.3 ns per row below 128 B).  So
//  * a contiguous run (host_link_copy) is cut into chunks, and
//  * rows of one strided dimension (host_link_rows) into chunks of rows,
// that go host -> device staging on the caller's stream and staging -> host
// on link_stream(), kStages chunks in flight; the strided side of each chunk
// is one 2-D copy.  The reference sends contiguous types to cudaMemcpyAsync
// the same way (Packer1D, src/internal/packer_1d.cu:16-50); layouts with two
// or more strided dimensions, or rows under kHostLinkMinRow, stay on the
// kernels.
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

// The staged pipeline: chunk i (of `nchunks`, at most `slot` bytes each)
// goes in by in(i, slot_ptr, stream) and out by out(i, slot_ptr, stream).
template <typename In, typename Out>
static int pipeline(size_t nchunks, size_t slot, cudaStream_t s, In in_copy,
                    Out out_copy) {
  cudaStream_t h = link_stream();
  if (!h)
    return set_error(TEMPI_ERR_CUDA, "host link: no helper stream");
  char *stage = static_cast<char *>(slab_alloc(Space::DEVICE, kStages * slot));
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
  cudaError_t e = have_events ? cudaEventRecord(start, s)
                              : cudaErrorMemoryAllocation;
  if (e == cudaSuccess)
    e = cudaStreamWaitEvent(h, start, 0);
  for (size_t i = 0; i < nchunks && e == cudaSuccess; ++i) {
    const int k = int(i % kStages);
    char *sl = stage + size_t(k) * slot;
    // slot k is free once its previous chunk has left for the host
    if (i >= size_t(kStages))
      e = cudaStreamWaitEvent(s, out[k], 0);
    if (e == cudaSuccess)
      e = in_copy(i, sl, s);
    if (e == cudaSuccess)
      e = cudaEventRecord(in[k], s);
    if (e == cudaSuccess)
      e = cudaStreamWaitEvent(h, in[k], 0);
    if (e == cudaSuccess)
      e = out_copy(i, sl, h);
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

int host_link_copy(void *dst, const void *src, size_t n, cudaStream_t s) {
  if (n == 0)
    return TEMPI_OK;
  // at least 2 * kStages chunks so both directions overlap for most of it;
  // whole MiB, so every staging slot and chunk offset stays aligned
  const size_t want = (n / (2 * kStages) + kMinChunk - 1) / kMinChunk * kMinChunk;
  const size_t chunk = env().host_link_chunk_kb > 0
                           ? size_t(env().host_link_chunk_kb) << 10
                           : std::min(kMaxChunk, std::max(kMinChunk, want));
  const char *sp = static_cast<const char *>(src);
  char *dp = static_cast<char *>(dst);
  return pipeline(
      (n + chunk - 1) / chunk, chunk, s,
      [&](size_t i, char *slot, cudaStream_t st) {
        const size_t off = i * chunk, len = std::min(chunk, n - off);
        return cudaMemcpyAsync(slot, sp + off, len, cudaMemcpyHostToDevice, st);
      },
      [&](size_t i, char *slot, cudaStream_t st) {
        const size_t off = i * chunk, len = std::min(chunk, n - off);
        return cudaMemcpyAsync(dp + off, slot, len, cudaMemcpyDeviceToHost, st);
      });
}

bool host_rows(const tempi_desc &d, int64_t incount, HostRows *out) {
  Geometry g;
  bool empty = false;
  if (make_geometry(&d, incount, 0, 0, 16, &g, &empty) != TEMPI_OK || empty ||
      g.nd != 1)
    return false;
  if (g.block < kHostLinkMinRow || g.block > int64_t(kMaxChunk) ||
      g.strides[0] < g.block)
    return false;
  out->rows = g.rows;
  out->width = g.block;
  out->pitch = g.strides[0];
  return true;
}

int host_link_rows(void *dst, int64_t dpitch, const void *src, int64_t spitch,
                   int64_t width, int64_t rows, cudaStream_t s) {
  if (rows <= 0 || width <= 0)
    return TEMPI_OK;
  if (width > int64_t(kMaxChunk) || dpitch < width || spitch < width)
    return set_error(TEMPI_ERR_ARG, "host link rows: bad shape");
  // rows per chunk: about 2 * kStages chunks, each at most kMaxChunk bytes
  const int64_t per = std::max<int64_t>(
      1, std::min<int64_t>(int64_t(kMaxChunk) / width,
                           (rows + 2 * kStages - 1) / (2 * kStages)));
  const char *sp = static_cast<const char *>(src);
  char *dp = static_cast<char *>(dst);
  const size_t w = size_t(width);
  return pipeline(
      size_t((rows + per - 1) / per), size_t(per * width), s,
      [&](size_t i, char *slot, cudaStream_t st) {
        const int64_t r0 = int64_t(i) * per, n = std::min(per, rows - r0);
        return cudaMemcpy2DAsync(slot, w, sp + r0 * spitch, size_t(spitch), w,
                                 size_t(n), cudaMemcpyHostToDevice, st);
      },
      [&](size_t i, char *slot, cudaStream_t st) {
        const int64_t r0 = int64_t(i) * per, n = std::min(per, rows - r0);
        return cudaMemcpy2DAsync(dp + r0 * dpitch, size_t(dpitch), slot, w, w,
                                 size_t(n), cudaMemcpyDeviceToHost, st);
      });
}

} // namespace tempi
