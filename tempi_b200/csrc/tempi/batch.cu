// Batched pack/unpack: every region of a step in one launch.
//
// The reference packs one object per MPI_Pack call, each with its own launch
// and stream synchronisation (src/pack.cpp:56, packer_2d.cu:101-109), so the
// 26 halo regions of a 3-D grid cost 26 launches and 26 synchronisations.
// Here the regions become a table in device memory; one grid-stride kernel
// walks it.  The work is cut into equal chunks of kChunkWords words (one
// chunk per CTA iteration); a region owns a contiguous range of chunks, found
// by binary search over the table's prefix offsets.  Each region keeps its
// own geometry and proven vector width, so a 16-B-row face and a 2-KiB-row
// face run at their own best width inside the same launch.
//
// A batch can capture one launch into a CUDA graph and replay it; because
// the pointers live in the table, replays see new buffer contents without
// re-capture.
//
// A copy batch (tempi_batch_create_copy) fuses pack, transfer and unpack:
// each entry pairs a source layout with a destination layout of the same
// byte count, and word w of the entry is read at the source geometry's
// offset of w and written at the destination geometry's offset of w.  Both
// geometries are built at the same proven width, so one word index walks
// both.

#include "internal.hpp"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

namespace tempi {

namespace {

constexpr int kBatchThreads = 256;
constexpr int kBatchUnroll = 4;
constexpr uint32_t kChunkWords = kBatchThreads * kBatchUnroll;

struct BatchRegion {
  char *strided; // origin + start
  char *packed;
  Geometry g;
  uint32_t chunk_begin; // first chunk of this region
  uint32_t pad;
};

__device__ __forceinline__ uint32_t bdiv(uint32_t n, const FastDiv &f) {
  return f.m ? (__umulhi(n, f.m) >> f.s) : n;
}

__device__ __forceinline__ int64_t brow_offset(uint32_t row, const Geometry &g) {
  int64_t off = 0;
#pragma unroll
  for (int k = 0; k < KDIMS; ++k) {
    if (k >= int(g.nd))
      break;
    if (k == int(g.nd) - 1) {
      off += int64_t(row) * g.strides[k];
    } else {
      const uint32_t q = bdiv(row, g.cdiv[k]);
      off += int64_t(row - q * g.cdiv[k].d) * g.strides[k];
      row = q;
    }
  }
  return off;
}

template <int W>
__device__ __forceinline__ void copy_chunk(const BatchRegion &r, uint32_t w0,
                                           bool unpack) {
  using T = typename std::conditional<
      W == 16, uint4,
      typename std::conditional<
          W == 8, uint2,
          typename std::conditional<
              W == 4, uint32_t,
              typename std::conditional<W == 2, uint16_t,
                                        uint8_t>::type>::type>::type>::type;
  const Geometry &g = r.g;
  const uint32_t total = g.total_words;
  int64_t so[kBatchUnroll];
  uint32_t ww[kBatchUnroll];
#pragma unroll
  for (int u = 0; u < kBatchUnroll; ++u) {
    ww[u] = w0 + threadIdx.x + u * kBatchThreads;
    if (ww[u] < total) {
      const uint32_t row = bdiv(ww[u], g.wdiv);
      so[u] = brow_offset(row, g) + int64_t(ww[u] - row * g.wpr) * W;
    }
  }
  T v[kBatchUnroll];
  if (!unpack) {
#pragma unroll
    for (int u = 0; u < kBatchUnroll; ++u)
      if (ww[u] < total)
        v[u] = __ldg(reinterpret_cast<const T *>(r.strided + so[u]));
#pragma unroll
    for (int u = 0; u < kBatchUnroll; ++u)
      if (ww[u] < total)
        reinterpret_cast<T *>(r.packed)[ww[u]] = v[u];
  } else {
#pragma unroll
    for (int u = 0; u < kBatchUnroll; ++u)
      if (ww[u] < total)
        v[u] = __ldg(reinterpret_cast<const T *>(r.packed) + ww[u]);
#pragma unroll
    for (int u = 0; u < kBatchUnroll; ++u)
      if (ww[u] < total)
        *reinterpret_cast<T *>(r.strided + so[u]) = v[u];
  }
}

// Index of the last region whose first chunk is <= chunk, found by warp 0:
// each round the lanes sample 32 evenly spaced entries of the remaining
// stretch with one coalesced load and a ballot narrows it 32-fold, so n
// regions take ceil(log32 n) dependent loads (one for a 26-region halo, two
// for up to 1024 regions) instead of a binary search's log2 n.
template <typename Rec>
__device__ __forceinline__ int find_region(const Rec *__restrict__ r, int n,
                                           uint32_t chunk, uint32_t lane) {
  int base = 0, len = n;
  while (true) {
    const int step = (len + 31) / 32;
    const int off = int(lane) * step;
    const bool le = off < len && r[base + off].chunk_begin <= chunk;
    const unsigned m = __ballot_sync(0xffffffffu, le);
    const int seg = 31 - __clz(m); // the stretch's first entry always qualifies
    base += seg * step;
    if (step == 1)
      return base;
    len = min(step, len - seg * step);
  }
}

__global__ void __launch_bounds__(kBatchThreads, 3)
    k_batch(const BatchRegion *__restrict__ regions, int nregions,
            uint32_t total_chunks, int unpack) {
  __shared__ BatchRegion sr;
  __shared__ int cur;
  const uint32_t lane = threadIdx.x & 31;
  if (threadIdx.x == 0)
    cur = -1;
  __syncthreads();
  for (uint32_t chunk = blockIdx.x; chunk < total_chunks; chunk += gridDim.x) {
    if (threadIdx.x < 32) {
      const int idx = find_region(regions, nregions, chunk, lane);
      if (idx != cur) { // the warp copies the record, a word per lane
        constexpr int kWords = sizeof(BatchRegion) / 4;
        const uint32_t *from = reinterpret_cast<const uint32_t *>(regions + idx);
        uint32_t *to = reinterpret_cast<uint32_t *>(&sr);
        for (int w = lane; w < kWords; w += 32)
          to[w] = from[w];
        __syncwarp();
        if (lane == 0)
          cur = idx;
      }
    }
    __syncthreads();
    const uint32_t w0 = (chunk - sr.chunk_begin) * kChunkWords;
    switch (sr.g.width) {
    case 16: copy_chunk<16>(sr, w0, unpack); break;
    case 8: copy_chunk<8>(sr, w0, unpack); break;
    case 4: copy_chunk<4>(sr, w0, unpack); break;
    case 2: copy_chunk<2>(sr, w0, unpack); break;
    default: copy_chunk<1>(sr, w0, unpack); break;
    }
    __syncthreads();
  }
}

struct CopyPair {
  const char *src; // src origin + start
  char *dst;       // dst origin + start
  Geometry gs, gd; // same width and word count
  uint32_t chunk_begin;
  uint32_t pad;
};

template <int W>
__device__ __forceinline__ void copy_pair_chunk(const CopyPair &r, uint32_t w0) {
  using T = typename std::conditional<
      W == 16, uint4,
      typename std::conditional<
          W == 8, uint2,
          typename std::conditional<
              W == 4, uint32_t,
              typename std::conditional<W == 2, uint16_t,
                                        uint8_t>::type>::type>::type>::type;
  const uint32_t total = r.gs.total_words;
  // each load is issued as soon as its source offset is known; only the
  // destination offsets and the loaded words stay live until the stores
  int64_t dof[kBatchUnroll];
  T v[kBatchUnroll];
#pragma unroll
  for (int u = 0; u < kBatchUnroll; ++u) {
    const uint32_t ww = w0 + threadIdx.x + u * kBatchThreads;
    if (ww < total) {
      const uint32_t rs = bdiv(ww, r.gs.wdiv);
      v[u] = __ldg(reinterpret_cast<const T *>(
          r.src + brow_offset(rs, r.gs) + int64_t(ww - rs * r.gs.wpr) * W));
      const uint32_t rd = bdiv(ww, r.gd.wdiv);
      dof[u] = brow_offset(rd, r.gd) + int64_t(ww - rd * r.gd.wpr) * W;
    }
  }
#pragma unroll
  for (int u = 0; u < kBatchUnroll; ++u)
    if (w0 + threadIdx.x + u * kBatchThreads < total)
      *reinterpret_cast<T *>(r.dst + dof[u]) = v[u];
}

__global__ void __launch_bounds__(kBatchThreads, 3)
    k_batch_copy(const CopyPair *__restrict__ pairs, int npairs,
                 uint32_t total_chunks) {
  __shared__ CopyPair sp;
  __shared__ int cur;
  const uint32_t lane = threadIdx.x & 31;
  if (threadIdx.x == 0)
    cur = -1;
  __syncthreads();
  for (uint32_t chunk = blockIdx.x; chunk < total_chunks; chunk += gridDim.x) {
    if (threadIdx.x < 32) {
      const int idx = find_region(pairs, npairs, chunk, lane);
      if (idx != cur) {
        constexpr int kWords = sizeof(CopyPair) / 4;
        const uint32_t *from = reinterpret_cast<const uint32_t *>(pairs + idx);
        uint32_t *to = reinterpret_cast<uint32_t *>(&sp);
        for (int w = lane; w < kWords; w += 32)
          to[w] = from[w];
        __syncwarp();
        if (lane == 0)
          cur = idx;
      }
    }
    __syncthreads();
    const uint32_t w0 = (chunk - sp.chunk_begin) * kChunkWords;
    switch (sp.gs.width) {
    case 16: copy_pair_chunk<16>(sp, w0); break;
    case 8: copy_pair_chunk<8>(sp, w0); break;
    case 4: copy_pair_chunk<4>(sp, w0); break;
    case 2: copy_pair_chunk<2>(sp, w0); break;
    default: copy_pair_chunk<1>(sp, w0); break;
    }
    __syncthreads();
  }
}

} // namespace

struct BatchImpl {
  std::vector<BatchRegion> host;
  BatchRegion *dev = nullptr;
  std::vector<CopyPair> host_pairs; // a copy batch
  CopyPair *dev_pairs = nullptr;
  uint32_t total_chunks = 0;
  int unpack = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

} // namespace tempi

struct tempi_batch {
  tempi::BatchImpl impl;
};

using namespace tempi;

extern "C" int tempi_batch_create(const tempi_region *regions, int32_t n,
                                  int32_t unpack, tempi_batch **out) {
  if (!out || n < 0 || (n > 0 && !regions))
    return set_error(TEMPI_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  auto *b = new tempi_batch();
  b->impl.unpack = unpack ? 1 : 0;
  uint64_t chunks = 0;
  for (int32_t i = 0; i < n; ++i) {
    const tempi_region &r = regions[i];
    BatchRegion br{};
    char *strided = (char *)r.origin + r.desc.start;
    bool empty = false;
    int err = make_geometry(&r.desc, r.incount, uintptr_t(strided),
                            uintptr_t(r.packed), 0, &br.g, &empty);
    if (err) {
      delete b;
      return err;
    }
    if (empty)
      continue;
    br.strided = strided;
    br.packed = (char *)r.packed;
    br.chunk_begin = uint32_t(chunks);
    chunks += (br.g.total_words + kChunkWords - 1) / kChunkWords;
    if (chunks > UINT32_MAX) {
      delete b;
      return set_error(TEMPI_ERR_ARG, "batch too large");
    }
    b->impl.host.push_back(br);
  }
  b->impl.total_chunks = uint32_t(chunks);
  if (!b->impl.host.empty()) {
    const size_t bytes = b->impl.host.size() * sizeof(BatchRegion);
    cudaError_t e = cudaMalloc(&b->impl.dev, bytes);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->impl.dev, b->impl.host.data(), bytes,
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(b->impl.dev);
      delete b;
      return cuda_error(e, "batch table upload");
    }
  }
  *out = b;
  return TEMPI_OK;
}

static int batch_launch(tempi_batch *b, cudaStream_t s) {
  BatchImpl &bi = b->impl;
  if (!bi.host_pairs.empty()) {
    const uint32_t grid = std::max<uint32_t>(
        1, std::min<uint32_t>(bi.total_chunks, num_sms() * 8));
    k_batch_copy<<<grid, kBatchThreads, 0, s>>>(
        bi.dev_pairs, int(bi.host_pairs.size()), bi.total_chunks);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      return cuda_error(e, "copy batch launch");
    counters().kernel_launches++;
    set_last_kernel("batch_copy");
    return TEMPI_OK;
  }
  if (bi.host.empty())
    return TEMPI_OK;
  const int sms = num_sms();
  const uint32_t grid =
      std::max<uint32_t>(1, std::min<uint32_t>(bi.total_chunks, sms * 8));
  k_batch<<<grid, kBatchThreads, 0, s>>>(bi.dev, int(bi.host.size()),
                                        bi.total_chunks, bi.unpack);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "batch launch");
  counters().kernel_launches++;
  set_last_kernel(bi.unpack ? "batch_unpack" : "batch_pack");
  return TEMPI_OK;
}

// Copy pairs for `regions`; empty regions are dropped.  Returns the chunk
// count through *chunks_out.
static int build_pairs(const tempi_copy_region *regions, int32_t n,
                       std::vector<CopyPair> *pairs, uint32_t *chunks_out) {
  uint64_t chunks = 0;
  pairs->clear();
  for (int32_t i = 0; i < n; ++i) {
    const tempi_copy_region &r = regions[i];
    if (r.src_count < 0 || r.dst_count < 0 ||
        r.src_desc.size * r.src_count != r.dst_desc.size * r.dst_count) {
      return set_error(TEMPI_ERR_ARG,
                       "copy region %d: source and destination sizes differ",
                       int(i));
    }
    const char *src = (const char *)r.src_origin + r.src_desc.start;
    char *dst = (char *)r.dst_origin + r.dst_desc.start;
    CopyPair cp{};
    bool es = false, ed = false;
    // the widest width both layouts prove, then both geometries at it
    int err = make_geometry(&r.src_desc, r.src_count, uintptr_t(src), 0, 0,
                            &cp.gs, &es);
    if (!err)
      err = make_geometry(&r.dst_desc, r.dst_count, uintptr_t(dst), 0, 0,
                          &cp.gd, &ed);
    if (!err && !es && !ed) {
      const int w = int(std::min(cp.gs.width, cp.gd.width));
      err = make_geometry(&r.src_desc, r.src_count, uintptr_t(src), 0, w,
                          &cp.gs, &es);
      if (!err)
        err = make_geometry(&r.dst_desc, r.dst_count, uintptr_t(dst), 0, w,
                            &cp.gd, &ed);
    }
    if (err)
      return err;
    if (es || ed)
      continue; // nothing to copy
    if (cp.gs.width != cp.gd.width || cp.gs.total_words != cp.gd.total_words)
      return set_error(TEMPI_ERR_ARG, "copy region %d: layouts disagree",
                       int(i));
    cp.src = src;
    cp.dst = dst;
    cp.chunk_begin = uint32_t(chunks);
    chunks += (cp.gs.total_words + kChunkWords - 1) / kChunkWords;
    if (chunks > UINT32_MAX)
      return set_error(TEMPI_ERR_ARG, "batch too large");
    pairs->push_back(cp);
  }
  *chunks_out = uint32_t(chunks);
  return TEMPI_OK;
}

extern "C" int tempi_batch_create_copy(const tempi_copy_region *regions,
                                       int32_t n, tempi_batch **out) {
  if (!out || n < 0 || (n > 0 && !regions))
    return set_error(TEMPI_ERR_ARG, "bad copy batch arguments");
  *out = nullptr;
  auto *b = new tempi_batch();
  int err = build_pairs(regions, n, &b->impl.host_pairs, &b->impl.total_chunks);
  if (err) {
    delete b;
    return err;
  }
  if (!b->impl.host_pairs.empty()) {
    const size_t bytes = b->impl.host_pairs.size() * sizeof(CopyPair);
    cudaError_t e = cudaMalloc(&b->impl.dev_pairs, bytes);
    if (e == cudaSuccess)
      e = cudaMemcpy(b->impl.dev_pairs, b->impl.host_pairs.data(), bytes,
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      cudaFree(b->impl.dev_pairs);
      delete b;
      return cuda_error(e, "copy batch table upload");
    }
  }
  *out = b;
  return TEMPI_OK;
}

namespace tempi {

// One copy batch on `s` with the pair table in a grow-only device buffer:
// no allocation once the buffer is large enough.  The caller synchronises
// `s` before the next call (the table is rewritten by every call).
int copy_batch_run(const tempi_copy_region *regions, int32_t n,
                   cudaStream_t s) {
  static std::mutex mu;
  static CopyPair *table = nullptr;
  static size_t capacity = 0;
  static std::vector<CopyPair> pairs, on_device;
  std::lock_guard<std::mutex> l(mu);
  uint32_t chunks = 0;
  int err = build_pairs(regions, n, &pairs, &chunks);
  if (err || pairs.empty())
    return err;
  if (pairs.size() > capacity) {
    cudaFree(table);
    table = nullptr;
    capacity = 0;
    on_device.clear();
    const size_t want = std::max<size_t>(pairs.size(), 64);
    cudaError_t e = cudaMalloc(&table, want * sizeof(CopyPair));
    if (e != cudaSuccess)
      return cuda_error(e, "copy table allocation");
    capacity = want;
  }
  // a loop that exchanges the same regions every step uploads its table once
  const size_t bytes = pairs.size() * sizeof(CopyPair);
  if (on_device.size() != pairs.size() ||
      std::memcmp(on_device.data(), pairs.data(), bytes) != 0) {
    on_device.clear();
    cudaError_t e = cudaMemcpyAsync(table, pairs.data(), bytes,
                                    cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
      return cuda_error(e, "copy table upload");
    on_device = pairs;
  }
  cudaError_t e;
  const uint32_t grid =
      std::max<uint32_t>(1, std::min<uint32_t>(chunks, num_sms() * 8));
  k_batch_copy<<<grid, kBatchThreads, 0, s>>>(table, int(pairs.size()), chunks);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "copy batch launch");
  counters().kernel_launches++;
  set_last_kernel("batch_copy");
  return TEMPI_OK;
}

} // namespace tempi

extern "C" int tempi_batch_launch(tempi_batch *b, void *stream) {
  if (!b)
    return set_error(TEMPI_ERR_ARG, "null batch");
  return batch_launch(b, static_cast<cudaStream_t>(stream));
}

extern "C" int tempi_batch_capture(tempi_batch *b, void *stream) {
  if (!b)
    return set_error(TEMPI_ERR_ARG, "null batch");
  BatchImpl &bi = b->impl;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (bi.exec) {
    cudaGraphExecDestroy(bi.exec);
    cudaGraphDestroy(bi.graph);
    bi.exec = nullptr;
    bi.graph = nullptr;
  }
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return cuda_error(e, "begin capture");
  int err = batch_launch(b, s);
  e = cudaStreamEndCapture(s, &bi.graph);
  if (err)
    return err;
  if (e != cudaSuccess)
    return cuda_error(e, "end capture");
  e = cudaGraphInstantiate(&bi.exec, bi.graph, 0);
  if (e != cudaSuccess)
    return cuda_error(e, "graph instantiate");
  return TEMPI_OK;
}

extern "C" int tempi_batch_replay(tempi_batch *b, void *stream) {
  if (!b || !b->impl.exec)
    return set_error(TEMPI_ERR_ARG, "batch has no captured graph");
  cudaError_t e = cudaGraphLaunch(b->impl.exec, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return cuda_error(e, "graph launch");
  if (!b->impl.host.empty() || !b->impl.host_pairs.empty())
    counters().kernel_launches++;
  return TEMPI_OK;
}

// ---- batched pack without allocation ------------------------------------
//
// tempi_batch_create puts the region table in memory it obtains with
// cudaMalloc.  Some callers cannot allocate device memory where they pack:
// a halo-exchange step inside a latency-critical loop (cudaMalloc can
// synchronise the whole device), or an application whose memory pool
// already owns the GPU's memory, so any further cudaMalloc fails.  For them
// tempi_batch_run_static keeps the table in the fixed array below instead.
//
// The array is a file-scope device variable: every GPU that loads this
// library holds it (kStaticBatchRegions = 1024 entries of 168 B: 168 KiB) until the
// process exits.  Host code cannot use the name `g_static_regions` as a
// device address (it denotes a host-side stand-in), so the first call on
// each device, with that device current, asks the runtime for the array's
// device address once (cudaGetSymbolAddress) and every call passes that
// address to the kernel.  Because of that set-up, the first call on a
// device should come before any stream capture.  The cached address is not
// refreshed if the application resets the device (cudaDeviceReset).
//
// The table reaches the array without a host-to-device copy: the host
// builds it in pieces of up to kFillPiece entries and passes each piece BY
// VALUE as the parameter of a small kernel (k_static_fill) that writes it
// into the array, on the caller's stream ahead of the batch kernel.  Kernel
// parameters are copied when the launch is issued, so the host's piece can
// be reused at once, and the host never waits for earlier work on the
// stream (a copy from pageable host memory would).  All calls share the one
// array and it keeps the last call's table; each call rewrites every entry
// it uses, so nothing needs clearing, but calls whose launches can overlap
// on the GPU (different streams, no ordering) race on the table.
constexpr int kStaticBatchRegions = 1024;
constexpr int kMaxDevices = 64;
constexpr int kFillPiece = 128; // 21.5 KB of parameters (the limit is 32,764 B)

static_assert(sizeof(BatchRegion) == 168 && sizeof(BatchRegion) % 4 == 0,
              "table entry size is documented");
static __device__ __align__(256) BatchRegion g_static_regions[kStaticBatchRegions];

template <int P> struct StaticPiece {
  BatchRegion r[P];
};
static_assert(sizeof(StaticPiece<kFillPiece>) + 8 <= 32764,
              "a piece fits the kernel parameter space");

// entries [first, first + count) of the array from the piece, a 32-bit
// word per thread; the host guarantees first + count <= kStaticBatchRegions
// and count <= P
template <int P>
__global__ void __launch_bounds__(256)
    k_static_fill(const __grid_constant__ StaticPiece<P> piece, int first,
                  int count) {
  constexpr int kWords = sizeof(BatchRegion) / 4;
  const uint32_t *from = reinterpret_cast<const uint32_t *>(piece.r);
  uint32_t *to = reinterpret_cast<uint32_t *>(g_static_regions + first);
  for (int w = threadIdx.x; w < count * kWords; w += blockDim.x)
    to[w] = from[w];
}

static std::mutex g_static_mu;
static BatchRegion *g_static_ptr[kMaxDevices] = {};

static int static_table(BatchRegion **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return cuda_error(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(TEMPI_ERR_ARG, "device %d out of range", dev);
  std::lock_guard<std::mutex> l(g_static_mu);
  if (!g_static_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_regions);
    if (e != cudaSuccess)
      return cuda_error(e, "cudaGetSymbolAddress of the static region table");
    g_static_ptr[dev] = static_cast<BatchRegion *>(p);
  }
  *out = g_static_ptr[dev];
  return TEMPI_OK;
}

// launch k_static_fill for entries [first, first + count) of `piece`
static int static_fill(const StaticPiece<kFillPiece> &piece, int first,
                       int count, cudaStream_t s) {
  if (count <= 32) { // a small table: a 5.4 KB parameter block
    StaticPiece<32> small;
    std::memcpy(small.r, piece.r, size_t(count) * sizeof(BatchRegion));
    k_static_fill<32><<<1, 256, 0, s>>>(small, first, count);
  } else {
    k_static_fill<kFillPiece><<<1, 256, 0, s>>>(piece, first, count);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "static region table fill");
  counters().kernel_launches++;
  return TEMPI_OK;
}

extern "C" int tempi_batch_run_static(const tempi_region *regions, int32_t n,
                                      int32_t unpack, void *stream) {
  if (n < 0 || (n > 0 && !regions))
    return set_error(TEMPI_ERR_ARG, "bad batch arguments");
  if (n > kStaticBatchRegions)
    return set_error(TEMPI_ERR_ARG,
                     "tempi_batch_run_static takes at most %d regions, got %d",
                     kStaticBatchRegions, n);
  BatchRegion *table = nullptr;
  int err = static_table(&table);
  if (err)
    return err;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // every region is checked before anything is launched, so a bad region
  // leaves the array and the stream untouched
  StaticPiece<kFillPiece> piece;
  int used = 0, filled = 0;
  uint64_t chunks = 0;
  for (int pass = 0; pass < 2; ++pass) {
    used = filled = 0;
    chunks = 0;
    for (int32_t i = 0; i < n; ++i) {
      const tempi_region &r = regions[i];
      BatchRegion &br = piece.r[filled];
      br = BatchRegion{};
      char *strided = (char *)r.origin + r.desc.start;
      bool empty = false;
      err = make_geometry(&r.desc, r.incount, uintptr_t(strided),
                          uintptr_t(r.packed), 0, &br.g, &empty);
      if (err)
        return err;
      if (empty)
        continue;
      br.strided = strided;
      br.packed = (char *)r.packed;
      br.chunk_begin = uint32_t(chunks);
      chunks += (br.g.total_words + kChunkWords - 1) / kChunkWords;
      if (chunks > UINT32_MAX)
        return set_error(TEMPI_ERR_ARG, "batch too large");
      if (++filled == kFillPiece) {
        if (pass == 1 && (err = static_fill(piece, used, filled, s)))
          return err;
        used += filled;
        filled = 0;
      }
    }
    if (filled) { // a partial last piece (empty regions are never stored)
      if (pass == 1 && (err = static_fill(piece, used, filled, s)))
        return err;
      used += filled;
      filled = 0;
    }
  }
  if (used == 0)
    return TEMPI_OK;
  const uint32_t total = uint32_t(chunks);
  const uint32_t grid =
      std::max<uint32_t>(1, std::min<uint32_t>(total, num_sms() * 8));
  k_batch<<<grid, kBatchThreads, 0, s>>>(table, used, total, unpack ? 1 : 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "static batch launch");
  counters().kernel_launches++;
  set_last_kernel(unpack ? "batch_unpack_static" : "batch_pack_static");
  return TEMPI_OK;
}

extern "C" int tempi_batch_destroy(tempi_batch *b) {
  if (!b)
    return TEMPI_OK;
  if (b->impl.exec)
    cudaGraphExecDestroy(b->impl.exec);
  if (b->impl.graph)
    cudaGraphDestroy(b->impl.graph);
  cudaFree(b->impl.dev);
  cudaFree(b->impl.dev_pairs);
  delete b;
  return TEMPI_OK;
}
