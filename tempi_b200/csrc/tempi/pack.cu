// Strided pack / unpack kernels for sm_100a.
//
// What they compute is the reference packers' job (pack_2d/unpack_2d,
// include/pack_kernels.cuh:64-120; pack_3d/unpack_3d, :350-433; Packer1D's
// cudaMemcpyAsync, src/internal/packer_1d.cu:16-50): copy the described bytes
// of `incount` objects, in type-map order, to or from a contiguous buffer.
//
// How is this library's own design:
//  * one launch covers every object: the object count is just the slowest
//    strided dimension (stride = extent), and dimensions that are contiguous
//    with each other are merged on the host first (make_geometry);
//  * offsets are 64-bit; rows and words are 32-bit indices (packed sizes are
//    bounded by MPI's int counts), decomposed with exact multiply-high
//    division (FastDiv) instead of hardware division;
//  * the vector width is the widest power of two (up to 16 B) that divides
//    the block length, every stride and BOTH runtime base pointers, so every
//    access is naturally aligned (the reference checks only block length and
//    start offset, pack_kernels.cuh:129-157, and never uses 16-B words);
//  * k_words: one thread per output word, U independent loads in flight per
//    thread; packed-side accesses are contiguous across a warp.  Used for
//    short rows, where a warp spans many rows.
//  * k_rows: one warp per row, lanes stride across the row's words, U loads
//    in flight per lane; the row offset is computed once per row.  Used for
//    wide rows.
//  * k_rows_shift: a group of lanes per row, 16-B words realigned by funnel
//    shifts, for rows whose two sides disagree modulo 16.
//  * k_unpack_staged: 8 KB chunks of the packed stream move into shared
//    memory by bulk asynchronous copies counted on mbarriers (bounded
//    waits), and are scattered to the rows by plain vector stores.
//  * k_staged_bulk: the staged pack, and the staged unpack of wide 16-B
//    aligned rows: one warp per CTA moves 16 KB chunks through shared memory
//    with bulk copies in both directions (row pieces on the strided side,
//    one copy on the packed side).
//  * grids are a multiple of the SM count and grid-stride over the work.

#include "internal.hpp"
#include "runtime.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <set>
#include <utility>

namespace tempi {

template <int W> struct Word;
template <> struct Word<1> { using T = uint8_t; };
template <> struct Word<2> { using T = uint16_t; };
template <> struct Word<4> { using T = uint32_t; };
template <> struct Word<8> { using T = uint2; };
template <> struct Word<16> { using T = uint4; };

__device__ __forceinline__ uint32_t fastdiv(uint32_t n, const FastDiv &f) {
  return f.m ? (__umulhi(n, f.m) >> f.s) : n;
}

template <int ND>
__device__ __forceinline__ int64_t row_offset(uint32_t row, const Geometry &g) {
  int64_t off = 0;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    if (k == ND - 1) {
      off += int64_t(row) * g.strides[k];
    } else {
      const uint32_t q = fastdiv(row, g.cdiv[k]);
      off += int64_t(row - q * g.cdiv[k].d) * g.strides[k];
      row = q;
    }
  }
  return off;
}

constexpr int kUnroll = 4;

template <int W, int ND, bool UNPACK>
__global__ void __launch_bounds__(512)
    k_words(char *__restrict__ strided, char *__restrict__ packed,
            const __grid_constant__ Geometry g) {
  using T = typename Word<W>::T;
  constexpr int U = kUnroll;
  const uint32_t nthreads = gridDim.x * blockDim.x;
  const uint32_t total = g.total_words;
  // every pass keeps U independent loads in flight; the last pass is
  // predicated instead of falling back to one load at a time
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < total;
       w += U * nthreads) {
    int64_t so[U];
    bool in[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t ww = w + u * nthreads;
      in[u] = ww < total;
      const uint32_t row = fastdiv(in[u] ? ww : 0, g.wdiv);
      const uint32_t col = (in[u] ? ww : 0) - row * g.wpr;
      so[u] = row_offset<ND>(row, g) + int64_t(col) * W;
    }
    T v[U];
    if (!UNPACK) {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (in[u])
          v[u] = __ldg(reinterpret_cast<const T *>(strided + so[u]));
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (in[u])
          reinterpret_cast<T *>(packed)[w + u * nthreads] = v[u];
    } else {
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (in[u])
          v[u] = __ldg(reinterpret_cast<const T *>(packed) + (w + u * nthreads));
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (in[u])
          *reinterpret_cast<T *>(strided + so[u]) = v[u];
    }
  }
}

template <int W, int ND, bool UNPACK>
__global__ void __launch_bounds__(512)
    k_rows(char *__restrict__ strided, char *__restrict__ packed,
           const __grid_constant__ Geometry g) {
  using T = typename Word<W>::T;
  constexpr int U = kUnroll;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t wpr = g.wpr;
  for (uint32_t row = warp; row < g.rows; row += nwarps) {
    T *s = reinterpret_cast<T *>(strided + row_offset<ND>(row, g));
    T *p = reinterpret_cast<T *>(packed + int64_t(row) * g.block);
    const T *src = UNPACK ? p : s;
    T *dst = UNPACK ? s : p;
    // U predicated loads in flight per lane, whatever the row length
    for (uint32_t c = lane; c < wpr; c += 32 * U) {
      T v[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (c + 32 * u < wpr)
          v[u] = __ldg(src + c + 32 * u);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (c + 32 * u < wpr)
          dst[c + 32 * u] = v[u];
    }
  }
}

// Row copy for rows whose source and destination disagree modulo 16.
// The destination row is covered by nw 16-B aligned words, the first and the
// last possibly partial.  Each group of L lanes owns one row and each lane K
// of its words per pass (lane l: words base + l + k*L), so K independent
// loads are in flight per lane and every instruction of a group touches L
// consecutive words: behind the L2 the order would not matter, but reads of
// host memory over the link are issued per instruction, and wide contiguous
// requests are what the link moves efficiently.  Word j is assembled with
// funnel shifts from the 16-B aligned source words j and j+1 that cover it;
// word j+1 comes from the next lane by shuffle, so every source word is
// loaded once.  A source word is loaded only if it holds a byte of the row,
// so no access leaves the 16-B chunks the row touches.  Whole words are
// stored as one 16-B store; the partial end words as aligned 8/4/2/1-byte
// pieces of exactly the row's bytes.
constexpr int kShiftWords = 4;

__device__ __forceinline__ uint4 realign(const uint4 &a, const uint4 &b,
                                         uint32_t q, uint32_t sh) {
  uint32_t x0, x1, x2, x3, x4; // the five 32-bit words covering the output
  switch (q) {
  case 0: x0 = a.x, x1 = a.y, x2 = a.z, x3 = a.w, x4 = b.x; break;
  case 1: x0 = a.y, x1 = a.z, x2 = a.w, x3 = b.x, x4 = b.y; break;
  case 2: x0 = a.z, x1 = a.w, x2 = b.x, x3 = b.y, x4 = b.z; break;
  default: x0 = a.w, x1 = b.x, x2 = b.y, x3 = b.z, x4 = b.w; break;
  }
  return make_uint4(__funnelshift_r(x0, x1, sh), __funnelshift_r(x1, x2, sh),
                    __funnelshift_r(x2, x3, sh), __funnelshift_r(x3, x4, sh));
}

__device__ __forceinline__ uint32_t word32(const uint4 &v, uint32_t i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// bytes [a, b) of v to w + a (w 16-B aligned), in the widest aligned pieces
__device__ __forceinline__ void store_part(char *w, const uint4 &v, uint32_t a,
                                           uint32_t b) {
  while (a < b) {
    const uint32_t x = word32(v, a >> 2);
    if ((a & 7) == 0 && a + 8 <= b) {
      *reinterpret_cast<uint2 *>(w + a) = make_uint2(x, word32(v, (a >> 2) + 1));
      a += 8;
    } else if ((a & 3) == 0 && a + 4 <= b) {
      *reinterpret_cast<uint32_t *>(w + a) = x;
      a += 4;
    } else if ((a & 1) == 0 && a + 2 <= b) {
      *reinterpret_cast<uint16_t *>(w + a) = uint16_t(x >> ((a & 3) * 8));
      a += 2;
    } else {
      w[a] = char(x >> ((a & 3) * 8));
      a += 1;
    }
  }
}

template <int L>
__device__ __forceinline__ void shifted_row(const char *__restrict__ s,
                                            char *__restrict__ d, uint32_t n,
                                            uint32_t lane) {
  constexpr int K = kShiftWords;
  // destination words dw[0, nw) hold the row at bytes [lo, end)
  const uint32_t lo = uint32_t(reinterpret_cast<uintptr_t>(d) & 15);
  uint4 *dw = reinterpret_cast<uint4 *>(d - lo);
  const uint32_t end = lo + n;
  const uint32_t nw = (end + 15) >> 4;
  // destination byte x of the words comes from source byte aw + o + x
  const char *s0 = s - lo;
  const uint32_t o = uint32_t(reinterpret_cast<uintptr_t>(s0) & 15);
  const uint4 *aw = reinterpret_cast<const uint4 *>(s0 - o);
  const uint32_t j_first = (o + lo) >> 4, j_last = (o + end - 1) >> 4;
  const uint32_t q = o >> 2, sh = (o & 3) * 8;
  constexpr unsigned kMask = L == 32 ? 0xffffffffu : ((1u << L) - 1u);
  const unsigned mask = kMask << (threadIdx.x & 31 & ~(L - 1));
  const uint32_t from = (lane + 1) & (L - 1);
  // every lane of a group runs the same number of passes (uniform `nw`)
  for (uint32_t base = 0; base < nw; base += L * K) {
    // a[k] = source word base + k*L + lane; lane 0 also loads the word after
    // the pass, base + K*L
    uint4 a[K + 1];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const uint32_t j = base + k * L + lane;
      a[k] = (j >= j_first && j <= j_last) ? __ldg(aw + j) : make_uint4(0, 0, 0, 0);
    }
    {
      const uint32_t j = base + K * L;
      a[K] = (lane == 0 && j >= j_first && j <= j_last) ? __ldg(aw + j)
                                                         : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      // the word after lane l's word k is lane l+1's word k, and for the
      // group's last lane it is lane 0's word k+1
      const uint4 send = lane == 0 ? a[k + 1] : a[k];
      uint4 next;
      next.x = __shfl_sync(mask, send.x, from, L);
      next.y = __shfl_sync(mask, send.y, from, L);
      next.z = __shfl_sync(mask, send.z, from, L);
      next.w = __shfl_sync(mask, send.w, from, L);
      const uint32_t j = base + k * L + lane;
      if (j < nw) {
        const uint4 v = realign(a[k], next, q, sh);
        const uint32_t b0 = j == 0 ? lo : 0;
        const uint32_t b1 = j == nw - 1 ? end - 16 * j : 16;
        if (b0 == 0 && b1 == 16)
          dw[j] = v;
        else
          store_part(reinterpret_cast<char *>(dw + j), v, b0, b1);
      }
    }
  }
}

template <int L, int ND, bool UNPACK>
__global__ void __launch_bounds__(256)
    k_rows_shift(char *__restrict__ strided, char *__restrict__ packed,
                 const __grid_constant__ Geometry g) {
  const uint32_t lane = threadIdx.x & (L - 1);
  const uint32_t group = (blockIdx.x * blockDim.x + threadIdx.x) / L;
  const uint32_t ngroups = (gridDim.x * blockDim.x) / L;
  const uint32_t n = uint32_t(g.block);
  for (uint32_t row = group; row < g.rows; row += ngroups) {
    char *s = strided + row_offset<ND>(row, g);
    char *p = packed + int64_t(row) * g.block;
    if (UNPACK)
      shifted_row<L>(p, s, n, lane);
    else
      shifted_row<L>(s, p, n, lane);
  }
}

// Staged unpack (kernel 4): the contiguous packed side is pulled into shared
// memory with bulk asynchronous copies (cp.async.bulk, completion counted on
// an mbarrier), kStagedStages chunks in flight per CTA, and the threads
// scatter each chunk's words to the typed rows from shared memory with
// consecutive threads storing consecutive words.  Meant for rows whose
// alignment forces narrow typed-side words: the plain kernels then keep too
// few bytes of loads in flight.  The host launches it only when the packed
// base is 16-B aligned and the packed size a multiple of 16 bytes, which is
// what a bulk copy requires.  Every wait on an mbarrier is bounded (about a
// second of SM clock); a CTA that gives up sets the failure word of
// StagedCtl (mapped pinned host memory, read by the host after it
// synchronises: staged_failed), waits (bounded again) for its other copies
// and returns, leaving its chunks uncopied.
constexpr int kStagedBytes = 8192;
constexpr int kStagedStages = 3;
constexpr int kStagedThreads = 256;

struct StagedCtl {
  int *fail;          // device address of the host-mapped failure word
  uint32_t shortfall; // bytes each chunk's barrier expects beyond its copies:
                      // 0, except to exercise the give-up path in tests
};

__device__ __forceinline__ void staged_give_up(const StagedCtl &ctl) {
  *reinterpret_cast<volatile int *>(ctl.fail) = 1;
  __threadfence_system();
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar))
               : "memory");
}

// one bulk copy of `bytes` into shared memory, its barrier told to expect
// `bytes + shortfall`
__device__ __forceinline__ void bulk_load(void *dst, const void *src,
                                          uint32_t bytes, uint32_t shortfall,
                                          uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes + shortfall)
               : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::"
               "bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_done(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// false after about 2^31 SM cycles (about a second) without completion
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar,
                                                  uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_done(bar, parity)) {
    if (clock64() - t0 > (1ll << 31))
      return false;
    __nanosleep(64);
  }
  return true;
}

// mbarrier.try_wait suspends the thread until the phase completes or a
// hardware time limit passes, so a waiting warp neither spins nor sleeps
// past the completion; false after about 2^31 SM cycles (about a second)
__device__ __forceinline__ bool mbar_try_wait_bounded(uint64_t *bar,
                                                      uint32_t parity) {
  const long long t0 = clock64();
  for (;;) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    if (ok)
      return true;
    if (clock64() - t0 > (1ll << 31))
      return false;
  }
}

// The give-up path of a staged CTA, run by one thread: report the failure,
// then wait once more (bounded again) on every stage that still has copies
// counted -- the stage whose wait ran out included -- so that a copy that
// was only slow lands before the CTA exits.  A copy still in flight after
// this second bound (about two seconds in all) would write into the shared
// memory of an exited CTA; nothing in this library issues such a copy (every
// bulk copy reads device memory proper), so that case is a GPU fault, not a
// path this code expects.
__device__ __forceinline__ void staged_drain(const StagedCtl &ctl,
                                             uint64_t *bar, uint32_t c,
                                             uint32_t it, uint32_t nchunks) {
  staged_give_up(ctl);
  for (int k = 0; k < kStagedStages; ++k) {
    const uint32_t ck = c + uint32_t(k) * gridDim.x;
    if (ck < nchunks)
      mbar_wait_bounded(&bar[(it + k) % kStagedStages],
                        ((it + k) / kStagedStages) & 1);
  }
}

template <int W, int ND>
__global__ void __launch_bounds__(kStagedThreads)
    k_unpack_staged(char *__restrict__ strided,
                    const char *__restrict__ packed,
                    const __grid_constant__ Geometry g, uint32_t nchunks,
                    uint64_t total_bytes, StagedCtl ctl) {
  using T = typename Word<W>::T;
  __shared__ __align__(128) char stage[kStagedStages][kStagedBytes];
  __shared__ __align__(8) uint64_t bar[kStagedStages];
  __shared__ int gave_up;
  auto chunk_bytes = [&](uint32_t c) {
    const uint64_t left = total_bytes - uint64_t(c) * kStagedBytes;
    return uint32_t(left < uint64_t(kStagedBytes) ? left : kStagedBytes);
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStagedStages; ++s)
      mbar_init(&bar[s]);
    gave_up = 0;
    // the initialised barriers are visible to the copy engine's proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int s = 0; s < kStagedStages; ++s) {
      const uint32_t c = blockIdx.x + uint32_t(s) * gridDim.x;
      if (c < nchunks)
        bulk_load(stage[s], packed + uint64_t(c) * kStagedBytes,
                  chunk_bytes(c), ctl.shortfall, &bar[s]);
    }
  }
  __syncthreads();
  uint32_t it = 0;
  for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x, ++it) {
    const int s = int(it % kStagedStages);
    const uint32_t parity = (it / kStagedStages) & 1;
    if (!mbar_wait_bounded(&bar[s], parity))
      gave_up = 1;
    __syncthreads();
    if (gave_up) {
      if (threadIdx.x == 0)
        staged_drain(ctl, bar, c, it, nchunks);
      return;
    }
    const uint32_t words = chunk_bytes(c) / W;
    const uint32_t w0 = c * uint32_t(kStagedBytes / W);
    const T *src = reinterpret_cast<const T *>(stage[s]);
    for (uint32_t j = threadIdx.x; j < words; j += blockDim.x) {
      const uint32_t w = w0 + j;
      const uint32_t row = fastdiv(w, g.wdiv);
      const uint32_t col = w - row * g.wpr;
      *reinterpret_cast<T *>(strided + row_offset<ND>(row, g) +
                             int64_t(col) * W) = src[j];
    }
    __syncthreads(); // every thread is done with stage s
    if (threadIdx.x == 0) {
      const uint32_t cn = c + uint32_t(kStagedStages) * gridDim.x;
      if (cn < nchunks)
        bulk_load(stage[s], packed + uint64_t(cn) * kStagedBytes,
                  chunk_bytes(cn), ctl.shortfall, &bar[s]);
    }
  }
}

// The bulk kernels: the staged pack, and the staged unpack of 16-B aligned
// rows of at least kBulkMinRow bytes (or of a contiguous run).  One warp per
// CTA moves kBulkChunk-byte chunks of the packed stream through kBulkStages
// shared-memory stages with bulk asynchronous copies in both directions, and
// no thread touches the data:
//   pack    the row pieces of chunk c are gathered into a stage (one bulk
//           copy per piece, the lanes issuing pieces in parallel, all
//           counted on the stage's mbarrier); lane 0 writes the stage to
//           the packed buffer with one bulk store;
//   unpack  lane 0 pulls chunk c into a stage with one bulk copy; the lanes
//           write its row pieces out with one bulk store each.
// A stage is refilled once the bulk stores that read it have finished
// reading (cp.async.bulk.wait_group.read), one iteration behind, so
// kBulkStages - 1 chunks are on their way in while one goes out.  Every
// piece is 16-B aligned with a multiple of 16 bytes (width 16: block,
// strides and both bases), as bulk copies require.  Each wait on an
// mbarrier is bounded as in k_unpack_staged; a CTA that gives up sets the
// failure word, waits (bounded) on every chunk it has requested, waits for
// its stores and returns.
constexpr uint32_t kBulkChunk = 16384;
constexpr int kBulkStages = 4;
constexpr int kBulkSmem = int(kBulkChunk) * kBulkStages;
constexpr int kBulkMaxPerSm = 3;       // 3 x 64 KB of shared memory per SM
constexpr uint64_t kBulkMinRow = 512;  // narrower unpacks scatter by words
// Measured on B200, contiguous copies back to back: one CTA per SM moves 128
// MiB and more 3-4 % faster than two or three (fewer interleaved streams),
// while below that the extra CTAs win (64 MiB: 21.0 us at 2-3 per SM
// against 25.0 at one)
constexpr uint64_t kBulkOnePerSm = uint64_t(96) << 20;

__device__ __forceinline__ void bulk_expect(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// global -> shared, completion counted on `bar`
__device__ __forceinline__ void bulk_in(void *dst, const void *src,
                                        uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::"
               "bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// shared -> global, in this thread's current bulk group
__device__ __forceinline__ void bulk_out(void *dst, const void *src,
                                         uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::
                   "l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
}

template <int ND, bool UNPACK>
__global__ void __launch_bounds__(32)
    k_staged_bulk(char *__restrict__ strided, char *__restrict__ packed,
                  const __grid_constant__ Geometry g, uint32_t nchunks,
                  uint64_t total_bytes, StagedCtl ctl) {
  extern __shared__ __align__(128) char stage[]; // kBulkStages x kBulkChunk
  __shared__ __align__(8) uint64_t bar[kBulkStages];
  const uint32_t lane = threadIdx.x;
  const uint64_t block = uint64_t(g.block);
  auto chunk_bytes = [&](uint32_t c) {
    const uint64_t left = total_bytes - uint64_t(c) * kBulkChunk;
    return uint32_t(left < uint64_t(kBulkChunk) ? left : kBulkChunk);
  };
  // piece k of chunk c (lane l takes k = l, l + 32, ...): stage bytes
  // [d, d + len) and the strided bytes of row row0 + k from offset o
  auto pieces = [&](uint32_t c, auto &&f) {
    const uint64_t p0 = uint64_t(c) * kBulkChunk;
    const uint32_t n = chunk_bytes(c);
    const uint32_t row0 = uint32_t(p0 / block);
    const uint64_t off0 = p0 - uint64_t(row0) * block;
    const uint64_t first = block - off0; // bytes of the first row's piece
    for (uint32_t k = lane;; k += 32) {
      const uint64_t d = k == 0 ? 0 : first + uint64_t(k - 1) * block;
      if (d >= n)
        break;
      const uint64_t o = k == 0 ? off0 : 0;
      const uint64_t len = block - o < n - d ? block - o : n - d;
      f(uint32_t(d), strided + row_offset<ND>(row0 + k, g) + o, uint32_t(len));
    }
  };
  // warp-wide: chunk c into stage s
  auto fill = [&](uint32_t c, int s) {
    char *st = stage + size_t(s) * kBulkChunk;
    if (lane == 0)
      bulk_expect(&bar[s], chunk_bytes(c) + ctl.shortfall);
    __syncwarp();
    if (UNPACK) {
      if (lane == 0)
        bulk_in(st, packed + uint64_t(c) * kBulkChunk, chunk_bytes(c), &bar[s]);
    } else {
      pieces(c, [&](uint32_t d, const char *src, uint32_t len) {
        bulk_in(st + d, src, len, &bar[s]);
      });
    }
  };
  // warp-wide: stage s out to where chunk c belongs, one bulk group per lane
  auto empty = [&](uint32_t c, int s) {
    const char *st = stage + size_t(s) * kBulkChunk;
    if (UNPACK) {
      pieces(c, [&](uint32_t d, char *dst, uint32_t len) {
        bulk_out(dst, st + d, len);
      });
    } else if (lane == 0) {
      bulk_out(packed + uint64_t(c) * kBulkChunk, st, chunk_bytes(c));
    }
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  };
  if (lane == 0) {
    for (int s = 0; s < kBulkStages; ++s)
      mbar_init(&bar[s]);
    // the initialised barriers are visible to the copy engine's proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  uint32_t issued = 0; // iterations whose chunk has been requested
  for (int s = 0; s < kBulkStages; ++s) {
    const uint32_t c = blockIdx.x + uint32_t(s) * gridDim.x;
    if (c >= nchunks)
      break;
    fill(c, s);
    ++issued;
  }
  uint32_t it = 0;
  for (uint32_t c = blockIdx.x; c < nchunks; c += gridDim.x, ++it) {
    const int s = int(it % kBulkStages);
    const bool ok = mbar_try_wait_bounded(&bar[s], (it / kBulkStages) & 1);
    if (!__all_sync(0xffffffffu, ok)) {
      if (lane == 0) {
        staged_give_up(ctl);
        for (uint32_t j = it; j < issued; ++j)
          mbar_try_wait_bounded(&bar[j % kBulkStages], (j / kBulkStages) & 1);
      }
      __syncwarp();
      break;
    }
    empty(c, s);
    // the stage emptied one iteration ago is free once its stores have read
    // it: refill it with the chunk kBulkStages - 1 iterations ahead
    asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
    __syncwarp();
    if (it >= 1) {
      const uint32_t cn = c + uint32_t(kBulkStages - 1) * gridDim.x;
      if (cn < nchunks) {
        fill(cn, int((it - 1) % kBulkStages));
        ++issued;
      }
    }
  }
  // every store complete before the CTA (and its shared memory) goes
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

using StagedFn = void (*)(char *, const char *, Geometry, uint32_t, uint64_t,
                          StagedCtl);
using BulkFn = void (*)(char *, char *, Geometry, uint32_t, uint64_t,
                        StagedCtl);

template <bool UNPACK> BulkFn pick_bulk(uint32_t nd) {
  switch (nd) {
  case 0: return k_staged_bulk<0, UNPACK>;
  case 1: return k_staged_bulk<1, UNPACK>;
  case 2: return k_staged_bulk<2, UNPACK>;
  case 3: return k_staged_bulk<3, UNPACK>;
  case 4: return k_staged_bulk<4, UNPACK>;
  default: return k_staged_bulk<5, UNPACK>;
  }
}

// The bulk kernels take more than the default 48 KB of dynamic shared
// memory; the limit is raised once per kernel and device.
bool bulk_smem_ready(BulkFn fn) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  static std::mutex mu;
  static std::set<std::pair<int, const void *>> done;
  const auto key = std::make_pair(dev, reinterpret_cast<const void *>(fn));
  std::lock_guard<std::mutex> l(mu);
  if (done.count(key))
    return true;
  if (cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kBulkSmem) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  done.insert(key);
  return true;
}

// The failure word of the staged kernels: one int of mapped pinned host
// memory (portable to every device), allocated by MPI_Init, or else at the
// first staged launch outside a stream capture.  Until it exists the plain
// kernels run instead.
namespace {
std::once_flag g_fail_once;
// written once inside g_fail_once, then published by g_fail_ready
int *g_fail_host = nullptr, *g_fail_dev = nullptr;
std::atomic<bool> g_fail_ready{false};
std::atomic<int64_t> g_fail_count{0};
} // namespace

bool staged_channel(cudaStream_t stream) {
  if (g_fail_ready.load(std::memory_order_acquire))
    return true;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (cs != cudaStreamCaptureStatusNone)
    return false;
  std::call_once(g_fail_once, [] {
    void *h = nullptr, *d = nullptr;
    if (cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable) !=
        cudaSuccess) {
      cudaGetLastError();
      return;
    }
    if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
      cudaGetLastError();
      cudaFreeHost(h);
      return;
    }
    *static_cast<volatile int *>(h) = 0;
    g_fail_host = static_cast<int *>(h);
    g_fail_dev = static_cast<int *>(d);
    g_fail_ready.store(true, std::memory_order_release);
  });
  return g_fail_ready.load(std::memory_order_acquire);
}

bool staged_failed() {
  if (!g_fail_ready.load(std::memory_order_acquire))
    return false;
  // one reader takes the word, so two threads never report one failure twice
  if (__atomic_exchange_n(g_fail_host, 0, __ATOMIC_ACQ_REL) == 0)
    return false;
  g_fail_count++;
  return true;
}

int64_t staged_timeouts() {
  int64_t n = g_fail_count.load();
  if (g_fail_ready.load(std::memory_order_acquire) &&
      *static_cast<volatile int *>(g_fail_host))
    ++n;
  return n;
}

template <int W> StagedFn pick_staged_nd(uint32_t nd) {
  switch (nd) {
  case 0: return k_unpack_staged<W, 0>;
  case 1: return k_unpack_staged<W, 1>;
  case 2: return k_unpack_staged<W, 2>;
  case 3: return k_unpack_staged<W, 3>;
  case 4: return k_unpack_staged<W, 4>;
  default: return k_unpack_staged<W, 5>;
  }
}

StagedFn pick_staged(uint32_t width, uint32_t nd) {
  switch (width) {
  case 16: return pick_staged_nd<16>(nd);
  case 8: return pick_staged_nd<8>(nd);
  case 4: return pick_staged_nd<4>(nd);
  case 2: return pick_staged_nd<2>(nd);
  default: return pick_staged_nd<1>(nd);
  }
}

using KernelFn = void (*)(char *, char *, Geometry);

template <int L, bool UNPACK> KernelFn pick_shift(uint32_t nd) {
  switch (nd) {
  case 0: return k_rows_shift<L, 0, UNPACK>;
  case 1: return k_rows_shift<L, 1, UNPACK>;
  case 2: return k_rows_shift<L, 2, UNPACK>;
  case 3: return k_rows_shift<L, 3, UNPACK>;
  case 4: return k_rows_shift<L, 4, UNPACK>;
  default: return k_rows_shift<L, 5, UNPACK>;
  }
}

template <int W, bool UNPACK> KernelFn pick_words(uint32_t nd) {
  switch (nd) {
  case 0: return k_words<W, 0, UNPACK>;
  case 1: return k_words<W, 1, UNPACK>;
  case 2: return k_words<W, 2, UNPACK>;
  case 3: return k_words<W, 3, UNPACK>;
  case 4: return k_words<W, 4, UNPACK>;
  default: return k_words<W, 5, UNPACK>;
  }
}

template <int W, bool UNPACK> KernelFn pick_rows(uint32_t nd) {
  switch (nd) {
  case 0: return k_rows<W, 0, UNPACK>;
  case 1: return k_rows<W, 1, UNPACK>;
  case 2: return k_rows<W, 2, UNPACK>;
  case 3: return k_rows<W, 3, UNPACK>;
  case 4: return k_rows<W, 4, UNPACK>;
  default: return k_rows<W, 5, UNPACK>;
  }
}

template <bool UNPACK> KernelFn pick(int kernel, uint32_t width, uint32_t nd) {
  if (kernel == 3) { // `width` carries the lanes per row here
    switch (width) {
    case 4: return pick_shift<4, UNPACK>(nd);
    case 8: return pick_shift<8, UNPACK>(nd);
    case 16: return pick_shift<16, UNPACK>(nd);
    default: return pick_shift<32, UNPACK>(nd);
    }
  }
  if (kernel == 2) {
    switch (width) {
    case 16: return pick_rows<16, UNPACK>(nd);
    case 8: return pick_rows<8, UNPACK>(nd);
    case 4: return pick_rows<4, UNPACK>(nd);
    case 2: return pick_rows<2, UNPACK>(nd);
    default: return pick_rows<1, UNPACK>(nd);
    }
  }
  switch (width) {
  case 16: return pick_words<16, UNPACK>(nd);
  case 8: return pick_words<8, UNPACK>(nd);
  case 4: return pick_words<4, UNPACK>(nd);
  case 2: return pick_words<2, UNPACK>(nd);
  default: return pick_words<1, UNPACK>(nd);
  }
}

static const char *kernel_name(int kernel, uint32_t width, bool unpack) {
  static char names[4][2][33][32];
  static std::once_flag once;
  std::call_once(once, [] {
    const char *k_names[4] = {"words", "rows", "shift", "staged"};
    for (int k = 0; k < 4; ++k)
      for (int u = 0; u < 2; ++u)
        for (int w = 1; w <= 32; w *= 2)
          std::snprintf(names[k][u][w], 32, "%s_%s_%s%d", k_names[k],
                        u ? "unpack" : "pack", k == 2 ? "l" : "w", w);
  });
  return names[kernel - 1][unpack][width];
}

// SM count of the current device, cached per device index (a process may
// drive GPUs with different SM counts)
int num_sms() {
  constexpr int kDevs = 64;
  static std::atomic<int> cache[kDevs];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = -1;
  }
  if (dev >= 0 && dev < kDevs) {
    const int c = cache[dev].load(std::memory_order_relaxed);
    if (c > 0)
      return c;
  }
  int sms = 0;
  if (dev < 0 ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
          cudaSuccess ||
      sms <= 0) {
    cudaGetLastError();
    return 148;
  }
  if (dev < kDevs)
    cache[dev].store(sms, std::memory_order_relaxed);
  return sms;
}

int make_geometry(const tempi_desc *d, int64_t incount, uintptr_t sbase,
                  uintptr_t pbase, int max_width, Geometry *g, bool *empty) {
  *empty = false;
  if (!d || !g)
    return set_error(TEMPI_ERR_ARG, "null descriptor");
  if (d->ndims < 0 || d->ndims > TEMPI_MAX_DIMS || d->block < 0 || incount < 0)
    return set_error(TEMPI_ERR_ARG, "bad descriptor (ndims=%d block=%lld)",
                     d->ndims, (long long)d->block);
  if (incount == 0 || d->block == 0) {
    *empty = true;
    return TEMPI_OK;
  }
  int64_t cnt[KDIMS], str[KDIMS];
  int n = 0;
  for (int k = 0; k < d->ndims; ++k) {
    if (d->counts[k] < 0)
      return set_error(TEMPI_ERR_ARG, "negative count");
    if (d->counts[k] == 0) {
      *empty = true;
      return TEMPI_OK;
    }
    if (d->counts[k] != 1) {
      cnt[n] = d->counts[k];
      str[n] = d->strides[k];
      ++n;
    }
  }
  if (incount != 1) {
    cnt[n] = incount;
    str[n] = d->extent;
    ++n;
  }
  int64_t block = d->block;
  for (bool changed = true; changed;) {
    changed = false;
    if (n > 0 && str[0] == block) { // rows are adjacent: one longer block
      block *= cnt[0];
      for (int k = 1; k < n; ++k)
        cnt[k - 1] = cnt[k], str[k - 1] = str[k];
      --n;
      changed = true;
      continue;
    }
    for (int k = 0; k + 1 < n; ++k) {
      if (str[k + 1] == cnt[k] * str[k]) { // dim k+1 continues dim k
        cnt[k] *= cnt[k + 1];
        for (int j = k + 2; j < n; ++j)
          cnt[j - 1] = cnt[j], str[j - 1] = str[j];
        --n;
        changed = true;
        break;
      }
    }
  }
  int64_t rows = 1;
  for (int k = 0; k < n; ++k) {
    rows *= cnt[k];
    if (rows > INT32_MAX)
      return set_error(TEMPI_ERR_ARG, "too many rows");
  }
  if (block > INT32_MAX || rows * block > INT32_MAX)
    return set_error(TEMPI_ERR_ARG, "packed size exceeds 2^31-1 bytes");
  for (int k = 0; k < n; ++k)
    if (cnt[k] > INT32_MAX)
      return set_error(TEMPI_ERR_ARG, "count too large");

  uint64_t bits = uint64_t(block) | uint64_t(sbase) | uint64_t(pbase);
  for (int k = 0; k < n; ++k)
    bits |= uint64_t(str[k]);
  uint32_t w = 16;
  while (w > 1 && (bits & (w - 1)))
    w >>= 1;
  while (max_width > 0 && w > uint32_t(max_width))
    w >>= 1;

  std::memset(g, 0, sizeof(*g));
  g->nd = n;
  for (int k = 0; k < n; ++k) {
    g->strides[k] = str[k];
    g->cdiv[k] = make_fastdiv(uint32_t(cnt[k]));
  }
  g->width = w;
  g->wpr = uint32_t(block / w);
  g->wdiv = make_fastdiv(g->wpr);
  g->rows = uint32_t(rows);
  g->total_words = uint32_t(rows) * g->wpr;
  g->block = block;
  return TEMPI_OK;
}

int launch_geometry(const Geometry &g, const char *strided, char *packed,
                    bool unpack, const tempi_config *cfg, cudaStream_t stream,
                    int both_device) {
  const int sms = num_sms();
  int kernel = cfg ? cfg->kernel : 0;
  // the staged kernels (4), where their bulk copies are allowed: unpack
  // needs a 16-B aligned packed base and a packed size that is a multiple of
  // 16 bytes; pack needs every row piece 16-B aligned on both sides (width
  // 16).  Both sides must be device memory proper: host-mapped and managed
  // buffers take the plain kernels; so do launches before the failure word
  // exists (see staged_channel).
  const uint64_t bytes = uint64_t(g.rows) * uint64_t(g.block);
  const bool wide = g.width == 16 && bytes >= (uint64_t(32) << 20);
  const bool narrow_unpack =
      unpack && bytes >= (uint64_t(1) << 20) && g.block <= 512;
  bool staged =
      (kernel == 4 || ((kernel < 1 || kernel > 4) && (wide || narrow_unpack))) &&
      bytes % 16 == 0 &&
      (unpack ? (reinterpret_cast<uintptr_t>(packed) & 15) == 0
              : g.width == 16) &&
      (both_device >= 0
           ? both_device == 1
           : classify(strided).is_device && classify(packed).is_device) &&
      staged_channel(stream);
  // packs, and unpacks of wide aligned rows, run the bulk kernels
  BulkFn bulk = nullptr;
  if (staged &&
      (!unpack || (g.width == 16 && (g.nd == 0 || g.block >= kBulkMinRow)))) {
    bulk = unpack ? pick_bulk<true>(g.nd) : pick_bulk<false>(g.nd);
    if (!bulk_smem_ready(bulk)) {
      bulk = nullptr;
      staged = unpack; // a pack then takes the plain kernels
    }
  }
  if (staged) {
    const StagedCtl ctl{g_fail_dev, uint32_t(env().staged_shortfall)};
    const int req =
        (cfg && cfg->blocks_per_sm >= 1 && cfg->blocks_per_sm <= 8)
            ? cfg->blocks_per_sm
            : 0;
    if (bulk) {
      // one warp per CTA: one CTA per SM for long streams, else as many as
      // their shared memory allows; a requested count caps it
      const uint32_t nchunks = uint32_t((bytes + kBulkChunk - 1) / kBulkChunk);
      const int own = bytes >= kBulkOnePerSm ? 1 : kBulkMaxPerSm;
      const int bps = req ? std::min(req, own) : own;
      const uint32_t blocks = std::max<uint32_t>(
          1, std::min<uint32_t>(nchunks, uint32_t(sms) * uint32_t(bps)));
      bulk<<<blocks, 32, kBulkSmem, stream>>>(const_cast<char *>(strided),
                                               packed, g, nchunks, bytes, ctl);
    } else {
      const uint32_t nchunks =
          uint32_t((bytes + kStagedBytes - 1) / kStagedBytes);
      // measured on the strided sweep: 3 CTAs per SM for long aligned
      // streams, a full SM (8 CTAs of 256 threads) for narrow scatters
      const int bps = req ? req : wide ? 3 : 8;
      const uint32_t blocks = std::max<uint32_t>(
          1, std::min<uint32_t>(nchunks, uint32_t(sms) * uint32_t(bps)));
      pick_staged(g.width, g.nd)<<<blocks, kStagedThreads, 0, stream>>>(
          const_cast<char *>(strided), packed, g, nchunks, bytes, ctl);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
      return cuda_error(e, "staged kernel launch");
    counters().kernel_launches++;
    set_last_kernel(kernel_name(4, g.width, unpack));
    return TEMPI_OK;
  }
  if (kernel < 1 || kernel > 3) {
    if (!unpack && g.width < 16 && g.block >= 128 && g.rows >= uint32_t(sms))
      kernel = 3; // misaligned wide rows: realign with funnel shifts
    else if (g.wpr >= 64 && g.rows >= uint32_t(2 * sms))
      kernel = 2;
    else
      kernel = 1;
  }
  // rows per group of lanes for the shift kernel
  uint32_t lanes = 32;
  if (kernel == 3) {
    const int req = cfg ? cfg->unroll : 0; // reused: lanes per row
    // one pass of a group covers lanes * kShiftWords * 16 bytes of a row
    lanes = (req == 4 || req == 8 || req == 16 || req == 32)
                ? uint32_t(req)
                : (g.block > 1024 ? 32u
                   : g.block > 512 ? 16u
                   : g.block > 256 ? 8u
                                   : 4u);
  }
  int threads = (cfg && cfg->threads) ? cfg->threads : 256;
  threads = std::max(32, std::min(kernel == 3 ? 256 : 512, threads / 32 * 32));
  int bps = (cfg && cfg->blocks_per_sm) ? cfg->blocks_per_sm : 2048 / threads;
  int64_t need;
  if (kernel == 2)
    need = (int64_t(g.rows) * 32 + threads - 1) / threads;
  else if (kernel == 3)
    need = (int64_t(g.rows) * lanes + threads - 1) / threads;
  else
    need = (int64_t(g.total_words) + int64_t(threads) * kUnroll - 1) /
           (int64_t(threads) * kUnroll);
  int64_t blocks = std::min<int64_t>(need, int64_t(sms) * bps);
  blocks = std::max<int64_t>(blocks, 1);
  const uint32_t sel = kernel == 3 ? lanes : g.width;
  KernelFn fn = unpack ? pick<true>(kernel, sel, g.nd)
                       : pick<false>(kernel, sel, g.nd);
  fn<<<unsigned(blocks), threads, 0, stream>>>(const_cast<char *>(strided),
                                               packed, g);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "pack kernel launch");
  counters().kernel_launches++;
  set_last_kernel(kernel_name(kernel, sel, unpack));
  return TEMPI_OK;
}

int pack_known(const tempi_desc *d, const void *origin, int64_t incount,
               void *packed, const tempi_config *cfg, cudaStream_t stream,
               int both_device) {
  if (!d)
    return set_error(TEMPI_ERR_ARG, "null descriptor");
  const char *base = static_cast<const char *>(origin) + d->start;
  Geometry g;
  bool empty;
  int err = make_geometry(d, incount, uintptr_t(base), uintptr_t(packed),
                          cfg ? cfg->width : 0, &g, &empty);
  if (err || empty)
    return err;
  counters().packs++;
  counters().pack_bytes += int64_t(g.rows) * g.block;
  return launch_geometry(g, base, static_cast<char *>(packed), false, cfg,
                         stream, both_device);
}

int unpack_known(const tempi_desc *d, const void *packed, int64_t incount,
                 void *origin, const tempi_config *cfg, cudaStream_t stream,
                 int both_device) {
  if (!d)
    return set_error(TEMPI_ERR_ARG, "null descriptor");
  char *base = static_cast<char *>(origin) + d->start;
  Geometry g;
  bool empty;
  int err = make_geometry(d, incount, uintptr_t(base), uintptr_t(packed),
                          cfg ? cfg->width : 0, &g, &empty);
  if (err || empty)
    return err;
  counters().unpacks++;
  counters().unpack_bytes += int64_t(g.rows) * g.block;
  return launch_geometry(
      g, base, const_cast<char *>(static_cast<const char *>(packed)), true,
      cfg, stream, both_device);
}

} // namespace tempi

using namespace tempi;

extern "C" int tempi_pack(const tempi_desc *d, const void *origin,
                          int64_t incount, void *packed,
                          const tempi_config *cfg, void *stream) {
  return pack_known(d, origin, incount, packed, cfg,
                    static_cast<cudaStream_t>(stream), -1);
}

extern "C" int tempi_unpack(const tempi_desc *d, const void *packed,
                            int64_t incount, void *origin,
                            const tempi_config *cfg, void *stream) {
  return unpack_known(d, packed, incount, origin, cfg,
                      static_cast<cudaStream_t>(stream), -1);
}

extern "C" int tempi_staged_check(void) {
  if (staged_failed())
    return set_error(TEMPI_ERR_TIMEOUT,
                     "a staged pack/unpack kernel gave up waiting on its bulk "
                     "copies; its output is incomplete");
  return TEMPI_OK;
}
