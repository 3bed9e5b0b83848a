// Batched pack/unpack: every region of a step in one launch.
//
// The reference packs one object per MPI_Pack call, each with its own launch
// and stream synchronisation (src/pack.cpp:56, packer_2d.cu:101-109), so the
// 26 halo regions of a 3-D grid cost 26 launches and 26 synchronisations.
// Here the regions become a table in device memory; one grid-stride kernel
// walks it.
//
// Work is cut into warp chunks: one warp copies one chunk in `passes`
// passes of 32 x L words, where L (words in flight per lane: 4 for 16-byte
// words, 8 for narrower ones) is fixed by the region's proven width and
// `passes` (1, 2 or 4) is chosen per region class.  Warps take chunks
// warp_id, warp_id + total warps, ... with no CTA-wide barrier; each finds
// its chunk's region by ballot rounds over the table's first-chunk column.
// A table of up to kSmemTableBytes is copied into shared memory once per
// CTA (one round trip), so those lookups never touch global memory.  Each
// region keeps its own geometry and proven vector width, so a 16-B row face
// and a 2-KiB row face run at their own width inside the same launch.
//
// The passes of each region class (width x words per row) and the launch
// shape of a batch (threads per CTA, CTAs per SM) come from defaults or from
// tempi_batch_tune, a measured autotuner whose choices are kept per batch
// signature for later batches of the same classes (and in
// TEMPI_CACHE_DIR/tempi_b200_batch_tune.txt).
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
#include "runtime.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

namespace tempi {

namespace {

constexpr int kSmemTableBytes = 32768; // tables up to this size are staged
constexpr int kClasses = 40;           // 5 widths x 8 row-length buckets
constexpr int kPassChoices[3] = {1, 2, 4};

// words each lane keeps in flight in one pass: 64 bytes for 8- and 16-byte
// words (registers allow no more), 8 words for narrower ones
template <int W> constexpr int lane_words() { return W == 16 ? 4 : 8; }
__host__ __device__ constexpr uint32_t lane_words_of(uint32_t w) {
  return w == 16 ? 4u : 8u;
}

struct BatchRegion {
  char *strided; // origin + start
  char *packed;
  Geometry g;
  uint32_t chunk_begin; // first warp chunk of this region
  uint32_t passes;      // passes of a warp over one chunk: 1, 2 or 4
};

struct CopyPair {
  const char *src; // src origin + start
  char *dst;       // dst origin + start
  Geometry gs, gd; // same width and word count
  uint32_t chunk_begin;
  uint32_t passes;
};

// the geometry that sets a record's words and class
const Geometry &geometry_of(const BatchRegion &r) { return r.g; }
const Geometry &geometry_of(const CopyPair &r) { return r.gs; }

template <int W> struct BWord;
template <> struct BWord<1> { using T = uint8_t; };
template <> struct BWord<2> { using T = uint16_t; };
template <> struct BWord<4> { using T = uint32_t; };
template <> struct BWord<8> { using T = uint2; };
template <> struct BWord<16> { using T = uint4; };

__device__ __forceinline__ uint32_t bdiv(uint32_t n, const FastDiv &f) {
  return f.m ? (__umulhi(n, f.m) >> f.s) : n;
}

// strided-side offset of row `row`: its digits over the counts, fastest
// first (a runtime loop, so that the unrolled word loops around it keep few
// registers live)
__device__ __forceinline__ int64_t brow_offset(uint32_t row, const Geometry &g) {
  const int nd = int(g.nd);
  if (nd == 0)
    return 0;
  int64_t off = 0;
#pragma unroll 1
  for (int k = 0; k + 1 < nd; ++k) {
    const uint32_t q = bdiv(row, g.cdiv[k]);
    off += int64_t(row - q * g.cdiv[k].d) * g.strides[k];
    row = q;
  }
  return off + int64_t(row) * g.strides[nd - 1];
}

// byte offset of word w on the strided side of g
template <int W>
__device__ __forceinline__ int64_t word_offset(uint32_t w, const Geometry &g) {
  const uint32_t row = bdiv(w, g.wdiv);
  return brow_offset(row, g) + int64_t(w - row * g.wpr) * W;
}

// One warp chunk of a pack or unpack region: words w0 + lane + 32 u.  Each
// load issues as soon as its address is known and only the loaded words
// stay live until the stores, so U loads are in flight per lane without
// holding U offsets in registers.
template <int W, int U>
__device__ __forceinline__ void pack_chunk(const BatchRegion &r, uint32_t w0,
                                           uint32_t lane, bool unpack) {
  using T = typename BWord<W>::T;
  const uint32_t total = r.g.total_words;
  char *strided = r.strided;
  T *packed = reinterpret_cast<T *>(r.packed);
  T v[U];
  if (!unpack) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t w = w0 + lane + 32 * u;
      if (w < total)
        v[u] = __ldg(reinterpret_cast<const T *>(strided + word_offset<W>(w, r.g)));
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (w0 + lane + 32 * u < total)
        packed[w0 + lane + 32 * u] = v[u];
  } else {
#pragma unroll
    for (int u = 0; u < U; ++u)
      if (w0 + lane + 32 * u < total)
        v[u] = __ldg(packed + (w0 + lane + 32 * u));
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t w = w0 + lane + 32 * u;
      if (w < total)
        *reinterpret_cast<T *>(strided + word_offset<W>(w, r.g)) = v[u];
    }
  }
}

// one warp chunk of a copy pair: the loads at the source geometry first,
// then the stores at the destination geometry
template <int W, int U>
__device__ __forceinline__ void copy_chunk(const CopyPair &r, uint32_t w0,
                                           uint32_t lane) {
  using T = typename BWord<W>::T;
  const uint32_t total = r.gs.total_words;
  T v[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const uint32_t w = w0 + lane + 32 * u;
    if (w < total)
      v[u] = __ldg(reinterpret_cast<const T *>(r.src + word_offset<W>(w, r.gs)));
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    const uint32_t w = w0 + lane + 32 * u;
    if (w < total)
      *reinterpret_cast<T *>(r.dst + word_offset<W>(w, r.gd)) = v[u];
  }
}

// a warp chunk is `passes` passes of 32 x lane_words<W>() words
template <int W>
__device__ __forceinline__ void pack_chunk_p(const BatchRegion &r, uint32_t c,
                                             uint32_t lane, bool unpack) {
  constexpr uint32_t kPass = 32u * lane_words<W>();
  const uint32_t passes = r.passes;
  uint32_t w0 = (c - r.chunk_begin) * passes * kPass;
  for (uint32_t p = 0; p < passes && w0 < r.g.total_words; ++p, w0 += kPass)
    pack_chunk<W, lane_words<W>()>(r, w0, lane, unpack);
}

template <int W>
__device__ __forceinline__ void copy_chunk_p(const CopyPair &r, uint32_t c,
                                             uint32_t lane) {
  constexpr uint32_t kPass = 32u * lane_words<W>();
  const uint32_t passes = r.passes;
  uint32_t w0 = (c - r.chunk_begin) * passes * kPass;
  for (uint32_t p = 0; p < passes && w0 < r.gs.total_words; ++p, w0 += kPass)
    copy_chunk<W, lane_words<W>()>(r, w0, lane);
}

// Index of the last entry whose first chunk is <= chunk, found by one warp:
// each round the lanes sample 32 evenly spaced entries of the remaining
// stretch and a ballot narrows it 32-fold, so n entries take ceil(log32 n)
// rounds (one for a 26-region halo, two for up to 1024 regions).
template <typename Rec>
__device__ __forceinline__ int find_region(const Rec *r, int n, uint32_t chunk,
                                           uint32_t lane) {
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

// The table in shared memory when `staged` (the caller sized the dynamic
// shared memory for it), else in global memory.
template <typename Rec, int THREADS>
__device__ __forceinline__ const Rec *stage_table(const Rec *__restrict__ g,
                                                  int n, int staged,
                                                  uint32_t *s_table) {
  if (!staged)
    return g;
  const uint32_t *from = reinterpret_cast<const uint32_t *>(g);
  const int words = n * int(sizeof(Rec) / 4);
  for (int i = threadIdx.x; i < words; i += THREADS)
    s_table[i] = from[i];
  __syncthreads();
  return reinterpret_cast<const Rec *>(s_table);
}

// every warp chunk of the table `tab`, warps taking chunks warp_id,
// warp_id + total warps, ...
template <int THREADS>
__device__ __forceinline__ void batch_chunks(const BatchRegion *tab,
                                             int nregions,
                                             uint32_t total_chunks,
                                             int unpack) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = gridDim.x * (THREADS / 32);
  for (uint32_t c = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5);
       c < total_chunks; c += nwarps) {
    const BatchRegion &r = tab[find_region(tab, nregions, c, lane)];
    switch (r.g.width) {
    case 16: pack_chunk_p<16>(r, c, lane, unpack); break;
    case 8: pack_chunk_p<8>(r, c, lane, unpack); break;
    case 4: pack_chunk_p<4>(r, c, lane, unpack); break;
    case 2: pack_chunk_p<2>(r, c, lane, unpack); break;
    default: pack_chunk_p<1>(r, c, lane, unpack); break;
    }
  }
}

// at least 768 threads per SM: registers are capped at 85 per thread
template <int THREADS>
__global__ void __launch_bounds__(THREADS, (768 + THREADS - 1) / THREADS)
    k_batch(const BatchRegion *__restrict__ regions, int nregions,
            uint32_t total_chunks, int unpack, int staged) {
  extern __shared__ __align__(16) uint32_t s_table[];
  const BatchRegion *tab =
      stage_table<BatchRegion, THREADS>(regions, nregions, staged, s_table);
  batch_chunks<THREADS>(tab, nregions, total_chunks, unpack);
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, (768 + THREADS - 1) / THREADS)
    k_batch_copy(const CopyPair *__restrict__ pairs, int npairs,
                 uint32_t total_chunks, int staged) {
  extern __shared__ __align__(16) uint32_t s_table[];
  const CopyPair *tab =
      stage_table<CopyPair, THREADS>(pairs, npairs, staged, s_table);
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = gridDim.x * (THREADS / 32);
  for (uint32_t c = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5);
       c < total_chunks; c += nwarps) {
    const CopyPair &r = tab[find_region(tab, npairs, c, lane)];
    switch (r.gs.width) {
    case 16: copy_chunk_p<16>(r, c, lane); break;
    case 8: copy_chunk_p<8>(r, c, lane); break;
    case 4: copy_chunk_p<4>(r, c, lane); break;
    case 2: copy_chunk_p<2>(r, c, lane); break;
    default: copy_chunk_p<1>(r, c, lane); break;
    }
  }
}

// read every 16-B word of a buffer larger than the L2 (the autotuner's
// flush between timed launches), leaving clean lines behind
__global__ void k_tune_flush(const uint4 *__restrict__ buf, size_t n,
                             unsigned *__restrict__ sink) {
  unsigned acc = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    const uint4 v = __ldcg(buf + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9e3779b9u)
    *sink = acc;
}

// ---- region classes and launch shapes --------------------------------------

int ilog2(uint32_t x) { return x ? 31 - __builtin_clz(x) : 0; }

// class of a geometry: its width and the log2 of its words per row (7 for
// 128 words or more)
int region_class(const Geometry &g) {
  return 8 * ilog2(g.width) + std::min(7, ilog2(g.wpr));
}

// passes per chunk of a class before any tuning
uint32_t default_passes(int cls) {
  (void)cls;
  return 1;
}

struct Shape {
  int threads = 256;
  int ctas_per_sm = 0; // 0: as many as fit
};

// how many CTAs of a batch kernel fit one SM (cached per kernel and size)
int max_ctas(bool copy, int threads, int smem) {
  static std::mutex mu;
  static std::map<std::tuple<bool, int, int, int>, int> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> l(mu);
  auto key = std::make_tuple(copy, threads, smem, dev);
  auto it = cache.find(key);
  if (it != cache.end())
    return it->second;
  const void *fn = nullptr;
  if (copy)
    fn = threads == 128   ? (const void *)k_batch_copy<128>
         : threads == 512 ? (const void *)k_batch_copy<512>
                          : (const void *)k_batch_copy<256>;
  else
    fn = threads == 128   ? (const void *)k_batch<128>
         : threads == 512 ? (const void *)k_batch<512>
                          : (const void *)k_batch<256>;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) !=
          cudaSuccess ||
      n < 1) {
    cudaGetLastError();
    n = 1;
  }
  cache[key] = n;
  return n;
}

// warp chunks of every record, in order; the total (or more than
// UINT32_MAX when the batch is too large)
template <typename Rec> uint64_t assign_chunks(std::vector<Rec> &recs) {
  uint64_t chunks = 0;
  for (Rec &r : recs) {
    const Geometry &g = geometry_of(r);
    r.chunk_begin = uint32_t(std::min<uint64_t>(chunks, UINT32_MAX));
    const uint64_t per = 32ull * lane_words_of(g.width) * r.passes;
    chunks += (g.total_words + per - 1) / per;
  }
  return chunks;
}

} // namespace

// Launch the pack kernel (or, for pairs, the copy kernel) over a table in
// device memory on `s`.
template <typename Rec>
static int launch_table(const Rec *table, int n, uint32_t total_chunks,
                        int unpack, Shape shape, cudaStream_t s) {
  constexpr bool kCopy = std::is_same<Rec, CopyPair>::value;
  if (n <= 0 || total_chunks == 0)
    return TEMPI_OK;
  const int smem_need = n * int(sizeof(Rec));
  const int staged = smem_need <= kSmemTableBytes ? 1 : 0;
  const int smem = staged ? smem_need : 0;
  const int threads = shape.threads == 128 || shape.threads == 512
                          ? shape.threads
                          : 256;
  const int fit = max_ctas(kCopy, threads, smem);
  const int per_sm = shape.ctas_per_sm > 0 ? std::min(shape.ctas_per_sm, fit)
                                           : fit;
  const uint32_t warps_per_cta = uint32_t(threads / 32);
  const uint32_t want = (total_chunks + warps_per_cta - 1) / warps_per_cta;
  const uint32_t grid = std::max<uint32_t>(
      1, std::min<uint32_t>(want, uint32_t(num_sms()) * uint32_t(per_sm)));
  if constexpr (kCopy) {
    if (threads == 128)
      k_batch_copy<128><<<grid, 128, smem, s>>>(table, n, total_chunks, staged);
    else if (threads == 512)
      k_batch_copy<512><<<grid, 512, smem, s>>>(table, n, total_chunks, staged);
    else
      k_batch_copy<256><<<grid, 256, smem, s>>>(table, n, total_chunks, staged);
  } else {
    if (threads == 128)
      k_batch<128><<<grid, 128, smem, s>>>(table, n, total_chunks, unpack, staged);
    else if (threads == 512)
      k_batch<512><<<grid, 512, smem, s>>>(table, n, total_chunks, unpack, staged);
    else
      k_batch<256><<<grid, 256, smem, s>>>(table, n, total_chunks, unpack, staged);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, kCopy ? "copy batch launch" : "batch launch");
  counters().kernel_launches++;
  set_last_kernel(kCopy ? "batch_copy" : unpack ? "batch_unpack" : "batch_pack");
  return TEMPI_OK;
}

// ---- tuned choices, kept per batch signature -------------------------------

namespace {

struct Tuned {
  Shape shape;
  uint8_t passes[kClasses] = {}; // 0: the class's default
};

std::mutex g_tune_mu;
std::map<uint64_t, Tuned> g_tuned;
bool g_tune_loaded = false;

std::string tune_path() {
  return env().cache_dir + "/tempi_b200_batch_tune.txt";
}

void load_tuned_locked() {
  if (g_tune_loaded)
    return;
  g_tune_loaded = true;
  FILE *f = std::fopen(tune_path().c_str(), "r");
  if (!f)
    return;
  unsigned long long sig;
  int th, cps;
  while (std::fscanf(f, "%llx %d %d", &sig, &th, &cps) == 3) {
    Tuned t;
    t.shape.threads = th;
    t.shape.ctas_per_sm = cps;
    bool ok = true;
    for (int c = 0; c < kClasses && ok; ++c) {
      unsigned u;
      ok = std::fscanf(f, "%u", &u) == 1;
      t.passes[c] = uint8_t(u == 1 || u == 2 || u == 4 ? u : 0);
    }
    if (!ok)
      break;
    g_tuned[sig] = t;
  }
  std::fclose(f);
}

// signature of a batch: what kind of launch it is, and the multiset of its
// records' (class, log2 words)
template <typename Rec> uint64_t signature(const std::vector<Rec> &recs, int unpack) {
  std::vector<uint32_t> keys;
  keys.reserve(recs.size());
  for (const Rec &r : recs) {
    const Geometry &g = geometry_of(r);
    keys.push_back(uint32_t(region_class(g)) << 8 | uint32_t(ilog2(g.total_words)));
  }
  std::sort(keys.begin(), keys.end());
  uint64_t h = 1469598103934665603ull; // FNV-1a
  auto mix = [&](uint32_t v) {
    for (int i = 0; i < 4; ++i) {
      h ^= (v >> (8 * i)) & 0xff;
      h *= 1099511628211ull;
    }
  };
  mix(std::is_same<Rec, CopyPair>::value ? 2u : uint32_t(unpack));
  for (uint32_t k : keys)
    mix(k);
  return h;
}

// the passes of every record from `t` (or the defaults) and the chunk count
template <typename Rec>
uint64_t apply_passes(std::vector<Rec> &recs, const Tuned *t) {
  for (Rec &r : recs) {
    const int c = region_class(geometry_of(r));
    r.passes = t && t->passes[c] ? t->passes[c] : default_passes(c);
  }
  return assign_chunks(recs);
}

} // namespace

struct BatchImpl {
  std::vector<BatchRegion> host;
  BatchRegion *dev = nullptr;
  std::vector<CopyPair> host_pairs; // a copy batch
  CopyPair *dev_pairs = nullptr;
  uint32_t total_chunks = 0;
  int unpack = 0;
  Shape shape;
  Tuned tuned;       // this batch's choices
  bool has_tuned = false;
  uint64_t sig = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

} // namespace tempi

struct tempi_batch {
  tempi::BatchImpl impl;
};

using namespace tempi;

// choices for a new batch: the tuned ones of its signature if any; sets the
// records' passes and chunks, returns the chunk total
template <typename Rec>
static uint64_t plan_batch(BatchImpl &bi, std::vector<Rec> &recs) {
  bi.sig = signature(recs, bi.unpack);
  {
    std::lock_guard<std::mutex> l(g_tune_mu);
    load_tuned_locked();
    auto it = g_tuned.find(bi.sig);
    if (it != g_tuned.end()) {
      bi.tuned = it->second;
      bi.has_tuned = true;
      bi.shape = it->second.shape;
    }
  }
  return apply_passes(recs, bi.has_tuned ? &bi.tuned : nullptr);
}

template <typename Rec>
static int upload(const std::vector<Rec> &recs, Rec **dev) {
  if (recs.empty())
    return TEMPI_OK;
  const size_t bytes = recs.size() * sizeof(Rec);
  cudaError_t e = cudaSuccess;
  if (!*dev)
    e = cudaMalloc(dev, bytes);
  if (e == cudaSuccess)
    e = copy_complete(*dev, recs.data(), bytes);
  if (e != cudaSuccess)
    return cuda_error(e, "batch table upload");
  return TEMPI_OK;
}

extern "C" int tempi_batch_create(const tempi_region *regions, int32_t n,
                                  int32_t unpack, tempi_batch **out) {
  if (!out || n < 0 || (n > 0 && !regions))
    return set_error(TEMPI_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  auto *b = new tempi_batch();
  b->impl.unpack = unpack ? 1 : 0;
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
    b->impl.host.push_back(br);
  }
  const uint64_t chunks = plan_batch(b->impl, b->impl.host);
  if (chunks > UINT32_MAX) {
    delete b;
    return set_error(TEMPI_ERR_ARG, "batch too large");
  }
  b->impl.total_chunks = uint32_t(chunks);
  int err = upload(b->impl.host, &b->impl.dev);
  if (err) {
    cudaFree(b->impl.dev);
    delete b;
    return err;
  }
  *out = b;
  return TEMPI_OK;
}

template <int P> struct StaticPiece {
  BatchRegion r[P];
};

// A batch of up to kParamRegions regions in one launch with its table in the
// kernel's parameters (5.4 KB): each CTA copies it from there into shared
// memory instead of from global memory.  Used by the allocation-free entry
// point (neither a fill kernel nor the fixed array is involved) and by
// small batches at the default launch shape.  256 threads, 3 CTAs per SM by
// the launch bounds.
constexpr int kParamRegions = 32;

template <int P>
__global__ void __launch_bounds__(256, 3)
    k_batch_param(const __grid_constant__ StaticPiece<P> piece, int nregions,
                  uint32_t total_chunks, int unpack) {
  // read in place: a warp's region search reads one field of up to 32
  // entries, its copy loop one entry that every lane shares
  batch_chunks<256>(piece.r, nregions, total_chunks, unpack);
}

// k_batch_param over `n` <= kParamRegions entries of `table` (host memory),
// `per_sm` CTAs per SM (at most 3)
static int launch_param(const BatchRegion *table, int n, uint32_t total_chunks,
                        int unpack, int per_sm, cudaStream_t s) {
  StaticPiece<kParamRegions> piece;
  std::memcpy(piece.r, table, size_t(n) * sizeof(BatchRegion));
  const uint32_t grid = std::max<uint32_t>(
      1, std::min<uint32_t>((total_chunks + 7) / 8,
                            uint32_t(num_sms()) * uint32_t(per_sm)));
  k_batch_param<kParamRegions><<<grid, 256, 0, s>>>(piece, n, total_chunks,
                                                     unpack);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return cuda_error(e, "batch launch");
  counters().kernel_launches++;
  return TEMPI_OK;
}

// `direct`: a launch of its own (tempi_batch_launch).  There a small table at
// a 256-thread shape rides in the kernel's parameters instead of being read
// from device memory by every CTA (measured on the 256^3 halo: 11.3 against
// 12.0-12.3 us by events, 7.3-7.6 against 7.6-7.9 us in-kernel).  Graph
// captures and the tuner's timings keep the table in device memory: a
// replayed kernel node with 5.4 KB of parameters measured 1-2 us slower.
static int batch_launch(tempi_batch *b, cudaStream_t s, bool direct) {
  BatchImpl &bi = b->impl;
  if (!bi.host_pairs.empty())
    return launch_table(bi.dev_pairs, int(bi.host_pairs.size()),
                        bi.total_chunks, 0, bi.shape, s);
  const int n = int(bi.host.size());
  if (direct && n > 0 && n <= kParamRegions && bi.total_chunks > 0 &&
      (bi.shape.threads == 0 || bi.shape.threads == 256) &&
      bi.shape.ctas_per_sm <= 3) {
    const int per_sm = bi.shape.ctas_per_sm > 0 ? bi.shape.ctas_per_sm : 3;
    const int err = launch_param(bi.host.data(), n, bi.total_chunks, bi.unpack,
                                 per_sm, s);
    if (!err)
      set_last_kernel(bi.unpack ? "batch_unpack" : "batch_pack");
    return err;
  }
  return launch_table(bi.dev, n, bi.total_chunks, bi.unpack, bi.shape, s);
}

// Copy pairs for `regions`, each at the default passes of its class; empty
// regions are dropped.  Returns the chunk count through *chunks_out.
static int build_pairs(const tempi_copy_region *regions, int32_t n,
                       std::vector<CopyPair> *pairs, uint64_t *chunks_out) {
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
    pairs->push_back(cp);
  }
  *chunks_out = apply_passes(*pairs, nullptr);
  if (*chunks_out > UINT32_MAX)
    return set_error(TEMPI_ERR_ARG, "batch too large");
  return TEMPI_OK;
}

extern "C" int tempi_batch_create_copy(const tempi_copy_region *regions,
                                       int32_t n, tempi_batch **out) {
  if (!out || n < 0 || (n > 0 && !regions))
    return set_error(TEMPI_ERR_ARG, "bad copy batch arguments");
  *out = nullptr;
  auto *b = new tempi_batch();
  uint64_t chunks = 0;
  int err = build_pairs(regions, n, &b->impl.host_pairs, &chunks);
  if (!err) {
    chunks = plan_batch(b->impl, b->impl.host_pairs);
    if (chunks > UINT32_MAX)
      err = set_error(TEMPI_ERR_ARG, "batch too large");
  }
  if (!err) {
    b->impl.total_chunks = uint32_t(chunks);
    err = upload(b->impl.host_pairs, &b->impl.dev_pairs);
  }
  if (err) {
    cudaFree(b->impl.dev_pairs);
    delete b;
    return err;
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
  static Shape shape;
  static uint64_t on_device_sig = 0;
  std::lock_guard<std::mutex> l(mu);
  uint64_t chunks = 0;
  int err = build_pairs(regions, n, &pairs, &chunks);
  if (err || pairs.empty())
    return err;
  // a batch of a tuned signature takes the tuned choices
  const uint64_t sig = signature(pairs, 0);
  if (sig != on_device_sig || on_device.size() != pairs.size()) {
    std::lock_guard<std::mutex> t(g_tune_mu);
    load_tuned_locked();
    auto it = g_tuned.find(sig);
    shape = it != g_tuned.end() ? it->second.shape : Shape{};
    if (it != g_tuned.end())
      chunks = apply_passes(pairs, &it->second);
  } else {
    // same signature as the table on the device: same choices
    for (size_t i = 0; i < pairs.size(); ++i)
      pairs[i].passes = on_device[i].passes;
    chunks = assign_chunks(pairs);
  }
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
    on_device_sig = sig;
  }
  return launch_table(table, int(pairs.size()), uint32_t(chunks), 0, shape, s);
}

} // namespace tempi

extern "C" int tempi_batch_launch(tempi_batch *b, void *stream) {
  if (!b)
    return set_error(TEMPI_ERR_ARG, "null batch");
  return batch_launch(b, static_cast<cudaStream_t>(stream), true);
}

static void drop_graph(BatchImpl &bi) {
  if (bi.exec) {
    cudaGraphExecDestroy(bi.exec);
    cudaGraphDestroy(bi.graph);
    bi.exec = nullptr;
    bi.graph = nullptr;
  }
}

extern "C" int tempi_batch_capture(tempi_batch *b, void *stream) {
  if (!b)
    return set_error(TEMPI_ERR_ARG, "null batch");
  BatchImpl &bi = b->impl;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  drop_graph(bi);
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return cuda_error(e, "begin capture");
  int err = batch_launch(b, s, false);
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

// ---- the autotuner ----------------------------------------------------------

namespace {

// median device time (ms) of `reps` launches of the batch as configured,
// the L2 flushed before each
float time_batch(tempi_batch *b, cudaStream_t s, const uint4 *flush,
                 size_t flush_words, unsigned *sink, cudaEvent_t e0,
                 cudaEvent_t e1, int reps, int *err) {
  std::vector<float> ts;
  for (int r = 0; r < reps && !*err; ++r) {
    k_tune_flush<<<num_sms() * 8, 256, 0, s>>>(flush, flush_words, sink);
    cudaEventRecord(e0, s);
    *err = batch_launch(b, s, false);
    cudaEventRecord(e1, s);
    if (cudaEventSynchronize(e1) != cudaSuccess) {
      *err = cuda_error(cudaGetLastError(), "tuning launch");
      break;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    ts.push_back(ms);
  }
  if (ts.empty())
    return 1e30f;
  std::sort(ts.begin(), ts.end());
  return ts[ts.size() / 2];
}

// re-plan the records with `t`, upload the table
int replan(tempi_batch *b, const Tuned &t) {
  BatchImpl &bi = b->impl;
  bi.shape = t.shape;
  uint64_t chunks;
  int err;
  if (!bi.host_pairs.empty()) {
    chunks = apply_passes(bi.host_pairs, &t);
    err = upload(bi.host_pairs, &bi.dev_pairs);
  } else {
    chunks = apply_passes(bi.host, &t);
    err = upload(bi.host, &bi.dev);
  }
  if (chunks > UINT32_MAX)
    return set_error(TEMPI_ERR_ARG, "batch too large");
  bi.total_chunks = uint32_t(chunks);
  return err;
}

template <typename Rec> std::vector<int> classes_of(const std::vector<Rec> &recs) {
  std::vector<int> out;
  for (const Rec &r : recs)
    out.push_back(region_class(geometry_of(r)));
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

} // namespace

extern "C" int tempi_batch_tune(tempi_batch *b, void *stream, int32_t reps) {
  if (!b)
    return set_error(TEMPI_ERR_ARG, "null batch");
  BatchImpl &bi = b->impl;
  if (bi.host.empty() && bi.host_pairs.empty())
    return TEMPI_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  reps = std::max(1, std::min(50, int(reps)));
  drop_graph(bi);
  int dev = 0, l2 = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess)
    l2 = 128 << 20;
  const size_t flush_bytes = (size_t(l2) * 2 + 15) & ~size_t(15);
  void *flush = nullptr;
  unsigned *sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t ce = cudaMalloc(&flush, flush_bytes + 16);
  if (ce == cudaSuccess)
    ce = cudaMemsetAsync(flush, 0, flush_bytes + 16, s);
  if (ce == cudaSuccess)
    ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess)
    ce = cudaEventCreate(&e1);
  int err = ce == cudaSuccess ? TEMPI_OK : cuda_error(ce, "tuning set-up");
  sink = reinterpret_cast<unsigned *>(static_cast<char *>(flush) + flush_bytes);
  const uint4 *fl = static_cast<const uint4 *>(flush);
  const size_t fw = flush_bytes / 16;
  Tuned best = bi.has_tuned ? bi.tuned : Tuned{};
  const std::vector<int> cls = !bi.host_pairs.empty() ? classes_of(bi.host_pairs)
                                                      : classes_of(bi.host);
  float t_best = 1e30f;
  if (!err) {
    err = replan(b, best);
    if (!err) {
      time_batch(b, s, fl, fw, sink, e0, e1, 2, &err); // warm
      t_best = time_batch(b, s, fl, fw, sink, e0, e1, reps, &err);
    }
  }
  // each class's passes in turn, the others held
  for (int c : cls) {
    for (int p : kPassChoices) {
      if (err)
        break;
      Tuned t = best;
      t.passes[c] = uint8_t(p);
      if ((best.passes[c] ? best.passes[c] : default_passes(c)) == uint32_t(p))
        continue;
      err = replan(b, t);
      const float tt = err ? 1e30f : time_batch(b, s, fl, fw, sink, e0, e1, reps, &err);
      if (tt < t_best) {
        t_best = tt;
        best = t;
      }
    }
  }
  // then the launch shape
  for (int th : {128, 256, 512}) {
    for (int cps : {1, 2, 3, 4, 6, 8, 12, 16}) {
      if (err)
        break;
      Tuned t = best;
      t.shape.threads = th;
      t.shape.ctas_per_sm = cps;
      if (cps > max_ctas(!bi.host_pairs.empty(), th, 0) ||
          (th == best.shape.threads && cps == best.shape.ctas_per_sm))
        continue;
      err = replan(b, t);
      const float tt = err ? 1e30f : time_batch(b, s, fl, fw, sink, e0, e1, reps, &err);
      if (tt < t_best) {
        t_best = tt;
        best = t;
      }
    }
  }
  if (!err)
    err = replan(b, best);
  if (e0)
    cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
  cudaStreamSynchronize(s);
  cudaFree(flush);
  if (err)
    return err;
  for (int c = 0; c < kClasses; ++c) // record resolved choices
    if (!best.passes[c])
      best.passes[c] = uint8_t(default_passes(c));
  bi.tuned = best;
  bi.has_tuned = true;
  std::lock_guard<std::mutex> l(g_tune_mu);
  load_tuned_locked();
  g_tuned[bi.sig] = best;
  if (FILE *f = std::fopen(tune_path().c_str(), "a")) {
    std::fprintf(f, "%llx %d %d", (unsigned long long)bi.sig, best.shape.threads,
                 best.shape.ctas_per_sm);
    for (int c = 0; c < kClasses; ++c)
      std::fprintf(f, " %u", unsigned(best.passes[c]));
    std::fprintf(f, "\n");
    std::fclose(f);
  }
  return TEMPI_OK;
}

extern "C" int tempi_batch_config(const tempi_batch *b, int32_t *threads,
                                  int32_t *ctas_per_sm, int32_t *classes,
                                  int32_t *passes, int32_t max_classes) {
  if (!b)
    return -set_error(TEMPI_ERR_ARG, "null batch");
  const BatchImpl &bi = b->impl;
  if (threads)
    *threads = bi.shape.threads;
  if (ctas_per_sm)
    *ctas_per_sm = bi.shape.ctas_per_sm;
  std::vector<std::pair<int, int>> cu;
  auto add = [&](const Geometry &g, uint32_t u) { // u: passes
    const int c = region_class(g);
    for (auto &p : cu)
      if (p.first == c)
        return;
    cu.push_back({c, int(u)});
  };
  for (const BatchRegion &r : bi.host)
    add(r.g, r.passes);
  for (const CopyPair &r : bi.host_pairs)
    add(r.gs, r.passes);
  std::sort(cu.begin(), cu.end());
  int k = 0;
  for (auto &p : cu) {
    if (k >= max_classes)
      break;
    if (classes)
      classes[k] = p.first;
    if (passes)
      passes[k] = p.second;
    ++k;
  }
  return k;
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
// A table of up to kParamRegions entries is passed BY VALUE as the batch
// kernel's own parameter (k_batch_param): one launch, the array untouched.
// A larger table reaches the array without a host-to-device copy: the host
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
    if (pass == 1 && used <= kParamRegions) { // pass 0 left them all in piece
      if (used == 0)
        return TEMPI_OK;
      err = launch_param(piece.r, used, uint32_t(chunks), unpack ? 1 : 0, 3, s);
      if (!err)
        set_last_kernel(unpack ? "batch_unpack_static" : "batch_pack_static");
      return err;
    }
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
      br.passes = default_passes(region_class(br.g));
      br.chunk_begin = uint32_t(chunks);
      const uint64_t per = 32ull * lane_words_of(br.g.width) * br.passes;
      chunks += (br.g.total_words + per - 1) / per;
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
  err = launch_table(table, used, uint32_t(chunks), unpack ? 1 : 0, Shape{}, s);
  if (err)
    return err;
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
