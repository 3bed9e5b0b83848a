// Host runtime of the interposer: environment knobs, type cache, device
// stream, slab allocators and event pool.
#pragma once

#include "internal.hpp"
#include "symbols.hpp"

#include <cstddef>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace tempi {

// ---- environment (reference include/env.hpp:10-37, src/internal/env.cpp) --
enum class Method { AUTO = 0, DEVICE = 1, ONESHOT = 2, STAGED = 3 };
enum class Contiguous { NONE, AUTO, STAGED };
enum class Dispatch { LEARNED, TABLE, EXHAUSTIVE, HEURISTIC };
// the reference's MPI_Alltoallv methods (src/internal/alltoallv_impl.cpp)
enum class Alltoallv { AUTO, STAGED, REMOTE_FIRST, ISIR_STAGED, ISIR_REMOTE_STAGED, NONE };

struct Env {
  bool disable = false;      // TEMPI_DISABLE
  bool no_pack = false;      // TEMPI_NO_PACK
  bool no_type_commit = false; // TEMPI_NO_TYPE_COMMIT
  Method datatype = Method::AUTO; // TEMPI_DATATYPE_{ONESHOT,DEVICE,STAGED,AUTO}
  Contiguous contiguous = Contiguous::NONE; // TEMPI_CONTIGUOUS_{STAGED,AUTO}
  Dispatch dispatch = Dispatch::LEARNED; // TEMPI_DISPATCH=learned|table|exhaustive|heuristic
  std::string cache_dir;     // TEMPI_CACHE_DIR
  double wait_timeout_s = 30; // TEMPI_WAIT_TIMEOUT_S: bound on MPI_Wait polling
  // TEMPI_HOST_LINK=kernel: contiguous runs between pinned host buffers go
  // through the kernels too, instead of the copy-engine pipeline
  bool host_link_dma = true;
  // TEMPI_HOST_LINK_CHUNK_KB: chunk size of the copy-engine pipeline for
  // contiguous runs, a multiple of 256 KiB (0: the built-in rule)
  long host_link_chunk_kb = 0;
  // TEMPI_TEST_STAGED_SHORTFALL=<bytes>: the staged kernels' barriers expect
  // that many bytes per chunk beyond what their copies deliver, so every
  // bounded wait runs out (about a second) and the give-up path reports a
  // timeout.  For tests of that path only; 0 (the default) in normal use.
  int staged_shortfall = 0;
  // TEMPI_SLAB_CACHE_MB: bytes of freed slabs kept for reuse, per memory
  // space; freed slabs beyond it go back to CUDA.  Large enough by default
  // that a loop of 1 GiB self-sends (a send slab and a receive slab) reuses
  // its slabs instead of pinning (or allocating) gigabytes for every message.
  long slab_cache_mb = 4096;
  // TEMPI_ALLTOALLV_{STAGED,REMOTE_FIRST,ISIR_STAGED,ISIR_REMOTE_STAGED},
  // TEMPI_NO_ALLTOALLV (reference src/internal/env.cpp:35-49)
  Alltoallv alltoallv = Alltoallv::AUTO;
  // TEMPI_RANKS_PER_NODE=k: ranks r and s share a node when r/k == s/k
  // (0, the default: every rank of the job shares one node)
  int ranks_per_node = 0;
};
const Env &env();
void read_env(); // re-read the environment (MPI_Init does this)

// ---- canonicaliser ---------------------------------------------------------
// Describe `t` as a strided block; TEMPI_ERR_UNSUPPORTED when it is not one.
int canonicalize(MPI_Datatype t, tempi_desc *out);

// ---- type cache (reference include/type_cache.hpp:23-30) ------------------
struct TypeRecord {
  tempi_desc desc{};
  bool packable = false; // desc describes the type and a kernel handles it
  // method chosen per packed byte count (reference SendRecvND's
  // modelChoiceCache_, sender.cpp:259-277)
  std::unordered_map<int64_t, Method> methods;
  // kernel configuration chosen per (object count, typed-buffer kind,
  // packed-buffer kind); -1 = the fixed rules
  std::unordered_map<uint64_t, int> configs;
};

// Returns nullptr when the type is unknown.  The pointer stays valid until
// the type is released.
TypeRecord *find_type(MPI_Datatype t);
TypeRecord *commit_type(MPI_Datatype t);
void release_type(MPI_Datatype t);

// ---- device state ---------------------------------------------------------
// Lazily creates TEMPI's non-blocking stream on the current device
// (reference kernStream, src/internal/streams.cpp:19-28).
cudaStream_t pack_stream();
// A second non-blocking stream, for work that runs beside pack_stream()
// (the copy-engine pipeline's device-to-host half).
cudaStream_t link_stream();
bool cuda_available();

// Where a pointer lives.  device_ptr is what a kernel should use.
struct PtrInfo {
  bool device_accessible = false; // device memory, managed, or mapped host
  bool is_device = false;         // device memory proper
  bool is_host = false;           // pinned host memory (not managed)
  void *device_ptr = nullptr;
};
PtrInfo classify(const void *p);

// ---- slab allocators (reference include/allocator_slab.hpp) ---------------
// Power-of-two size classes up to 64 MiB with O(1) free lists, blocks
// rounded to 2 MiB above that; freed blocks are kept while the cached bytes
// stay within TEMPI_SLAB_CACHE_MB per space.  Device slabs come from
// cudaMalloc; host slabs from cudaHostAlloc(Mapped|Portable), so kernels can
// write them directly (the ONE_SHOT path).  slab_alloc returns null when the
// allocation fails (tempi_last_error says why).
enum class Space { DEVICE, HOST_MAPPED };
void *slab_alloc(Space s, size_t bytes);
void slab_free(Space s, void *p);
// test hook behind TEMPI_TEST_FAIL_SLAB: the n-th slab_alloc from now fails
// (0: none)
void slab_test_fail_after(int64_t n);
void slab_release_all();

// ---- copy-engine path between pinned host buffers -------------------------
// Bytes of the one contiguous run that `incount` objects of `d` describe, or
// -1 when they describe more than one run.
int64_t contiguous_run(const tempi_desc &d, int64_t incount);
// Smallest run worth the copy-engine pipeline.
constexpr int64_t kHostLinkMinBytes = int64_t(8) << 20;
// Copy `n` bytes from pinned host `src` to pinned host `dst` through device
// staging with the copy engines, both link directions busy at once; enqueued
// on `s` and on link_stream(), and synchronised before it returns.
int host_link_copy(void *dst, const void *src, size_t n, cudaStream_t s);
// Narrowest row worth the 2-D copy-engine pipeline (used for unpacks).
// Measured on the sweep's host-to-host points: 256-B rows at byte 28 unpack
// in 2.61 ms instead of 3.25 ms by the kernels, 1-KiB rows gain 2-7 %, while
// 64-B rows at byte 120 unpack slower (1.52 against 1.33 ms) although a lone
// 2-D copy of them runs at 14-18 GB/s: in the pipeline the two directions
// overlap poorly.
constexpr int64_t kHostLinkMinRow = 128;
// `incount` objects of `d` as `rows` rows of `width` bytes at `pitch`, when
// they have exactly one strided dimension with rows of kHostLinkMinRow bytes
// or more (and at most one staging chunk) that do not overlap.
struct HostRows {
  int64_t rows, width, pitch;
};
bool host_rows(const tempi_desc &d, int64_t incount, HostRows *out);
// Copy `rows` rows of `width` bytes from pinned host `src` (row pitch
// `spitch`) to pinned host `dst` (row pitch `dpitch`) through device staging,
// as host_link_copy does; each chunk's host side is one 2-D copy.
int host_link_rows(void *dst, int64_t dpitch, const void *src, int64_t spitch,
                   int64_t width, int64_t rows, cudaStream_t s);

// ---- event pool (reference src/internal/events.cpp:17-86) -----------------
cudaEvent_t event_acquire();
void event_release(cudaEvent_t e);
void events_release_all();

} // namespace tempi
