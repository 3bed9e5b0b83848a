/* tempi_b200.h -- the drop-in boundary of libtempi_b200.so.

   Two surfaces:

   1. Interposed MPI entry points.  libtempi_b200.so exports these MPI-3.1
      functions with their standard C signatures (declared by the MPI
      library's own mpi.h, so they are listed here only as a comment).  An
      application links libtempi_b200.so ahead of its MPI library, or
      preloads it; each call reaches the real MPI through
      dlsym(RTLD_NEXT, name) when TEMPI cannot or should not handle it.

        MPI_Init          replaces reference src/init.cpp:22-67
        MPI_Init_thread   replaces reference src/init_thread.cpp:22-65
        MPI_Finalize      replaces reference src/finalize.cpp:20-46
        MPI_Type_commit   replaces reference src/type_commit.cpp:16-114
        MPI_Type_free     replaces reference src/type_free.cpp:14-26
        MPI_Pack          replaces reference src/pack.cpp:28-68
        MPI_Unpack        replaces reference src/unpack.cpp:20-60
        MPI_Send          replaces reference src/send.cpp + src/internal/send.cpp:21-53
        MPI_Recv          replaces reference src/recv.cpp:19-52
        MPI_Isend         replaces reference src/isend.cpp + src/internal/isend.cpp:15-45
        MPI_Irecv         replaces reference src/irecv.cpp + src/internal/irecv.cpp:15-44
        MPI_Wait          replaces reference src/wait.cpp:11-16
        MPI_Neighbor_alltoallw
                          replaces reference src/neighbor_alltoallw.cpp:11-17
                          + src/internal/neighbor_alltoallw.cpp:19-85
        MPI_Alltoallv     replaces reference src/alltoallv.cpp:14-66
                          + src/internal/alltoallv_impl.cpp:21-258

      Signatures are those of include/symbols.hpp in the reference
      (PARAMS_MPI_* macros, lines 10-178).

   2. The thin kernel ABI below: plain pointers and sizes, no MPI or torch
      types, every function returning 0 (TEMPI_OK) or a TEMPI_ERR_* code.
      The MPI layer is built on it; tests, benchmarks and non-MPI callers use
      it directly.
*/
#ifndef TEMPI_B200_H
#define TEMPI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TEMPI_OK 0
#define TEMPI_ERR_ARG 1         /* bad argument or descriptor */
#define TEMPI_ERR_CUDA 2        /* a CUDA call failed (message via tempi_last_error) */
#define TEMPI_ERR_UNSUPPORTED 3 /* type cannot be described as a strided block */
#define TEMPI_ERR_TIMEOUT 4     /* a bounded wait ran out */
#define TEMPI_ERR_NO_MEM 5
#define TEMPI_ERR_TRUNCATE 6    /* output buffer too small */
#define TEMPI_ERR_NOT_BUILT 7   /* compiled without the kernel */

#define TEMPI_MAX_DIMS 4

/* A canonical strided block: the bytes of one object are
     for i[nd-1] .. for i[0]: copy `block` bytes from
       origin + start + sum_k i[k]*strides[k]
   in that order (counts[0]/strides[0] vary fastest).  Object j of a
   multi-object call starts at origin + j*extent.  `align` is the largest
   power of two <= 16 dividing start, block, every stride and extent.  The
   same information as the reference's StridedBlock
   (include/strided_block.hpp:12-67), whose counts[0] is the block length. */
typedef struct tempi_desc {
  int64_t start;
  int64_t extent;
  int64_t block;
  int64_t size; /* packed bytes of one object = block * prod(counts) */
  int32_t ndims;
  int32_t align;
  int64_t counts[TEMPI_MAX_DIMS];
  int64_t strides[TEMPI_MAX_DIMS];
} tempi_desc;

/* Kernel choice for one launch.  Zero fields mean "let the library pick".
   kernel: 0 auto, 1 word kernel (a thread per vector word), 2 row kernel (a
   warp per row), 3 shift kernel (a group of `unroll` = 4/8/16/32 lanes per
   row, 16-B accesses at any alignment), 4 staged kernels (chunks of the packed
   stream move through shared memory by bulk asynchronous copies: a pack
   gathers 16 KB chunks' row pieces in and writes each chunk out with one
   bulk store, and needs width 16 throughout; an unpack needs a 16-B aligned
   packed base, and for 16-B aligned rows of 512 B or more (or one
   contiguous run) pulls 16 KB chunks in and writes their row pieces out
   with bulk stores, else pulls 8 KB chunks in and scatters them by vector
   words.  Every staged launch needs a packed size that is a multiple
   of 16 and device memory on both sides; calls that do not qualify take the
   automatic rules).  width: vector bytes for kernels 1, 2 and 4
   (1,2,4,8,16; never above what the alignment proof allows).
   blocks_per_sm: resident blocks per SM the grid is sized for (kernel 4:
   1..8; the 16 KB-chunk kernels run one warp per block, one block per SM
   for 96 MiB or more and 3 below, and blocks_per_sm only lowers that; the
   scattering unpack defaults to 3 for aligned copies of 32 MiB or more,
   else 8). */
typedef struct tempi_config {
  int32_t kernel;
  int32_t width;
  int32_t threads;
  int32_t unroll;
  int32_t blocks_per_sm;
  int32_t reserved;
} tempi_config;

/* ---- strided pack / unpack (reference Packer::pack/unpack_async,
        include/packer.hpp:14-49; kernels pack_kernels.cuh:64-120, 350-433) */

/* Pack `incount` objects described by `d` from `origin` (device-accessible)
   into `packed` (device-accessible, incount*d->size bytes).  Asynchronous
   on `stream` (a cudaStream_t; 0 = legacy default stream). */
int tempi_pack(const tempi_desc *d, const void *origin, int64_t incount,
               void *packed, const tempi_config *cfg, void *stream);
/* Inverse of tempi_pack; bytes of `origin` outside the description are
   never written. */
int tempi_unpack(const tempi_desc *d, const void *packed, int64_t incount,
                 void *origin, const tempi_config *cfg, void *stream);

/* Canonicalise a committed MPI datatype handle (MPI_Datatype passed as an
   integer or pointer-sized value) the way MPI_Type_commit does.  Returns
   TEMPI_ERR_UNSUPPORTED if the type is not a strided block. */
int tempi_describe(int64_t datatype, tempi_desc *out);

/* ---- batched pack: many (object, region) pairs in one launch -------------
   A region is `incount` objects of a strided block whose typed buffer has
   its origin at `origin`, packed to (or unpacked from) `packed`.  The table
   lives in device memory, so a captured graph replays with new data and no
   re-capture.  No counterpart in the reference, which packs one object per
   launch (src/pack.cpp:56). */
typedef struct tempi_region {
  void *origin; /* typed buffer (read by pack, written by unpack) */
  void *packed; /* contiguous bytes of this region */
  tempi_desc desc;
  int64_t incount;
} tempi_region;

typedef struct tempi_batch tempi_batch; /* opaque */

int tempi_batch_create(const tempi_region *regions, int32_t n, int32_t unpack,
                       tempi_batch **out);
int tempi_batch_launch(tempi_batch *b, void *stream);
/* capture one launch into a CUDA graph and replay it with tempi_batch_replay */
int tempi_batch_capture(tempi_batch *b, void *stream);
int tempi_batch_replay(tempi_batch *b, void *stream);
int tempi_batch_destroy(tempi_batch *b);

/* The batch autotuner.  A batch launch is one kernel over warp chunks; its
   choices are the launch shape (threads per block 128/256/512, blocks per
   SM) and, per region class (class = 8 * log2(width) + min(7, log2(words
   per row)): the proven vector width and the row length), the passes of a
   warp over one chunk (1, 2 or 4: the chunk size).  tempi_batch_tune times
   the batch on `stream` (`reps` launches per candidate, the L2 flushed
   before each; it allocates and frees a flush buffer of twice the L2),
   keeps the fastest choices for this batch, and remembers them for every
   later batch with the same signature (the same region classes and sizes)
   in this process and in TEMPI_CACHE_DIR/tempi_b200_batch_tune.txt.  It
   drops a captured graph: capture again after tuning.  The reference has
   no counterpart (it packs one object per launch). */
int tempi_batch_tune(tempi_batch *b, void *stream, int32_t reps);
/* The choices a batch launches with: threads per block, blocks per SM (0:
   as many as fit), and for each region class present (ascending, at most
   max_classes) its passes.  Returns the number of classes written, or a
   negative TEMPI_ERR_* code. */
int tempi_batch_config(const tempi_batch *b, int32_t *threads,
                       int32_t *ctas_per_sm, int32_t *classes,
                       int32_t *passes, int32_t max_classes);

/* Batched exchange: every region is copied from one strided layout straight
   into another (typed -> typed, no packed buffer between them), all regions
   in one launch, through the same batch handle (launch / capture / replay /
   destroy above).  The bytes of `src_count` objects of `src_desc` at
   `src_origin`, in type-map order, go to the bytes of `dst_count` objects of
   `dst_desc` at `dst_origin`, in type-map order; both must describe the same
   number of bytes.  This is a pack, a transfer and an unpack fused into one
   kernel: a halo exchange with a periodic neighbour that is the same rank
   (each send region lands in the opposite ghost region), and the local part
   of MPI_Neighbor_alltoallw.  Replaces the pack -> MPI_Neighbor_alltoallv ->
   unpack sequence of the reference's bin/bench_halo_exchange.cpp:560-625
   and the Isend/Irecv pairs of src/internal/neighbor_alltoallw.cpp:19-85
   for edges that stay on this GPU. */
typedef struct tempi_copy_region {
  const void *src_origin;
  void *dst_origin;
  tempi_desc src_desc;
  tempi_desc dst_desc;
  int64_t src_count;
  int64_t dst_count;
} tempi_copy_region;

int tempi_batch_create_copy(const tempi_copy_region *regions, int32_t n,
                            tempi_batch **out);

/* Batched pack (unpack != 0: unpack) of `n` regions in one launch on
   `stream`, allocating nothing.  No counterpart in the reference.  For
   callers that cannot allocate device memory where they pack -- a step of
   a latency-critical loop (cudaMalloc can synchronise the whole device), or
   an application whose memory pool already owns the GPU's memory -- the
   region table is kept in a fixed array inside the library instead of
   memory from cudaMalloc.  At most 1024 regions per call (larger n returns
   TEMPI_ERR_ARG, and so does any invalid region, before anything is
   launched).  Every GPU that loads the library holds that 168 KiB array
   until exit.  A table of up to 32 (non-empty) regions travels in the
   batch kernel's own parameters (one launch, the array untouched); a
   larger one reaches the array through the parameters of small fill
   kernels (one per 128 regions) launched on `stream` ahead of the batch
   kernel.  Either way the call copies nothing from host memory and never
   waits for earlier work on the stream.  The first call on a device, with
   that device current, looks up the array's device address, so make it
   before any stream capture; that address is not looked up again after a
   cudaDeviceReset.  All calls share the array: calls whose launches can
   overlap on the GPU race on it. */
int tempi_batch_run_static(const tempi_region *regions, int32_t n,
                           int32_t unpack, void *stream);

/* ---- learned cost model --------------------------------------------------
   Replaces the reference's measured-parameter tables (perf.json;
   src/internal/measure_system.cpp:106-299, include/measure_system.hpp:30-106)
   as the predictor behind the choice of kernel configuration and transfer
   method.  An FP32 perceptron 12 -> 64 -> 64 -> 23 (ReLU), an ensemble of
   `members` copies; one member's parameters are TEMPI_MLP_PARAMS floats laid
   out W1[64][12] b1[64] W2[64][64] b2[64] W3[23][64] b3[23].  All pointers
   below are device memory. */
#define TEMPI_MLP_IN 12
#define TEMPI_MLP_HIDDEN 64
#define TEMPI_MLP_OUT 23
#define TEMPI_MLP_PARAMS 6487
#define TEMPI_MLP_MEMBERS 5
/* entries of tempi_measure's output: the model's outputs, then the fixed
   rules' pack and unpack */
#define TEMPI_MEASURED 25

/* seeded uniform(+-1/sqrt(fan_in)) weights, zero biases */
int tempi_mlp_init(float *params, int members, uint64_t seed);
/* Adam on the masked mean squared error of y (n x 23; mask 1 = observed,
   NULL = all observed) from x (n x 12); one CTA per member, mini-batches of
   `batch` <= 64 rows drawn with replacement.  loss_out (optional,
   members x epochs) receives each epoch's mean loss. */
int tempi_mlp_train(float *params, int members, const float *x,
                    const float *y, const float *mask, int n, int epochs,
                    int batch, float lr, uint64_t seed, float *loss_out,
                    void *stream);
/* out[member][row][23] for n rows of x */
int tempi_mlp_predict(const float *params, int members, const float *x, int n,
                      float *out, void *stream);
/* gradient (TEMPI_MLP_PARAMS floats) and loss of one member on rows
   [0, n), n <= 64: checked against a float64 CPU restatement */
int tempi_mlp_grad(const float *params, const float *x, const float *y,
                   const float *mask, int n, float *grad, float *loss,
                   void *stream);

/* ---- dispatch -------------------------------------------------------------
   The model's twenty-three outputs are log2 microseconds of: [0..9] a pack
   of the objects with kernel configuration 0..9 (word kernel with 256, 512,
   128 threads; row kernel; shift kernel with 4, 8, 16, 32 lanes per row;
   staged kernel with 3 and with 8 CTAs per SM), [10..19] an unpack with
   configuration 0..9, [20..22] a self-send round trip (MPI_Send + MPI_Recv)
   by DEVICE, ONE_SHOT, STAGED.  Pack and unpack are
   chosen separately: they can prefer different kernels (a shift kernel packs
   misaligned rows from host memory well, but its partial end stores make it
   a poor unpacker into host memory).  `typed_host` / `packed_host`: the
   typed or packed buffer is in mapped pinned host memory. */

/* the twelve model inputs for `incount` objects of `d` */
int tempi_features(const tempi_desc *d, int64_t incount, int typed_host,
                   int packed_host, float *out12);
/* time every candidate on scratch buffers shaped like the object (the
   exhaustive autotuner; reference bin/measure_system.cpp,
   src/internal/measure_system.cu:381-610).  what: bit 0 configurations,
   bit 1 methods.  times_us[TEMPI_MEASURED]: the twenty-three candidates above,
   then the fixed rules' (no model) pack and unpack; NaN where not
   measured. */
int tempi_measure(const tempi_desc *d, int64_t incount, int typed_host,
                  int packed_host, int what, int reps, float *times_us);
/* load a trained cost model and/or measured tables (NULL to skip one);
   MPI_Init loads them from TEMPI_CACHE_DIR or tempi_b200/models/ */
int tempi_dispatch_load(const char *model_path, const char *table_path);
/* what a policy would choose.  mode 0: learned, 1: the reference's
   perf-table model restated (method only), 2: the fixed rules.
   pack_config / unpack_config: 0..9 or -1 (fixed rules); method: 1 DEVICE,
   2 ONE_SHOT, 3 STAGED.  predicted/spread (optional, 23 each): ensemble mean
   and standard deviation, log2 microseconds (mode 0 only). */
int tempi_dispatch_choose(const tempi_desc *d, int64_t incount,
                          int typed_host, int packed_host, int mode,
                          int *pack_config, int *unpack_config, int *method,
                          float *predicted, float *spread);

/* The table model's interpolation (reference measure_system.cpp:181-299):
   cols <= 0: a 1-D table, entry i = 2^i bytes; otherwise rows x cols, entry
   [i][j] = 2^(2i+6) bytes packed from blocks of 2^j bytes. */
double tempi_table_interp(const double *table, int rows, int cols,
                          int64_t bytes, int64_t block);

/* ---- runtime ------------------------------------------------------------ */
/* TEMPI's internal non-blocking stream (a cudaStream_t) on which the MPI
   entry points launch (reference kernStream, src/internal/streams.cpp:16-28).
   Exposed so callers can order or time work against it. */
void *tempi_stream(void);
/* re-read the TEMPI_* environment knobs (MPI_Init reads them once) */
int tempi_reload_env(void);

/* ---- diagnostics -------------------------------------------------------- */
const char *tempi_last_error(void);
/* number of kernel launches issued by this library since load */
int64_t tempi_kernel_launches(void);
/* name of the kernel variant the last tempi_pack/unpack used */
const char *tempi_last_kernel(void);
/* value of a named counter (reference include/counters.hpp groups):
   "kernel_launches", "packs", "unpacks", "pack_bytes", "unpack_bytes",
   "lib_pack", "lib_unpack", "cached_types", "send_device", "send_oneshot",
   "send_staged", "send_lib", "recv_device", "recv_oneshot", "recv_staged",
   "recv_lib", "isend_managed", "irecv_managed", "dispatch_hit",
   "dispatch_miss", "dispatch_measured" (kernel choices made by timing the
   candidates: the exhaustive fallback), "slab_hits", "slab_misses", "slab_bytes" (bytes of
   slabs held from CUDA), "slab_live_bytes" (handed out), "slab_cached_bytes"
   (kept for reuse, at most TEMPI_SLAB_CACHE_MB per memory space),
   "host_link_copies", "send_contig_staged", "recv_contig_staged",
   "neighbor_fused", "neighbor_isir", "neighbor_lib", "alltoallv_staged",
   "alltoallv_remote_first", "alltoallv_isir_staged",
   "alltoallv_isir_remote_staged", "alltoallv_lib", and "staged_timeouts"
   (staged launches whose bounded waits gave up, as far as the host has seen:
   see tempi_staged_check); -1 for an unknown name */
int64_t tempi_counter(const char *name);
/* The staged kernels (kernel 4) wait on their bulk copies with a bound of
   about a second; a kernel that gives up leaves its chunks uncopied and sets
   a failure word in pinned host memory.  After synchronising the stream of a
   tempi_pack / tempi_unpack call, this returns TEMPI_ERR_TIMEOUT if any staged
   kernel gave up since the last check (and clears the word), else TEMPI_OK.
   The interposed MPI calls check it themselves and return MPI_ERR_OTHER.  No
   reference counterpart: the reference's kernels have no waits. */
int tempi_staged_check(void);

#ifdef __cplusplus
}
#endif

#endif /* TEMPI_B200_H */
