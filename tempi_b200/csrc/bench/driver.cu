// Benchmark driver: runs sequences of interposed MPI_Pack / MPI_Unpack calls
// from C, the way the reference's bin/bench_mpi_pack.cpp drives them, so the
// measured per-call cost is the library's and not a scripting layer's.
// Linked against libtempi_b200.so, so MPI_Pack/MPI_Unpack here resolve to
// the interposed entry points.  Device time per pass comes from CUDA events
// recorded on TEMPI's own stream (tempi_stream()), which every interposed
// call launches on and synchronises.
#include <mpi.h>

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>

#include "tempi_b200.h"

namespace {

// read every 16-B word of `buf` so the L2 holds clean lines afterwards
__global__ void read_all(const uint4 *__restrict__ buf, size_t n,
                         unsigned *__restrict__ sink) {
  unsigned acc = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x) {
    uint4 v = __ldcg(buf + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == 0x9e3779b9u)
    *sink = acc; // practically never taken; keeps the loads alive
}

unsigned *g_sink = nullptr;

__global__ void k_bench_empty() {}

// one 4-B load per thread from rows `stride` bytes apart, stored densely:
// the least work a kernel that reads scattered DRAM lines can do
__global__ void k_bench_gather(const char *__restrict__ base, long long stride,
                               int rows, uint32_t *__restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < rows)
    out[t] = __ldg(reinterpret_cast<const uint32_t *>(base + t * stride));
}

} // namespace

extern "C" {

typedef struct tempi_bench_op {
  int unpack; // 0: MPI_Pack(typed -> packed), 1: MPI_Unpack(packed -> typed)
  int datatype;
  void *typed;
  void *packed;
  int incount;
  int position;
  int capacity;
  int reserved;
} tempi_bench_op;

// Evict the L2: write `bytes` of `buf`, then read them back so that the
// lines left behind are clean (a dirty L2 would bill its write-back to the
// next timed kernel).
// One copy-engine 2-D copy of `height` rows of `width` bytes (cudaMemcpy2DAsync)
// on `stream`: to_host != 0 copies device -> host, else host -> device.  For
// the host-link measurements of 2-D copies.
int tempi_bench_copy2d(void *dst, size_t dpitch, const void *src, size_t spitch,
                       size_t width, size_t height, int to_host, void *stream) {
  cudaError_t e = cudaMemcpy2DAsync(
      dst, dpitch, src, spitch, width, height,
      to_host ? cudaMemcpyDeviceToHost : cudaMemcpyHostToDevice,
      static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 2;
  }
  return 0;
}

// One launch of an empty kernel on `stream`: the fixed cost of any launch,
// measured beside the pack kernels (by CUDA events, or by ncu's duration).
int tempi_bench_empty(void *stream) {
  k_bench_empty<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>();
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// k_bench_gather over `rows` rows of `base`; the caller keeps
// (rows - 1) * stride + 4 bytes of `base` and 4 * rows bytes of `out` valid
int tempi_bench_gather(const void *base, long long stride, int rows, void *out,
                       void *stream) {
  if (rows <= 0 || stride < 4)
    return 1;
  k_bench_gather<<<(rows + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const char *>(base), stride, rows, static_cast<uint32_t *>(out));
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Host wall-clock cost per call of the pieces of a synchronous MPI_Pack:
// us_out[0] MPI_Pack of `incount` objects of `datatype` (typed -> packed),
// us_out[1] an empty kernel launch + cudaStreamSynchronize on TEMPI's stream,
// us_out[2] the empty launch alone, us_out[3] cudaStreamSynchronize of the
// idle stream, us_out[4] cudaPointerGetAttributes of both buffers.  Each is
// the median over 5 batches of `n` calls (after 200 untimed calls) of the
// mean per call.
int tempi_bench_call_overhead(int datatype, void *typed, void *packed,
                              int incount, int capacity, int n,
                              double *us_out) {
  if (n < 1 || !us_out)
    return 1;
  cudaStream_t s = static_cast<cudaStream_t>(tempi_stream());
  int err = 0;
  auto per_call = [&](auto f) {
    for (int i = 0; i < 200; ++i)
      f();
    double v[5];
    for (double &x : v) {
      const auto t0 = std::chrono::steady_clock::now();
      for (int i = 0; i < n; ++i)
        f();
      x = std::chrono::duration<double, std::micro>(
              std::chrono::steady_clock::now() - t0)
              .count() /
          n;
    }
    std::sort(v, v + 5);
    return v[2];
  };
  us_out[0] = per_call([&] {
    int pos = 0;
    if (MPI_Pack(typed, incount, datatype, packed, capacity, &pos,
                 MPI_COMM_WORLD) != MPI_SUCCESS)
      err = 2;
  });
  us_out[1] = per_call([&] {
    k_bench_empty<<<1, 32, 0, s>>>();
    if (cudaStreamSynchronize(s) != cudaSuccess)
      err = 2;
  });
  us_out[2] = per_call([&] { k_bench_empty<<<1, 32, 0, s>>>(); });
  if (cudaStreamSynchronize(s) != cudaSuccess)
    err = 2;
  us_out[3] = per_call([&] { cudaStreamSynchronize(s); });
  us_out[4] = per_call([&] {
    cudaPointerAttributes a, b;
    cudaPointerGetAttributes(&a, typed);
    cudaPointerGetAttributes(&b, packed);
  });
  return err ? err : (cudaGetLastError() == cudaSuccess ? 0 : 2);
}

int tempi_bench_flush(void *buf, size_t bytes, void *stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (!g_sink && cudaMalloc(&g_sink, sizeof(unsigned)) != cudaSuccess)
    return 2;
  if (cudaMemsetAsync(buf, 1, bytes, s) != cudaSuccess)
    return 2;
  read_all<<<1184, 256, 0, s>>>(static_cast<const uint4 *>(buf), bytes / 16,
                                g_sink);
  return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// Run `iters` passes over `ops`; ms_out[i] is pass i's device time.  With
// `flush` non-null the L2 is flushed (untimed) before each pass.
int tempi_bench_mpi_ops(const tempi_bench_op *ops, int n, int iters,
                        void *flush, size_t flush_bytes, float *ms_out) {
  cudaStream_t s = static_cast<cudaStream_t>(tempi_stream());
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
    return 2;
  int err = 0;
  for (int it = 0; it < iters && !err; ++it) {
    if (flush && tempi_bench_flush(flush, flush_bytes, s))
      err = 2;
    cudaEventRecord(a, s);
    for (int i = 0; i < n && !err; ++i) {
      const tempi_bench_op &o = ops[i];
      int pos = o.position;
      err = o.unpack ? MPI_Unpack(o.packed, o.capacity, &pos, o.typed,
                                  o.incount, o.datatype, MPI_COMM_WORLD)
                     : MPI_Pack(o.typed, o.incount, o.datatype, o.packed,
                                o.capacity, &pos, MPI_COMM_WORLD);
    }
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms_out)
      ms_out[it] = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return err;
}

// A periodic halo exchange of one grid with itself over a graph
// communicator of n self-edges, `iters` times; ms_out[i] is step i's device
// time (events on TEMPI's stream; every call below returns only when its
// work is done).  mode 0: the reference's sequence (bin/bench_halo_exchange.cpp
// :560-625): MPI_Pack of every send region into sendbuf, MPI_Neighbor_alltoallv
// of the packed bytes, MPI_Unpack of every region from recvbuf.  mode 1: one
// MPI_Neighbor_alltoallw with a send and a receive datatype per edge.
int tempi_bench_halo(int mode, int n, const int *sendtypes,
                     const int *recvtypes, const int *counts,
                     const int *displs, void *grid, void *sendbuf,
                     void *recvbuf, int packed_bytes, int comm, int iters,
                     float *ms_out) {
  cudaStream_t s = static_cast<cudaStream_t>(tempi_stream());
  cudaEvent_t a, b;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
    return 2;
  int *ones = new int[n];
  MPI_Aint *zeros = new MPI_Aint[n];
  for (int i = 0; i < n; ++i) {
    ones[i] = 1;
    zeros[i] = 0;
  }
  int err = 0;
  for (int it = 0; it < iters && !err; ++it) {
    cudaEventRecord(a, s);
    if (mode == 0) {
      int pos = 0;
      for (int i = 0; i < n && !err; ++i)
        err = MPI_Pack(grid, 1, sendtypes[i], sendbuf, packed_bytes, &pos, comm);
      if (!err)
        err = MPI_Neighbor_alltoallv(sendbuf, counts, displs, MPI_BYTE,
                                     recvbuf, counts, displs, MPI_BYTE, comm);
      pos = 0;
      for (int i = 0; i < n && !err; ++i)
        err = MPI_Unpack(recvbuf, packed_bytes, &pos, grid, 1, recvtypes[i],
                         comm);
    } else {
      err = MPI_Neighbor_alltoallw(grid, ones, zeros, sendtypes, grid, ones,
                                   zeros, recvtypes, comm);
    }
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms_out)
      ms_out[it] = ms;
  }
  delete[] ones;
  delete[] zeros;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return err;
}

} // extern "C"
