// Choice of kernel configuration and transfer method for strided objects.
//
// The reference picks DEVICE or ONE_SHOT from measured tables (perf.json,
// src/internal/measure_system.cpp:106-299, cached per (colocated, bytes) in
// sender.cpp:259-277 and async_operation.cpp:341-368) and picks its kernel
// word size by a fixed rule.  Here a learned cost model (an FP32 MLP
// ensemble, mlp.cu) predicts the time of every candidate -- eight kernel
// configurations and three transfer methods -- from twelve features of the
// object; the candidate with the smallest predicted time wins, for a pack
// and for an unpack separately.  When the ensemble disagrees about the
// winner, the candidates are timed for real (exhaustive autotuning).
// Choices are cached per type.
#pragma once

#include "runtime.hpp"

namespace tempi {

constexpr int kNumConfigs = 10; // kernel configurations
constexpr int kNumMethods = 3; // DEVICE, ONE_SHOT, STAGED
// model outputs: pack with configuration k, unpack with configuration k,
// self-send by method m
constexpr int kPackOut = 0, kUnpackOut = kNumConfigs,
              kMethodOut = 2 * kNumConfigs;
static_assert(kMethodOut + kNumMethods == TEMPI_MLP_OUT, "model outputs");
extern const tempi_config kCandidates[kNumConfigs];
// measured entries: the model's outputs, then the fixed rules' pack and
// unpack times (the policy without the model)
constexpr int kFixedPack = TEMPI_MLP_OUT, kFixedUnpack = TEMPI_MLP_OUT + 1;
constexpr int kMeasured = TEMPI_MEASURED;
static_assert(kFixedUnpack + 1 == kMeasured, "measured entries");

// Whether candidate configuration k suits `incount` objects of `d`: a warp
// per row needs rows of at least 64 B, a shift group of L lanes rows of at
// least 4L bytes (16 B for L = 4), and both need at least two rows per SM;
// the staged kernels need a packed size of at least 64 KiB that is a
// multiple of 16 bytes (where a launch is not eligible for their bulk
// copies it takes the fixed rules).
// The harness measures only eligible candidates and the dispatcher chooses
// only among them.
bool eligible(const tempi_desc &d, int64_t incount, int k);

// Twelve model inputs for `incount` objects of `d`.
void features(const tempi_desc &d, int64_t incount, bool src_host,
              bool dst_host, float out[TEMPI_MLP_IN]);

// Transfer method for `count` objects of a committed type (cached per
// packed byte count in the record).  TEMPI_DATATYPE_* overrides everything.
Method choose_method(TypeRecord &r, int count);
// TEMPI_CONTIGUOUS_AUTO for a contiguous device buffer of `bytes`: whether
// staging through host memory (copy to host, host send, copy back) beats a
// send straight from device memory, by the measured tables (reference
// SendRecv1D::send/recv, src/internal/sender.cpp:63-88).  False without
// tables.
bool contiguous_staged_faster(int64_t bytes);

// Kernel configuration for one pack (unpack = false) or unpack launch of a
// committed type; src_host / dst_host: the typed / packed buffer is host
// memory.
tempi_config choose_config(TypeRecord &r, int64_t incount, bool src_host,
                           bool dst_host, bool unpack);
// ...and for an object with no record (the fixed rules)
tempi_config choose_config(const tempi_desc &d, int64_t incount);

// Prepare the choice for a newly committed type (MPI_Type_commit).
void on_commit(TypeRecord &r);

// Load models from TEMPI_CACHE_DIR or next to the library (MPI_Init).
void dispatch_init();

// Time every candidate: times_us[0..9] = pack and [10..19] = unpack with
// each kernel configuration, [20..22] = self-send round trip by each method,
// [23] / [24] = pack / unpack by the fixed rules (NaN where not measured).
// `what`: bit 0 configurations, bit 1 methods.
int measure_candidates(const tempi_desc &d, int64_t incount, bool src_host,
                       bool dst_host, int what, int reps, float *times_us);
// Free the scratch buffers measure_candidates keeps between calls (the
// training harness reuses them; a one-off measurement need not hold them).
void measure_release();

// Forced method for measurement (-1: none)
void force_method(int m);
// While set, kernel configurations come from the fixed rules (the harness
// measures; it must not recurse into itself).
void set_measuring(bool on);

} // namespace tempi
