// Dispatch: learned cost model, measured fallback, the restated perf-table
// selector, and the fixed rules.  See dispatch.hpp.

#include "dispatch.hpp"

#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <fstream>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

namespace tempi {

// the kernel configurations the model scores (outputs 0..9)
const tempi_config kCandidates[kNumConfigs] = {
    {1, 0, 256, 0, 0, 0},  // word kernel, 256 threads
    {1, 0, 512, 0, 0, 0},  // word kernel, 512 threads
    {1, 0, 128, 0, 0, 0},  // word kernel, 128 threads
    {2, 0, 256, 0, 0, 0},  // row kernel (warp per row)
    {3, 0, 256, 4, 0, 0},  // shift kernel, 4 lanes per row
    {3, 0, 256, 8, 0, 0},  // shift kernel, 8 lanes per row
    {3, 0, 256, 16, 0, 0}, // shift kernel, 16 lanes per row
    {3, 0, 256, 32, 0, 0}, // shift kernel, 32 lanes per row
    {4, 0, 256, 0, 3, 0},  // staged kernel, 3 CTAs per SM
    {4, 0, 256, 0, 8, 0},  // staged kernel, 8 CTAs per SM
};

namespace {

float lg(double v) { return v > 0 ? float(std::log2(v)) : 0.f; }

// ---- the learned model ------------------------------------------------------

struct Model {
  bool loaded = false;
  int members = 0;
  float y_mean[TEMPI_MLP_OUT], y_std[TEMPI_MLP_OUT];
  std::vector<float> params;
  float *dev_params = nullptr;
  // one inference's input row and outputs, in mapped pinned host memory
  // (the kernel reads and writes them over the link: no copies to wait for)
  float *host_io = nullptr, *dev_io = nullptr;
  std::string source;
};

struct Table {
  bool loaded = false;
  std::vector<double> pp_dev, pp_host, d2h, h2d;
  std::vector<std::vector<double>> pack_dev, unpack_dev, pack_host, unpack_host;
};

std::mutex g_mu;
Model g_model;
// Choices by layout, shared by every type handle with the same descriptor,
// object count, buffer kinds, direction and policy, so committing a shape
// again (a new handle for a layout seen before) costs no inference or
// measurement.  Guarded by g_mu; cleared when a new model loads, and when it
// grows past kMaxLayouts.
std::unordered_map<std::string, int> g_layouts;
constexpr size_t kMaxLayouts = size_t(1) << 16;
Table g_table;
int g_forced = -1;
double g_spread_limit = 0.5; // log2 units: the members disagree by ~41 %

const char kModelMagic[8] = {'T', 'M', 'L', 'P', 'v', '0', '0', '1'};
const char kTableMagic[8] = {'T', 'T', 'A', 'B', 'v', '0', '0', '1'};

int load_model_file(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f)
    return TEMPI_ERR_ARG;
  char magic[8];
  int32_t dims[4];
  f.read(magic, 8);
  f.read(reinterpret_cast<char *>(dims), sizeof(dims));
  if (!f || std::memcmp(magic, kModelMagic, 8) || dims[0] != TEMPI_MLP_IN ||
      dims[1] != TEMPI_MLP_HIDDEN || dims[2] != TEMPI_MLP_OUT || dims[3] <= 0 ||
      dims[3] > 64)
    return set_error(TEMPI_ERR_ARG, "%s is not a cost model file", path.c_str());
  Model m;
  m.members = dims[3];
  f.read(reinterpret_cast<char *>(m.y_mean), sizeof(m.y_mean));
  f.read(reinterpret_cast<char *>(m.y_std), sizeof(m.y_std));
  m.params.resize(size_t(m.members) * TEMPI_MLP_PARAMS);
  f.read(reinterpret_cast<char *>(m.params.data()),
         m.params.size() * sizeof(float));
  if (!f)
    return set_error(TEMPI_ERR_ARG, "%s is truncated", path.c_str());
  m.loaded = true;
  m.source = path;
  std::lock_guard<std::mutex> l(g_mu);
  cudaFree(g_model.dev_params);
  if (g_model.host_io)
    cudaFreeHost(g_model.host_io);
  g_model = std::move(m);
  g_layouts.clear(); // choices made with the previous model
  LOG_INFO("cost model loaded from %s (%d members)", path.c_str(),
           g_model.members);
  return TEMPI_OK;
}

template <class T> bool rd(std::ifstream &f, std::vector<T> &v, size_t n) {
  v.resize(n);
  f.read(reinterpret_cast<char *>(v.data()), n * sizeof(T));
  return bool(f);
}

int load_table_file(const std::string &path) {
  std::ifstream f(path, std::ios::binary);
  if (!f)
    return TEMPI_ERR_ARG;
  char magic[8];
  int32_t dims[3];
  f.read(magic, 8);
  f.read(reinterpret_cast<char *>(dims), sizeof(dims));
  if (!f || std::memcmp(magic, kTableMagic, 8) || dims[0] <= 0 ||
      dims[1] <= 0 || dims[2] <= 0 || dims[0] > 64 || dims[1] > 64 ||
      dims[2] > 64)
    return set_error(TEMPI_ERR_ARG, "%s is not a table file", path.c_str());
  Table t;
  bool ok = rd(f, t.pp_dev, dims[0]) && rd(f, t.pp_host, dims[0]) &&
            rd(f, t.d2h, dims[0]) && rd(f, t.h2d, dims[0]);
  for (auto *tab : {&t.pack_dev, &t.unpack_dev, &t.pack_host, &t.unpack_host}) {
    tab->resize(dims[1]);
    for (auto &row : *tab)
      ok = ok && rd(f, row, dims[2]);
  }
  if (!ok)
    return set_error(TEMPI_ERR_ARG, "%s is truncated", path.c_str());
  t.loaded = true;
  std::lock_guard<std::mutex> l(g_mu);
  g_table = std::move(t);
  return TEMPI_OK;
}

// Ensemble prediction (log2 microseconds) for one feature row: the mean
// over members and the spread (standard deviation) of each output.
int predict(const float f[TEMPI_MLP_IN], float mean[TEMPI_MLP_OUT],
            float spread[TEMPI_MLP_OUT]) {
  std::lock_guard<std::mutex> l(g_mu);
  Model &m = g_model;
  if (!m.loaded || !cuda_available())
    return TEMPI_ERR_UNSUPPORTED;
  cudaError_t e = cudaSuccess;
  const size_t io_floats = TEMPI_MLP_IN + size_t(m.members) * TEMPI_MLP_OUT;
  if (!m.dev_params) {
    e = cudaMalloc(&m.dev_params, m.params.size() * sizeof(float));
    if (e == cudaSuccess)
      e = copy_complete(m.dev_params, m.params.data(),
                        m.params.size() * sizeof(float));
    void *h = nullptr, *d = nullptr;
    if (e == cudaSuccess)
      e = cudaHostAlloc(&h, io_floats * sizeof(float), cudaHostAllocMapped);
    if (e == cudaSuccess)
      e = cudaHostGetDevicePointer(&d, h, 0);
    if (e != cudaSuccess) {
      if (h)
        cudaFreeHost(h);
      cudaFree(m.dev_params);
      m.dev_params = nullptr;
      return cuda_error(e, "cost model upload");
    }
    m.host_io = static_cast<float *>(h);
    m.dev_io = static_cast<float *>(d);
  }
  cudaStream_t s = pack_stream();
  std::memcpy(m.host_io, f, TEMPI_MLP_IN * sizeof(float));
  std::atomic_thread_fence(std::memory_order_seq_cst); // before the launch
  int err = tempi_mlp_predict(m.dev_params, m.members, m.dev_io, 1,
                              m.dev_io + TEMPI_MLP_IN, s);
  if (err)
    return err;
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    return cuda_error(e, "cost model output");
  const float *out = m.host_io + TEMPI_MLP_IN;
  for (int j = 0; j < TEMPI_MLP_OUT; ++j) {
    double s1 = 0, s2 = 0;
    for (int k = 0; k < m.members; ++k) {
      const double v = out[k * TEMPI_MLP_OUT + j] * m.y_std[j] + m.y_mean[j];
      s1 += v;
      s2 += v * v;
    }
    mean[j] = float(s1 / m.members);
    spread[j] = float(std::sqrt(std::max(0.0, s2 / m.members - (s1 / m.members) *
                                                               (s1 / m.members))));
  }
  return TEMPI_OK;
}

// ---- the restated perf-table selector ---------------------------------------
// Same model as the reference's Performance::model_device / model_oneshot
// (measure_system.cpp:106-138): pack + transfer + unpack, each interpolated
// from tables measured on this machine.  1-D tables: entry i is 2^i bytes;
// 2-D tables: entry [i][j] is 2^(2i+6) bytes packed from blocks of 2^j bytes.

int floor_log2(int64_t x) { return x <= 1 ? 0 : 63 - __builtin_clzll(uint64_t(x)); }
int ceil_log2(int64_t x) {
  const int f = floor_log2(x);
  return (x > 1 && (x & (x - 1))) ? f + 1 : f;
}

double table_1d(const std::vector<double> &a, int64_t bytes) {
  if (a.empty())
    return INFINITY;
  const int lo = floor_log2(bytes), hi = ceil_log2(bytes);
  if (hi >= int(a.size())) // beyond the table: scale the last entry linearly
    return a.back() * double(bytes) / double(int64_t(1) << (a.size() - 1));
  if (lo == hi)
    return a[lo];
  const float f = float(bytes - (int64_t(1) << lo)) /
                  float((int64_t(1) << hi) - (int64_t(1) << lo));
  return a[lo] * (1 - f) + a[hi] * f;
}

double table_2d(const std::vector<std::vector<double>> &a, int64_t bytes,
                int64_t block) {
  if (a.empty())
    return INFINITY;
  block = std::max<int64_t>(1, std::min<int64_t>(block, 512));
  const int yi1 = (floor_log2(bytes) - 6) / 2;
  const int64_t y1 = int64_t(1) << (2 * std::max(yi1, 0) + 6);
  const int yi2 = y1 == bytes ? yi1 : yi1 + 1;
  const int64_t y2 = int64_t(1) << (2 * yi2 + 6);
  int xi1 = floor_log2(block), xi2 = ceil_log2(block);
  const int rows = int(a.size());
  const std::vector<double> &ref = a[std::min(std::max(yi2, 0), rows - 1)];
  xi2 = std::min(xi2, int(ref.size()) - 1);
  xi1 = std::min(xi1, xi2);
  const int64_t x1 = int64_t(1) << xi1, x2 = int64_t(1) << xi2;
  const float sx = xi1 == xi2 ? 0.f : float(block - x1) / float(x2 - x1);
  const float sy = yi1 == yi2 ? 0.f : float(bytes - y1) / float(y2 - y1);
  if (yi2 >= rows) {
    const std::vector<double> &last = a.back();
    const double base = (1 - sx) * last[xi1] + sx * last[xi2];
    const double ymax = double(int64_t(1) << (2 * (rows - 1) + 6));
    return base / ymax * double(bytes);
  }
  const int r1 = std::max(yi1, 0);
  const double f1 = (1 - sx) * a[r1][xi1] + sx * a[r1][xi2];
  const double f2 = (1 - sx) * a[yi2][xi1] + sx * a[yi2][xi2];
  return (1 - sy) * f1 + sy * f2;
}

Method table_method(int64_t bytes, int64_t block) {
  std::lock_guard<std::mutex> l(g_mu);
  const Table &t = g_table;
  const double dev = table_2d(t.pack_dev, bytes, block) +
                     table_1d(t.pp_dev, bytes) +
                     table_2d(t.unpack_dev, bytes, block);
  const double one = table_2d(t.pack_host, bytes, block) +
                     table_1d(t.pp_host, bytes) +
                     table_2d(t.unpack_host, bytes, block);
  return one < dev ? Method::ONESHOT : Method::DEVICE;
}

std::string library_dir() {
  Dl_info info{};
  if (dladdr(reinterpret_cast<void *>(&dispatch_init), &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    const size_t slash = p.rfind('/');
    return slash == std::string::npos ? "." : p.substr(0, slash);
  }
  return ".";
}

// the winner among candidates [lo, hi) by predicted time (skipping those
// `ok` rules out), and whether the ensemble agrees well enough to trust it
int pick(const float *mean, const float *spread, int lo, int hi, bool *trust,
         const bool *ok = nullptr) {
  int best = -1;
  for (int j = lo; j < hi; ++j)
    if ((!ok || ok[j - lo]) && (best < 0 || mean[j] < mean[best]))
      best = j;
  if (best < 0)
    best = lo;
  *trust = spread[best] <= g_spread_limit;
  return best;
}

// Whether a host-resident layout lies where the cost model was trained: up
// to 4 MiB packed in a span of up to 16 MiB (tempi_b200/dispatch_train.py
// random_layout).  Beyond that the model extrapolates, and its picks for the
// strided sweep's host-resident points were measured 7.6 % slower than the
// fastest candidates in total (shift kernels unpacking small rows into host
// memory at half the speed of the word kernel).  Device layouts larger than
// the trained 256 MiB keep the model: they are long streams, where the
// candidates differ little, and measuring them would hold scratch memory of
// their size.
constexpr int64_t kTrainedHostBytes = int64_t(4) << 20;
constexpr int64_t kTrainedHostSpan = int64_t(16) << 20;
// Host-resident layouts are measured (on pinned scratch buffers the size of
// their span, freed again afterwards) up to this span; beyond it the fixed
// rules choose
constexpr int64_t kMeasureHostSpan = int64_t(512) << 20;

int64_t layout_span(const tempi_desc &d, int64_t incount) {
  int64_t hi = d.start + d.block + (incount - 1) * d.extent;
  for (int k = 0; k < d.ndims; ++k)
    hi += (d.counts[k] - 1) * d.strides[k];
  return hi;
}

enum class Range { TRAINED, MEASURE, FIXED };
Range trained_range(const tempi_desc &d, int64_t incount, bool src_host,
                    bool dst_host) {
  const int64_t bytes = incount * d.size;
  if (!src_host && !dst_host)
    return Range::TRAINED;
  const int64_t span = layout_span(d, incount);
  if (bytes <= kTrainedHostBytes && span <= kTrainedHostSpan)
    return Range::TRAINED;
  return span <= kMeasureHostSpan ? Range::MEASURE : Range::FIXED;
}

uint64_t config_key(int64_t incount, bool src_host, bool dst_host,
                    bool unpack) {
  return (uint64_t(incount) << 3) | (unpack ? 4 : 0) | (src_host ? 2 : 0) |
         (dst_host ? 1 : 0);
}

} // namespace

bool contiguous_staged_faster(int64_t bytes) {
  std::lock_guard<std::mutex> l(g_mu);
  const Table &t = g_table;
  if (!t.loaded)
    return false;
  const double staged = table_1d(t.d2h, bytes) + table_1d(t.pp_host, bytes) +
                        table_1d(t.h2d, bytes);
  return staged < table_1d(t.pp_dev, bytes);
}

bool eligible(const tempi_desc &d, int64_t incount, int k) {
  Geometry g;
  bool empty = false;
  if (k < 0 || k >= kNumConfigs)
    return false;
  if (make_geometry(&d, std::max<int64_t>(incount, 1), 0, 0, 0, &g, &empty) ||
      empty)
    return k == 0;
  const tempi_config &c = kCandidates[k];
  // the row kernels spread rows, not bytes, over the GPU: they need rows to
  // fill it
  const bool many_rows = g.rows >= uint32_t(2 * num_sms());
  if (c.kernel == 2)
    return g.block >= 64 && many_rows;
  if (c.kernel == 3)
    return g.block >= std::max<int64_t>(16, 4 * c.unroll) && many_rows;
  if (c.kernel == 4) {
    const int64_t bytes = int64_t(g.rows) * g.block;
    return bytes >= (int64_t(64) << 10) && bytes % 16 == 0;
  }
  return true;
}

void force_method(int m) { g_forced = m; }

// set while the harness measures: its own packs and sends use the fixed
// rules (and never re-enter the harness)
thread_local bool g_measuring = false;
void set_measuring(bool on) { g_measuring = on; }

void features(const tempi_desc &d, int64_t incount, bool src_host,
              bool dst_host, float f[TEMPI_MLP_IN]) {
  Geometry g;
  bool empty = false;
  std::memset(f, 0, sizeof(float) * TEMPI_MLP_IN);
  // pointers are assumed 256-B aligned here; the type's own alignment counts
  if (make_geometry(&d, std::max<int64_t>(incount, 1), 0, 0, 0, &g, &empty) ||
      empty)
    return;
  int64_t rest = 1;
  for (uint32_t k = 1; k < g.nd; ++k)
    rest *= g.cdiv[k].d;
  const int64_t total = int64_t(g.rows) * g.block;
  const float s = 1.f / 32.f; // log2 features scaled into [0, ~1]
  f[0] = float(g.nd) / 5.f;
  f[1] = lg(g.block) * s;
  f[2] = g.nd > 0 ? lg(g.cdiv[0].d) * s : 0.f;
  f[3] = lg(rest) * s;
  f[4] = g.nd > 0 ? lg(std::abs(double(g.strides[0]))) * s : 0.f;
  f[5] = g.nd > 1 ? lg(std::abs(double(g.strides[1]))) * s : 0.f;
  f[6] = lg(total) * s;
  f[7] = lg(incount) * s;
  f[8] = lg(g.width) / 4.f;
  f[9] = src_host ? 1.f : 0.f;
  f[10] = dst_host ? 1.f : 0.f;
  f[11] = lg(std::abs(double(d.extent)) * std::max<int64_t>(incount, 1)) * s;
}

tempi_config choose_config(const tempi_desc &d, int64_t incount) {
  (void)d;
  (void)incount;
  return tempi_config{}; // the fixed rules in launch_geometry
}

// The layout cache's key: the descriptor's fields in use, the object count,
// the buffer kinds, what is chosen ('p' pack, 'u' unpack, 'm' method) and
// the policy.
std::string layout_key(const tempi_desc &d, int64_t n, bool a, bool b,
                       char what) {
  int64_t v[5 + 2 * TEMPI_MAX_DIMS];
  int k = 0;
  v[k++] = d.start;
  v[k++] = d.extent;
  v[k++] = d.block;
  v[k++] = d.ndims;
  v[k++] = n;
  for (int i = 0; i < d.ndims && i < TEMPI_MAX_DIMS; ++i) {
    v[k++] = d.counts[i];
    v[k++] = d.strides[i];
  }
  std::string key(reinterpret_cast<const char *>(v), size_t(k) * sizeof(int64_t));
  key.push_back(char(a));
  key.push_back(char(b));
  key.push_back(what);
  key.push_back(char(env().dispatch));
  return key;
}

// under g_mu
void remember_layout(const std::string &key, int choice) {
  if (g_layouts.size() >= kMaxLayouts)
    g_layouts.clear();
  g_layouts[key] = choice;
}

tempi_config choose_config(TypeRecord &r, int64_t incount, bool src_host,
                           bool dst_host, bool unpack) {
  const Dispatch mode = env().dispatch;
  if (mode == Dispatch::HEURISTIC || mode == Dispatch::TABLE || g_measuring)
    return tempi_config{};
  const uint64_t key = config_key(incount, src_host, dst_host, unpack);
  const int lo = unpack ? kUnpackOut : kPackOut;
  {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = r.configs.find(key); // every call after the first: no strings
    if (it != r.configs.end()) {
      counters().dispatch_hit++;
      return it->second < 0 ? tempi_config{} : kCandidates[it->second];
    }
  }
  const std::string lkey =
      layout_key(r.desc, incount, src_host, dst_host, unpack ? 'u' : 'p');
  const std::string lkey2 =
      layout_key(r.desc, incount, src_host, dst_host, unpack ? 'p' : 'u');
  {
    std::lock_guard<std::mutex> l(g_mu);
    auto lt = g_layouts.find(lkey); // another handle of the same layout
    if (lt != g_layouts.end()) {
      counters().dispatch_hit++;
      r.configs[key] = lt->second;
      return lt->second < 0 ? tempi_config{} : kCandidates[lt->second];
    }
  }
  counters().dispatch_miss++;
  int choice = -1;
  bool trust = false;
  bool ok[kNumConfigs];
  for (int k = 0; k < kNumConfigs; ++k)
    ok[k] = eligible(r.desc, incount, k);
  const Range range = trained_range(r.desc, incount, src_host, dst_host);
  if (mode == Dispatch::LEARNED && range == Range::TRAINED) {
    float f[TEMPI_MLP_IN], mean[TEMPI_MLP_OUT], spread[TEMPI_MLP_OUT];
    features(r.desc, incount, src_host, dst_host, f);
    if (predict(f, mean, spread) == TEMPI_OK) {
      choice = pick(mean, spread, lo, lo + kNumConfigs, &trust, ok) - lo;
      // one inference predicts both directions: keep the other's pick too,
      // when the ensemble agrees on it
      const int lo2 = unpack ? kPackOut : kUnpackOut;
      bool trust2 = false;
      const int other =
          pick(mean, spread, lo2, lo2 + kNumConfigs, &trust2, ok) - lo2;
      if (trust2) {
        std::lock_guard<std::mutex> l(g_mu);
        r.configs.emplace(config_key(incount, src_host, dst_host, !unpack),
                          other);
        remember_layout(lkey2, other);
      }
    }
  }
  if (mode == Dispatch::EXHAUSTIVE || (choice >= 0 && !trust) ||
      (mode == Dispatch::LEARNED && range == Range::MEASURE)) {
    counters().dispatch_measured++;
    float t[kMeasured];
    const int me = measure_candidates(r.desc, incount, src_host, dst_host, 1, 2, t);
    // a choice made at run time holds no scratch memory afterwards (its
    // buffers are the size of the layout's span)
    measure_release();
    if (me == TEMPI_OK) {
      int best = -1;
      for (int j = 0; j < kNumConfigs; ++j)
        if (std::isfinite(t[lo + j]) && (best < 0 || t[lo + j] < t[lo + best]))
          best = j;
      choice = best;
      // the same measurement answers the other direction too
      int other = -1;
      const int lo2 = unpack ? kPackOut : kUnpackOut;
      for (int j = 0; j < kNumConfigs; ++j)
        if (std::isfinite(t[lo2 + j]) &&
            (other < 0 || t[lo2 + j] < t[lo2 + other]))
          other = j;
      std::lock_guard<std::mutex> l(g_mu);
      r.configs[config_key(incount, src_host, dst_host, !unpack)] = other;
      remember_layout(lkey2, other);
    }
  }
  std::lock_guard<std::mutex> l(g_mu);
  r.configs[key] = choice;
  remember_layout(lkey, choice);
  return choice < 0 ? tempi_config{} : kCandidates[choice];
}

Method choose_method(TypeRecord &r, int count) {
  if (g_forced >= 1 && g_forced <= 3)
    return Method(g_forced);
  switch (env().datatype) {
  case Method::DEVICE:
  case Method::ONESHOT:
  case Method::STAGED:
    return env().datatype;
  default:
    break;
  }
  const int64_t bytes = int64_t(count) * r.desc.size;
  const std::string lkey = layout_key(r.desc, count, false, false, 'm');
  {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = r.methods.find(bytes);
    if (it != r.methods.end()) {
      counters().dispatch_hit++;
      return it->second;
    }
    auto lt = g_layouts.find(lkey);
    if (lt != g_layouts.end()) {
      counters().dispatch_hit++;
      r.methods[bytes] = Method(lt->second);
      return Method(lt->second);
    }
  }
  counters().dispatch_miss++;
  Method m = Method::DEVICE; // the fixed rule: stay on the GPU
  const Dispatch mode = env().dispatch;
  if (mode == Dispatch::TABLE && g_table.loaded) {
    m = table_method(bytes, r.desc.block);
  } else if (mode == Dispatch::LEARNED) {
    float f[TEMPI_MLP_IN], mean[TEMPI_MLP_OUT], spread[TEMPI_MLP_OUT];
    features(r.desc, count, false, false, f);
    bool trust = false;
    if (predict(f, mean, spread) == TEMPI_OK) {
      const int j =
          pick(mean, spread, kMethodOut, kMethodOut + kNumMethods, &trust);
      // an untrusted prediction keeps the fixed rule: timing a transfer
      // needs a matching receive, which a send cannot arrange by itself
      if (trust)
        m = Method(j - kMethodOut + 1);
    }
  }
  std::lock_guard<std::mutex> l(g_mu);
  r.methods[bytes] = m;
  remember_layout(lkey, int(m));
  return m;
}

void on_commit(TypeRecord &r) {
  if (!r.packable || r.desc.size == 0 || env().dispatch != Dispatch::LEARNED ||
      !g_model.loaded || g_measuring)
    return;
  // cached for device-to-device packs and unpacks (one inference serves
  // both unless the ensemble disagrees about the unpack)
  choose_config(r, 1, false, false, false);
  choose_config(r, 1, false, false, true);
}

void dispatch_init() {
  const std::string names[] = {env().cache_dir + "/tempi_b200_dispatch.bin",
                               library_dir() + "/../models/tempi_b200_dispatch.bin"};
  for (const std::string &n : names)
    if (load_model_file(n) == TEMPI_OK)
      break;
  const std::string tables[] = {env().cache_dir + "/tempi_b200_table.bin",
                                library_dir() + "/../models/tempi_b200_table.bin"};
  for (const std::string &n : tables)
    if (load_table_file(n) == TEMPI_OK)
      break;
  if (const char *s = std::getenv("TEMPI_DISPATCH_SPREAD"))
    g_spread_limit = std::atof(s);
}

} // namespace tempi

using namespace tempi;

extern "C" int tempi_features(const tempi_desc *d, int64_t incount,
                              int src_host, int dst_host, float *out) {
  if (!d || !out)
    return set_error(TEMPI_ERR_ARG, "null argument");
  features(*d, incount, src_host != 0, dst_host != 0, out);
  return TEMPI_OK;
}

extern "C" int tempi_dispatch_load(const char *model_path,
                                   const char *table_path) {
  int err = TEMPI_OK;
  if (model_path && (err = load_model_file(model_path)))
    return err ? err : set_error(TEMPI_ERR_ARG, "cannot read %s", model_path);
  if (table_path && (err = load_table_file(table_path)))
    return err;
  return TEMPI_OK;
}

extern "C" int tempi_dispatch_choose(const tempi_desc *d, int64_t incount,
                                     int src_host, int dst_host, int mode,
                                     int *pack_config, int *unpack_config,
                                     int *method, float *predicted,
                                     float *spread) {
  if (!d)
    return set_error(TEMPI_ERR_ARG, "null descriptor");
  int pc = -1, uc = -1, mi = int(Method::DEVICE);
  float f[TEMPI_MLP_IN], mean[TEMPI_MLP_OUT], sp[TEMPI_MLP_OUT];
  for (int j = 0; j < TEMPI_MLP_OUT; ++j)
    mean[j] = sp[j] = NAN;
  if (mode == 0) { // learned
    features(*d, incount, src_host != 0, dst_host != 0, f);
    int err = predict(f, mean, sp);
    if (err)
      return err == TEMPI_ERR_UNSUPPORTED
                 ? set_error(err, "no cost model loaded")
                 : err;
    bool trust, ok[kNumConfigs];
    for (int k = 0; k < kNumConfigs; ++k)
      ok[k] = eligible(*d, incount, k);
    pc = pick(mean, sp, kPackOut, kPackOut + kNumConfigs, &trust, ok) -
         kPackOut;
    uc = pick(mean, sp, kUnpackOut, kUnpackOut + kNumConfigs, &trust, ok) -
         kUnpackOut;
    mi = pick(mean, sp, kMethodOut, kMethodOut + kNumMethods, &trust) -
         kMethodOut + 1;
  } else if (mode == 1) { // restated perf tables
    if (!g_table.loaded)
      return set_error(TEMPI_ERR_UNSUPPORTED, "no tables loaded");
    mi = int(table_method(int64_t(incount) * d->size, d->block));
  } // mode 2: fixed rules (-1: launch_geometry's choice, DEVICE)
  if (pack_config)
    *pack_config = pc;
  if (unpack_config)
    *unpack_config = uc;
  if (method)
    *method = mi;
  for (int j = 0; j < TEMPI_MLP_OUT; ++j) {
    if (predicted)
      predicted[j] = mean[j];
    if (spread)
      spread[j] = sp[j];
  }
  return TEMPI_OK;
}

extern "C" double tempi_table_interp(const double *table, int rows, int cols,
                                     int64_t bytes, int64_t block) {
  using namespace tempi;
  if (!table || rows <= 0)
    return NAN;
  if (cols <= 0)
    return table_1d(std::vector<double>(table, table + rows), bytes);
  std::vector<std::vector<double>> a(rows);
  for (int i = 0; i < rows; ++i)
    a[i].assign(table + size_t(i) * cols, table + size_t(i + 1) * cols);
  return table_2d(a, bytes, block);
}
