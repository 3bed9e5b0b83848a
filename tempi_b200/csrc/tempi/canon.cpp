// Canonicalisation of committed MPI datatypes into strided blocks, and the
// type cache.
//
// Same job as the reference's traverse/simplify/to_strided_block
// (src/internal/types.cpp:42-715): read the constructor tree through
// MPI_Type_get_envelope / MPI_Type_get_contents and reduce it to
// {start, block, (count, stride)...}.  This version builds a loop nest
// directly (outermost loop first, each constructor prepending its loops) and
// then applies only rewrites that keep the type-map order:
//   * a loop of count 1 is dropped;
//   * an innermost loop whose stride equals the block length widens the
//     block (rows are adjacent);
//   * two adjacent loops where the outer stride equals inner count x inner
//     stride become one loop.
// The reference additionally swaps loops so larger strides sit outside
// (stream_swap, types.cpp:378-404); that changes the packed byte order for
// types such as an hvector of columns, so it is deliberately not done here.
// Extra coverage over the reference: dup, resized, and (h)indexed(_block)
// types whose blocks are equal and equally spaced.

#include "runtime.hpp"

#include <algorithm>
#include <cstring>
#include <vector>

namespace tempi {

namespace {

struct Loop {
  int64_t count, stride;
};

struct Nest {
  int64_t off = 0;   // byte offset of the first described byte
  int64_t block = 0; // contiguous bytes at the bottom
  std::vector<Loop> loops; // outermost first
};

int64_t extent_of(MPI_Datatype t) {
  MPI_Aint lb = 0, ext = 0;
  libmpi.Type_get_extent(t, &lb, &ext);
  return ext;
}

bool build(MPI_Datatype t, Nest &n, int depth);

// child nest prefixed by `outer` loops and shifted by `off`
bool with_child(MPI_Datatype child, const std::vector<Loop> &outer, int64_t off,
                Nest &n, int depth) {
  Nest c;
  if (!build(child, c, depth + 1))
    return false;
  n.off = off + c.off;
  n.block = c.block;
  n.loops = outer;
  n.loops.insert(n.loops.end(), c.loops.begin(), c.loops.end());
  return true;
}

// equally sized, equally spaced blocks at byte displacements d[i]
bool regular_blocks(const std::vector<int64_t> &bl,
                    const std::vector<int64_t> &d, int64_t &off,
                    int64_t &count, int64_t &blen, int64_t &stride) {
  count = (int64_t)bl.size();
  if (count == 0)
    return false;
  blen = bl[0];
  for (int64_t b : bl)
    if (b != blen)
      return false;
  off = d[0];
  stride = count > 1 ? d[1] - d[0] : 0;
  for (int64_t i = 1; i < count; ++i)
    if (d[i] - d[i - 1] != stride)
      return false;
  return true;
}

bool build(MPI_Datatype t, Nest &n, int depth) {
  if (depth > 64)
    return false;
  int ni = 0, na = 0, nd = 0, combiner = 0;
  if (libmpi.Type_get_envelope(t, &ni, &na, &nd, &combiner) != MPI_SUCCESS)
    return false;
  if (combiner == MPI_COMBINER_NAMED) {
    int size = 0;
    libmpi.Type_size(t, &size);
    if (extent_of(t) != size)
      return false;
    n.off = 0;
    n.block = size;
    n.loops.clear();
    return true;
  }
  std::vector<int> ints(std::max(ni, 1));
  std::vector<MPI_Aint> addrs(std::max(na, 1));
  std::vector<MPI_Datatype> types(std::max(nd, 1));
  if (libmpi.Type_get_contents(t, ni, na, nd, ints.data(), addrs.data(),
                               types.data()) != MPI_SUCCESS)
    return false;
  switch (combiner) {
  case MPI_COMBINER_DUP:
  case MPI_COMBINER_RESIZED:
    // the child's byte layout is unchanged; parents step by this type's
    // extent, which they read with MPI_Type_get_extent
    return with_child(types[0], {}, 0, n, depth);
  case MPI_COMBINER_CONTIGUOUS: {
    const int64_t e = extent_of(types[0]);
    return with_child(types[0], {{ints[0], e}}, 0, n, depth);
  }
  case MPI_COMBINER_VECTOR: {
    const int64_t e = extent_of(types[0]);
    return with_child(types[0], {{ints[0], int64_t(ints[2]) * e}, {ints[1], e}},
                      0, n, depth);
  }
  case MPI_COMBINER_HVECTOR: {
    const int64_t e = extent_of(types[0]);
    return with_child(types[0], {{ints[0], int64_t(addrs[0])}, {ints[1], e}}, 0,
                      n, depth);
  }
  case MPI_COMBINER_INDEXED:
  case MPI_COMBINER_HINDEXED:
  case MPI_COMBINER_INDEXED_BLOCK:
  case MPI_COMBINER_HINDEXED_BLOCK: {
    const int64_t e = extent_of(types[0]);
    const int count = ints[0];
    std::vector<int64_t> bl(count), d(count);
    for (int i = 0; i < count; ++i) {
      switch (combiner) {
      case MPI_COMBINER_INDEXED:
        bl[i] = ints[1 + i], d[i] = int64_t(ints[1 + count + i]) * e;
        break;
      case MPI_COMBINER_HINDEXED:
        bl[i] = ints[1 + i], d[i] = addrs[i];
        break;
      case MPI_COMBINER_INDEXED_BLOCK:
        bl[i] = ints[1], d[i] = int64_t(ints[2 + i]) * e;
        break;
      default:
        bl[i] = ints[1], d[i] = addrs[i];
      }
    }
    int64_t off, cnt, blen, stride;
    if (!regular_blocks(bl, d, off, cnt, blen, stride))
      return false;
    return with_child(types[0], {{cnt, stride}, {blen, e}}, off, n, depth);
  }
  case MPI_COMBINER_SUBARRAY: {
    const int ndims = ints[0];
    const int *sizes = &ints[1], *subs = &ints[1 + ndims],
              *starts = &ints[1 + 2 * ndims];
    const bool corder = ints[1 + 3 * ndims] == MPI_ORDER_C;
    const int64_t e = extent_of(types[0]);
    std::vector<Loop> loops;
    int64_t off = 0;
    for (int k = 0; k < ndims; ++k) { // slowest-varying dimension first
      const int d = corder ? k : ndims - 1 - k;
      int64_t s = e;
      if (corder)
        for (int j = d + 1; j < ndims; ++j)
          s *= sizes[j];
      else
        for (int j = 0; j < d; ++j)
          s *= sizes[j];
      loops.push_back({subs[d], s});
      off += int64_t(starts[d]) * s;
    }
    return with_child(types[0], loops, off, n, depth);
  }
  default:
    return false; // struct, darray, ...: the library packs these
  }
}

// order-preserving normal form; returns false when a count is zero
bool normalize(Nest &n) {
  std::vector<Loop> l;
  for (const Loop &x : n.loops) {
    if (x.count == 0)
      return false;
    if (x.count != 1)
      l.push_back(x);
  }
  for (bool changed = true; changed;) {
    changed = false;
    if (!l.empty() && l.back().stride == n.block) {
      n.block *= l.back().count;
      l.pop_back();
      changed = true;
      continue;
    }
    for (size_t k = 0; k + 1 < l.size(); ++k) {
      if (l[k].stride == l[k + 1].count * l[k + 1].stride) {
        l[k].count *= l[k + 1].count;
        l[k].stride = l[k + 1].stride;
        l.erase(l.begin() + k + 1);
        changed = true;
        break;
      }
    }
  }
  n.loops = l;
  return true;
}

int align_of(const tempi_desc &d) {
  uint64_t bits = uint64_t(d.start) | uint64_t(d.block) | uint64_t(d.extent);
  for (int k = 0; k < d.ndims; ++k)
    bits |= uint64_t(d.strides[k]);
  int a = 16;
  while (a > 1 && (bits & (a - 1)))
    a >>= 1;
  return a;
}

std::mutex g_mu;
std::unordered_map<MPI_Datatype, TypeRecord> g_cache;

} // namespace

int canonicalize(MPI_Datatype t, tempi_desc *out) {
  if (!resolve_symbols())
    return set_error(TEMPI_ERR_UNSUPPORTED, "no underlying MPI library");
  std::memset(out, 0, sizeof(*out));
  int size = 0;
  if (libmpi.Type_size(t, &size) != MPI_SUCCESS)
    return set_error(TEMPI_ERR_ARG, "MPI_Type_size failed");
  out->extent = extent_of(t);
  out->align = 16;
  Nest n;
  if (!build(t, n, 0))
    return TEMPI_ERR_UNSUPPORTED;
  if (!normalize(n) || size == 0) { // nothing is described
    out->size = 0;
    return TEMPI_OK;
  }
  if ((int)n.loops.size() > TEMPI_MAX_DIMS)
    return TEMPI_ERR_UNSUPPORTED;
  out->start = n.off;
  out->block = n.block;
  out->ndims = (int32_t)n.loops.size();
  int64_t total = n.block;
  for (int k = 0; k < out->ndims; ++k) { // fastest first in the descriptor
    const Loop &x = n.loops[n.loops.size() - 1 - k];
    out->counts[k] = x.count;
    out->strides[k] = x.stride;
    total *= x.count;
  }
  out->size = total;
  if (total != size) // a reading of the type we do not trust
    return TEMPI_ERR_UNSUPPORTED;
  out->align = align_of(*out);
  return TEMPI_OK;
}

TypeRecord *find_type(MPI_Datatype t) {
  std::lock_guard<std::mutex> l(g_mu);
  auto it = g_cache.find(t);
  return it == g_cache.end() ? nullptr : &it->second;
}

TypeRecord *commit_type(MPI_Datatype t) {
  {
    std::lock_guard<std::mutex> l(g_mu);
    auto it = g_cache.find(t);
    if (it != g_cache.end())
      return &it->second;
  }
  TypeRecord r;
  r.packable = canonicalize(t, &r.desc) == TEMPI_OK;
  std::lock_guard<std::mutex> l(g_mu);
  auto res = g_cache.emplace(t, std::move(r));
  if (res.second)
    counters().cached_types++;
  return &res.first->second;
}

void release_type(MPI_Datatype t) {
  std::lock_guard<std::mutex> l(g_mu);
  if (g_cache.erase(t))
    counters().cached_types--;
}

} // namespace tempi

extern "C" int tempi_describe(int64_t datatype, tempi_desc *out) {
  if (!out)
    return tempi::set_error(TEMPI_ERR_ARG, "null output");
  return tempi::canonicalize(static_cast<MPI_Datatype>(datatype), out);
}
