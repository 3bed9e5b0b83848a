#include "symbols.hpp"

#include "internal.hpp"

#include <dlfcn.h>

#include <mutex>

namespace tempi {

LibMPI libmpi{};

static void *g_handle = nullptr;

static void *open_fallback() {
  if (g_handle)
    return g_handle;
  const char *names[] = {std::getenv("TEMPI_LIBMPI"), "libmpi.so",
                         "libminimpi.so"};
  for (const char *n : names) {
    if (!n)
      continue;
    g_handle = dlopen(n, RTLD_NOW | RTLD_GLOBAL);
    if (g_handle) {
      LOG_INFO("underlying MPI opened from %s", n);
      return g_handle;
    }
  }
  return nullptr;
}

static void *find(const char *name) {
  void *p = dlsym(RTLD_NEXT, name);
  if (!p) {
    void *h = open_fallback();
    if (h)
      p = dlsym(h, name);
  }
  if (!p)
    LOG_ERROR("could not resolve %s in the underlying MPI library", name);
  return p;
}

template <class F> static bool load(F &slot, const char *name) {
  slot = reinterpret_cast<F>(find(name));
  return slot != nullptr;
}

bool resolve_symbols() {
  static std::once_flag once;
  static bool ok = false;
  std::call_once(once, [] {
    bool r = true;
#define LOAD(fn) r &= load(libmpi.fn, "MPI_" #fn)
    LOAD(Init);
    LOAD(Init_thread);
    LOAD(Finalize);
    LOAD(Comm_rank);
    LOAD(Comm_size);
    LOAD(Type_commit);
    LOAD(Type_free);
    LOAD(Type_size);
    LOAD(Type_get_extent);
    LOAD(Type_get_envelope);
    LOAD(Type_get_contents);
    LOAD(Pack);
    LOAD(Unpack);
    LOAD(Pack_size);
    LOAD(Send);
    LOAD(Recv);
    LOAD(Isend);
    LOAD(Irecv);
    LOAD(Send_init);
    LOAD(Start);
    LOAD(Test);
    LOAD(Wait);
    LOAD(Request_free);
    LOAD(Type_contiguous);
    LOAD(Type_create_hvector);
    LOAD(Type_create_resized);
    LOAD(Dist_graph_neighbors_count);
    LOAD(Dist_graph_neighbors);
    LOAD(Neighbor_alltoallw);
    LOAD(Alltoallv);
#undef LOAD
    ok = r;
  });
  return ok;
}

} // namespace tempi
