// Method and kernel-configuration choice.  Replaced in part by the learned
// model in model.cpp; the fixed rules here are its fallback.

#include "dispatch.hpp"

namespace tempi {

Method choose_method(TypeRecord &r, int count) {
  switch (env().datatype) {
  case Method::DEVICE:
  case Method::ONESHOT:
  case Method::STAGED:
    return env().datatype;
  default:
    break;
  }
  const int64_t bytes = int64_t(count) * r.desc.size;
  auto it = r.methods.find(bytes);
  if (it != r.methods.end()) {
    counters().dispatch_hit++;
    return it->second;
  }
  counters().dispatch_miss++;
  Method m = Method::DEVICE;
  r.methods[bytes] = m;
  return m;
}

tempi_config choose_config(const tempi_desc &d, int64_t incount) {
  (void)d;
  (void)incount;
  return tempi_config{};
}

void dispatch_init() {}

} // namespace tempi
