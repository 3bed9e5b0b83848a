// Choice of transfer method and kernel configuration for a strided object.
#pragma once

#include "runtime.hpp"

namespace tempi {

// Transfer method for `count` objects of a committed type (cached per
// packed byte count in the record).  TEMPI_DATATYPE_* overrides everything.
Method choose_method(TypeRecord &r, int count);

// Kernel configuration for one pack/unpack launch.
tempi_config choose_config(const tempi_desc &d, int64_t incount);

// Load cached models from TEMPI_CACHE_DIR (called from MPI_Init).
void dispatch_init();

} // namespace tempi
