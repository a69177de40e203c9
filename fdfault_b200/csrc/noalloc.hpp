#pragma once
// Fixed-size device buffer used by the allocation-free read-back entry point.

#include "../../include/fdfault_b200.h"   // FDF_NOALLOC_MAX_VALUES: capacity in doubles (8 MiB)

namespace fdf {

// Device address of the static buffer on `device` (the calling thread's
// current device); looked up once per device, then cached.
double* noalloc_field_buffer(int device);

}  // namespace fdf
