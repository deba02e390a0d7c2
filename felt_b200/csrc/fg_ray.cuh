// Surface::ray (include/Felt/Surface.hpp:468-616, 1450-1598) for batches of rays on the device.
#pragma once

#include <cstddef>

#include "fg_engine.cuh"

namespace fg {

/// Casts n rays (origins and directions, n*D floats each) at surface s of the pool; hits
/// receives n*D floats, FLT_MAX in every component for a ray that misses. With device_ptrs the
/// three arrays are device memory of the pool's GPU, else host memory. exact_order: find each
/// next candidate partition by a full walk of the planes instead of merging the per-axis walks
/// (the same order; used to test the merge).
void ray_batch(EngineBase& eng, int s, const float* origins, const float* dirs, size_t n,
               float* hits, bool device_ptrs, bool exact_order = false);

}  // namespace fg
