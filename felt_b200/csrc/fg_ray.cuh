// Surface::ray (include/Felt/Surface.hpp:468-616, 1450-1598) for batches of rays on the device.
#pragma once

#include <cstddef>

#include "fg_engine.cuh"

namespace fg {

/// Casts n rays (origins and directions, n*D floats each) at surface s of the pool; hits
/// receives n*D floats, FLT_MAX in every component for a ray that misses. With device_ptrs the
/// three arrays are device memory of the pool's GPU, else host memory. mode: how each ray's
/// candidate partitions are put in order, all giving the reference's order: 0 merges the
/// per-axis lists of a walk kernel (rays with long lists fall back to 2), 1 finds each next
/// candidate by a full walk of the planes, 2 merges per-axis cursors. 1 and 2 exist to test 0.
void ray_batch(EngineBase& eng, int s, const float* origins, const float* dirs, size_t n,
               float* hits, bool device_ptrs, int mode = 0);

}  // namespace fg
