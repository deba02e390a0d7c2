// Surface::ray (include/Felt/Surface.hpp:468-616, 1450-1598) for batches of rays on the device.
#pragma once

#include <cstddef>

#include "fg_engine.cuh"

namespace fg {

/// Casts n rays (origins and directions, n*D floats each) at surface s of the pool; hits
/// receives n*D floats, FLT_MAX in every component for a ray that misses. With device_ptrs the
/// three arrays are device memory of the pool's GPU, else host memory. buffer: candidate
/// partitions a ray sorts in registers/local memory before it falls back to re-walking its
/// planes (< 0 = the default, ray_buffer_max()); the result does not depend on it.
void ray_batch(EngineBase& eng, int s, const float* origins, const float* dirs, size_t n,
               float* hits, bool device_ptrs, int buffer = -1);

/// Largest candidate buffer a ray keeps.
int ray_buffer_max();

}  // namespace fg
