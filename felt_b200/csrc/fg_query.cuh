// The isogrid's Numeric API evaluated at host-given positions (fg_query.cu).
#pragma once

#include <cstddef>

#include "fg_engine.cuh"

namespace fg {

/// Evaluates query `what` (FG_Q_*) of surface s at n nodes (ipos, D ints each) or real positions
/// (fpos, D floats each; used when ipos is null), host arrays; out gets n values, or n * D for
/// the gradients.
void query(EngineBase& eng, int s, int what, const float* fpos, const int* ipos, size_t n, float* out);

}  // namespace fg
