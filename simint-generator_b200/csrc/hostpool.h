// Host worker pool for the data movement around simint_compute_eri: packing
// large pair sets into the pinned staging buffer and copying large results
// out of it run on all host cores.
#pragma once

#include <cstddef>
#include <functional>

namespace sb200 {

// Run fn(lo, hi) over [0, n) split into contiguous pieces on the pool's
// threads and the caller; returns when all pieces are done.  Small n runs
// inline.  Calls from several host threads are serialised.
void parallel_for(size_t n, size_t min_piece, const std::function<void(size_t, size_t)> & fn);

// memcpy on the pool for large sizes.
void parallel_copy(void * dst, const void * src, size_t bytes);

} // namespace sb200
