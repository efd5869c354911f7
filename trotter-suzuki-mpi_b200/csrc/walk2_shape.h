// Shared-memory geometry of the look-ahead walk (walk2.cuh), for the host.
#pragma once

namespace tsb {

// Entries of the per-warp vertical pair coefficient table for segments of
// seg_h rows: the walk's seg_h + 8 rows, 4 entries before its first row and
// the last row's pair, rounded up to an even count.
__host__ __device__ inline int w2_vlen(int seg_h) { return (seg_h + 8 + 4 + 2 + 1) & ~1; }

}  // namespace tsb
