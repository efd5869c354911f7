// Shared-memory geometry of the look-ahead walk (walk2.cuh), for the host.
#pragma once

namespace tsb {

// Entries of the per-warp vertical pair coefficient table for segments of
// seg_h rows: the walk's seg_h + 2 HY rows, VPAD entries before its first
// row and the last row's pair, rounded up to an even count (HY = VPAD = 4;
// 6 in a rotating frame).
__host__ __device__ inline int w2_vlen(int seg_h, bool rot = false) {
    return rot ? (seg_h + 12 + 6 + 2 + 1) & ~1 : (seg_h + 8 + 4 + 2 + 1) & ~1;
}

}  // namespace tsb
