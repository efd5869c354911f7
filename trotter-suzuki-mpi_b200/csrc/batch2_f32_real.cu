// Batched step on the look-ahead walk: single precision, real time.
#include "batch2_launch.h"

namespace tsb {

cudaError_t launch_batch2_f32_real(int phase, const BatchArgs<float> &b, int warps, size_t smem,
                                   int blocks, cudaStream_t st, int *bps) {
    return launch_batch2_t<float, false>(phase, b, warps, smem, blocks, st, bps);
}

}  // namespace tsb
