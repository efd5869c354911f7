// Batched step-kernel variants: float.
#include "batch_launch.h"

namespace tsb {

cudaError_t launch_batch_f32(bool imag, int phase, const BatchArgs<float> &b, int warps, size_t smem,
                             int blocks, cudaStream_t st, int *bps) {
    return imag ? launch_batch_t<float, true>(phase, b, warps, smem, blocks, st, bps)
                : launch_batch_t<float, false>(phase, b, warps, smem, blocks, st, bps);
}

}  // namespace tsb
