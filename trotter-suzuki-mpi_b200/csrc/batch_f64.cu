// Batched step-kernel variants: double.
#include "batch_launch.h"

namespace tsb {

cudaError_t launch_batch_f64(bool imag, int phase, const BatchArgs<double> &b, int warps, size_t smem,
                             int blocks, cudaStream_t st, int *bps) {
    return imag ? launch_batch_t<double, true>(phase, b, warps, smem, blocks, st, bps)
                : launch_batch_t<double, false>(phase, b, warps, smem, blocks, st, bps);
}

}  // namespace tsb
