// Batched step on the look-ahead walk: double precision, imaginary time.
#include "batch2_launch.h"

namespace tsb {

cudaError_t launch_batch2_f64_imag(int phase, const BatchArgs<double> &b, int warps, size_t smem,
                                   int blocks, cudaStream_t st, int *bps) {
    return launch_batch2_t<double, true>(phase, b, warps, smem, blocks, st, bps);
}

}  // namespace tsb
