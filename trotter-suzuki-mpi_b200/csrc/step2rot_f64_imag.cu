// Look-ahead walk variants in a rotating frame: double, imaginary time.
#include "step2_launch.h"

namespace tsb {

cudaError_t launch_step2rot_f64_imag(int C, int R, int phase, const StepArgs<double> &a,
                                     int warps, size_t smem, int blocks, cudaStream_t st, int *bps,
                                     bool pdl) {
    return launch_step2rot_t<double, true>(C, R, phase, a, warps, smem, blocks, st, bps, pdl);
}

}  // namespace tsb
