// Step-kernel variants: double, imaginary time.
#include "step_launch.h"

namespace tsb {

cudaError_t launch_step_f64_imag(int C, bool rot, int phase, const StepArgs<double> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st, int *bps) {
    return launch_step_imag_t<double, true>(C, rot, phase, a, warps, smem, blocks, st, bps);
}

}  // namespace tsb
