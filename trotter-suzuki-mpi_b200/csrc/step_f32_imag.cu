// Step-kernel variants: float, imaginary time.
#include "step_launch.h"

namespace tsb {

cudaError_t launch_step_f32_imag(int C, bool rot, int phase, const StepArgs<float> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st, int *bps) {
    return launch_step_imag_t<float, true>(C, rot, phase, a, warps, smem, blocks, st, bps);
}

}  // namespace tsb
