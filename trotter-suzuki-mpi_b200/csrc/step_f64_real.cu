// Step-kernel variants: double, real time.
#include "step_launch.h"

namespace tsb {

cudaError_t launch_step_f64_real(int C, bool rot, bool phase, const StepArgs<double> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st) {
    return launch_step_imag_t<double, false>(C, rot, phase, a, warps, smem, blocks, st);
}

}  // namespace tsb
