// Look-ahead walk variants for one species of a pair: float, real time.
#include "step2_launch.h"

namespace tsb {

cudaError_t launch_step2pair_f32_real(int R, int phase, const StepArgs<float> &a,
                                      int warps, size_t smem, int blocks, cudaStream_t st, int *bps,
                                      bool pdl) {
    return launch_step2pair_t<float, false>(R, phase, a, warps, smem, blocks, st, bps, pdl);
}

}  // namespace tsb
