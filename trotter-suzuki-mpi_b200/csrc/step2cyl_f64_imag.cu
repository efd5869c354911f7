// Look-ahead walk variants on a cylindrical lattice: double, imaginary time.
#include "step2_launch.h"

namespace tsb {

cudaError_t launch_step2cyl_f64_imag(int R, int phase, const StepArgs<double> &a,
                                     int warps, size_t smem, int blocks, cudaStream_t st, int *bps,
                                     bool pdl) {
    return launch_step2cyl_t<double, true>(R, phase, a, warps, smem, blocks, st, bps, pdl);
}

}  // namespace tsb
