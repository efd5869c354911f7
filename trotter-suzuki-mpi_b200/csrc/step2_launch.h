// Launch templates of the look-ahead walk (walk2.cuh); one translation unit
// per precision and time mode (step2_f{64,32}_{real,imag}.cu).
#pragma once
#include "step_launch.h"
#include "walk2.cuh"

namespace tsb {

template <class V>
cudaError_t launch_step2_variant(const StepArgs<typename V::T> &a, int warps, size_t smem,
                                 int blocks, cudaStream_t st, int *blocks_per_sm) {
    auto fn = step2_kernel<V>;
    static int configured_smem = -1;
    if ((int)smem > configured_smem) {
        cudaError_t e =
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured_smem = (int)smem;
    }
    if (blocks_per_sm) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, warps * 32, smem);
        if (e != cudaSuccess) return e;
    }
    if (blocks == 0) return cudaSuccess;
    fn<<<blocks, warps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <typename T, bool IMAG>
cudaError_t launch_step2_t(int C, int phase, const StepArgs<T> &a, int warps, size_t smem,
                           int blocks, cudaStream_t st, int *bps) {
    if (C == 2) {
        if (phase == 0) return launch_step2_variant<Variant<T, 2, IMAG, false, 0>>(a, warps, smem, blocks, st, bps);
        if (phase == 1) return launch_step2_variant<Variant<T, 2, IMAG, false, 1>>(a, warps, smem, blocks, st, bps);
        if (phase == 2) return launch_step2_variant<Variant<T, 2, IMAG, false, 2>>(a, warps, smem, blocks, st, bps);
    } else if (C == 4) {
        if (phase == 0) return launch_step2_variant<Variant<T, 4, IMAG, false, 0>>(a, warps, smem, blocks, st, bps);
        if (phase == 1) return launch_step2_variant<Variant<T, 4, IMAG, false, 1>>(a, warps, smem, blocks, st, bps);
        if (phase == 2) return launch_step2_variant<Variant<T, 4, IMAG, false, 2>>(a, warps, smem, blocks, st, bps);
    }
    return cudaErrorInvalidValue;
}

}  // namespace tsb
