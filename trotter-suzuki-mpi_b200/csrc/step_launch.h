// Entry points of the separately compiled step-kernel variants.
#pragma once
#include <cuda_runtime.h>

#include "step_kernel.cuh"

namespace tsb {

// blocks == 0 only configures the kernel attributes (no launch); when
// blocks_per_sm is not null it receives the number of resident blocks per SM.
cudaError_t launch_step_f64_real(int C, bool rot, int phase, const StepArgs<double> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_step_f64_imag(int C, bool rot, int phase, const StepArgs<double> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_step_f32_real(int C, bool rot, int phase, const StepArgs<float> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_step_f32_imag(int C, bool rot, int phase, const StepArgs<float> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm);

template <class V>
cudaError_t launch_step_variant(const StepArgs<typename V::T> &a, int warps, size_t smem,
                                int blocks, cudaStream_t st, int *blocks_per_sm) {
    auto fn = step_kernel<V>;
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

// Rotation variants exist with 2 cells per lane only (the 7-row window with
// 4 cells per lane would exceed the register budget).
template <typename T, bool IMAG, int C, bool ROT>
cudaError_t launch_phase(int phase, const StepArgs<T> &a, int warps, size_t smem, int blocks,
                         cudaStream_t st, int *bps) {
    if constexpr (C == 2 && !ROT) {
        if (phase == 3)
            return launch_step_variant<Variant<T, C, IMAG, ROT, 3>>(a, warps, smem, blocks, st, bps);
        if (phase == 4)
            return launch_step_variant<Variant<T, C, IMAG, ROT, 4>>(a, warps, smem, blocks, st, bps);
        if (phase == 5)
            return launch_step_variant<Variant<T, C, IMAG, ROT, 5>>(a, warps, smem, blocks, st, bps);
        if (phase == 6)
            return launch_step_variant<Variant<T, C, IMAG, ROT, 6>>(a, warps, smem, blocks, st, bps);
        if constexpr (!IMAG) {
            if (phase == 7)
                return launch_step_variant<Variant<T, C, IMAG, ROT, 11>>(a, warps, smem, blocks,
                                                                         st, bps);
        }
    }
    if (phase > 3) return cudaErrorInvalidValue;
    if (phase == 2) return launch_step_variant<Variant<T, C, IMAG, ROT, 2>>(a, warps, smem, blocks, st, bps);
    if (phase == 1) return launch_step_variant<Variant<T, C, IMAG, ROT, 1>>(a, warps, smem, blocks, st, bps);
    return launch_step_variant<Variant<T, C, IMAG, ROT, 0>>(a, warps, smem, blocks, st, bps);
}

// phase: 0 none, 1 g|psi|^2, 2 g|psi|^2 + Lee-Huang-Yang, 3 two components
// (g|psi|^2 + g_ab|psi_b|^2; 2 cells per lane, no rotating frame); 4-6: 0-2 on
// a cylindrical lattice (2 cells per lane, no rotating frame); 7: 3 in real
// time with the previous step's Rabi rotation applied as the rows are loaded.
template <typename T, bool IMAG>
cudaError_t launch_step_imag_t(int C, bool rot, int phase, const StepArgs<T> &a, int warps,
                               size_t smem, int blocks, cudaStream_t st, int *bps) {
    if (C == 2) {
        if (rot) return launch_phase<T, IMAG, 2, true>(phase, a, warps, smem, blocks, st, bps);
        return launch_phase<T, IMAG, 2, false>(phase, a, warps, smem, blocks, st, bps);
    }
    if (C == 4 && !rot) return launch_phase<T, IMAG, 4, false>(phase, a, warps, smem, blocks, st, bps);
    return cudaErrorInvalidValue;
}

}  // namespace tsb
