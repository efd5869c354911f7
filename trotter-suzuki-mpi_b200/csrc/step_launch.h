// Entry points of the separately compiled step-kernel variants.
#pragma once
#include <cuda_runtime.h>

#include "step_kernel.cuh"

namespace tsb {

// blocks == 0 only configures the kernel attributes (no launch).
cudaError_t launch_step_f64_real(int C, bool rot, bool phase, const StepArgs<double> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st);
cudaError_t launch_step_f64_imag(int C, bool rot, bool phase, const StepArgs<double> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st);
cudaError_t launch_step_f32_real(int C, bool rot, bool phase, const StepArgs<float> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st);
cudaError_t launch_step_f32_imag(int C, bool rot, bool phase, const StepArgs<float> &a, int warps,
                                 size_t smem, int blocks, cudaStream_t st);

template <class V>
cudaError_t launch_step_variant(const StepArgs<typename V::T> &a, int warps, size_t smem,
                                int blocks, cudaStream_t st) {
    auto fn = step_kernel<V>;
    static int configured_smem = -1;
    if ((int)smem > configured_smem) {
        cudaError_t e =
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured_smem = (int)smem;
    }
    if (blocks == 0) return cudaSuccess;
    fn<<<blocks, warps * 32, smem, st>>>(a);
    return cudaGetLastError();
}

// Rotation variants exist with 2 cells per lane only (the 7-row window with
// 4 cells per lane would exceed the register budget).
template <typename T, bool IMAG>
cudaError_t launch_step_imag_t(int C, bool rot, bool phase, const StepArgs<T> &a, int warps,
                               size_t smem, int blocks, cudaStream_t st) {
    if (C == 2) {
        if (rot) {
            if (phase) return launch_step_variant<Variant<T, 2, IMAG, true, true>>(a, warps, smem, blocks, st);
            return launch_step_variant<Variant<T, 2, IMAG, true, false>>(a, warps, smem, blocks, st);
        }
        if (phase) return launch_step_variant<Variant<T, 2, IMAG, false, true>>(a, warps, smem, blocks, st);
        return launch_step_variant<Variant<T, 2, IMAG, false, false>>(a, warps, smem, blocks, st);
    }
    if (C == 4 && !rot) {
        if (phase) return launch_step_variant<Variant<T, 4, IMAG, false, true>>(a, warps, smem, blocks, st);
        return launch_step_variant<Variant<T, 4, IMAG, false, false>>(a, warps, smem, blocks, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace tsb
