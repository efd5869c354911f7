// Entry points of the separately compiled batched step-kernel variants
// (2 cells per lane, no rotating frame).
#pragma once
#include <cuda_runtime.h>

#include "step_kernel.cuh"

namespace tsb {

// blocks == 0 only configures the kernel attributes (no launch); when
// blocks_per_sm is not null it receives the number of resident blocks per SM.
cudaError_t launch_batch_f64(bool imag, int phase, const BatchArgs<double> &b, int warps,
                             size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_batch_f32(bool imag, int phase, const BatchArgs<float> &b, int warps,
                             size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm);

// The batched step on the look-ahead walk (walk2.cuh, two rows per
// iteration; batch2_f{64,32}_{real,imag}.cu), same arguments.
cudaError_t launch_batch2_f64_real(int phase, const BatchArgs<double> &b, int warps, size_t smem,
                                   int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_batch2_f64_imag(int phase, const BatchArgs<double> &b, int warps, size_t smem,
                                   int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_batch2_f32_real(int phase, const BatchArgs<float> &b, int warps, size_t smem,
                                   int blocks, cudaStream_t st, int *blocks_per_sm);
cudaError_t launch_batch2_f32_imag(int phase, const BatchArgs<float> &b, int warps, size_t smem,
                                   int blocks, cudaStream_t st, int *blocks_per_sm);

template <class V>
cudaError_t launch_batch_variant(const BatchArgs<typename V::T> &b, int warps, size_t smem,
                                 int blocks, cudaStream_t st, int *blocks_per_sm) {
    auto fn = batch_step_kernel<V>;
    static int configured_smem = -1;
    if ((int)smem > configured_smem) {
        cudaError_t e =
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured_smem = (int)smem;
    }
    if (blocks_per_sm) {
        cudaError_t e =
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, fn, warps * 32, smem);
        if (e != cudaSuccess) return e;
    }
    if (blocks == 0) return cudaSuccess;
    fn<<<blocks, warps * 32, smem, st>>>(b);
    return cudaGetLastError();
}

template <typename T, bool IMAG>
cudaError_t launch_batch_t(int phase, const BatchArgs<T> &b, int warps, size_t smem, int blocks,
                           cudaStream_t st, int *bps) {
    if (phase == 2) return launch_batch_variant<Variant<T, 2, IMAG, false, 2>>(b, warps, smem, blocks, st, bps);
    if (phase == 1) return launch_batch_variant<Variant<T, 2, IMAG, false, 1>>(b, warps, smem, blocks, st, bps);
    return launch_batch_variant<Variant<T, 2, IMAG, false, 0>>(b, warps, smem, blocks, st, bps);
}

}  // namespace tsb
