// Launch templates of the batched step on the look-ahead walk; one
// translation unit per precision and time mode (batch2_f{64,32}_{real,imag}.cu).
#pragma once
#include "batch_launch.h"
#include "walk2.cuh"

namespace tsb {

template <class V>
cudaError_t launch_batch2_variant(const BatchArgs<typename V::T> &b, int warps, size_t smem,
                                  int blocks, cudaStream_t st, int *blocks_per_sm) {
    auto fn = batch2_kernel<V, 2>;
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
cudaError_t launch_batch2_t(int phase, const BatchArgs<T> &b, int warps, size_t smem, int blocks,
                            cudaStream_t st, int *bps) {
    if (phase == 2) return launch_batch2_variant<Variant<T, 2, IMAG, false, 2>>(b, warps, smem, blocks, st, bps);
    if (phase == 1) return launch_batch2_variant<Variant<T, 2, IMAG, false, 1>>(b, warps, smem, blocks, st, bps);
    return launch_batch2_variant<Variant<T, 2, IMAG, false, 0>>(b, warps, smem, blocks, st, bps);
}

}  // namespace tsb
