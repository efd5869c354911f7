// Launch templates of the look-ahead walk (walk2.cuh); one translation unit
// per precision and time mode (step2_f{64,32}_{real,imag}.cu).
#pragma once
#include "step2_decl.h"
#include "walk2.cuh"

namespace tsb {

// pdl: launch with a programmatic dependency on the stream's previous kernel
// (the set-up of this step overlaps the end of the previous one)
template <class V, int R = 1>
cudaError_t launch_step2_variant(const StepArgs<typename V::T> &a, int warps, size_t smem,
                                 int blocks, cudaStream_t st, int *blocks_per_sm, bool pdl) {
    auto fn = step2_kernel<V, R>;
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
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3((unsigned)(warps * 32));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, fn, a);
}

// R: rows per iteration of the walk (2: cells per lane 2 only)
template <typename T, bool IMAG>
cudaError_t launch_step2_t(int C, int R, int phase, const StepArgs<T> &a, int warps, size_t smem,
                           int blocks, cudaStream_t st, int *bps, bool pdl) {
    if constexpr (std::is_same<T, double>::value && !IMAG) {
        // the table's entries from potential rows (phase bit 16)
        if (C == 2 && R == 2 && phase >= 16) {
            if (phase == 16) return launch_step2_variant<Variant<T, 2, false, false, 16>, 2>(a, warps, smem, blocks, st, bps, pdl);
            if (phase == 17) return launch_step2_variant<Variant<T, 2, false, false, 17>, 2>(a, warps, smem, blocks, st, bps, pdl);
            if (phase == 18) return launch_step2_variant<Variant<T, 2, false, false, 18>, 2>(a, warps, smem, blocks, st, bps, pdl);
        }
    }
    if (C == 2 && R == 2) {
        if (phase == 0) return launch_step2_variant<Variant<T, 2, IMAG, false, 0>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 1) return launch_step2_variant<Variant<T, 2, IMAG, false, 1>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 2) return launch_step2_variant<Variant<T, 2, IMAG, false, 2>, 2>(a, warps, smem, blocks, st, bps, pdl);
        return cudaErrorInvalidValue;
    }
    if (R != 1) return cudaErrorInvalidValue;
    if (C == 2) {
        if (phase == 0) return launch_step2_variant<Variant<T, 2, IMAG, false, 0>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 1) return launch_step2_variant<Variant<T, 2, IMAG, false, 1>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 2) return launch_step2_variant<Variant<T, 2, IMAG, false, 2>>(a, warps, smem, blocks, st, bps, pdl);
    } else if (C == 4) {
        if (phase == 0) return launch_step2_variant<Variant<T, 4, IMAG, false, 0>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 1) return launch_step2_variant<Variant<T, 4, IMAG, false, 1>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 2) return launch_step2_variant<Variant<T, 4, IMAG, false, 2>>(a, warps, smem, blocks, st, bps, pdl);
    }
    return cudaErrorInvalidValue;
}

// The rotating frame (2 cells per lane; 4 in single precision), R rows per
// iteration.
template <typename T, bool IMAG>
cudaError_t launch_step2rot_t(int C, int R, int phase, const StepArgs<T> &a, int warps, size_t smem,
                              int blocks, cudaStream_t st, int *bps, bool pdl) {
    if constexpr (sizeof(T) == 4) {
        if (C == 4 && R == 2) {
            if (phase == 0) return launch_step2_variant<Variant<T, 4, IMAG, true, 0>, 2>(a, warps, smem, blocks, st, bps, pdl);
            if (phase == 1) return launch_step2_variant<Variant<T, 4, IMAG, true, 1>, 2>(a, warps, smem, blocks, st, bps, pdl);
            if (phase == 2) return launch_step2_variant<Variant<T, 4, IMAG, true, 2>, 2>(a, warps, smem, blocks, st, bps, pdl);
            return cudaErrorInvalidValue;
        }
        if (C == 4 && R == 1) {
            if (phase == 0) return launch_step2_variant<Variant<T, 4, IMAG, true, 0>>(a, warps, smem, blocks, st, bps, pdl);
            if (phase == 1) return launch_step2_variant<Variant<T, 4, IMAG, true, 1>>(a, warps, smem, blocks, st, bps, pdl);
            if (phase == 2) return launch_step2_variant<Variant<T, 4, IMAG, true, 2>>(a, warps, smem, blocks, st, bps, pdl);
            return cudaErrorInvalidValue;
        }
    }
    if (C != 2) return cudaErrorInvalidValue;
    if (R == 2) {
        if (phase == 0) return launch_step2_variant<Variant<T, 2, IMAG, true, 0>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 1) return launch_step2_variant<Variant<T, 2, IMAG, true, 1>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 2) return launch_step2_variant<Variant<T, 2, IMAG, true, 2>, 2>(a, warps, smem, blocks, st, bps, pdl);
    } else if (R == 1) {
        if (phase == 0) return launch_step2_variant<Variant<T, 2, IMAG, true, 0>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 1) return launch_step2_variant<Variant<T, 2, IMAG, true, 1>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 2) return launch_step2_variant<Variant<T, 2, IMAG, true, 2>>(a, warps, smem, blocks, st, bps, pdl);
    }
    return cudaErrorInvalidValue;
}

// One species of a pair (2 cells per lane): phase 3, and 7 (the Rabi
// rotation at load, Variant phase 11, real time), R rows per iteration.
template <typename T, bool IMAG>
cudaError_t launch_step2pair_t(int R, int phase, const StepArgs<T> &a, int warps, size_t smem,
                               int blocks, cudaStream_t st, int *bps, bool pdl) {
    if (R == 2) {
        if (phase == 3) return launch_step2_variant<Variant<T, 2, IMAG, false, 3>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if constexpr (!IMAG)
            if (phase == 7) return launch_step2_variant<Variant<T, 2, IMAG, false, 11>, 2>(a, warps, smem, blocks, st, bps, pdl);
    } else if (R == 1) {
        if (phase == 3) return launch_step2_variant<Variant<T, 2, IMAG, false, 3>>(a, warps, smem, blocks, st, bps, pdl);
        if constexpr (!IMAG)
            if (phase == 7) return launch_step2_variant<Variant<T, 2, IMAG, false, 11>>(a, warps, smem, blocks, st, bps, pdl);
    }
    return cudaErrorInvalidValue;
}

// Cylindrical lattices (2 cells per lane): phases 4-6, R rows per iteration.
template <typename T, bool IMAG>
cudaError_t launch_step2cyl_t(int R, int phase, const StepArgs<T> &a, int warps, size_t smem,
                              int blocks, cudaStream_t st, int *bps, bool pdl) {
    if (R == 2) {
        if (phase == 4) return launch_step2_variant<Variant<T, 2, IMAG, false, 4>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 5) return launch_step2_variant<Variant<T, 2, IMAG, false, 5>, 2>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 6) return launch_step2_variant<Variant<T, 2, IMAG, false, 6>, 2>(a, warps, smem, blocks, st, bps, pdl);
    } else if (R == 1) {
        if (phase == 4) return launch_step2_variant<Variant<T, 2, IMAG, false, 4>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 5) return launch_step2_variant<Variant<T, 2, IMAG, false, 5>>(a, warps, smem, blocks, st, bps, pdl);
        if (phase == 6) return launch_step2_variant<Variant<T, 2, IMAG, false, 6>>(a, warps, smem, blocks, st, bps, pdl);
    }
    return cudaErrorInvalidValue;
}

}  // namespace tsb
