// Entry points of the separately compiled look-ahead walk variants
// (step2_f{64,32}_{real,imag}.cu) and the walk's shared-memory geometry.
#pragma once
#include <cuda_runtime.h>

#include "step_kernel.cuh"
#include "walk2_shape.h"

namespace tsb {

// The look-ahead walk (walk2.cuh): phases 0-2, cartesian, one component;
// R rows per iteration (1, or 2 with 2 cells per lane); pdl: programmatic
// dependent launch after the stream's previous kernel.
cudaError_t launch_step2_f64_real(int C, int R, int phase, const StepArgs<double> &a, int warps,
                                  size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                  bool pdl);
cudaError_t launch_step2_f64_imag(int C, int R, int phase, const StepArgs<double> &a, int warps,
                                  size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                  bool pdl);
cudaError_t launch_step2_f32_real(int C, int R, int phase, const StepArgs<float> &a, int warps,
                                  size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                  bool pdl);
cudaError_t launch_step2_f32_imag(int C, int R, int phase, const StepArgs<float> &a, int warps,
                                  size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                  bool pdl);

// The same in a rotating frame (2 cells per lane, or 4 in single precision;
// step2rot_f{64,32}_{real,imag}.cu), for one species of a pair (phases 3 and
// 7; step2pair_*.cu) and on cylindrical lattices (phases 4-6; step2cyl_*.cu).
cudaError_t launch_step2rot_f64_real(int C, int R, int phase, const StepArgs<double> &a,
                                     int warps, size_t smem, int blocks, cudaStream_t st,
                                     int *blocks_per_sm, bool pdl);
cudaError_t launch_step2rot_f64_imag(int C, int R, int phase, const StepArgs<double> &a,
                                     int warps, size_t smem, int blocks, cudaStream_t st,
                                     int *blocks_per_sm, bool pdl);
cudaError_t launch_step2rot_f32_real(int C, int R, int phase, const StepArgs<float> &a,
                                     int warps, size_t smem, int blocks, cudaStream_t st,
                                     int *blocks_per_sm, bool pdl);
cudaError_t launch_step2rot_f32_imag(int C, int R, int phase, const StepArgs<float> &a,
                                     int warps, size_t smem, int blocks, cudaStream_t st,
                                     int *blocks_per_sm, bool pdl);
cudaError_t launch_step2pair_f64_real(int R, int phase, const StepArgs<double> &a, int warps,
                                      size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                      bool pdl);
cudaError_t launch_step2pair_f64_imag(int R, int phase, const StepArgs<double> &a, int warps,
                                      size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                      bool pdl);
cudaError_t launch_step2pair_f32_real(int R, int phase, const StepArgs<float> &a, int warps,
                                      size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                      bool pdl);
cudaError_t launch_step2pair_f32_imag(int R, int phase, const StepArgs<float> &a, int warps,
                                      size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                      bool pdl);
cudaError_t launch_step2cyl_f64_real(int R, int phase, const StepArgs<double> &a, int warps,
                                     size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                     bool pdl);
cudaError_t launch_step2cyl_f64_imag(int R, int phase, const StepArgs<double> &a, int warps,
                                     size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                     bool pdl);
cudaError_t launch_step2cyl_f32_real(int R, int phase, const StepArgs<float> &a, int warps,
                                     size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                     bool pdl);
cudaError_t launch_step2cyl_f32_imag(int R, int phase, const StepArgs<float> &a, int warps,
                                     size_t smem, int blocks, cudaStream_t st, int *blocks_per_sm,
                                     bool pdl);

}  // namespace tsb
