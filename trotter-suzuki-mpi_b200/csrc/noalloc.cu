// Squared norm of a caller-owned device tile without any device allocation.
//
// Some callers of this library cannot call cudaMalloc: code whose device
// memory is owned by another allocator (a framework's caching allocator or a
// fixed pool sized at start-up, where a foreign cudaMalloc can fail or
// fragment the pool), and code that must not allocate after start-up because
// cudaMalloc/cudaFree can synchronise the device and stall a pipeline of
// queued work.  ts_b200_squared_norm_noalloc serves them: the caller passes the
// tile and the output, and the reduction's scratch lives in a file-scope
// device array of this library.
//
// The scratch holds one FP64 partial per inner row plus a completion ticket:
// at most TSB_NOALLOC_MAX_ROWS rows (128 KiB), held by every GPU that loads
// the library until the process exits.  Every call shares it and it keeps the
// last call's contents; the ticket is cleared before each launch, the row
// partials are always written before they are read.  Calls that overlap on the
// GPU (different streams, no ordering between them) race on the scratch.
#include <cuda_runtime.h>

#include <mutex>

#include "step_kernel.cuh"
#include "ts_b200.h"

namespace {

constexpr int TSB_NOALLOC_MAX_ROWS = 16384;
constexpr int NA_THREADS = 256;
constexpr int NA_MAX_DEVICES = 64;

struct NoallocScratch {
    double row_sum[TSB_NOALLOC_MAX_ROWS];
    unsigned int ticket;
};

static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch, looked up once per device.
NoallocScratch *g_scratch_ptr[NA_MAX_DEVICES] = {};
std::mutex g_scratch_mutex;

int scratch_for_current_device(NoallocScratch **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TS_B200_NO_DEVICE;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return TS_B200_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
            return TS_B200_CUDA_ERROR;
        g_scratch_ptr[dev] = static_cast<NoallocScratch *>(p);
    }
    *out = g_scratch_ptr[dev];
    return TS_B200_OK;
}

// One warp per row (rows strided over the grid's warps), lanes stride the
// row's inner columns; then the last block to finish adds the row partials in
// row order, so the result does not depend on the grid size.
template <typename T>
__global__ void __launch_bounds__(NA_THREADS)
    noalloc_norm_kernel(const tsb::Cx<T> *psi, size_t pitch, int x0, int x1, int y0, int rows,
                        double dxdy, NoallocScratch *scratch, double *out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int warps_total = gridDim.x * (blockDim.x >> 5);
    for (int r = blockIdx.x * (blockDim.x >> 5) + warp; r < rows; r += warps_total) {
        const tsb::Cx<T> *row = psi + (size_t)(y0 + r) * pitch;
        double s = 0.0;
        for (int x = x0 + lane; x < x1; x += 32) {
            const double re = (double)row[x].re, im = (double)row[x].im;
            s += re * re + im * im;
        }
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) scratch->row_sum[r] = s;
    }
    __shared__ unsigned int s_last;
    __shared__ double red[NA_THREADS];
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&scratch->ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double s = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) s += __ldcg(&scratch->row_sum[r]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = red[0] * dxdy;
        scratch->ticket = 0u;
    }
}

}  // namespace

extern "C" int ts_b200_squared_norm_noalloc(const void *psi, int precision, size_t pitch,
                                            int dim_x, int dim_y, int inner_x0, int inner_x1,
                                            int inner_y0, int inner_y1, double delta_x,
                                            double delta_y, double *out, void *stream) {
    if (!psi || !out || dim_x < 1 || dim_y < 1 || pitch < (size_t)dim_x || inner_x0 < 0 ||
        inner_x1 > dim_x || inner_x0 >= inner_x1 || inner_y0 < 0 || inner_y1 > dim_y ||
        inner_y0 >= inner_y1 || (precision != TS_B200_FP64 && precision != TS_B200_FP32))
        return TS_B200_INVALID_ARGUMENT;
    const int rows = inner_y1 - inner_y0;
    if (rows > TSB_NOALLOC_MAX_ROWS) return TS_B200_UNSUPPORTED;  // scratch holds 16384 rows
    NoallocScratch *scratch = nullptr;
    int st = scratch_for_current_device(&scratch);
    if (st != TS_B200_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(&scratch->ticket, 0, sizeof(unsigned int), s) != cudaSuccess)
        return TS_B200_CUDA_ERROR;
    const int blocks = (rows + (NA_THREADS / 32) - 1) / (NA_THREADS / 32);
    const int grid = blocks < 1184 ? blocks : 1184;
    const double dxdy = delta_x * delta_y;
    if (precision == TS_B200_FP64)
        noalloc_norm_kernel<double><<<grid, NA_THREADS, 0, s>>>(
            static_cast<const tsb::Cx<double> *>(psi), pitch, inner_x0, inner_x1, inner_y0, rows,
            dxdy, scratch, out);
    else
        noalloc_norm_kernel<float><<<grid, NA_THREADS, 0, s>>>(
            static_cast<const tsb::Cx<float> *>(psi), pitch, inner_x0, inner_x1, inner_y0, rows,
            dxdy, scratch, out);
    return cudaGetLastError() == cudaSuccess ? TS_B200_OK : TS_B200_CUDA_ERROR;
}
