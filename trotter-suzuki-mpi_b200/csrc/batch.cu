// Batched evolution: many tiles of uneven sizes advanced together, one
// persistent launch per Trotter step (include/ts_b200.h, ts_b200_batch_*).
//
// A batch borrows the device buffers of existing tile handles
// (ts_b200_kernel): their state, exponential tables and scalars.  Per step it
// launches the batched step kernel (batch2_kernel on the look-ahead walk,
// batch_step_kernel on the checked walk) over the task list of all tiles, then (in
// imaginary time) one reduction block per tile that turns the task partials
// into the tile's squared norm and renormalisation factor, then (for tiles
// with periodic boundaries, except on the last step of an evolve) one
// batched halo refresh.  Runs of 32 steps are replayed from a CUDA graph.
//
// The tile shape (rows per segment task, warps per block) is chosen by a
// timing autotuner over a small candidate set; the choice is cached per batch
// signature (precision, time mode, tile sizes) for the process.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "batch_launch.h"
#include "halo.cuh"
#include "handle.h"
#include "ts_b200.h"
#include "walk2_shape.h"

using tsb::BatchArgs;
using tsb::Cx;
using tsb::Scalars;
using tsb::StepArgs;
using tsbh::div_up;
using tsbh::g_launches;

namespace {

// Per tile: where its tasks sit in the task list (imaginary-time reduction).
struct TileNorm {
    int first, count;
    double dxdy, norm0;
    Scalars *scal;
};

// Per periodic tile: the halo refresh geometry.
struct TileHalo {
    int tile;
    int W, H, P, hx, hy, px, py, iy0;
};

constexpr int kGraphSteps = 32;
constexpr int kNormThreads = 256;

__global__ void batch_norm_kernel(const TileNorm *tn, const double *task_norm) {
    const TileNorm n = tn[blockIdx.x];
    __shared__ double red[kNormThreads];
    double s = 0.0;
    for (int i = threadIdx.x; i < n.count; i += blockDim.x) s += task_norm[n.first + i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double tot = red[0] * n.dxdy;
        n.scal->last_norm = tot;
        if (n.scal->renorm) n.scal->pending_inv = 1.0 / sqrt(tot / n.norm0);
    }
}

// FP32 real time: every tile's coefficient schedule advances by one step
// (the single-tile kernel's last block does this for its own tile).
__global__ void batch_step_count_kernel(const TileNorm *tn, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) tn[i].scal->step += 1u;
}

// blockIdx.y: periodic tile; the x blocks stride over its destination cells.
template <typename T>
__global__ void batch_halo_kernel(const StepArgs<T> *inst, const TileHalo *th) {
    const TileHalo h = th[blockIdx.y];
    Cx<T> *psi = reinterpret_cast<Cx<T> *>(const_cast<void *>(inst[h.tile].psi_out));
    tsb::halo_cells(psi, h.W, h.H, h.P, h.hx, h.hy, h.px, h.py, h.iy0, h.iy0 + h.H - 2 * h.hy,
                    blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

struct Shape {
    int seg_rows;  // rows per segment task (even)
    int warps;     // warps per block
};

std::mutex g_tune_mutex;
std::map<std::vector<long>, Shape> g_tuned;  // batch signature -> shape

}  // namespace

struct ts_b200_batch {
    std::vector<ts_b200_kernel *> k;
    bool fp32 = false, imag = false;
    int phase = 0;
    int device = 0, num_sms = 148;
    Shape shape{128, 4};
    // row walk: 2 the look-ahead walk (two rows per iteration, a ring of 6
    // rows), 0 the checked walk (a ring of `ring` rows)
    int walk = 0;
    int ring = 4;
    int resident_blocks = 0;  // of the current shape (0: unknown)
    int n_tasks = 0;
    int sum_strips = 0, sum_segs = 0;
    size_t args_bytes = 0;        // sizeof(StepArgs<T>)
    void *d_args[2] = {nullptr, nullptr};  // per tile, step parity 0 / 1
    int2 *d_tasks = nullptr;
    size_t tasks_cap = 0;
    double *d_task_norm = nullptr;
    TileNorm *d_norm = nullptr;
    TileHalo *d_halo = nullptr;
    int n_halo = 0, halo_cells_max = 0;
    int *d_error = nullptr;
    std::vector<int> args_cur;    // cur of each tile the argument tables were built for
    bool layout_valid = false;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaEvent_t ev = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::string err;
};

namespace {

int bfail(ts_b200_batch *b, int status, const std::string &msg) {
    if (b) b->err = msg;
    return status;
}

int bcuda(ts_b200_batch *b, cudaError_t e, const char *what) {
    if (b) b->err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR;
}

#define TSBB_CHECK(b, call)                                  \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return bcuda(b, e_, #call);   \
    } while (0)

constexpr int kHX = 4, kHY = 4;   // halo of the 2-cell, rotation-free strips
constexpr int kWO = 64 - 2 * kHX; // output columns per strip

int even_up(int n) { return n + (n & 1); }

int tile_seg_rows(const ts_b200_kernel *t, int seg_rows) {
    return std::max(2, std::min(even_up(t->H), even_up(seg_rows)));
}

// Look-ahead walk: vertical pair table entries per warp, for the tallest
// segment of the batch.
int batch_vlen(const ts_b200_batch *b) {
    int seg = 2;
    for (const ts_b200_kernel *t : b->k) seg = std::max(seg, tile_seg_rows(t, b->shape.seg_rows));
    return tsb::w2_vlen(seg, false);
}

size_t batch_smem(const ts_b200_batch *b, int warps) {
    if (b->walk) {
        // per warp: the ring, the vertical pair table and one mbarrier per
        // ring slot of two rows
        return (size_t)warps * (b->ring * tsbh::slot_bytes(2, b->fp32, b->imag) +
                                (size_t)batch_vlen(b) * (b->fp32 ? 8 : 16) + (b->ring / 2) * 8);
    }
    return (size_t)warps * (b->ring * tsbh::slot_bytes(2, b->fp32, b->imag) + 8 * b->ring);
}

void drop_batch_graph(ts_b200_batch *b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
}

template <typename T>
cudaError_t launch_batch_kernel(ts_b200_batch *b, const BatchArgs<T> &a, int blocks, int *bps);

template <>
cudaError_t launch_batch_kernel<double>(ts_b200_batch *b, const BatchArgs<double> &a, int blocks,
                                        int *bps) {
    const size_t smem = batch_smem(b, b->shape.warps);
    if (b->walk)
        return b->imag ? tsb::launch_batch2_f64_imag(b->phase, a, b->shape.warps, smem, blocks,
                                                     b->stream, bps)
                       : tsb::launch_batch2_f64_real(b->phase, a, b->shape.warps, smem, blocks,
                                                     b->stream, bps);
    return tsb::launch_batch_f64(b->imag, b->phase, a, b->shape.warps, smem, blocks, b->stream, bps);
}
template <>
cudaError_t launch_batch_kernel<float>(ts_b200_batch *b, const BatchArgs<float> &a, int blocks,
                                       int *bps) {
    const size_t smem = batch_smem(b, b->shape.warps);
    if (b->walk)
        return b->imag ? tsb::launch_batch2_f32_imag(b->phase, a, b->shape.warps, smem, blocks,
                                                     b->stream, bps)
                       : tsb::launch_batch2_f32_real(b->phase, a, b->shape.warps, smem, blocks,
                                                     b->stream, bps);
    return tsb::launch_batch_f32(b->imag, b->phase, a, b->shape.warps, smem, blocks, b->stream, bps);
}

// Task list, per-tile reduction table and halo table for the current shape.
template <typename T>
int build_layout(ts_b200_batch *b) {
    const int n = (int)b->k.size();
    std::vector<int2> tasks;
    std::vector<TileNorm> norms(n);
    std::vector<TileHalo> halos;
    b->sum_strips = b->sum_segs = 0;
    b->halo_cells_max = 0;
    for (int i = 0; i < n; ++i) {
        const ts_b200_kernel *t = b->k[i];
        const int sh = tile_seg_rows(t, b->shape.seg_rows);
        const int strips = div_up(t->W, kWO), segs = div_up(t->H, sh);
        norms[i] = TileNorm{(int)tasks.size(), strips * segs, t->d.delta_x * t->d.delta_y,
                            t->d.norm0, t->scal};
        for (int j = 0; j < strips * segs; ++j) tasks.push_back(make_int2(i, j));
        b->sum_strips += strips;
        b->sum_segs += segs;
        if (t->d.periodic_x || t->d.periodic_y) {
            halos.push_back(TileHalo{i, t->W, t->H, t->P, t->d.halo_x, t->d.halo_y,
                                     t->d.periodic_x, t->d.periodic_y, t->d.inner_y0});
            b->halo_cells_max = std::max(b->halo_cells_max,
                                         tsb::halo_cell_count(t->W, t->H, t->d.halo_x, t->d.halo_y,
                                                              t->d.periodic_x, t->d.periodic_y));
        }
    }
    b->n_tasks = (int)tasks.size();
    b->n_halo = (int)halos.size();
    if (tasks.size() > b->tasks_cap) {
        if (b->d_tasks) cudaFree(b->d_tasks);
        if (b->d_task_norm) cudaFree(b->d_task_norm);
        b->d_tasks = nullptr;
        b->d_task_norm = nullptr;
        TSBB_CHECK(b, cudaMalloc(&b->d_tasks, tasks.size() * sizeof(int2)));
        TSBB_CHECK(b, cudaMalloc(&b->d_task_norm, tasks.size() * sizeof(double)));
        b->tasks_cap = tasks.size();
    }
    TSBB_CHECK(b, cudaMemcpyAsync(b->d_tasks, tasks.data(), tasks.size() * sizeof(int2),
                                  cudaMemcpyHostToDevice, b->stream));
    TSBB_CHECK(b, cudaMemcpyAsync(b->d_norm, norms.data(), n * sizeof(TileNorm),
                                  cudaMemcpyHostToDevice, b->stream));
    if (!halos.empty())
        TSBB_CHECK(b, cudaMemcpyAsync(b->d_halo, halos.data(), halos.size() * sizeof(TileHalo),
                                      cudaMemcpyHostToDevice, b->stream));
    // the host vectors die here: the copies must have read them
    TSBB_CHECK(b, cudaStreamSynchronize(b->stream));
    b->layout_valid = true;
    b->args_cur.assign(n, -1);  // the argument tables carry the task geometry too
    drop_batch_graph(b);
    if (b->resident_blocks <= 0) {
        BatchArgs<T> a0{};
        int bps = 0;
        cudaError_t e = launch_batch_kernel<T>(b, a0, 0, &bps);
        if (e != cudaSuccess) return bcuda(b, e, "batch kernel configuration");
        if (bps < 1) return bfail(b, TS_B200_UNSUPPORTED, "batch kernel does not fit on an SM");
        b->resident_blocks = bps * b->num_sms;
    }
    return TS_B200_OK;
}

// Argument tables for both step parities from the tiles' current buffers.
template <typename T>
int build_args(ts_b200_batch *b) {
    const int n = (int)b->k.size();
    bool same = (int)b->args_cur.size() == n;
    for (int i = 0; same && i < n; ++i) same = b->args_cur[i] == b->k[i]->cur;
    if (same) return TS_B200_OK;
    std::vector<StepArgs<T>> par[2];
    par[0].resize(n);
    par[1].resize(n);
    for (int i = 0; i < n; ++i) {
        ts_b200_kernel *t = b->k[i];
        StepArgs<T> a{};
        tsbh::fill_step_constants(t, a);
        const int sh = tile_seg_rows(t, b->shape.seg_rows);
        a.n_strips = div_up(t->W, kWO);
        a.n_segs = div_up(t->H, sh);
        a.seg_h = sh;
        a.ring = b->ring;
        a.partials = nullptr;
        for (int p = 0; p < 2; ++p) {
            a.psi_in = t->psi[t->cur ^ p];
            a.psi_out = t->psi[t->cur ^ p ^ 1];
            par[p][i] = a;
        }
    }
    for (int p = 0; p < 2; ++p)
        TSBB_CHECK(b, cudaMemcpyAsync(b->d_args[p], par[p].data(), n * sizeof(StepArgs<T>),
                                      cudaMemcpyHostToDevice, b->stream));
    TSBB_CHECK(b, cudaStreamSynchronize(b->stream));
    for (int i = 0; i < n; ++i) b->args_cur[i] = b->k[i]->cur;
    return TS_B200_OK;
}

// One step of every tile: parity p selects the argument table.
template <typename T>
int launch_batch_step(ts_b200_batch *b, int p, bool exchange, bool renorm_pass = true) {
    BatchArgs<T> a{};
    a.inst = static_cast<const StepArgs<T> *>(b->d_args[p]);
    a.tasks = b->d_tasks;
    a.task_norm = b->d_task_norm;
    a.error = b->d_error;
    a.n_tasks = b->n_tasks;
    a.ring = b->ring;
    a.vlen = b->walk ? batch_vlen(b) : 0;
    const int blocks = std::max(1, std::min(b->resident_blocks, div_up(b->n_tasks, b->shape.warps)));
    cudaError_t e = launch_batch_kernel<T>(b, a, blocks, nullptr);
    if (e != cudaSuccess) return bcuda(b, e, "batch step launch");
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (b->fp32 && !b->imag && renorm_pass) {
        const int n = (int)b->k.size();
        batch_step_count_kernel<<<div_up(n, 256), 256, 0, b->stream>>>(b->d_norm, n);
        e = cudaGetLastError();
        if (e != cudaSuccess) return bcuda(b, e, "batch step count launch");
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    if (b->imag && renorm_pass) {
        batch_norm_kernel<<<(unsigned)b->k.size(), kNormThreads, 0, b->stream>>>(b->d_norm,
                                                                               b->d_task_norm);
        e = cudaGetLastError();
        if (e != cudaSuccess) return bcuda(b, e, "batch norm launch");
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    if (exchange && b->n_halo > 0) {
        const unsigned gx = (unsigned)std::max(1, std::min(div_up(b->halo_cells_max, 256), 1024));
        batch_halo_kernel<T><<<dim3(gx, (unsigned)b->n_halo), 256, 0, b->stream>>>(
            static_cast<const StepArgs<T> *>(b->d_args[p]), b->d_halo);
        e = cudaGetLastError();
        if (e != cudaSuccess) return bcuda(b, e, "batch halo launch");
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
    return TS_B200_OK;
}

int kernels_per_batch_step(const ts_b200_batch *b, bool exchange) {
    return 1 + ((b->imag || b->fp32) ? 1 : 0) + ((exchange && b->n_halo > 0) ? 1 : 0);
}

// The batch stream waits for every tile's queued work, or the tiles' streams
// wait for the batch.
int join_tiles(ts_b200_batch *b, bool tiles_first) {
    for (ts_b200_kernel *t : b->k) {
        if (t->stream == b->stream) continue;
        if (tiles_first) {
            TSBB_CHECK(b, cudaEventRecord(b->ev, t->stream));
            TSBB_CHECK(b, cudaStreamWaitEvent(b->stream, b->ev, 0));
        } else {
            TSBB_CHECK(b, cudaStreamWaitEvent(t->stream, b->ev, 0));
        }
    }
    if (!tiles_first) return TS_B200_OK;
    return TS_B200_OK;
}

template <typename T>
int evolve_t(ts_b200_batch *b, int iterations) {
    if (!b->layout_valid) {
        int s = build_layout<T>(b);
        if (s) return s;
    }
    int s = join_tiles(b, true);
    if (s) return s;
    s = build_args<T>(b);
    if (s) return s;
    // Steps 0 .. iterations-2 refresh the halos, the last one does not
    // (src/solver.cpp:203-209).  Step j uses argument table j & 1.
    int remaining = iterations - 1;
    int parity = 0;
    if (remaining >= kGraphSteps) {
        if (!b->graph) {
            cudaGraph_t g = nullptr;
            TSBB_CHECK(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = g_launches.load();
            int st = TS_B200_OK;
            for (int i = 0; i < kGraphSteps && st == TS_B200_OK; ++i) st = launch_batch_step<T>(b, i & 1, true);
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            g_launches.store(before);
            if (st != TS_B200_OK || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                (void)cudaGetLastError();
                if (st != TS_B200_OK) return st;
                return bcuda(b, e, "batch graph capture");
            }
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return bcuda(b, e, "batch graph instantiate");
        }
        const int per = kernels_per_batch_step(b, true);
        while (remaining >= kGraphSteps) {
            TSBB_CHECK(b, cudaGraphLaunch(b->graph, b->stream));
            g_launches.fetch_add((uint64_t)kGraphSteps * per, std::memory_order_relaxed);
            remaining -= kGraphSteps;
        }
    }
    for (; remaining > 0; --remaining) {
        s = launch_batch_step<T>(b, parity, true);
        if (s) return s;
        parity ^= 1;
    }
    s = launch_batch_step<T>(b, parity, false);
    if (s) return s;
    for (ts_b200_kernel *t : b->k) t->cur ^= (iterations & 1);
    TSBB_CHECK(b, cudaEventRecord(b->ev, b->stream));
    return join_tiles(b, false);
}

// Device time of `steps` batched steps that all read the tiles' current
// buffers and write the other ones (the state the tiles hold is unchanged;
// no renormalisation pass), after one untimed step.
template <typename T>
int time_shape(ts_b200_batch *b, int steps, float *ms) {
    int s = build_layout<T>(b);
    if (s) return s;
    s = build_args<T>(b);
    if (s) return s;
    s = launch_batch_step<T>(b, 0, false, false);
    if (s) return s;
    cudaEvent_t e0, e1;
    TSBB_CHECK(b, cudaEventCreate(&e0));
    TSBB_CHECK(b, cudaEventCreate(&e1));
    cudaEventRecord(e0, b->stream);
    for (int i = 0; i < steps && s == TS_B200_OK; ++i) s = launch_batch_step<T>(b, 0, false, false);
    cudaEventRecord(e1, b->stream);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s) return s;
    if (e != cudaSuccess) return bcuda(b, e, "autotune timing");
    return TS_B200_OK;
}

std::vector<long> signature(const ts_b200_batch *b) {
    std::vector<long> sig{b->fp32 ? 1L : 0L, b->imag ? 1L : 0L, (long)b->phase};
    for (const ts_b200_kernel *t : b->k) {
        sig.push_back(t->W);
        sig.push_back(t->H);
    }
    return sig;
}

template <typename T>
int autotune_t(ts_b200_batch *b, int trial_steps, int use_cache) {
    const std::vector<long> sig = signature(b);
    if (use_cache) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tuned.find(sig);
        if (it != g_tuned.end()) {
            if (it->second.seg_rows != b->shape.seg_rows || it->second.warps != b->shape.warps) {
                b->shape = it->second;
                b->resident_blocks = 0;
                b->layout_valid = false;
            }
            return TS_B200_OK;
        }
    }
    int s = join_tiles(b, true);
    if (s) return s;
    static const int kSegRows[] = {16, 32, 64, 96, 128, 192, 256};
    static const int kWarps[] = {4, 2};
    constexpr int kShapes = 14;
    // two passes over the candidates, each keeping its faster time: a clock
    // that moves during the search (power capping) then favours no shape
    float shape_ms[kShapes];
    for (int pass = 0; pass < 2; ++pass) {
        int i = 0;
        for (int wv : kWarps) {
            for (int sr : kSegRows) {
                b->shape = Shape{sr, wv};
                b->resident_blocks = 0;
                b->layout_valid = false;
                float ms = 0.0f;
                s = time_shape<T>(b, trial_steps, &ms);
                if (s) return s;
                shape_ms[i] = pass == 0 ? ms : std::min(shape_ms[i], ms);
                ++i;
            }
        }
    }
    Shape best = b->shape;
    float best_ms = -1.0f;
    {
        int i = 0;
        for (int wv : kWarps) {
            for (int sr : kSegRows) {
                if (best_ms < 0.0f || shape_ms[i] < best_ms) {
                    best_ms = shape_ms[i];
                    best = Shape{sr, wv};
                }
                ++i;
            }
        }
    }
    b->shape = best;
    b->resident_blocks = 0;
    b->layout_valid = false;
    s = build_layout<T>(b);
    if (s) return s;
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tuned[sig] = best;
    }
    TSBB_CHECK(b, cudaEventRecord(b->ev, b->stream));
    return join_tiles(b, false);
}

}  // namespace

extern "C" {

int ts_b200_batch_create(ts_b200_kernel *const *kernels, int n, ts_b200_batch **out) {
    if (!out) return TS_B200_INVALID_ARGUMENT;
    *out = nullptr;
    if (!kernels || n < 1) return TS_B200_INVALID_ARGUMENT;
    const ts_b200_kernel *k0 = kernels[0];
    if (!k0) return TS_B200_INVALID_ARGUMENT;
    int phase = 0;
    bool walk2 = true;
    for (int i = 0; i < n; ++i) {
        const ts_b200_kernel *t = kernels[i];
        if (!t) return TS_B200_INVALID_ARGUMENT;
        for (int j = 0; j < i; ++j)
            if (kernels[j] == t) return TS_B200_INVALID_ARGUMENT;  // a tile appears once
        if (t->fp32 != k0->fp32 || t->imag != k0->imag || t->device != k0->device)
            return TS_B200_INVALID_ARGUMENT;
        // batched strips carry no rotating frame, second species or radial term
        if (t->rot || t->pair_mode || t->cyl) return TS_B200_UNSUPPORTED;
        phase = std::max(phase, t->phase);
        walk2 = walk2 && t->walk2 > 0;
    }
    ts_b200_batch *b = new (std::nothrow) ts_b200_batch();
    if (!b) return TS_B200_OUT_OF_MEMORY;
    b->k.assign(kernels, kernels + n);
    b->fp32 = k0->fp32;
    b->imag = k0->imag;
    b->phase = phase;
    b->walk = walk2 ? 2 : 0;
    b->ring = walk2 ? 6 : 4;
    b->device = k0->device;
    b->num_sms = k0->num_sms;
    b->args_bytes = b->fp32 ? sizeof(StepArgs<float>) : sizeof(StepArgs<double>);
    cudaError_t e = cudaSetDevice(b->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking);
    b->stream = b->own_stream;
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
    for (int p = 0; p < 2 && e == cudaSuccess; ++p) e = cudaMalloc(&b->d_args[p], n * b->args_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_norm, n * sizeof(TileNorm));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_halo, n * sizeof(TileHalo));
    if (e == cudaSuccess) e = cudaMalloc(&b->d_error, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_error, 0, sizeof(int));
    if (e != cudaSuccess) {
        const int st = e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR;
        ts_b200_batch_destroy(b);
        return st;
    }
    *out = b;
    return TS_B200_OK;
}

void ts_b200_batch_destroy(ts_b200_batch *b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_batch_graph(b);
    for (void *p : b->d_args) cudaFree(p);
    cudaFree(b->d_tasks);
    cudaFree(b->d_task_norm);
    cudaFree(b->d_norm);
    cudaFree(b->d_halo);
    cudaFree(b->d_error);
    if (b->ev) cudaEventDestroy(b->ev);
    if (b->own_stream) cudaStreamDestroy(b->own_stream);
    delete b;
}

int ts_b200_batch_evolve(ts_b200_batch *b, int iterations) {
    if (!b || iterations < 0) return TS_B200_INVALID_ARGUMENT;
    if (iterations == 0) return TS_B200_OK;
    return b->fp32 ? evolve_t<float>(b, iterations) : evolve_t<double>(b, iterations);
}

int ts_b200_batch_synchronize(ts_b200_batch *b) {
    if (!b) return TS_B200_INVALID_ARGUMENT;
    int err = 0;
    TSBB_CHECK(b, cudaMemcpyAsync(&err, b->d_error, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    TSBB_CHECK(b, cudaStreamSynchronize(b->stream));
    if (err) return bfail(b, TS_B200_DEVICE_TIMEOUT, "a bounded wait in the batched step gave up");
    return TS_B200_OK;
}

int ts_b200_batch_set_stream(ts_b200_batch *b, void *stream) {
    if (!b) return TS_B200_INVALID_ARGUMENT;
    // work queued so far finishes before the batch moves to the other stream
    TSBB_CHECK(b, cudaStreamSynchronize(b->stream));
    b->stream = stream ? static_cast<cudaStream_t>(stream) : b->own_stream;
    return TS_B200_OK;
}

int ts_b200_batch_set_launch(ts_b200_batch *b, int segment_rows, int warps_per_block) {
    if (!b || segment_rows < 0) return TS_B200_INVALID_ARGUMENT;
    if (warps_per_block != 0 && warps_per_block != 1 && warps_per_block != 2 && warps_per_block != 4)
        return TS_B200_INVALID_ARGUMENT;
    if (segment_rows) b->shape.seg_rows = even_up(std::max(2, segment_rows));
    if (warps_per_block) b->shape.warps = warps_per_block;
    b->resident_blocks = 0;
    b->layout_valid = false;
    return TS_B200_OK;
}

int ts_b200_batch_autotune(ts_b200_batch *b, int trial_steps, int use_cache) {
    if (!b || trial_steps < 1) return TS_B200_INVALID_ARGUMENT;
    return b->fp32 ? autotune_t<float>(b, trial_steps, use_cache)
                   : autotune_t<double>(b, trial_steps, use_cache);
}

int ts_b200_batch_launch_info(ts_b200_batch *b, ts_b200_launch_shape *out) {
    if (!b || !out) return TS_B200_INVALID_ARGUMENT;
    if (!b->layout_valid) {
        const int s = b->fp32 ? build_layout<float>(b) : build_layout<double>(b);
        if (s) return s;
    }
    out->cells_per_lane = 2;
    out->segment_rows = b->shape.seg_rows;
    out->warps_per_block = b->shape.warps;
    out->ring_depth = b->ring;
    out->strips = b->sum_strips;
    out->segments = b->sum_segs;
    out->blocks = std::max(1, std::min(b->resident_blocks, div_up(b->n_tasks, b->shape.warps)));
    out->threads = 32 * b->shape.warps;
    out->smem_bytes = (int64_t)batch_smem(b, b->shape.warps);
    out->walk = b->walk;
    out->reserved = 0;
    return TS_B200_OK;
}

int ts_b200_batch_size(const ts_b200_batch *b) { return b ? (int)b->k.size() : 0; }

const char *ts_b200_batch_last_error(const ts_b200_batch *b) {
    return b ? b->err.c_str() : "null batch";
}

}  // extern "C"
