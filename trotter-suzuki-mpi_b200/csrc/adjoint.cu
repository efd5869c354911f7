// Adjoint engine (include/ts_b200.h, ts_b200_adjoint_*): forward evolution
// with the state kept for the reverse pass, and the reverse pass that maps
// dL/dpsi(T) to dL/dpsi(0) and dL/dV (adjoint_kernel.cuh).
//
// INVERSE mode (checkpoint_every == 0; linear real time): the forward pass
// keeps only psi(T); the reverse pass recovers psi_n from psi_{n+1} with the
// inverse step, fused with the adjoint step.
// CHECKPOINT mode: the forward pass stores psi every `every` steps; the
// reverse pass recomputes each segment's states from its checkpoint (forward
// step kernel into a segment buffer) and runs the adjoint steps over them in
// reverse.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <string>

#include "adjoint_kernel.cuh"
#include "handle.h"
#include "ts_b200.h"

using tsb::AdjArgs;
using tsb::AdjVariant;
using tsb::Cx;
using tsbh::div_up;
using tsbh::g_launches;

struct ts_b200_adjoint {
    ts_b200_kernel *k = nullptr;  // the tile: table, forward buffers, stream
    double dt = 0.0;
    int steps = 0, every = 0, n_ckpt = 0;
    int W = 0, H = 0, P = 0;
    void *lam[2] = {nullptr, nullptr};
    double *gv = nullptr;
    void *ckpt = nullptr;  // n_ckpt states
    void *seg = nullptr;   // every - 1 recomputed states
    int *error = nullptr;
    int seg_h = 32, warps = 2, ring = 4, blocks = 0;
    bool forward_done = false;
    void *state0 = nullptr;           // a segment's first state (graph-fixed address)
    cudaGraphExec_t inv_graph = nullptr;  // kInvGraphSteps inverse adjoint steps
    cudaGraphExec_t seg_graph = nullptr;  // one full checkpoint segment
    std::string err;
};

namespace {

constexpr int kAdjThreadsPerWarp = 32;
constexpr int kInvGraphSteps = 32;  // even: the buffers end where they started

int afail(ts_b200_adjoint *a, int status, const std::string &msg) {
    if (a) a->err = msg;
    return status;
}

int acuda(ts_b200_adjoint *a, cudaError_t e, const char *what) {
    if (a) a->err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR;
}

#define TSBA_CHECK(a, call)                                  \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return acuda(a, e_, #call);   \
    } while (0)

// exp(-i V dt) per cell (the reference tabulates it with std::exp(complex),
// src/solver.cpp:74-109); padding columns [W, P) get 0.
__global__ void table_from_potential_kernel(const double *V, int W, int H, int P, double dt,
                                            Cx<double> *tab) {
    const size_t n = (size_t)P * H;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / P), x = (int)(i % P);
        Cx<double> e{0.0, 0.0};
        if (x < W) {
            double s, c;
            sincos(V[(size_t)y * W + x] * dt, &s, &c);
            e.re = c;
            e.im = -s;
        }
        tab[i] = e;
    }
}

size_t state_bytes(const ts_b200_adjoint *a) { return (size_t)a->P * a->H * sizeof(Cx<double>); }

void *ckpt_at(ts_b200_adjoint *a, int j) {
    return static_cast<unsigned char *>(a->ckpt) + (size_t)j * state_bytes(a);
}

void *seg_at(ts_b200_adjoint *a, int j) {  // recomputed state j (1 .. every-1)
    return static_cast<unsigned char *>(a->seg) + (size_t)(j - 1) * state_bytes(a);
}

size_t adj_smem(const ts_b200_adjoint *a) {
    return (size_t)a->warps * (a->ring * AdjVariant<0, 0>::SLOT + 8 * a->ring);
}

template <class A>
cudaError_t launch_adj_variant(ts_b200_adjoint *a, const AdjArgs &args, int blocks, int *bps) {
    auto fn = tsb::adjoint_kernel<A>;
    const size_t smem = adj_smem(a);
    static int configured = -1;
    if ((int)smem > configured) {
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured = (int)smem;
    }
    if (bps) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            bps, fn, a->warps * kAdjThreadsPerWarp, smem);
        if (e != cudaSuccess) return e;
    }
    if (blocks == 0) return cudaSuccess;
    fn<<<blocks, a->warps * kAdjThreadsPerWarp, smem, a->k->stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_adj(ts_b200_adjoint *a, int mode, int phase, const AdjArgs &args, int blocks,
                       int *bps) {
    if (mode == 0) return launch_adj_variant<AdjVariant<0, 0>>(a, args, blocks, bps);
    if (phase == 2) return launch_adj_variant<AdjVariant<1, 2>>(a, args, blocks, bps);
    if (phase == 1) return launch_adj_variant<AdjVariant<1, 1>>(a, args, blocks, bps);
    return launch_adj_variant<AdjVariant<1, 0>>(a, args, blocks, bps);
}

AdjArgs adj_args(ts_b200_adjoint *a) {
    const ts_b200_desc &d = a->k->d;
    AdjArgs x{};
    x.pot = a->k->tab;
    x.gv = a->gv;
    x.error = a->error;
    x.W = a->W;
    x.H = a->H;
    x.P = a->P;
    x.n_strips = div_up(a->W, AdjVariant<0, 0>::WO);
    x.n_segs = div_up(a->H, a->seg_h);
    x.seg_h = a->seg_h;
    x.ring = a->ring;
    x.aH = d.a_h;
    x.bH = d.b_h;
    x.aV = d.a_v;
    x.bV = d.b_v;
    x.ca = d.coupling;
    x.caa = d.lhy_coupling;
    x.dt = a->dt;
    return x;
}

int adj_step(ts_b200_adjoint *a, int mode, const void *psi_in, void *psi_out, const void *lam_in,
             void *lam_out) {
    AdjArgs x = adj_args(a);
    x.psi_in = psi_in;
    x.psi_out = psi_out;
    x.lam_in = lam_in;
    x.lam_out = lam_out;
    const int tasks = x.n_strips * x.n_segs;
    const int blocks = std::max(1, std::min(a->blocks, div_up(tasks, a->warps)));
    cudaError_t e = launch_adj(a, mode, a->k->phase, x, blocks, nullptr);
    if (e != cudaSuccess) return acuda(a, e, "adjoint kernel launch");
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
}

int tile_status(ts_b200_adjoint *a, int s) {
    if (s) a->err = std::string("tile: ") + ts_b200_last_error(a->k);
    return s;
}

// Capture the launches `body` queues on the tile's stream into *exec.
template <class F>
int capture(ts_b200_adjoint *a, cudaGraphExec_t *exec, F body) {
    cudaStream_t st = a->k->stream;
    cudaGraph_t g = nullptr;
    TSBA_CHECK(a, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const uint64_t before = g_launches.load();
    const int s = body();
    cudaError_t e = cudaStreamEndCapture(st, &g);
    g_launches.store(before);  // counted when replayed
    if (s != TS_B200_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        if (s != TS_B200_OK) return s;
        return acuda(a, e, "adjoint graph capture");
    }
    e = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return acuda(a, e, "adjoint graph instantiate");
    return TS_B200_OK;
}

// Reverse pass of one checkpoint segment of `len` steps starting from the
// state in a->state0: recompute states 1 .. len-1, then len adjoint steps
// (lambda ping-pongs from lam[l]).
int segment_pass(ts_b200_adjoint *a, int len, int l) {
    int s = TS_B200_OK;
    for (int i = 1; i < len && s == TS_B200_OK; ++i)
        s = tile_status(a, tsbh::launch_step_buffers(a->k, i == 1 ? a->state0 : seg_at(a, i - 1),
                                                     seg_at(a, i)));
    for (int i = len - 1; i >= 0 && s == TS_B200_OK; --i) {
        const void *psi_n = i == 0 ? a->state0 : seg_at(a, i);
        s = adj_step(a, 1, psi_n, nullptr, a->lam[l], a->lam[l ^ 1]);
        l ^= 1;
    }
    return s;
}

}  // namespace

extern "C" {

int ts_b200_adjoint_create(const ts_b200_desc *d, double delta_t, int steps, int checkpoint_every,
                           ts_b200_adjoint **out) {
    if (!out) return TS_B200_INVALID_ARGUMENT;
    *out = nullptr;
    if (!d || steps < 1 || checkpoint_every < 0 || !(delta_t > 0.0)) return TS_B200_INVALID_ARGUMENT;
    if (d->imag_time || d->precision != TS_B200_FP64 || d->periodic_x || d->periodic_y ||
        (d->alpha_x != 0.0 && d->alpha_y != 0.0) || d->cylindrical)
        return TS_B200_UNSUPPORTED;  // real time, FP64, closed cartesian tile, no rotating frame
    if (checkpoint_every == 0 && (d->coupling != 0.0 || d->lhy_coupling != 0.0))
        return TS_B200_INVALID_ARGUMENT;  // inverse steps need the linear step
    ts_b200_adjoint *a = new (std::nothrow) ts_b200_adjoint();
    if (!a) return TS_B200_OUT_OF_MEMORY;
    int s = ts_b200_create(d, &a->k);
    if (s) {
        delete a;
        return s;
    }
    a->dt = delta_t;
    a->steps = steps;
    a->every = checkpoint_every;
    a->W = a->k->W;
    a->H = a->k->H;
    a->P = a->k->P;
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    const size_t sb = state_bytes(a);
    alloc(&a->lam[0], sb);
    alloc(&a->lam[1], sb);
    alloc(reinterpret_cast<void **>(&a->gv), (size_t)a->P * a->H * sizeof(double));
    alloc(reinterpret_cast<void **>(&a->error), sizeof(int));
    if (a->every > 0) {
        a->n_ckpt = (steps + a->every - 1) / a->every;  // states at 0, every, 2 every, ...
        alloc(&a->ckpt, sb * a->n_ckpt);
        if (a->every > 1) alloc(&a->seg, sb * (a->every - 1));
        alloc(&a->state0, sb);
    }
    if (e == cudaSuccess) {
        int bps = 0;
        AdjArgs x{};
        e = launch_adj(a, a->every > 0 ? 1 : 0, a->k->phase, x, 0, &bps);
        if (e == cudaSuccess && bps < 1) e = cudaErrorInvalidConfiguration;
        a->blocks = bps * a->k->num_sms;
        // one round of tasks over the resident warps (the tile is often small)
        const int strips = div_up(a->W, AdjVariant<0, 0>::WO);
        const int per_strip = std::max(1, a->blocks * a->warps / strips);
        a->seg_h = std::max(8, div_up(a->H, per_strip));
        a->seg_h += a->seg_h & 1;
    }
    if (e != cudaSuccess) {
        const int st = e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR;
        ts_b200_adjoint_destroy(a);
        return st;
    }
    *out = a;
    return TS_B200_OK;
}

void ts_b200_adjoint_destroy(ts_b200_adjoint *a) {
    if (!a) return;
    if (a->k) cudaStreamSynchronize(a->k->stream);
    cudaFree(a->lam[0]);
    cudaFree(a->lam[1]);
    cudaFree(a->gv);
    cudaFree(a->ckpt);
    cudaFree(a->seg);
    cudaFree(a->error);
    cudaFree(a->state0);
    if (a->inv_graph) cudaGraphExecDestroy(a->inv_graph);
    if (a->seg_graph) cudaGraphExecDestroy(a->seg_graph);
    ts_b200_destroy(a->k);
    delete a;
}

int ts_b200_adjoint_set_stream(ts_b200_adjoint *a, void *stream) {
    if (!a) return TS_B200_INVALID_ARGUMENT;
    return tile_status(a, ts_b200_set_stream(a->k, stream));
}

int ts_b200_adjoint_forward(ts_b200_adjoint *a, const double *potential, const void *psi0,
                            void *psi_t) {
    if (!a || !potential || !psi0) return TS_B200_INVALID_ARGUMENT;
    ts_b200_kernel *k = a->k;
    const size_t n = (size_t)a->P * a->H;
    const int grid = (int)std::min<size_t>((n + 255) / 256, 4096);
    table_from_potential_kernel<<<grid, 256, 0, k->stream>>>(
        potential, a->W, a->H, a->P, a->dt, static_cast<Cx<double> *>(k->tab));
    TSBA_CHECK(a, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    int s = tile_status(a, ts_b200_set_state_device(k, psi0, (size_t)a->W));
    if (s) return s;
    if (a->every > 0) {
        for (int j = 0; j < a->n_ckpt; ++j) {
            TSBA_CHECK(a, cudaMemcpyAsync(ckpt_at(a, j), k->psi[k->cur], state_bytes(a),
                                          cudaMemcpyDeviceToDevice, k->stream));
            const int len = std::min(a->every, a->steps - j * a->every);
            s = tile_status(a, ts_b200_evolve(k, len));
            if (s) return s;
        }
    } else {
        s = tile_status(a, ts_b200_evolve(k, a->steps));
        if (s) return s;
    }
    a->forward_done = true;
    if (psi_t) return tile_status(a, ts_b200_get_state_device(k, psi_t, (size_t)a->W));
    return TS_B200_OK;
}

int ts_b200_adjoint_backward(ts_b200_adjoint *a, const void *grad_psi_t, double *grad_potential,
                             void *grad_psi0) {
    if (!a || !grad_psi_t) return TS_B200_INVALID_ARGUMENT;
    if (!a->forward_done) return afail(a, TS_B200_INVALID_ARGUMENT, "backward before forward");
    ts_b200_kernel *k = a->k;
    const size_t cell = sizeof(Cx<double>);
    TSBA_CHECK(a, cudaMemcpy2DAsync(a->lam[0], a->P * cell, grad_psi_t, a->W * cell, a->W * cell,
                                    a->H, cudaMemcpyDeviceToDevice, k->stream));
    TSBA_CHECK(a, cudaMemsetAsync(a->gv, 0, (size_t)a->P * a->H * sizeof(double), k->stream));
    int l = 0;
    int s = TS_B200_OK;
    if (a->every == 0) {
        // ping-pong from (psi[cur], lam[0]); runs of kInvGraphSteps replayed
        int c = k->cur;  // psi(T)
        int n = a->steps;
        if (n >= kInvGraphSteps && c == 0) {
            if (!a->inv_graph) {
                s = capture(a, &a->inv_graph, [&] {
                    int st = TS_B200_OK, cc = 0, ll = 0;
                    for (int i = 0; i < kInvGraphSteps && st == TS_B200_OK; ++i) {
                        st = adj_step(a, 0, k->psi[cc], k->psi[cc ^ 1], a->lam[ll], a->lam[ll ^ 1]);
                        cc ^= 1;
                        ll ^= 1;
                    }
                    return st;
                });
                if (s) return s;
            }
            while (n >= kInvGraphSteps) {
                TSBA_CHECK(a, cudaGraphLaunch(a->inv_graph, k->stream));
                g_launches.fetch_add(kInvGraphSteps, std::memory_order_relaxed);
                n -= kInvGraphSteps;
            }
        }
        for (; n > 0 && s == TS_B200_OK; --n) {
            s = adj_step(a, 0, k->psi[c], k->psi[c ^ 1], a->lam[l], a->lam[l ^ 1]);
            c ^= 1;
            l ^= 1;
        }
        k->cur = c;  // the tile now holds the recomputed psi(0)
    } else {
        for (int j = a->n_ckpt - 1; j >= 0 && s == TS_B200_OK; --j) {
            const int len = std::min(a->every, a->steps - j * a->every);
            TSBA_CHECK(a, cudaMemcpyAsync(a->state0, ckpt_at(a, j), state_bytes(a),
                                          cudaMemcpyDeviceToDevice, k->stream));
            if (len == a->every && (len & 1) == 0) {
                // full segments of an even length leave lambda in lam[l]
                if (!a->seg_graph) {
                    s = capture(a, &a->seg_graph, [&] { return segment_pass(a, len, 0); });
                    if (s) return s;
                }
                if (l != 0) {  // the graph starts from lam[0]
                    TSBA_CHECK(a, cudaMemcpyAsync(a->lam[0], a->lam[1], state_bytes(a),
                                                  cudaMemcpyDeviceToDevice, k->stream));
                    l = 0;
                }
                TSBA_CHECK(a, cudaGraphLaunch(a->seg_graph, k->stream));
                g_launches.fetch_add(2 * len - 1, std::memory_order_relaxed);
            } else {
                s = segment_pass(a, len, l);
                if (len & 1) l ^= 1;
            }
        }
    }
    if (s) return s;
    a->forward_done = false;  // the reverse pass consumed the kept states
    if (grad_potential)
        TSBA_CHECK(a, cudaMemcpy2DAsync(grad_potential, a->W * sizeof(double), a->gv,
                                        a->P * sizeof(double), a->W * sizeof(double), a->H,
                                        cudaMemcpyDeviceToDevice, k->stream));
    if (grad_psi0)
        TSBA_CHECK(a, cudaMemcpy2DAsync(grad_psi0, a->W * cell, a->lam[l], a->P * cell, a->W * cell,
                                        a->H, cudaMemcpyDeviceToDevice, k->stream));
    return TS_B200_OK;
}

int ts_b200_adjoint_synchronize(ts_b200_adjoint *a) {
    if (!a) return TS_B200_INVALID_ARGUMENT;
    int err = 0;
    TSBA_CHECK(a, cudaMemcpyAsync(&err, a->error, sizeof(int), cudaMemcpyDeviceToHost, a->k->stream));
    TSBA_CHECK(a, cudaStreamSynchronize(a->k->stream));
    if (err) return afail(a, TS_B200_DEVICE_TIMEOUT, "a bounded wait in the adjoint step gave up");
    return tile_status(a, ts_b200_synchronize(a->k));
}

const char *ts_b200_adjoint_last_error(const ts_b200_adjoint *a) {
    return a ? a->err.c_str() : "null adjoint";
}

}  // extern "C"
