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
// IMAGINARY mode (imaginary time, checkpoints): as CHECKPOINT, with the
// renormalisation after every step: the forward pass takes norm0 = N(psi_0)
// (read back once per forward: it is a launch parameter of the step), each
// checkpoint keeps its tile with the pending factor c, the recomputation
// records every step's factor, and the reverse pass of each step also reads
// the next state for the transposed renormalisation.
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
    int *error = nullptr;
    int seg_h = 32, warps = 2, ring = 4, blocks = 0;
    bool forward_done = false;
    // imaginary time: factors c of the checkpoints and of a segment's states,
    // the projection coefficients mu (ping-pong), the running sum of the
    // inner products, block partials and ticket of the reductions; norm0
    bool imag = false;
    double *ckpt_c = nullptr, *mu = nullptr, *ksum = nullptr;
    double *partials = nullptr;
    unsigned int *ticket = nullptr;
    double norm0 = 0.0;
    // checkpointed reverse pass: up to two buffer sets, so that the states of
    // one segment are recomputed (on rstream) while the adjoint passes of the
    // next run (on the tile's stream); one set when memory is short
    int nsets = 1;
    void *seg[2] = {nullptr, nullptr};     // a segment's recomputed states
    void *state0[2] = {nullptr, nullptr};  // its first state (graph-fixed address)
    double *seg_c[2] = {nullptr, nullptr}; // imaginary time: their factors
    cudaStream_t rstream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_ready[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    cudaGraphExec_t inv_graph = nullptr;  // kInvGraphSteps inverse adjoint steps
    cudaGraphExec_t rec_graph[2] = {nullptr, nullptr};   // recomputation of a full segment
    cudaGraphExec_t pass_graph[2] = {nullptr, nullptr};  // the passes of a full segment
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

// exp(-V dt) per cell (imaginary time, real table, src/solver.cpp:74-109);
// padding columns [W, P) get 0.
__global__ void table_imag_from_potential_kernel(const double *V, int W, int H, int P, double dt,
                                                 double *tab) {
    const size_t n = (size_t)P * H;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / P), x = (int)(i % P);
        tab[i] = x < W ? exp(-V[(size_t)y * W + x] * dt) : 0.0;
    }
}

// Re<Lambda, c phi> over the tile (W x H, pitch P; Lambda of pitch W) with c
// the pending factor of phi: block sums, then the last block adds them in a
// fixed order and writes mu = scale * sum and the running sum (= the sum).
__global__ void adj_dot_kernel(const Cx<double> *lam, const Cx<double> *phi, const double *c,
                               int W, int H, int P, double scale, double *partials,
                               unsigned int *ticket, double *mu, double *ksum) {
    double s = 0.0;
    const size_t n = (size_t)W * H;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t y = i / W, x = i % W;
        const Cx<double> l = lam[i], f = phi[y * P + x];
        s = __fma_rn(l.re, f.re, __fma_rn(l.im, f.im, s));
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    __shared__ double sw[8];
    __shared__ unsigned int last;
    if ((threadIdx.x & 31) == 0) sw[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) b += sw[i];
        partials[blockIdx.x] = b;
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double tot = 0.0;
        for (int i = 0; i < (int)gridDim.x; ++i) tot += __ldcg(&partials[i]);
        tot *= *c;
        *mu = scale * tot;
        *ksum = tot;
        *ticket = 0u;
    }
}

// dL/dpsi_0 = Lambda_0 + (dA / norm0) (sum of Re<Lambda_k, psi_k>, k >= 1) psi_0:
// the gradient through norm0 = N(psi_0).  Output of pitch W.
__global__ void adj_grad_psi0_kernel(const Cx<double> *lam, const Cx<double> *psi0, int W, int H,
                                     int P, double scale, const double *ksum, Cx<double> *out) {
    const double m = scale * *ksum;
    const size_t n = (size_t)W * H;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t y = i / W, x = i % W;
        const Cx<double> l = lam[y * P + x], p = psi0[y * P + x];
        out[i] = Cx<double>{__fma_rn(m, p.re, l.re), __fma_rn(m, p.im, l.im)};
    }
}

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

// recomputed state j (1 .. every-1; .. every in imaginary time) of buffer set b
void *seg_at(ts_b200_adjoint *a, int b, int j) {
    return static_cast<unsigned char *>(a->seg[b]) + (size_t)(j - 1) * state_bytes(a);
}

void drop_segment_graphs(ts_b200_adjoint *a) {
    for (int b = 0; b < 2; ++b)
        for (cudaGraphExec_t *g : {&a->rec_graph[b], &a->pass_graph[b]}) {
            if (*g) cudaGraphExecDestroy(*g);
            *g = nullptr;
        }
}

size_t adj_smem(const ts_b200_adjoint *a) {
    const int slot = a->imag ? AdjVariant<2, 0>::SLOT : AdjVariant<0, 0>::SLOT;
    return (size_t)a->warps * (a->ring * slot + 8 * a->ring);
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
    // programmatic dependent launch (the kernel waits for its predecessor
    // before it reads anything)
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3((unsigned)(a->warps * kAdjThreadsPerWarp));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = a->k->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, fn, args);
}

cudaError_t launch_adj(ts_b200_adjoint *a, int mode, int phase, const AdjArgs &args, int blocks,
                       int *bps) {
    if (mode == 0) return launch_adj_variant<AdjVariant<0, 0>>(a, args, blocks, bps);
    if (mode == 2) {
        if (phase == 2) return launch_adj_variant<AdjVariant<2, 2>>(a, args, blocks, bps);
        if (phase == 1) return launch_adj_variant<AdjVariant<2, 1>>(a, args, blocks, bps);
        return launch_adj_variant<AdjVariant<2, 0>>(a, args, blocks, bps);
    }
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
    x.partials = a->partials;
    x.ticket = a->ticket;
    x.kappa_sum = a->ksum;
    x.mu_scale = a->imag ? a->k->d.delta_x * a->k->d.delta_y / a->norm0 : 0.0;
    return x;
}

// One reverse imaginary-time step: psi_k = c_k phi_k (phi_k at psi_k_in, c_k
// at *c_k), Lambda_{k+1} and psi_{k+1} (phi at psn, c at *c_n); mu_{k+1} in,
// mu_k out; `accumulate` adds Re<Lambda_k, psi_k> to the running sum.
int adj_step_imag(ts_b200_adjoint *a, const void *psi_k_in, const double *c_k, const void *psn,
                  const double *c_n, const void *lam_in, void *lam_out, const double *mu_in,
                  double *mu_out, bool accumulate) {
    AdjArgs x = adj_args(a);
    x.psi_in = psi_k_in;
    x.psi_out = nullptr;
    x.lam_in = lam_in;
    x.lam_out = lam_out;
    x.psn_in = psn;
    x.c_in = c_k;
    x.c_next = c_n;
    x.mu_next = mu_in;
    x.mu_out = mu_out;
    x.accumulate = accumulate ? 1 : 0;
    const int tasks = x.n_strips * x.n_segs;
    const int blocks = std::max(1, std::min(a->blocks, div_up(tasks, a->warps)));
    cudaError_t e = launch_adj(a, 2, a->k->phase, x, blocks, nullptr);
    if (e != cudaSuccess) return acuda(a, e, "adjoint kernel launch");
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return TS_B200_OK;
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

// Capture the launches `body` queues on stream `st` into *exec.
template <class F>
int capture(ts_b200_adjoint *a, cudaStream_t st, cudaGraphExec_t *exec, F body) {
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

// Recompute the states of a checkpoint segment of `len` steps from
// state0[b] into buffer set b, on the recomputation stream: states 1 .. len-1
// (real time) or 1 .. len with each step's renormalisation factor into
// seg_c[b][i] (imaginary time, from the factor seg_c[b][0]; the step writes
// it itself, so that the steps follow one another without a copy between).
int recompute(ts_b200_adjoint *a, int b, int len) {
    ts_b200_kernel *k = a->k;
    if (a->imag) {
        cudaError_t e = cudaMemcpyAsync(&k->scal->pending_inv, &a->seg_c[b][0], sizeof(double),
                                        cudaMemcpyDeviceToDevice, a->rstream);
        if (e != cudaSuccess) return acuda(a, e, "segment factor");
    }
    tsbh::StepPart part;
    part.pdl = true;
    part.stream = a->rstream;
    const int n = a->imag ? len : len - 1;
    int s = TS_B200_OK;
    for (int i = 1; i <= n && s == TS_B200_OK; ++i) {
        if (a->imag) part.inv_copy = &a->seg_c[b][i];
        s = tile_status(a, tsbh::launch_step_part(k, i == 1 ? a->state0[b] : seg_at(a, b, i - 1),
                                                  seg_at(a, b, i), part));
    }
    return s;
}

// The len reverse steps of a segment from its states in buffer set b
// (lambda ping-pongs from lam[l]; in imaginary time mu from mu[l], `first`
// the global index of the segment's first step: the step 0 pass adds nothing
// to the sum), on the tile's stream.
int passes(ts_b200_adjoint *a, int b, int len, int l, int first) {
    int s = TS_B200_OK;
    for (int i = len - 1; i >= 0 && s == TS_B200_OK; --i) {
        const void *psi_n = i == 0 ? a->state0[b] : seg_at(a, b, i);
        if (a->imag)
            s = adj_step_imag(a, psi_n, &a->seg_c[b][i], seg_at(a, b, i + 1), &a->seg_c[b][i + 1],
                              a->lam[l], a->lam[l ^ 1], &a->mu[l], &a->mu[l ^ 1], first + i > 0);
        else
            s = adj_step(a, 1, psi_n, nullptr, a->lam[l], a->lam[l ^ 1]);
        l ^= 1;
    }
    return s;
}

// The checkpointed reverse pass, segments from the last: segment j's states
// are recomputed into buffer set j % nsets on the recomputation stream while
// the passes of segment j + 1 run on the tile's stream (with two sets; one
// set orders them one after the other).  Full segments of an even length
// replay graphs (the recomputation of a set; its passes, which leave lambda
// and mu in [0]); returns the final lambda index in *l_out.
int checkpointed_reverse(ts_b200_adjoint *a, int *l_out) {
    ts_b200_kernel *k = a->k;
    cudaStream_t A = k->stream, B = a->rstream;
    int l = 0;
    int s = TS_B200_OK;
    TSBA_CHECK(a, cudaEventRecord(a->ev_start, A));
    TSBA_CHECK(a, cudaStreamWaitEvent(B, a->ev_start, 0));
    for (int b = 0; b < 2; ++b) TSBA_CHECK(a, cudaEventRecord(a->ev_free[b], A));
    for (int j = a->n_ckpt - 1; j >= 0 && s == TS_B200_OK; --j) {
        const int b = j % a->nsets;
        const int len = std::min(a->every, a->steps - j * a->every);
        const bool full = len == a->every && (len & 1) == 0;
        // recompute segment j once set b is free
        TSBA_CHECK(a, cudaStreamWaitEvent(B, a->ev_free[b], 0));
        TSBA_CHECK(a, cudaMemcpyAsync(a->state0[b], ckpt_at(a, j), state_bytes(a),
                                      cudaMemcpyDeviceToDevice, B));
        if (a->imag)
            TSBA_CHECK(a, cudaMemcpyAsync(&a->seg_c[b][0], &a->ckpt_c[j], sizeof(double),
                                          cudaMemcpyDeviceToDevice, B));
        if (full) {
            if (!a->rec_graph[b]) {
                s = capture(a, B, &a->rec_graph[b], [&] { return recompute(a, b, len); });
                if (s) return s;
            }
            TSBA_CHECK(a, cudaGraphLaunch(a->rec_graph[b], B));
            g_launches.fetch_add(a->imag ? len : len - 1, std::memory_order_relaxed);
        } else {
            s = recompute(a, b, len);
            if (s) return s;
        }
        TSBA_CHECK(a, cudaEventRecord(a->ev_ready[b], B));
        // its passes once its states are there
        TSBA_CHECK(a, cudaStreamWaitEvent(A, a->ev_ready[b], 0));
        if (full && (!a->imag || j > 0)) {
            if (!a->pass_graph[b]) {
                s = capture(a, A, &a->pass_graph[b], [&] { return passes(a, b, len, 0, 1); });
                if (s) return s;
            }
            if (l != 0) {  // the graph starts from lam[0] (and mu[0])
                TSBA_CHECK(a, cudaMemcpyAsync(a->lam[0], a->lam[1], state_bytes(a),
                                              cudaMemcpyDeviceToDevice, A));
                if (a->imag)
                    TSBA_CHECK(a, cudaMemcpyAsync(&a->mu[0], &a->mu[1], sizeof(double),
                                                  cudaMemcpyDeviceToDevice, A));
                l = 0;
            }
            TSBA_CHECK(a, cudaGraphLaunch(a->pass_graph[b], A));
            g_launches.fetch_add(len, std::memory_order_relaxed);
        } else {
            s = passes(a, b, len, l, j * a->every);
            if (len & 1) l ^= 1;
        }
        TSBA_CHECK(a, cudaEventRecord(a->ev_free[b], A));
    }
    *l_out = l;
    return s;
}

}  // namespace

extern "C" {

int ts_b200_adjoint_create(const ts_b200_desc *d, double delta_t, int steps, int checkpoint_every,
                           ts_b200_adjoint **out) {
    if (!out) return TS_B200_INVALID_ARGUMENT;
    *out = nullptr;
    if (!d || steps < 1 || checkpoint_every < 0 || !(delta_t > 0.0)) return TS_B200_INVALID_ARGUMENT;
    if (d->precision != TS_B200_FP64 || d->periodic_x || d->periodic_y ||
        (d->alpha_x != 0.0 && d->alpha_y != 0.0) || d->cylindrical)
        return TS_B200_UNSUPPORTED;  // FP64, closed cartesian tile, no rotating frame
    if (checkpoint_every == 0 && (d->coupling != 0.0 || d->lhy_coupling != 0.0 || d->imag_time))
        return TS_B200_INVALID_ARGUMENT;  // inverse steps need the linear unitary step
    ts_b200_adjoint *a = new (std::nothrow) ts_b200_adjoint();
    if (!a) return TS_B200_OUT_OF_MEMORY;
    ts_b200_desc dd = *d;
    if (dd.imag_time) dd.norm0 = 1.0;  // renormalised; the forward pass sets N(psi_0)
    int s = ts_b200_create(&dd, &a->k);
    if (s) {
        delete a;
        return s;
    }
    a->dt = delta_t;
    a->steps = steps;
    a->every = checkpoint_every;
    a->imag = d->imag_time != 0;
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
        // imaginary time also recomputes the next segment's first state; a
        // second buffer set (recomputation overlapping the passes) when it
        // takes under a quarter of the free device memory
        const int nseg = a->imag ? a->every : a->every - 1;
        size_t free_b = 0, total_b = 0;
        if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
        a->nsets = (a->n_ckpt > 1 && sb * (nseg + 1) * 4 <= free_b) ? 2 : 1;
        for (int b = 0; b < a->nsets; ++b) {
            if (nseg > 0) alloc(&a->seg[b], sb * nseg);
            alloc(&a->state0[b], sb);
            if (a->imag)
                alloc(reinterpret_cast<void **>(&a->seg_c[b]), sizeof(double) * (a->every + 1));
        }
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&a->rstream, cudaStreamNonBlocking);
        for (cudaEvent_t *ev : {&a->ev_start, &a->ev_ready[0], &a->ev_ready[1], &a->ev_free[0],
                                &a->ev_free[1]})
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    }
    if (a->imag) {
        alloc(reinterpret_cast<void **>(&a->ckpt_c), sizeof(double) * a->n_ckpt);
        alloc(reinterpret_cast<void **>(&a->mu), sizeof(double) * 2);
        alloc(reinterpret_cast<void **>(&a->ksum), sizeof(double));
        alloc(reinterpret_cast<void **>(&a->ticket), sizeof(unsigned int));
    }
    if (e == cudaSuccess) {
        int bps = 0;
        AdjArgs x{};
        e = launch_adj(a, a->imag ? 2 : (a->every > 0 ? 1 : 0), a->k->phase, x, 0, &bps);
        if (e == cudaSuccess && bps < 1) e = cudaErrorInvalidConfiguration;
        a->blocks = bps * a->k->num_sms;
        // one round of tasks over the resident warps (the tile is often
        // small), segments of at least 4 rows (6 in imaginary time): on
        // 512^2 the pass took 63.6 / 128.3 / 162.8 ms (linear, checkpointed,
        // imaginary time, 3000 steps) at 4 / 4 / 6 rows against 67.2 /
        // 144.3 / 169.0 at 8 and 89 / 195 / 235 at 2
        const int strips = div_up(a->W, AdjVariant<0, 0>::WO);
        const int per_strip = std::max(1, a->blocks * a->warps / strips);
        a->seg_h = std::max(a->imag ? 6 : 4, div_up(a->H, per_strip));
        a->seg_h += a->seg_h & 1;
        // block partials of the reductions (adjoint steps and the dot kernel)
        if (a->imag) alloc(reinterpret_cast<void **>(&a->partials),
                           sizeof(double) * std::max(a->blocks, 1024));
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
    if (a->rstream) cudaStreamSynchronize(a->rstream);
    cudaFree(a->lam[0]);
    cudaFree(a->lam[1]);
    cudaFree(a->gv);
    cudaFree(a->ckpt);
    for (int b = 0; b < 2; ++b) {
        cudaFree(a->seg[b]);
        cudaFree(a->state0[b]);
        cudaFree(a->seg_c[b]);
    }
    cudaFree(a->error);
    cudaFree(a->ckpt_c);
    cudaFree(a->mu);
    cudaFree(a->ksum);
    cudaFree(a->partials);
    cudaFree(a->ticket);
    if (a->inv_graph) cudaGraphExecDestroy(a->inv_graph);
    drop_segment_graphs(a);
    for (cudaEvent_t ev : {a->ev_start, a->ev_ready[0], a->ev_ready[1], a->ev_free[0], a->ev_free[1]})
        if (ev) cudaEventDestroy(ev);
    if (a->rstream) cudaStreamDestroy(a->rstream);
    ts_b200_destroy(a->k);
    delete a;
}

int ts_b200_adjoint_set_stream(ts_b200_adjoint *a, void *stream) {
    if (!a) return TS_B200_INVALID_ARGUMENT;
    return tile_status(a, ts_b200_set_stream(a->k, stream));
}

int ts_b200_adjoint_set_segments(ts_b200_adjoint *a, int adjoint_rows, int forward_rows) {
    if (!a || adjoint_rows < 0 || forward_rows < 0 || (adjoint_rows & 1) || adjoint_rows == 1)
        return TS_B200_INVALID_ARGUMENT;
    if (forward_rows > 0) {
        const int s = tile_status(a, ts_b200_set_launch(a->k, 0, forward_rows, 0, 0));
        if (s) return s;
        drop_segment_graphs(a);
    }
    if (adjoint_rows > 0 && adjoint_rows != a->seg_h) {
        a->seg_h = adjoint_rows;
        if (a->inv_graph) cudaGraphExecDestroy(a->inv_graph);
        a->inv_graph = nullptr;
        drop_segment_graphs(a);
    }
    return TS_B200_OK;
}

int ts_b200_adjoint_forward(ts_b200_adjoint *a, const double *potential, const void *psi0,
                            void *psi_t) {
    if (!a || !potential || !psi0) return TS_B200_INVALID_ARGUMENT;
    ts_b200_kernel *k = a->k;
    const size_t n = (size_t)a->P * a->H;
    const int grid = (int)std::min<size_t>((n + 255) / 256, 4096);
    if (a->imag)
        table_imag_from_potential_kernel<<<grid, 256, 0, k->stream>>>(
            potential, a->W, a->H, a->P, a->dt, static_cast<double *>(k->tab));
    else
        table_from_potential_kernel<<<grid, 256, 0, k->stream>>>(
            potential, a->W, a->H, a->P, a->dt, static_cast<Cx<double> *>(k->tab));
    TSBA_CHECK(a, cudaGetLastError());
    g_launches.fetch_add(1, std::memory_order_relaxed);
    int s = tile_status(a, ts_b200_set_state_device(k, psi0, (size_t)a->W));
    if (s) return s;
    if (a->imag) {
        // norm0 = N(psi_0), the norm every step restores (src/solver.cpp:155);
        // a launch parameter of the step, so the graphs follow a new value
        double n0 = 0.0;
        s = tile_status(a, ts_b200_squared_norm(k, &n0));
        if (s) return s;
        if (!(n0 > 0.0)) return afail(a, TS_B200_INVALID_ARGUMENT, "psi0 has zero norm");
        if (n0 != a->norm0) {
            a->norm0 = n0;
            s = tile_status(a, tsbh::set_norm0(k, n0));
            if (s) return s;
            drop_segment_graphs(a);
        }
    }
    if (a->every > 0) {
        for (int j = 0; j < a->n_ckpt; ++j) {
            TSBA_CHECK(a, cudaMemcpyAsync(ckpt_at(a, j), k->psi[k->cur], state_bytes(a),
                                          cudaMemcpyDeviceToDevice, k->stream));
            if (a->imag)
                TSBA_CHECK(a, cudaMemcpyAsync(&a->ckpt_c[j], &k->scal->pending_inv,
                                              sizeof(double), cudaMemcpyDeviceToDevice,
                                              k->stream));
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
    if (a->imag) {
        // mu_T and the running sum from Re<Lambda_T, psi_T>, psi_T = c_T phi_T
        TSBA_CHECK(a, cudaMemsetAsync(a->ticket, 0, sizeof(unsigned int), k->stream));
        const double scale = k->d.delta_x * k->d.delta_y / a->norm0;
        adj_dot_kernel<<<std::min(1024, div_up((long)a->W * a->H, 256)), 256, 0, k->stream>>>(
            static_cast<const Cx<double> *>(grad_psi_t), static_cast<const Cx<double> *>(k->psi[k->cur]),
            &k->scal->pending_inv, a->W, a->H, a->P, scale, a->partials, a->ticket, &a->mu[0],
            a->ksum);
        TSBA_CHECK(a, cudaGetLastError());
        g_launches.fetch_add(1, std::memory_order_relaxed);
        s = checkpointed_reverse(a, &l);
        if (s) return s;
        a->forward_done = false;
        if (grad_potential)
            TSBA_CHECK(a, cudaMemcpy2DAsync(grad_potential, a->W * sizeof(double), a->gv,
                                            a->P * sizeof(double), a->W * sizeof(double), a->H,
                                            cudaMemcpyDeviceToDevice, k->stream));
        if (grad_psi0) {
            // psi_0 is checkpoint 0 (factor 1: a state set from outside)
            adj_grad_psi0_kernel<<<std::min(1024, div_up((long)a->W * a->H, 256)), 256, 0,
                                   k->stream>>>(
                static_cast<const Cx<double> *>(a->lam[l]),
                static_cast<const Cx<double> *>(ckpt_at(a, 0)), a->W, a->H, a->P, scale, a->ksum,
                static_cast<Cx<double> *>(grad_psi0));
            TSBA_CHECK(a, cudaGetLastError());
            g_launches.fetch_add(1, std::memory_order_relaxed);
        }
        return TS_B200_OK;
    }
    if (a->every == 0) {
        // ping-pong from (psi[cur], lam[0]); runs of kInvGraphSteps replayed
        int c = k->cur;  // psi(T)
        int n = a->steps;
        if (n >= kInvGraphSteps && c == 0) {
            if (!a->inv_graph) {
                s = capture(a, k->stream, &a->inv_graph, [&] {
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
        s = checkpointed_reverse(a, &l);
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
