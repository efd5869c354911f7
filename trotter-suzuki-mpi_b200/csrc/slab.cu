// One lattice in slabs of rows, each slab a tile of its own: the halo
// exchange between the slabs and their joint imaginary-time norm, issued on
// the tiles' streams (no host synchronisation per step) and captured in CUDA
// graphs, the exchange overlapping each slab's interior.
//
// The reference splits a lattice over MPI ranks (Lattice2D on
// MPI_Cart_create, tile borders src/common.cpp:83-102) and, per step, runs
// the kernel on the halo bands first, starts the halo exchange, runs the
// interior and then waits for the exchange (src/solver.cpp:202-210,
// src/cpukernel.cpp:691-747); the imaginary-time renormalisation sums the
// squared norm over the ranks (src/cpukernel.cpp:537-546).  Here each step of
// a slab is two launches of the fused step over disjoint row windows:
//
//   edge stream (high priority):  edge bands -> send/receive halo rows ->
//                                 [x halo, norm sum, renormalisation]
//   interior stream:              interior rows
//
// The edge bands are the rows [0, inner_y0 + h) when there is an upper
// neighbour and [inner_y1 - h, rows) (start rounded down to even) when there
// is a lower one, h the halo rows; they contain the rows sent to the
// neighbours.  The interior reads no halo row (its walk reaches HY <= h rows
// past its window), so it does not wait for the exchange: the interior of
// step i waits only for the edge launch of step i - 1 (whose rows it reads,
// and whose input rows it overwrites), the edge launch of step i for the
// interior of step i - 1.  Both launches read the same input buffer and write
// disjoint rows of the other; the second to finish sums their norms in a
// fixed order (StepArgs::pair_norm).  In imaginary time, with a periodic x
// halo, or when the slab is too short to split, the next step also waits for
// the end of the previous one.
//
// Transports: NCCL between processes (one slab per rank; ncclSend/ncclRecv
// and a one-double ncclAllReduce on the edge stream; NCCL is loaded at run
// time, the copy the process already holds when there is one), or device
// copies between slabs of one process on one GPU (copy engines, ordered by
// events).  The messages are those of the reference's exchange: the last h
// inner rows go down into the lower neighbour's top halo, the first h inner
// rows up into the upper neighbour's bottom halo; on the last step of an
// evolve() call the messages across the lattice's periodic wrap are left out,
// as a single tile skips its periodic halo copy there (src/solver.cpp:203-
// 209), while those between slabs are kept, so that the slabs reproduce the
// single tile.
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <string>
#include <vector>

#include "handle.h"

namespace {

using tsbh::div_up;

// ------------------------------------------------------------------ NCCL
struct NcclApi {
    bool ok = false;
    std::string why;
    ncclResult_t (*GetUniqueId)(ncclUniqueId *) = nullptr;
    ncclResult_t (*CommInitRank)(ncclComm_t *, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
    ncclResult_t (*Send)(const void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*Recv)(void *, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
    ncclResult_t (*AllReduce)(const void *, void *, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                              cudaStream_t) = nullptr;
    ncclResult_t (*GroupStart)() = nullptr;
    ncclResult_t (*GroupEnd)() = nullptr;
    const char *(*GetErrorString)(ncclResult_t) = nullptr;
};

template <typename F>
bool bind(void *h, const char *name, F *fn) {
    *fn = reinterpret_cast<F>(dlsym(h, name));
    return *fn != nullptr;
}

NcclApi load_nccl() {
    NcclApi a;
    // the library already in the process (a framework's), else the loader's
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
        const char *e = dlerror();
        a.why = std::string("libnccl.so.2 not found: ") + (e ? e : "");
        return a;
    }
    bool ok = bind(h, "ncclGetUniqueId", &a.GetUniqueId) &&
              bind(h, "ncclCommInitRank", &a.CommInitRank) &&
              bind(h, "ncclCommDestroy", &a.CommDestroy) && bind(h, "ncclSend", &a.Send) &&
              bind(h, "ncclRecv", &a.Recv) && bind(h, "ncclAllReduce", &a.AllReduce) &&
              bind(h, "ncclGroupStart", &a.GroupStart) && bind(h, "ncclGroupEnd", &a.GroupEnd) &&
              bind(h, "ncclGetErrorString", &a.GetErrorString);
    if (!ok) a.why = "libnccl.so.2 lacks a symbol";
    a.ok = ok;
    return a;
}

NcclApi &nccl() {
    static NcclApi api = load_nccl();
    return api;
}

// ------------------------------------------------------------ device work
// Imaginary time, slabs of one process: the lattice's squared norm as the
// slabs' norms summed in slab order, and each slab's pending factor from it.
__global__ void slab_norm_kernel(tsb::Scalars *const *scal, const double *norm0, int n) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double tot = 0.0;
    for (int i = 0; i < n; ++i) tot += scal[i]->last_norm;
    for (int i = 0; i < n; ++i)
        if (scal[i]->renorm) scal[i]->pending_inv = 1.0 / sqrt(tot / norm0[i]);
}

// The same from a norm already summed over the ranks.
__global__ void slab_renorm_kernel(tsb::Scalars *scal, const double *total, double norm0) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && scal->renorm)
        scal->pending_inv = 1.0 / sqrt(*total / norm0);
}

}  // namespace

// ------------------------------------------------------------------ group
struct SlabTile {
    ts_b200_kernel *k = nullptr;
    ts_b200_slab_link link{-1, -1, 0, 0, 0, 0};
    int h = 0;                // halo rows
    bool split = false;       // edge bands and interior as two launches
    bool chained = false;     // the interior waits for the end of the previous step
    tsbh::StepPart edge, inner, whole;
    cudaStream_t se = nullptr, si = nullptr;
    cudaEvent_t ev_edge = nullptr, ev_int = nullptr, ev_step = nullptr, ev_aux = nullptr;
    double *scratch = nullptr;  // partials (edge | interior | whole), pair norms, ranks' total
    size_t scratch_n = 0;
    unsigned int *tickets = nullptr;  // edge, interior, whole, pair
    double *pair_norm = nullptr, *total = nullptr;
};

struct ts_b200_slabs {
    std::vector<SlabTile> t;
    bool use_nccl = false;
    ncclComm_t comm = nullptr;
    int rank = 0, nranks = 1;
    bool split_on = true;
    bool imag = false;
    int device = 0;
    cudaStream_t origin = nullptr;  // tile 0's stream: the group's work starts and ends here
    cudaEvent_t ev_fork = nullptr;
    tsb::Scalars **d_scal = nullptr;  // slabs of one process: their scalars and norm0
    double *d_norm0 = nullptr;
    std::vector<double> norm0;        // the values in d_norm0
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    std::vector<long long> signature;
    int launches_per_step = 0;
    std::string err;
};

namespace {

int sfail(ts_b200_slabs *s, int status, const std::string &msg) {
    if (s) s->err = msg;
    return status;
}

int scuda(ts_b200_slabs *s, cudaError_t e, const char *what) {
    return sfail(s, e == cudaErrorMemoryAllocation ? TS_B200_OUT_OF_MEMORY : TS_B200_CUDA_ERROR,
                 std::string(what) + ": " + cudaGetErrorString(e));
}

int snccl(ts_b200_slabs *s, ncclResult_t r, const char *what) {
    return sfail(s, TS_B200_CUDA_ERROR,
                 std::string(what) + ": " + (nccl().GetErrorString ? nccl().GetErrorString(r) : "?"));
}

#define TSS_CHECK(s, call)                                     \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return scuda(s, e_, #call);     \
    } while (0)

#define TSS_NCCL(s, call)                                      \
    do {                                                       \
        ncclResult_t r_ = (call);                              \
        if (r_ != ncclSuccess) return snccl(s, r_, #call);     \
    } while (0)

#define TSS_OK(call)             \
    do {                         \
        const int st_ = (call);  \
        if (st_) return st_;     \
    } while (0)

size_t cell_bytes(const ts_b200_kernel *k) { return k->fp32 ? 8 : 16; }

// Rows of the message span: h rows of the tile at `row`, pitch included.
size_t span_bytes(const SlabTile &x) { return (size_t)x.h * x.k->P * cell_bytes(x.k); }
unsigned char *row_ptr(const SlabTile &x, void *buf, int row) {
    return static_cast<unsigned char *>(buf) + (size_t)row * x.k->P * cell_bytes(x.k);
}

// The tile's part of a step and the group's launch counts.  Returns nonzero
// when a tile does not satisfy the slab layout.
int plan_tile(ts_b200_slabs *s, SlabTile &x) {
    ts_b200_kernel *k = x.k;
    const ts_b200_desc &d = k->d;
    int32_t w[8];
    const int st = ts_b200_slab_windows(k->H, d.inner_y0, d.inner_y1, d.halo_y,
                                        tsbh::step_reach_rows(k), x.link.up >= 0,
                                        x.link.down >= 0, w);
    if (st) return sfail(s, st, "slab layout: the tile's rows do not fit its halo and neighbours");
    x.h = d.halo_y;
    x.split = s->split_on && w[6] != 0;
    x.chained = k->imag || d.periodic_x;
    x.edge = tsbh::StepPart{};
    x.inner = tsbh::StepPart{};
    x.whole = tsbh::StepPart{};
    if (x.split) {
        x.edge.a0 = w[0];
        x.edge.a1 = w[1];
        x.edge.b0 = w[2];
        x.edge.b1 = w[3];
        x.inner.a0 = w[4];
        x.inner.a1 = w[5];
    }
    TSS_OK(tsbh::configure_step(k));
    const int nb_e = x.split ? tsbh::part_blocks(k, x.edge) : 0;
    const int nb_i = x.split ? tsbh::part_blocks(k, x.inner) : 0;
    const int nb_w = tsbh::part_blocks(k, x.whole);
    const size_t need = (size_t)nb_e + nb_i + nb_w + 3;
    if (need > x.scratch_n) {
        if (x.scratch) cudaFree(x.scratch);
        x.scratch = nullptr;
        x.scratch_n = 0;
        TSS_CHECK(s, cudaMalloc(&x.scratch, need * sizeof(double)));
        x.scratch_n = need;
    }
    if (!x.tickets) {
        TSS_CHECK(s, cudaMalloc(&x.tickets, 4 * sizeof(unsigned int)));
        TSS_CHECK(s, cudaMemset(x.tickets, 0, 4 * sizeof(unsigned int)));
    }
    x.edge.partials = x.scratch;
    x.inner.partials = x.scratch + nb_e;
    x.whole.partials = x.scratch + nb_e + nb_i;
    x.pair_norm = x.scratch + nb_e + nb_i + nb_w;
    x.total = x.pair_norm + 2;
    x.edge.ticket = x.tickets + 0;
    x.inner.ticket = x.tickets + 1;
    x.whole.ticket = x.tickets + 2;
    x.edge.stream = x.se;
    x.inner.stream = x.si;
    x.whole.stream = x.se;
    if (x.split) {
        x.edge.pair_norm = x.inner.pair_norm = x.pair_norm;
        x.edge.pair_ticket = x.inner.pair_ticket = x.tickets + 3;
        x.edge.pair_slot = 0;
        x.inner.pair_slot = 1;
    }
    return TS_B200_OK;
}

int plan(ts_b200_slabs *s) {
    std::vector<long long> sig;
    s->launches_per_step = 0;
    for (SlabTile &x : s->t) {
        TSS_OK(plan_tile(s, x));
        const ts_b200_kernel *k = x.k;
        sig.insert(sig.end(), {(long long)k->C, k->seg_h, k->warps, k->ring, k->walk2,
                               k->resident_blocks, (long long)(k->d.norm0 * 1e6), x.split,
                               (long long)(uintptr_t)k->psi[0], (long long)(uintptr_t)k->psi[1],
                               (long long)(uintptr_t)x.scratch});
        s->launches_per_step += (x.split ? 2 : 1) + (k->d.periodic_x ? 1 : 0);
    }
    if (s->imag) s->launches_per_step += 1;
    if (s->d_norm0) {
        std::vector<double> n0;
        for (const SlabTile &x : s->t) n0.push_back(x.k->d.norm0);
        if (n0 != s->norm0) {
            TSS_CHECK(s, cudaMemcpyAsync(s->d_norm0, n0.data(), n0.size() * sizeof(double),
                                         cudaMemcpyHostToDevice, s->origin));
            TSS_CHECK(s, cudaStreamSynchronize(s->origin));
            s->norm0 = n0;
        }
    }
    if (sig != s->signature) {
        if (s->graph) cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        s->graph_steps = 0;
        s->signature = sig;
    }
    return TS_B200_OK;
}

// Messages of a tile for one step: the spans to send to and receive from
// its neighbours, in the order both ends post them (per peer, the reference's
// tags 1 then 2).
struct Msg {
    int peer;  // tile index (local) or rank (NCCL)
    int row;   // first row of the span in the tile
    int tag;   // 1: rows moving down the lattice, 2: moving up
    bool send;
};

void messages(const SlabTile &x, bool final, std::vector<Msg> &out) {
    out.clear();
    int32_t m[16];
    const int n = ts_b200_slab_messages(x.k->d.inner_y0, x.k->d.inner_y1, x.h, &x.link,
                                        final ? 1 : 0, m);
    for (int i = 0; i < n; ++i) out.push_back({m[4 * i], m[4 * i + 1], m[4 * i + 2], m[4 * i + 3] != 0});
}

// The group's streams join the origin stream (start of a sequence, also
// inside a capture) and leave it (end).
int fork_from_origin(ts_b200_slabs *s) {
    TSS_CHECK(s, cudaEventRecord(s->ev_fork, s->origin));
    for (SlabTile &x : s->t) {
        TSS_CHECK(s, cudaStreamWaitEvent(x.se, s->ev_fork, 0));
        TSS_CHECK(s, cudaStreamWaitEvent(x.si, s->ev_fork, 0));
        // the first step's waits find these records
        TSS_CHECK(s, cudaEventRecord(x.ev_int, x.si));
        TSS_CHECK(s, cudaEventRecord(x.ev_edge, x.se));
        TSS_CHECK(s, cudaEventRecord(x.ev_step, x.se));
    }
    return TS_B200_OK;
}

int join_to_origin(ts_b200_slabs *s) {
    for (SlabTile &x : s->t) {
        TSS_CHECK(s, cudaEventRecord(x.ev_aux, x.si));
        TSS_CHECK(s, cudaStreamWaitEvent(s->origin, x.ev_aux, 0));
        TSS_CHECK(s, cudaEventRecord(x.ev_aux, x.se));
        TSS_CHECK(s, cudaStreamWaitEvent(s->origin, x.ev_aux, 0));
    }
    return TS_B200_OK;
}

int issue_exchange(ts_b200_slabs *s, bool final) {
    std::vector<Msg> ms;
    if (s->use_nccl) {
        SlabTile &x = s->t[0];
        messages(x, final, ms);
        if (ms.empty()) return TS_B200_OK;
        void *out = x.k->psi[x.k->cur];
        const size_t n = span_bytes(x);
        TSS_NCCL(s, nccl().GroupStart());
        for (const Msg &m : ms) {
            if (m.send) {
                ncclResult_t r = nccl().Send(row_ptr(x, out, m.row), n, ncclUint8, m.peer, s->comm, x.se);
                if (r != ncclSuccess) {
                    (void)nccl().GroupEnd();
                    return snccl(s, r, "ncclSend");
                }
            } else {
                ncclResult_t r = nccl().Recv(row_ptr(x, out, m.row), n, ncclUint8, m.peer, s->comm, x.se);
                if (r != ncclSuccess) {
                    (void)nccl().GroupEnd();
                    return snccl(s, r, "ncclRecv");
                }
            }
        }
        TSS_NCCL(s, nccl().GroupEnd());
        return TS_B200_OK;
    }
    // one process: each slab pulls its halo rows from its neighbours' output
    // once their edge launches are done
    for (SlabTile &x : s->t) {
        messages(x, final, ms);
        for (const Msg &m : ms) {
            if (m.send) continue;
            SlabTile &y = s->t[m.peer];
            // the rows the neighbour sends: its last h inner rows into our top
            // halo (tag 1), its first h inner rows into our bottom halo (tag 2)
            const int src_row = (m.tag == 1) ? y.k->d.inner_y1 - y.h : y.k->d.inner_y0;
            if (&y != &x) TSS_CHECK(s, cudaStreamWaitEvent(x.se, y.ev_edge, 0));
            TSS_CHECK(s, cudaMemcpyAsync(row_ptr(x, x.k->psi[x.k->cur], m.row),
                                         row_ptr(y, y.k->psi[y.k->cur], src_row), span_bytes(x),
                                         cudaMemcpyDeviceToDevice, x.se));
        }
    }
    return TS_B200_OK;
}

// One step of every slab of the group (see the stream plan at the top).
int issue_step(ts_b200_slabs *s, bool final) {
    // compute: edge bands, then the interior
    for (SlabTile &x : s->t) {
        ts_b200_kernel *k = x.k;
        const void *in = k->psi[k->cur];
        void *out = k->psi[1 - k->cur];
        if (x.split) {
            TSS_CHECK(s, cudaStreamWaitEvent(x.se, x.ev_int, 0));
            TSS_CHECK(s, cudaStreamWaitEvent(x.si, x.chained ? x.ev_step : x.ev_edge, 0));
            TSS_OK(tsbh::launch_step_part(k, in, out, x.edge));
            TSS_CHECK(s, cudaEventRecord(x.ev_edge, x.se));
            TSS_OK(tsbh::launch_step_part(k, in, out, x.inner));
            TSS_CHECK(s, cudaEventRecord(x.ev_int, x.si));
        } else {
            TSS_OK(tsbh::launch_step_part(k, in, out, x.whole));
            TSS_CHECK(s, cudaEventRecord(x.ev_edge, x.se));
        }
        k->cur = 1 - k->cur;
    }
    TSS_OK(issue_exchange(s, final));
    // what needs the whole step: the x halo (not after the last step of a
    // call, as a single tile skips its halo copy there) and the norm
    for (SlabTile &x : s->t) {
        if (x.split && x.chained) TSS_CHECK(s, cudaStreamWaitEvent(x.se, x.ev_int, 0));
        if (x.k->d.periodic_x && !final && x.link.xhalo_row1 > x.link.xhalo_row0)
            TSS_OK(tsbh::launch_halo_on(x.k, x.se, x.link.xhalo_row0, x.link.xhalo_row1));
    }
    if (s->imag) {
        if (s->use_nccl) {
            SlabTile &x = s->t[0];
            TSS_NCCL(s, nccl().AllReduce(&x.k->scal->last_norm, x.total, 1, ncclFloat64, ncclSum,
                                         s->comm, x.se));
            slab_renorm_kernel<<<1, 32, 0, x.se>>>(x.k->scal, x.total, x.k->d.norm0);
            TSS_CHECK(s, cudaGetLastError());
            tsbh::g_launches.fetch_add(1, std::memory_order_relaxed);
        } else {
            SlabTile &x0 = s->t[0];
            for (size_t i = 1; i < s->t.size(); ++i) {
                TSS_CHECK(s, cudaEventRecord(s->t[i].ev_aux, s->t[i].se));
                TSS_CHECK(s, cudaStreamWaitEvent(x0.se, s->t[i].ev_aux, 0));
            }
            slab_norm_kernel<<<1, 32, 0, x0.se>>>(s->d_scal, s->d_norm0, (int)s->t.size());
            TSS_CHECK(s, cudaGetLastError());
            tsbh::g_launches.fetch_add(1, std::memory_order_relaxed);
            TSS_CHECK(s, cudaEventRecord(x0.ev_aux, x0.se));
            for (size_t i = 1; i < s->t.size(); ++i)
                TSS_CHECK(s, cudaStreamWaitEvent(s->t[i].se, x0.ev_aux, 0));
        }
    }
    for (SlabTile &x : s->t) {
        TSS_CHECK(s, cudaEventRecord(x.ev_step, x.se));
        if (!x.split) {
            // the next step's edge launch orders after this one by the stream;
            // keep the interior stream's record current for the join
            TSS_CHECK(s, cudaEventRecord(x.ev_int, x.se));
        }
    }
    return TS_B200_OK;
}

int issue_steps(ts_b200_slabs *s, int n, bool last_final) {
    TSS_OK(fork_from_origin(s));
    for (int i = 0; i < n; ++i) TSS_OK(issue_step(s, last_final && i == n - 1));
    return join_to_origin(s);
}

int make_streams(ts_b200_slabs *s, SlabTile &x) {
    int least = 0, greatest = 0;
    TSS_CHECK(s, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    TSS_CHECK(s, cudaStreamCreateWithPriority(&x.se, cudaStreamNonBlocking, greatest));
    TSS_CHECK(s, cudaStreamCreateWithPriority(&x.si, cudaStreamNonBlocking, least));
    for (cudaEvent_t *e : {&x.ev_edge, &x.ev_int, &x.ev_step, &x.ev_aux})
        TSS_CHECK(s, cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return TS_B200_OK;
}

int check_tile(ts_b200_slabs *s, const ts_b200_kernel *k) {
    if (!k) return sfail(s, TS_B200_INVALID_ARGUMENT, "null tile");
    if (k->pair_mode) return sfail(s, TS_B200_UNSUPPORTED, "slabs of a two-component pair");
    if (k->cyl) return sfail(s, TS_B200_UNSUPPORTED, "slabs of a cylindrical lattice");
    if (k->d.periodic_y)
        return sfail(s, TS_B200_INVALID_ARGUMENT,
                     "a slab tile is closed in y: its neighbours supply the halo rows");
    return TS_B200_OK;
}

int finish_create(ts_b200_slabs *s) {
    s->imag = s->t[0].k->imag;
    s->device = s->t[0].k->device;
    for (SlabTile &x : s->t) {
        if (x.k->imag != s->imag || x.k->fp32 != s->t[0].k->fp32 || x.k->W != s->t[0].k->W ||
            x.k->P != s->t[0].k->P || x.k->device != s->device)
            return sfail(s, TS_B200_INVALID_ARGUMENT,
                         "slabs differ in time mode, precision, width or device");
        TSS_OK(make_streams(s, x));
    }
    TSS_CHECK(s, cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
    s->origin = s->t[0].k->stream;
    if (s->imag && !s->use_nccl) {
        const size_t n = s->t.size();
        std::vector<tsb::Scalars *> sc(n);
        std::vector<double> n0(n);
        for (size_t i = 0; i < n; ++i) {
            sc[i] = s->t[i].k->scal;
            n0[i] = s->t[i].k->d.norm0;
        }
        TSS_CHECK(s, cudaMalloc(&s->d_scal, n * sizeof(tsb::Scalars *)));
        TSS_CHECK(s, cudaMalloc(&s->d_norm0, n * sizeof(double)));
        TSS_CHECK(s, cudaMemcpy(s->d_scal, sc.data(), n * sizeof(tsb::Scalars *), cudaMemcpyHostToDevice));
        TSS_CHECK(s, cudaMemcpy(s->d_norm0, n0.data(), n * sizeof(double), cudaMemcpyHostToDevice));
        s->norm0 = n0;
    }
    return TS_B200_OK;
}

void destroy(ts_b200_slabs *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (SlabTile &x : s->t) {
        if (x.se) cudaStreamSynchronize(x.se);
        if (x.si) cudaStreamSynchronize(x.si);
        for (cudaEvent_t e : {x.ev_edge, x.ev_int, x.ev_step, x.ev_aux})
            if (e) cudaEventDestroy(e);
        if (x.se) cudaStreamDestroy(x.se);
        if (x.si) cudaStreamDestroy(x.si);
        cudaFree(x.scratch);
        cudaFree(x.tickets);
    }
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    cudaFree(s->d_scal);
    cudaFree(s->d_norm0);
    if (s->comm) nccl().CommDestroy(s->comm);
    delete s;
}

}  // namespace

// ================================================================== C ABI
extern "C" {

int ts_b200_slab_windows(int rows, int inner_y0, int inner_y1, int halo, int reach, int has_up,
                         int has_down, int32_t out[8]) {
    if (!out || rows < 1 || halo < 0 || reach < 0 || inner_y0 < 0 || inner_y1 > rows ||
        inner_y1 <= inner_y0)
        return TS_B200_INVALID_ARGUMENT;
    for (int i = 0; i < 8; ++i) out[i] = 0;
    // neighbours supply exactly `halo` rows on their side; the tile has at
    // least `halo` inner rows to send; the halo covers the walk's reach
    if ((has_up && inner_y0 != halo) || (!has_up && inner_y0 != 0) ||
        (has_down && rows - inner_y1 != halo) || (!has_down && inner_y1 != rows))
        return TS_B200_INVALID_ARGUMENT;
    if ((has_up || has_down) && (inner_y1 - inner_y0 < halo || halo < reach || (halo & 1)))
        return TS_B200_INVALID_ARGUMENT;
    const int top_end = has_up ? inner_y0 + halo : 0;
    const int bot_start = has_down ? ((inner_y1 - halo) & ~1) : rows;
    // windows: edge [a0, a1) and [b0, b1) (the non-empty one first), interior
    // [i0, i1); split when there is a neighbour and an interior of at least
    // two walks' reach
    const bool split = (has_up || has_down) && bot_start - top_end >= 2 * reach + 2;
    out[6] = split ? 1 : 0;
    if (!split) return TS_B200_OK;
    if (has_up) {
        out[0] = 0;
        out[1] = top_end;
        if (has_down) {
            out[2] = bot_start;
            out[3] = rows;
        }
    } else {
        out[0] = bot_start;
        out[1] = rows;
    }
    out[4] = top_end;
    out[5] = bot_start;
    return TS_B200_OK;
}

int ts_b200_slab_messages(int inner_y0, int inner_y1, int halo, const ts_b200_slab_link *link,
                          int final, int32_t out[16]) {
    if (!link || !out) return -TS_B200_INVALID_ARGUMENT;
    const bool down_ok = link->down >= 0 && !(final && link->down_wraps);
    const bool up_ok = link->up >= 0 && !(final && link->up_wraps);
    int n = 0;
    auto add = [&](int peer, int row, int tag, int send) {
        out[4 * n] = peer;
        out[4 * n + 1] = row;
        out[4 * n + 2] = tag;
        out[4 * n + 3] = send;
        ++n;
    };
    // sends: the last h inner rows down into the lower neighbour's top halo
    // (tag 1), the first h inner rows up into the upper one's bottom halo
    // (tag 2); receives in the same tag order from each side
    if (down_ok) add(link->down, inner_y1 - halo, 1, 1);
    if (up_ok) add(link->up, inner_y0, 2, 1);
    if (up_ok) add(link->up, 0, 1, 0);
    if (down_ok) add(link->down, inner_y1, 2, 0);
    return n;
}

int ts_b200_nccl_unique_id(void *id, size_t bytes) {
    if (!id || bytes < sizeof(ncclUniqueId)) return TS_B200_INVALID_ARGUMENT;
    if (!nccl().ok) return TS_B200_UNSUPPORTED;
    ncclUniqueId u;
    if (nccl().GetUniqueId(&u) != ncclSuccess) return TS_B200_CUDA_ERROR;
    memcpy(id, &u, sizeof(u));
    return TS_B200_OK;
}

int ts_b200_slabs_create_local(ts_b200_slabs **out, ts_b200_kernel *const *tiles,
                               const ts_b200_slab_link *links, int n_tiles) {
    if (!out || !tiles || !links || n_tiles < 1) return TS_B200_INVALID_ARGUMENT;
    *out = nullptr;
    ts_b200_slabs *s = new ts_b200_slabs();
    int st = TS_B200_OK;
    for (int i = 0; i < n_tiles && !st; ++i) {
        st = check_tile(s, tiles[i]);
        const ts_b200_slab_link &l = links[i];
        if (!st && (l.up >= n_tiles || l.down >= n_tiles || l.up < -1 || l.down < -1))
            st = sfail(s, TS_B200_INVALID_ARGUMENT, "slab link to a tile outside the group");
        if (!st && ((l.up >= 0 && links[l.up].down != i) || (l.down >= 0 && links[l.down].up != i)))
            st = sfail(s, TS_B200_INVALID_ARGUMENT, "slab links are not mutual");
        if (!st) {
            SlabTile x;
            x.k = tiles[i];
            x.link = l;
            s->t.push_back(x);
        }
    }
    if (!st) {
        cudaSetDevice(tiles[0]->device);
        st = finish_create(s);
    }
    if (st) {
        // the reason stays readable on the first tile (ts_b200_last_error)
        tiles[0]->err = s->err;
        destroy(s);
        return st;
    }
    *out = s;
    return TS_B200_OK;
}

int ts_b200_slabs_create_nccl(ts_b200_slabs **out, ts_b200_kernel *tile,
                              const ts_b200_slab_link *link, const void *nccl_id, size_t id_bytes,
                              int nranks, int rank) {
    if (!out || !tile || !link || !nccl_id || id_bytes < sizeof(ncclUniqueId) || nranks < 1 ||
        rank < 0 || rank >= nranks || link->up >= nranks || link->down >= nranks)
        return TS_B200_INVALID_ARGUMENT;
    *out = nullptr;
    if (!nccl().ok) {
        tile->err = nccl().why;
        return TS_B200_UNSUPPORTED;
    }
    ts_b200_slabs *s = new ts_b200_slabs();
    int st = check_tile(s, tile);
    if (!st) {
        SlabTile x;
        x.k = tile;
        x.link = *link;
        s->t.push_back(x);
        s->use_nccl = true;
        s->rank = rank;
        s->nranks = nranks;
        cudaSetDevice(tile->device);
        ncclUniqueId u;
        memcpy(&u, nccl_id, sizeof(u));
        ncclResult_t r = nccl().CommInitRank(&s->comm, nranks, u, rank);
        if (r != ncclSuccess) {
            s->comm = nullptr;
            st = snccl(s, r, "ncclCommInitRank");
        }
    }
    if (!st) st = finish_create(s);
    if (st) {
        tile->err = s->err;
        destroy(s);
        return st;
    }
    *out = s;
    return TS_B200_OK;
}

int ts_b200_slabs_set_split(ts_b200_slabs *s, int on) {
    if (!s || (on != 0 && on != 1)) return TS_B200_INVALID_ARGUMENT;
    s->split_on = on != 0;
    return TS_B200_OK;
}

int ts_b200_slabs_plan(ts_b200_slabs *s, int tile, int32_t out[8]) {
    if (!s || !out || tile < 0 || tile >= (int)s->t.size()) return TS_B200_INVALID_ARGUMENT;
    cudaSetDevice(s->device);
    TSS_OK(plan(s));
    const SlabTile &x = s->t[tile];
    const tsbh::StepPart &e = x.edge, &i = x.inner;
    const int32_t v[8] = {e.a0, e.a1, e.b0, e.b1, i.a0, i.a1, x.split ? 1 : 0, s->launches_per_step};
    for (int j = 0; j < 8; ++j) out[j] = v[j];
    return TS_B200_OK;
}

int ts_b200_slabs_evolve(ts_b200_slabs *s, int iterations) {
    if (!s || iterations < 0) return TS_B200_INVALID_ARGUMENT;
    if (iterations == 0) return TS_B200_OK;
    cudaSetDevice(s->device);
    TSS_OK(plan(s));
    // work queued on the other tiles' streams comes first
    for (size_t i = 1; i < s->t.size(); ++i) {
        TSS_CHECK(s, cudaEventRecord(s->t[i].ev_aux, s->t[i].k->stream));
        TSS_CHECK(s, cudaStreamWaitEvent(s->origin, s->t[i].ev_aux, 0));
    }
    // Runs of G non-final steps from buffer 0 replay one CUDA graph (G even:
    // the graph leaves every tile's buffers as it found them); the rest are
    // issued directly, the last step with the final messages.
    const int G = 16;
    int remaining = iterations - 1;
    if (remaining > 0 && s->t[0].k->cur != 0) {
        TSS_OK(issue_steps(s, 1, false));
        --remaining;
    }
    if (remaining >= G) {
        if (!s->graph) {
            cudaGraph_t g = nullptr;
            const int cur0 = s->t[0].k->cur;
            TSS_CHECK(s, cudaStreamBeginCapture(s->origin, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = tsbh::g_launches.load();
            const int st = issue_steps(s, G, false);
            cudaError_t e = cudaStreamEndCapture(s->origin, &g);
            tsbh::g_launches.store(before);
            for (SlabTile &x : s->t) x.k->cur = cur0;  // the capture ran no step
            if (st != TS_B200_OK || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                (void)cudaGetLastError();
                if (st != TS_B200_OK) return st;
                return scuda(s, e, "slab graph capture");
            }
            e = cudaGraphInstantiate(&s->graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return scuda(s, e, "slab graph instantiate");
            s->graph_steps = G;
        }
        while (remaining >= G) {
            TSS_CHECK(s, cudaGraphLaunch(s->graph, s->origin));
            tsbh::g_launches.fetch_add((uint64_t)G * s->launches_per_step, std::memory_order_relaxed);
            remaining -= G;
        }
    }
    if (remaining > 0) TSS_OK(issue_steps(s, remaining, false));
    TSS_OK(issue_steps(s, 1, true));
    // the tiles' own streams continue after the group's work
    TSS_CHECK(s, cudaEventRecord(s->ev_fork, s->origin));
    for (size_t i = 1; i < s->t.size(); ++i)
        TSS_CHECK(s, cudaStreamWaitEvent(s->t[i].k->stream, s->ev_fork, 0));
    return TS_B200_OK;
}

const char *ts_b200_slabs_last_error(const ts_b200_slabs *s) { return s ? s->err.c_str() : ""; }

int ts_b200_slabs_destroy(ts_b200_slabs *s) {
    destroy(s);
    return TS_B200_OK;
}

}  // extern "C"
