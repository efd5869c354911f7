/*
 * ts_b200.h -- C ABI of the B200 Trotter-Suzuki evolution kernel.
 *
 * This is the boundary behind which the checkerboard Trotter-Suzuki step of
 * trotter-suzuki-mpi 1.6.2 runs on one NVIDIA B200 (sm_100a).  It replaces
 * the reference's kernel plug-in interface ITrotterKernel
 * (src/trottersuzuki.h:502-520) and its CUDA implementation CC2Kernel
 * (src/kernel.h:173-269, src/gpukernel.cu:122-728).  The C++ host layer
 * (class B200Kernel, an ITrotterKernel) and the Python binding both call only
 * these functions.
 *
 * Conventions
 *  - Plain pointers and sizes; no C++ types, no exceptions cross this ABI.
 *  - Every function returns a ts_b200_status; TS_B200_OK is 0.  The message
 *    of the last failure on a handle is returned by ts_b200_last_error().
 *    (The reference turns CUDA failures into my_abort() ->
 *    std::runtime_error, src/gpukernel.cu:24-36, src/common.cpp:104-115; the
 *    C++ host layer does the same with these codes.)
 *  - A "tile" is the reference's per-process lattice tile: dim_x * dim_y
 *    cells, row-major, including the periodic halo (src/model.cpp:103-158).
 *    Host arrays are the reference's SoA layout (p_real, p_imag,
 *    src/trottersuzuki.h:125-126); on the device the tile is stored as
 *    interleaved complex numbers (AoS) with a row pitch of a multiple of 4
 *    cells.
 *  - All work is queued on the handle's CUDA stream; calls that return data
 *    to the host synchronise that stream.
 */
#ifndef TS_B200_H
#define TS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TS_B200_OK = 0,
    TS_B200_INVALID_ARGUMENT = 1,
    TS_B200_CUDA_ERROR = 2,
    TS_B200_OUT_OF_MEMORY = 3,
    TS_B200_UNSUPPORTED = 4,
    TS_B200_DEVICE_TIMEOUT = 5,
    TS_B200_NO_DEVICE = 6
} ts_b200_status;

typedef enum {
    TS_B200_FP64 = 0,      /* psi and the exponential table stored and updated in double */
    TS_B200_FP32 = 1       /* psi and the table stored in float, pair updates in float;
                              norm, energies and the renormalisation factor in double */
} ts_b200_precision;

/* Everything a step needs.  Field meanings follow the reference's CPUBlock
 * constructor (src/cpukernel.cpp:172-272) and Lattice (src/trottersuzuki.h:34-56). */
typedef struct {
    int32_t dim_x, dim_y;            /* tile size, halo included (Lattice::dim_x/dim_y) */
    int32_t inner_x0, inner_x1;      /* inner (non-halo) columns, tile coordinates */
    int32_t inner_y0, inner_y1;      /* inner rows, tile coordinates */
    int32_t halo_x, halo_y;          /* Lattice::halo_x/halo_y (4, or 8 with rotation) */
    int32_t periodic_x, periodic_y;  /* Lattice::periods[1] / periods[0] */
    int32_t imag_time;               /* imaginary-time evolution */
    int32_t precision;               /* ts_b200_precision */
    double a_h, b_h, a_v, b_v;       /* cos/sin (cosh/sinh) of dt/(4 m dx^2), dt/(4 m dy^2) */
    double coupling;                 /* g * dt            (coupling_const[0]) */
    double lhy_coupling;             /* g_LHY * dt        (LeeHuangYang_coupling[0]) */
    double alpha_x, alpha_y;         /* rotating-frame constants; both non-zero enable it */
    double rot_offset_x;             /* start_x - rot_coord_x (truncated to int per column) */
    double rot_offset_y;             /* start_y - rot_coord_y */
    double delta_x, delta_y;
    double norm0;                    /* imaginary time: squared norm kept after each step;
                                        0 disables the renormalisation (as the reference) */
    int32_t cylindrical;             /* radial axis x (Lattice::coordinate_system
                                        "cylindrical"): the radial kinetic term and, in
                                        imaginary time, column 0 mirroring column 1 */
    int32_t angular_momentum;        /* State::angular_momentum: parity of that mirror */
    double kin_radial;               /* dt / (8 m dx^2) (kin_radial[0]) */
} ts_b200_desc;

typedef struct ts_b200_kernel ts_b200_kernel;

/* Create a kernel on the current CUDA device.  Allocates the two tile
 * buffers, the exponential table and the reduction scratch.
 * Replaces: CC2Kernel::CC2Kernel (src/gpukernel.cu:122-238),
 *           CPUBlock::CPUBlock (src/cpukernel.cpp:172-272). */
int ts_b200_create(const ts_b200_desc *desc, ts_b200_kernel **out);

/* Free everything.  Replaces: CC2Kernel::~CC2Kernel (src/gpukernel.cu:240-273). */
int ts_b200_destroy(ts_b200_kernel *k);

/* Upload the tile from host SoA arrays with row stride `stride` (cells).
 * Replaces: the state upload in CC2Kernel::CC2Kernel (src/gpukernel.cu:196-206). */
int ts_b200_set_state(ts_b200_kernel *k, const double *p_real, const double *p_imag,
                      size_t stride);

/* Upload exp(-i dt V) (real time) or exp(-dt V) (imaginary time; only the
 * real part is read) for the tile, host SoA with row stride `stride`.
 * Replaces: ITrotterKernel::update_potential (src/trottersuzuki.h:514,
 *           src/gpukernel.cu:378-387). */
int ts_b200_set_exp_potential(ts_b200_kernel *k, const double *pot_real, const double *pot_imag,
                              size_t stride);

/* One Trotter step of the whole tile: the 8 checkerboard pair sweeps, the
 * potential/GPE/LHY phase and (if enabled) the rotating-frame sweeps, fused
 * in one pass.  When `exchange` is non-zero the periodic halo is refreshed
 * afterwards; in imaginary time the step's squared norm is computed and the
 * renormalisation is applied when the tile is next read.
 * Replaces: ITrotterKernel::run_kernel_on_halo + run_kernel +
 *           start/finish_halo_exchange + wait_for_completion
 *           (src/trottersuzuki.h:505-507,517-518; src/gpukernel.cu:439-521). */
int ts_b200_step(ts_b200_kernel *k, int exchange);

/* Refresh the periodic halo of the current tile (no-op for closed lattices).
 * Replaces: ITrotterKernel::start_halo_exchange + finish_halo_exchange
 *           (src/trottersuzuki.h:517-518; single process:
 *           src/cpukernel.cpp:706-716,738-746). */
int ts_b200_halo_exchange(ts_b200_kernel *k);

/* `iterations` steps with the reference's evolve() semantics: the halo is
 * refreshed after every step but the last (src/solver.cpp:186-230).  Steps
 * are replayed from a CUDA graph; nothing synchronises the host. */
int ts_b200_evolve(ts_b200_kernel *k, int iterations);

/* Copy a width x height window at (x, y) of the tile to host SoA arrays with
 * row stride dest_stride (cells), applying any pending renormalisation.
 * Replaces: ITrotterKernel::get_sample (src/trottersuzuki.h:508,
 *           src/gpukernel.cu:547-561). */
int ts_b200_get_sample(ts_b200_kernel *k, size_t dest_stride, size_t x, size_t y, size_t width,
                       size_t height, double *dest_real, double *dest_imag);

/* Squared norm of the inner region times delta_x * delta_y, in double.
 * Replaces: ITrotterKernel::calculate_squared_norm (src/trottersuzuki.h:511,
 *           src/gpukernel.cu:479-500). */
int ts_b200_squared_norm(ts_b200_kernel *k, double *out);

/* Energy functional of src/solver.cpp:244-564 (single component) on the
 * device, FP64 accumulation.  `potential` is the tile of V values (host,
 * row stride dim_x) or NULL to reuse the last one uploaded. */
typedef struct {
    double mass, coupling, lhy_coupling, angular_velocity;
    int32_t start_x, start_y;                    /* Lattice::start_x/start_y */
    int32_t global_no_halo_dim_x, global_no_halo_dim_y;
    double length_x, length_y;
} ts_b200_energy_params;

typedef struct {
    double total, kinetic, potential, rotational, intra, lhy, norm2;
} ts_b200_energy_result;

int ts_b200_energies(ts_b200_kernel *k, const double *potential,
                     const ts_b200_energy_params *params, ts_b200_energy_result *out);

/* Expectation values of src/model.cpp:385-536 (2D, cartesian) on the device. */
typedef struct {
    double norm2, mean_x, mean_xx, mean_y, mean_yy, mean_px, mean_pxpx, mean_py, mean_pypy,
        mean_lz;
} ts_b200_expectation_result;

int ts_b200_expectations(ts_b200_kernel *k, const ts_b200_energy_params *params,
                         ts_b200_expectation_result *out);

/* Squared norm of a caller-owned device tile (AoS complex in `precision`, row
 * pitch `pitch` cells) over the inner region, times delta_x * delta_y, written
 * to the device double `*out` on `stream` (a cudaStream_t, NULL for the
 * default stream).  Allocates nothing: for callers that cannot call cudaMalloc
 * (device memory owned by another allocator or fixed pool; no allocation, and
 * so no implicit device synchronisation, after start-up).  Its scratch is a
 * static device array of the library (128 KiB per GPU, kept until exit):
 * tiles with more than 16384 inner rows are rejected (TS_B200_UNSUPPORTED);
 * the first call on a device looks the array up (cudaGetSymbolAddress), so
 * make it before any stream capture; calls that overlap on the GPU race on
 * the shared scratch.  No counterpart in the reference (which reduces the
 * norm on the host, src/cpukernel.cpp:526-549). */
int ts_b200_squared_norm_noalloc(const void *psi, int precision, size_t pitch, int dim_x,
                                 int dim_y, int inner_x0, int inner_x1, int inner_y0,
                                 int inner_y1, double delta_x, double delta_y, double *out,
                                 void *stream);

/* Device-resident access (for callers that already hold device memory, such
 * as a torch binding or a benchmark).  `aos` is a device array of dim_y rows
 * of dim_x interleaved complex numbers in the kernel's precision with row
 * pitch `pitch` cells. */
int ts_b200_set_state_device(ts_b200_kernel *k, const void *aos, size_t pitch);
int ts_b200_get_state_device(ts_b200_kernel *k, void *aos, size_t pitch);
int ts_b200_set_exp_potential_device(ts_b200_kernel *k, const void *table, size_t pitch);

/* The exponential table from a potential already on the device: `potential`
 * holds dim_y rows of dim_x doubles V(x, y) with row pitch `pitch` doubles;
 * the table exp(-i dt V) (real time) or exp(-dt V) (imaginary time) is built
 * on the device in the kernel's precision.  Replaces, for a potential that
 * changes every step, the host re-tabulation and upload of the reference's
 * Solver::evolve (src/solver.cpp:187-200 with initialize_exp_potential,
 * src/solver.cpp:74-109, and the kernel's update_potential). */
int ts_b200_set_potential_device(ts_b200_kernel *k, const double *potential, size_t pitch,
                                 double delta_t);

/* `count` steps, step i with the potential V_i already on the device:
 * V_i = potentials + i * slab doubles (dim_y rows, row pitch `pitch`), its
 * table built as by ts_b200_set_potential_device before the step.  Every
 * step refreshes the halo when `exchange` is nonzero, none does otherwise
 * (a run of the reference's per-step Python loop, classes_extension.py:
 * 393-403, where each step is an evolve call of its own).  With count >= 2
 * in FP64 real time on cartesian one-component tiles (no rotating frame, the
 * default row walk) with an even dim_x, even `pitch` and `slab` and 16-byte
 * aligned planes, each step forms the table's entries from V_i itself (the
 * same values) instead of a table pass; the table of the last potential is
 * then built once, so later steps see the same table either way. */
int ts_b200_evolve_potentials(ts_b200_kernel *k, const double *potentials, size_t pitch,
                              size_t slab, int count, double delta_t, int exchange);

/* One lattice split across ranks in slabs of rows (the reference's MPI
 * tiles, src/common.cpp:83-102, and their halo exchange,
 * src/cpukernel.cpp:691-747): the current buffer's rows [row0, row0 + nrows)
 * as one device span of `bytes` (rows are contiguous, pitch included), for
 * sending the edge rows and receiving the halo rows; the device address of
 * the squared norm of the tile's inner region after the last step (times
 * dx dy, before renormalisation), to be summed over the ranks; and the
 * imaginary-time renormalisation from that sum (device pointer), which
 * replaces the one the step took from the tile alone. */
int ts_b200_rows(ts_b200_kernel *k, int row0, int nrows, void **ptr, size_t *bytes);
int ts_b200_last_norm(ts_b200_kernel *k, double **device_ptr);
int ts_b200_renormalize_from(ts_b200_kernel *k, const double *total_norm);

/* ---- Slabs driven natively: the same lattice split, with the exchange and
 * the joint norm issued on the tiles' streams (no host step per step),
 * replayed from CUDA graphs, and each step run as its edge bands (the rows
 * the neighbours need) and its interior (which reads no halo row) on two
 * streams, so that the exchange overlaps the interior: the reference's
 * halo-first step, src/solver.cpp:202-210 with src/cpukernel.cpp:691-747
 * (run_kernel_on_halo, start_halo_exchange, run_kernel,
 * finish_halo_exchange).  A slab tile is closed in y (periodic_y = 0): inner
 * rows [inner_y0, inner_y1), halo_y rows above it when it has an upper
 * neighbour (inner_y0 = halo_y, else 0) and below it when it has a lower one
 * (dim_y - inner_y1 = halo_y, else inner_y1 = dim_y); periodic x is kept on
 * the tile.  Imaginary-time tiles carry the whole lattice's norm0. */
typedef struct ts_b200_slabs ts_b200_slabs;

/* A slab's neighbours: up (smaller rows) and down; a tile index of the group
 * (slabs of one process) or a rank of the communicator (NCCL); -1 none.  The
 * *_wraps flags mark a link across the lattice's periodic wrap, whose
 * messages the last step of an evolve call leaves out (src/solver.cpp:
 * 203-209, where a single tile skips its periodic halo copy). */
typedef struct {
    int32_t up, down;
    int32_t up_wraps, down_wraps;
    /* periodic x: the tile rows [xhalo_row0, xhalo_row1) whose x halo the
     * slab refreshes after a step, the rows whose lattice row the whole
     * tile refreshes (src/cpukernel.cpp:706-716: its rows [inner_y0,
     * inner_y0 + dim_y - 2 halo_y); for a lattice periodic in y every row,
     * its y-halo rows taking refreshed rows).  The received halo rows are
     * refreshed by the receiver: a row's x halo comes from its own cells. */
    int32_t xhalo_row0, xhalo_row1;
} ts_b200_slab_link;

/* Row windows of a slab's split step (host only, no device needed): out[0..3]
 * the edge windows [a0, a1) and [b0, b1) (b0 = b1 = 0 for one), out[4..5] the
 * interior, out[6] 1 when the step splits (a neighbour and an interior of
 * at least 2 reach + 2 rows), out[7] 0.  reach: rows a segment's walk reads
 * past its output rows (4; 6 in a rotating frame), at most halo. */
int ts_b200_slab_windows(int rows, int inner_y0, int inner_y1, int halo, int reach, int has_up,
                         int has_down, int32_t out[8]);

/* The messages of a slab's step (host only): up to 4 entries of
 * (peer, first tile row of the h-row span, tag, 1 send / 0 receive) in the
 * order both ends post them, as src/cpukernel.cpp:717-747: the last h inner
 * rows go down into the lower neighbour's top halo (tag 1), the first h
 * inner rows up into the upper neighbour's bottom halo (tag 2).  final: the
 * last step of an evolve call (links across the wrap left out).  Returns the
 * number of entries (negative: invalid arguments). */
int ts_b200_slab_messages(int inner_y0, int inner_y1, int halo, const ts_b200_slab_link *link,
                          int final, int32_t out[16]);

/* Slabs of one process on one GPU (their exchange by device copies). */
int ts_b200_slabs_create_local(ts_b200_slabs **out, ts_b200_kernel *const *tiles,
                               const ts_b200_slab_link *links, int n_tiles);

/* One slab per process, the exchange and the norm sum over NCCL (loaded at
 * run time: the libnccl.so.2 already in the process, else the loader's).
 * Rank 0 draws the id with ts_b200_nccl_unique_id and the ranks share it;
 * creation is collective over the nranks ranks. */
int ts_b200_nccl_unique_id(void *id, size_t bytes);
int ts_b200_slabs_create_nccl(ts_b200_slabs **out, ts_b200_kernel *tile,
                              const ts_b200_slab_link *link, const void *nccl_id, size_t id_bytes,
                              int nranks, int rank);

/* 1 (default): split steps where a slab allows; 0: one launch per step. */
int ts_b200_slabs_set_split(ts_b200_slabs *s, int on);

/* The plan of tile `tile`: out[0..6] as ts_b200_slab_windows (as used),
 * out[7] the group's kernel launches per step. */
int ts_b200_slabs_plan(ts_b200_slabs *s, int tile, int32_t out[8]);

/* `iterations` steps of every slab, ordered after the work queued on the
 * tiles' streams, and the tiles' streams ordered after them (no host
 * synchronisation).  Steps 0 .. iterations-2 exchange every message, the
 * last leaves out the ones across the periodic wrap. */
int ts_b200_slabs_evolve(ts_b200_slabs *s, int iterations);
const char *ts_b200_slabs_last_error(const ts_b200_slabs *s);
int ts_b200_slabs_destroy(ts_b200_slabs *s);

/* Queue all work of this handle on `stream` (a cudaStream_t); NULL restores
 * the handle's own stream.  Every call that reads or writes device memory the
 * caller owns (the *_device calls) is ordered on the handle's stream only:
 * the caller orders its own stream against it, with these two or with
 * ts_b200_set_stream to its own stream.  ts_b200_stream_wait: the handle's
 * stream waits for the work queued so far on `stream` (NULL: the legacy
 * default stream); ts_b200_stream_signal: `stream` waits for the work queued
 * so far on the handle's. */
int ts_b200_set_stream(ts_b200_kernel *k, void *stream);
int ts_b200_stream_wait(ts_b200_kernel *k, void *stream);
int ts_b200_stream_signal(ts_b200_kernel *k, void *stream);
int ts_b200_synchronize(ts_b200_kernel *k);

/* Geometry of the fused step launch chosen for this tile (for reporting):
 * cells per lane, rows per segment, warps per block, ring depth, tasks, and
 * the row walk (0 checked; 1 or 2: look-ahead, rows per iteration). */
typedef struct {
    int32_t cells_per_lane, segment_rows, warps_per_block, ring_depth;
    int32_t strips, segments, blocks, threads;
    int64_t smem_bytes;
    int32_t walk, reserved;
} ts_b200_launch_shape;

int ts_b200_launch_info(const ts_b200_kernel *k, ts_b200_launch_shape *out);

/* Override the launch shape (autotuner / tests).  Zero fields keep the
 * current choice.  Only shapes this build instantiates are accepted. */
int ts_b200_set_launch(ts_b200_kernel *k, int cells_per_lane, int segment_rows, int warps_per_block,
                       int ring_depth);

/* Row walk of the fused step (no counterpart in the reference; every walk
 * performs the same operations per cell): 2 (default) the look-ahead walk of
 * every variant, with even segments, a ring of 6 rows (8 in a rotating
 * frame), 4 or 8 warps per block (4 in a rotating frame) and two rows per
 * iteration (one mbarrier per row pair; with 4 cells per lane one row,
 * except in a single-precision rotating frame); 1 the same walk with one row
 * per iteration; 0 the checked walk (a rotating frame then takes 2 cells per
 * lane).  ts_b200_launch_info reports the rows per iteration in use (0 for
 * the checked walk). */
int ts_b200_set_walk(ts_b200_kernel *k, int walk);

/* The look-ahead walk launches each fused step with a programmatic
 * dependency on the previous kernel of the stream (on = 1, the default): the
 * step's blocks are scheduled as the previous step's blocks retire and set up
 * their shared memory, then wait for the previous kernel to complete before
 * they read the tile.  on = 0 launches each step after the previous kernel
 * has completed.  No counterpart in the reference. */
int ts_b200_set_overlap(ts_b200_kernel *k, int on);

/* ---- Batched evolution (no counterpart in the reference, which evolves one
 * lattice per Solver; the batch replaces a loop of per-tile evolve() calls).
 *
 * A batch advances many tiles of uneven sizes together: each Trotter step is
 * one persistent launch over the tasks of all tiles (plus, in imaginary time,
 * one per-tile norm reduction launch, in FP32 real time one launch advancing
 * the tiles' coefficient schedules, and for periodic tiles one batched halo
 * refresh), 32-step runs replayed from a CUDA graph.  The batch borrows the
 * tiles' device state: set states and tables, read results, energies and
 * norms through the tiles' own calls.  All tiles must share precision, time
 * mode and device and have no rotating frame (TS_B200_UNSUPPORTED); a tile
 * appears once.  The batch orders itself after work queued on the tiles'
 * streams and the tiles' streams after the batch's work.  The batched step
 * runs the row walk its tiles are set to at creation (ts_b200_set_walk): the
 * look-ahead walk with two rows per iteration, or the checked walk if any
 * tile is set to it; ts_b200_batch_launch_info reports it. */
typedef struct ts_b200_batch ts_b200_batch;

int ts_b200_batch_create(ts_b200_kernel *const *kernels, int n, ts_b200_batch **out);
void ts_b200_batch_destroy(ts_b200_batch *b);
int ts_b200_batch_size(const ts_b200_batch *b);

/* `iterations` Trotter steps of every tile, with the per-tile protocol of
 * ts_b200_evolve (halo refresh after every step but the last). */
int ts_b200_batch_evolve(ts_b200_batch *b, int iterations);

/* Wait for the batch's queued work; TS_B200_DEVICE_TIMEOUT if a bounded wait
 * in the batched step gave up. */
int ts_b200_batch_synchronize(ts_b200_batch *b);

/* Queue the batch's work on `stream` (a cudaStream_t); NULL restores the
 * batch's own stream. */
int ts_b200_batch_set_stream(ts_b200_batch *b, void *stream);

/* Tile shape of the batched launch: rows per segment task (even; capped by
 * each tile's height) and warps per block (1, 2 or 4).  Zero keeps a field. */
int ts_b200_batch_set_launch(ts_b200_batch *b, int segment_rows, int warps_per_block);

/* Autotuner: times `trial_steps` batched steps for each candidate shape (rows
 * per segment 16..256, 2 or 4 warps per block), twice over the candidate list,
 * and keeps the shape with the fastest of its two times.  The
 * trials read the tiles' current state and write only the scratch buffer, so
 * the state is unchanged.  With use_cache != 0 a shape tuned earlier in this
 * process for the same precision, time mode and tile sizes is reused
 * without timing.  Synchronises the batch's stream. */
int ts_b200_batch_autotune(ts_b200_batch *b, int trial_steps, int use_cache);

/* Current shape: strips and segments are summed over the tiles. */
int ts_b200_batch_launch_info(ts_b200_batch *b, ts_b200_launch_shape *out);
const char *ts_b200_batch_last_error(const ts_b200_batch *b);

/* ---- Adjoint (reverse mode) of a real-time evolution (no counterpart in the
 * reference, which has no derivatives).  For a loss L(psi(T)) the reverse
 * pass turns dL/dpsi(T) into dL/dpsi(0) and dL/dV(x, y) for the `steps`
 * Trotter steps of the forward pass.  Complex fields are device arrays of
 * interleaved doubles (re, im) with row stride dim_x cells; gradients follow
 * the real-pair convention dL/dre + i dL/dim.  The potential V is a device
 * array of dim_x * dim_y doubles; its table exp(-i V dt) is built on the
 * device.  Real time, FP64, closed boundaries, no rotating frame
 * (TS_B200_UNSUPPORTED otherwise).
 * checkpoint_every == 0: the reverse pass recovers the forward states by
 * inverse steps; linear evolution only (coupling = lhy_coupling = 0, else
 * TS_B200_INVALID_ARGUMENT).  checkpoint_every = k > 0: the forward pass
 * stores every k-th state and the reverse pass recomputes each segment
 * (device memory: ceil(steps / k) + k - 1 extra states).  One backward per
 * forward; the engine works on its own stream (ts_b200_adjoint_set_stream). */
typedef struct ts_b200_adjoint ts_b200_adjoint;

int ts_b200_adjoint_create(const ts_b200_desc *d, double delta_t, int steps, int checkpoint_every,
                           ts_b200_adjoint **out);
void ts_b200_adjoint_destroy(ts_b200_adjoint *a);
int ts_b200_adjoint_set_stream(ts_b200_adjoint *a, void *stream);
/* Rows per segment task of the adjoint pass (even, >= 2) and of the forward
 * and recomputation steps (ts_b200_set_launch); 0 keeps the choice. */
int ts_b200_adjoint_set_segments(ts_b200_adjoint *a, int adjoint_rows, int forward_rows);
/* psi_t may be NULL (the final state stays in the engine). */
int ts_b200_adjoint_forward(ts_b200_adjoint *a, const double *potential, const void *psi0,
                            void *psi_t);
/* grad_potential and grad_psi0 may be NULL. */
int ts_b200_adjoint_backward(ts_b200_adjoint *a, const void *grad_psi_t, double *grad_potential,
                             void *grad_psi0);
/* Wait for the engine's queued work; TS_B200_DEVICE_TIMEOUT if a bounded
 * wait gave up. */
int ts_b200_adjoint_synchronize(ts_b200_adjoint *a);
const char *ts_b200_adjoint_last_error(const ts_b200_adjoint *a);

/* ------------------------------------------------------------ two components
 * Two species evolved together: the reference's two-wavefunction kernel and
 * loop (CPUBlock two-state constructor src/cpukernel.cpp:274-392,
 * rabi_coupling / normalization src/cpukernel.cpp:581-667, the coupled phase
 * src/cpucartesian.cpp:73-92,113-126, the Rabi rotation
 * src/cpucartesian.cpp:264-290, Solver::evolve src/solver.cpp:172-230).
 * `a` and `b` are two tiles of the same geometry, precision and time mode,
 * each with its own state, table and step constants (mass, g * dt, norm0 of
 * its ts_b200_desc); no rotating frame and no Lee-Huang-Yang term, as in the
 * reference's two-component path.  While paired the tiles step only through
 * the pair (ts_b200_step / ts_b200_evolve on them return
 * TS_B200_UNSUPPORTED); their states are read and written with the tiles' own
 * calls, and b's work is queued on a's stream. */
typedef struct ts_b200_pair ts_b200_pair;

/* coupling_ab: g_ab; omega_r, omega_i: the Rabi coupling omega (the
 * reference's Hamiltonian2Component::omega_r, omega_i). */
int ts_b200_pair_create(ts_b200_kernel *a, ts_b200_kernel *b, double coupling_ab,
                        double omega_r, double omega_i, double delta_t, ts_b200_pair **out);
/* The Rabi rotation by var * delta_t alone: Solver::evolve's half step before
 * the loop (src/solver.cpp:172-177, rabi_coupling(0.5, delta_t)). */
int ts_b200_pair_rabi(ts_b200_pair *p, double var);
/* `iterations` steps of the loop: species a, species b (with a's state from
 * before a's step), the Rabi rotation (a half one on the last step), and in
 * imaginary time with a Rabi coupling the joint normalisation.  Every step
 * but the last refreshes the halos. */
int ts_b200_pair_evolve(ts_b200_pair *p, int iterations);
/* `steps` steps of that loop; with final_steps == 0 none of them is the
 * call's last (all refresh the halos and take a full Rabi rotation), so a
 * caller can re-tabulate a time-dependent potential between runs. */
int ts_b200_pair_steps(ts_b200_pair *p, int steps, int final_steps);
/* The plug-in protocol's pieces (ITrotterKernel::run_kernel for species
 * `which`, 0 = a, 1 = b, without the halo refresh, which ts_b200_halo_exchange
 * on the species' tile does; ITrotterKernel::normalization).  Species b's step
 * must follow species a's. */
int ts_b200_pair_step_species(ts_b200_pair *p, int which);
int ts_b200_pair_normalize(ts_b200_pair *p);
/* Inter-species and Rabi energies of Solver::calculate_energy_expected_values
 * (src/solver.cpp:340-353,438-439,549-550), as the reference writes them:
 * sum g_ab |a|^4 |b|^4 and 0.5 sum |a|^2 |b|^2 2 Re(conj(a) b omega), each over
 * (sum |a|^2)(sum |b|^2) on the inner region.  Synchronises a's stream. */
int ts_b200_pair_cross_energies(ts_b200_pair *p, double *inter_species, double *rabi);
const char *ts_b200_pair_last_error(const ts_b200_pair *p);
/* Unpairs the tiles (each then steps alone again) and frees the pair. */
int ts_b200_pair_destroy(ts_b200_pair *p);

/* Autotuner for this tile: times `trial_steps` steps for each balanced launch
 * shape (rows per segment such that every SM holds the same number of
 * blocks, for 1 .. the resident blocks per SM, 4 or 2 warps per block; 4 or 8
 * with the look-ahead walk, each with and without programmatic dependent
 * launch) and for segments of 32, 64 and 128 rows taken by the persistent
 * warps in turn, and keeps the fastest.  The trials read the current state and write the other
 * buffer, the scalars a step updates are restored: the state is unchanged.
 * Synchronises the tile's stream.  No counterpart in the reference. */
int ts_b200_autotune(ts_b200_kernel *k, int trial_steps);

/* Pinned host memory for the state arrays (page-locked so that host<->device
 * copies run at full PCIe/C2C rate). */
int ts_b200_host_alloc(void **ptr, size_t bytes);
int ts_b200_host_free(void *ptr);

const char *ts_b200_last_error(const ts_b200_kernel *k);
const char *ts_b200_status_string(int status);

/* Library version string and the number of kernel launches made by this
 * process so far (used to report how many launches a measurement made). */
const char *ts_b200_version(void);
uint64_t ts_b200_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* TS_B200_H */
