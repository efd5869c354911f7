// Internal: the per-tile handle behind the C ABI and the helpers the
// batched path (batch.cu) shares with the single-tile path (ts_b200.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>

#include "step_kernel.cuh"
#include "ts_b200.h"

// =================================================================== handle
struct ts_b200_kernel {
    ts_b200_desc d{};
    int W = 0, H = 0, P = 0;
    bool fp32 = false, imag = false, rot = false;
    int phase = 0;  // 0 none, 1 g|psi|^2, 2 with Lee-Huang-Yang, 3 one component of a pair
                    // (7: the same with the Rabi rotation applied at load), | 4 cylindrical
    size_t cell = 0, tab_cell = 0;
    void *psi[2] = {nullptr, nullptr};
    int cur = 0;
    void *tab = nullptr;
    void *row_ab = nullptr, *col_ab = nullptr;
    double *partials = nullptr;
    size_t partials_cap = 0;
    tsb::Scalars *scal = nullptr;
    double *staging = nullptr;  // 2 * W * H doubles
    double *vtab = nullptr;     // V for energies (W * H)
    bool have_v = false;
    double *red_partials = nullptr;
    double *red_out = nullptr;
    unsigned int *red_ticket = nullptr;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaEvent_t ev_order = nullptr;  // ts_b200_stream_wait / _signal
    // ts_b200_evolve_potentials in progress with the table made inside the
    // step: the potential the next step reads (row pitch in bytes) and dt
    const double *vpot = nullptr;
    size_t vpot_pitch = 0;
    double vpot_dt = 0.0;
    int C = 2, seg_h = 64, warps = 4, ring = 4;
    int resident_blocks = 0;  // blocks of the current launch shape resident on the GPU (0: unknown)
    bool auto_seg = true;     // pick the segment height from the resident grid
    bool overlap = true;      // look-ahead walk: programmatic dependent launch of each step
    int walk2 = 2;            // rows per iteration of the look-ahead walk (walk2.cuh) where
                              // the variant has one; 0: the checked walk
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0;
    float4 *kin_sched = nullptr;  // FP32 real time: per-step kinetic coefficients
    int num_sms = 148;
    int device = 0;
    // two components (pair.cu): the tile is one species of a ts_b200_pair;
    // pb / pb_scale / cab are the other species' tile for the next step
    bool cyl = false;        // cylindrical lattice (radial axis x)
    void *rad = nullptr;     // per column: radial pair (a, b), (c, 0) in the tile's precision
    bool pair_mode = false;
    int phase_alone = 0;  // phase outside the pair
    const void *pb = nullptr;
    const double *pb_scale = nullptr;
    double cab = 0.0;
    // phase 7: cos (minus 1 in single precision), the other cell's factor in
    // this species' rotation (re, im), this cell's factor in the other's
    double rabi[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    std::string err;
};

namespace tsbh {

// Kernel launches made through the library (reported by ts_b200_launch_count).
extern std::atomic<uint64_t> g_launches;

inline int div_up(long a, long b) { return (int)((a + b - 1) / b); }

// Entries of the FP32 real-time kinetic coefficient schedule (repeats after).
constexpr int kSchedLen = 4096;

// Bytes of one ring slot: a row of 32*C cells of psi and of the table (and,
// for one species of a pair, of the other species).
inline int slot_bytes(int C, bool fp32, bool imag, bool pb = false) {
    const int cell = fp32 ? 8 : 16;
    const int tab = imag ? cell / 2 : cell;
    return 32 * C * (cell + tab + (pb ? cell : 0));
}

// Kernel launches of one step of the tile (exchange: with the halo refresh).
int launch_step_tile(ts_b200_kernel *k, int exchange);

// Step constants of a tile in the kernel's precision (delta form in float):
// every StepArgs field except the buffers, the task geometry and the scratch.
template <typename T>
void fill_step_constants(const ts_b200_kernel *k, tsb::StepArgs<T> &a);

// One fused step of the tile from device buffer `in` to `out` (tile layout,
// row pitch k->P), on the tile's stream; the tile's own buffers are untouched.
int launch_step_buffers(ts_b200_kernel *k, const void *in, void *out);

// Imaginary time: the squared norm every step restores (a launch parameter of
// the step, so a captured evolve graph is dropped when it changes).
int set_norm0(ts_b200_kernel *k, double norm0);

// One launch of the fused step over some of the tile's output rows: window
// [a0, a1) and, if b1 > b0, window [b0, b1) (even starts; a1 = 0: the whole
// tile), on `stream` (null: the tile's), with its own block ticket and, in
// imaginary time, its own block partials (null: the tile's).  pair_norm /
// pair_ticket non-null: the step is split over two such launches (pair_slot
// 0 and 1) that read the same input buffer and write disjoint rows; the
// second to finish ends the step.  blocks > 0 caps the grid.
struct StepPart {
    int a0 = 0, a1 = 0, b0 = 0, b1 = 0;
    cudaStream_t stream = nullptr;
    double *partials = nullptr;
    unsigned int *ticket = nullptr;
    double *pair_norm = nullptr;
    unsigned int *pair_ticket = nullptr;
    int pair_slot = 0;
    int blocks = 0;
    double *inv_copy = nullptr;  // imaginary time: the step's factor also written here
    bool pdl = false;            // programmatic dependent launch (whole-tile parts)
};

// Resident grid and segment height of the tile's step (once per shape).
int configure_step(ts_b200_kernel *k);
// Grid of a part's launch (after configure_step).
int part_blocks(const ts_b200_kernel *k, const StepPart &p);
int launch_step_part(ts_b200_kernel *k, const void *in, void *out, const StepPart &p);
// Rows a segment's walk reads beyond its output rows (the variant's HY).
int step_reach_rows(const ts_b200_kernel *k);
// Periodic halo of the current buffer (x only for a slab tile) on `stream`;
// xr1 > xr0: the x halo of rows [xr0, xr1) (default: the reference's rows).
int launch_halo_on(ts_b200_kernel *k, cudaStream_t stream, int xr0 = 0, int xr1 = 0);

}  // namespace tsbh
