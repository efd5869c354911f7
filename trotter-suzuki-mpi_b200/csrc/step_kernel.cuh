// Fused Trotter-Suzuki step for sm_100a.
//
// One launch advances the whole tile by one full step: the checkerboard pair
// sweeps V0 H0 V1 H1 P [R] H1 V1 H0 V0 of src/cpukernel.cpp:22-92 with the
// pair updates of src/cpucartesian.cpp:4-70, the potential / GPE / LHY phase
// of src/cpucartesian.cpp:94-108,128-136 and the rotating-frame sweeps of
// src/cpucartesian.cpp:141-262, each tile cell read once and written once.
//
// Work decomposition ("streaming strips"):
//   * The tile is cut into column strips.  A warp owns one strip of
//     32 lanes x C cells (C consecutive columns per lane) and walks down a
//     segment of rows.  The outer HX columns on each side are recomputed
//     halo (4 for the 4 horizontal sweeps, 8 when the 4 rotation row sweeps
//     are added); the strip writes only its middle 32*C - 2*HX columns.
//   * Walking down the rows, each lane keeps a window of NWIN rows of its C
//     cells in registers.  A vertical sweep pairs a row with the one below,
//     so every vertical stage of the sequence runs one row behind the
//     previous one: with rows r (just loaded) ... r-NWIN+1 in the window,
//     stage k works on the row pair that has become complete for it.  Row
//     r-NWIN+1 leaves the window finished and is stored.  A segment reads HY
//     rows above and below the rows it writes (4 vertical sweeps, 6 with the
//     two rotation column sweeps).
//   * Horizontal pairs inside a lane's C cells are register operations;
//     pairs that straddle two lanes exchange the neighbour cell with a warp
//     shuffle.  Pairs that would cross the tile edge are skipped, which is
//     the reference's closed boundary (and its tile edge in periodic mode).
//   * Rows reach shared memory through cp.async.bulk (the TMA bulk-copy
//     engine) into a per-warp ring of D slots completed by mbarriers; a
//     slot holds one row of psi and one row of the exponential table.  The
//     table row is consumed two iterations after the psi row, then the slot
//     is refilled D rows ahead.  Every mbarrier wait is bounded; a wait that
//     gives up sets the error word and abandons the segment.
//
// Imaginary time (IMAG): the pair matrix is [[a, b], [b, a]], the table is
// real, and the squared norm of the written inner cells is reduced in FP64
// (per-warp partials, then the last block to finish sums them in a fixed
// order).  The renormalisation of src/cpukernel.cpp:551-562 is deferred: the
// next launch multiplies every cell it reads by 1/sqrt(norm/norm0).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace tsb {

template <typename T>
struct Cx {
    T re, im;
};

struct Scalars {
    double pending_inv;  // factor applied to the tile when it is next read
    double last_norm;    // squared norm * dx * dy of the unnormalised tile of the last step
    unsigned int ticket; // blocks finished in the current launch
    int error;           // non-zero: a bounded wait gave up
    int renorm;          // imaginary-time renormalisation enabled (norm0 != 0)
    unsigned int step;   // steps taken (indexes the coefficient schedule)
    // two components: pending_inv before the last step's update (the factor
    // of the buffer that step read) and the norm the next step keeps
    double prev_inv;
    double norm_target;
};

template <typename T>
struct StepArgs {
    const void *psi_in;
    void *psi_out;
    const void *pot;     // Cx<T> per cell in real time, T per cell in imaginary time
    const void *row_ab;  // Cx<T> per tile row: (a, b) of the rotation row sweeps
    const void *col_ab;  // Cx<T> per tile column: (a, b) of the rotation column sweeps
    int W, H, P;         // tile width, height, row pitch (cells, multiple of 4)
    int ix0, ix1, iy0, iy1;
    int n_strips, n_segs, seg_h, ring;
    T aH, bH, aV, bV;
    T ca, caa;           // g*dt and g_LHY*dt
    double *partials;    // one per task (imaginary time)
    // FP32 real time: per-step kinetic coefficients (aH-1, bH, aV-1, bV),
    // entry scal->step mod sched_len; null: aH..bV above
    const float4 *kin_sched;
    int sched_len;
    Scalars *scal;
    double dxdy, norm0;
    // two components: the other species' tile at the start of this step, the
    // factor that normalises it, and g_ab * dt
    const void *pb;
    const double *pb_scale;
    T cab;
    // two components in real time, phase bit 8: the Rabi rotation that
    // follows the previous step, applied to (own, other) as the rows arrive:
    // cos (minus 1 in delta form), the complex factor of the other species'
    // cell in the own cell's rotation and that of the own cell in the other's
    T rabi_cc, rabi_sr, rabi_si, rabi_or, rabi_oi;
    // cylindrical: per tile column x, the radial pair (x, x+1) as (a, b, c, 0)
    // (a - 1 in delta form); the sign of the mirrored axis column
    const void *rad;
    T mirror_sign;
    // Output rows of the launch.  win_n0 = 0: the whole tile, segment s the
    // rows [s seg_h, (s + 1) seg_h) clipped to H.  Otherwise two windows of
    // rows (even starts): segments 0 .. win_n0-1 cover [win_a0, win_a1),
    // the rest [win_b0, win_b1).  A slab's step runs as two launches over
    // disjoint windows (its edge bands, then its interior), which read the
    // same input buffer.
    int win_n0, win_a0, win_a1, win_b0, win_b1;
    // The launch's block ticket (null: scal->ticket).  pair_norm non-null:
    // the step is split over two launches, each writes its squared norm to
    // pair_norm[pair_slot]; the last block of the second launch to finish
    // (pair_ticket) sums them, slot 0 first, and ends the step (norm,
    // renormalisation, coefficient schedule).
    unsigned int *ticket;
    double *pair_norm;
    unsigned int *pair_ticket;
    int pair_slot;
    // imaginary time, non-null: the step's renormalisation factor is also
    // written here (a recomputation keeping each step's factor)
    double *inv_copy;
    // pot's row pitch in bytes (0: P cells of the table type) and, for the
    // variants that read V instead of the table (phase bit 16), dt
    size_t pot_pitch;
    double pot_dt;
};

// Output rows [oy0, oy1) of segment `seg` of the launch.
template <typename T>
__device__ __forceinline__ void segment_rows(const StepArgs<T> &a, int seg, int &oy0, int &oy1) {
    if (a.win_n0 == 0) {
        oy0 = seg * a.seg_h;
        oy1 = min(oy0 + a.seg_h, a.H);
    } else if (seg < a.win_n0) {
        oy0 = a.win_a0 + seg * a.seg_h;
        oy1 = min(oy0 + a.seg_h, a.win_a1);
    } else {
        oy0 = a.win_b0 + (seg - a.win_n0) * a.seg_h;
        oy1 = min(oy0 + a.seg_h, a.win_b1);
    }
}

template <typename T>
__device__ __forceinline__ unsigned int *launch_ticket(const StepArgs<T> &a) {
    return a.ticket ? a.ticket : &a.scal->ticket;
}

// Called by the last block of a launch (one thread): true when the step ends
// with this launch (a single launch, or the second of a split step to finish).
template <typename T>
__device__ __forceinline__ bool step_ends_here(const StepArgs<T> &a) {
    if (!a.pair_ticket) return true;
    __threadfence();
    if (atomicAdd(a.pair_ticket, 1u) != 1u) return false;
    *a.pair_ticket = 0u;
    __threadfence();
    return true;
}

// Imaginary time, the last block of a launch with the launch's squared norm
// in *tot: true when the step ends here, with the step's norm in *tot (for a
// split step, the two launches' norms, slot 0 first).
template <typename T>
__device__ __forceinline__ bool split_norm_total(const StepArgs<T> &a, double *tot) {
    if (!a.pair_norm) return true;
    a.pair_norm[a.pair_slot] = *tot;
    if (!step_ends_here(a)) return false;
    *tot = __ldcg(&a.pair_norm[0]) + __ldcg(&a.pair_norm[1]);
    return true;
}

// ---------------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up after `limit_ns` nanoseconds of polling.  Called by
// all lanes of a warp for the same barrier and phase; the vote keeps the loop
// warp-uniform.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  uint64_t limit_ns = 1000000000ull) {
    if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
    const uint64_t t0 = global_ns();
    while (true) {
        if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
        if (__any_sync(0xffffffffu, global_ns() - t0 > limit_ns)) return false;
    }
}

// ------------------------------------------------------------- pair algebra
// Multiply-adds are written as explicit fused operations so that every
// kernel variant (cells per lane, rotation on/off) performs the same
// rounding for a given cell: the result does not depend on the launch shape.
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double mul_t(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_t(float a, float b) { return __fmul_rn(a, b); }

// FP32 storage works in "delta form": a coefficient a that is close to 1 is
// carried as a - 1, and an update x' = a x + y is evaluated as
// x + ((a - 1) x + y).  Stored in float, a itself would be off by up to half an
// ulp of 1 (6e-8), the same on every sweep, and the norm would drift by that
// much per sweep; a - 1 is small, so its rounding error is tiny.  The FP64 path
// keeps the reference's form a x + y.
template <typename T>
struct DeltaForm {
    static constexpr bool value = std::is_same<T, float>::value;
};

// z + ((a - 1) z + p) in delta form, a z + p otherwise (a is a - 1 in delta form).
template <typename T>
__device__ __forceinline__ T lin(T a, T z, T p) {
    if (DeltaForm<T>::value) return z + fma_t(a, z, p);
    return fma_t(a, z, p);
}

// The two pair forms, for a coefficient pair (a, b) and a cell s with its
// partner p:
//   direct: s + (a s + b p) per component (a s + b p without delta form),
//   cross:  the same with b p replaced by i b p (re <- -b p.im, im <- b p.re).
template <typename T>
__device__ __forceinline__ Cx<T> pair_direct(Cx<T> s, Cx<T> p, T a, T b) {
    return Cx<T>{lin(a, s.re, mul_t(b, p.re)), lin(a, s.im, mul_t(b, p.im))};
}
template <typename T>
__device__ __forceinline__ Cx<T> pair_cross(Cx<T> s, Cx<T> p, T a, T b) {
    return Cx<T>{lin(a, s.re, -mul_t(b, p.im)), lin(a, s.im, mul_t(b, p.re))};
}
// Single precision: both components in packed pairs (FMUL2 / FFMA2 / FADD2
// of sm_100) with the same roundings as the scalar forms.  In the cross form
// the partner enters with its halves swapped, so its two fused multiply-adds
// stay scalar: a packed one would need the swap first.
template <>
__device__ __forceinline__ Cx<float> pair_direct<float>(Cx<float> s, Cx<float> p, float a,
                                                        float b) {
    const float2 s2 = make_float2(s.re, s.im);
    const float2 t = __fmul2_rn(make_float2(b, b), make_float2(p.re, p.im));
    const float2 r = __fadd2_rn(s2, __ffma2_rn(make_float2(a, a), s2, t));
    return Cx<float>{r.x, r.y};
}
template <>
__device__ __forceinline__ Cx<float> pair_cross<float>(Cx<float> s, Cx<float> p, float a,
                                                       float b) {
    const float2 t = __fmul2_rn(make_float2(b, b), make_float2(p.re, p.im));
    const float2 u = make_float2(__fmaf_rn(a, s.re, -t.y), __fmaf_rn(a, s.im, t.x));
    const float2 r = __fadd2_rn(make_float2(s.re, s.im), u);
    return Cx<float>{r.x, r.y};
}

// Kinetic pair (src/cpucartesian.cpp:8-11 real time, :29-32 imaginary time);
// the update is symmetric, so each cell is updated from (self, partner).
template <bool IMAG, typename T>
__device__ __forceinline__ Cx<T> kin(Cx<T> s, Cx<T> p, T a, T b) {
    return IMAG ? pair_direct(s, p, a, b) : pair_cross(s, p, a, b);
}

// v * f for a real factor f (both components, one packed multiply in single precision).
__device__ __forceinline__ Cx<double> scale_cx(Cx<double> v, double f) {
    return Cx<double>{mul_t(f, v.re), mul_t(f, v.im)};
}
__device__ __forceinline__ Cx<float> scale_cx(Cx<float> v, float f) {
    const float2 r = __fmul2_rn(make_float2(f, f), make_float2(v.re, v.im));
    return Cx<float>{r.x, r.y};
}

// Rotation pair (src/cpucartesian.cpp:149-153 real, :210-214 imaginary):
// `first` is the lower-index cell of the pair, `second` the higher one.
// (-b) x is -(b x) exactly, so signs move onto the coefficient.
template <bool IMAG, typename T>
__device__ __forceinline__ Cx<T> rot_first(Cx<T> f, Cx<T> s, T a, T b) {
    return IMAG ? pair_cross(f, s, a, -b) : pair_direct(f, s, a, b);
}

template <bool IMAG, typename T>
__device__ __forceinline__ Cx<T> rot_second(Cx<T> s, Cx<T> f, T a, T b) {
    return IMAG ? pair_cross(s, f, a, b) : pair_direct(s, f, a, -b);
}

template <typename T>
__device__ __forceinline__ Cx<T> shfl_down1(Cx<T> v) {
    Cx<T> r;
    r.re = __shfl_down_sync(0xffffffffu, v.re, 1);
    r.im = __shfl_down_sync(0xffffffffu, v.im, 1);
    return r;
}

template <typename T>
__device__ __forceinline__ Cx<T> shfl_up1(Cx<T> v) {
    Cx<T> r;
    r.re = __shfl_up_sync(0xffffffffu, v.re, 1);
    r.im = __shfl_up_sync(0xffffffffu, v.im, 1);
    return r;
}

// Per-lane masks of a strip (which cells exist, which horizontal pairs are live).
template <int C>
struct LaneMask {
    bool pair_int[C];  // pair (i, i+1) inside the lane, both cells in the tile
    bool pair_left;    // pair (lane-1 cell C-1, cell 0) exists
    bool pair_right;   // pair (cell C-1, lane+1 cell 0) exists
};

// Vertical kinetic sweep on rows (u, u+1): cells with (x + u) % 2 == s pair,
// i.e. lane cells with (i & 1) == PAR where PAR = (u + s) & 1 (strips start
// on an even column).
template <bool IMAG, int C, int PAR, typename T>
__device__ __forceinline__ void vsweep(Cx<T> (&up)[C], Cx<T> (&lo)[C], T a, T b) {
#pragma unroll
    for (int i = PAR; i < C; i += 2) {
        Cx<T> u = up[i], l = lo[i];
        up[i] = kin<IMAG>(u, l, a, b);
        lo[i] = kin<IMAG>(l, u, a, b);
    }
}

// Horizontal kinetic sweep on one row: pairs (x, x+1) with (x + u) % 2 == s
// start at lane cells with (i & 1) == PAR, PAR = (u + s) & 1.  Only strips
// that touch the tile edge (EDGE) mask pairs: in an interior strip the cells
// of lanes 0 and 31 are recomputed halo that is never stored, so their
// missing partners do not matter.
template <bool IMAG, int C, int PAR, bool EDGE, typename T>
__device__ __forceinline__ void hsweep(Cx<T> (&w)[C], T a, T b, const LaneMask<C> &m) {
    if (PAR == 0) {
#pragma unroll
        for (int i = 0; i + 1 < C; i += 2) {
            Cx<T> p = w[i], q = w[i + 1];
            Cx<T> np = kin<IMAG>(p, q, a, b), nq = kin<IMAG>(q, p, a, b);
            w[i] = (!EDGE || m.pair_int[i]) ? np : p;
            w[i + 1] = (!EDGE || m.pair_int[i]) ? nq : q;
        }
    } else {
        Cx<T> right = shfl_down1(w[0]);
        Cx<T> left = shfl_up1(w[C - 1]);
#pragma unroll
        for (int i = 1; i + 1 < C; i += 2) {
            Cx<T> p = w[i], q = w[i + 1];
            Cx<T> np = kin<IMAG>(p, q, a, b), nq = kin<IMAG>(q, p, a, b);
            w[i] = (!EDGE || m.pair_int[i]) ? np : p;
            w[i + 1] = (!EDGE || m.pair_int[i]) ? nq : q;
        }
        Cx<T> n0 = kin<IMAG>(w[0], left, a, b);
        Cx<T> nl = kin<IMAG>(w[C - 1], right, a, b);
        if (!EDGE || m.pair_left) w[0] = n0;
        if (!EDGE || m.pair_right) w[C - 1] = nl;
    }
}

// Horizontal kinetic sweep with per-lane pair coefficients (2 cells per
// lane): (ai, bi) for the pair inside the lane, (al, bl) for the pair with the
// left neighbour lane, (ar, br) for the pair with the right one.  A pair whose
// partner lies outside the tile carries the identity, (1, 0) ((0, 0) in delta
// form), so one code path serves edge and interior strips alike.
template <bool IMAG, int PAR, typename T>
__device__ __forceinline__ void hsweep_lane(Cx<T> (&w)[2], T ai, T bi, T al, T bl, T ar, T br) {
    if (PAR == 0) {
        const Cx<T> p = w[0], q = w[1];
        w[0] = kin<IMAG>(p, q, ai, bi);
        w[1] = kin<IMAG>(q, p, ai, bi);
    } else {
        const Cx<T> right = shfl_down1(w[0]);
        const Cx<T> left = shfl_up1(w[1]);
        w[0] = kin<IMAG>(w[0], left, al, bl);
        w[1] = kin<IMAG>(w[1], right, ar, br);
    }
}

// Radial kinetic sweep (src/cpucylindrical.cpp:4-81) on one row, 2 cells per
// lane: the pair (x, x+1) with x = PAR (mod 2) updates its first cell with
// (a, b) and its second with (a, c); (a0, b0) and (a1, b1) are the
// coefficients of this lane's cells 0 and 1 for the sweep's parity.
template <bool IMAG, int PAR, typename T>
__device__ __forceinline__ void rsweep_lane(Cx<T> (&w)[2], T a0, T b0, T a1, T b1) {
    if (PAR == 0) {
        const Cx<T> p = w[0], q = w[1];
        w[0] = kin<IMAG>(p, q, a0, b0);
        w[1] = kin<IMAG>(q, p, a1, b1);
    } else {
        const Cx<T> right = shfl_down1(w[0]);
        const Cx<T> left = shfl_up1(w[1]);
        w[0] = kin<IMAG>(w[0], left, a0, b0);
        w[1] = kin<IMAG>(w[1], right, a1, b1);
    }
}

// The same for C cells per lane: (pa[i], pb[i]) for the pair (i, i+1) inside
// the lane, (al, bl) / (ar, br) for the pairs with the neighbour lanes.
template <bool IMAG, int PAR, int C, typename T>
__device__ __forceinline__ void hsweep_lanes(Cx<T> (&w)[C], const T (&pa)[C - 1],
                                             const T (&pb)[C - 1], T al, T bl, T ar, T br) {
    if (PAR == 0) {
#pragma unroll
        for (int i = 0; i + 1 < C; i += 2) {
            const Cx<T> p = w[i], q = w[i + 1];
            w[i] = kin<IMAG>(p, q, pa[i], pb[i]);
            w[i + 1] = kin<IMAG>(q, p, pa[i], pb[i]);
        }
    } else {
        const Cx<T> right = shfl_down1(w[0]);
        const Cx<T> left = shfl_up1(w[C - 1]);
#pragma unroll
        for (int i = 1; i + 1 < C; i += 2) {
            const Cx<T> p = w[i], q = w[i + 1];
            w[i] = kin<IMAG>(p, q, pa[i], pb[i]);
            w[i + 1] = kin<IMAG>(q, p, pa[i], pb[i]);
        }
        w[0] = kin<IMAG>(w[0], left, al, bl);
        w[C - 1] = kin<IMAG>(w[C - 1], right, ar, br);
    }
}

// Rotation row sweep on one row: pairs (x, x+1) with x % 2 == PAR.
template <bool IMAG, int C, int PAR, bool EDGE, typename T>
__device__ __forceinline__ void rrow(Cx<T> (&w)[C], T a, T b, const LaneMask<C> &m) {
    if (PAR == 0) {
#pragma unroll
        for (int i = 0; i + 1 < C; i += 2) {
            Cx<T> f = w[i], s = w[i + 1];
            Cx<T> nf = rot_first<IMAG>(f, s, a, b), ns = rot_second<IMAG>(s, f, a, b);
            w[i] = (!EDGE || m.pair_int[i]) ? nf : f;
            w[i + 1] = (!EDGE || m.pair_int[i]) ? ns : s;
        }
    } else {
        Cx<T> right = shfl_down1(w[0]);
        Cx<T> left = shfl_up1(w[C - 1]);
#pragma unroll
        for (int i = 1; i + 1 < C; i += 2) {
            Cx<T> f = w[i], s = w[i + 1];
            Cx<T> nf = rot_first<IMAG>(f, s, a, b), ns = rot_second<IMAG>(s, f, a, b);
            w[i] = (!EDGE || m.pair_int[i]) ? nf : f;
            w[i + 1] = (!EDGE || m.pair_int[i]) ? ns : s;
        }
        Cx<T> n0 = rot_second<IMAG>(w[0], left, a, b);
        Cx<T> nl = rot_first<IMAG>(w[C - 1], right, a, b);
        if (!EDGE || m.pair_left) w[0] = n0;
        if (!EDGE || m.pair_right) w[C - 1] = nl;
    }
}

// Rotation column sweep on rows (u, u+1) (every column pairs; u has the sweep's parity).
template <bool IMAG, int C, typename T>
__device__ __forceinline__ void rcol(Cx<T> (&up)[C], Cx<T> (&lo)[C], const Cx<T> (&ab)[C]) {
#pragma unroll
    for (int i = 0; i < C; ++i) {
        Cx<T> f = up[i], s = lo[i];
        up[i] = rot_first<IMAG>(f, s, ab[i].re, ab[i].im);
        lo[i] = rot_second<IMAG>(s, f, ab[i].re, ab[i].im);
    }
}

// Library paths for large phase arguments: kept out of line so that the
// unrolled row loop does not carry copies of them.
static __device__ __noinline__ void sincos_t(double x, double *s, double *c) { sincos(x, s, c); }
static __device__ __noinline__ void sincos_t(float x, float *s, float *c) { sincosf(x, s, c); }
static __device__ __noinline__ double exp_t(double x) { return exp(x); }
static __device__ __noinline__ double sin_t(double x) { return sin(x); }
static __device__ __noinline__ float sin_t(float x) { return sinf(x); }
static __device__ __noinline__ float exp_t(float x) { return expf(x); }
__device__ __forceinline__ double sqrt_t(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_t(float x) { return sqrtf(x); }

// Phase factors of the GPE / LHY term for small arguments.  The nonlinear
// phase g*dt*|psi|^2 is far below 1/32 in practice, where truncated Maclaurin
// series of cos, sin and exp (Horner's rule) leave a remainder well under half
// an ulp; larger arguments take the CUDA math library.  Two tiers, chosen for
// the whole warp:
//   |th| < 2^-8: double cos / sin to the t^3 terms (t = th^2), exp to x^6
//                (remainders below 3e-21; Estrin's scheme, a shorter
//                dependency chain than Horner's); float cos / sin to t^2,
//                exp to x^4 (below 1e-14);
//   |th| < 1/32: cos / sin to t^5, exp to x^8 (remainders below 1e-19).
// Returns sin(th) and cos(th) (cos(th) - 1 in delta form).  The comparisons
// are exact in either precision.
__device__ __forceinline__ bool phase_tiny(double th) { return fabs(th) < 0.00390625; }
__device__ __forceinline__ bool phase_tiny(float th) { return fabsf(th) < 0.00390625f; }
__device__ __forceinline__ bool phase_small(double th) { return fabs(th) < 0.03125; }
__device__ __forceinline__ bool phase_small(float th) { return fabsf(th) < 0.03125f; }

// TIERS = false: the 1/32 tier and the library only (less code, for the
// kernels whose row body is long enough for instruction fetch to limit them).
template <typename T, bool TIERS = true>
__device__ __forceinline__ void phase_sincos(T th, T *s, T *c) {
    constexpr bool F = std::is_same<T, float>::value;
    // warp-uniform choice: the shorter series if every lane allows it, the
    // library path only if some lane needs it
    if (TIERS && !__any_sync(0xffffffffu, !phase_tiny(th))) {
        const T t = th * th;
        if (F) {
            const T pc = fma_t(T(4.1666666666666664e-02), t, T(-0.5));               // 1/4!, -1/2!
            const T ps = fma_t(T(8.3333333333333332e-03), t, T(-1.6666666666666666e-01));  // 1/5!, -1/3!
            *c = DeltaForm<T>::value ? mul_t(pc, t) : fma_t(pc, t, T(1));
            *s = fma_t(mul_t(ps, t), th, th);
        } else {
            // Estrin's scheme (two levels instead of Horner's three):
            // cos = (1 - t/2!) + t^2 (1/4! - t/6!),
            // sin = th + (th t) ((-1/3! + t/5!) - t^2/7!)
            const T t2 = mul_t(t, t);
            const T c0 = fma_t(t, T(-0.5), T(1));
            const T c1 = fma_t(t, T(-1.3888888888888889e-03), T(4.1666666666666664e-02));
            const T s0 = fma_t(t, T(8.3333333333333332e-03), T(-1.6666666666666666e-01));
            const T ps = fma_t(t2, T(-1.9841269841269841e-04), s0);
            *c = fma_t(c1, t2, c0);
            *s = fma_t(mul_t(th, t), ps, th);
        }
    } else if (!__any_sync(0xffffffffu, !phase_small(th))) {
        const T t = th * th;
        T pc = T(-2.7557319223985893e-07);            // -1/10!
        pc = fma_t(pc, t, T(2.4801587301587302e-05));  //  1/8!
        pc = fma_t(pc, t, T(-1.3888888888888889e-03)); // -1/6!
        pc = fma_t(pc, t, T(4.1666666666666664e-02));  //  1/4!
        pc = fma_t(pc, t, T(-0.5));                    // -1/2!
        T ps = T(-2.5052108385441720e-08);             // -1/11!
        ps = fma_t(ps, t, T(2.7557319223985888e-06));  //  1/9!
        ps = fma_t(ps, t, T(-1.9841269841269841e-04)); // -1/7!
        ps = fma_t(ps, t, T(8.3333333333333332e-03));  //  1/5!
        ps = fma_t(ps, t, T(-1.6666666666666666e-01)); // -1/3!
        *c = DeltaForm<T>::value ? mul_t(pc, t) : fma_t(pc, t, T(1));
        *s = fma_t(mul_t(ps, t), th, th);
    } else {
        sincos_t(th, s, c);
        if (DeltaForm<T>::value) {
            // cos(th) - 1 = -2 sin^2(th / 2), without cancellation
            const T h = sin_t(T(0.5) * th);
            *c = T(-2) * h * h;
        }
    }
}

// exp(-th) for the imaginary-time nonlinear factor (same tiers).
template <typename T, bool TIERS = true>
__device__ __forceinline__ T phase_expneg(T th) {
    constexpr bool F = std::is_same<T, float>::value;
    if (TIERS && !__any_sync(0xffffffffu, !phase_tiny(th))) {
        const T x = -th;
        if (F) {
            T p = fma_t(T(4.1666666666666664e-02), x, T(1.6666666666666666e-01));  // 1/4!, 1/3!
            p = fma_t(p, x, T(0.5));  // 1/2!
            p = fma_t(p, x, T(1));
            return fma_t(p, x, T(1));
        }
        // Estrin's scheme (three levels instead of Horner's seven):
        // (1 + x + x^2/2! + x^3/3!) + x^4 (1/4! + x/5! + x^2/6!)
        const T x2 = mul_t(x, x);
        const T x4 = mul_t(x2, x2);
        const T a0 = x + T(1);
        const T a1 = fma_t(x, T(1.6666666666666666e-01), T(0.5));
        const T b0 = fma_t(x, T(8.3333333333333332e-03), T(4.1666666666666664e-02));
        const T lo = fma_t(a1, x2, a0);
        const T hi = fma_t(x2, T(1.3888888888888889e-03), b0);
        return fma_t(hi, x4, lo);
    }
    if (!__any_sync(0xffffffffu, !phase_small(th))) {
        const T x = -th;
        T p = T(2.4801587301587302e-05);             // 1/8!
        p = fma_t(p, x, T(1.9841269841269841e-04)); // 1/7!
        p = fma_t(p, x, T(1.3888888888888889e-03)); // 1/6!
        p = fma_t(p, x, T(8.3333333333333332e-03)); // 1/5!
        p = fma_t(p, x, T(4.1666666666666664e-02)); // 1/4!
        p = fma_t(p, x, T(1.6666666666666666e-01)); // 1/3!
        p = fma_t(p, x, T(0.5));                    // 1/2!
        p = fma_t(p, x, T(1));
        return fma_t(p, x, T(1));
    }
    return exp_t(-th);
}

// exp(-th0), exp(-th1) of two single-precision cells: the series of both in
// one packed pair, each cell with the roundings of phase_expneg.
template <bool TIERS = true>
__device__ __forceinline__ float2 phase_expneg2(float th0, float th1) {
    if (TIERS && !__any_sync(0xffffffffu, !(phase_tiny(th0) && phase_tiny(th1)))) {
        const float2 x = make_float2(-th0, -th1);
        constexpr double k[4] = {1.6666666666666666e-01, 0.5, 1.0, 1.0};
        float2 p = make_float2(float(4.1666666666666664e-02), float(4.1666666666666664e-02));
#pragma unroll
        for (int j = 0; j < 4; ++j) p = __ffma2_rn(p, x, make_float2(float(k[j]), float(k[j])));
        return p;
    }
    if (!__any_sync(0xffffffffu, !(phase_small(th0) && phase_small(th1)))) {
        const float2 x = make_float2(-th0, -th1);
        constexpr double k[8] = {1.9841269841269841e-04, 1.3888888888888889e-03,
                                 8.3333333333333332e-03, 4.1666666666666664e-02,
                                 1.6666666666666666e-01, 0.5, 1.0, 1.0};
        float2 p = make_float2(float(2.4801587301587302e-05), float(2.4801587301587302e-05));
#pragma unroll
        for (int j = 0; j < 8; ++j) p = __ffma2_rn(p, x, make_float2(float(k[j]), float(k[j])));
        return p;
    }
    return make_float2(phase_expneg<float, TIERS>(th0), phase_expneg<float, TIERS>(th1));
}

// sin(a) and cos(a) - 1 for |a| <= 1/16 from their Maclaurin series (Horner's
// rule in a^2).  With the last terms a^9/9! and a^10/10! the truncation error
// is below 2^-64 relative, and a, -a^2/2 carry the leading bits exactly, so
// both are within about half an ulp of the true values: no range reduction
// and a few FMAs instead of a full sincos.
constexpr double kSmallAngle = 0.0625;
__device__ inline void small_angle_sincos(double a, double *s, double *cm1) {
    const double a2 = a * a;
    double ps = 1.0 / 362880.0;  // 1/9!
    ps = fma(ps, a2, -1.0 / 5040.0);
    ps = fma(ps, a2, 1.0 / 120.0);
    ps = fma(ps, a2, -1.0 / 6.0);
    *s = fma(a * a2, ps, a);
    double pc = -1.0 / 3628800.0;  // -1/10!
    pc = fma(pc, a2, 1.0 / 40320.0);
    pc = fma(pc, a2, -1.0 / 720.0);
    pc = fma(pc, a2, 1.0 / 24.0);
    pc = fma(pc, a2, -0.5);
    *cm1 = a2 * pc;
}

// The FP64 real-time table entry exp(-i ang), ang = dt V: (cos, -sin), the
// series for small angles (src/solver.cpp:74-109 tabulates the same with
// std::exp(complex)).
__device__ inline Cx<double> vpot_table_entry(double ang) {
    double s;
    if (fabs(ang) <= kSmallAngle) {
        double cm1;
        small_angle_sincos(ang, &s, &cm1);
        return Cx<double>{1.0 + cm1, -s};
    }
    double c;
    sincos(ang, &s, &c);
    return Cx<double>{c, -s};
}

template <typename T>
struct Vec2T;
template <>
struct Vec2T<double> {
    using type = double2;
};
template <>
struct Vec2T<float> {
    using type = float2;
};

template <typename T>
__device__ __forceinline__ Cx<T> ld_cx_shared(const Cx<T> *p) {
    typename Vec2T<T>::type v = *reinterpret_cast<const typename Vec2T<T>::type *>(p);
    Cx<T> r;
    r.re = v.x;
    r.im = v.y;
    return r;
}

template <typename T>
__device__ __forceinline__ void st_cx_global(Cx<T> *p, Cx<T> v) {
    typename Vec2T<T>::type o;
    o.x = v.re;
    o.y = v.im;
    *reinterpret_cast<typename Vec2T<T>::type *>(p) = o;
}

// Rabi rotation of one cell (src/cpucartesian.cpp:264-290, real time):
// cc * self + (sr + i si) * other, cc - 1 in delta form.
template <typename T>
__device__ __forceinline__ Cx<T> rabi_cell(Cx<T> self, Cx<T> other, T cc, T sr, T si) {
    Cx<T> r;
    r.re = lin(cc, self.re, fma_t(sr, other.re, -mul_t(si, other.im)));
    r.im = lin(cc, self.im, fma_t(sr, other.im, mul_t(si, other.re)));
    return r;
}

// Potential, GPE and LHY phase on one row (src/cpucartesian.cpp:96-106,130-134).
// |psi|^2 is taken before the table multiply, as the reference does.
// PB (two components): the phase adds g_ab dt |psi_b|^2, psi_b the other
// species' cell at the start of this step (`ub`, already scaled)
// (src/cpucartesian.cpp:73-92,113-126).
template <bool IMAG, bool PHASE, bool LHY, bool PB, int C, bool TIERS = true, typename T,
          typename TabT>
__device__ __forceinline__ void potential_row(Cx<T> (&w)[C], const TabT *tab, T ca, T caa,
                                              const Cx<T> (*ub)[C] = nullptr, T cab = T(0)) {
    if constexpr (IMAG && PHASE && std::is_same<T, float>::value && C % 2 == 0) {
        // single precision: the factors of two cells at a time in packed pairs
        T th[C];
#pragma unroll
        for (int i = 0; i < C; ++i) {
            const Cx<T> v = w[i];
            const T n2 = fma_t(v.re, v.re, mul_t(v.im, v.im));
            th[i] = mul_t(ca, n2);
            if (LHY) th[i] = fma_t(caa, mul_t(n2, sqrt_t(n2)), th[i]);
            if (PB) {
                const Cx<T> u = (*ub)[i];
                th[i] = th[i] + mul_t(cab, fma_t(u.re, u.re, mul_t(u.im, u.im)));
            }
        }
#pragma unroll
        for (int i = 0; i < C; i += 2) {
            const float2 pr = make_float2(reinterpret_cast<const T *>(tab)[i],
                                          reinterpret_cast<const T *>(tab)[i + 1]);
            const float2 f = __fmul2_rn(phase_expneg2<TIERS>(th[i], th[i + 1]), pr);
            w[i] = scale_cx(w[i], f.x);
            w[i + 1] = scale_cx(w[i + 1], f.y);
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < C; ++i) {
        Cx<T> v = w[i];
        T thb = T(0);
        if (PB) {
            const Cx<T> u = (*ub)[i];
            thb = mul_t(cab, fma_t(u.re, u.re, mul_t(u.im, u.im)));
        }
        if (IMAG) {
            const T pr = reinterpret_cast<const T *>(tab)[i];
            if (PHASE) {
                const T n2 = fma_t(v.re, v.re, mul_t(v.im, v.im));
                T th = mul_t(ca, n2);
                if (LHY) th = fma_t(caa, mul_t(n2, sqrt_t(n2)), th);
                if (PB) th = th + thb;
                v = scale_cx(v, mul_t(phase_expneg<T, TIERS>(th), pr));
            } else {
                v = scale_cx(v, pr);
            }
        } else {
            const Cx<T> e = reinterpret_cast<const Cx<T> *>(tab)[i];
            T c = DeltaForm<T>::value ? T(0) : T(1), s = T(0);
            if (PHASE) {
                const T n2 = fma_t(v.re, v.re, mul_t(v.im, v.im));
                T th = mul_t(ca, n2);
                if (LHY) th = fma_t(caa, mul_t(n2, sqrt_t(n2)), th);
                if (PB) th = th + thb;
                phase_sincos<T, TIERS>(th, &s, &c);
            }
            // the table holds (cos, sin) of -dt V; in delta form (cos - 1, sin):
            // v (cos + i sin), the kinetic pair's form with the cell as its own
            // partner; the phase multiplies by (c - i s)
            v = kin<false>(v, v, e.re, e.im);
            if (PHASE) v = kin<false>(v, v, c, -s);
        }
        w[i] = v;
    }
}


// Compile-time description of a kernel variant.
// PHASE & 3: 0 no nonlinear phase, 1 g|psi|^2 only, 2 with the Lee-Huang-Yang
// term, 3 g|psi|^2 + g_ab|psi_b|^2 (one component of a two-component system);
// PHASE & 4: cylindrical lattice (radial kinetic sweeps, mirrored axis column);
// PHASE & 8 (with 3, real time): the Rabi rotation of the previous step
// applied to both species' cells as they are loaded.
template <typename T_, int C_, bool IMAG_, bool ROT_, int PHASE_>
struct Variant {
    using T = T_;
    static constexpr int C = C_;
    static constexpr bool IMAG = IMAG_;
    static constexpr bool ROT = ROT_;
    static constexpr bool PHASE = (PHASE_ & 3) != 0;
    static constexpr bool LHY = (PHASE_ & 3) == 2;
    static constexpr bool PB = (PHASE_ & 3) == 3;
    static constexpr bool CYL = (PHASE_ & 4) != 0;
    static constexpr bool RABI = (PHASE_ & 8) != 0;
    static_assert(!RABI || (PB && !IMAG_ && !CYL), "Rabi loads: two components, real time");
    // PHASE & 16: the table's entries made in the step from a potential V
    // (FP64, real time, cartesian, one component): the ring carries rows of
    // V, one double per cell, and the potential stage forms exp(-i dt V)
    // as the table kernel does
    static constexpr bool VPOT = (PHASE_ & 16) != 0;
    static_assert(!VPOT || (!IMAG_ && !ROT_ && (PHASE_ & 12) == 0 && (PHASE_ & 3) != 3 &&
                            std::is_same<T_, double>::value),
                  "potential rows: double, real time, cartesian, one component");
    // recomputed halo columns: one per horizontal pair sweep of the step
    // (4 kinetic; 4 more rotation row sweeps or radial sweeps)
    static constexpr int HX = (ROT_ || (PHASE_ & 4)) ? 8 : 4;
    static constexpr int HY = ROT_ ? 6 : 4;
    // Register window (rows); the body is unrolled over two windows so that
    // the parity of every row index is a compile-time constant.
    static constexpr int NWIN = ROT_ ? 7 : 5;
    static constexpr int UNROLL = 2 * NWIN;
    static constexpr int OUT_LAG = NWIN - 1;
    static constexpr int SW = 32 * C_;
    static constexpr int WO = SW - 2 * HX;
    // Per-lane horizontal coefficients instead of edge masks (no second,
    // masked copy of the row body): variants with 2 cells per lane and no
    // rotating frame.
    static constexpr bool LANE_COEF = !ROT_;
    // Resident blocks of 4 warps per SM the register allocation aims at.  The
    // default launch runs 4 blocks per SM (balanced tasks, fewer and taller
    // segments); a cap of 4 lets the compiler keep ~90 registers in double,
    // which schedules the row body better (46 vs 54 us per 2048^2 step than
    // the 80-register cap of 6 blocks); float keeps a cap of 6.
    static constexpr int MIN_BLOCKS =
        LANE_COEF ? (C_ == 2 ? (sizeof(T_) == 4 ? 6 : 4) : (sizeof(T_) == 4 ? 4 : 2)) : 4;
    // The batched kernel runs many tasks per warp: more resident warps (6
    // blocks in double, 8 in float: 80 / 64 registers) hide more latency.
    static constexpr int BATCH_MIN_BLOCKS = LANE_COEF ? (sizeof(T_) == 4 ? 8 : 6) : 4;  // C = 2
    using TabT = typename std::conditional<IMAG_ || VPOT, T_, Cx<T_>>::type;
    static constexpr int PSI_BYTES = SW * (int)sizeof(Cx<T_>);
    static constexpr int TAB_BYTES = SW * (int)sizeof(TabT);
    // a slot: one row of psi, of the table and (PB) of the other species
    static constexpr int SLOT = PSI_BYTES + TAB_BYTES + (PB ? PSI_BYTES : 0);
};


// Per-warp state of one segment walk.  Every member is indexed with
// compile-time constants after inlining, so the whole struct lives in
// registers.  Ring slots are tracked incrementally: row ra of a segment goes
// to slot 0, row ra+1 to slot 1, ...; the parity each slot's mbarrier will
// show next is kept in phase_bits (bit q for slot q) across segments.
template <class V>
struct Walk {
    using T = typename V::T;
    using TabT = typename V::TabT;
    static constexpr int C = V::C, NWIN = V::NWIN;

    Cx<T> win[NWIN][C];
    Cx<T> colab[C];
    LaneMask<C> m;
    bool present[C], out_col[C], norm_col[C];
    int ra, rb, oy0, oy1, xl, lane, D;
    int lslot;            // slot of the next row to load
    int tslot;            // slot of the row whose table is read next
    uint32_t phase_bits;  // expected completion parity of each slot
    int issued_to;        // rows [ra, issued_to) have had their copy issued
    int loaded_to;        // rows [ra, loaded_to) have been waited for
    const unsigned char *gpsi, *gtab;  // row 0, column cs of psi and of the table
    const unsigned char *gpb;          // PB: row 0, column cs of the other species
    size_t gpsi_pitch, gtab_pitch;
    uint32_t psi_off, psi_bytes, tab_off, tab_bytes;
    unsigned char *ring;
    uint64_t *bars;
    double nacc;
    bool failed;
    T inv;
    T aH, bH, aV, bV, ca, caa;  // step constants, read from the parameters once
    T pbs, cab;                 // PB: factor of the other species' tile, g_ab * dt
    T rcc, rsr, rsi, ror, roi;  // RABI: rotation of the own and of the other cell
    T rca[2][2], rcb[2][2];     // CYL: radial (a, b_self) of cell [i] for parity [p]
    T msign;                    // CYL, imaginary time: mirror sign on the lane of column 0
    T hpa[C - 1], hpb[C - 1];        // LANE_COEF: this lane's pairs (i, i+1)
    T hal, hbl, har, hbr;            //   and its pairs with the neighbour lanes

    __device__ __forceinline__ void issue(int row, int slot) {
        unsigned char *sb = ring + slot * V::SLOT;
        mbar_expect_tx(&bars[slot], psi_bytes + tab_bytes + (V::PB ? psi_bytes : 0u));
        bulk_g2s(sb + psi_off, gpsi + (size_t)row * gpsi_pitch, psi_bytes, &bars[slot]);
        bulk_g2s(sb + V::PSI_BYTES + tab_off, gtab + (size_t)row * gtab_pitch, tab_bytes,
                 &bars[slot]);
        if constexpr (V::PB)
            bulk_g2s(sb + V::PSI_BYTES + V::TAB_BYTES + psi_off, gpb + (size_t)row * gpsi_pitch,
                     psi_bytes, &bars[slot]);
    }
    __device__ __forceinline__ int next(int q) const { return q + 1 == D ? 0 : q + 1; }
};

// Horizontal sweep of one window row, PAR the pair parity.
template <class V, int PAR, bool EDGE>
__device__ __forceinline__ void hsw(Walk<V> &w, Cx<typename V::T> (&row)[V::C]) {
    if constexpr (V::LANE_COEF) {
        hsweep_lanes<V::IMAG, PAR, V::C>(row, w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
    } else {
        hsweep<V::IMAG, V::C, PAR, EDGE>(row, w.aH, w.bH, w.m);
    }
}

// Zero the parts of this warp's ring slots that the current task's copies do
// not cover (strips that reach past the row), so that cells outside the tile
// read as 0 without a per-row mask.
template <class V>
__device__ __forceinline__ void zero_ring_outside(Walk<V> &w) {
    uint32_t *ring32 = reinterpret_cast<uint32_t *>(w.ring);
    const int words = w.D * V::SLOT / 4;
    for (int i = w.lane; i < words; i += 32) {
        const uint32_t off = (uint32_t)(i * 4) % (uint32_t)V::SLOT;
        bool copied;
        if (off < (uint32_t)V::PSI_BYTES) {
            copied = off >= w.psi_off && off < w.psi_off + w.psi_bytes;
        } else if (off < (uint32_t)(V::PSI_BYTES + V::TAB_BYTES)) {
            const uint32_t t = off - (uint32_t)V::PSI_BYTES;
            copied = t >= w.tab_off && t < w.tab_off + w.tab_bytes;
        } else {
            const uint32_t t = off - (uint32_t)(V::PSI_BYTES + V::TAB_BYTES);
            copied = t >= w.psi_off && t < w.psi_off + w.psi_bytes;
        }
        if (!copied) ring32[i] = 0u;
    }
}

// One iteration of the walk for row r = base + K (base even, so the parity of
// every row index below is known at compile time).
// GUARD: the iteration may touch rows outside [ra, rb) (segment prologue and
// epilogue); without it every stage is known to be valid.  EDGE: the strip
// touches the tile edge and needs the per-lane masks.
template <class V, int K, bool GUARD, bool EDGE>
__device__ __forceinline__ void walk_row(Walk<V> &w, const StepArgs<typename V::T> &a, int r) {
    using T = typename V::T;
    using TabT = typename V::TabT;
    constexpr int C = V::C, NWIN = V::NWIN;
    constexpr bool IMAG = V::IMAG, ROT = V::ROT, PHASE = V::PHASE;
    // row r - j lives in win[(K - j) mod NWIN]
#define WS(j) w.win[((K) - (j) + 2 * NWIN) % NWIN]
    const int ra = w.ra, rb = w.rb;
    const T aH = w.aH, bH = w.bH, aV = w.aV, bV = w.bV;

    // ---- load row r
    if (!GUARD || (r >= ra && r < rb)) {
        const int q = w.lslot;
        if (!mbar_wait_bounded(&w.bars[q], (w.phase_bits >> q) & 1u)) {
            w.failed = true;
            return;
        }
        w.phase_bits ^= 1u << q;
        w.lslot = w.next(q);
        w.loaded_to = r + 1;
        const Cx<T> *sp = reinterpret_cast<const Cx<T> *>(w.ring + q * V::SLOT) + C * w.lane;
#pragma unroll
        for (int i = 0; i < C; ++i) {
            Cx<T> v = ld_cx_shared(sp + i);
            if constexpr (V::RABI) {
                const Cx<T> *bp = reinterpret_cast<const Cx<T> *>(w.ring + q * V::SLOT +
                                                                  V::PSI_BYTES + V::TAB_BYTES) +
                                  C * w.lane;
                Cx<T> u = ld_cx_shared(bp + i);
                v = rabi_cell(v, scale_cx(u, w.pbs), w.rcc, w.rsr, w.rsi);
            }
            if (IMAG) v = scale_cx(v, w.inv);
            WS(0)[i] = (!EDGE || w.present[i]) ? v : Cx<T>{T(0), T(0)};
        }
    }
    // ---- S1: V0 on rows (r-1, r)
    if (!GUARD || (r - 1 >= ra && r < rb)) vsweep<IMAG, C, ((K + 1) & 1)>(WS(1), WS(0), aV, bV);
    // ---- S2: H0 on row r-1
    if (!GUARD || (r - 1 >= ra && r - 1 < rb)) hsw<V, ((K + 1) & 1), EDGE>(w, WS(1));
    // ---- S3: V1 on rows (r-2, r-1)
    if (!GUARD || (r - 2 >= ra && r - 1 < rb)) vsweep<IMAG, C, ((K + 1) & 1)>(WS(2), WS(1), aV, bV);
    // ---- S4: H1, P, then H1 (or the rotation row sweeps) on row r-2; free its slot
    if (!GUARD || (r - 2 >= ra && r - 2 < rb)) {
        const int u = r - 2;
        hsw<V, ((K + 1) & 1), EDGE>(w, WS(2));
        if constexpr (V::CYL) {
            rsweep_lane<IMAG, 0>(WS(2), w.rca[0][0], w.rcb[0][0], w.rca[0][1], w.rcb[0][1]);
            rsweep_lane<IMAG, 1>(WS(2), w.rca[1][0], w.rcb[1][0], w.rca[1][1], w.rcb[1][1]);
        }
        const int q = w.tslot;
        const TabT *tp =
            reinterpret_cast<const TabT *>(w.ring + q * V::SLOT + V::PSI_BYTES) + C * w.lane;
        if constexpr (V::PB) {
            const Cx<T> *bp = reinterpret_cast<const Cx<T> *>(w.ring + q * V::SLOT +
                                                              V::PSI_BYTES + V::TAB_BYTES) +
                              C * w.lane;
            Cx<T> ub[C];
#pragma unroll
            for (int i = 0; i < C; ++i) {
                Cx<T> u = scale_cx(ld_cx_shared(bp + i), w.pbs);
                if constexpr (V::RABI) {
                    // the other species rotated from the cells this row started from
                    const Cx<T> o = ld_cx_shared(
                        reinterpret_cast<const Cx<T> *>(w.ring + q * V::SLOT) + C * w.lane + i);
                    u = rabi_cell(u, o, w.rcc, w.ror, w.roi);
                }
                ub[i] = u;
            }
            potential_row<IMAG, PHASE, false, true, C, false>(WS(2), tp, w.ca, w.caa, &ub, w.cab);
        } else {
            potential_row<IMAG, PHASE, V::LHY, false, C>(WS(2), tp, w.ca, w.caa);
        }
        if constexpr (ROT) {
            const Cx<T> ab = reinterpret_cast<const Cx<T> *>(a.row_ab)[u];
            rrow<IMAG, C, 0, EDGE>(WS(2), ab.re, ab.im, w.m);
            rrow<IMAG, C, 1, EDGE>(WS(2), ab.re, ab.im, w.m);
        } else {
            if constexpr (V::CYL) {
                rsweep_lane<IMAG, 1>(WS(2), w.rca[1][0], w.rcb[1][0], w.rca[1][1], w.rcb[1][1]);
                rsweep_lane<IMAG, 0>(WS(2), w.rca[0][0], w.rcb[0][0], w.rca[0][1], w.rcb[0][1]);
            }
            hsw<V, ((K + 1) & 1), EDGE>(w, WS(2));
        }
        __syncwarp();
        if (u + w.D < rb) {
            if (w.lane == 0) {
                // the slot's last generic-proxy reads happen-before the bulk copy refills it
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                w.issue(u + w.D, q);
            }
            w.issued_to = u + w.D + 1;
        }
        w.tslot = w.next(q);
    }
    if constexpr (!ROT) {
        // ---- S5: V1 on rows (r-3, r-2)
        if (!GUARD || (r - 3 >= ra && r - 2 < rb)) vsweep<IMAG, C, ((K) & 1)>(WS(3), WS(2), aV, bV);
        // ---- S6: H0 on row r-3
        if (!GUARD || (r - 3 >= ra && r - 3 < rb)) hsw<V, ((K + 1) & 1), EDGE>(w, WS(3));
        // ---- S7: V0 on rows (r-4, r-3)
        if (!GUARD || (r - 4 >= ra && r - 3 < rb)) vsweep<IMAG, C, ((K) & 1)>(WS(4), WS(3), aV, bV);
    } else {
        // ---- S5: rotation columns, even rows: pair (r-3, r-2) when r-3 is even
        if (((K + 1) & 1) == 0 && (!GUARD || (r - 3 >= ra && r - 2 < rb))) rcol<IMAG, C>(WS(3), WS(2), w.colab);
        // ---- S6: rotation columns, odd rows: pair (r-4, r-3) when r-4 is odd
        if (((K) & 1) == 1 && (!GUARD || (r - 4 >= ra && r - 3 < rb))) rcol<IMAG, C>(WS(4), WS(3), w.colab);
        // ---- S7: rotation rows again, then H1, on row r-4
        if (!GUARD || (r - 4 >= ra && r - 4 < rb)) {
            const Cx<T> ab = reinterpret_cast<const Cx<T> *>(a.row_ab)[r - 4];
            rrow<IMAG, C, 0, EDGE>(WS(4), ab.re, ab.im, w.m);
            rrow<IMAG, C, 1, EDGE>(WS(4), ab.re, ab.im, w.m);
            hsw<V, ((K + 1) & 1), EDGE>(w, WS(4));
        }
        // ---- S8: V1 on rows (r-5, r-4)
        if (!GUARD || (r - 5 >= ra && r - 4 < rb)) vsweep<IMAG, C, ((K) & 1)>(WS(5), WS(4), aV, bV);
        // ---- S9: H0 on row r-5
        if (!GUARD || (r - 5 >= ra && r - 5 < rb)) hsw<V, ((K + 1) & 1), EDGE>(w, WS(5));
        // ---- S10: V0 on rows (r-6, r-5)
        if (!GUARD || (r - 6 >= ra && r - 5 < rb)) vsweep<IMAG, C, ((K) & 1)>(WS(6), WS(5), aV, bV);
    }
    // ---- store the finished row r - (NWIN-1)
    {
        const int u = r - (NWIN - 1);
        if (u >= w.oy0 && u < w.oy1) {
            Cx<T> *orow = reinterpret_cast<Cx<T> *>(a.psi_out) + (size_t)u * a.P + w.xl;
            const bool norm_row = IMAG && u >= a.iy0 && u < a.iy1;
            if constexpr (V::CYL && IMAG) {
                // column 0 mirrors column 1 (src/cpukernel.cpp:669-689); msign is
                // 0 on every other lane
                if (w.msign != T(0)) {
                    WS(NWIN - 1)[0].re = w.msign * WS(NWIN - 1)[1].re;
                    WS(NWIN - 1)[0].im = w.msign * WS(NWIN - 1)[1].im;
                }
            }
#pragma unroll
            for (int i = 0; i < C; ++i) {
                const Cx<T> v = WS(NWIN - 1)[i];
                if (w.out_col[i]) st_cx_global(orow + i, v);
                if (norm_row && w.norm_col[i])
                    w.nacc += (double)v.re * (double)v.re + (double)v.im * (double)v.im;
            }
        }
    }
#undef WS
}

template <class V, int K, bool GUARD, bool EDGE>
__device__ __forceinline__ void walk_rows(Walk<V> &w, const StepArgs<typename V::T> &a, int base,
                                          int rlast) {
    if constexpr (K < V::UNROLL) {
        const int r = base + K;
        if ((GUARD && r > rlast) || w.failed) return;
        walk_row<V, K, GUARD, EDGE>(w, a, r);
        walk_rows<V, K + 1, GUARD, EDGE>(w, a, base, rlast);
    }
}

// Walk one segment in chunks of UNROLL rows.  With SPLIT, chunks whose rows
// are all inside the segment and past the window's fill run a copy of the
// body without the per-stage row checks.  The single-tile kernel splits in
// real time (2048^2 FP32: 51 -> 45 us per step, FP64: 55 -> 53 us); in
// imaginary time (FP64: 46 -> 52 us) and in the batched kernel (FP64 -8 %,
// FP32 -14 %) the second copy of the body made the step slower.
template <class V, bool EDGE, bool SPLIT>
__device__ __forceinline__ void walk_segment(Walk<V> &w, const StepArgs<typename V::T> &a) {
    const int rlast = w.rb - 1 + V::OUT_LAG;
    for (int base = w.ra & ~1; base <= rlast && !w.failed; base += V::UNROLL) {
        if constexpr (SPLIT) {
            if (base >= w.ra + V::NWIN - 1 && base + V::UNROLL <= w.rb) {
                walk_rows<V, 0, false, EDGE>(w, a, base, rlast);
                continue;
            }
        }
        walk_rows<V, 0, true, EDGE>(w, a, base, rlast);
    }
}

// ------------------------------------------------------------ task pieces
// Per-warp set-up shared by the single-tile and the batched kernels: this
// warp's ring slots (D of them) and their mbarriers.
template <class V>
__device__ __forceinline__ void warp_setup(Walk<V> &w, unsigned char *smem, int warps, int warp,
                                           int lane, int D) {
    w.nacc = 0.0;
    w.failed = false;
    w.D = D;
    w.lane = lane;
    // each warp: D ring slots, then (after all warps' rings) D mbarriers
    w.ring = smem + (size_t)warp * D * V::SLOT;
    w.bars = reinterpret_cast<uint64_t *>(smem + (size_t)warps * D * V::SLOT) + warp * D;
    w.phase_bits = 0u;
    // Zero this warp's ring once: cells never written by a copy (outside the
    // tile) are then finite, so masked-off pair updates cannot produce NaNs.
    {
        uint4 *z = reinterpret_cast<uint4 *>(w.ring);
        const int n16 = D * V::SLOT / 16;
        for (int i = lane; i < n16; i += 32) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (lane == 0) {
        for (int q = 0; q < D; ++q) mbar_init(&w.bars[q], 1);
        fence_mbar_init();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
}

// The step constants of one tile.  In FP32 real time the kinetic
// coefficients come from a per-step schedule: float pairs rounded with the
// carried error of the previous steps (sigma-delta), so that the coefficient
// error summed over any run of steps stays within half an ulp instead of
// growing with the step count (a fixed float pair would rotate every step
// by the same wrong angle and scale the norm by the same factor).
template <class V>
__device__ __forceinline__ void bind_args(Walk<V> &w, const StepArgs<typename V::T> &a) {
    using T = typename V::T;
    w.inv = V::IMAG ? (T)a.scal->pending_inv : T(1);
    w.aH = a.aH;
    w.bH = a.bH;
    w.aV = a.aV;
    w.bV = a.bV;
    if constexpr (DeltaForm<T>::value && !V::IMAG) {
        if (a.kin_sched) {
            const unsigned int step = __ldcg(&a.scal->step);
            const float4 c = __ldg(&a.kin_sched[step % (unsigned int)a.sched_len]);
            w.aH = c.x;
            w.bH = c.y;
            w.aV = c.z;
            w.bV = c.w;
        }
    }
    w.ca = a.ca;
    w.caa = a.caa;
    if constexpr (V::PB) {
        w.pbs = (T)__ldcg(a.pb_scale);
        w.cab = a.cab;
    }
    if constexpr (V::RABI) {
        w.rcc = a.rabi_cc;
        w.rsr = a.rabi_sr;
        w.rsi = a.rabi_si;
        w.ror = a.rabi_or;
        w.roi = a.rabi_oi;
    }
    w.gpsi_pitch = (size_t)a.P * sizeof(Cx<T>);
    w.gtab_pitch = (size_t)a.P * sizeof(typename V::TabT);
}

// One task of a tile: strip x segment `task`, interior strips first.
template <class V, bool SPLIT>
__device__ __forceinline__ void run_task(Walk<V> &w, const StepArgs<typename V::T> &a, int task) {
    using T = typename V::T;
    using TabT = typename V::TabT;
    constexpr int C = V::C, NWIN = V::NWIN, HX = V::HX, HY = V::HY, SW = V::SW, WO = V::WO;
    constexpr bool ROT = V::ROT;
    const int lane = w.lane;
    const int D = w.D;
    // tasks of interior strips come first and those of the first and last
    // strip (the only ones that need masks) last, so that few SMs run both
    // code paths
    int strip, seg;
    {
        const int n_int = a.n_strips > 2 ? (a.n_strips - 2) * a.n_segs : 0;
        if (task < n_int) {
            strip = 1 + task % (a.n_strips - 2);
            seg = task / (a.n_strips - 2);
        } else {
            const int e = task - n_int;
            const int n_edge_strips = a.n_strips > 2 ? 2 : a.n_strips;
            const int es = e % n_edge_strips;
            strip = (a.n_strips > 2 && es == 1) ? a.n_strips - 1 : es;
            seg = e / n_edge_strips;
        }
    }
    const int ox0 = strip * WO, ox1 = min(ox0 + WO, a.W);
    const int c0 = ox0 - HX;
    segment_rows(a, seg, w.oy0, w.oy1);
    w.ra = max(w.oy0 - HY, 0);
    w.rb = min(w.oy1 + HY, a.H);
    const int cs = max(c0, 0);
    const int ce = min(c0 + SW, a.P);
    w.psi_off = (uint32_t)(cs - c0) * sizeof(Cx<T>);
    w.psi_bytes = (uint32_t)(ce - cs) * sizeof(Cx<T>);
    w.tab_off = (uint32_t)(cs - c0) * sizeof(TabT);
    w.tab_bytes = (uint32_t)(ce - cs) * sizeof(TabT);
    w.gpsi = reinterpret_cast<const unsigned char *>(a.psi_in) + (size_t)cs * sizeof(Cx<T>);
    w.gtab = reinterpret_cast<const unsigned char *>(a.pot) + (size_t)cs * sizeof(TabT);
    if constexpr (V::PB)
        w.gpb = reinterpret_cast<const unsigned char *>(a.pb) + (size_t)cs * sizeof(Cx<T>);
    w.xl = c0 + C * lane;
#pragma unroll
    for (int i = 0; i < C; ++i) {
        const int x = w.xl + i;
        w.present[i] = x >= 0 && x < a.W;
        w.out_col[i] = x >= ox0 && x < ox1;
        w.norm_col[i] = w.out_col[i] && x >= a.ix0 && x < a.ix1;
    }
#pragma unroll
    for (int i = 0; i + 1 < C; ++i) w.m.pair_int[i] = w.present[i] && w.present[i + 1];
    w.m.pair_int[C - 1] = false;
    w.m.pair_left = lane > 0 && w.present[0] && w.xl - 1 >= 0;
    w.m.pair_right = lane < 31 && w.present[C - 1] && w.xl + C < a.W;
    if constexpr (V::LANE_COEF) {
        const T one = DeltaForm<T>::value ? T(0) : T(1);
#pragma unroll
        for (int i = 0; i + 1 < C; ++i) {
            w.hpa[i] = w.m.pair_int[i] ? w.aH : one;
            w.hpb[i] = w.m.pair_int[i] ? w.bH : T(0);
        }
        w.hal = w.m.pair_left ? w.aH : one;
        w.hbl = w.m.pair_left ? w.bH : T(0);
        w.har = w.m.pair_right ? w.aH : one;
        w.hbr = w.m.pair_right ? w.bH : T(0);
    }
    if constexpr (ROT) {
#pragma unroll
        for (int i = 0; i < C; ++i)
            w.colab[i] = reinterpret_cast<const Cx<T> *>(a.col_ab)[w.present[i] ? w.xl + i : 0];
    }
    if constexpr (V::CYL) {
        // pair starting at column x: valid when x >= 0 and x + 1 < W
        const T one = DeltaForm<T>::value ? T(0) : T(1);
        const Cx<T> *rad = reinterpret_cast<const Cx<T> *>(a.rad);  // (a, b), (c, 0) per column
        auto pair_ok = [&](int x) { return x >= 0 && x + 1 < a.W; };
        const int x0 = w.xl;
        // parity 0: cells 0, 1 pair with each other (pair at x0)
        const bool p0 = pair_ok(x0);
        w.rca[0][0] = p0 ? rad[2 * x0].re : one;
        w.rcb[0][0] = p0 ? rad[2 * x0].im : T(0);
        w.rca[0][1] = w.rca[0][0];
        w.rcb[0][1] = p0 ? rad[2 * x0 + 1].re : T(0);
        // parity 1: cell 0 is the second cell of the pair at x0 - 1, cell 1 the
        // first of the pair at x0 + 1
        const bool pl = pair_ok(x0 - 1), pr = pair_ok(x0 + 1);
        w.rca[1][0] = pl ? rad[2 * (x0 - 1)].re : one;
        w.rcb[1][0] = pl ? rad[2 * (x0 - 1) + 1].re : T(0);
        w.rca[1][1] = pr ? rad[2 * (x0 + 1)].re : one;
        w.rcb[1][1] = pr ? rad[2 * (x0 + 1)].im : T(0);
        w.msign = (V::IMAG && x0 == 0) ? a.mirror_sign : T(0);
    }
#pragma unroll
    for (int j = 0; j < NWIN; ++j)
#pragma unroll
        for (int i = 0; i < C; ++i) w.win[j][i] = Cx<T>{T(0), T(0)};

    w.lslot = 0;
    w.tslot = 0;
    w.loaded_to = w.ra;
    w.issued_to = min(w.ra + D, w.rb);
    __syncwarp();  // the previous task's reads of the ring are done
    if constexpr (V::LANE_COEF) {
        if (c0 < 0 || c0 + SW > a.P) {
            zero_ring_outside(w);
            __syncwarp();
        }
    }
    if (lane == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int row = w.ra; row < w.issued_to; ++row) w.issue(row, row - w.ra);
    }

    if constexpr (V::LANE_COEF) {
        walk_segment<V, false, SPLIT>(w, a);
    } else {
        if (c0 >= 0 && c0 + SW <= a.W) walk_segment<V, false, SPLIT>(w, a);
        else walk_segment<V, true, SPLIT>(w, a);
    }

    if (w.failed) {
        if (lane == 0) atomicExch(&a.scal->error, 1);
        // let copies already issued land before the block can exit
        int q = w.lslot;
        for (int row = w.loaded_to; row < w.issued_to; ++row) {
            (void)mbar_wait_bounded(&w.bars[q], (w.phase_bits >> q) & 1u, 100000000ull);
            w.phase_bits ^= 1u << q;
            q = w.next(q);
        }
    }
}

// Grid: any number of blocks of 1..4 warps; each warp loops over the tasks
// (strip, segment) t = warp_global, warp_global + total_warps, ...
template <class V>
__global__ void __launch_bounds__(128, V::MIN_BLOCKS) step_kernel(StepArgs<typename V::T> a) {
    constexpr bool IMAG = V::IMAG;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warps = blockDim.x >> 5;
    // broadcast from lane 0 so that the compiler knows the warp index, and
    // every task quantity derived from it, to be warp-uniform
    const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const int lane = threadIdx.x & 31;
    const int n_tasks = a.n_strips * a.n_segs;

    Walk<V> w;
    warp_setup(w, smem, warps, warp, lane, a.ring);
    bind_args(w, a);
    for (int task = blockIdx.x * warps + warp; task < n_tasks && !w.failed;
         task += gridDim.x * warps)
        run_task<V, !IMAG && !V::PB>(w, a, task);

    if constexpr (!IMAG && DeltaForm<typename V::T>::value) {
        // the last block to finish advances the schedule's step (every block
        // has read it: each takes a ticket only after its whole walk)
        if (a.kin_sched) {
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                unsigned int *tk = launch_ticket(a);
                if (atomicAdd(tk, 1u) == gridDim.x - 1) {
                    *tk = 0u;
                    if (step_ends_here(a)) a.scal->step += 1u;
                    __threadfence();
                }
            }
        }
    }

    if constexpr (IMAG) {
        // block partial: the block's warps in warp order (a warp's tasks in
        // task order); then the last block to finish sums the block partials
        // in a fixed order, eight independent loads in flight per thread.
        double nacc = w.nacc;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) nacc += __shfl_xor_sync(0xffffffffu, nacc, off);
        __shared__ double s_warp[4];
        __shared__ unsigned int s_last;
        __shared__ double red[128];
        if (lane == 0) s_warp[warp] = nacc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int i = 0; i < warps; ++i) b += s_warp[i];
            a.partials[blockIdx.x] = b;
            __threadfence();
            const unsigned int t = atomicAdd(launch_ticket(a), 1u);
            s_last = (t == gridDim.x - 1) ? 1u : 0u;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            const int nb = gridDim.x;
            double acc[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[j] = 0.0;
            for (int base = threadIdx.x; base < nb; base += 8 * (int)blockDim.x) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int t = base + j * (int)blockDim.x;
                    if (t < nb) acc[j] += __ldcg(&a.partials[t]);
                }
            }
            red[threadIdx.x] = ((acc[0] + acc[1]) + (acc[2] + acc[3])) +
                               ((acc[4] + acc[5]) + (acc[6] + acc[7]));
            __syncthreads();
            for (int h = blockDim.x >> 1; h > 0; h >>= 1) {
                if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
                __syncthreads();
            }
            if (threadIdx.x == 0) {
                double tot = red[0] * a.dxdy;
                *launch_ticket(a) = 0u;
                if constexpr (V::PB) {
                    a.scal->last_norm = tot;
                    // the other species' next step reads this step's input
                    // buffer with the factor that was pending on it
                    a.scal->prev_inv = a.scal->pending_inv;
                    // the kept norm moves with the joint normalisation: a
                    // species that started empty is renormalised once it has
                    // a share (src/cpukernel.cpp:551, norm[i] != 0)
                    const double n0 = a.scal->norm_target;
                    if (n0 != 0.0) a.scal->pending_inv = 1.0 / sqrt(tot / n0);
                } else if (split_norm_total(a, &tot)) {
                    a.scal->last_norm = tot;
                    if (a.scal->renorm) a.scal->pending_inv = 1.0 / sqrt(tot / a.norm0);
                    if (a.inv_copy) *a.inv_copy = a.scal->pending_inv;
                }
            }
        }
    }
}

// ------------------------------------------------------------------ batch
// Many tiles of uneven sizes advanced by one Trotter step in one launch: the
// tasks (strip x segment) of all tiles form one list that the persistent
// grid walks; each task binds its tile's buffers and constants.
template <typename T>
struct BatchArgs {
    const StepArgs<T> *inst;  // per tile: this step's buffers, constants and task geometry
    const int2 *tasks;        // (tile, task of the tile), tile-major
    double *task_norm;        // imaginary time: squared norm of each task's inner cells
    int *error;               // set when a bounded wait gives up
    int n_tasks;
    int ring;  // ring slots per warp (checked walk)
    int vlen;  // vertical pair table entries per warp (look-ahead walk)
};

template <typename X>
__device__ __forceinline__ X bcast0(X x) {
    return __shfl_sync(0xffffffffu, x, 0);
}
template <typename X>
__device__ __forceinline__ X *ldg_ptr(X *const *addr) {
    return reinterpret_cast<X *>(__ldg(reinterpret_cast<const unsigned long long *>(addr)));
}
template <typename X>
__device__ __forceinline__ X *bcast0_ptr(X *p) {
    return reinterpret_cast<X *>(__shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(p), 0));
}

// The tile's arguments as warp-uniform values (read by every lane from the
// same address, broadcast from lane 0 so that the compiler knows it).
template <typename T>
__device__ __forceinline__ StepArgs<T> load_tile_args(const StepArgs<T> *p) {
    StepArgs<T> a;
    a.psi_in = bcast0_ptr(ldg_ptr(&p->psi_in));
    a.psi_out = bcast0_ptr(ldg_ptr(&p->psi_out));
    a.pot = bcast0_ptr(ldg_ptr(&p->pot));
    a.row_ab = bcast0_ptr(ldg_ptr(&p->row_ab));
    a.col_ab = bcast0_ptr(ldg_ptr(&p->col_ab));
    a.W = bcast0(__ldg(&p->W));
    a.H = bcast0(__ldg(&p->H));
    a.P = bcast0(__ldg(&p->P));
    a.ix0 = bcast0(__ldg(&p->ix0));
    a.ix1 = bcast0(__ldg(&p->ix1));
    a.iy0 = bcast0(__ldg(&p->iy0));
    a.iy1 = bcast0(__ldg(&p->iy1));
    a.n_strips = bcast0(__ldg(&p->n_strips));
    a.n_segs = bcast0(__ldg(&p->n_segs));
    a.seg_h = bcast0(__ldg(&p->seg_h));
    a.ring = bcast0(__ldg(&p->ring));
    a.aH = bcast0(__ldg(&p->aH));
    a.bH = bcast0(__ldg(&p->bH));
    a.aV = bcast0(__ldg(&p->aV));
    a.bV = bcast0(__ldg(&p->bV));
    a.ca = bcast0(__ldg(&p->ca));
    a.caa = bcast0(__ldg(&p->caa));
    a.partials = nullptr;
    a.kin_sched = bcast0_ptr(ldg_ptr(&p->kin_sched));
    a.sched_len = bcast0(__ldg(&p->sched_len));
    a.scal = bcast0_ptr(ldg_ptr(&p->scal));
    a.dxdy = bcast0(__ldg(&p->dxdy));
    a.norm0 = bcast0(__ldg(&p->norm0));
    a.win_n0 = 0;
    a.ticket = nullptr;
    a.pair_norm = nullptr;
    a.pair_ticket = nullptr;
    a.inv_copy = nullptr;
    a.pot_pitch = 0;
    a.pot_dt = 0.0;
    return a;
}

template <class V>
__global__ void __launch_bounds__(128, V::BATCH_MIN_BLOCKS) batch_step_kernel(BatchArgs<typename V::T> b) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warps = blockDim.x >> 5;
    const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const int lane = threadIdx.x & 31;

    Walk<V> w;
    warp_setup(w, smem, warps, warp, lane, b.ring);
    for (int t = blockIdx.x * warps + warp; t < b.n_tasks && !w.failed; t += gridDim.x * warps) {
        const int2 it = __ldg(&b.tasks[t]);
        const int tile = bcast0(it.x), task = bcast0(it.y);
        const StepArgs<typename V::T> a = load_tile_args(b.inst + tile);
        bind_args(w, a);
        w.nacc = 0.0;
        run_task<V, false>(w, a, task);
        if constexpr (V::IMAG) {
            double n = w.nacc;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) n += __shfl_xor_sync(0xffffffffu, n, off);
            if (lane == 0) b.task_norm[t] = n;
        }
    }
    if (w.failed && lane == 0) atomicExch(b.error, 1);
}

}  // namespace tsb
