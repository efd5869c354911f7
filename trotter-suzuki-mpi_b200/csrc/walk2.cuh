// Streamed step without per-stage row checks ("look-ahead walk").
//
// Same work decomposition as step_kernel (a warp walks one strip of 32 x C
// columns down a segment of rows, keeping a register window of rows and
// running every stage of V0 H0 V1 H1 P H1 V1 H0 V0 one row behind the
// previous one), arranged so that the row body carries no row checks:
//
//   * The walk of a segment with output rows [oy0, oy1) visits the rows
//     oy0 - HY .. oy1 + HY - 1 (the HY vertical sweeps, 4, or 6 in a
//     rotating frame, spoil one row per sweep at each end of the walk, so
//     these halo rows absorb everything that happens beyond them).  Rows of the walk outside the tile are not copied: their
//     ring slot keeps an older row (finite values), which only ever meets a
//     tile row through a vertical pair across the tile edge, and those pairs
//     carry the identity (1, 0) from a per-warp table of pair coefficients
//     (src/cpucartesian.cpp:4-70 skips them: closed boundary).  Every other
//     stage needs no check at all.
//   * The walk stores row c - HY in the iteration that loads row c; with
//     the HY halo rows below the segment the last stored row is finished in
//     the iteration of the last loaded row, so there is no drain.
//   * Ring slots and window rows are compile-time indices: the body is
//     unrolled over NW rows (6; 8 in a rotating frame), which is the ring
//     depth and the window height (the window holds the row being loaded one
//     iteration ahead plus rows c .. c-HY), and even, so row parities are
//     compile-time as well.  The
//     mbarriers are re-initialised for every task, so their phases are
//     compile-time up to one bit per chunk.
//   * Loads run one row ahead: the iteration of row c waits for row c + 1
//     and moves it to registers while the stages of row c run, so the
//     shared-memory latency is off the stage chain.
//   * Or (R = 2) two rows per iteration: one ring slot and one mbarrier per
//     pair of rows, and the stages of both rows in one basic block, where
//     the second row's chain of stages runs one stage behind the first's
//     (row c + 1's V0 needs only row c's V0), so the two chains overlap.
//
// Variants: every one of step_kernel: cartesian (phases 0-2; 2 or 4 cells per
// lane, 2 in a double-precision rotating frame), one species of a pair
// (phases 3 and 7: the other species' rows ride in the ring, the Rabi
// rotation at load) and cylindrical lattices (phases 4-6: radial sweeps,
// the mirrored axis column at the store), both precisions and time modes.  The arithmetic of
// each cell is that of step_kernel (the same pair forms, potential row,
// rotation sweeps and reductions), so both give the same bits; the rotating
// frame's row and column rotations across the tile's edges take the identity
// as its vertical pairs do.
#pragma once
#include "step_kernel.cuh"
#include "walk2_shape.h"

namespace tsb {

template <class V, int R_ = 1>
struct W2Shape {
    static constexpr int C = V::C;
    static constexpr bool ROT = V::ROT;
    static constexpr int R = R_;               // rows per iteration (and per ring slot)
    // window rows: the row loaded ahead and rows c .. c-4 (c-6 in a rotating
    // frame, whose step has 6 vertical sweeps)
    static constexpr int NW = ROT ? 8 : 6;
    static constexpr int D = NW / R_;          // ring slots per warp
    static constexpr int UNROLL = NW;          // rows per unrolled chunk
    static constexpr bool CYL = V::CYL;
    // halo columns: one per horizontal sweep (4 kinetic, 4 more rotation row
    // or radial sweeps); halo rows: one per vertical sweep
    static constexpr int HX = (ROT || CYL) ? 8 : 4, HY = ROT ? 6 : 4;
    static constexpr int SO = 2 * HY;          // walk index of the first stored row
    // slot indices in flight ahead of the current one: the slot of row c-2
    // (whose table the current iteration reads) is refilled with row c-2+NW
    static constexpr int AHEAD = D - 2 / R_;
    static constexpr int SW = 32 * C, WO = SW - 2 * HX;
    // one row of psi and of the table (and, for one species of a pair, of
    // the other species' psi)
    static constexpr int ROWB = V::PSI_BYTES + V::TAB_BYTES + (V::PB ? V::PSI_BYTES : 0);
    static constexpr int PB_OFF = V::PSI_BYTES + V::TAB_BYTES;
    static constexpr int SLOT = R_ * ROWB;
    // vertical pair coefficients: entry j is the pair (u - 1, u) with
    // u = ra + j - VPAD; the first stages of a walk read up to VPAD - 1
    // entries before the first row
    static constexpr int VPAD = ROT ? 6 : 4;
    static_assert(V::HX == HX && (!ROT || V::C == 2 || sizeof(typename V::T) == 4),
                  "look-ahead walk geometry (4 cells per lane in a rotating frame: float)");
    static_assert((!CYL && !V::PB) || (V::C == 2 && !ROT && !(CYL && V::PB)),
                  "look-ahead walk: cylinder or pair with 2 cells per lane, no rotating frame");
    static_assert(R_ == 1 || R_ == 2, "one or two rows per iteration");
    static_assert(D * R == UNROLL && NW == UNROLL && UNROLL % 2 == 0,
                  "compile-time slots and parities");
};


__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

template <class V, int R = 1>
struct Walk2 {
    using T = typename V::T;
    using TabT = typename V::TabT;
    using S = W2Shape<V, R>;
    static constexpr int C = V::C;

    Cx<T> win[S::NW][C];
    T hpa[C - 1], hpb[C - 1];  // this lane's horizontal pairs (i, i+1)
    T hal, hbl, har, hbr;      // and its pairs with the neighbour lanes
    // rotating frame: this lane's column rotation coefficients, its pair
    // masks for the row rotation sweeps, the per-row coefficients
    Cx<T> colab[C];
    LaneMask<C> m;
    const Cx<T> *row_ab;
    // single precision: the row rotation coefficients of walk rows t-4 .. t-1
    // (row j in rab[j % 4]), each loaded two rows ahead of its first use
    // (measured 624 -> 600 us per 8192^2 step; in double the four registers
    // cost more than the loads: 967 -> 991 us)
    static constexpr bool AB_AHEAD = sizeof(T) == 4;
    Cx<T> rab[4];
    // cylindrical: radial (a, b) of cell [i] for the sweep of parity [p]; the
    // mirror sign on the lane of column 0 (imaginary time), else 0
    T rca[2][2], rcb[2][2];
    T msign;
    bool out_col[C], norm_col[C];
    bool partial_out;  // a pair of this lane's cells is cut by the output's edge
    int ra, nit, lane;
    int n_lo, n_hi;  // iterations whose stored row is in the norm region
    const unsigned char *gpsi, *gtab;  // row 0 of the strip's first copied column
    const unsigned char *gpb;          // pair: the other species' row 0, same column
    // the first row of the next slot to issue (slot indices advance by one
    // per issue); the walk indices [t_lo, t_lo + t_span) of copied rows (in
    // the tile and in the walk); row_tx: the bytes of one copied row
    const unsigned char *cpsi, *ctab, *cpb;
    uint32_t t_lo, t_span, row_tx;
    // pair: the other species' pending factor, g_ab dt; with the Rabi
    // rotation at load (real time) its coefficients for the own and the
    // other species' cell
    T pbs, cab;
    T rcc, rsr, rsi, ror, roi;
    size_t gpsi_pitch, gtab_pitch;
    uint32_t psi_off, psi_bytes, tab_off, tab_bytes;
    int H;
    unsigned char *ring;
    Cx<T> *vco;
    uint64_t *bars;
    Cx<T> *orow;  // row oy0 - 8 of the output at this lane's first column (moved per row)
    size_t opitch;  // output row pitch in cells
    double nacc;
    bool failed;
    int fail_idx;  // ring slot index (rows R * fail_idx ..) whose wait gave up
    T inv;
    T aH, bH, aV, bV, ca, caa;
    T vdt;  // potential rows (phase bit 16): dt

    // copy the rows of slot index `si` of the walk (rows R si .. R si + R - 1)
    // into ring slot q; rows outside the tile or past the walk are not
    // copied, and a slot without any row completes its phase by a plain
    // arrive.  Lane 0 issues, through predicates (no divergent branch in the
    // row body).  Slot indices are issued in order, one more per call, so
    // the copy addresses advance from the walk's first row; a walk index tp
    // is a copied row when t_lo <= tp < t_lo + t_span.  In a rotating frame
    // the addresses are computed from the row instead: loop-carried pointers
    // took the double kernel from 158 to 174 registers, 2 blocks per SM
    // instead of 3 (1182 against 1039 us per 8192^2 step).
    __device__ __forceinline__ void issue(int si, int q) {
        const uint32_t sb = smem_u32(ring + q * S::SLOT);
        const uint32_t bar = smem_u32(&bars[q]);
        uint32_t p[R], n = 0;
        const unsigned char *src_psi[R], *src_tab[R];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const bool real = (uint32_t)(R * si + k - t_lo) < t_span;
            p[k] = (lane == 0 && real) ? 1u : 0u;
            n += real ? 1u : 0u;
            if constexpr (S::ROT) {
                const int rr = real ? ra + R * si + k : 0;
                src_psi[k] = gpsi + (size_t)rr * gpsi_pitch;
                src_tab[k] = gtab + (size_t)rr * gtab_pitch;
            } else {
                src_psi[k] = cpsi + k * gpsi_pitch;
                src_tab[k] = ctab + k * gtab_pitch;
            }
        }
        const uint32_t pc = (lane == 0 && n > 0) ? 1u : 0u;
        const uint32_t pa = (lane == 0 && n == 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred pc, pa;\n\t"
            "setp.ne.u32 pc, %0, 0;\n\t"
            "setp.ne.u32 pa, %1, 0;\n\t"
            "@pc mbarrier.arrive.expect_tx.shared::cta.b64 _, [%2], %3;\n\t"
            "@pa mbarrier.arrive.shared::cta.b64 _, [%2];\n\t}" ::"r"(pc),
            "r"(pa), "r"(bar), "r"(n * row_tx)
            : "memory");
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t rb = sb + (uint32_t)(k * S::ROWB);
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.u32 p, %0, 0;\n\t"
                "@p cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%1], [%2], %3, [%4];\n\t"
                "@p cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%5], [%6], %7, [%4];\n\t}" ::"r"(p[k]),
                "r"(rb + psi_off), "l"(src_psi[k]), "r"(psi_bytes), "r"(bar),
                "r"(rb + (uint32_t)V::PSI_BYTES + tab_off), "l"(src_tab[k]), "r"(tab_bytes)
                : "memory");
            if constexpr (V::PB)
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.u32 p, %0, 0;\n\t"
                    "@p cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%1], [%2], %3, [%4];\n\t}" ::"r"(p[k]),
                    "r"(rb + (uint32_t)S::PB_OFF + psi_off), "l"(cpb + k * gpsi_pitch), "r"(psi_bytes),
                    "r"(bar)
                    : "memory");
        }
        if constexpr (!S::ROT) {
            cpsi += R * gpsi_pitch;
            ctab += R * gtab_pitch;
            if constexpr (V::PB) cpb += R * gpsi_pitch;
        }
    }
};

// Cells of this lane from a ring slot row (vector loads of 16 bytes).
template <typename T, int C>
__device__ __forceinline__ void load_row_cells(const unsigned char *p, Cx<T> (&v)[C]) {
    if constexpr (sizeof(T) == 4 && C % 2 == 0) {
#pragma unroll
        for (int i = 0; i < C; i += 2) {
            const float4 q = reinterpret_cast<const float4 *>(p)[i / 2];
            v[i] = Cx<T>{q.x, q.y};
            v[i + 1] = Cx<T>{q.z, q.w};
        }
    } else {
#pragma unroll
        for (int i = 0; i < C; ++i) v[i] = ld_cx_shared(reinterpret_cast<const Cx<T> *>(p) + i);
    }
}

// Table values of this lane from a ring slot row.
template <typename TabT, int C>
__device__ __forceinline__ void load_tab_cells(const unsigned char *p, TabT (&v)[C]) {
    constexpr int BYTES = C * (int)sizeof(TabT);
    if constexpr (BYTES % 16 == 0) {
        uint4 *d = reinterpret_cast<uint4 *>(v);
#pragma unroll
        for (int i = 0; i < BYTES / 16; ++i) d[i] = reinterpret_cast<const uint4 *>(p)[i];
    } else if constexpr (BYTES % 8 == 0) {
        uint2 *d = reinterpret_cast<uint2 *>(v);
#pragma unroll
        for (int i = 0; i < BYTES / 8; ++i) d[i] = reinterpret_cast<const uint2 *>(p)[i];
    } else {
#pragma unroll
        for (int i = 0; i < C; ++i) v[i] = reinterpret_cast<const TabT *>(p)[i];
    }
}

template <typename T, int C>
__device__ __forceinline__ void store_row_cells(Cx<T> *o, const Cx<T> (&v)[C],
                                                const bool (&in)[C], bool partial) {
    if constexpr (sizeof(T) == 4 && C % 2 == 0) {
        // a pair of cells in one 16-byte store where both are output cells
        // (predicated stores: no divergent branch at the strip's halo
        // lanes); with 4 cells per lane the single cells of a pair cut by
        // the tile's edge sit behind a branch that only such a lane takes
        // (8192^2 rotating-frame step about 1 % faster), with 2 they are
        // predicated as well (24.5 against 25.4 us per 2048^2 step)
#pragma unroll
        for (int i = 0; i < C; i += 2) {
            const bool both = in[i] && in[i + 1];
            if (both)
                reinterpret_cast<float4 *>(o)[i / 2] =
                    make_float4(v[i].re, v[i].im, v[i + 1].re, v[i + 1].im);
            if constexpr (C == 2) {
                if (in[i] && !both) st_cx_global(o + i, v[i]);
                if (in[i + 1] && !both) st_cx_global(o + i + 1, v[i + 1]);
            }
        }
        if constexpr (C > 2) {
            if (partial) {
#pragma unroll
                for (int i = 0; i < C; i += 2) {
                    if (in[i] && !in[i + 1]) st_cx_global(o + i, v[i]);
                    if (in[i + 1] && !in[i]) st_cx_global(o + i + 1, v[i + 1]);
                }
            }
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < C; ++i)
        if (in[i]) st_cx_global(o + i, v[i]);
}

// Rotating frame: the row rotation coefficients of tile row u (rows of the
// walk outside the tile take row 0's or row H-1's: their results never reach
// a tile row).
template <class V, int R>
__device__ __forceinline__ Cx<typename V::T> w2_row_ab(const Walk2<V, R> &w, int u) {
    u = u < 0 ? 0 : (u >= w.H ? w.H - 1 : u);
    return w.row_ab[u];
}

// Rotating frame: the column rotation sweep on rows (u - 1, u), the identity
// unless both rows are in the tile.
template <class V, int R>
__device__ __forceinline__ void w2_rcol(const Walk2<V, R> &w, Cx<typename V::T> (&up)[V::C],
                                        Cx<typename V::T> (&lo)[V::C], int u) {
    using T = typename V::T;
    const bool ok = u >= 1 && u < w.H;
    Cx<T> ab[V::C];
#pragma unroll
    for (int i = 0; i < V::C; ++i)
        ab[i] = ok ? w.colab[i] : Cx<T>{DeltaForm<T>::value ? T(0) : T(1), T(0)};
    rcol<V::IMAG, V::C>(up, lo, ab);
}

// The stages of current row c = ra + t (t = base + K, base a multiple of
// UNROLL): V0 H0 V1 (H1 P H1) V1 H0 V0 one row behind each other, then the
// store of the finished row c - 4; in a rotating frame V0 H0 V1 (H1 P R R)
// Rc Rc (R R H1) V1 H0 V0 (R: a row rotation sweep of parity 0 then 1, Rc:
// the column rotation sweeps on the pairs starting at even, then odd rows,
// src/cpucartesian.cpp:139-177), the store of row c - 6.
template <class V, int R, int K>
__device__ __forceinline__ void w2_stages(Walk2<V, R> &w, int t) {
    using T = typename V::T;
    using TabT = typename V::TabT;
    using S = W2Shape<V, R>;
    constexpr int C = V::C;
    constexpr bool IMAG = V::IMAG, PHASE = V::PHASE;
    // row c - j lives in win[(K - j) mod NW]
#define W2S(j) w.win[((K) - (j) + 2 * S::NW) % S::NW]
    const Cx<T> *vc = w.vco + t + S::VPAD;
    if constexpr (S::ROT) {
        const int c = w.ra + t;
        // ---- S1: V0 on rows (c-1, c)
        {
            const Cx<T> cv = vc[0];
            vsweep<IMAG, C, ((K + 1) & 1)>(W2S(1), W2S(0), cv.re, cv.im);
        }
        // ---- S2: H0 on row c-1
        hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(1), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
        // ---- S3: V1 on rows (c-2, c-1)
        {
            const Cx<T> cv = vc[-1];
            vsweep<IMAG, C, ((K + 1) & 1)>(W2S(2), W2S(1), cv.re, cv.im);
        }
        // ---- S4: H1, P and the row rotations on row c-2
        {
            constexpr int RT = (K + S::UNROLL - 2) % S::UNROLL;
            constexpr int q = RT / R, pos = RT % R;
            hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(2), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
            alignas(16) TabT tv[C];
            load_tab_cells<TabT, C>(w.ring + q * S::SLOT + pos * S::ROWB + V::PSI_BYTES +
                                        C * (int)sizeof(TabT) * w.lane,
                                    tv);
            potential_row<IMAG, PHASE, V::LHY, false, C>(W2S(2), tv, w.ca, w.caa);
            const Cx<T> ab = Walk2<V, R>::AB_AHEAD ? w.rab[(K + 2) % 4] : w2_row_ab(w, c - 2);
            rrow<IMAG, C, 0, true>(W2S(2), ab.re, ab.im, w.m);
            rrow<IMAG, C, 1, true>(W2S(2), ab.re, ab.im, w.m);
        }
        if constexpr ((K & 1) == 1) {
            // ---- S5: column rotations on rows (c-3, c-2), c-3 even
            w2_rcol(w, W2S(3), W2S(2), c - 2);
            // ---- S6: column rotations on rows (c-4, c-3), c-4 odd
            w2_rcol(w, W2S(4), W2S(3), c - 3);
        }
        // ---- S7: the row rotations again, then H1, on row c-4 (ahead: its
        // coefficients' register takes row c's, used two and four rows on)
        {
            constexpr bool AHEAD = Walk2<V, R>::AB_AHEAD;
            const Cx<T> ab = AHEAD ? w.rab[K % 4] : w2_row_ab(w, c - 4);
            rrow<IMAG, C, 0, true>(W2S(4), ab.re, ab.im, w.m);
            rrow<IMAG, C, 1, true>(W2S(4), ab.re, ab.im, w.m);
            hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(4), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
            if constexpr (AHEAD) w.rab[K % 4] = w2_row_ab(w, c);
        }
        // ---- S8: V1 on rows (c-5, c-4)
        {
            const Cx<T> cv = vc[-4];
            vsweep<IMAG, C, ((K) & 1)>(W2S(5), W2S(4), cv.re, cv.im);
        }
        // ---- S9: H0 on row c-5
        hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(5), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
        // ---- S10: V0 on rows (c-6, c-5)
        {
            const Cx<T> cv = vc[-5];
            vsweep<IMAG, C, ((K) & 1)>(W2S(6), W2S(5), cv.re, cv.im);
        }
    } else {
        // ---- S1: V0 on rows (c-1, c)
        {
            const Cx<T> cv = vc[0];
            vsweep<IMAG, C, ((K + 1) & 1)>(W2S(1), W2S(0), cv.re, cv.im);
        }
        // ---- S2: H0 on row c-1
        hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(1), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
        // ---- S3: V1 on rows (c-2, c-1)
        {
            const Cx<T> cv = vc[-1];
            vsweep<IMAG, C, ((K + 1) & 1)>(W2S(2), W2S(1), cv.re, cv.im);
        }
        // ---- S4: H1, P, H1 on row c-2 (its table from its ring slot); in a
        // cylinder the radial sweeps of both parities around P
        // (src/cpukernel.cpp:22-92 with src/cpucylindrical.cpp:4-81)
        {
            constexpr int RT = (K + S::UNROLL - 2) % S::UNROLL;  // row c-2 within the chunk
            constexpr int q = RT / R, pos = RT % R;
            hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(2), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
            if constexpr (S::CYL) {
                rsweep_lane<IMAG, 0>(W2S(2), w.rca[0][0], w.rcb[0][0], w.rca[0][1], w.rcb[0][1]);
                rsweep_lane<IMAG, 1>(W2S(2), w.rca[1][0], w.rcb[1][0], w.rca[1][1], w.rcb[1][1]);
            }
            const unsigned char *row = w.ring + q * S::SLOT + pos * S::ROWB;
            alignas(16) TabT tv[C];
            load_tab_cells<TabT, C>(row + V::PSI_BYTES + C * (int)sizeof(TabT) * w.lane, tv);
            if constexpr (V::PB) {
                // the other species' cells, scaled (and, with the Rabi
                // rotation at load, rotated with the cells this row started
                // from); the short phase tier left out as in step_kernel,
                // whose bits this walk keeps
                Cx<T> ub[C];
                load_row_cells<T, C>(row + S::PB_OFF + C * (int)sizeof(Cx<T>) * w.lane, ub);
                Cx<T> own[C];
                if constexpr (V::RABI) load_row_cells<T, C>(row + C * (int)sizeof(Cx<T>) * w.lane, own);
#pragma unroll
                for (int i = 0; i < C; ++i) {
                    ub[i] = scale_cx(ub[i], w.pbs);
                    if constexpr (V::RABI) ub[i] = rabi_cell(ub[i], own[i], w.rcc, w.ror, w.roi);
                }
                potential_row<IMAG, PHASE, false, true, C, false>(W2S(2), tv, w.ca, w.caa, &ub,
                                                                  w.cab);
            } else if constexpr (V::VPOT) {
                // the table's entries from the potential row, as the table
                // kernel forms them
                Cx<T> te[C];
#pragma unroll
                for (int i = 0; i < C; ++i) te[i] = vpot_table_entry(w.vdt * tv[i]);
                potential_row<IMAG, PHASE, V::LHY, false, C>(W2S(2), te, w.ca, w.caa);
            } else {
                potential_row<IMAG, PHASE, V::LHY, false, C>(W2S(2), tv, w.ca, w.caa);
            }
            if constexpr (S::CYL) {
                rsweep_lane<IMAG, 1>(W2S(2), w.rca[1][0], w.rcb[1][0], w.rca[1][1], w.rcb[1][1]);
                rsweep_lane<IMAG, 0>(W2S(2), w.rca[0][0], w.rcb[0][0], w.rca[0][1], w.rcb[0][1]);
            }
            hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(2), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
        }
        // ---- S5: V1 on rows (c-3, c-2)
        {
            const Cx<T> cv = vc[-2];
            vsweep<IMAG, C, ((K) & 1)>(W2S(3), W2S(2), cv.re, cv.im);
        }
        // ---- S6: H0 on row c-3
        hsweep_lanes<IMAG, ((K + 1) & 1), C>(W2S(3), w.hpa, w.hpb, w.hal, w.hbl, w.har, w.hbr);
        // ---- S7: V0 on rows (c-4, c-3)
        {
            const Cx<T> cv = vc[-3];
            vsweep<IMAG, C, ((K) & 1)>(W2S(4), W2S(3), cv.re, cv.im);
        }
    }
    // ---- row c-HY is finished: store it (the first 2 HY rows of a walk are halo;
    // with two rows per iteration the second row can lie past the walk)
    if (t >= S::SO && (R == 1 || t < w.nit)) {
        if constexpr (S::CYL && IMAG) {
            // column 0 mirrors column 1 (src/cpukernel.cpp:669-689); msign
            // is 0 on every other lane
            if (w.msign != T(0)) {
                W2S(S::HY)[0].re = w.msign * W2S(S::HY)[1].re;
                W2S(S::HY)[0].im = w.msign * W2S(S::HY)[1].im;
            }
        }
        store_row_cells<T, C>(w.orow, W2S(S::HY), w.out_col, w.partial_out);
        if (IMAG && t >= w.n_lo && t < w.n_hi) {
#pragma unroll
            for (int i = 0; i < C; ++i) {
                const Cx<T> v = W2S(S::HY)[i];
                if (w.norm_col[i])
                    w.nacc += (double)v.re * (double)v.re + (double)v.im * (double)v.im;
            }
        }
    }
    w.orow += w.opitch;
#undef W2S
}

// This lane's cells of row `pos` of ring slot q into window row `dst`.
template <class V, int R>
__device__ __forceinline__ void w2_load(Walk2<V, R> &w, int q, int pos,
                                        Cx<typename V::T> (&dst)[V::C]) {
    using T = typename V::T;
    using S = W2Shape<V, R>;
    constexpr int C = V::C;
    const unsigned char *row = w.ring + q * S::SLOT + pos * S::ROWB;
    Cx<T> v[C];
    load_row_cells<T, C>(row + C * (int)sizeof(Cx<T>) * w.lane, v);
    if constexpr (V::RABI) {
        // one species of a pair, real time: the Rabi rotation of the previous
        // step with the other species' cell of the same row
        Cx<T> u[C];
        load_row_cells<T, C>(row + S::PB_OFF + C * (int)sizeof(Cx<T>) * w.lane, u);
#pragma unroll
        for (int i = 0; i < C; ++i) v[i] = rabi_cell(v[i], scale_cx(u[i], w.pbs), w.rcc, w.rsr, w.rsi);
    }
#pragma unroll
    for (int i = 0; i < C; ++i) dst[i] = V::IMAG ? scale_cx(v[i], w.inv) : v[i];
}

// One iteration (row t = base + K with R = 1; rows t, t + 1 with R = 2, K
// even); ph is the chunk's mbarrier parity.
template <class V, int R, int K>
__device__ __forceinline__ void w2_iter(Walk2<V, R> &w, int t, uint32_t ph) {
    using S = W2Shape<V, R>;
#define W2S(j) w.win[((K) - (j) + 2 * S::NW) % S::NW]
    if constexpr (R == 1) {
        // look-ahead: wait for row t + 1 and move it to the window
        constexpr int q = (K + 1) % S::D;
        const uint32_t par = (K + 1 < S::D) ? ph : (ph ^ 1u);
        if (!mbar_wait_bounded(&w.bars[q], par)) {
            w.failed = true;
            w.fail_idx = t + 1;
            return;
        }
        w2_load(w, q, 0, W2S(-1));
        w2_stages<V, R, K>(w, t);
        // the slot of row t-2 is free: copy row t-2+NW into it
        constexpr int qi = (K + S::AHEAD) % S::D;
        __syncwarp();
        // the slot's generic-proxy reads happen-before the bulk copy refills it
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        w.issue(t + S::AHEAD, qi);
    } else {
        // rows t and t + 1 arrive together in slot K / 2
        constexpr int q = K / 2;
        if (!mbar_wait_bounded(&w.bars[q], ph)) {
            w.failed = true;
            w.fail_idx = t / 2;
            return;
        }
        w2_load(w, q, 0, W2S(0));
        w2_load(w, q, 1, W2S(-1));
        w2_stages<V, R, K>(w, t);
        w2_stages<V, R, K + 1>(w, t + 1);
        // the slot of rows t-2, t-1 is free: copy rows t-2+NW, t-1+NW into it
        constexpr int qi = (q + S::AHEAD) % S::D;
        __syncwarp();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        w.issue(t / 2 + S::AHEAD, qi);
    }
#undef W2S
}

template <class V, int R, int K>
__device__ __forceinline__ bool w2_rows(Walk2<V, R> &w, int base, uint32_t ph) {
    if constexpr (K < W2Shape<V, R>::UNROLL) {
        const int t = base + K;
        if (t >= w.nit) return false;
        w2_iter<V, R, K>(w, t, ph);
        if (w.failed) return false;
        return w2_rows<V, R, K + R>(w, base, ph);
    }
    return true;
}

// One task: strip x segment.  The first and last strips come first: their
// tasks start with extra set-up (clearing the ring bytes outside the tile),
// and the lowest task indices go to the blocks the SMs schedule first (the
// warp scheduler favours older blocks; tasks in the youngest blocks of an SM
// start and finish last).
template <class V, int R>
__device__ __forceinline__ void w2_task(Walk2<V, R> &w, const StepArgs<typename V::T> &a, int task) {
    using T = typename V::T;
    using TabT = typename V::TabT;
    using S = W2Shape<V, R>;
    constexpr int C = V::C;
    const int lane = w.lane;
    int strip, seg;
    {
        const int n_edge_strips = a.n_strips > 2 ? 2 : a.n_strips;
        const int n_edge = n_edge_strips * a.n_segs;
        if (task < n_edge) {
            const int es = task % n_edge_strips;
            strip = (a.n_strips > 2 && es == 1) ? a.n_strips - 1 : es;
            seg = task / n_edge_strips;
        } else {
            const int e = task - n_edge;
            strip = 1 + e % (a.n_strips - 2);
            seg = e / (a.n_strips - 2);
        }
    }
    const int ox0 = strip * S::WO, ox1 = min(ox0 + S::WO, a.W);
    const int c0 = ox0 - S::HX;
    int oy0, oy1;
    segment_rows(a, seg, oy0, oy1);
    w.ra = oy0 - S::HY;
    w.nit = (oy1 - oy0) + 2 * S::HY;
    w.n_lo = a.iy0 - oy0 + S::SO;
    w.n_hi = a.iy1 - oy0 + S::SO;
    const int cs = max(c0, 0);
    const int ce = min(c0 + S::SW, a.P);
    w.psi_off = (uint32_t)(cs - c0) * sizeof(Cx<T>);
    w.psi_bytes = (uint32_t)(ce - cs) * sizeof(Cx<T>);
    w.tab_off = (uint32_t)(cs - c0) * sizeof(TabT);
    // a potential's rows hold the tile's W columns only
    w.tab_bytes = (uint32_t)((V::VPOT ? min(ce, a.W) : ce) - cs) * sizeof(TabT);
    w.gpsi = reinterpret_cast<const unsigned char *>(a.psi_in) + (size_t)cs * sizeof(Cx<T>);
    w.gtab = reinterpret_cast<const unsigned char *>(a.pot) + (size_t)cs * sizeof(TabT);
    if constexpr (V::PB) w.gpb = reinterpret_cast<const unsigned char *>(a.pb) + (size_t)cs * sizeof(Cx<T>);
    // running copy addresses from the walk's first row (which may lie above
    // the tile: only rows inside it are ever read through them)
    w.cpsi = w.gpsi + (ptrdiff_t)w.ra * (ptrdiff_t)w.gpsi_pitch;
    w.ctab = w.gtab + (ptrdiff_t)w.ra * (ptrdiff_t)w.gtab_pitch;
    if constexpr (V::PB) w.cpb = w.gpb + (ptrdiff_t)w.ra * (ptrdiff_t)w.gpsi_pitch;
    {
        const int lo = max(0, -w.ra);               // the first walk row inside the tile
        const int hi = min(a.H - w.ra, w.nit);      // past the tile's last row and the walk's
        w.t_lo = (uint32_t)lo;
        w.t_span = (uint32_t)max(0, hi - lo);
    }
    w.row_tx = w.psi_bytes + w.tab_bytes + (V::PB ? w.psi_bytes : 0u);
    const int xl = c0 + C * lane;
    bool present[C];
#pragma unroll
    for (int i = 0; i < C; ++i) {
        const int x = xl + i;
        present[i] = x >= 0 && x < a.W;
        w.out_col[i] = x >= ox0 && x < ox1;
        w.norm_col[i] = w.out_col[i] && x >= a.ix0 && x < a.ix1;
    }
    w.partial_out = false;
#pragma unroll
    for (int i = 0; i + 1 < C; i += 2) {
        w.partial_out = w.partial_out || (w.out_col[i] != w.out_col[i + 1]);
    }
    {
        const T one = DeltaForm<T>::value ? T(0) : T(1);
#pragma unroll
        for (int i = 0; i + 1 < C; ++i) {
            const bool p = present[i] && present[i + 1];
            w.hpa[i] = p ? w.aH : one;
            w.hpb[i] = p ? w.bH : T(0);
        }
        const bool pl = lane > 0 && present[0] && xl - 1 >= 0;
        const bool pr = lane < 31 && present[C - 1] && xl + C < a.W;
        w.hal = pl ? w.aH : one;
        w.hbl = pl ? w.bH : T(0);
        w.har = pr ? w.aH : one;
        w.hbr = pr ? w.bH : T(0);
        if constexpr (S::CYL) {
            // radial pairs (x, x+1), valid when x >= 0 and x + 1 < W; the
            // table holds (a, b), (c, 0) per column x
            const Cx<T> *rad = reinterpret_cast<const Cx<T> *>(a.rad);
            auto pair_ok = [&](int x) { return x >= 0 && x + 1 < a.W; };
            // parity 0: cells 0, 1 pair with each other (pair at xl)
            const bool p0 = pair_ok(xl);
            w.rca[0][0] = p0 ? rad[2 * xl].re : one;
            w.rcb[0][0] = p0 ? rad[2 * xl].im : T(0);
            w.rca[0][1] = w.rca[0][0];
            w.rcb[0][1] = p0 ? rad[2 * xl + 1].re : T(0);
            // parity 1: cell 0 is the second cell of the pair at xl - 1,
            // cell 1 the first of the pair at xl + 1
            const bool q0 = pair_ok(xl - 1), q1 = pair_ok(xl + 1);
            w.rca[1][0] = q0 ? rad[2 * (xl - 1)].re : one;
            w.rcb[1][0] = q0 ? rad[2 * (xl - 1) + 1].re : T(0);
            w.rca[1][1] = q1 ? rad[2 * (xl + 1)].re : one;
            w.rcb[1][1] = q1 ? rad[2 * (xl + 1)].im : T(0);
            w.msign = (V::IMAG && xl == 0) ? a.mirror_sign : T(0);
        }
        if constexpr (S::ROT) {
            // the row rotation sweeps' pair masks and this lane's column
            // rotation coefficients
#pragma unroll
            for (int i = 0; i + 1 < C; ++i) w.m.pair_int[i] = present[i] && present[i + 1];
            w.m.pair_int[C - 1] = false;
            w.m.pair_left = pl;
            w.m.pair_right = pr;
#pragma unroll
            for (int i = 0; i < C; ++i)
                w.colab[i] = reinterpret_cast<const Cx<T> *>(a.col_ab)[present[i] ? xl + i : 0];
            // the row coefficients of the rows before the walk's first
            if constexpr (Walk2<V, R>::AB_AHEAD) {
#pragma unroll
                for (int j = 0; j < 4; ++j) w.rab[j] = w2_row_ab(w, w.ra - 4 + j);
            }
        }
        // vertical pairs (u - 1, u): the identity unless both rows are in the tile
        const int vl = w2_vlen(a.seg_h, S::ROT);
        for (int j = lane; j < vl; j += 32) {
            const int u = w.ra + j - S::VPAD;
            const bool ok = u >= 1 && u < a.H;
            w.vco[j] = ok ? Cx<T>{w.aV, w.bV} : Cx<T>{one, T(0)};
        }
    }
    w.orow = reinterpret_cast<Cx<T> *>(a.psi_out) + (ptrdiff_t)(oy0 - S::SO) * a.P + xl;
    __syncwarp();  // the previous task's reads of the ring are done
    if (c0 < 0 || c0 + S::SW > a.P) {
        // cells of the strip outside the tile read as 0 (copies do not cover them)
        uint32_t *ring32 = reinterpret_cast<uint32_t *>(w.ring);
        for (int i = lane; i < S::D * S::SLOT / 4; i += 32) {
            const uint32_t off = (uint32_t)(i * 4) % (uint32_t)S::ROWB;
            bool copied;
            if (off < (uint32_t)V::PSI_BYTES) {
                copied = off >= w.psi_off && off < w.psi_off + w.psi_bytes;
            } else if (off < (uint32_t)S::PB_OFF) {
                const uint32_t tt = off - (uint32_t)V::PSI_BYTES;
                copied = tt >= w.tab_off && tt < w.tab_off + w.tab_bytes;
            } else {
                const uint32_t tt = off - (uint32_t)S::PB_OFF;
                copied = tt >= w.psi_off && tt < w.psi_off + w.psi_bytes;
            }
            if (!copied) ring32[i] = 0u;
        }
    }
    __syncwarp();
    if (lane == 0) {
        // fresh barriers: every slot starts at phase 0 for this task
#pragma unroll
        for (int q = 0; q < S::D; ++q) {
            mbar_inval(&w.bars[q]);
            mbar_init(&w.bars[q], 1);
        }
        fence_mbar_init();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    // the first rows of the walk (slots 0 .. AHEAD-1)
    constexpr int PRE = S::AHEAD;
#pragma unroll
    for (int q = 0; q < PRE; ++q) w.issue(q, q);
    bool ok = true;
    if constexpr (R == 1) {
        // row 0 of the walk; the iterations load one row ahead
        ok = mbar_wait_bounded(&w.bars[0], 0u);
        if (!ok) {
            w.failed = true;
            w.fail_idx = 0;
        } else {
            w2_load(w, 0, 0, w.win[0]);
        }
    }
    if (ok) {
        for (int base = 0; !w.failed; base += S::UNROLL) {
            const uint32_t ph = (uint32_t)(base / S::UNROLL) & 1u;
            if (!w2_rows<V, R, 0>(w, base, ph)) break;
        }
    }
    if (w.failed) {
        if (lane == 0) atomicExch(&a.scal->error, 1);
        // let the copies still in flight land before the block can exit:
        // slots [0, PRE) were issued before the walk and one more by each
        // completed iteration (R = 1: iteration t waits for row t + 1 and
        // issues row t + AHEAD; R = 2: iteration k waits for pair k and
        // issues pair k + AHEAD); the wait for slot index fail_idx gave up
        const int issued_to =
            R == 1 ? max(PRE, w.fail_idx - 1 + S::AHEAD) : max(PRE, w.fail_idx + S::AHEAD);
        for (int j = w.fail_idx; j < issued_to; ++j)
            (void)mbar_wait_bounded(&w.bars[j % S::D], (uint32_t)(j / S::D) & 1u, 100000000ull);
    }
}

// The end of a step launch, shared with step_kernel: in FP32 real time the
// last block advances the coefficient schedule; in imaginary time the block
// partials of the squared norm are summed in a fixed order by the last block,
// which sets the renormalisation factor the next step applies.
template <class V>
__device__ __forceinline__ void w2_finish(const StepArgs<typename V::T> &a, double nacc, int warps,
                                          int warp, int lane) {
    if constexpr (!V::IMAG && DeltaForm<typename V::T>::value) {
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
    if constexpr (V::IMAG) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) nacc += __shfl_xor_sync(0xffffffffu, nacc, off);
        __shared__ double s_warp[32];
        __shared__ unsigned int s_last;
        __shared__ double red[32];
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
            // the block partials in a fixed order: thread i adds partials i,
            // i + threads, ... (all loads in flight), the warps fold their
            // lanes by shuffles, thread 0 adds the warps in order
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
            double v =
                ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (lane == 0) red[warp] = v;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int i = 0; i < warps; ++i) t += red[i];
                double tot = t * a.dxdy;
                *launch_ticket(a) = 0u;
                if constexpr (V::PB) {
                    // one species of a pair (as step_kernel): the other
                    // species' next step reads this step's input buffer with
                    // the factor that was pending on it; the kept norm moves
                    // with the joint normalisation (src/cpukernel.cpp:551)
                    a.scal->last_norm = tot;
                    a.scal->prev_inv = a.scal->pending_inv;
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

// Blocks of 4 or 8 warps (4 in a rotating frame); each warp loops over the
// tasks t = warp_global, warp_global + total_warps, ...
// Register budget: 2 cells per lane fit 128 registers, so 16 warps of the
// default 4-warp blocks stay resident per SM; 4 cells per lane take up to
// 255.  In a rotating frame (blocks of at most 4 warps) the 8-row window
// takes ~160 registers in double, 3 blocks per SM as its 8-row ring allows
// (capping the registers at 170 for 3 blocks made the compiler's schedule
// slower: 1039 -> 1072 us per 8192^2 step; with more live state, 174
// registers, 2 blocks per SM, it took 1182 us); in float a cap of 170 (3
// blocks per SM) ran 600 us against 621 at a cap of 128 (5 blocks).
template <class V>
struct W2Bounds {
    static constexpr bool ROT32 = V::ROT && sizeof(typename V::T) == 4;
    static constexpr int THREADS = ROT32 ? 128 : 256;
    static constexpr int MIN_BLOCKS = ROT32 ? 3 : ((V::C == 2 && !V::ROT) ? 2 : 1);
};

// Per-warp set-up: this warp's ring (D slots), its vertical pair table of
// `vl` entries and its mbarriers, the ring zeroed and the window finite.
template <class V, int R>
__device__ __forceinline__ void w2_warp_setup(Walk2<V, R> &w, unsigned char *smem, int warps,
                                              int warp, int lane, int vl) {
    using T = typename V::T;
    using S = W2Shape<V, R>;
    w.lane = lane;
    w.nacc = 0.0;
    w.failed = false;
    w.ring = smem + (size_t)warp * S::D * S::SLOT;
    w.vco = reinterpret_cast<Cx<T> *>(smem + (size_t)warps * S::D * S::SLOT) + (size_t)warp * vl;
    w.bars = reinterpret_cast<uint64_t *>(smem + (size_t)warps * S::D * S::SLOT +
                                          (size_t)warps * vl * sizeof(Cx<T>)) +
             warp * S::D;
    {
        uint4 *z = reinterpret_cast<uint4 *>(w.ring);
        for (int i = lane; i < S::D * S::SLOT / 16; i += 32) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (lane == 0) {
        for (int q = 0; q < S::D; ++q) mbar_init(&w.bars[q], 1);
        fence_mbar_init();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    // finite window contents before the first task (the first rows of every
    // walk meet whatever the window holds only in halo rows)
#pragma unroll
    for (int j = 0; j < S::NW; ++j)
#pragma unroll
        for (int i = 0; i < V::C; ++i) w.win[j][i] = Cx<T>{T(0), T(0)};
}

// The step constants of one tile (read after the previous step completed:
// the renormalisation factor and, in FP32 real time, the step of the
// kinetic coefficient schedule).
template <class V, int R>
__device__ __forceinline__ void w2_bind(Walk2<V, R> &w, const StepArgs<typename V::T> &a) {
    using T = typename V::T;
    w.H = a.H;
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
    w.row_ab = reinterpret_cast<const Cx<T> *>(a.row_ab);
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
    w.opitch = (size_t)a.P;
    w.gpsi_pitch = (size_t)a.P * sizeof(Cx<T>);
    w.gtab_pitch = a.pot_pitch ? a.pot_pitch : (size_t)a.P * sizeof(typename V::TabT);
    if constexpr (V::VPOT) w.vdt = (T)a.pot_dt;
}

template <class V, int R>
__global__ void __launch_bounds__(W2Bounds<V>::THREADS, W2Bounds<V>::MIN_BLOCKS)
    step2_kernel(StepArgs<typename V::T> a) {
    extern __shared__ __align__(128) unsigned char smem[];
    // the next step's blocks may be scheduled as this step's blocks retire
    // (programmatic dependent launch): their set-up below overlaps this
    // step's tail, and they wait for this step's completion before reading
    // its output
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int warps = blockDim.x >> 5;
    const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const int lane = threadIdx.x & 31;
    const int n_tasks = a.n_strips * a.n_segs;

    Walk2<V, R> w;
    w2_warp_setup(w, smem, warps, warp, lane, w2_vlen(a.seg_h, W2Shape<V, R>::ROT));
    // everything below reads what the previous step wrote (the tile, the
    // renormalisation factor, the schedule's step): wait for its completion
    // (immediate without a programmatic dependency)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    w2_bind(w, a);

    for (int task = blockIdx.x * warps + warp; task < n_tasks && !w.failed;
         task += gridDim.x * warps)
        w2_task(w, a, task);

    w2_finish<V>(a, w.nacc, warps, warp, lane);
}

// Many tiles of one precision and time mode in one persistent launch (the
// batched step on the look-ahead walk): the task list of all tiles is
// walked as by batch_step_kernel, each task binding its tile's buffers and
// constants; in imaginary time each task's squared norm goes to
// task_norm[task], which a per-tile pass sums into the tile's
// renormalisation factor.  b.vlen: vertical pair table entries per warp (for
// the tallest segment of the batch).
template <class V, int R>
__global__ void __launch_bounds__(128, 4) batch2_kernel(BatchArgs<typename V::T> b) {
    using T = typename V::T;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warps = blockDim.x >> 5;
    const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const int lane = threadIdx.x & 31;

    Walk2<V, R> w;
    w2_warp_setup(w, smem, warps, warp, lane, b.vlen);
    for (int t = blockIdx.x * warps + warp; t < b.n_tasks && !w.failed; t += gridDim.x * warps) {
        const int2 it = __ldg(&b.tasks[t]);
        const int tile = bcast0(it.x), task = bcast0(it.y);
        const StepArgs<T> a = load_tile_args(b.inst + tile);
        w2_bind(w, a);
        w.nacc = 0.0;
        w2_task(w, a, task);
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
