// Adjoint (reverse-mode) Trotter step for real-time evolution on a closed
// tile, FP64: one fused streaming pass per step carries the adjoint field
// lambda backwards through the transposed stages and accumulates dL/dV.
//
// Forward step (src/cpukernel.cpp:22-92, real time): stages in application
// order V0 H0 V1 H1 P H1 V1 H0 V0.  Every kinetic stage is a pair rotation
// [[a, ib], [ib, a]] (src/cpucartesian.cpp:8-11): as a real 4x4 map on
// (re_i, im_i, re_j, im_j) it is orthogonal, so its transpose is its inverse,
// the same rotation with b -> -b.  The potential stage (src/cpucartesian.cpp:
// 96-106) is psi' = R psi with R = E exp(-i theta), E = exp(-i V dt) from the
// table, theta = g dt |psi|^2 (+ g_LHY dt |psi|^3), |psi|^2 taken before the
// table multiply.  With <u, w> = Re(conj(u) w) and q = Im(conj(lambda') psi'):
//     lambda = conj(R) lambda' + 2 theta'(|psi|^2) q psi,
//     dL/dV += dt q,                       (dE/dV = -i dt E)
// where lambda' is the adjoint at the stage's output and theta' = d theta /
// d|psi|^2 = g dt (+ 1.5 g_LHY dt |psi|).
//
// Two modes:
//  INVERSE (g = g_LHY = 0): the step is linear and unitary, so the forward
//    state is recovered backwards too: psi_n = S^-1 psi_{n+1} is the same
//    palindromic stage sequence with b -> -b and conj(E).  One pass maps
//    (psi_{n+1}, lambda_{n+1}) to (psi_n, lambda_n).
//  CHECKPOINT (any g): psi_n comes from a recomputed forward state; the pass
//    runs the forward stages V0 H0 V1 H1 on psi_n (up to the potential) and
//    the transposed stages on lambda, mapping (psi_n, lambda_{n+1}) to
//    lambda_n.
//
// IMAGINARY (imaginary time, checkpoints): the forward step is
// phi_{k+1} = S(psi_k), psi_{k+1} = c_{k+1} phi_{k+1} with
// c = sqrt(norm0 / N(phi)) (src/cpukernel.cpp:551-562), N(x) = dA sum |x|^2.
// Every imaginary-time pair matrix [[a, b], [b, a]] (src/cpucartesian.cpp:
// 25-44,59-70) is symmetric, so the transposed sweeps are the sweeps
// themselves; the potential stage psi' = f E x (E = exp(-V dt) from the real
// table, f = exp(-theta(|x|^2)), src/cpucartesian.cpp:128-136) has
//     lambda = f E (lambda' - 2 theta' s x),  s = Re(conj(lambda') x),
//     dL/dV += -dt f E s.
// The pass of step k reads psi_k (stored phi_k with its factor c_k) and the
// adjoint Lambda_{k+1} = dL/dpsi_{k+1}; it applies the transpose of the
// renormalisation as the rows arrive,
//     lambda = c_{k+1} (Lambda_{k+1} - mu_{k+1} psi_{k+1}),
//     mu_{k+1} = (dA / norm0) Re<Lambda_{k+1}, psi_{k+1}>,
// which needs psi_{k+1} (stored phi_{k+1}, factor c_{k+1}) as a third field.
// The pass also produces mu_k for the next pass: Re<Lambda_k, psi_k> with
// Lambda_k = J^T lambda equals Re<K_2^T lambda, J_P chi> summed over the
// cells (J = K_2 J_P K_1, K_1 the stages before the potential, K_2 those
// after, chi = K_1 psi_k), and both factors are in registers at the
// potential stage: J_P chi = f E (1 - 2 theta' |chi|^2) chi.  The owned cells
// add it to a per-lane sum, the blocks' sums meet in a fixed order in the
// last block to finish, which writes mu_k (and adds the sum to the running
// total the gradient of the initial norm needs).
//
// The walk is the forward kernel's (column strips of 32 lanes x 2 cells,
// a 5-row register window per field, rows streamed through a shared-memory
// ring by bulk copies); each ring slot holds a row of psi, lambda, (in
// imaginary time) psi_{k+1}, the table and dL/dV.
#pragma once
#include "step_kernel.cuh"

namespace tsb {

struct AdjArgs {
    const void *psi_in;  // Cx<double>: INVERSE psi_{n+1}; CHECKPOINT psi_n
    void *psi_out;       // INVERSE: psi_n
    const void *lam_in;  // lambda_{n+1}
    void *lam_out;       // lambda_n
    const void *pot;     // Cx<double>: exp(-i V dt)
    double *gv;          // dL/dV, accumulated (read, add, write)
    int *error;          // set when a bounded wait gives up
    int W, H, P;         // tile width, height, row pitch (cells, multiple of 4)
    int n_strips, n_segs, seg_h, ring;
    double aH, bH, aV, bV;
    double ca, caa, dt;  // g dt, g_LHY dt, dt
    // IMAGINARY: psi_{k+1} (stored phi_{k+1}), the factors c_k, c_{k+1}, the
    // projection coefficient mu_{k+1} in, mu_k out, the running sum of the
    // inner products (added to when `accumulate`), dA / norm0, and the
    // per-block partials with the ticket of the last block
    const void *psn_in;
    const double *c_in, *c_next, *mu_next;
    double *mu_out, *kappa_sum;
    double *partials;
    unsigned int *ticket;
    double mu_scale;
    int accumulate;
};

template <int MODE_, int PHASE_>
struct AdjVariant {
    static constexpr int MODE = MODE_;  // 0 INVERSE, 1 CHECKPOINT, 2 IMAGINARY
    static constexpr int PHASE = PHASE_;
    static constexpr bool IMAG = MODE_ == 2;
    static constexpr int C = 2, NWIN = 5, HX = 4, HY = 4, UNROLL = 10, OUT_LAG = 4;
    static constexpr int SW = 64, WO = SW - 2 * HX;
    static constexpr int ROW = SW * 16;             // bytes of one Cx<double> row
    // slot: psi | lambda | [psi_{k+1}] | table | dL/dV
    static constexpr int PSN_OFF = 2 * ROW;
    static constexpr int TAB_OFF = IMAG ? 3 * ROW : 2 * ROW;
    static constexpr int TAB_CELL = IMAG ? 8 : 16;  // real table in imaginary time
    static constexpr int GV_OFF = TAB_OFF + SW * TAB_CELL;
    static constexpr int SLOT = GV_OFF + SW * 8;
};

struct AdjWalk {
    Cx<double> ps[5][2], la[5][2];
    bool out_col[2];
    int ra, rb, oy0, oy1, xl, lane, D;
    int lslot, tslot, issued_to, loaded_to;
    uint32_t phase_bits;
    const unsigned char *gpsi, *glam, *gtab, *ggv;  // row 0, column cs
    const unsigned char *gpsn;                      // IMAGINARY: psi_{k+1}
    double cin, cnext, m2;  // IMAGINARY: c_k, c_{k+1}, mu_{k+1} c_{k+1}
    double kacc;            // IMAGINARY: this lane's part of Re<Lambda_k, psi_k>
    size_t pitch16, pitch8;
    uint32_t off16, bytes16, off8, bytes8;
    unsigned char *ring;
    uint64_t *bars;
    bool failed;
    double hai, hbi, hal, hbl, har, hbr;  // per-lane horizontal pair coefficients
    double aVv, bVv;                      // vertical pair coefficients

    template <class A>
    __device__ __forceinline__ void issue(int row, int q) {
        unsigned char *sb = ring + q * A::SLOT;
        if constexpr (A::IMAG) {
            mbar_expect_tx(&bars[q], 3 * bytes16 + 2 * bytes8);
            bulk_g2s(sb + off16, gpsi + (size_t)row * pitch16, bytes16, &bars[q]);
            bulk_g2s(sb + A::ROW + off16, glam + (size_t)row * pitch16, bytes16, &bars[q]);
            bulk_g2s(sb + A::PSN_OFF + off16, gpsn + (size_t)row * pitch16, bytes16, &bars[q]);
            bulk_g2s(sb + A::TAB_OFF + off8, gtab + (size_t)row * pitch8, bytes8, &bars[q]);
            bulk_g2s(sb + A::GV_OFF + off8, ggv + (size_t)row * pitch8, bytes8, &bars[q]);
        } else {
            mbar_expect_tx(&bars[q], 3 * bytes16 + bytes8);
            bulk_g2s(sb + off16, gpsi + (size_t)row * pitch16, bytes16, &bars[q]);
            bulk_g2s(sb + A::ROW + off16, glam + (size_t)row * pitch16, bytes16, &bars[q]);
            bulk_g2s(sb + A::TAB_OFF + off16, gtab + (size_t)row * pitch16, bytes16, &bars[q]);
            bulk_g2s(sb + A::GV_OFF + off8, ggv + (size_t)row * pitch8, bytes8, &bars[q]);
        }
    }
    __device__ __forceinline__ int next(int q) const { return q + 1 == D ? 0 : q + 1; }
};

// Horizontal sweep; NEG: the transposed (inverse) rotation; IM: the
// imaginary-time pair matrix (symmetric: its own transpose).
template <int PAR, bool NEG, bool IM = false>
__device__ __forceinline__ void adj_h(AdjWalk &w, Cx<double> (&row)[2]) {
    const double s = NEG ? -1.0 : 1.0;
    hsweep_lane<IM, PAR>(row, w.hai, s * w.hbi, w.hal, s * w.hbl, w.har, s * w.hbr);
}

// Potential stage of row u (both fields at this point of the pipeline).
template <class A>
__device__ __forceinline__ void adj_potential(AdjWalk &w, const AdjArgs &a, Cx<double> (&ps)[2],
                                              Cx<double> (&la)[2], int q, int u) {
    const unsigned char *sb = w.ring + q * A::SLOT;
    const double *gp = reinterpret_cast<const double *>(sb + A::GV_OFF) + 2 * w.lane;
    const bool out_row = u >= w.oy0 && u < w.oy1;
    double *grow = a.gv + (size_t)u * a.P + w.xl;
    if constexpr (A::IMAG) {
        const double *ep = reinterpret_cast<const double *>(sb + A::TAB_OFF) + 2 * w.lane;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            // psi is chi (the stage's input), lambda is at the stage's output
            const Cx<double> x = ps[i];
            const Cx<double> l = la[i];
            const double n2 = __fma_rn(x.re, x.re, __dmul_rn(x.im, x.im));
            double th = 0.0, dth = 0.0;
            if (A::PHASE) {
                th = __dmul_rn(a.ca, n2);
                dth = a.ca;
                if (A::PHASE == 2) {
                    const double r = sqrt(n2);
                    th = __fma_rn(a.caa, __dmul_rn(n2, r), th);
                    dth = __fma_rn(1.5 * a.caa, r, dth);
                }
            }
            const double fe = A::PHASE ? __dmul_rn(phase_expneg(th), ep[i]) : ep[i];
            const double sd = __fma_rn(l.re, x.re, __dmul_rn(l.im, x.im));
            const double k2 = 2.0 * dth * sd;
            if (out_row && w.out_col[i]) {
                grow[i] = __fma_rn(-a.dt, __dmul_rn(fe, sd), gp[i]);
                w.kacc = __fma_rn(__dmul_rn(fe, __fma_rn(-2.0 * dth, n2, 1.0)), sd, w.kacc);
            }
            la[i].re = __dmul_rn(fe, __fma_rn(-k2, x.re, l.re));
            la[i].im = __dmul_rn(fe, __fma_rn(-k2, x.im, l.im));
        }
        return;
    }
    const Cx<double> *tp = reinterpret_cast<const Cx<double> *>(sb + A::TAB_OFF) + 2 * w.lane;
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const Cx<double> e = ld_cx_shared(tp + i);
        const double g_old = gp[i];
        const Cx<double> l = la[i];
        if (A::MODE == 0) {
            // psi, lambda are at the stage's output: psi' and lambda'
            const Cx<double> p = ps[i];
            const double qv = __fma_rn(l.re, p.im, -__dmul_rn(l.im, p.re));
            if (out_row && w.out_col[i]) grow[i] = __fma_rn(a.dt, qv, g_old);
            ps[i].re = __fma_rn(e.re, p.re, __dmul_rn(e.im, p.im));
            ps[i].im = __fma_rn(e.re, p.im, -__dmul_rn(e.im, p.re));
            la[i].re = __fma_rn(e.re, l.re, __dmul_rn(e.im, l.im));
            la[i].im = __fma_rn(e.re, l.im, -__dmul_rn(e.im, l.re));
        } else {
            // psi is at the stage's input, lambda at its output
            const Cx<double> x = ps[i];
            const double n2 = __fma_rn(x.re, x.re, __dmul_rn(x.im, x.im));
            double c = 1.0, s = 0.0, dth = 0.0;
            if (A::PHASE) {
                double th = __dmul_rn(a.ca, n2);
                dth = a.ca;
                if (A::PHASE == 2) {
                    const double r = sqrt(n2);
                    th = __fma_rn(a.caa, __dmul_rn(n2, r), th);
                    dth = __fma_rn(1.5 * a.caa, r, dth);
                }
                phase_sincos(th, &s, &c);
            }
            // psi' = exp(-i theta) (E x)
            const double tr = __fma_rn(e.re, x.re, -__dmul_rn(e.im, x.im));
            const double ti = __fma_rn(e.re, x.im, __dmul_rn(e.im, x.re));
            const double pr = __fma_rn(c, tr, __dmul_rn(s, ti));
            const double pi = __fma_rn(c, ti, -__dmul_rn(s, tr));
            const double qv = __fma_rn(l.re, pi, -__dmul_rn(l.im, pr));
            if (out_row && w.out_col[i]) grow[i] = __fma_rn(a.dt, qv, g_old);
            // lambda = conj(E) exp(+i theta) lambda' + 2 theta' q x
            const double ur = __fma_rn(c, l.re, -__dmul_rn(s, l.im));
            const double ui = __fma_rn(c, l.im, __dmul_rn(s, l.re));
            const double k2 = A::PHASE ? 2.0 * dth * qv : 0.0;
            la[i].re = __fma_rn(e.re, ur, __fma_rn(e.im, ui, __dmul_rn(k2, x.re)));
            la[i].im = __fma_rn(e.re, ui, __fma_rn(-e.im, ur, __dmul_rn(k2, x.im)));
        }
    }
}

// One iteration of the adjoint walk for row r = base + K (base even).
template <class A, int K, bool GUARD>
__device__ __forceinline__ void adj_row(AdjWalk &w, const AdjArgs &a, int r) {
    constexpr int NWIN = 5;
    constexpr bool INV = A::MODE == 0;
    constexpr bool IM = A::IMAG;
#define PS(j) w.ps[((K) - (j) + 2 * NWIN) % NWIN]
#define LA(j) w.la[((K) - (j) + 2 * NWIN) % NWIN]
    const int ra = w.ra, rb = w.rb;
    const double aV = w.aVv, bV = w.bVv;
    // psi: inverse rotations (INVERSE) or forward ones (CHECKPOINT, IMAGINARY);
    // lambda: the transposed stages (b -> -b in real time, the same in
    // imaginary time)
    const double bVp = INV ? -bV : bV;
    const double bVl = IM ? bV : -bV;

    if (!GUARD || (r >= ra && r < rb)) {
        const int q = w.lslot;
        if (!mbar_wait_bounded(&w.bars[q], (w.phase_bits >> q) & 1u)) {
            w.failed = true;
            return;
        }
        w.phase_bits ^= 1u << q;
        w.lslot = w.next(q);
        w.loaded_to = r + 1;
        const unsigned char *sb = w.ring + q * A::SLOT;
        const Cx<double> *sp = reinterpret_cast<const Cx<double> *>(sb) + 2 * w.lane;
        const Cx<double> *sl = reinterpret_cast<const Cx<double> *>(sb + A::ROW) + 2 * w.lane;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            PS(0)[i] = ld_cx_shared(sp + i);
            LA(0)[i] = ld_cx_shared(sl + i);
        }
        if constexpr (A::IMAG) {
            // psi_k = c_k phi_k; lambda = c_{k+1} (Lambda - mu c_{k+1} phi_{k+1})
            const Cx<double> *sn =
                reinterpret_cast<const Cx<double> *>(sb + A::PSN_OFF) + 2 * w.lane;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const Cx<double> n = ld_cx_shared(sn + i);
                PS(0)[i] = scale_cx(PS(0)[i], w.cin);
                LA(0)[i].re = __dmul_rn(w.cnext, __fma_rn(-w.m2, n.re, LA(0)[i].re));
                LA(0)[i].im = __dmul_rn(w.cnext, __fma_rn(-w.m2, n.im, LA(0)[i].im));
            }
        }
    }
    // S1: V0 on rows (r-1, r)
    if (!GUARD || (r - 1 >= ra && r < rb)) {
        vsweep<IM, 2, ((K + 1) & 1)>(PS(1), PS(0), aV, bVp);
        vsweep<IM, 2, ((K + 1) & 1)>(LA(1), LA(0), aV, bVl);
    }
    // S2: H0 on row r-1
    if (!GUARD || (r - 1 >= ra && r - 1 < rb)) {
        adj_h<((K + 1) & 1), INV, IM>(w, PS(1));
        adj_h<((K + 1) & 1), !IM, IM>(w, LA(1));
    }
    // S3: V1 on rows (r-2, r-1)
    if (!GUARD || (r - 2 >= ra && r - 1 < rb)) {
        vsweep<IM, 2, ((K + 1) & 1)>(PS(2), PS(1), aV, bVp);
        vsweep<IM, 2, ((K + 1) & 1)>(LA(2), LA(1), aV, bVl);
    }
    // S4: H1, potential, H1 on row r-2; refill its slot
    if (!GUARD || (r - 2 >= ra && r - 2 < rb)) {
        const int u = r - 2;
        adj_h<((K + 1) & 1), INV, IM>(w, PS(2));
        adj_h<((K + 1) & 1), !IM, IM>(w, LA(2));
        const int q = w.tslot;
        adj_potential<A>(w, a, PS(2), LA(2), q, u);
        adj_h<((K + 1) & 1), !IM, IM>(w, LA(2));
        if (INV) adj_h<((K + 1) & 1), true>(w, PS(2));
        __syncwarp();
        if (u + w.D < rb) {
            if (w.lane == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                w.issue<A>(u + w.D, q);
            }
            w.issued_to = u + w.D + 1;
        }
        w.tslot = w.next(q);
    }
    // S5: V1 on rows (r-3, r-2)
    if (!GUARD || (r - 3 >= ra && r - 2 < rb)) {
        vsweep<IM, 2, ((K) & 1)>(LA(3), LA(2), aV, bVl);
        if (INV) vsweep<false, 2, ((K) & 1)>(PS(3), PS(2), aV, -bV);
    }
    // S6: H0 on row r-3
    if (!GUARD || (r - 3 >= ra && r - 3 < rb)) {
        adj_h<((K + 1) & 1), !IM, IM>(w, LA(3));
        if (INV) adj_h<((K + 1) & 1), true>(w, PS(3));
    }
    // S7: V0 on rows (r-4, r-3)
    if (!GUARD || (r - 4 >= ra && r - 3 < rb)) {
        vsweep<IM, 2, ((K) & 1)>(LA(4), LA(3), aV, bVl);
        if (INV) vsweep<false, 2, ((K) & 1)>(PS(4), PS(3), aV, -bV);
    }
    // store the finished row r - 4
    {
        const int u = r - (NWIN - 1);
        if (u >= w.oy0 && u < w.oy1) {
            Cx<double> *lrow = reinterpret_cast<Cx<double> *>(a.lam_out) + (size_t)u * a.P + w.xl;
            Cx<double> *prow = reinterpret_cast<Cx<double> *>(a.psi_out) + (size_t)u * a.P + w.xl;
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                if (w.out_col[i]) {
                    st_cx_global(lrow + i, LA(NWIN - 1)[i]);
                    if (INV) st_cx_global(prow + i, PS(NWIN - 1)[i]);
                }
            }
        }
    }
#undef PS
#undef LA
}

template <class A, int K, bool GUARD>
__device__ __forceinline__ void adj_rows(AdjWalk &w, const AdjArgs &a, int base, int rlast) {
    if constexpr (K < A::UNROLL) {
        const int r = base + K;
        if (w.failed || (GUARD && r > rlast)) return;
        adj_row<A, K, GUARD>(w, a, r);
        adj_rows<A, K + 1, GUARD>(w, a, base, rlast);
    }
}

template <class A>
__global__ void __launch_bounds__(64, 6) adjoint_kernel(AdjArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    // programmatic dependent launch: the next pass's blocks may be placed as
    // this pass's blocks retire and set up their shared memory; they wait
    // (griddepcontrol.wait below) for this pass to complete before reading
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int warps = blockDim.x >> 5;
    const int warp = __shfl_sync(0xffffffffu, (int)(threadIdx.x >> 5), 0);
    const int lane = threadIdx.x & 31;
    const int D = a.ring;
    const int n_tasks = a.n_strips * a.n_segs;

    AdjWalk w;
    w.failed = false;
    w.D = D;
    w.lane = lane;
    w.aVv = a.aV;
    w.bVv = a.bV;
    w.ring = smem + (size_t)warp * D * A::SLOT;
    w.bars = reinterpret_cast<uint64_t *>(smem + (size_t)warps * D * A::SLOT) + warp * D;
    w.phase_bits = 0u;
    w.pitch16 = (size_t)a.P * 16;
    w.pitch8 = (size_t)a.P * 8;
    w.kacc = 0.0;
    {
        uint4 *z = reinterpret_cast<uint4 *>(w.ring);
        const int n16 = D * A::SLOT / 16;
        for (int i = lane; i < n16; i += 32) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (lane == 0) {
        for (int q = 0; q < D; ++q) mbar_init(&w.bars[q], 1);
        fence_mbar_init();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();
    // the previous kernel of the stream (recomputation or pass) has completed
    // and its writes are visible from here on
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if constexpr (A::IMAG) {
        w.cin = *a.c_in;
        w.cnext = *a.c_next;
        w.m2 = *a.mu_next * w.cnext;
    }

    for (int task = blockIdx.x * warps + warp; task < n_tasks && !w.failed;
         task += gridDim.x * warps) {
        const int strip = task % a.n_strips, seg = task / a.n_strips;
        const int ox0 = strip * A::WO, ox1 = min(ox0 + A::WO, a.W);
        const int c0 = ox0 - A::HX;
        w.oy0 = seg * a.seg_h;
        w.oy1 = min(w.oy0 + a.seg_h, a.H);
        w.ra = max(w.oy0 - A::HY, 0);
        w.rb = min(w.oy1 + A::HY, a.H);
        const int cs = max(c0, 0);
        const int ce = min(c0 + A::SW, a.P);
        w.off16 = (uint32_t)(cs - c0) * 16u;
        w.bytes16 = (uint32_t)(ce - cs) * 16u;
        w.off8 = (uint32_t)(cs - c0) * 8u;
        w.bytes8 = (uint32_t)(ce - cs) * 8u;
        w.gpsi = reinterpret_cast<const unsigned char *>(a.psi_in) + (size_t)cs * 16;
        w.glam = reinterpret_cast<const unsigned char *>(a.lam_in) + (size_t)cs * 16;
        w.gtab = reinterpret_cast<const unsigned char *>(a.pot) + (size_t)cs * A::TAB_CELL;
        if constexpr (A::IMAG) w.gpsn = reinterpret_cast<const unsigned char *>(a.psn_in) + (size_t)cs * 16;
        w.ggv = reinterpret_cast<const unsigned char *>(a.gv) + (size_t)cs * 8;
        w.xl = c0 + 2 * lane;
        bool present[2];
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int x = w.xl + i;
            present[i] = x >= 0 && x < a.W;
            w.out_col[i] = x >= ox0 && x < ox1;
        }
        const bool pint = present[0] && present[1];
        const bool pleft = lane > 0 && present[0] && w.xl - 1 >= 0;
        const bool pright = lane < 31 && present[1] && w.xl + 2 < a.W;
        w.hai = pint ? a.aH : 1.0;
        w.hbi = pint ? a.bH : 0.0;
        w.hal = pleft ? a.aH : 1.0;
        w.hbl = pleft ? a.bH : 0.0;
        w.har = pright ? a.aH : 1.0;
        w.hbr = pright ? a.bH : 0.0;
#pragma unroll
        for (int j = 0; j < 5; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                w.ps[j][i] = Cx<double>{0.0, 0.0};
                w.la[j][i] = Cx<double>{0.0, 0.0};
            }
        w.lslot = 0;
        w.tslot = 0;
        w.loaded_to = w.ra;
        w.issued_to = min(w.ra + D, w.rb);
        __syncwarp();
        if (c0 < 0 || c0 + A::SW > a.P) {
            // zero the slot bytes this task's copies do not cover
            uint32_t *ring32 = reinterpret_cast<uint32_t *>(w.ring);
            const int words = D * A::SLOT / 4;
            for (int i = lane; i < words; i += 32) {
                const uint32_t off = (uint32_t)(i * 4) % (uint32_t)A::SLOT;
                bool copied;
                if (off < (uint32_t)A::TAB_OFF) {
                    const uint32_t t = off % (uint32_t)A::ROW;
                    copied = t >= w.off16 && t < w.off16 + w.bytes16;
                } else if (off < (uint32_t)A::GV_OFF) {
                    const uint32_t t = off - (uint32_t)A::TAB_OFF;
                    copied = A::TAB_CELL == 16 ? (t >= w.off16 && t < w.off16 + w.bytes16)
                                               : (t >= w.off8 && t < w.off8 + w.bytes8);
                } else {
                    const uint32_t t = off - (uint32_t)A::GV_OFF;
                    copied = t >= w.off8 && t < w.off8 + w.bytes8;
                }
                if (!copied) ring32[i] = 0u;
            }
            __syncwarp();
        }
        if (lane == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (int row = w.ra; row < w.issued_to; ++row) w.issue<A>(row, row - w.ra);
        }
        const int rlast = w.rb - 1 + A::OUT_LAG;
        for (int base = w.ra & ~1; base <= rlast && !w.failed; base += A::UNROLL)
            adj_rows<A, 0, true>(w, a, base, rlast);
        if (w.failed) {
            if (lane == 0) atomicExch(a.error, 1);
            int q = w.lslot;
            for (int row = w.loaded_to; row < w.issued_to; ++row) {
                (void)mbar_wait_bounded(&w.bars[q], (w.phase_bits >> q) & 1u, 100000000ull);
                w.phase_bits ^= 1u << q;
                q = w.next(q);
            }
        }
    }
    if constexpr (A::IMAG) {
        // Re<Lambda_k, psi_k>: lanes, warps of the block, then the blocks in
        // a fixed order by the last block to finish
        double v = w.kacc;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        __shared__ double s_warp[32];
        __shared__ unsigned int s_last;
        if (lane == 0) s_warp[warp] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int i = 0; i < warps; ++i) b += s_warp[i];
            a.partials[blockIdx.x] = b;
            __threadfence();
            s_last = (atomicAdd(a.ticket, 1u) == gridDim.x - 1) ? 1u : 0u;
        }
        __syncthreads();
        if (s_last && threadIdx.x == 0) {
            __threadfence();
            double tot = 0.0;
            for (int i = 0; i < (int)gridDim.x; ++i) tot += __ldcg(&a.partials[i]);
            *a.mu_out = a.mu_scale * tot;
            if (a.accumulate) *a.kappa_sum += tot;
            *a.ticket = 0u;
        }
    }
}

}  // namespace tsb
