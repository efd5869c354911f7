/*
 * ts_oracle.c -- CPU restatement of the reference's Trotter-Suzuki evolution
 * path.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it as a checker.  No product code path
 * links or calls it.
 *
 * It restates, in plain C99 double arithmetic with the same operation order
 * per cell, the single-component path of trotter-suzuki-mpi 1.6.2:
 *   - pair sweeps            src/cpucartesian.cpp:4-70
 *   - potential / GPE / LHY   src/cpucartesian.cpp:73-138
 *   - rotating frame          src/cpucartesian.cpp:141-262
 *   - the Strang sequence     src/cpukernel.cpp:22-92
 *   - step constants          src/cpukernel.cpp:185-217
 *   - periodic halo exchange  src/cpukernel.cpp:691-747 (single process)
 *   - imaginary-time renorm   src/cpukernel.cpp:526-570
 *   - evolve loop             src/solver.cpp:150-242
 *   - energies                src/solver.cpp:244-564 (single component)
 *   - two components          src/cpucartesian.cpp:73-126,264-290,
 *                             src/cpukernel.cpp:581-667, src/solver.cpp:172-230
 *   - expectation values      src/model.cpp:385-536
 *
 * The reference evolves the tile in 128x128 cache blocks with a 4 (8 with
 * rotation) cell overlap; every written cell lies at least that far from an
 * interior block edge, so the blocked result equals one sweep over the whole
 * tile.  This restatement sweeps the whole tile at once.  Two places where
 * the reference's blocking itself is defective are not restated (see the
 * project design notes): tile widths 128+120q (112q with rotation) leave a
 * band of columns unwritten, and the periodic x-halo copy can read columns
 * that the current step has not written yet.
 *
 * Compile with -ffp-contract=off so that no multiply-add is fused (the
 * reference's plain -O2 x86-64 build has no FMA instructions either).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "ts_oracle.h"

/* ---- pair sweeps (src/cpucartesian.cpp:4-70) ------------------------- */

/* Pair (i, j): real time uses [[a, ib], [ib, a]], imaginary time [[a, b], [b, a]]. */
static inline void pair_real(double a, double b, double *re, double *im, size_t i, size_t j) {
    double tr = re[i], ti = im[i];
    re[i] = a * tr - b * im[j];
    im[i] = a * ti + b * re[j];
    re[j] = a * re[j] - b * ti;
    im[j] = a * im[j] + b * tr;
}

static inline void pair_imag(double a, double b, double *re, double *im, size_t i, size_t j) {
    double tr = re[i], ti = im[i];
    re[i] = a * tr + b * re[j];
    im[i] = a * ti + b * im[j];
    re[j] = a * re[j] + b * tr;
    im[j] = a * im[j] + b * ti;
}

/* Vertical sweep s: pairs (x,y)-(x,y+1) with (x+y)%2 == s and y+1 < H. */
static void sweep_vertical(const tso_params *p, int s, double a, double b, double *re, double *im) {
    const size_t W = (size_t)p->W;
    for (int y = 0; y + 1 < p->H; ++y)
        for (int x = (s + y) & 1; x < p->W; x += 2) {
            size_t i = (size_t)y * W + x;
            if (p->imag_time) pair_imag(a, b, re, im, i, i + W);
            else pair_real(a, b, re, im, i, i + W);
        }
}

/* Horizontal sweep s: pairs (x,y)-(x+1,y) with (x+y)%2 == s and x+1 < W. */
static void sweep_horizontal(const tso_params *p, int s, double a, double b, double *re, double *im) {
    const size_t W = (size_t)p->W;
    for (int y = 0; y < p->H; ++y)
        for (int x = (s + y) & 1; x + 1 < p->W; x += 2) {
            size_t i = (size_t)y * W + x;
            if (p->imag_time) pair_imag(a, b, re, im, i, i + 1);
            else pair_real(a, b, re, im, i, i + 1);
        }
}

/* ---- potential, GPE and LHY phase (src/cpucartesian.cpp:94-108,128-136) */
static void potential_step(const tso_params *p, const double *pot_re, const double *pot_im,
                           double *re, double *im) {
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        double n2 = re[k] * re[k] + im[k] * im[k];
        double n3 = n2 * sqrt(n2);
        if (p->imag_time) {
            double t = exp(-1. * (p->coupling * n2 + p->lhy_coupling * n3));
            re[k] = t * pot_re[k] * re[k];
            im[k] = t * pot_re[k] * im[k];
        } else {
            double c = cos(p->coupling * n2 + p->lhy_coupling * n3);
            double s = sin(p->coupling * n2 + p->lhy_coupling * n3);
            double t = re[k];
            re[k] = pot_re[k] * t - pot_im[k] * im[k];
            im[k] = pot_re[k] * im[k] + pot_im[k] * t;
            t = re[k];
            re[k] = c * t + s * im[k];
            im[k] = c * im[k] - s * t;
        }
    }
}

/* ---- rotating frame (src/cpucartesian.cpp:141-262) ---------------------- */
static inline void rot_pair(int imag_time, double a, double b, double *re, double *im,
                            size_t i, size_t j) {
    double tr = re[i], ti = im[i];
    if (imag_time) {
        re[i] = a * re[i] + b * im[j];
        im[i] = a * im[i] - b * re[j];
        re[j] = -b * ti + a * re[j];
        im[j] = b * tr + a * im[j];
    } else {
        re[i] = a * re[i] + b * re[j];
        im[i] = a * im[i] + b * im[j];
        re[j] = a * re[j] - b * tr;
        im[j] = a * im[j] - b * ti;
    }
}

static void rotation_rows(const tso_params *p, double *re, double *im) {
    const size_t W = (size_t)p->W;
    for (int y = 0; y < p->H; ++y) {
        double ang = -0.5 * p->alpha_y * (y + p->rot_off_y);
        double a = p->imag_time ? cosh(ang) : cos(ang);
        double b = p->imag_time ? sinh(ang) : sin(ang);
        for (int par = 0; par < 2; ++par)
            for (int x = par; x + 1 < p->W; x += 2)
                rot_pair(p->imag_time, a, b, re, im, (size_t)y * W + x, (size_t)y * W + x + 1);
    }
}

static void rotation_cols(const tso_params *p, double *re, double *im) {
    const size_t W = (size_t)p->W;
    for (int x = 0; x < p->W; ++x) {
        double ang = p->alpha_x * (x + p->rot_off_x);
        double a = p->imag_time ? cosh(ang) : cos(ang);
        double b = p->imag_time ? sinh(ang) : sin(ang);
        for (int par = 0; par < 2; ++par)
            for (int y = par; y + 1 < p->H; y += 2)
                rot_pair(p->imag_time, a, b, re, im, (size_t)y * W + x, (size_t)(y + 1) * W + x);
    }
}

/* ---- radial kinetic term (src/cpucylindrical.cpp:4-81) ---------------------
 * Pairs (i, i+1) of the radial (x) axis with i = start_offset (mod 2), every
 * row; x = i is the radial index (the tile starts at the axis).  The pair
 * (0, 1) has its own coupling.  Restated as the reference writes it,
 * including its choice of hyperbolic functions in real time and circular ones
 * in imaginary time for the pairs past the first. */
static void radial_pair(int imag_time, double a, double b, double c, double *re, double *im,
                        size_t i, size_t j) {
    double tr = re[i], ti = im[i];
    if (imag_time) {
        re[i] = a * tr + b * re[j];
        im[i] = a * ti + b * im[j];
        re[j] = a * re[j] + c * tr;
        im[j] = a * im[j] + c * ti;
    } else {
        re[i] = a * tr - b * im[j];
        im[i] = a * ti + b * re[j];
        re[j] = a * re[j] - c * ti;
        im[j] = a * im[j] + c * tr;
    }
}

static void radial_sweep(const tso_params *p, int start_offset, double *re, double *im) {
    const size_t W = (size_t)p->W;
    int start_i = 0;
    if (start_offset == 0) {
        double kr = 2 * p->kin_radial;
        double a = p->imag_time ? cosh(kr) : cos(kr);
        double b = p->imag_time ? -sinh(kr) : -sin(kr);
        for (int y = 0; y < p->H; ++y)
            radial_pair(p->imag_time, a, b, b, re, im, (size_t)y * W, (size_t)y * W + 1);
        start_i = 2;
    }
    double x = (double)start_i + start_offset;
    for (int i = start_i + start_offset; i < p->W - 1; i += 2, x += 2) {
        double kr = p->kin_radial / sqrt(x * x - 0.25);
        double ratio = sqrt((2 * x + 1) / (2 * x - 1));
        double sk = p->imag_time ? sin(kr) : sinh(kr);
        double a = p->imag_time ? cos(kr) : cosh(kr), b = sk * ratio, c = -sk / ratio;
        for (int y = 0; y < p->H; ++y)
            radial_pair(p->imag_time, a, b, c, re, im, (size_t)y * W + i, (size_t)y * W + i + 1);
    }
}

/* Column 0 (r = -dx/2) mirrors column 1 with the parity of the angular
 * momentum, after every imaginary-time step (src/cpukernel.cpp:669-689). */
static void mirror_axis(const tso_params *p, double *re, double *im) {
    const size_t W = (size_t)p->W;
    for (int y = 0; y < p->H; ++y) {
        re[(size_t)y * W] = p->mirror_sign * re[(size_t)y * W + 1];
        im[(size_t)y * W] = p->mirror_sign * im[(size_t)y * W + 1];
    }
}

/* ---- one full step (src/cpukernel.cpp:22-92) ----------------------------- */
void tso_full_step(const tso_params *p, double *re, double *im, const double *pot_re,
                   const double *pot_im) {
    const int vert = p->H > 1;
    if (vert) sweep_vertical(p, 0, p->aV, p->bV, re, im);
    sweep_horizontal(p, 0, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 1, p->aV, p->bV, re, im);
    sweep_horizontal(p, 1, p->aH, p->bH, re, im);
    if (p->cylindrical) {
        radial_sweep(p, 0, re, im);
        radial_sweep(p, 1, re, im);
    }
    potential_step(p, pot_re, pot_im, re, im);
    if (p->alpha_x != 0. && p->alpha_y != 0.) {
        rotation_rows(p, re, im);
        rotation_cols(p, re, im);
        rotation_rows(p, re, im);
    }
    if (p->cylindrical) {
        radial_sweep(p, 1, re, im);
        radial_sweep(p, 0, re, im);
    }
    sweep_horizontal(p, 1, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 1, p->aV, p->bV, re, im);
    sweep_horizontal(p, 0, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 0, p->aV, p->bV, re, im);
}

/* ---- periodic halo refresh (src/cpukernel.cpp:706-716,738-746) ----------- */
void tso_halo_exchange(const tso_params *p, double *re, double *im) {
    const size_t W = (size_t)p->W;
    if (p->periodic_x) {
        /* rows [iy0, iy0 + H - 2*halo_y), as the reference copies them */
        int nrows = p->H - 2 * p->halo_y;
        int n_in = p->W - 2 * p->halo_x;
        for (int r = 0; r < nrows; ++r) {
            size_t row = (size_t)(p->iy0 + r) * W;
            for (int c = 0; c < p->halo_x; ++c) {
                re[row + c] = re[row + c + n_in];
                im[row + c] = im[row + c + n_in];
                re[row + p->W - p->halo_x + c] = re[row + p->halo_x + c];
                im[row + p->W - p->halo_x + c] = im[row + p->halo_x + c];
            }
        }
    }
    if (p->periodic_y) {
        int n_in = p->H - 2 * p->halo_y;
        for (int r = 0; r < p->halo_y; ++r) {
            memcpy(re + (size_t)r * W, re + (size_t)(r + n_in) * W, W * sizeof(double));
            memcpy(im + (size_t)r * W, im + (size_t)(r + n_in) * W, W * sizeof(double));
            memcpy(re + (size_t)(p->H - p->halo_y + r) * W, re + (size_t)(p->halo_y + r) * W,
                   W * sizeof(double));
            memcpy(im + (size_t)(p->H - p->halo_y + r) * W, im + (size_t)(p->halo_y + r) * W,
                   W * sizeof(double));
        }
    }
}

/* ---- norm and renormalisation (src/cpukernel.cpp:526-562) ---------------- */
double tso_squared_norm(const tso_params *p, const double *re, const double *im) {
    double s = 0.;
    for (int y = p->iy0; y < p->iy1; ++y)
        for (int x = p->ix0; x < p->ix1; ++x) {
            size_t k = (size_t)y * p->W + x;
            s += re[k] * re[k] + im[k] * im[k];
        }
    return s * p->delta_x * p->delta_y;
}

static void renormalise(const tso_params *p, double *re, double *im) {
    if (!p->imag_time || p->norm0 == 0) return;
    double f = sqrt(tso_squared_norm(p, re, im) / p->norm0);
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        re[k] /= f;
        im[k] /= f;
    }
}

/* ---- evolve loop (src/solver.cpp:186-230, single component) -------------- */
void tso_evolve(const tso_params *p, double *re, double *im, const double *pot_re,
                const double *pot_im, int iterations) {
    for (int i = 0; i < iterations; ++i) {
        tso_full_step(p, re, im, pot_re, pot_im);
        if (i != iterations - 1) tso_halo_exchange(p, re, im);
        renormalise(p, re, im);
        if (p->cylindrical && p->imag_time) mirror_axis(p, re, im);
    }
}

/* ---- two components ------------------------------------------------------
 * The two-wavefunction path of the reference: the step of one component with
 * the other's density in the nonlinear phase (src/cpucartesian.cpp:73-92,
 * 113-126: exp(-i (g dt |a|^2 + g_ab dt |b|^2)), |b|^2 from the other
 * component's buffer at the start of the component's step), the Rabi
 * rotation (src/cpucartesian.cpp:264-290 with the angle of
 * src/cpukernel.cpp:581-606) and, in imaginary time with a Rabi coupling,
 * the joint normalisation (src/cpukernel.cpp:608-667); the loop is
 * src/solver.cpp:172-230 (B steps with A's state from before A's step). */
static void potential_step2(const tso_params *p, double coupling_ab, const double *pot_re,
                            const double *pot_im, const double *pb_re, const double *pb_im,
                            double *re, double *im) {
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        double n2 = re[k] * re[k] + im[k] * im[k];
        double n2b = pb_re[k] * pb_re[k] + pb_im[k] * pb_im[k];
        if (p->imag_time) {
            double t = exp(-1. * (p->coupling * n2 + coupling_ab * n2b));
            re[k] = t * pot_re[k] * re[k];
            im[k] = t * pot_re[k] * im[k];
        } else {
            double c = cos(p->coupling * n2 + coupling_ab * n2b);
            double s = sin(p->coupling * n2 + coupling_ab * n2b);
            double t = re[k];
            re[k] = pot_re[k] * t - pot_im[k] * im[k];
            im[k] = pot_re[k] * im[k] + pot_im[k] * t;
            t = re[k];
            re[k] = c * t + s * im[k];
            im[k] = c * im[k] - s * t;
        }
    }
}

void tso_full_step2(const tso_params *p, double coupling_ab, double *re, double *im,
                    const double *pot_re, const double *pot_im, const double *pb_re,
                    const double *pb_im) {
    const int vert = p->H > 1;
    if (vert) sweep_vertical(p, 0, p->aV, p->bV, re, im);
    sweep_horizontal(p, 0, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 1, p->aV, p->bV, re, im);
    sweep_horizontal(p, 1, p->aH, p->bH, re, im);
    potential_step2(p, coupling_ab, pot_re, pot_im, pb_re, pb_im, re, im);
    if (p->alpha_x != 0. && p->alpha_y != 0.) {
        rotation_rows(p, re, im);
        rotation_cols(p, re, im);
        rotation_rows(p, re, im);
    }
    sweep_horizontal(p, 1, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 1, p->aV, p->bV, re, im);
    sweep_horizontal(p, 0, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 0, p->aV, p->bV, re, im);
}

void tso_rabi(const tso_params *p, double omega_r, double omega_i, double var, double delta_t,
              double *a_re, double *a_im, double *b_re, double *b_im) {
    const double c3 = 0.5 * omega_r, c4 = 0.5 * omega_i;
    const double norm_omega = sqrt(c3 * c3 + c4 * c4);
    double cc, cs_r, cs_i;
    if (p->imag_time) {
        cc = cosh(-delta_t * var * norm_omega);
        cs_r = norm_omega == 0 ? 0 : c3 / norm_omega * sinh(-delta_t * var * norm_omega);
        cs_i = norm_omega == 0 ? 0 : c4 / norm_omega * sinh(-delta_t * var * norm_omega);
    } else {
        cc = cos(-delta_t * var * norm_omega);
        cs_r = norm_omega == 0 ? 0 : c3 / norm_omega * sin(-delta_t * var * norm_omega);
        cs_i = norm_omega == 0 ? 0 : c4 / norm_omega * sin(-delta_t * var * norm_omega);
    }
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        double r = a_re[k], i = a_im[k];
        if (p->imag_time) {
            a_re[k] = cc * r + cs_r * b_re[k] - cs_i * b_im[k];
            a_im[k] = cc * i + cs_i * b_re[k] + cs_r * b_im[k];
            b_re[k] = cc * b_re[k] + cs_r * r + cs_i * i;
            b_im[k] = cc * b_im[k] - cs_i * r + cs_r * i;
        } else {
            a_re[k] = cc * r - cs_i * b_re[k] - cs_r * b_im[k];
            a_im[k] = cc * i + cs_r * b_re[k] - cs_i * b_im[k];
            b_re[k] = cc * b_re[k] + cs_i * r - cs_r * i;
            b_im[k] = cc * b_im[k] + cs_r * r + cs_i * i;
        }
    }
}

static double inner_sum(const tso_params *p, const double *re, const double *im) {
    double s = 0.;
    for (int y = p->iy0; y < p->iy1; ++y)
        for (int x = p->ix0; x < p->ix1; ++x) {
            size_t k = (size_t)y * p->W + x;
            s += re[k] * re[k] + im[k] * im[k];
        }
    return s;
}

static void scale_tile(const tso_params *p, double f, double *re, double *im) {
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        re[k] /= f;
        im[k] /= f;
    }
}

int tso_evolve2(const tso_params *pa, const tso_params *pb, double coupling_ab, double omega_r,
                double omega_i, double delta_t, double *norms, double tot_norm, double *a_re,
                double *a_im, double *b_re, double *b_im, const double *ta_re,
                const double *ta_im, const double *tb_re, const double *tb_im, int iterations,
                int rabi_first_half) {
    const size_t n = (size_t)pa->W * pa->H;
    double *old_re = malloc(n * sizeof(double)), *old_im = malloc(n * sizeof(double));
    if (!old_re || !old_im) {
        free(old_re);
        free(old_im);
        return 1;
    }
    if (rabi_first_half) tso_rabi(pa, omega_r, omega_i, 0.5, delta_t, a_re, a_im, b_re, b_im);
    for (int i = 0; i < iterations; ++i) {
        memcpy(old_re, a_re, n * sizeof(double));
        memcpy(old_im, a_im, n * sizeof(double));
        tso_full_step2(pa, coupling_ab, a_re, a_im, ta_re, ta_im, b_re, b_im);
        if (i != iterations - 1) tso_halo_exchange(pa, a_re, a_im);
        if (pa->imag_time && norms[0] != 0)
            scale_tile(pa, sqrt(tso_squared_norm(pa, a_re, a_im) / norms[0]), a_re, a_im);
        tso_full_step2(pb, coupling_ab, b_re, b_im, tb_re, tb_im, old_re, old_im);
        if (i != iterations - 1) tso_halo_exchange(pb, b_re, b_im);
        if (pb->imag_time && norms[1] != 0)
            scale_tile(pb, sqrt(tso_squared_norm(pb, b_re, b_im) / norms[1]), b_re, b_im);
        tso_rabi(pa, omega_r, omega_i, i == iterations - 1 ? 0.5 : 1., delta_t, a_re, a_im, b_re,
                 b_im);
        if (pa->imag_time && (omega_r != 0 || omega_i != 0)) {
            double sa = inner_sum(pa, a_re, a_im), sb = inner_sum(pa, b_re, b_im);
            double f = sqrt((sa + sb) * pa->delta_x * pa->delta_y / tot_norm);
            scale_tile(pa, f, a_re, a_im);
            scale_tile(pa, f, b_re, b_im);
            norms[0] = sa / (sa + sb) * tot_norm;
            norms[1] = sb / (sa + sb) * tot_norm;
        }
    }
    free(old_re);
    free(old_im);
    return 0;
}

/* ---- reverse mode of tso_evolve (real time, closed tile) ----------------
 * Not a restatement of the reference (it has no derivatives): the
 * transpose, stage by stage, of the forward step above, used as the FP64
 * CPU check of the B200 adjoint kernel.  Every pair sweep is orthogonal as a
 * real map, so its transpose is the same sweep with b -> -b.  The potential
 * stage psi' = exp(-i theta(|x|^2)) E x (x its input) has the transpose
 *     lambda = conj(E) exp(+i theta) lambda' + 2 theta' q x,
 *     q = Im(conj(lambda') psi'),   dL/dV += dt q   (dE/dV = -i dt E),
 * with theta = g|x|^2 + g_lhy|x|^3 (g, g_lhy already times dt) and
 * theta' = g + 1.5 g_lhy |x|.  All forward states are stored (small tiles). */
static void forward_half(const tso_params *p, double *re, double *im) {
    const int vert = p->H > 1;
    if (vert) sweep_vertical(p, 0, p->aV, p->bV, re, im);
    sweep_horizontal(p, 0, p->aH, p->bH, re, im);
    if (vert) sweep_vertical(p, 1, p->aV, p->bV, re, im);
    sweep_horizontal(p, 1, p->aH, p->bH, re, im);
}

static void adjoint_potential(const tso_params *p, const double *pot_re, const double *pot_im,
                              double dt, const double *xr, const double *xi, double *lr,
                              double *li, double *grad_v) {
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        double n2 = xr[k] * xr[k] + xi[k] * xi[k];
        double r = sqrt(n2);
        double th = p->coupling * n2 + p->lhy_coupling * n2 * r;
        double dth = p->coupling + 1.5 * p->lhy_coupling * r;
        double c = cos(th), s = sin(th);
        double tr = pot_re[k] * xr[k] - pot_im[k] * xi[k];
        double ti = pot_re[k] * xi[k] + pot_im[k] * xr[k];
        double pr = c * tr + s * ti, pi = c * ti - s * tr;
        double q = lr[k] * pi - li[k] * pr;
        grad_v[k] += dt * q;
        double ur = c * lr[k] - s * li[k], ui = c * li[k] + s * lr[k];
        double nr = pot_re[k] * ur + pot_im[k] * ui + 2. * dth * q * xr[k];
        double ni = pot_re[k] * ui - pot_im[k] * ur + 2. * dth * q * xi[k];
        lr[k] = nr;
        li[k] = ni;
    }
}

int tso_adjoint_real(const tso_params *p, const double *pot_re, const double *pot_im, double dt,
                     const double *psi0_re, const double *psi0_im, int steps,
                     const double *lam_re, const double *lam_im, double *grad_v,
                     double *grad_re, double *grad_im) {
    const size_t n = (size_t)p->W * p->H;
    const int vert = p->H > 1;
    if (p->imag_time || p->periodic_x || p->periodic_y || (p->alpha_x != 0. && p->alpha_y != 0.))
        return 1;
    double *states = (double *)malloc(sizeof(double) * 2 * n * (size_t)steps);
    double *xr = (double *)malloc(sizeof(double) * n), *xi = (double *)malloc(sizeof(double) * n);
    if (!states || !xr || !xi) {
        free(states); free(xr); free(xi);
        return 2;
    }
    double *cr = states, *ci = states + n;
    memcpy(cr, psi0_re, sizeof(double) * n);
    memcpy(ci, psi0_im, sizeof(double) * n);
    for (int s = 1; s < steps; ++s) {
        double *pr = states + 2 * n * (size_t)(s - 1), *nr = states + 2 * n * (size_t)s;
        memcpy(nr, pr, sizeof(double) * 2 * n);
        tso_full_step(p, nr, nr + n, pot_re, pot_im);
    }
    memcpy(grad_re, lam_re, sizeof(double) * n);
    memcpy(grad_im, lam_im, sizeof(double) * n);
    memset(grad_v, 0, sizeof(double) * n);
    for (int s = steps - 1; s >= 0; --s) {
        memcpy(xr, states + 2 * n * (size_t)s, sizeof(double) * n);
        memcpy(xi, states + 2 * n * (size_t)s + n, sizeof(double) * n);
        forward_half(p, xr, xi);  /* x: the potential stage's input */
        if (vert) sweep_vertical(p, 0, p->aV, -p->bV, grad_re, grad_im);
        sweep_horizontal(p, 0, p->aH, -p->bH, grad_re, grad_im);
        if (vert) sweep_vertical(p, 1, p->aV, -p->bV, grad_re, grad_im);
        sweep_horizontal(p, 1, p->aH, -p->bH, grad_re, grad_im);
        adjoint_potential(p, pot_re, pot_im, dt, xr, xi, grad_re, grad_im, grad_v);
        sweep_horizontal(p, 1, p->aH, -p->bH, grad_re, grad_im);
        if (vert) sweep_vertical(p, 1, p->aV, -p->bV, grad_re, grad_im);
        sweep_horizontal(p, 0, p->aH, -p->bH, grad_re, grad_im);
        if (vert) sweep_vertical(p, 0, p->aV, -p->bV, grad_re, grad_im);
    }
    free(states); free(xr); free(xi);
    return 0;
}

/* ---- reverse mode of the imaginary-time evolution (closed tile) ----------
 * Not a restatement of the reference (it has no derivatives): the transpose
 * of tso_evolve in imaginary time, the CPU FP64 check of the B200 imaginary-
 * time adjoint.  Forward: norm0 = N(psi_0) (the State's norm when the
 * imaginary-time evolution starts, src/solver.cpp:155), then per step
 *     phi_{k+1} = S(psi_k),  psi_{k+1} = c_{k+1} phi_{k+1},
 *     c = sqrt(norm0 / N(phi))                      (src/cpukernel.cpp:551-562)
 * with N(x) = dA sum |x|^2 over the tile.  Reverse, from Lambda = dL/dpsi_T:
 *   - normalisation of step k's output: kappa_k = Re<Lambda, psi_k>,
 *         Lambda <- c_k (Lambda - (dA / norm0) kappa_k psi_k);
 *   - the step: every imaginary-time pair matrix [[a, b], [b, a]] is
 *     symmetric, so the transposed sweeps are the sweeps themselves, in
 *     reverse order; the potential stage psi' = f E x (E = exp(-V dt),
 *     f = exp(-theta(|x|^2)), theta = g|x|^2 + g_lhy|x|^3, g and g_lhy
 *     already times dt) has the transpose
 *         lambda = f E (lambda' - 2 theta' s x),  s = Re(conj(lambda') x),
 *         dL/dV += -dt f E s,                 theta' = g + 1.5 g_lhy |x|;
 *   - norm0 depends on psi_0: dL/dpsi_0 += (dA / norm0) sum_{k>=1} kappa_k psi_0.
 * All forward states are stored (small tiles). */
static void adjoint_potential_imag(const tso_params *p, const double *pot_re, double dt,
                                   const double *xr, const double *xi, double *lr, double *li,
                                   double *grad_v) {
    const size_t n = (size_t)p->W * p->H;
    for (size_t k = 0; k < n; ++k) {
        double n2 = xr[k] * xr[k] + xi[k] * xi[k];
        double r = sqrt(n2);
        double th = p->coupling * n2 + p->lhy_coupling * n2 * r;
        double dth = p->coupling + 1.5 * p->lhy_coupling * r;
        double fe = exp(-th) * pot_re[k];
        double sdot = lr[k] * xr[k] + li[k] * xi[k];
        grad_v[k] += -dt * fe * sdot;
        lr[k] = fe * (lr[k] - 2. * dth * sdot * xr[k]);
        li[k] = fe * (li[k] - 2. * dth * sdot * xi[k]);
    }
}

int tso_adjoint_imag(const tso_params *p, const double *pot_re, double dt, const double *psi0_re,
                     const double *psi0_im, int steps, const double *lam_re, const double *lam_im,
                     double *grad_v, double *grad_re, double *grad_im) {
    const size_t n = (size_t)p->W * p->H;
    const int vert = p->H > 1;
    if (!p->imag_time || p->periodic_x || p->periodic_y || (p->alpha_x != 0. && p->alpha_y != 0.) ||
        p->cylindrical)
        return 1;
    const double dA = p->delta_x * p->delta_y;
    /* states psi_0 .. psi_T (normalised) and factors c_1 .. c_T */
    double *states = (double *)malloc(sizeof(double) * 2 * n * (size_t)(steps + 1));
    double *cs = (double *)malloc(sizeof(double) * (size_t)(steps + 1));
    double *xr = (double *)malloc(sizeof(double) * n), *xi = (double *)malloc(sizeof(double) * n);
    if (!states || !cs || !xr || !xi) {
        free(states); free(cs); free(xr); free(xi);
        return 2;
    }
    memcpy(states, psi0_re, sizeof(double) * n);
    memcpy(states + n, psi0_im, sizeof(double) * n);
    const double norm0 = tso_squared_norm(p, psi0_re, psi0_im);
    cs[0] = 1.;
    for (int s = 1; s <= steps; ++s) {
        double *pr = states + 2 * n * (size_t)(s - 1), *nr = states + 2 * n * (size_t)s;
        memcpy(nr, pr, sizeof(double) * 2 * n);
        tso_full_step(p, nr, nr + n, pot_re, NULL);
        double f = sqrt(tso_squared_norm(p, nr, nr + n) / norm0);
        for (size_t k = 0; k < n; ++k) {
            nr[k] /= f;
            nr[n + k] /= f;
        }
        cs[s] = 1. / f;
    }
    memcpy(grad_re, lam_re, sizeof(double) * n);
    memcpy(grad_im, lam_im, sizeof(double) * n);
    memset(grad_v, 0, sizeof(double) * n);
    double kappa_sum = 0.;
    for (int s = steps; s >= 1; --s) {
        const double *pr = states + 2 * n * (size_t)s, *pi = pr + n;
        double kappa = 0.;
        for (size_t k = 0; k < n; ++k) kappa += grad_re[k] * pr[k] + grad_im[k] * pi[k];
        kappa_sum += kappa;
        const double m = dA / norm0 * kappa;
        for (size_t k = 0; k < n; ++k) {
            grad_re[k] = cs[s] * (grad_re[k] - m * pr[k]);
            grad_im[k] = cs[s] * (grad_im[k] - m * pi[k]);
        }
        memcpy(xr, states + 2 * n * (size_t)(s - 1), sizeof(double) * n);
        memcpy(xi, states + 2 * n * (size_t)(s - 1) + n, sizeof(double) * n);
        forward_half(p, xr, xi);  /* x: the potential stage's input */
        if (vert) sweep_vertical(p, 0, p->aV, p->bV, grad_re, grad_im);
        sweep_horizontal(p, 0, p->aH, p->bH, grad_re, grad_im);
        if (vert) sweep_vertical(p, 1, p->aV, p->bV, grad_re, grad_im);
        sweep_horizontal(p, 1, p->aH, p->bH, grad_re, grad_im);
        adjoint_potential_imag(p, pot_re, dt, xr, xi, grad_re, grad_im, grad_v);
        sweep_horizontal(p, 1, p->aH, p->bH, grad_re, grad_im);
        if (vert) sweep_vertical(p, 1, p->aV, p->bV, grad_re, grad_im);
        sweep_horizontal(p, 0, p->aH, p->bH, grad_re, grad_im);
        if (vert) sweep_vertical(p, 0, p->aV, p->bV, grad_re, grad_im);
    }
    const double m0 = dA / norm0 * kappa_sum;
    for (size_t k = 0; k < n; ++k) {
        grad_re[k] += m0 * psi0_re[k];
        grad_im[k] += m0 * psi0_im[k];
    }
    free(states); free(cs); free(xr); free(xi);
    return 0;
}

/* ---- step constants (src/cpukernel.cpp:185-217) and table (src/solver.cpp:74-109) */
void tso_init_constants(tso_params *p, double delta_t, double mass, double g, double g_lhy,
                        double omega, double delta_x, double delta_y) {
    double kx = delta_t / (4. * mass * delta_x * delta_x);
    double ky = delta_t / (4. * mass * delta_y * delta_y);
    if (p->imag_time) {
        p->aH = cosh(kx); p->bH = sinh(kx);
        p->aV = cosh(ky); p->bV = sinh(ky);
    } else {
        p->aH = cos(kx); p->bH = sin(kx);
        p->aV = cos(ky); p->bV = sin(ky);
    }
    p->alpha_x = omega * delta_t * delta_x / (2 * delta_y);
    p->alpha_y = omega * delta_t * delta_y / (2 * delta_x);
    p->coupling = g * delta_t;
    p->lhy_coupling = g_lhy * delta_t;
    p->delta_x = delta_x;
    p->delta_y = delta_y;
}

/* exp(-i dt V) in real time, exp(-dt V) in imaginary time: the real and
 * imaginary parts of std::exp(complex) for a purely imaginary / purely real
 * argument are (cos, sin) / (exp, 0) of the component. */
void tso_exp_table(int imag_time, double delta_t, const double *V, size_t n, double *out_re,
                   double *out_im) {
    for (size_t k = 0; k < n; ++k) {
        if (imag_time) {
            out_re[k] = exp(-delta_t * V[k]);
            out_im[k] = 0.;
        } else {
            double ang = -delta_t * V[k];
            out_re[k] = cos(ang);
            out_im[k] = sin(ang);
        }
    }
}

/* ---- coordinates (src/common.cpp:45-65, cartesian) ----------------------- */
static void coords(const tso_geometry *g, int x_in, int y_in, double *x_out, double *y_out) {
    if (g->cylindrical) {
        /* the radial axis x starts at the tile's edge (src/common.cpp:66-81) */
        double idy = g->start_y * g->delta_y + 0.5 * g->delta_y + y_in * g->delta_y;
        double idx = g->start_x * g->delta_x + x_in * g->delta_x - 0.5 * g->delta_x;
        double y_c = g->global_no_halo_dim_y * g->delta_y * 0.5;
        if (idy - y_c < -g->length_y * 0.5) idy += g->length_y;
        if (idy - y_c > g->length_y * 0.5) idy -= g->length_y;
        *x_out = idx;
        *y_out = idy - y_c;
        return;
    }
    double idy = g->start_y * g->delta_y + 0.5 * g->delta_y + y_in * g->delta_y;
    double idx = g->start_x * g->delta_x + 0.5 * g->delta_x + x_in * g->delta_x;
    double x_c = g->global_no_halo_dim_x * g->delta_x * 0.5;
    double y_c = g->global_no_halo_dim_y * g->delta_y * 0.5;
    if (idx - x_c < -g->length_x * 0.5) idx += g->length_x;
    if (idx - x_c > g->length_x * 0.5) idx -= g->length_x;
    if (idy - y_c < -g->length_y * 0.5) idy += g->length_y;
    if (idy - y_c > g->length_y * 0.5) idy -= g->length_y;
    *x_out = idx - x_c;
    *y_out = idy - y_c;
}

void tso_coordinates(const tso_geometry *g, int x_in, int y_in, double *x_out, double *y_out) {
    coords(g, x_in, y_in, x_out, y_out);
}

/* ---- energies (src/solver.cpp:244-564, single component, cartesian) ------- */
typedef struct { double re, im; } cplx;

static inline cplx cload(const double *re, const double *im, size_t k) {
    cplx c = {re[k], im[k]};
    return c;
}

/* complex<double>(c, 0) * z, as std::complex evaluates it for finite values */
static inline cplx rscale(double c, cplx z) {
    cplx r = {c * z.re - 0. * z.im, c * z.im + 0. * z.re};
    return r;
}
static inline cplx cadd(cplx a, cplx b) {
    cplx r = {a.re + b.re, a.im + b.im};
    return r;
}
static inline cplx cmul(cplx a, cplx b) {
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx conjc(cplx a) {
    cplx r = {a.re, -a.im};
    return r;
}

void tso_energies(const tso_geometry *g, const double *re, const double *im, const double *V,
                  double mass, double g_coupling, double g_lhy, double omega,
                  tso_energy_result *out) {
    const int W = g->W;
    double s_n2 = 0, s_n2k = 0, s_kin = 0, s_pot = 0, s_rot = 0, s_intra = 0, s_lhy = 0;
    const int ihx = g->ix0, ihy = g->iy0;           /* inner_start - start */
    const int ehx = W - g->ix1, ehy = g->H - g->iy1; /* end - inner_end */
    const double dx = g->delta_x, dy = g->delta_y;
    const double cost_E = -1. / (2. * mass);
    const double c1 = -1. / 12., c2 = 4. / 3., c3 = -2.5;
    const double d1 = 1. / 6., d2 = -1., d3 = 0.5, d4 = 1. / 3.;
    const int xlim = g->cylindrical ? 3 : 0; /* src/solver.cpp:301 */
    for (int i = g->iy0; i < g->iy1; ++i) {
        for (int j = g->ix0; j < g->ix1; ++j) {
            size_t k = (size_t)i * W + j;
            cplx c = cload(re, im, k);
            double x, y;
            coords(g, j, i, &x, &y);
            double n2 = cmul(conjc(c), c).re;
            s_n2 += n2;
            s_pot += n2 * V[k];
            s_intra += n2 * n2 * 0.5 * g_coupling;
            s_lhy += pow(n2, 2.5) * 0.4 * g_lhy;
            if (((i - g->iy0 >= (ihy == 0) * 2 && i < g->iy1 - (ehy == 0) * 2) || g->H == 1) &&
                (j - g->ix0 >= (ihx == 0) * 2 + xlim && j < g->ix1 - (ehx == 0) * 2)) {
                cplx r = cload(re, im, k + 1), l = cload(re, im, k - 1);
                cplx rr = cload(re, im, k + 2), ll = cload(re, im, k - 2);
                s_n2k += cmul(conjc(c), c).re;
                /* cost_E * conj(c) * (lap) / (dx*dx): the division applies to the product */
                cplx lap = cadd(cadd(cadd(cadd(rscale(c1, rr), rscale(c2, r)), rscale(c2, l)),
                                     rscale(c1, ll)), rscale(c3, c));
                cplx t = {cost_E * c.re, cost_E * (-c.im)};
                s_kin += cmul(t, lap).re / (dx * dx);
                if (g->H > 1) {
                    cplx up = cload(re, im, k - W), dn = cload(re, im, k + W);
                    cplx uu = cload(re, im, k - 2 * (size_t)W), dd = cload(re, im, k + 2 * (size_t)W);
                    cplx lapy = cadd(cadd(cadd(cadd(rscale(c1, dd), rscale(c2, dn)), rscale(c2, up)),
                                          rscale(c1, uu)), rscale(c3, c));
                    s_kin += cmul(t, lapy).re / (dy * dy);
                    /* rot_x = (complex(y) * omega / dx) * i, rot_y likewise with x, dy */
                    cplx yo = {y * omega / dx, 0. * omega / dx};
                    cplx xo = {x * omega / dy, 0. * omega / dy};
                    cplx iu = {0., 1.};
                    cplx rot_x = cmul(yo, iu), rot_y = cmul(xo, iu);
                    cplx dyv = cadd(cadd(cadd(rscale(d4, up), rscale(d3, c)), rscale(d2, dn)),
                                    rscale(d1, dd));
                    cplx dxv = cadd(cadd(cadd(rscale(d4, r), rscale(d3, c)), rscale(d2, l)),
                                    rscale(d1, ll));
                    s_rot += cmul(conjc(c), cadd(cmul(rot_y, dyv), cmul(rot_x, dxv))).re;
                }
            }
        }
    }
    out->kinetic = s_kin / s_n2k;
    out->rotational = s_rot / s_n2k;
    out->potential = s_pot / s_n2;
    out->intra = s_intra / s_n2;
    out->lhy = s_lhy / s_n2;
    out->total = out->kinetic + out->potential + out->intra + out->rotational + out->lhy;
    out->norm2 = s_n2 * (dy * g->length_x / (g->global_no_halo_dim_x - (g->cylindrical ? 1 : 0)));
}

/* ---- expectation values (src/model.cpp:385-536, cartesian 2D) ------------- */
void tso_expectations(const tso_geometry *g, const double *re, const double *im,
                      tso_expectation_result *out) {
    const int W = g->W;
    const int ihx = g->ix0, ihy = g->iy0;
    const int ehx = W - g->ix1, ehy = g->H - g->iy1;
    double s_n2 = 0, sx = 0, sxx = 0, sy = 0, syy = 0, spx = 0, spxpx = 0, spy = 0, spypy = 0,
           slz = 0;
    const double param_px = -1. / g->delta_x, param_py = 1. / g->delta_y;
    const double c1 = -1. / 12., c2 = 4. / 3., c3 = -2.5;
    const double d1 = 1. / 6., d2 = -1., d3 = 0.5, d4 = 1. / 3.;
    for (int i = ihy; i < g->iy1; ++i) {
        for (int j = ihx; j < g->ix1; ++j) {
            size_t k = (size_t)i * W + j;
            cplx c = cload(re, im, k);
            double x, y;
            coords(g, j, i, &x, &y);
            cplx cc = cmul(conjc(c), c);
            cplx xr = {x, 0.}, yr = {y, 0.};
            s_n2 += cc.re;
            sx += cmul(cc, xr).re;
            sy += cmul(cc, yr).re;
            sxx += cmul(cmul(cc, xr), xr).re;
            syy += cmul(cmul(cc, yr), yr).re;
            if (i - ihy >= (ihy == 0) * 2 && i < g->iy1 - (ehy == 0) * 2 &&
                j - ihx >= (ihx == 0) * 2 && j < g->ix1 - (ehx == 0) * 2) {
                cplx up = cload(re, im, k - W), dn = cload(re, im, k + W);
                cplx r = cload(re, im, k + 1), l = cload(re, im, k - 1);
                cplx uu = cload(re, im, k - 2 * (size_t)W), dd = cload(re, im, k + 2 * (size_t)W);
                cplx rr = cload(re, im, k + 2), ll = cload(re, im, k - 2);
                cplx dxv = cadd(cadd(cadd(rscale(d4, r), rscale(d3, c)), rscale(d2, l)),
                                rscale(d1, ll));
                cplx dyv = cadd(cadd(cadd(rscale(d4, up), rscale(d3, c)), rscale(d2, dn)),
                                rscale(d1, dd));
                spx += cmul(conjc(c), dxv).im;
                spy += cmul(conjc(c), dyv).im;
                spxpx += cmul(conjc(c), cadd(cadd(cadd(cadd(rscale(c1, rr), rscale(c2, r)),
                                                      rscale(c2, l)), rscale(c1, ll)),
                                             rscale(c3, c))).re;
                spypy += cmul(conjc(c), cadd(cadd(cadd(cadd(rscale(c1, dd), rscale(c2, dn)),
                                                      rscale(c2, up)), rscale(c1, uu)),
                                             rscale(c3, c))).re;
                /* y_r / delta_x * (...) + x_r / delta_y * (...) */
                cplx ydx = {y / g->delta_x, 0. / g->delta_x};
                cplx xdy = {x / g->delta_y, 0. / g->delta_y};
                slz += cmul(conjc(c), cadd(cmul(ydx, dxv), cmul(xdy, dyv))).im;
            }
        }
    }
    out->mean_x = sx / s_n2;
    out->mean_y = sy / s_n2;
    out->mean_xx = sxx / s_n2;
    out->mean_yy = syy / s_n2;
    out->mean_px = -spx * param_px / s_n2;
    out->mean_py = -spy * param_py / s_n2;
    out->mean_pxpx = -spxpx * param_px * param_px / s_n2;
    out->mean_pypy = -spypy * param_py * param_py / s_n2;
    out->mean_lz = slz / s_n2;
    out->norm2 = s_n2 * (g->delta_x * g->delta_y);
}

/* Cross terms of the two-component energy (src/solver.cpp:340-353,438-439,
 * 549-550), kept as the reference writes them: g_ab |a|^4 |b|^4 summed and
 * divided by (sum |a|^2)(sum |b|^2), and 0.5 * sum |a|^2 |b|^2 2 Re(conj(a) b
 * omega) likewise. */
void tso_cross_energies(const tso_geometry *g, const double *a_re, const double *a_im,
                        const double *b_re, const double *b_im, double coupling_ab,
                        double omega_r, double omega_i, double *inter, double *rabi) {
    double s_a = 0, s_b = 0, s_inter = 0, s_rabi = 0;
    for (int i = g->iy0; i < g->iy1; ++i)
        for (int j = g->ix0; j < g->ix1; ++j) {
            size_t k = (size_t)i * g->W + j;
            cplx a = cload(a_re, a_im, k), b = cload(b_re, b_im, k);
            cplx om = {omega_r, omega_i};
            double na = cmul(conjc(a), a).re, nb = cmul(conjc(b), b).re;
            s_a += na;
            s_b += nb;
            /* left to right, as the reference's expressions evaluate */
            cplx t = cmul(conjc(a), a);
            t = cmul(t, conjc(a));
            t = cmul(t, a);
            t = cmul(t, conjc(b));
            t = cmul(t, b);
            t = cmul(t, conjc(b));
            t = cmul(t, b);
            s_inter += cmul(t, (cplx){coupling_ab, 0.}).re;
            cplx u = cadd(cmul(cmul(conjc(a), b), om), cmul(conjc(cmul(b, om)), a));
            cplx v = cmul(cmul(cmul(conjc(a), a), conjc(b)), b);
            s_rabi += cmul(v, u).re;
        }
    *inter = s_inter / (s_a * s_b);
    *rabi = 0.5 * s_rabi / (s_a * s_b);
}
