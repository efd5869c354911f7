/* ts_oracle.h -- CPU restatement of the reference path (test infrastructure only). */
#ifndef TS_ORACLE_H
#define TS_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One tile in the reference's layout: W x H cells, row-major, inner region
 * [ix0, ix1) x [iy0, iy1) (src/common.cpp:83-102, src/model.cpp:103-158). */
typedef struct {
    int W, H;
    int ix0, ix1, iy0, iy1;
    int periodic_x, periodic_y;
    int halo_x, halo_y;
    int imag_time;
    double aH, bH, aV, bV;          /* src/cpukernel.cpp:195-212 */
    double coupling, lhy_coupling;  /* g*dt, g_LHY*dt (src/cpukernel.cpp:213-216) */
    double alpha_x, alpha_y;        /* src/cpukernel.cpp:185-186 */
    int rot_off_x, rot_off_y;       /* trunc(start - rot_coord) (src/cpukernel.cpp:417) */
    double delta_x, delta_y;
    double norm0;                   /* squared norm kept in imaginary time (src/solver.cpp:155) */
    int cylindrical;                /* radial axis x (src/cpucylindrical.cpp) */
    double kin_radial;              /* dt / (8 m dx^2) (src/cpukernel.cpp:200-210) */
    int mirror_sign;                /* (-1)^l, column 0 = sign * column 1 (src/cpukernel.cpp:669-689) */
} tso_params;

typedef struct {
    int W, H, ix0, ix1, iy0, iy1;
    int start_x, start_y;
    int global_no_halo_dim_x, global_no_halo_dim_y;
    double delta_x, delta_y, length_x, length_y;
    int cylindrical;
} tso_geometry;

typedef struct {
    double total, kinetic, potential, rotational, intra, lhy, norm2;
} tso_energy_result;

typedef struct {
    double norm2, mean_x, mean_xx, mean_y, mean_yy, mean_px, mean_pxpx, mean_py, mean_pypy, mean_lz;
} tso_expectation_result;

void tso_init_constants(tso_params *p, double delta_t, double mass, double g, double g_lhy,
                        double omega, double delta_x, double delta_y);
void tso_exp_table(int imag_time, double delta_t, const double *V, size_t n, double *out_re,
                   double *out_im);
void tso_full_step(const tso_params *p, double *re, double *im, const double *pot_re,
                   const double *pot_im);
void tso_halo_exchange(const tso_params *p, double *re, double *im);
double tso_squared_norm(const tso_params *p, const double *re, const double *im);
/* Reverse mode of `steps` real-time steps on a closed tile (test check of
 * the B200 adjoint; not in the reference): from lambda = dL/dpsi(T) (real
 * pairs) to dL/dV (dt = time step) and dL/dpsi0.  Returns non-zero for
 * unsupported tiles or when out of memory. */
int tso_adjoint_real(const tso_params *p, const double *pot_re, const double *pot_im, double dt,
                     const double *psi0_re, const double *psi0_im, int steps,
                     const double *lam_re, const double *lam_im, double *grad_v,
                     double *grad_re, double *grad_im);

/* Reverse mode of `steps` imaginary-time steps on a closed tile, with the
 * renormalisation after every step to norm0 = N(psi_0) (test check of the
 * B200 imaginary-time adjoint; not in the reference): from lambda =
 * dL/dpsi(T) to dL/dV and dL/dpsi0 (the table is exp(-V dt), pot_re). */
int tso_adjoint_imag(const tso_params *p, const double *pot_re, double dt, const double *psi0_re,
                     const double *psi0_im, int steps, const double *lam_re, const double *lam_im,
                     double *grad_v, double *grad_re, double *grad_im);

void tso_evolve(const tso_params *p, double *re, double *im, const double *pot_re,
                const double *pot_im, int iterations);
/* Two components: one component's step with the other's density (pb) in
 * the phase; the Rabi rotation of both tiles; `iterations` steps of the
 * two-component loop.  norms[2] (the per-component norms kept in imaginary
 * time) are updated by the joint normalisation; tot_norm is their initial
 * sum.  Returns non-zero when out of memory. */
void tso_full_step2(const tso_params *p, double coupling_ab, double *re, double *im,
                    const double *pot_re, const double *pot_im, const double *pb_re,
                    const double *pb_im);
void tso_rabi(const tso_params *p, double omega_r, double omega_i, double var, double delta_t,
              double *a_re, double *a_im, double *b_re, double *b_im);
int tso_evolve2(const tso_params *pa, const tso_params *pb, double coupling_ab, double omega_r,
                double omega_i, double delta_t, double *norms, double tot_norm, double *a_re,
                double *a_im, double *b_re, double *b_im, const double *ta_re,
                const double *ta_im, const double *tb_re, const double *tb_im, int iterations,
                int rabi_first_half);
void tso_coordinates(const tso_geometry *g, int x_in, int y_in, double *x_out, double *y_out);
void tso_cross_energies(const tso_geometry *g, const double *a_re, const double *a_im,
                        const double *b_re, const double *b_im, double coupling_ab,
                        double omega_r, double omega_i, double *inter, double *rabi);
void tso_energies(const tso_geometry *g, const double *re, const double *im, const double *V,
                  double mass, double g_coupling, double g_lhy, double omega,
                  tso_energy_result *out);
void tso_expectations(const tso_geometry *g, const double *re, const double *im,
                      tso_expectation_result *out);

#ifdef __cplusplus
}
#endif
#endif
