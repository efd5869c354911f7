/*
 * ts_host.h -- flat C ABI of the C++ host layer (Lattice, State, Potential,
 * Hamiltonian, Solver) of the B200 Trotter-Suzuki engine.
 *
 * This is what a foreign-language binding of the C++ API calls; the Python
 * package trottersuzuki_b200 uses it through ctypes.  It plays the role of the
 * reference's SWIG interface (src/Python/trottersuzuki/trottersuzuki.i), which
 * wraps the same classes (src/trottersuzuki.h:34-602).  Objects are opaque
 * handles; every function returns 0 on success and a non-zero code after a
 * C++ exception, whose message tsh_last_error() returns (thread-local).
 */
#ifndef TS_HOST_H
#define TS_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "ts_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t dim_x, dim_y;
    int32_t global_no_halo_dim_x, global_no_halo_dim_y;
    int32_t start_x, start_y, end_x, end_y;
    int32_t inner_start_x, inner_start_y, inner_end_x, inner_end_y;
    int32_t halo_x, halo_y, periodic_x, periodic_y;
    double length_x, length_y, delta_x, delta_y;
} tsh_lattice_info;

const char *tsh_last_error(void);

/* Lattice2D(dim_x, length_x, dim_y, length_y, periodic_x, periodic_y,
 * angular_velocity, "cartesian") -- src/trottersuzuki.h:110-112 */
int tsh_lattice2d_new(int dim_x, double length_x, int dim_y, double length_y, int periodic_x,
                      int periodic_y, double angular_velocity, void **out);
/* Lattice1D(dim, length, periodic_x, "cartesian") -- src/trottersuzuki.h:74 */
int tsh_lattice1d_new(int dim, double length, int periodic_x, void **out);
/* The same with Lattice::coordinate_system ("cartesian" or "cylindrical",
 * src/model.cpp:32-158). */
int tsh_lattice2d_new_cs(int dim_x, double length_x, int dim_y, double length_y, int periodic_x,
                         int periodic_y, double angular_velocity, const char *coordinate_system,
                         void **out);
int tsh_lattice1d_new_cs(int dim_x, double length_x, int periodic_x,
                         const char *coordinate_system, void **out);
int tsh_lattice_info_get(void *lattice, tsh_lattice_info *out);
int tsh_lattice_free(void *lattice);

/* State(grid) (zero), GaussianState, ExponentialState, SinusoidState
 * -- src/trottersuzuki.h:138,209-336 */
int tsh_state_new(void *lattice, void **out);
/* State(grid, angular_momentum) (src/trottersuzuki.h:138) */
int tsh_state_new_l(void *lattice, int angular_momentum, void **out);
int tsh_gaussian_state_new(void *lattice, double omega_x, double omega_y, double mean_x,
                           double mean_y, double norm, double phase, void **out);
int tsh_exponential_state_new(void *lattice, int n_x, int n_y, double norm, double phase,
                              void **out);
int tsh_sinusoid_state_new(void *lattice, int n_x, int n_y, double norm, double phase, void **out);
/* Pointers to the state's p_real / p_imag tile arrays (dim_y x dim_x). */
int tsh_state_arrays(void *state, double **p_real, double **p_imag);
/* Mark the arrays as changed (the expectation values are recomputed). */
int tsh_state_touch(void *state);
/* norm2, mean_x, mean_xx, mean_y, mean_yy, mean_px, mean_pxpx, mean_py,
 * mean_pypy, mean_lz -- State::get_* (src/trottersuzuki.h:150-159) */
int tsh_state_expectations(void *state, double out[10]);
int tsh_state_free(void *state);
/* State::write_to_file (kind 0, the file `name`), write_particle_density
 * (kind 1, name + "-density"), write_phase (kind 2, name + "-phase") and
 * loadtxt: the reference's text format (src/model.cpp:254-383,636-638,
 * src/common.cpp:161-181). */
int tsh_state_write(void *state, int kind, const char *name);
int tsh_state_loadtxt(void *state, const char *name);

/* Potential(grid, matrix) (the matrix is copied) and HarmonicPotential
 * -- src/trottersuzuki.h:365,410 */
int tsh_potential_matrix_new(void *lattice, const double *matrix, void **out);
int tsh_harmonic_potential_new(void *lattice, double omega_x, double omega_y, double mass,
                               double mean_x, double mean_y, void **out);
int tsh_potential_free(void *potential);

/* Hamiltonian(grid, potential, mass, coupling_a, LeeHuangYang_coupling_a,
 * angular_velocity, rot_coord_x, rot_coord_y) -- src/trottersuzuki.h:446-448 */
int tsh_hamiltonian_new(void *lattice, void *potential, double mass, double coupling_a,
                        double lhy_coupling_a, double angular_velocity, double rot_coord_x,
                        double rot_coord_y, void **out);
int tsh_hamiltonian_free(void *hamiltonian);
/* Hamiltonian2Component(grid, potential, potential_b, mass, mass_b, coupling_a,
 * coupling_ab, coupling_b, omega_r, omega_i, angular_velocity, rot_coord_x,
 * rot_coord_y) -- src/trottersuzuki.h:455-497 (freed with tsh_hamiltonian_free) */
int tsh_hamiltonian2_new(void *lattice, void *potential, void *potential_b, double mass,
                         double mass_b, double coupling_a, double coupling_ab, double coupling_b,
                         double omega_r, double omega_i, double angular_velocity,
                         double rot_coord_x, double rot_coord_y, void **out);

/* Solver(grid, state, hamiltonian, delta_t, kernel_type) and its methods
 * -- src/trottersuzuki.h:541-569 */
int tsh_solver_new(void *lattice, void *state, void *hamiltonian, double delta_t,
                   const char *kernel_type, void **out);
/* Solver(grid, state1, state2, hamiltonian2, delta_t, kernel_type) --
 * src/trottersuzuki.h:554-555 */
int tsh_solver2_new(void *lattice, void *state1, void *state2, void *hamiltonian2,
                    double delta_t, const char *kernel_type, void **out);
int tsh_solver_evolve(void *solver, int iterations, int imag_time);
/* Two components: total, kinetic (1, 2), potential (1, 2), rotational (1, 2),
 * intra-species (1, 2), inter-species, Rabi, squared norm (1, 2). */
int tsh_solver_energies2(void *solver, double out[13]);
/* total, kinetic, potential, rotational, intra-species, Lee-Huang-Yang, squared norm */
int tsh_solver_energies(void *solver, double out[7]);
int tsh_solver_set_exp_potential(void *solver, const double *re, const double *im, int length,
                                 int which);
int tsh_solver_update_parameters(void *solver);
/* Build (or rebuild) the solver's kernel for the time mode as evolve() does
 * (src/solver.cpp:150-171), without a step or a copy back into the State. */
int tsh_solver_prepare(void *solver, int imag_time);
/* The device handle of the solver's kernel (NULL before the first evolve). */
int tsh_solver_kernel_handle(void *solver, void **out);
int tsh_solver_free(void *solver);

/* The step descriptor the solver's kernel would get for this lattice and
 * Hamiltonian (the constants of the reference's CPUBlock constructor,
 * src/cpukernel.cpp:172-272), for the adjoint engine and other direct users
 * of include/ts_b200.h.  No counterpart in the reference. */
int tsh_make_desc(void *lattice, void *hamiltonian, double delta_t, double norm, int imag_time,
                  int precision, ts_b200_desc *out);

#ifdef __cplusplus
}
#endif
#endif
