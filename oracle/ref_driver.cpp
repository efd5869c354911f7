// Test-infrastructure driver around the reference's own CPU implementation.
//
// This file is compiled together with the reference's unmodified C++ sources
// (src/{common,cpukernel,cpucartesian,cpucylindrical,model,solver}.cpp of
// trotter-suzuki-mpi 1.6.2, read in place, never copied) into
// oracle/_ref/libtsref*.so by oracle/build_ref.sh.  It is a checker and a CPU
// baseline only: tests/, bench.py's reference arm and the golden-fixture
// generator load it; no product code path does.
//
// The driver builds the reference objects through the reference's public API
// (Lattice1D/Lattice2D, State/GaussianState/ExponentialState, Potential/
// HarmonicPotential, Hamiltonian, Solver with kernel_type "cpu", or "gpu" in
// the build that also compiles the reference's CUDA kernel,
// src/trottersuzuki.h:34-597), runs Solver::evolve (src/solver.cpp:150-242)
// and returns the tile, the energies (src/solver.cpp:566-680) and the state
// expectation values (src/model.cpp:385-536).
#include <algorithm>
#include <cstring>
#include <cstdio>
#include <chrono>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "trottersuzuki.h"

extern "C" {

struct tsref_config {
    int dim_x, dim_y;            // dim_y == 0 selects Lattice1D
    double length_x, length_y;
    int periodic_x, periodic_y;
    double lattice_angular_velocity;   // decides the halo width (src/model.cpp:140-141)
    int init_kind;               // 0: arrays given, 1: GaussianState, 2: ExponentialState
    double g_omega_x, g_omega_y, g_mean_x, g_mean_y, g_norm, g_phase;
    int e_nx, e_ny;
    int pot_kind;                // 0: matrix given, 1: HarmonicPotential, 2: none (V = 0)
    double h_omega_x, h_omega_y, h_mass, h_mean_x, h_mean_y;
    double mass, coupling, lhy_coupling, angular_velocity, rot_coord_x, rot_coord_y;
    int force_rotation_periodic; // fill the fields the Hamiltonian leaves unset for periodic+rotation
    double delta_t;
    int n_segments;              // evolve() calls made in order
    int seg_iterations[8];
    int seg_imag[8];
    int omp_threads;             // <= 0: leave OpenMP's default
    int kernel_gpu;              // 1: kernel_type "gpu", the reference's CUDA kernel
                                 // (CC2Kernel, src/gpukernel.cu; libtsref_gpu.so only)
    int cylindrical;             // 1: coordinate_system "cylindrical" (2D lattices)
    int angular_momentum;        // of the State (init_kind 0)
};

struct tsref_result {
    int dim_x, dim_y;            // tile dims of the reference lattice
    int halo_x, halo_y;
    int start_x, start_y, inner_start_x, inner_start_y, inner_end_x, inner_end_y;
    double delta_x, delta_y;
    double total_energy, kinetic_energy, potential_energy, rotational_energy;
    double intra_energy, lhy_energy, squared_norm;
    double mean_x, mean_xx, mean_y, mean_yy, mean_px, mean_pxpx, mean_py, mean_pypy, mean_lz;
    double state_norm;
    double initial_total_energy, initial_squared_norm;
    double seconds;              // wall time of the evolve() calls only
    double seg_seconds[8];       // wall time of each evolve() call
};

static char g_err[512];

const char *tsref_last_error(void) { return g_err; }

// Query the reference lattice geometry without evolving.
int tsref_geometry(const tsref_config *cfg, tsref_result *res) {
    try {
        Lattice *grid;
        if (cfg->dim_y == 0)
            grid = new Lattice1D(cfg->dim_x, cfg->length_x, cfg->periodic_x != 0);
        else
            grid = new Lattice2D(cfg->dim_x, cfg->length_x, cfg->dim_y, cfg->length_y,
                                 cfg->periodic_x != 0, cfg->periodic_y != 0,
                                 cfg->lattice_angular_velocity,
                                 cfg->cylindrical ? "cylindrical" : "cartesian");
        res->dim_x = grid->dim_x; res->dim_y = grid->dim_y;
        res->halo_x = grid->halo_x; res->halo_y = grid->halo_y;
        res->start_x = grid->start_x; res->start_y = grid->start_y;
        res->inner_start_x = grid->inner_start_x; res->inner_start_y = grid->inner_start_y;
        res->inner_end_x = grid->inner_end_x; res->inner_end_y = grid->inner_end_y;
        res->delta_x = grid->delta_x; res->delta_y = grid->delta_y;
        delete grid;
    } catch (std::exception &e) {
        snprintf(g_err, sizeof g_err, "%s", e.what());
        return 1;
    }
    return 0;
}

// Run the reference.  psi_re/psi_im (tile sized, row-major, stride dim_x) are
// the initial state when init_kind == 0 and receive the final state.
// potential (tile sized) is read when pot_kind == 0.
int tsref_run(const tsref_config *cfg, double *psi_re, double *psi_im,
              const double *potential, tsref_result *res) {
    try {
#ifdef _OPENMP
        if (cfg->omp_threads > 0) omp_set_num_threads(cfg->omp_threads);
#endif
        Lattice *grid;
        Lattice1D *g1 = nullptr;
        Lattice2D *g2 = nullptr;
        if (cfg->dim_y == 0) {
            g1 = new Lattice1D(cfg->dim_x, cfg->length_x, cfg->periodic_x != 0);
            grid = g1;
        } else {
            g2 = new Lattice2D(cfg->dim_x, cfg->length_x, cfg->dim_y, cfg->length_y,
                               cfg->periodic_x != 0, cfg->periodic_y != 0,
                               cfg->lattice_angular_velocity,
                               cfg->cylindrical ? "cylindrical" : "cartesian");
            grid = g2;
        }
        const size_t n = size_t(grid->dim_x) * grid->dim_y;
        State *state;
        std::vector<double> own_re, own_im;
        if (cfg->init_kind == 0) {
            own_re.assign(psi_re, psi_re + n);
            own_im.assign(psi_im, psi_im + n);
            state = new State(grid, cfg->angular_momentum, own_re.data(), own_im.data());
        } else if (cfg->init_kind == 1) {
            if (g2) state = new GaussianState(g2, cfg->g_omega_x, cfg->g_omega_y, cfg->g_mean_x,
                                              cfg->g_mean_y, cfg->g_norm, cfg->g_phase);
            else state = new GaussianState(g1, cfg->g_omega_x, cfg->g_mean_x, cfg->g_norm, cfg->g_phase);
        } else {
            if (g2) state = new ExponentialState(g2, cfg->e_nx, cfg->e_ny, cfg->g_norm, cfg->g_phase);
            else state = new ExponentialState(g1, cfg->e_nx, cfg->g_norm, cfg->g_phase);
        }
        Potential *pot = nullptr;
        std::vector<double> own_pot;
        if (cfg->pot_kind == 0) {
            own_pot.assign(potential, potential + n);
            pot = new Potential(grid, own_pot.data());
        } else if (cfg->pot_kind == 1) {
            if (!g2) throw std::runtime_error("HarmonicPotential needs a 2D lattice");
            pot = new HarmonicPotential(g2, cfg->h_omega_x, cfg->h_omega_y, cfg->h_mass,
                                        cfg->h_mean_x, cfg->h_mean_y);
        }
        Hamiltonian *ham = new Hamiltonian(grid, pot, cfg->mass, cfg->coupling, cfg->lhy_coupling,
                                           cfg->angular_velocity, cfg->rot_coord_x, cfg->rot_coord_y);
        if (cfg->force_rotation_periodic) {
            // The reference returns early for periodic + rotation
            // (src/model.cpp:936-940) and leaves these public fields unset;
            // set them with the closed-boundary formulas (src/model.cpp:950-964).
            ham->rot_coord_x = (grid->global_dim_x - grid->periods[1] * 2 * grid->halo_x) * 0.5 +
                               cfg->rot_coord_x / grid->delta_x;
            ham->rot_coord_y = (grid->global_dim_y - grid->periods[0] * 2 * grid->halo_y) * 0.5 +
                               cfg->rot_coord_y / grid->delta_y;
            ham->potential = pot ? pot : new Potential(grid, const_potential);
        }
        Solver *solver = new Solver(grid, state, ham, cfg->delta_t,
                                    cfg->kernel_gpu ? "gpu" : "cpu");
        res->initial_total_energy = solver->get_total_energy();
        res->initial_squared_norm = solver->get_squared_norm();
        auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < cfg->n_segments; ++s) {
            auto ts = std::chrono::steady_clock::now();
            solver->evolve(cfg->seg_iterations[s], cfg->seg_imag[s] != 0);
            res->seg_seconds[s] =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
        }
        auto t1 = std::chrono::steady_clock::now();
        res->seconds = std::chrono::duration<double>(t1 - t0).count();
        res->total_energy = solver->get_total_energy();
        res->kinetic_energy = solver->get_kinetic_energy();
        res->potential_energy = solver->get_potential_energy();
        res->rotational_energy = solver->get_rotational_energy();
        res->intra_energy = solver->get_intra_species_energy();
        res->lhy_energy = solver->get_LeeHuangYang_energy();
        res->squared_norm = solver->get_squared_norm();
        if (g2) {
            res->mean_x = state->get_mean_x();
            res->mean_xx = state->get_mean_xx();
            res->mean_y = state->get_mean_y();
            res->mean_yy = state->get_mean_yy();
            res->mean_px = state->get_mean_px();
            res->mean_pxpx = state->get_mean_pxpx();
            res->mean_py = state->get_mean_py();
            res->mean_pypy = state->get_mean_pypy();
            res->mean_lz = state->get_mean_angular_momentum();
        }
        res->state_norm = state->get_squared_norm();
        res->dim_x = grid->dim_x; res->dim_y = grid->dim_y;
        res->halo_x = grid->halo_x; res->halo_y = grid->halo_y;
        res->start_x = grid->start_x; res->start_y = grid->start_y;
        res->inner_start_x = grid->inner_start_x; res->inner_start_y = grid->inner_start_y;
        res->inner_end_x = grid->inner_end_x; res->inner_end_y = grid->inner_end_y;
        res->delta_x = grid->delta_x; res->delta_y = grid->delta_y;
        memcpy(psi_re, state->p_real, n * sizeof(double));
        memcpy(psi_im, state->p_imag, n * sizeof(double));
        delete solver;
        // With force_rotation_periodic the reference constructor returned
        // before setting its ownership flag, so the Hamiltonian is leaked on
        // purpose instead of running a destructor on an unset field.
        if (!cfg->force_rotation_periodic) delete ham;
        delete pot;
        delete state;
        delete grid;
    } catch (std::exception &e) {
        snprintf(g_err, sizeof g_err, "%s", e.what());
        return 1;
    }
    return 0;
}

// State text I/O of the reference (src/model.cpp:254-383,636-638): load = 0
// writes the state given in re/im (kind 0 state, 1 density, 2 phase) to
// `name`; load = 1 reads `name` into a fresh State and returns its tile.
int tsref_state_io(const tsref_config *cfg, double *re, double *im, int kind, const char *name,
                   int load) {
    try {
        Lattice *grid;
        if (cfg->dim_y == 0)
            grid = new Lattice1D(cfg->dim_x, cfg->length_x, cfg->periodic_x != 0);
        else
            grid = new Lattice2D(cfg->dim_x, cfg->length_x, cfg->dim_y, cfg->length_y,
                                 cfg->periodic_x != 0, cfg->periodic_y != 0,
                                 cfg->lattice_angular_velocity,
                                 cfg->cylindrical ? "cylindrical" : "cartesian");
        const size_t n = size_t(grid->dim_x) * grid->dim_y;
        std::vector<double> r(n, 0.0), i(n, 0.0);
        if (!load) {
            std::copy(re, re + n, r.begin());
            std::copy(im, im + n, i.begin());
        }
        State *st = new State(grid, 0, r.data(), i.data());
        if (load) {
            std::vector<char> nm(name, name + strlen(name) + 1);
            st->loadtxt(nm.data());
            std::copy(r.begin(), r.end(), re);
            std::copy(i.begin(), i.end(), im);
        } else if (kind == 0) {
            st->write_to_file(name);
        } else if (kind == 1) {
            st->write_particle_density(name);
        } else {
            st->write_phase(name);
        }
        delete st;
        delete grid;
    } catch (std::exception &e) {
        snprintf(g_err, sizeof g_err, "%s", e.what());
        return 1;
    }
    return 0;
}

// Two components: Hamiltonian2Component and the two-state Solver
// (src/trottersuzuki.h:455-497,541-569).  Lattice and time fields come from
// `cfg` (arrays given for both states, matrix potentials for both); the
// second component's constants from `c2`.
struct tsref_config2 {
    double mass_b, coupling_b, coupling_ab, omega_r, omega_i;
};

struct tsref_result2 {
    double total_energy;
    double kinetic[2], potential[2], rotational[2], intra[2];
    double inter_species, rabi;
    double squared_norm[2];
    double seconds;
    double seg_seconds[8];
};

int tsref_run2(const tsref_config *cfg, const tsref_config2 *c2, double *a_re, double *a_im,
               double *b_re, double *b_im, const double *pot_a, const double *pot_b,
               tsref_result2 *res) {
    try {
#ifdef _OPENMP
        if (cfg->omp_threads > 0) omp_set_num_threads(cfg->omp_threads);
#endif
        Lattice2D *grid = new Lattice2D(cfg->dim_x, cfg->length_x, cfg->dim_y, cfg->length_y,
                                        cfg->periodic_x != 0, cfg->periodic_y != 0, 0.);
        const size_t n = size_t(grid->dim_x) * grid->dim_y;
        std::vector<double> ar(a_re, a_re + n), ai(a_im, a_im + n), br(b_re, b_re + n),
            bi(b_im, b_im + n), va(pot_a, pot_a + n), vb(pot_b, pot_b + n);
        State *sa = new State(grid, 0, ar.data(), ai.data());
        State *sb = new State(grid, 0, br.data(), bi.data());
        Potential *pa = new Potential(grid, va.data());
        Potential *pb = new Potential(grid, vb.data());
        Hamiltonian2Component *ham = new Hamiltonian2Component(
            grid, pa, pb, cfg->mass, c2->mass_b, cfg->coupling, c2->coupling_ab, c2->coupling_b,
            c2->omega_r, c2->omega_i, 0., 0., 0.);
        Solver *solver = new Solver(grid, sa, sb, ham, cfg->delta_t,
                                    cfg->kernel_gpu ? "gpu" : "cpu");
        auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < cfg->n_segments; ++s) {
            auto ts = std::chrono::steady_clock::now();
            solver->evolve(cfg->seg_iterations[s], cfg->seg_imag[s] != 0);
            res->seg_seconds[s] =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
        }
        res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        res->total_energy = solver->get_total_energy();
        for (int c = 0; c < 2; ++c) {
            res->kinetic[c] = solver->get_kinetic_energy(c + 1);
            res->potential[c] = solver->get_potential_energy(c + 1);
            res->rotational[c] = solver->get_rotational_energy(c + 1);
            res->intra[c] = solver->get_intra_species_energy(c + 1);
            res->squared_norm[c] = solver->get_squared_norm(c + 1);
        }
        res->inter_species = solver->get_inter_species_energy();
        res->rabi = solver->get_rabi_energy();
        memcpy(a_re, sa->p_real, n * sizeof(double));
        memcpy(a_im, sa->p_imag, n * sizeof(double));
        memcpy(b_re, sb->p_real, n * sizeof(double));
        memcpy(b_im, sb->p_imag, n * sizeof(double));
        delete solver;
        delete ham;
        delete pa;
        delete pb;
        delete sa;
        delete sb;
        delete grid;
    } catch (std::exception &e) {
        snprintf(g_err, sizeof g_err, "%s", e.what());
        return 1;
    }
    return 0;
}

}  // extern "C"
