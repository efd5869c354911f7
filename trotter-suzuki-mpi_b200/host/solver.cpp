// Solver: the evolution driver of the B200 engine.
//
// Same protocol as the reference's Solver (src/solver.cpp:24-242): the
// exponential tables are built on the host with std::exp(complex) exactly as
// the reference does (src/solver.cpp:74-109), the kernel is (re)built when the
// time mode or the parameters change, and evolve() runs the iterations then
// copies the tile back into the State.  With the B200 kernel the iterations
// are queued as fused steps (CUDA-graph replay) instead of the per-step
// virtual calls; a time-dependent potential still re-uploads its table before
// the step that needs it.  Energies are the reference's functional
// (src/solver.cpp:244-564) reduced on the GPU in FP64 from the State arrays.
#include <cstring>
#include <iostream>
#include <vector>

#include "b200kernel.h"
#include "trottersuzuki.h"

Solver::Solver(Lattice *_grid, State *_state, Hamiltonian *_ham, double _delta_t,
               string _kernel_type)
    : grid(_grid), state(_state), state_b(NULL), hamiltonian(_ham), current_evolution_time(0),
      imag_time(false), delta_t(_delta_t), single_component(true), kernel_type(_kernel_type),
      kernel(NULL), has_parameters_changed(false), energy_expected_values_updated(false),
      is_python(false), kernel_state_current(false) {
    const size_t n = size_t(grid->dim_x) * grid->dim_y;
    external_pot_real = new double *[2];
    external_pot_imag = new double *[2];
    external_pot_real[0] = new double[n];
    external_pot_imag[0] = new double[n];
    external_pot_real[1] = NULL;
    external_pot_imag[1] = NULL;
    norm2[0] = norm2[1] = 0;
}

Solver::Solver(Lattice *_grid, State *s1, State *s2, Hamiltonian2Component *_ham,
               double _delta_t, string _kernel_type)
    : grid(_grid), state(s1), state_b(s2), hamiltonian(_ham), current_evolution_time(0),
      imag_time(false), delta_t(_delta_t), single_component(false), kernel_type(_kernel_type),
      kernel(NULL), has_parameters_changed(false), energy_expected_values_updated(false),
      is_python(false), kernel_state_current(false) {
    const size_t n = size_t(grid->dim_x) * grid->dim_y;
    external_pot_real = new double *[2];
    external_pot_imag = new double *[2];
    for (int i = 0; i < 2; ++i) {
        external_pot_real[i] = new double[n];
        external_pot_imag[i] = new double[n];
    }
    norm2[0] = norm2[1] = 0;
}

Solver::~Solver() {
    for (int i = 0; i < 2; ++i) {
        delete[] external_pot_real[i];
        delete[] external_pot_imag[i];
    }
    delete[] external_pot_real;
    delete[] external_pot_imag;
    delete kernel;
}

void Solver::initialize_exp_potential(double dt, int which) {
    Potential *pot = which == 0 ? hamiltonian->potential
                                : static_cast<Hamiltonian2Component *>(hamiltonian)->potential_b;
    const bool cyl = grid->coordinate_system == "cylindrical";
    for (int y = 0; y < grid->dim_y; ++y)
        for (int x = 0; x < grid->dim_x; ++x) {
            double v = pot->get_value(x, y);
            // the centrifugal term l^2 / (2 m r^2) (src/solver.cpp:85-96)
            if (cyl)
                v += which == 0 ? hamiltonian->azimuthal_potential(x, state->angular_momentum)
                                : static_cast<Hamiltonian2Component *>(hamiltonian)
                                      ->azimuthal_potential_b(x, state_b->angular_momentum);
            const complex<double> e = imag_time ? exp(complex<double>(-dt * v, 0.))
                                                : exp(complex<double>(0., -dt * v));
            external_pot_real[which][size_t(y) * grid->dim_x + x] = real(e);
            external_pot_imag[which][size_t(y) * grid->dim_x + x] = imag(e);
        }
}

void Solver::set_exp_potential(double *re, int re_len, double *im, int im_len, int which) {
    is_python = true;
    memcpy(external_pot_real[which], re, sizeof(double) * re_len);
    memcpy(external_pot_imag[which], im, sizeof(double) * im_len);
    // The reference's CPU kernel reads these arrays in place, so a new table
    // takes effect at the next step; the device kernel holds its own copy.
    if (kernel != NULL && (which == 0 || !single_component))
        kernel->update_potential(external_pot_real[which], external_pot_imag[which], which);
}

void Solver::init_kernel() {
    delete kernel;
    kernel = NULL;
    int precision;
    if (kernel_type == "gpu" || kernel_type == "b200")
        precision = TS_B200_FP64;
    else if (kernel_type == "gpu_fp32" || kernel_type == "b200_fp32")
        precision = TS_B200_FP32;
    else
        my_abort("Unknown kernel: \"" + kernel_type +
                 "\" (this build provides the B200 kernel: \"gpu\", \"gpu_fp32\")");
    if (single_component)
        kernel = new B200Kernel(grid, state, hamiltonian, external_pot_real[0],
                                external_pot_imag[0], delta_t, norm2[0], imag_time, precision);
    else
        kernel = new B200PairKernel(grid, state, state_b,
                                    static_cast<Hamiltonian2Component *>(hamiltonian),
                                    external_pot_real, external_pot_imag, delta_t, norm2,
                                    imag_time, precision);
    kernel_state_current = true;
}

void Solver::prepare_kernel(bool _imag_time) {
    if (_imag_time != imag_time || kernel == NULL || has_parameters_changed) {
        imag_time = _imag_time;
        if (imag_time) {
            initialize_exp_potential(delta_t, 0);
            norm2[0] = state->get_squared_norm();
            if (!single_component) {
                initialize_exp_potential(delta_t, 1);
                norm2[1] = state_b->get_squared_norm();
            }
        } else {
            if (!is_python) initialize_exp_potential(delta_t, 0);
            if (!single_component) initialize_exp_potential(delta_t, 1);
        }
        init_kernel();
        has_parameters_changed = false;
    }
}

void Solver::evolve(int iterations, bool _imag_time) {
    prepare_kernel(_imag_time);
    bool soft_update = false;
    if (iterations < 0) {
        iterations = -iterations;
        soft_update = true;
    }
    if (!single_component) {
        evolve_two_components(iterations, soft_update);
        return;
    }
    B200Kernel *bk = static_cast<B200Kernel *>(kernel);
    // Steps are queued in runs; a run is flushed when the potential changes
    // before the next step (the reference re-tabulates V there,
    // src/solver.cpp:187-192).  All flushed steps refresh the halo; the last
    // step of the call does not (src/solver.cpp:203-209).
    int pending = 0;
    for (int i = 0; i < iterations; ++i) {
        if (i > 0 && hamiltonian->potential->update(current_evolution_time)) {
            bk->steps_with_exchange(pending);
            pending = 0;
            if (!is_python) initialize_exp_potential(delta_t, 0);
            kernel->update_potential(external_pot_real[0], external_pot_imag[0], 0);
        }
        ++pending;
        current_evolution_time += delta_t;
    }
    bk->evolve(pending);
    if (!soft_update) {
        kernel->get_sample(grid->dim_x, 0, 0, grid->dim_x, grid->dim_y, state->p_real,
                           state->p_imag);
    }
    state->expected_values_updated = false;
    energy_expected_values_updated = false;
}

// Two components (src/solver.cpp:172-240): a Rabi half step first (every
// call from C++, only at t = 0 from Python), then the steps of the pair in
// runs between potential updates, the last one the call's last.
void Solver::evolve_two_components(int iterations, bool soft_update) {
    B200PairKernel *pk = static_cast<B200PairKernel *>(kernel);
    Hamiltonian2Component *h2 = static_cast<Hamiltonian2Component *>(hamiltonian);
    if (!is_python || current_evolution_time == 0) kernel->rabi_coupling(0.5, delta_t);
    int pending = 0;
    for (int i = 0; i < iterations; ++i) {
        if (i > 0) {
            const bool ua = hamiltonian->potential->update(current_evolution_time);
            const bool ub = h2->potential_b->update(current_evolution_time);
            if ((ua || ub) && pending > 0) {
                pk->steps(pending, false);
                pending = 0;
            }
            if (ua) {
                if (!is_python) initialize_exp_potential(delta_t, 0);
                kernel->update_potential(external_pot_real[0], external_pot_imag[0], 0);
            }
            if (ub) {
                if (!is_python) initialize_exp_potential(delta_t, 1);
                kernel->update_potential(external_pot_real[1], external_pot_imag[1], 1);
            }
        }
        ++pending;
        current_evolution_time += delta_t;
    }
    pk->steps(pending, true);
    if (!soft_update) {
        kernel->get_sample(grid->dim_x, 0, 0, grid->dim_x, grid->dim_y, state->p_real,
                           state->p_imag, state_b->p_real, state_b->p_imag);
        state_b->expected_values_updated = false;
    }
    state->expected_values_updated = false;
    energy_expected_values_updated = false;
}

void Solver::calculate_energy_expected_values(void) {
    if (!single_component) {
        calculate_energies_two_components();
        return;
    }
    std::vector<double> V(size_t(grid->dim_x) * grid->dim_y);
    for (int y = 0; y < grid->dim_y; ++y)
        for (int x = 0; x < grid->dim_x; ++x) {
            double v = hamiltonian->potential->get_value(x, y);
            if (grid->coordinate_system == "cylindrical")
                v += hamiltonian->azimuthal_potential(x, state->angular_momentum);
            V[size_t(y) * grid->dim_x + x] = v;
        }
    ts_b200_energy_result r = b200::reduce_energies(
        grid, state->p_real, state->p_imag, V.data(), hamiltonian->mass, hamiltonian->coupling_a,
        hamiltonian->LeeHuangYang_coupling_a, hamiltonian->angular_velocity);
    norm2[0] = r.norm2;
    kinetic_energy[0] = r.kinetic;
    potential_energy[0] = r.potential;
    rotational_energy[0] = r.rotational;
    intra_species_energy[0] = r.intra;
    LeeHuangYang_energy = r.lhy;
    total_energy = r.total;
    tot_kinetic_energy = r.kinetic;
    tot_potential_energy = r.potential;
    tot_rotational_energy = r.rotational;
    tot_intra_species_energy = r.intra;
    energy_expected_values_updated = true;
}

// src/solver.cpp:244-564 with two components: each species' terms as for one
// (its own mass, g, potential), the cross terms from the pair, and the totals
// of src/solver.cpp:544-558.
void Solver::calculate_energies_two_components(void) {
    Hamiltonian2Component *h2 = static_cast<Hamiltonian2Component *>(hamiltonian);
    const size_t n = size_t(grid->dim_x) * grid->dim_y;
    std::vector<double> Va(n), Vb(n);
    for (int y = 0; y < grid->dim_y; ++y)
        for (int x = 0; x < grid->dim_x; ++x) {
            Va[size_t(y) * grid->dim_x + x] = h2->potential->get_value(x, y);
            Vb[size_t(y) * grid->dim_x + x] = h2->potential_b->get_value(x, y);
        }
    const ts_b200_energy_result ra =
        b200::reduce_energies(grid, state->p_real, state->p_imag, Va.data(), h2->mass,
                              h2->coupling_a, h2->LeeHuangYang_coupling_a, h2->angular_velocity);
    const ts_b200_energy_result rb =
        b200::reduce_energies(grid, state_b->p_real, state_b->p_imag, Vb.data(), h2->mass_b,
                              h2->coupling_b, 0., h2->angular_velocity);
    b200::reduce_cross_energies(grid, state->p_real, state->p_imag, state_b->p_real,
                                state_b->p_imag, h2->coupling_ab, h2->omega_r, h2->omega_i,
                                &inter_species_energy, &rabi_energy);
    const ts_b200_energy_result *r[2] = {&ra, &rb};
    for (int c = 0; c < 2; ++c) {
        norm2[c] = r[c]->norm2;
        kinetic_energy[c] = r[c]->kinetic;
        potential_energy[c] = r[c]->potential;
        rotational_energy[c] = r[c]->rotational;
        intra_species_energy[c] = r[c]->intra;
    }
    LeeHuangYang_energy = ra.lhy;
    total_energy = kinetic_energy[0] + potential_energy[0] + intra_species_energy[0] +
                   rotational_energy[0] + kinetic_energy[1] + potential_energy[1] +
                   intra_species_energy[1] + rotational_energy[1] + inter_species_energy +
                   rabi_energy;
    tot_kinetic_energy = kinetic_energy[0] + kinetic_energy[1];
    tot_potential_energy = potential_energy[0] + potential_energy[1];
    tot_rotational_energy = rotational_energy[0] + rotational_energy[1];
    tot_intra_species_energy = intra_species_energy[0] + intra_species_energy[1];
    energy_expected_values_updated = true;
}

double Solver::get_total_energy(void) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return total_energy;
}

// which: 1 first component, 2 second, 3 total (src/solver.cpp:572-594).
static double pick(size_t which, bool single, double first, double second, double total) {
    if (which == 3) return total;
    if (which == 1) return first;
    if (which == 2) {
        if (single) {
            cout << "The system has only one component. No input have to be given\n";
            return 0;
        }
        return second;
    }
    cout << "Input may be 1, 2 or 3\n";
    return 0;
}

double Solver::get_squared_norm(size_t which) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return pick(which, single_component, norm2[0], norm2[1],
                single_component ? norm2[0] : norm2[0] + norm2[1]);
}

double Solver::get_kinetic_energy(size_t which) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return pick(which, single_component, kinetic_energy[0], kinetic_energy[1], tot_kinetic_energy);
}

double Solver::get_potential_energy(size_t which) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return pick(which, single_component, potential_energy[0], potential_energy[1],
                tot_potential_energy);
}

double Solver::get_rotational_energy(size_t which) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return pick(which, single_component, rotational_energy[0], rotational_energy[1],
                tot_rotational_energy);
}

double Solver::get_intra_species_energy(size_t which) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return pick(which, single_component, intra_species_energy[0], intra_species_energy[1],
                tot_intra_species_energy);
}

double Solver::get_LeeHuangYang_energy(void) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    return LeeHuangYang_energy;
}

double Solver::get_inter_species_energy(void) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    if (!single_component) return inter_species_energy;
    cout << "The system has only one component\n";
    return 0;
}

double Solver::get_rabi_energy(void) {
    if (!energy_expected_values_updated) calculate_energy_expected_values();
    if (!single_component) return rabi_energy;
    cout << "The system has only one component\n";
    return 0;
}

void Solver::update_parameters() { has_parameters_changed = true; }
