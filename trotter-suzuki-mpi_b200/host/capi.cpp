// Flat C ABI over the C++ host layer (include/ts_host.h).
#include <exception>
#include <string>
#include <vector>

#include "b200kernel.h"
#include "trottersuzuki.h"
#include "ts_host.h"

namespace {

thread_local std::string g_err;

template <class F>
int guard(F f) {
    try {
        f();
        return 0;
    } catch (std::exception &e) {
        g_err = e.what();
        return 1;
    } catch (...) {
        g_err = "unknown C++ exception";
        return 1;
    }
}

// A Potential built from a copied matrix owns that copy.
struct OwnedMatrixPotential : public Potential {
    std::vector<double> storage;
    OwnedMatrixPotential(Lattice *g, const double *m)
        : Potential(g, (double *)nullptr),
          storage(m, m + size_t(g->dim_x) * g->dim_y) {
        delete[] matrix;  // the zeroed matrix Potential allocated
        matrix = storage.data();
        self_init = false;
    }
};

}  // namespace

extern "C" {

const char *tsh_last_error(void) { return g_err.c_str(); }

int tsh_lattice2d_new(int nx, double lx, int ny, double ly, int px, int py, double omega,
                      void **out) {
    return guard([&] { *out = new Lattice2D(nx, lx, ny, ly, px != 0, py != 0, omega); });
}

int tsh_lattice1d_new(int n, double l, int px, void **out) {
    return guard([&] { *out = new Lattice1D(n, l, px != 0); });
}

int tsh_lattice2d_new_cs(int nx, double lx, int ny, double ly, int px, int py, double omega,
                         const char *cs, void **out) {
    return guard([&] { *out = new Lattice2D(nx, lx, ny, ly, px != 0, py != 0, omega, cs); });
}

int tsh_lattice1d_new_cs(int n, double l, int px, const char *cs, void **out) {
    return guard([&] { *out = new Lattice1D(n, l, px != 0, cs); });
}

int tsh_lattice_info_get(void *lp, tsh_lattice_info *o) {
    return guard([&] {
        Lattice *g = static_cast<Lattice *>(lp);
        o->dim_x = g->dim_x;
        o->dim_y = g->dim_y;
        o->global_no_halo_dim_x = g->global_no_halo_dim_x;
        o->global_no_halo_dim_y = g->global_no_halo_dim_y;
        o->start_x = g->start_x;
        o->start_y = g->start_y;
        o->end_x = g->end_x;
        o->end_y = g->end_y;
        o->inner_start_x = g->inner_start_x;
        o->inner_start_y = g->inner_start_y;
        o->inner_end_x = g->inner_end_x;
        o->inner_end_y = g->inner_end_y;
        o->halo_x = g->halo_x;
        o->halo_y = g->halo_y;
        o->periodic_x = g->periods[1];
        o->periodic_y = g->periods[0];
        o->length_x = g->length_x;
        o->length_y = g->length_y;
        o->delta_x = g->delta_x;
        o->delta_y = g->delta_y;
    });
}

int tsh_lattice_free(void *lp) {
    return guard([&] { delete static_cast<Lattice *>(lp); });
}

static Lattice2D *as2d(void *lp) {
    Lattice *g = static_cast<Lattice *>(lp);
    if (g->dim_y == 1 && g->global_no_halo_dim_y == 1 && g->length_y == 0)
        return nullptr;  // a Lattice1D
    return static_cast<Lattice2D *>(g);
}

int tsh_state_new(void *lp, void **out) {
    return guard([&] { *out = new State(static_cast<Lattice *>(lp)); });
}

int tsh_state_write(void *sp, int kind, const char *name) {
    return guard([&] {
        State *st = static_cast<State *>(sp);
        if (kind == 0) st->write_to_file(name);
        else if (kind == 1) st->write_particle_density(name);
        else if (kind == 2) st->write_phase(name);
        else my_abort("tsh_state_write: kind 0 (state), 1 (density) or 2 (phase)");
    });
}

int tsh_state_loadtxt(void *sp, const char *name) {
    return guard([&] { static_cast<State *>(sp)->loadtxt(const_cast<char *>(name)); });
}

int tsh_state_new_l(void *lp, int angular_momentum, void **out) {
    return guard([&] { *out = new State(static_cast<Lattice *>(lp), angular_momentum); });
}

int tsh_gaussian_state_new(void *lp, double wx, double wy, double mx, double my, double norm,
                           double phase, void **out) {
    return guard([&] {
        Lattice2D *g2 = as2d(lp);
        if (g2)
            *out = new GaussianState(g2, wx, wy, mx, my, norm, phase);
        else
            *out = new GaussianState(static_cast<Lattice1D *>(lp), wx, mx, norm, phase);
    });
}

int tsh_exponential_state_new(void *lp, int nx, int ny, double norm, double phase, void **out) {
    return guard([&] {
        Lattice2D *g2 = as2d(lp);
        if (g2)
            *out = new ExponentialState(g2, nx, ny, norm, phase);
        else
            *out = new ExponentialState(static_cast<Lattice1D *>(lp), nx, norm, phase);
    });
}

int tsh_sinusoid_state_new(void *lp, int nx, int ny, double norm, double phase, void **out) {
    return guard([&] {
        Lattice2D *g2 = as2d(lp);
        if (g2)
            *out = new SinusoidState(g2, nx, ny, norm, phase);
        else
            *out = new SinusoidState(static_cast<Lattice1D *>(lp), nx, norm, phase);
    });
}

int tsh_state_arrays(void *sp, double **re, double **im) {
    return guard([&] {
        State *s = static_cast<State *>(sp);
        *re = s->p_real;
        *im = s->p_imag;
    });
}

int tsh_state_touch(void *sp) {
    return guard([&] { static_cast<State *>(sp)->expected_values_updated = false; });
}

int tsh_state_expectations(void *sp, double out[10]) {
    return guard([&] {
        State *s = static_cast<State *>(sp);
        out[0] = s->get_squared_norm();
        out[1] = s->get_mean_x();
        out[2] = s->get_mean_xx();
        out[3] = s->get_mean_y();
        out[4] = s->get_mean_yy();
        out[5] = s->get_mean_px();
        out[6] = s->get_mean_pxpx();
        out[7] = s->get_mean_py();
        out[8] = s->get_mean_pypy();
        out[9] = s->get_mean_angular_momentum();
    });
}

int tsh_state_free(void *sp) {
    return guard([&] { delete static_cast<State *>(sp); });
}

int tsh_potential_matrix_new(void *lp, const double *m, void **out) {
    return guard([&] { *out = new OwnedMatrixPotential(static_cast<Lattice *>(lp), m); });
}

int tsh_harmonic_potential_new(void *lp, double wx, double wy, double mass, double mx, double my,
                               void **out) {
    return guard([&] {
        Lattice2D *g2 = as2d(lp);
        if (!g2) my_abort("HarmonicPotential needs a Lattice2D");
        *out = new HarmonicPotential(g2, wx, wy, mass, mx, my);
    });
}

int tsh_potential_free(void *pp) {
    return guard([&] { delete static_cast<Potential *>(pp); });
}

int tsh_hamiltonian_new(void *lp, void *pp, double mass, double ga, double glhy, double omega,
                        double rx, double ry, void **out) {
    return guard([&] {
        *out = new Hamiltonian(static_cast<Lattice *>(lp), static_cast<Potential *>(pp), mass, ga,
                               glhy, omega, rx, ry);
    });
}

int tsh_hamiltonian2_new(void *lp, void *pp, void *pbp, double mass, double mass_b, double ga,
                         double gab, double gb, double omega_r, double omega_i, double omega,
                         double rx, double ry, void **out) {
    return guard([&] {
        *out = new Hamiltonian2Component(static_cast<Lattice *>(lp), static_cast<Potential *>(pp),
                                         static_cast<Potential *>(pbp), mass, mass_b, ga, gab, gb,
                                         omega_r, omega_i, omega, rx, ry);
    });
}

int tsh_hamiltonian_free(void *hp) {
    return guard([&] { delete static_cast<Hamiltonian *>(hp); });
}

int tsh_solver_new(void *lp, void *sp, void *hp, double dt, const char *kt, void **out) {
    return guard([&] {
        *out = new Solver(static_cast<Lattice *>(lp), static_cast<State *>(sp),
                          static_cast<Hamiltonian *>(hp), dt, kt ? kt : "gpu");
    });
}

int tsh_solver2_new(void *lp, void *sp, void *sbp, void *hp, double delta_t,
                    const char *kernel_type, void **out) {
    return guard([&] {
        *out = new Solver(static_cast<Lattice *>(lp), static_cast<State *>(sp),
                          static_cast<State *>(sbp), static_cast<Hamiltonian2Component *>(hp),
                          delta_t, kernel_type);
    });
}

int tsh_solver_energies2(void *svp, double out[13]) {
    return guard([&] {
        Solver *s = static_cast<Solver *>(svp);
        out[0] = s->get_total_energy();
        out[1] = s->get_kinetic_energy(1);
        out[2] = s->get_kinetic_energy(2);
        out[3] = s->get_potential_energy(1);
        out[4] = s->get_potential_energy(2);
        out[5] = s->get_rotational_energy(1);
        out[6] = s->get_rotational_energy(2);
        out[7] = s->get_intra_species_energy(1);
        out[8] = s->get_intra_species_energy(2);
        out[9] = s->get_inter_species_energy();
        out[10] = s->get_rabi_energy();
        out[11] = s->get_squared_norm(1);
        out[12] = s->get_squared_norm(2);
    });
}

int tsh_solver_evolve(void *svp, int iterations, int imag) {
    return guard([&] { static_cast<Solver *>(svp)->evolve(iterations, imag != 0); });
}

int tsh_solver_prepare(void *svp, int imag) {
    return guard([&] { static_cast<Solver *>(svp)->prepare_kernel(imag != 0); });
}

int tsh_solver_energies(void *svp, double out[7]) {
    return guard([&] {
        Solver *s = static_cast<Solver *>(svp);
        out[0] = s->get_total_energy();
        out[1] = s->get_kinetic_energy();
        out[2] = s->get_potential_energy();
        out[3] = s->get_rotational_energy();
        out[4] = s->get_intra_species_energy();
        out[5] = s->get_LeeHuangYang_energy();
        out[6] = s->get_squared_norm();
    });
}

int tsh_solver_set_exp_potential(void *svp, const double *re, const double *im, int n, int w) {
    return guard([&] {
        static_cast<Solver *>(svp)->set_exp_potential(const_cast<double *>(re), n,
                                                      const_cast<double *>(im), n, w);
    });
}

int tsh_solver_update_parameters(void *svp) {
    return guard([&] { static_cast<Solver *>(svp)->update_parameters(); });
}

int tsh_solver_kernel_handle(void *svp, void **out) {
    return guard([&] {
        ITrotterKernel *k = static_cast<Solver *>(svp)->get_kernel();
        B200Kernel *b = dynamic_cast<B200Kernel *>(k);
        *out = b ? b->handle() : nullptr;
    });
}

int tsh_make_desc(void *lattice, void *hamiltonian, double delta_t, double norm, int imag_time,
                  int precision, ts_b200_desc *out) {
    return guard([&] {
        *out = b200::make_desc(static_cast<Lattice *>(lattice), static_cast<Hamiltonian *>(hamiltonian),
                               delta_t, norm, imag_time != 0, precision);
    });
}

int tsh_solver_free(void *svp) {
    return guard([&] { delete static_cast<Solver *>(svp); });
}

}  // extern "C"
