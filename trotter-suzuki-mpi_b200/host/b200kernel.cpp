// B200Kernel and the GPU reductions used by the model objects.
#include "b200kernel.h"

#include <cmath>
#include <stdexcept>
#include <string>

namespace b200 {

ts_b200_desc make_desc(Lattice *g, Hamiltonian *ham, double dt, double norm, bool imag,
                       int precision, int angular_momentum) {
    return make_species_desc(g, ham, dt, norm, imag, precision, ham->mass, ham->coupling_a,
                             ham->LeeHuangYang_coupling_a, angular_momentum);
}

ts_b200_desc make_species_desc(Lattice *g, Hamiltonian *ham, double dt, double norm, bool imag,
                               int precision, double mass, double coupling, double lhy,
                               int angular_momentum) {
    ts_b200_desc d = {};
    d.dim_x = g->dim_x;
    d.dim_y = g->dim_y;
    d.inner_x0 = g->inner_start_x - g->start_x;
    d.inner_x1 = g->inner_end_x - g->start_x;
    d.inner_y0 = g->inner_start_y - g->start_y;
    d.inner_y1 = g->inner_end_y - g->start_y;
    d.halo_x = g->halo_x;
    d.halo_y = g->halo_y;
    d.periodic_x = g->periods[1];
    d.periodic_y = g->periods[0];
    d.imag_time = imag ? 1 : 0;
    d.precision = precision;
    // step constants exactly as the reference's CPUBlock constructor computes
    // them (src/cpukernel.cpp:185-216)
    const double kx = dt / (4. * mass * g->delta_x * g->delta_x);
    const double ky = dt / (4. * mass * g->delta_y * g->delta_y);
    if (imag) {
        d.a_h = cosh(kx);
        d.b_h = sinh(kx);
        d.a_v = cosh(ky);
        d.b_v = sinh(ky);
    } else {
        d.a_h = cos(kx);
        d.b_h = sin(kx);
        d.a_v = cos(ky);
        d.b_v = sin(ky);
    }
    d.alpha_x = ham->angular_velocity * dt * g->delta_x / (2 * g->delta_y);
    d.alpha_y = ham->angular_velocity * dt * g->delta_y / (2 * g->delta_x);
    d.coupling = coupling * dt;
    d.lhy_coupling = lhy * dt;
    d.rot_offset_x = g->start_x - ham->rot_coord_x;
    d.rot_offset_y = g->start_y - ham->rot_coord_y;
    d.delta_x = g->delta_x;
    d.delta_y = g->delta_y;
    d.norm0 = imag ? norm : 0.0;
    if (g->coordinate_system == "cylindrical") {
        // src/cpukernel.cpp:200-210 (kin_radial) and :669-689 (the mirror's parity)
        d.cylindrical = 1;
        d.kin_radial = dt / (8. * mass * g->delta_x * g->delta_x);
        d.angular_momentum = angular_momentum;
    }
    return d;
}

namespace {

void fail(int status, ts_b200_kernel *h, const char *what) {
    std::string msg = std::string(what) + ": " + ts_b200_status_string(status);
    if (h) {
        const char *e = ts_b200_last_error(h);
        if (e && *e) msg += std::string(" (") + e + ")";
    }
    my_abort(msg);
}

// A short-lived FP64 real-time handle holding a host tile, for reductions.
struct ScratchTile {
    ts_b200_kernel *h = nullptr;
    ScratchTile(Lattice *g, const double *re, const double *im) {
        ts_b200_desc d = {};
        d.dim_x = g->dim_x;
        d.dim_y = g->dim_y;
        d.inner_x0 = g->inner_start_x - g->start_x;
        d.inner_x1 = g->inner_end_x - g->start_x;
        d.inner_y0 = g->inner_start_y - g->start_y;
        d.inner_y1 = g->inner_end_y - g->start_y;
        d.halo_x = g->halo_x;
        d.halo_y = g->halo_y;
        d.precision = TS_B200_FP64;
        d.a_h = d.a_v = 1.0;
        d.delta_x = g->delta_x;
        d.delta_y = g->delta_y;
        // the reductions' coordinates, energy region and norm follow the lattice
        d.cylindrical = g->coordinate_system == "cylindrical" ? 1 : 0;
        int s = ts_b200_create(&d, &h);
        if (s) fail(s, nullptr, "creating a device tile");
        s = ts_b200_set_state(h, re, im, g->dim_x);
        if (s) fail(s, h, "uploading the state");
    }
    ~ScratchTile() { ts_b200_destroy(h); }
};

ts_b200_energy_params params_of(Lattice *g) {
    ts_b200_energy_params p = {};
    p.start_x = g->start_x;
    p.start_y = g->start_y;
    p.global_no_halo_dim_x = g->global_no_halo_dim_x;
    p.global_no_halo_dim_y = g->global_no_halo_dim_y;
    p.length_x = g->length_x;
    p.length_y = g->length_y;
    return p;
}

}  // namespace

Expectations reduce_expectations(Lattice *g, const double *re, const double *im) {
    ScratchTile t(g, re, im);
    ts_b200_energy_params p = params_of(g);
    ts_b200_expectation_result r;
    int s = ts_b200_expectations(t.h, &p, &r);
    if (s) fail(s, t.h, "expectation values");
    Expectations e = {r.norm2,  r.mean_x,  r.mean_xx,   r.mean_y,    r.mean_yy,
                      r.mean_px, r.mean_pxpx, r.mean_py, r.mean_pypy, r.mean_lz};
    return e;
}

ts_b200_energy_result reduce_energies(Lattice *g, const double *re, const double *im,
                                      const double *V, double mass, double coupling,
                                      double lhy, double omega) {
    ScratchTile t(g, re, im);
    ts_b200_energy_params p = params_of(g);
    p.mass = mass;
    p.coupling = coupling;
    p.lhy_coupling = lhy;
    p.angular_velocity = omega;
    ts_b200_energy_result r;
    int s = ts_b200_energies(t.h, V, &p, &r);
    if (s) fail(s, t.h, "energies");
    return r;
}

void reduce_cross_energies(Lattice *g, const double *a_re, const double *a_im, const double *b_re,
                           const double *b_im, double coupling_ab, double omega_r, double omega_i,
                           double *inter, double *rabi) {
    ScratchTile ta(g, a_re, a_im), tb(g, b_re, b_im);
    ts_b200_pair *p = nullptr;
    int s = ts_b200_pair_create(ta.h, tb.h, coupling_ab, omega_r, omega_i, 1.0, &p);
    if (s) fail(s, ta.h, "pairing the tiles for the cross energies");
    s = ts_b200_pair_cross_energies(p, inter, rabi);
    const std::string e = s ? ts_b200_pair_last_error(p) : "";
    ts_b200_pair_destroy(p);
    if (s) my_abort("cross energies: " + e);
}

}  // namespace b200

B200Kernel::B200Kernel(Lattice *grid, State *state, Hamiltonian *ham, double *pot_re,
                       double *pot_im, double dt, double norm, bool imag, int precision)
    : h_(nullptr), dim_x_(grid->dim_x), dim_y_(grid->dim_y), imag_time_(imag) {
    ts_b200_desc d =
        b200::make_desc(grid, ham, dt, norm, imag, precision, state->angular_momentum);
    int s = ts_b200_create(&d, &h_);
    if (s) b200::fail(s, nullptr, "B200Kernel: creating the device tile");
    s = ts_b200_set_state(h_, state->p_real, state->p_imag, grid->dim_x);
    if (s == 0) s = ts_b200_set_exp_potential(h_, pot_re, pot_im, grid->dim_x);
    if (s) {
        const std::string e = ts_b200_last_error(h_);
        ts_b200_destroy(h_);
        h_ = nullptr;
        my_abort("B200Kernel: uploading the state: " + e);
    }
}

B200Kernel::~B200Kernel() { ts_b200_destroy(h_); }

void B200Kernel::check(int status, const char *what) const {
    if (status) b200::fail(status, h_, what);
}

void B200Kernel::run_kernel() { check(ts_b200_step(h_, 0), "B200Kernel::run_kernel"); }

void B200Kernel::finish_halo_exchange() {
    check(ts_b200_halo_exchange(h_), "B200Kernel::finish_halo_exchange");
}

void B200Kernel::evolve(int iterations) {
    check(ts_b200_evolve(h_, iterations), "B200Kernel::evolve");
}

void B200Kernel::steps_with_exchange(int n) {
    for (int i = 0; i < n; ++i) check(ts_b200_step(h_, 1), "B200Kernel::step");
}

void B200Kernel::get_sample(size_t dest_stride, size_t x, size_t y, size_t width, size_t height,
                            double *dest_real, double *dest_imag, double *, double *) const {
    check(ts_b200_get_sample(h_, dest_stride, x, y, width, height, dest_real, dest_imag),
          "B200Kernel::get_sample");
}

double B200Kernel::calculate_squared_norm(bool) const {
    double n = 0;
    check(ts_b200_squared_norm(h_, &n), "B200Kernel::calculate_squared_norm");
    return n;
}

void B200Kernel::update_potential(double *re, double *im, int which) {
    if (which != 0) my_abort("B200Kernel: single-component kernel (potential index 0 only)");
    check(ts_b200_set_exp_potential(h_, re, im, dim_x_), "B200Kernel::update_potential");
}

// ---------------------------------------------------------------- two species
B200PairKernel::B200PairKernel(Lattice *grid, State *state_a, State *state_b,
                               Hamiltonian2Component *ham, double **pot_re, double **pot_im,
                               double dt, double *norm, bool imag, int precision)
    : dim_x_(grid->dim_x) {
    if (ham->angular_velocity != 0.)
        my_abort("B200PairKernel: two components evolve without a rotating frame");
    const ts_b200_desc da = b200::make_species_desc(grid, ham, dt, norm[0], imag, precision,
                                                    ham->mass, ham->coupling_a, 0.);
    const ts_b200_desc db = b200::make_species_desc(grid, ham, dt, norm[1], imag, precision,
                                                    ham->mass_b, ham->coupling_b, 0.);
    State *st[2] = {state_a, state_b};
    const ts_b200_desc *ds[2] = {&da, &db};
    for (int c = 0; c < 2; ++c) {
        int s = ts_b200_create(ds[c], &h_[c]);
        if (s == 0) s = ts_b200_set_state(h_[c], st[c]->p_real, st[c]->p_imag, dim_x_);
        if (s == 0) s = ts_b200_set_exp_potential(h_[c], pot_re[c], pot_im[c], dim_x_);
        if (s) {
            const std::string e = h_[c] ? ts_b200_last_error(h_[c]) : "";
            release();
            my_abort("B200PairKernel: creating species " + std::to_string(c) + ": " + e);
        }
    }
    const int s = ts_b200_pair_create(h_[0], h_[1], ham->coupling_ab, ham->omega_r,
                                      ham->omega_i, dt, &p_);
    if (s) {
        release();
        my_abort(std::string("B200PairKernel: pairing the species: ") + ts_b200_status_string(s));
    }
}

void B200PairKernel::release() {
    ts_b200_pair_destroy(p_);
    p_ = nullptr;
    for (int c = 0; c < 2; ++c) {
        ts_b200_destroy(h_[c]);
        h_[c] = nullptr;
    }
}

B200PairKernel::~B200PairKernel() { release(); }

void B200PairKernel::check(int status, const char *what) const {
    if (status) my_abort(std::string(what) + ": " + ts_b200_status_string(status) + " (" +
                         ts_b200_pair_last_error(p_) + ")");
}

void B200PairKernel::run_kernel() {
    check(ts_b200_pair_step_species(p_, state_index_), "B200PairKernel::run_kernel");
}

void B200PairKernel::finish_halo_exchange() {
    check(ts_b200_halo_exchange(h_[state_index_]), "B200PairKernel::finish_halo_exchange");
}

void B200PairKernel::wait_for_completion() { state_index_ = 1 - state_index_; }

void B200PairKernel::rabi_coupling(double var, double) {
    check(ts_b200_pair_rabi(p_, var), "B200PairKernel::rabi_coupling");
}

void B200PairKernel::normalization() {
    check(ts_b200_pair_normalize(p_), "B200PairKernel::normalization");
}

void B200PairKernel::steps(int n, bool final_steps) {
    check(ts_b200_pair_steps(p_, n, final_steps ? 1 : 0), "B200PairKernel::steps");
}

void B200PairKernel::get_sample(size_t dest_stride, size_t x, size_t y, size_t width,
                                size_t height, double *dest_real, double *dest_imag,
                                double *dest_real2, double *dest_imag2) const {
    int s = ts_b200_get_sample(h_[0], dest_stride, x, y, width, height, dest_real, dest_imag);
    if (s == 0 && dest_real2)
        s = ts_b200_get_sample(h_[1], dest_stride, x, y, width, height, dest_real2, dest_imag2);
    check(s, "B200PairKernel::get_sample");
}

double B200PairKernel::calculate_squared_norm(bool) const {
    double n = 0;
    check(ts_b200_squared_norm(h_[state_index_], &n), "B200PairKernel::calculate_squared_norm");
    return n;
}

void B200PairKernel::update_potential(double *re, double *im, int which) {
    if (which != 0 && which != 1) my_abort("B200PairKernel: potential index 0 or 1");
    check(ts_b200_set_exp_potential(h_[which], re, im, dim_x_), "B200PairKernel::update_potential");
}
