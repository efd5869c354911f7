// The reference's GPU kernel class, CC2Kernel (declared by trotter-suzuki-mpi
// 1.6.2 in src/kernel.h when built with -DCUDA), implemented on the B200
// engine's C ABI (include/ts_b200.h) instead of src/gpukernel.cu.
//
// This is the binding a maintainer of the reference adds to run its own,
// unmodified Solver on a B200: compile the reference's sources with -DCUDA
// and this file in place of src/gpukernel.cu / src/gpucartesian.cu, and link
// libtsb200.so.  Solver::init_kernel (src/solver.cpp:118-148) then builds this
// class for kernel_type "gpu", and Solver::evolve (src/solver.cpp:150-242)
// drives it through the ITrotterKernel virtuals (src/trottersuzuki.h:502-520):
//
//   run_kernel_on_halo, start_halo_exchange   nothing to do: one fused launch
//                                             advances the whole tile
//   run_kernel                                ts_b200_step (the fused step; for
//                                             two components, the current
//                                             species' step)
//   finish_halo_exchange                      ts_b200_halo_exchange (periodic
//                                             halo refresh of the tile)
//   wait_for_completion                       nothing for one component (the
//                                             imaginary-time renormalisation is
//                                             applied when the tile is next
//                                             read); the next species for two
//   rabi_coupling, normalization              ts_b200_pair_rabi / _normalize
//   get_sample, calculate_squared_norm        ts_b200_get_sample / _squared_norm
//   update_potential                          ts_b200_set_exp_potential
//   cpy_first_positive_to_first_negative      nothing: the mirrored axis column
//                                             is written by the step itself
//
// The reference's CC2Kernel keeps its device state in private members; this
// implementation keeps the engine handles in a table keyed by the object, so
// the class layout stays the one src/kernel.h declares.  Errors go through
// the reference's my_abort (src/common.cpp:104-115), as CUDA errors do in the
// reference's kernel.  Solver::init_kernel refuses a rotating frame for
// kernel_type "gpu" (src/solver.cpp:132-134) before this class is built.
#include <cmath>
#include <map>
#include <mutex>
#include <string>

#include "common.h"
#include "kernel.h"
#include "trottersuzuki.h"
#include "ts_b200.h"

namespace {

struct Engine {
    ts_b200_kernel *h[2] = {nullptr, nullptr};
    ts_b200_pair *pair = nullptr;
    int species = 1;
    int current = 0;  // species the next run_kernel advances (two components)
    int dim_x = 0;
};

std::mutex g_mutex;
std::map<const void *, Engine> g_engines;

Engine &engine(const void *k) {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = g_engines.find(k);
    if (it == g_engines.end()) my_abort("CC2Kernel (B200): no engine for this kernel");
    return it->second;
}

void check(int status, ts_b200_kernel *h, const char *what) {
    if (!status) return;
    std::string msg = std::string("CC2Kernel (B200) ") + what + ": " + ts_b200_status_string(status);
    if (h) msg += std::string(" (") + ts_b200_last_error(h) + ")";
    my_abort(msg);
}

// The step descriptor of one species: the reference CPUBlock's constants
// (src/cpukernel.cpp:185-216) from the reference's Lattice and Hamiltonian.
ts_b200_desc species_desc(Lattice *g, Hamiltonian *ham, double dt, double norm, bool imag,
                          double mass, double coupling, double lhy, int angular_momentum) {
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
    d.precision = TS_B200_FP64;
    const double kx = dt / (4. * mass * g->delta_x * g->delta_x);
    const double ky = dt / (4. * mass * g->delta_y * g->delta_y);
    d.a_h = imag ? cosh(kx) : cos(kx);
    d.b_h = imag ? sinh(kx) : sin(kx);
    d.a_v = imag ? cosh(ky) : cos(ky);
    d.b_v = imag ? sinh(ky) : sin(ky);
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
        d.cylindrical = 1;
        d.kin_radial = dt / (8. * mass * g->delta_x * g->delta_x);
        d.angular_momentum = angular_momentum;
    }
    return d;
}

void release(Engine &e) {
    ts_b200_pair_destroy(e.pair);
    e.pair = nullptr;
    for (auto &h : e.h) {
        ts_b200_destroy(h);
        h = nullptr;
    }
}

}  // namespace

CC2Kernel::CC2Kernel(Lattice *grid, State *state, Hamiltonian *hamiltonian,
                     double *_external_pot_real, double *_external_pot_imag, double delta_t,
                     double _norm, bool _imag_time) {
    Engine e;
    e.dim_x = grid->dim_x;
    const ts_b200_desc d = species_desc(grid, hamiltonian, delta_t, _norm, _imag_time,
                                        hamiltonian->mass, hamiltonian->coupling_a,
                                        hamiltonian->LeeHuangYang_coupling_a,
                                        state->angular_momentum);
    int s = ts_b200_create(&d, &e.h[0]);
    check(s, nullptr, "creating the device tile");
    s = ts_b200_set_state(e.h[0], state->p_real, state->p_imag, grid->dim_x);
    if (!s) s = ts_b200_set_exp_potential(e.h[0], _external_pot_real, _external_pot_imag, grid->dim_x);
    if (s) {
        const std::string msg = ts_b200_last_error(e.h[0]);
        release(e);
        my_abort("CC2Kernel (B200) uploading the state and table: " + msg);
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    g_engines[this] = e;
}

CC2Kernel::CC2Kernel(Lattice *grid, State *state1, State *state2,
                     Hamiltonian2Component *hamiltonian, double **_external_pot_real,
                     double **_external_pot_imag, double delta_t, double *_norm,
                     bool _imag_time) {
    Engine e;
    e.species = 2;
    e.dim_x = grid->dim_x;
    const ts_b200_desc da = species_desc(grid, hamiltonian, delta_t, _norm[0], _imag_time,
                                         hamiltonian->mass, hamiltonian->coupling_a, 0., 0);
    const ts_b200_desc db = species_desc(grid, hamiltonian, delta_t, _norm[1], _imag_time,
                                         hamiltonian->mass_b, hamiltonian->coupling_b, 0., 0);
    State *st[2] = {state1, state2};
    const ts_b200_desc *ds[2] = {&da, &db};
    for (int c = 0; c < 2; ++c) {
        int s = ts_b200_create(ds[c], &e.h[c]);
        if (!s) s = ts_b200_set_state(e.h[c], st[c]->p_real, st[c]->p_imag, grid->dim_x);
        if (!s)
            s = ts_b200_set_exp_potential(e.h[c], _external_pot_real[c], _external_pot_imag[c],
                                          grid->dim_x);
        if (s) {
            const std::string msg = e.h[c] ? ts_b200_last_error(e.h[c]) : "";
            release(e);
            my_abort("CC2Kernel (B200) creating species " + std::to_string(c) + ": " + msg);
        }
    }
    const int s = ts_b200_pair_create(e.h[0], e.h[1], hamiltonian->coupling_ab,
                                      hamiltonian->omega_r, hamiltonian->omega_i, delta_t, &e.pair);
    if (s) {
        release(e);
        my_abort(std::string("CC2Kernel (B200) pairing the species: ") + ts_b200_status_string(s));
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    g_engines[this] = e;
}

CC2Kernel::~CC2Kernel() {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto it = g_engines.find(this);
    if (it != g_engines.end()) {
        release(it->second);
        g_engines.erase(it);
    }
}

void CC2Kernel::run_kernel_on_halo() {}

void CC2Kernel::run_kernel() {
    Engine &e = engine(this);
    if (e.species == 1) {
        check(ts_b200_step(e.h[0], 0), e.h[0], "run_kernel");
    } else {
        const int s = ts_b200_pair_step_species(e.pair, e.current);
        if (s) my_abort(std::string("CC2Kernel (B200) run_kernel: ") + ts_b200_pair_last_error(e.pair));
    }
}

void CC2Kernel::wait_for_completion() {
    Engine &e = engine(this);
    if (e.species == 2) e.current = 1 - e.current;
}

void CC2Kernel::get_sample(size_t dest_stride, size_t x, size_t y, size_t width, size_t height,
                           double *dest_real, double *dest_imag, double *dest_real2,
                           double *dest_imag2) const {
    Engine &e = engine(this);
    check(ts_b200_get_sample(e.h[0], dest_stride, x, y, width, height, dest_real, dest_imag),
          e.h[0], "get_sample");
    if (e.species == 2 && dest_real2)
        check(ts_b200_get_sample(e.h[1], dest_stride, x, y, width, height, dest_real2, dest_imag2),
              e.h[1], "get_sample");
}

void CC2Kernel::normalization() {
    Engine &e = engine(this);
    if (e.species != 2) return;
    const int s = ts_b200_pair_normalize(e.pair);
    if (s) my_abort(std::string("CC2Kernel (B200) normalization: ") + ts_b200_pair_last_error(e.pair));
}

void CC2Kernel::rabi_coupling(double var, double) {
    Engine &e = engine(this);
    if (e.species != 2) return;
    const int s = ts_b200_pair_rabi(e.pair, var);
    if (s) my_abort(std::string("CC2Kernel (B200) rabi_coupling: ") + ts_b200_pair_last_error(e.pair));
}

double CC2Kernel::calculate_squared_norm(bool) const {
    Engine &e = engine(this);
    double n = 0.0;
    ts_b200_kernel *h = e.h[e.species == 2 ? e.current : 0];
    check(ts_b200_squared_norm(h, &n), h, "calculate_squared_norm");
    return n;
}

void CC2Kernel::update_potential(double *_external_pot_real, double *_external_pot_imag,
                                 int which) {
    Engine &e = engine(this);
    if (which < 0 || which >= e.species) my_abort("CC2Kernel (B200) update_potential: index");
    check(ts_b200_set_exp_potential(e.h[which], _external_pot_real, _external_pot_imag, e.dim_x),
          e.h[which], "update_potential");
}

void CC2Kernel::cpy_first_positive_to_first_negative() {}

void CC2Kernel::start_halo_exchange() {}

void CC2Kernel::finish_halo_exchange() {
    Engine &e = engine(this);
    ts_b200_kernel *h = e.h[e.species == 2 ? e.current : 0];
    check(ts_b200_halo_exchange(h), h, "finish_halo_exchange");
}
