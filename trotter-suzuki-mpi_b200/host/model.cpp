// Lattice, State, Potential and Hamiltonian of the B200 engine.
//
// The behaviour follows the reference's model objects (src/model.cpp,
// src/common.cpp of trotter-suzuki-mpi 1.6.2) for one process: lattice
// geometry and halo (src/model.cpp:32-158, src/common.cpp:83-102),
// cell-centred coordinates (src/common.cpp:25-81), the analytic initial
// states (src/model.cpp:640-748) and potentials (src/model.cpp:826-926).
// The formulas are evaluated in the same order as the reference so that the
// same inputs give bit-identical tiles.  Expectation values are reduced on the
// GPU (ts_b200_expectations) from the host arrays.
#include <cmath>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <vector>

#include "b200kernel.h"
#include "trottersuzuki.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

void my_abort(string err) { throw std::runtime_error(err); }

double const_potential(double) { return 0.; }
double const_potential(double, double) { return 0.; }

namespace {

// Tile borders of one process along one axis (src/common.cpp:83-102 with a
// single process): a periodic axis gets a halo on both sides.
void borders(int length, int halo, bool periodic, int *start, int *end, int *inner_start,
             int *inner_end) {
    *inner_start = 0;
    *start = periodic ? -halo : 0;
    *end = length + (periodic ? halo : 0);
    *inner_end = length;
}

void check_coordinate_system(const string &cs, bool periodic_x) {
    if (cs != "cartesian" && cs != "cylindrical")
        my_abort("The coordinate system you have chosen is not implemented.");
    if (cs == "cylindrical" && periodic_x)
        my_abort("You cannot choose periodic boundary on the radial axis.");
}

}  // namespace

// ----------------------------------------------------------------- lattices
Lattice1D::Lattice1D(int dim, double length, bool periodic_x_axis, string cs) {
    check_coordinate_system(cs, periodic_x_axis);
    if (dim < 1) my_abort("Lattice1D: dim must be positive");
    coordinate_system = cs;
    length_x = length;
    length_y = 0;
    if (cs == "cylindrical") {
        dim += 1;
        delta_x = length_x / (double(dim) - 0.5);
    } else {
        delta_x = length_x / double(dim);
    }
    delta_y = 1.0;
    periods[0] = 0;
    periods[1] = periodic_x_axis ? 1 : 0;
    mpi_procs = 1;
    mpi_rank = 0;
    mpi_dims[0] = mpi_dims[1] = 1;
    mpi_coords[0] = mpi_coords[1] = 0;
    halo_x = 4;
    halo_y = 0;
    global_dim_x = dim + periods[1] * 2 * halo_x;
    global_dim_y = 1;
    global_no_halo_dim_x = dim;
    global_no_halo_dim_y = 1;
    borders(dim, halo_x, periods[1] != 0, &start_x, &end_x, &inner_start_x, &inner_end_x);
    if (cs == "cylindrical") inner_start_x += 1;
    dim_x = end_x - start_x;
    start_y = 0;
    end_y = 1;
    inner_start_y = 0;
    inner_end_y = 1;
    dim_y = 1;
}

Lattice2D::Lattice2D(int dim, double length, bool px, bool py, double omega, string cs) {
    init(dim, length, dim, length, px, py, omega, cs);
}

Lattice2D::Lattice2D(int dx, double lx, int dy, double ly, bool px, bool py, double omega,
                     string cs) {
    init(dx, lx, dy, ly, px, py, omega, cs);
}

void Lattice2D::init(int nx, double lx, int ny, double ly, bool px, bool py, double omega,
                     string cs) {
    check_coordinate_system(cs, px);
    if (nx < 1 || ny < 1) my_abort("Lattice2D: dimensions must be positive");
    length_x = lx;
    length_y = ly;
    if (cs == "cylindrical") {
        nx += 1;
        delta_x = length_x / (double(nx) - 0.5);
    } else {
        delta_x = length_x / double(nx);
    }
    delta_y = length_y / double(ny);
    coordinate_system = cs;
    periods[0] = py ? 1 : 0;
    periods[1] = px ? 1 : 0;
    mpi_procs = 1;
    mpi_rank = 0;
    mpi_dims[0] = mpi_dims[1] = 1;
    mpi_coords[0] = mpi_coords[1] = 0;
    halo_x = halo_y = (omega == 0. ? 4 : 8);
    global_dim_x = nx + periods[1] * 2 * halo_x;
    global_dim_y = ny + periods[0] * 2 * halo_y;
    global_no_halo_dim_x = nx;
    global_no_halo_dim_y = ny;
    borders(nx, halo_x, px, &start_x, &end_x, &inner_start_x, &inner_end_x);
    if (cs == "cylindrical") inner_start_x += 1;
    borders(ny, halo_y, py, &start_y, &end_y, &inner_start_y, &inner_end_y);
    dim_x = end_x - start_x;
    dim_y = end_y - start_y;
}

// --------------------------------------------------------------- coordinates
void map_lattice_to_coordinate_space(Lattice *g, int x_in, double *x_out) {
    if (g->coordinate_system == "cartesian") {
        double idx = g->start_x * g->delta_x + 0.5 * g->delta_x + x_in * g->delta_x;
        const double x_c = g->global_no_halo_dim_x * g->delta_x * 0.5;
        if (idx - x_c < -g->length_x * 0.5) idx += g->length_x;
        if (idx - x_c > g->length_x * 0.5) idx -= g->length_x;
        *x_out = idx - x_c;
    } else {
        *x_out = g->start_x * g->delta_x + x_in * g->delta_x - 0.5 * g->delta_x;
    }
}

void map_lattice_to_coordinate_space(Lattice *g, int x_in, int y_in, double *x_out,
                                     double *y_out) {
    double idy = g->start_y * g->delta_y + 0.5 * g->delta_y + y_in * g->delta_y;
    const double y_c = g->global_no_halo_dim_y * g->delta_y * 0.5;
    if (idy - y_c < -g->length_y * 0.5) idy += g->length_y;
    if (idy - y_c > g->length_y * 0.5) idy -= g->length_y;
    *y_out = idy - y_c;
    map_lattice_to_coordinate_space(g, x_in, x_out);
}

// -------------------------------------------------------------------- State
State::State(Lattice *_grid, int _angular_momentum, double *_p_real, double *_p_imag)
    : grid(_grid), angular_momentum(_angular_momentum) {
    expected_values_updated = false;
    const size_t n = size_t(grid->dim_x) * grid->dim_y;
    self_init = (_p_real == 0);
    p_real = _p_real ? _p_real : new double[n]();
    p_imag = _p_imag ? _p_imag : new double[n]();
}

State::State(const State &o)
    : grid(o.grid), angular_momentum(o.angular_momentum),
      expected_values_updated(o.expected_values_updated), self_init(true), mean_X(o.mean_X),
      mean_XX(o.mean_XX), mean_Y(o.mean_Y), mean_YY(o.mean_YY), mean_Px(o.mean_Px),
      mean_PxPx(o.mean_PxPx), mean_Py(o.mean_Py), mean_PyPy(o.mean_PyPy),
      mean_angular_momentum(o.mean_angular_momentum), norm2(o.norm2) {
    const size_t n = size_t(grid->dim_x) * grid->dim_y;
    p_real = new double[n];
    p_imag = new double[n];
    std::copy(o.p_real, o.p_real + n, p_real);
    std::copy(o.p_imag, o.p_imag + n, p_imag);
}

State::~State() {
    if (self_init) {
        delete[] p_real;
        delete[] p_imag;
    }
}

void State::init_state(complex<double> (*f)(double)) {
    double x = 0;
    for (int i = 0; i < grid->dim_x; ++i) {
        map_lattice_to_coordinate_space(grid, i, &x);
        const complex<double> v = f(x);
        p_real[i] = real(v);
        p_imag[i] = imag(v);
    }
    expected_values_updated = false;
}

void State::init_state(complex<double> (*f)(double, double)) {
    double x = 0, y = 0;
    for (int j = 0; j < grid->dim_y; ++j)
        for (int i = 0; i < grid->dim_x; ++i) {
            map_lattice_to_coordinate_space(grid, i, j, &x, &y);
            const complex<double> v = f(x, y);
            p_real[j * grid->dim_x + i] = real(v);
            p_imag[j * grid->dim_x + i] = imag(v);
        }
    expected_values_updated = false;
}

void State::imprint(complex<double> (*f)(double)) {
    double x = 0;
    for (int i = 0; i < grid->dim_x; ++i) {
        map_lattice_to_coordinate_space(grid, i, &x);
        const complex<double> v = f(x);
        const double re = p_real[i];
        p_real[i] = re * real(v) - p_imag[i] * imag(v);
        p_imag[i] = re * imag(v) + p_imag[i] * real(v);
    }
    expected_values_updated = false;
}

void State::imprint(complex<double> (*f)(double, double)) {
    double x = 0, y = 0;
    for (int j = 0; j < grid->dim_y; ++j)
        for (int i = 0; i < grid->dim_x; ++i) {
            map_lattice_to_coordinate_space(grid, i, j, &x, &y);
            const complex<double> v = f(x, y);
            const size_t k = size_t(j) * grid->dim_x + i;
            const double re = p_real[k];
            p_real[k] = re * real(v) - p_imag[k] * imag(v);
            p_imag[k] = re * imag(v) + p_imag[k] * real(v);
        }
    expected_values_updated = false;
}

// Text format of State::write_to_file: one line per lattice row, "(re,im) "
// per cell, lattice rows without halo.  On a periodic tile the halo is filled
// from the opposite side, as the reference's loader does (src/model.cpp:254-322).
void State::loadtxt(char *file_name) {
    std::ifstream in(file_name);
    if (!in) my_abort(string("cannot open ") + file_name);
    const int nx = grid->global_no_halo_dim_x, ny = grid->global_no_halo_dim_y;
    const int ox = grid->inner_start_x - grid->start_x, oy = grid->inner_start_y - grid->start_y;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            complex<double> v;
            in >> v;
            if (!in) my_abort(string("short read in ") + file_name);
            // every tile cell that shows lattice cell (i, j), halo copies included
            for (int ty = j + oy - ny; ty < grid->dim_y; ty += ny) {
                if (ty < 0) continue;
                for (int tx = i + ox - nx; tx < grid->dim_x; tx += nx) {
                    if (tx < 0) continue;
                    const size_t k = size_t(ty) * grid->dim_x + tx;
                    p_real[k] = real(v);
                    p_imag[k] = imag(v);
                }
            }
        }
    expected_values_updated = false;
}

double *State::get_particle_density(double *out) {
    const int w = grid->inner_end_x - grid->inner_start_x;
    const int h = grid->inner_end_y - grid->inner_start_y;
    double *d = out ? out : new double[size_t(w) * h];
    const int ox = grid->inner_start_x - grid->start_x, oy = grid->inner_start_y - grid->start_y;
    for (int j = 0; j < h; ++j)
        for (int i = 0; i < w; ++i) {
            const size_t k = size_t(j + oy) * grid->dim_x + (i + ox);
            d[size_t(j) * w + i] = p_real[k] * p_real[k] + p_imag[k] * p_imag[k];
        }
    return d;
}

double *State::get_phase(double *out) {
    const int w = grid->inner_end_x - grid->inner_start_x;
    const int h = grid->inner_end_y - grid->inner_start_y;
    double *d = out ? out : new double[size_t(w) * h];
    const int ox = grid->inner_start_x - grid->start_x, oy = grid->inner_start_y - grid->start_y;
    for (int j = 0; j < h; ++j)
        for (int i = 0; i < w; ++i) {
            const size_t k = size_t(j + oy) * grid->dim_x + (i + ox);
            const double n = sqrt(p_real[k] * p_real[k] + p_imag[k] * p_imag[k]);
            d[size_t(j) * w + i] =
                n == 0 ? 0 : acos(p_real[k] / n) * ((p_imag[k] >= 0) - (p_imag[k] < 0));
        }
    return d;
}

void State::calculate_expected_values(void) {
    b200::Expectations e = b200::reduce_expectations(grid, p_real, p_imag);
    norm2 = e.norm2;
    mean_X = e.mean_x;
    mean_XX = e.mean_xx;
    mean_Y = e.mean_y;
    mean_YY = e.mean_yy;
    mean_Px = e.mean_px;
    mean_PxPx = e.mean_pxpx;
    mean_Py = e.mean_py;
    mean_PyPy = e.mean_pypy;
    mean_angular_momentum = e.mean_lz;
    expected_values_updated = true;
}

double State::get_expected_value(string op) {
    if (!expected_values_updated) calculate_expected_values();
    if (op == "L_z") return mean_angular_momentum;
    if (op == "X") return mean_X;
    if (op == "X^2") return mean_XX;
    if (op == "Y") return mean_Y;
    if (op == "Y^2") return mean_YY;
    if (op == "P_x") return mean_Px;
    if (op == "P_x^2") return mean_PxPx;
    if (op == "P_y") return mean_Py;
    if (op == "P_y^2") return mean_PyPy;
    std::cerr << "The expected value of the operator " << op << " is not calculated.\n"
              << "Available operators are: L_z, X, X^2, Y, Y^2, P_x, P_x^2, P_y, P_y^2.\n";
    return std::numeric_limits<double>::quiet_NaN();
}

#define TS_STATE_GETTER(name, field)                           \
    double State::name(void) {                                 \
        if (!expected_values_updated) calculate_expected_values(); \
        return field;                                          \
    }
TS_STATE_GETTER(get_squared_norm, norm2)
TS_STATE_GETTER(get_mean_x, mean_X)
TS_STATE_GETTER(get_mean_xx, mean_XX)
TS_STATE_GETTER(get_mean_y, mean_Y)
TS_STATE_GETTER(get_mean_yy, mean_YY)
TS_STATE_GETTER(get_mean_px, mean_Px)
TS_STATE_GETTER(get_mean_pxpx, mean_PxPx)
TS_STATE_GETTER(get_mean_py, mean_Py)
TS_STATE_GETTER(get_mean_pypy, mean_PyPy)
TS_STATE_GETTER(get_mean_angular_momentum, mean_angular_momentum)
#undef TS_STATE_GETTER

// The reference's single-process stamp / print_complex_matrix
// (src/model.cpp:636-638, src/common.cpp:161-170,254-265): the file is named
// by the argument itself; each lattice row is a line of "(re,im) " with the
// stream's default formatting (6 significant digits), so files written here
// and by the reference are the same byte for byte.  The rows and columns are
// the lattice without its periodic halo; on a cylindrical lattice the columns
// are the inner ones (the reference's own width there, global_dim_x, runs one
// cell past each row).
void State::write_to_file(string filename) {
    std::ofstream out(filename.c_str(), std::ios::out | std::ios::trunc);
    const int ox = grid->inner_start_x - grid->start_x, oy = grid->inner_start_y - grid->start_y;
    const int w = grid->coordinate_system == "cylindrical"
                      ? grid->inner_end_x - grid->inner_start_x
                      : grid->global_dim_x - 2 * grid->periods[1] * grid->halo_x;
    const int h = grid->global_dim_y - 2 * grid->periods[0] * grid->halo_y;
    for (int j = 0; j < h; ++j) {
        for (int i = 0; i < w; ++i) {
            const size_t k = size_t(j + oy) * grid->dim_x + (i + ox);
            out << "(" << p_real[k] << "," << p_imag[k] << ") ";
        }
        out << std::endl;
    }
}

// print_matrix of src/common.cpp:172-181: "v " per cell, default formatting.
static void write_matrix(const string &name, const double *m, int w, int h) {
    std::ofstream out(name.c_str(), std::ios::out | std::ios::trunc);
    for (int j = 0; j < h; ++j) {
        for (int i = 0; i < w; ++i) out << m[size_t(j) * w + i] << " ";
        out << std::endl;
    }
}

void State::write_particle_density(string prefix) {
    double *d = get_particle_density();
    write_matrix(prefix + "-density", d, grid->inner_end_x - grid->inner_start_x,
                 grid->inner_end_y - grid->inner_start_y);
    delete[] d;
}

void State::write_phase(string prefix) {
    double *d = get_phase();
    write_matrix(prefix + "-phase", d, grid->inner_end_x - grid->inner_start_x,
                 grid->inner_end_y - grid->inner_start_y);
    delete[] d;
}

// ------------------------------------------------------------ analytic states
ExponentialState::ExponentialState(Lattice1D *g, int nx, double nm, double ph, double *re,
                                   double *im)
    : State(g, 0, re, im), n_x(nx), n_y(0), norm(nm), phase(ph) {
    double x = 0;
    for (int i = 0; i < grid->dim_x; ++i) {
        map_lattice_to_coordinate_space(grid, i, &x);
        const complex<double> v = exp_state(x, 0.);
        p_real[i] = real(v);
        p_imag[i] = imag(v);
    }
}

ExponentialState::ExponentialState(Lattice2D *g, int nx, int ny, double nm, double ph,
                                   double *re, double *im)
    : State(g, 0, re, im), n_x(nx), n_y(ny), norm(nm), phase(ph) {
    double x = 0, y = 0;
    for (int j = 0; j < grid->dim_y; ++j)
        for (int i = 0; i < grid->dim_x; ++i) {
            map_lattice_to_coordinate_space(grid, i, j, &x, &y);
            const complex<double> v = exp_state(x, y);
            p_real[size_t(j) * grid->dim_x + i] = real(v);
            p_imag[size_t(j) * grid->dim_x + i] = imag(v);
        }
}

complex<double> ExponentialState::exp_state(double x, double y) {
    const double lx = grid->global_no_halo_dim_x * grid->delta_x;
    const double ly = grid->global_no_halo_dim_y * grid->delta_y;
    return sqrt(norm / (lx * ly)) * exp(complex<double>(0., phase)) *
           exp(complex<double>(0., 2 * M_PI * double(n_x) / lx * x +
                                       2 * M_PI * double(n_y) / ly * y));
}

GaussianState::GaussianState(Lattice1D *g, double wx, double mx, double nm, double ph,
                             double *re, double *im)
    : State(g, 0, re, im), mean_x(mx), mean_y(0.), omega_x(wx), omega_y(1.), norm(nm),
      phase(ph) {
    double x = 0;
    for (int i = 0; i < grid->dim_x; ++i) {
        map_lattice_to_coordinate_space(grid, i, &x);
        const complex<double> v = gauss_state(x, 0.);
        p_real[i] = real(v);
        p_imag[i] = imag(v);
    }
}

GaussianState::GaussianState(Lattice2D *g, double wx, double wy, double mx, double my,
                             double nm, double ph, double *re, double *im)
    : State(g, 0, re, im), mean_x(mx), mean_y(my), omega_x(wx), omega_y(wy), norm(nm),
      phase(ph) {
    if (omega_y == -1.) omega_y = omega_x;
    double x = 0, y = 0;
    for (int j = 0; j < grid->dim_y; ++j)
        for (int i = 0; i < grid->dim_x; ++i) {
            map_lattice_to_coordinate_space(grid, i, j, &x, &y);
            const complex<double> v = gauss_state(x, y);
            p_real[size_t(j) * grid->dim_x + i] = real(v);
            p_imag[size_t(j) * grid->dim_x + i] = imag(v);
        }
}

complex<double> GaussianState::gauss_state(double x, double y) {
    const double amp = sqrt(norm * sqrt(omega_x * omega_y) / M_PI);
    const double arg = -(omega_x * pow(x - mean_x, 2.0) + omega_y * pow(y - mean_y, 2.0)) * 0.5;
    return complex<double>(amp * exp(arg), 0.) * exp(complex<double>(0., phase));
}

SinusoidState::SinusoidState(Lattice1D *g, int nx, double nm, double ph, double *re, double *im)
    : State(g, 0, re, im), n_x(nx), n_y(0), norm(nm), phase(ph) {
    double x = 0;
    for (int i = 0; i < grid->dim_x; ++i) {
        map_lattice_to_coordinate_space(grid, i, &x);
        const complex<double> v = sinusoid_state(x, 0.);
        p_real[i] = real(v);
        p_imag[i] = imag(v);
    }
}

SinusoidState::SinusoidState(Lattice2D *g, int nx, int ny, double nm, double ph, double *re,
                             double *im)
    : State(g, 0, re, im), n_x(nx), n_y(ny), norm(nm), phase(ph) {
    double x = 0, y = 0;
    for (int j = 0; j < grid->dim_y; ++j)
        for (int i = 0; i < grid->dim_x; ++i) {
            map_lattice_to_coordinate_space(grid, i, j, &x, &y);
            const complex<double> v = sinusoid_state(x, y);
            p_real[size_t(j) * grid->dim_x + i] = real(v);
            p_imag[size_t(j) * grid->dim_x + i] = imag(v);
        }
}

complex<double> SinusoidState::sinusoid_state(double x, double y) {
    const double lx = grid->global_no_halo_dim_x * grid->delta_x;
    const double ly = grid->global_no_halo_dim_y * grid->delta_y;
    return sqrt(norm / (lx * ly)) * 2. * exp(complex<double>(0., phase)) *
           complex<double>(sin(2 * M_PI * double(n_x) / lx * x) *
                               sin(2 * M_PI * double(n_y) / ly * y),
                           0.0);
}

// ---------------------------------------------------------------- potentials
Potential::Potential(Lattice *g, char *filename)
    : grid(g), updated_potential_matrix(false), current_evolution_time(0),
      static_potential(NULL), evolving_potential(NULL), self_init(true), is_static(true) {
    const size_t n = size_t(grid->dim_x) * grid->dim_y;
    matrix = new double[n];
    std::ifstream in(filename);
    if (!in) my_abort(string("cannot open ") + filename);
    for (size_t k = 0; k < n; ++k) in >> matrix[k];
}

Potential::Potential(Lattice *g, double *external_pot)
    : grid(g), updated_potential_matrix(false), current_evolution_time(0),
      static_potential(NULL), evolving_potential(NULL), is_static(true) {
    if (external_pot == 0) {
        matrix = new double[size_t(grid->dim_x) * grid->dim_y]();
        self_init = true;
    } else {
        matrix = external_pot;
        self_init = false;
    }
}

Potential::Potential(Lattice *g, double (*f)(double, double))
    : grid(g), matrix(NULL), updated_potential_matrix(false), current_evolution_time(0),
      static_potential(f), evolving_potential(NULL), self_init(false), is_static(true) {}

Potential::Potential(Lattice *g, double (*f)(double, double, double), int t)
    : grid(g), matrix(NULL), updated_potential_matrix(false), current_evolution_time(t),
      static_potential(NULL), evolving_potential(f), self_init(false), is_static(false) {}

Potential::~Potential() {
    if (self_init) delete[] matrix;
}

double Potential::get_value(int x) { return get_value(x, 0); }

double Potential::get_value(int x, int y) {
    if (matrix != NULL) return matrix[size_t(y) * grid->dim_x + x];
    double xr = 0, yr = 0;
    map_lattice_to_coordinate_space(grid, x, y, &xr, &yr);
    return is_static ? static_potential(xr, yr) : evolving_potential(xr, yr, current_evolution_time);
}

bool Potential::update(double t) {
    if (current_evolution_time != t) {
        current_evolution_time = t;
        if (!is_static || updated_potential_matrix) return true;
    }
    return false;
}

HarmonicPotential::HarmonicPotential(Lattice2D *g, double wx, double wy, double m, double mx,
                                     double my)
    : Potential(g, const_potential), omegax(wx), omegay(wy), mass(m), mean_x(mx), mean_y(my) {
    static_potential = NULL;
}

HarmonicPotential::~HarmonicPotential() {}

double HarmonicPotential::get_value(int x, int y) {
    double xr = 0, yr = 0;
    map_lattice_to_coordinate_space(grid, x, y, &xr, &yr);
    xr -= mean_x;
    yr -= mean_y;
    return 0.5 * mass * (omegax * omegax * xr * xr + omegay * omegay * yr * yr);
}

// -------------------------------------------------------------- Hamiltonians
Hamiltonian::Hamiltonian(Lattice *g, Potential *pot, double m, double ga, double glhy,
                         double omega, double rx, double ry)
    : mass(m), coupling_a(ga), LeeHuangYang_coupling_a(glhy), angular_velocity(omega), grid(g) {
    // A rotating frame needs 8-cell halos (src/model.cpp:941-944).  Periodic
    // boundaries are accepted here; see the header.
    if (angular_velocity != 0. && grid->mpi_procs == 1) {
        grid->halo_x = 8;
        grid->halo_y = 8;
    }
    rot_coord_x = grid->coordinate_system == "cylindrical"
                      ? 0
                      : grid->global_no_halo_dim_x * 0.5 + rx / grid->delta_x;
    rot_coord_y = grid->global_no_halo_dim_y * 0.5 + ry / grid->delta_y;
    if (pot == NULL) {
        self_init = true;
        potential = new Potential(grid, const_potential);
    } else {
        self_init = false;
        potential = pot;
    }
}

Hamiltonian::~Hamiltonian() {
    if (self_init) delete potential;
}

double Hamiltonian::azimuthal_potential(double x, int l) {
    double xr = 0, yr = 0;
    map_lattice_to_coordinate_space(grid, int(x), 0, &xr, &yr);
    return (l * l) / (2. * mass * xr * xr);
}

Hamiltonian2Component::Hamiltonian2Component(Lattice *g, Potential *pot, Potential *pot_b,
                                             double m, double m_b, double ga, double gab,
                                             double gb, double wr, double wi, double omega,
                                             double rx, double ry)
    : Hamiltonian(g, pot, m, ga, 0., omega, rx, ry), mass_b(m_b), coupling_ab(gab),
      coupling_b(gb), omega_r(wr), omega_i(wi) {
    potential_b = pot_b == NULL ? potential : pot_b;
}

Hamiltonian2Component::~Hamiltonian2Component() {}

double Hamiltonian2Component::azimuthal_potential_b(double x, int l) {
    double xr = 0, yr = 0;
    map_lattice_to_coordinate_space(grid, int(x), 0, &xr, &yr);
    return (l * l) / (2. * mass_b * xr * xr);
}
