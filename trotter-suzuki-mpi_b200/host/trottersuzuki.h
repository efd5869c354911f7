/*
 * trottersuzuki.h -- C++ API of the B200 Trotter-Suzuki engine.
 *
 * Class names, members and method signatures follow the public API of
 * trotter-suzuki-mpi 1.6.2 (src/trottersuzuki.h:34-602) so that programs
 * written against that library compile and run unchanged.  The evolution is
 * done by B200Kernel (b200kernel.h), an ITrotterKernel that runs the fused
 * sm_100a step behind the C ABI of include/ts_b200.h.
 *
 * Differences from the reference, all deliberate:
 *  - kernel_type: "gpu" and "b200" select the B200 kernel with FP64 storage,
 *    "gpu_fp32" / "b200_fp32" the FP32-storage form.  There is no CPU kernel
 *    in this build, so the default is "gpu" and "cpu" is rejected with the
 *    reference's "Unknown kernel" error path (std::runtime_error).
 *  - Rotating frame with periodic boundaries is accepted (the reference
 *    prints a message and leaves the Hamiltonian half-initialised).  The
 *    rotation coordinates are the extended tile coordinates, as the
 *    reference's formulas give them.
 *  - Energies, norms and expectation values are reduced on the GPU in FP64.
 *  - Two-component systems (Hamiltonian2Component, the two-state Solver, Rabi
 *    coupling) and cylindrical lattices run on the B200 kernel
 *    (B200PairKernel, the cylindrical step variants).  Not supported, as on
 *    the reference's own GPU path: two components with a rotating frame or the
 *    Lee-Huang-Yang term, and cylindrical lattices with a rotating frame.
 *    BesselState is not provided (cylindrical states come from
 *    init_state_matrix).
 */
#ifndef TS_B200_TROTTERSUZUKI_H
#define TS_B200_TROTTERSUZUKI_H

#include <complex>
#include <cstddef>
#include <string>

using namespace std;

/** Geometry of the lattice tile owned by this process (one GPU). */
class Lattice {
public:
    int mpi_rank;     ///< Always 0: one process per lattice.
    int mpi_procs;    ///< Always 1.
    double length_x, length_y;   ///< Physical side lengths.
    double delta_x, delta_y;     ///< Grid spacing.
    int dim_x, dim_y;            ///< Tile size including the periodic halo.
    int global_no_halo_dim_x, global_no_halo_dim_y;  ///< Lattice size without halo.
    int global_dim_x, global_dim_y;                  ///< Lattice size with halo.
    int periods[2];              ///< periods[0]: y periodic, periods[1]: x periodic.
    string coordinate_system;    ///< "cartesian" or "cylindrical".
    int halo_x, halo_y;          ///< Halo width (4; 8 with a rotating frame).
    int start_x, start_y;        ///< Lattice coordinate of the first tile cell.
    int end_x, end_y;            ///< One past the last tile cell.
    int inner_start_x, inner_start_y;  ///< First cell outside the halo.
    int inner_end_x, inner_end_y;      ///< One past the last cell outside the halo.
    int mpi_coords[2], mpi_dims[2];    ///< Process grid (always one process).
};

/** One-dimensional lattice (a chain); dim_y is 1. */
class Lattice1D : public Lattice {
public:
    Lattice1D(int dim, double length, bool periodic_x_axis = false,
              string coordinate_system = "cartesian");
};

/** Two-dimensional lattice. */
class Lattice2D : public Lattice {
public:
    Lattice2D(int dim, double length, bool periodic_x_axis = false, bool periodic_y_axis = false,
              double angular_velocity = 0., string coordinate_system = "cartesian");
    Lattice2D(int dim_x, double length_x, int dim_y, double length_y, bool periodic_x_axis = false,
              bool periodic_y_axis = false, double angular_velocity = 0.,
              string coordinate_system = "cartesian");

private:
    void init(int dim_x, double length_x, int dim_y, double length_y, bool periodic_x_axis,
              bool periodic_y_axis, double angular_velocity, string coordinate_system);
};

/** Wave function on the tile, real and imaginary parts in separate arrays. */
class State {
public:
    double *p_real;
    double *p_imag;
    Lattice *grid;
    int angular_momentum;

    State(Lattice *grid, int angular_momentum = 0, double *p_real = 0, double *p_imag = 0);
    State(const State &obj);
    ~State();
    void init_state(complex<double> (*ini_state)(double x));
    void init_state(complex<double> (*ini_state)(double x, double y));
    void loadtxt(char *file_name);
    void imprint(complex<double> (*function)(double x));
    void imprint(complex<double> (*function)(double x, double y));
    double *get_particle_density(double *density = 0);
    double *get_phase(double *phase = 0);
    double get_expected_value(string _operator);
    double get_squared_norm(void);
    double get_mean_x(void);
    double get_mean_xx(void);
    double get_mean_y(void);
    double get_mean_yy(void);
    double get_mean_px(void);
    double get_mean_pxpx(void);
    double get_mean_py(void);
    double get_mean_pypy(void);
    double get_mean_angular_momentum(void);
    void write_to_file(string fileprefix);
    void write_particle_density(string fileprefix);
    void write_phase(string fileprefix);
    bool expected_values_updated;

protected:
    bool self_init;
    void calculate_expected_values(void);
    double mean_X, mean_XX;
    double mean_Y, mean_YY;
    double mean_Px, mean_PxPx;
    double mean_Py, mean_PyPy;
    double mean_angular_momentum;
    double norm2;
};

/** Plane wave exp(i 2 pi (n_x x / L_x + n_y y / L_y)) with a given norm and phase. */
class ExponentialState : public State {
public:
    ExponentialState(Lattice1D *grid, int n_x = 1, double norm = 1, double phase = 0,
                     double *p_real = 0, double *p_imag = 0);
    ExponentialState(Lattice2D *grid, int n_x = 1, int n_y = 1, double norm = 1,
                     double phase = 0, double *p_real = 0, double *p_imag = 0);

private:
    int n_x, n_y;
    double norm, phase;
    complex<double> exp_state(double x, double y);
};

/** Gaussian with inverse variances omega_x, omega_y centred at (mean_x, mean_y). */
class GaussianState : public State {
public:
    GaussianState(Lattice1D *grid, double omega_x, double mean_x = 0, double norm = 1,
                  double phase = 0, double *p_real = 0, double *p_imag = 0);
    GaussianState(Lattice2D *grid, double omega_x, double omega_y = -1., double mean_x = 0,
                  double mean_y = 0, double norm = 1, double phase = 0, double *p_real = 0,
                  double *p_imag = 0);

private:
    double mean_x, mean_y, omega_x, omega_y, norm, phase;
    complex<double> gauss_state(double x, double y);
};

/** Product of sines sin(2 pi n_x x / L_x) sin(2 pi n_y y / L_y). */
class SinusoidState : public State {
public:
    SinusoidState(Lattice1D *grid, int n_x = 1, double norm = 1, double phase = 0,
                  double *p_real = 0, double *p_imag = 0);
    SinusoidState(Lattice2D *grid, int n_x = 1, int n_y = 1, double norm = 1, double phase = 0,
                  double *p_real = 0, double *p_imag = 0);

private:
    int n_x, n_y;
    double norm, phase;
    complex<double> sinusoid_state(double x, double y);
};

/** External potential: a matrix, a static function V(x, y) or V(x, y, t). */
class Potential {
public:
    Lattice *grid;
    double *matrix;

    Potential(Lattice *grid, char *filename);
    Potential(Lattice *grid, double *external_pot = 0);
    Potential(Lattice *grid, double (*potential_function)(double x, double y));
    Potential(Lattice *grid, double (*potential_function)(double x, double y, double t),
              int t = 0);
    virtual ~Potential();
    virtual double get_value(int x);
    virtual double get_value(int x, int y);
    bool update(double t);
    bool updated_potential_matrix;

protected:
    double current_evolution_time;
    double (*static_potential)(double x, double y);
    double (*evolving_potential)(double x, double y, double t);
    bool self_init;
    bool is_static;
};

/** V = m/2 (omega_x^2 (x - mean_x)^2 + omega_y^2 (y - mean_y)^2). */
class HarmonicPotential : public Potential {
public:
    HarmonicPotential(Lattice2D *grid, double omegax, double omegay, double mass = 1.,
                      double mean_x = 0., double mean_y = 0.);
    ~HarmonicPotential();
    double get_value(int x, int y);

private:
    double omegax, omegay, mass, mean_x, mean_y;
};

/** Single-component Hamiltonian: kinetic + V + g|psi|^2 + g_LHY|psi|^3 + rotating frame. */
class Hamiltonian {
public:
    Potential *potential;
    double mass;
    double coupling_a;
    double LeeHuangYang_coupling_a;
    double angular_velocity;
    double rot_coord_x;   ///< Rotation centre in lattice units.
    double rot_coord_y;
    double azimuthal_potential(double x, int angular_momentum);

    Hamiltonian(Lattice *grid, Potential *potential = 0, double mass = 1., double coupling_a = 0.,
                double LeeHuangYang_coupling_a = 0., double angular_velocity = 0.,
                double rot_coord_x = 0, double rot_coord_y = 0);
    virtual ~Hamiltonian();

protected:
    bool self_init;
    Lattice *grid;
};

/** Two-component Hamiltonian (declared for source compatibility; not evolved by B200Kernel). */
class Hamiltonian2Component : public Hamiltonian {
public:
    double mass_b;
    double coupling_ab;
    double coupling_b;
    double omega_r;
    double omega_i;
    Potential *potential_b;
    double azimuthal_potential_b(double x, int angular_momentum);

    Hamiltonian2Component(Lattice *grid, Potential *potential = 0, Potential *potential_b = 0,
                          double mass = 1., double mass_b = 1., double coupling_a = 0.,
                          double coupling_ab = 0., double coupling_b = 0., double omega_r = 0,
                          double omega_i = 0, double angular_velocity = 0.,
                          double rot_coord_x = 0, double rot_coord_y = 0);
    ~Hamiltonian2Component();
};

/** Kernel plug-in interface (same virtuals as the reference). */
class ITrotterKernel {
public:
    virtual ~ITrotterKernel() {}
    virtual void run_kernel() = 0;
    virtual void run_kernel_on_halo() = 0;
    virtual void wait_for_completion() = 0;
    virtual void get_sample(size_t dest_stride, size_t x, size_t y, size_t width, size_t height,
                            double *dest_real, double *dest_imag, double *dest_real2 = 0,
                            double *dest_imag2 = 0) const = 0;
    virtual void normalization() = 0;
    virtual void rabi_coupling(double var, double delta_t) = 0;
    virtual double calculate_squared_norm(bool global = true) const = 0;
    virtual bool runs_in_place() const = 0;
    virtual string get_name() const = 0;
    virtual void update_potential(double *_external_pot_real, double *_external_pot_imag,
                                  int which) = 0;
    virtual void cpy_first_positive_to_first_negative() = 0;
    virtual void start_halo_exchange() = 0;
    virtual void finish_halo_exchange() = 0;
};

/** Drives the evolution and computes energies. */
class Solver {
public:
    Lattice *grid;
    State *state;
    State *state_b;
    Hamiltonian *hamiltonian;
    double current_evolution_time;

    Solver(Lattice *grid, State *state, Hamiltonian *hamiltonian, double delta_t,
           string kernel_type = "gpu");
    Solver(Lattice *grid, State *state1, State *state2, Hamiltonian2Component *hamiltonian,
           double delta_t, string kernel_type = "gpu");
    ~Solver();
    void evolve(int iterations, bool imag_time = false);
    void update_parameters();
    double get_total_energy(void);
    double get_squared_norm(size_t which = 3);
    double get_kinetic_energy(size_t which = 3);
    double get_potential_energy(size_t which = 3);
    double get_rotational_energy(size_t which = 3);
    double get_intra_species_energy(size_t which = 3);
    double get_LeeHuangYang_energy(void);
    double get_inter_species_energy(void);
    double get_rabi_energy(void);
    void set_exp_potential(double *real, int real_length, double *imag, int imag_length,
                           int which);
    /** The kernel currently in use (NULL before the first evolve). */
    ITrotterKernel *get_kernel() { return kernel; }
    /** Build (or rebuild) the kernel for the time mode as evolve() does, with
     *  no step and no copy back into the State. */
    void prepare_kernel(bool imag_time);

private:
    bool imag_time;
    double **external_pot_real;
    double **external_pot_imag;
    double delta_t;
    double norm2[2];
    bool single_component;
    string kernel_type;
    ITrotterKernel *kernel;
    void initialize_exp_potential(double time_single_it, int which);
    void init_kernel();
    double total_energy;
    double kinetic_energy[2];
    double tot_kinetic_energy;
    double potential_energy[2];
    double tot_potential_energy;
    double rotational_energy[2];
    double tot_rotational_energy;
    double intra_species_energy[2];
    double tot_intra_species_energy;
    double LeeHuangYang_energy;
    double inter_species_energy;
    double rabi_energy;
    bool has_parameters_changed;
    bool energy_expected_values_updated;
    void calculate_energy_expected_values(void);
    void calculate_energies_two_components(void);
    void evolve_two_components(int iterations, bool soft_update);
    bool is_python;
    bool kernel_state_current;  ///< the kernel's device tile equals *state
};

double const_potential(double x);
double const_potential(double x, double y);
void map_lattice_to_coordinate_space(Lattice *grid, int x_in, double *x_out);
void map_lattice_to_coordinate_space(Lattice *grid, int x_in, int y_in, double *x_out,
                                     double *y_out);
/** Throws std::runtime_error(err), as the reference's my_abort does without MPI. */
void my_abort(string err);

#endif  // TS_B200_TROTTERSUZUKI_H
