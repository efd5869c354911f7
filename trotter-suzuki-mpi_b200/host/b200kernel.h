// B200Kernel: the ITrotterKernel of this engine.
//
// It keeps the tile and the exponential table on the GPU and runs the fused
// sm_100a step of include/ts_b200.h.  It replaces the reference's CUDA
// kernel class CC2Kernel (src/kernel.h:173-269) at the plug-in boundary
// ITrotterKernel (src/trottersuzuki.h:502-520); Solver::init_kernel creates it
// for kernel_type "gpu"/"b200" (FP64 storage) and "gpu_fp32"/"b200_fp32".
#ifndef TS_B200_B200KERNEL_H
#define TS_B200_B200KERNEL_H

#include <string>

#include "trottersuzuki.h"
#include "ts_b200.h"

class B200Kernel : public ITrotterKernel {
public:
    B200Kernel(Lattice *grid, State *state, Hamiltonian *hamiltonian, double *external_pot_real,
               double *external_pot_imag, double delta_t, double norm, bool imag_time,
               int precision = TS_B200_FP64);
    ~B200Kernel();

    // The fused step covers the whole tile, halo included, in one launch:
    // run_kernel_on_halo has nothing left to do.
    void run_kernel_on_halo() {}
    void run_kernel();
    // Imaginary-time renormalisation is computed on the device by the step
    // itself and applied when the tile is next read.
    void wait_for_completion() {}
    void get_sample(size_t dest_stride, size_t x, size_t y, size_t width, size_t height,
                    double *dest_real, double *dest_imag, double *dest_real2 = 0,
                    double *dest_imag2 = 0) const;
    // Two-component and cylindrical operations: not part of this kernel.
    void normalization() {}
    void rabi_coupling(double, double) {}
    void cpy_first_positive_to_first_negative() {}
    double calculate_squared_norm(bool global = true) const;
    bool runs_in_place() const { return false; }
    std::string get_name() const { return "B200"; }
    void update_potential(double *external_pot_real, double *external_pot_imag, int which);
    void start_halo_exchange() {}
    void finish_halo_exchange();

    /** Whole evolve() loop: steps 0..n-2 refresh the halo, the last does not. */
    void evolve(int iterations);
    /** Steps that all refresh the halo (used when a step is not the last one). */
    void steps_with_exchange(int n);
    ts_b200_kernel *handle() const { return h_; }

private:
    void check(int status, const char *what) const;
    ts_b200_kernel *h_;
    int dim_x_, dim_y_;
    bool imag_time_;
};

/** Two species evolved together (the reference's two-state CPUBlock,
 *  src/cpukernel.cpp:274-392,581-667), on a ts_b200_pair of two device tiles.
 *  The plug-in protocol alternates the species as the reference's kernel
 *  does: run_kernel / finish_halo_exchange act on the current species and
 *  wait_for_completion moves to the other one; steps() runs whole steps of
 *  the pair without the per-call protocol. */
class B200PairKernel : public ITrotterKernel {
public:
    B200PairKernel(Lattice *grid, State *state_a, State *state_b, Hamiltonian2Component *ham,
                   double **external_pot_real, double **external_pot_imag, double delta_t,
                   double *norm, bool imag_time, int precision = TS_B200_FP64);
    ~B200PairKernel();

    void run_kernel_on_halo() {}
    void run_kernel();
    void wait_for_completion();
    void get_sample(size_t dest_stride, size_t x, size_t y, size_t width, size_t height,
                    double *dest_real, double *dest_imag, double *dest_real2 = 0,
                    double *dest_imag2 = 0) const;
    void normalization();
    void rabi_coupling(double var, double delta_t);
    void cpy_first_positive_to_first_negative() {}
    double calculate_squared_norm(bool global = true) const;
    bool runs_in_place() const { return false; }
    std::string get_name() const { return "B200 (two components)"; }
    void update_potential(double *external_pot_real, double *external_pot_imag, int which);
    void start_halo_exchange() {}
    void finish_halo_exchange();

    /** n steps of the pair; with final_steps the last one is the evolve()
     *  call's last (no halo refresh, half Rabi rotation). */
    void steps(int n, bool final_steps);
    ts_b200_pair *pair() const { return p_; }

private:
    void check(int status, const char *what) const;
    void release();
    ts_b200_kernel *h_[2] = {nullptr, nullptr};
    ts_b200_pair *p_ = nullptr;
    int state_index_ = 0;
    int dim_x_;
};

namespace b200 {

struct Expectations {
    double norm2, mean_x, mean_xx, mean_y, mean_yy, mean_px, mean_pxpx, mean_py, mean_pypy,
        mean_lz;
};

/** Expectation values of a host tile (src/model.cpp:385-536), reduced on the GPU. */
Expectations reduce_expectations(Lattice *grid, const double *p_real, const double *p_imag);

/** Energy functional of a host tile (src/solver.cpp:244-564), reduced on the GPU. */
ts_b200_energy_result reduce_energies(Lattice *grid, const double *p_real, const double *p_imag,
                                      const double *V, double mass, double coupling,
                                      double lhy_coupling, double angular_velocity);

/** Step descriptor with the constants of the reference's CPUBlock constructor. */
ts_b200_desc make_desc(Lattice *grid, Hamiltonian *ham, double delta_t, double norm,
                       bool imag_time, int precision, int angular_momentum = 0);
/** The same for one species of mass `mass`, g = coupling, g_LHY = lhy. */
ts_b200_desc make_species_desc(Lattice *grid, Hamiltonian *ham, double delta_t, double norm,
                               bool imag_time, int precision, double mass, double coupling,
                               double lhy, int angular_momentum = 0);

/** Inter-species and Rabi energies of two host tiles (src/solver.cpp:340-353,
 *  549-550), reduced on the GPU. */
void reduce_cross_energies(Lattice *grid, const double *a_re, const double *a_im,
                           const double *b_re, const double *b_im, double coupling_ab,
                           double omega_r, double omega_i, double *inter, double *rabi);

}  // namespace b200

#endif
