"""The reference's own, unmodified Solver driving the B200 engine.

trotter-suzuki-mpi_b200/integration/build_with_reference.sh compiles the
reference's sources (src/{common,cpukernel,cpucartesian,cpucylindrical,model,
solver}.cpp, read in place) with -DCUDA and cc2kernel_b200.cpp, which
implements the reference's GPU kernel class CC2Kernel (src/kernel.h) on the
C ABI of include/ts_b200.h, into oracle/_ref/libtsref_b200.so.  Solver::evolve
(src/solver.cpp:150-242) then runs every step through the ITrotterKernel
virtuals (src/trottersuzuki.h:502-520) on the B200, and the reference's own
energy code (src/solver.cpp:244-564) reads the result.  Every golden fixture
the reference's GPU path accepts (no rotating frame: src/solver.cpp:132-134)
is reproduced to the FP64 parity bar.
"""
import json
import os

import numpy as np
import pytest

import tsref

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not tsref.available("b200"),
                                 reason="oracle/_ref/libtsref_b200.so not built")]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_PSI = 1e-10
TOL_E = 1e-10


def _load(path):
    z = np.load(path)
    return z, json.loads(str(z["meta"]))


def _single_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


@pytest.mark.parametrize("name", _single_names())
def test_reference_solver_on_b200_reproduces_golden(name):
    z, meta = _load(os.path.join(GOLDEN, name + ".npz"))
    if meta["omega"] != 0.0:
        pytest.skip("the reference's GPU kernel path refuses a rotating frame")
    N, L, Ny, px, py, omega, one_d = meta["lat"]
    cfg = tsref.make_config(N, L, 0 if one_d else Ny, None, px, py, omega, harmonic=None,
                            coupling=meta["g"], lhy_coupling=meta["lhy"],
                            angular_velocity=meta["omega"], delta_t=meta["dt"],
                            segments=meta["segments"], omp_threads=1, kernel_gpu=True)
    psi, res = tsref.run(cfg, z["psi0"], z["V"], flavour="b200")
    assert np.abs(psi - z["psi"]).max() <= TOL_PSI
    e = np.array([res.total_energy, res.kinetic_energy, res.potential_energy,
                  res.rotational_energy, res.intra_energy, res.lhy_energy, res.squared_norm])
    assert np.abs(e - z["energies"]).max() <= TOL_E * max(1.0, np.abs(z["energies"]).max())


@pytest.mark.parametrize("name", sorted(f[:-4] for f in os.listdir(os.path.join(GOLDEN, "cyl"))
                                        if f.endswith(".npz")))
def test_reference_solver_on_b200_cylindrical(name):
    z, meta = _load(os.path.join(GOLDEN, "cyl", name + ".npz"))
    N, L, Ny, Ly, py = meta["lat"]
    cfg = tsref.make_config(N, L, Ny, Ly, False, py, 0.0, harmonic=None, coupling=meta["g"],
                            delta_t=meta["dt"], segments=meta["segments"], omp_threads=1,
                            cylindrical=True, angular_momentum=meta["l"], kernel_gpu=True)
    psi, res = tsref.run(cfg, z["psi0"], z["V"], flavour="b200")
    assert np.abs(psi - z["psi"]).max() <= TOL_PSI
    assert abs(res.total_energy - z["energies"][0]) <= TOL_E * max(1.0, abs(z["energies"][0]))


@pytest.mark.parametrize("name", sorted(f[:-4] for f in os.listdir(os.path.join(GOLDEN, "two"))
                                        if f.endswith(".npz")))
def test_reference_solver_on_b200_two_components(name):
    z, meta = _load(os.path.join(GOLDEN, "two", name + ".npz"))
    N, L, Ny, px, py = meta["lat"]
    cfg = tsref.make_config(N, L, Ny, None, px, py, 0.0, harmonic=None, coupling=meta["g"],
                            delta_t=meta["dt"], segments=meta["segments"], omp_threads=1,
                            kernel_gpu=True)
    c2 = tsref.Config2(meta["mass_b"], meta["g_b"], meta["g_ab"], *meta["omega"])
    pa, pb, res = tsref.run2(cfg, c2, z["psi0_a"], z["psi0_b"], z["Va"], z["Vb"], flavour="b200")
    assert np.abs(pa - z["psi_a"]).max() <= TOL_PSI
    assert np.abs(pb - z["psi_b"]).max() <= TOL_PSI
    assert abs(res.total_energy - z["energies"][0]) <= TOL_E * max(1.0, abs(z["energies"][0]))


def test_cpu_kernel_type_still_runs_the_reference_cpu_path():
    """kernel_type "cpu" of the same library is the reference's CPUBlock."""
    name = "closed_real"
    z, meta = _load(os.path.join(GOLDEN, name + ".npz"))
    N, L, Ny, px, py, omega, one_d = meta["lat"]
    cfg = tsref.make_config(N, L, Ny, None, px, py, omega, harmonic=None, coupling=meta["g"],
                            lhy_coupling=meta["lhy"], delta_t=meta["dt"],
                            segments=meta["segments"], omp_threads=1, kernel_gpu=False)
    psi, _ = tsref.run(cfg, z["psi0"], z["V"], flavour="b200")
    assert np.abs(psi - z["psi"]).max() <= 1e-12
