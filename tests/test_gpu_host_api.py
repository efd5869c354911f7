"""The drop-in API on the GPU: golden fixtures, the reference's known-answer
tests (test/kerneltest.cpp) and the plain-method configuration, through the
C++ host layer (Lattice2D / State / Hamiltonian / Solver), plus the FP32
storage form against the FP64 path."""
import numpy as np
import pytest

import trottersuzuki_b200 as ts
from helpers import desc_from_params, energy_params, golden_names, load_golden

pytestmark = pytest.mark.gpu

TOL_PSI = 1e-10
TOLERANCE = 1e-3       # test/kerneltest.h:8
NORM_TOLERANCE = 1e-5  # test/kerneltest.h:9
ENERGY_KEYS = ("total", "kinetic", "potential", "rotational", "intra", "lhy", "norm2")


@pytest.mark.parametrize("name", golden_names())
def test_golden_through_c_abi(name):
    import oracle as O
    g = load_golden(name)
    m, lat = g["meta"], g["lat"]
    psi = g["psi0"]
    kernel = None
    prev = None
    n0 = 0.0
    for it, imag in m["segments"]:
        if kernel is None or imag != prev:
            if kernel is not None:
                psi = kernel.get_state()
                kernel.close()
            if imag:
                n0 = O.expectations(lat, psi)["norm2"]
            p = lat.params(m["dt"], imag, 1.0, m["g"], m["lhy"], m["omega"], norm0=n0)
            tr, ti = O.exp_table(g["V"], m["dt"], imag)
            kernel = ts.Kernel(desc_from_params(p))
            kernel.set_state(psi)
            kernel.set_exp_potential(tr, ti)
        kernel.evolve(it)
        prev = imag
    got = kernel.get_state()
    e = kernel.energies(g["V"], energy_params(lat, 1.0, m["g"], m["lhy"], m["omega"]))
    kernel.close()
    assert np.abs(got - g["psi"]).max() <= TOL_PSI
    for k, ref in zip(ENERGY_KEYS, g["energies"]):
        assert abs(e[k] - ref) <= 1e-10 * max(1.0, abs(ref)), (k, e[k], ref)


def _host_objects(g, kernel_type="gpu"):
    m, lat = g["meta"], g["lat"]
    N, L, Ny, px, py, omega, one_d = m["lat"]
    if one_d:
        grid = ts.Lattice1D(N, L, px)
    else:
        grid = ts.Lattice2D(N, L, Ny, None, px, py, omega)
    state = ts.State(grid)
    state.init_state_matrix(g["psi0"].real, g["psi0"].imag)
    pot = ts.Potential(grid, g["V"])
    ham = ts.Hamiltonian(grid, pot, 1.0, m["g"], m["lhy"], m["omega"])
    solver = ts.Solver(grid, state, ham, m["dt"], kernel_type=kernel_type)
    return grid, state, pot, ham, solver


@pytest.mark.parametrize("name", golden_names())
def test_golden_through_drop_in_solver(name):
    g = load_golden(name)
    grid, state, pot, ham, solver = _host_objects(g)
    for it, imag in g["meta"]["segments"]:
        solver.evolve(it, imag)
    assert np.abs(state.get_state() - g["psi"]).max() <= TOL_PSI
    got = solver._energies()
    for k, a, ref in zip(ENERGY_KEYS, got, g["energies"]):
        assert abs(a - ref) <= 1e-10 * max(1.0, abs(ref)), (k, a, ref)
    if not g["lat"].one_d:
        x = state._expect()
        assert np.allclose(x, g["expectations"], rtol=1e-10, atol=1e-12)


def test_plain_method_config():
    """256^2, L=20, closed, HO omega=1, Gaussian (sigma 1) at (1,0), dt=1e-4, 1000 steps.
    Values of the reference CPUBlock on the same inputs (oracle/_ref, -O2)."""
    grid = ts.Lattice2D(256, 20.0)
    state = ts.GaussianState(grid, 1.0, 1.0, 1.0, 0.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0))
    solver = ts.Solver(grid, state, ham, 1e-4)
    e0 = solver.get_total_energy()
    solver.evolve(1000)
    assert abs(e0 - 1.49999922537628) < 1e-12
    psi = state.get_state()
    assert abs(psi[128, 128] - (0.0962255019132641 + 0.343774225402042j)) < 1e-12
    assert abs(solver.get_total_energy() - 1.5000065920508816) < 1e-12
    assert abs(solver.get_kinetic_energy() - 0.5049899409347001) < 1e-12
    assert abs(solver.get_potential_energy() - 0.9950166511161814) < 1e-12
    assert abs(solver.get_squared_norm() - 1.0000000000007403) < 1e-12


# ------------------------------------------- test/kerneltest.cpp scenarios
@pytest.mark.parametrize("kernel_type", ["gpu", "gpu_fp32"])
def test_kat_free_particle(kernel_type):
    grid = ts.Lattice2D(250, 100.0, periodic_x_axis=True, periodic_y_axis=True)
    state = ts.ExponentialState(grid)
    ham = ts.Hamiltonian(grid)
    solver = ts.Solver(grid, state, ham, 5e-3, kernel_type=kernel_type)
    e0, n0 = solver.get_total_energy(), solver.get_squared_norm()
    solver.evolve(100)
    assert abs(e0 - solver.get_total_energy()) < TOLERANCE
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


@pytest.mark.parametrize("kernel_type", ["gpu", "gpu_fp32"])
def test_kat_harmonic_oscillator(kernel_type):
    grid = ts.Lattice2D(250, 100.0)
    state = ts.GaussianState(grid, 1.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0))
    solver = ts.Solver(grid, state, ham, 5e-3, kernel_type=kernel_type)
    e0, n0 = solver.get_total_energy(), solver.get_squared_norm()
    solver.evolve(100)
    assert abs(e0 - solver.get_total_energy()) < TOLERANCE
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


@pytest.mark.parametrize("kernel_type", ["gpu", "gpu_fp32"])
def test_kat_imaginary_harmonic_oscillator(kernel_type):
    grid = ts.Lattice2D(250, 100.0)
    state = ts.GaussianState(grid, 0.5)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0))
    solver = ts.Solver(grid, state, ham, 5e-3, kernel_type=kernel_type)
    n0 = solver.get_squared_norm()
    solver.evolve(1000, True)
    assert abs(1.00001 - solver.get_total_energy()) < TOLERANCE
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


def test_kat_intra_particle_interaction():
    grid = ts.Lattice2D(250, 100.0)
    state = ts.GaussianState(grid, 1.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0), 1.0, 10.0)
    solver = ts.Solver(grid, state, ham, 1e-3)
    e0, n0 = solver.get_total_energy(), solver.get_squared_norm()
    solver.evolve(1000)
    assert abs(e0 - solver.get_total_energy()) < TOLERANCE
    assert abs(1.02321 - state.get_mean_xx()) < TOLERANCE
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


def test_kat_imaginary_intra_particle_interaction():
    grid = ts.Lattice2D(250, 100.0)
    state = ts.GaussianState(grid, 1.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0), 1.0, 10.0)
    solver = ts.Solver(grid, state, ham, 1e-3)
    n0 = solver.get_squared_norm()
    solver.evolve(1000, True)
    assert abs(1.59273 - solver.get_total_energy()) < TOLERANCE
    assert abs(0.768148 - state.get_mean_xx()) < TOLERANCE
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


def test_kat_rotating_frame_lattice():
    """test/kerneltest.cpp:127-150 (the Hamiltonian's 5th argument is the LHY coupling)."""
    grid = ts.Lattice2D(300, 20.0, angular_velocity=0.7)
    state = ts.GaussianState(grid, 1.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0), 1.0, 100.0, 0.7)
    solver = ts.Solver(grid, state, ham, 1e-4)
    e0, n0 = solver.get_total_energy(), solver.get_squared_norm()
    solver.evolve(1000)
    assert abs(e0 - solver.get_total_energy()) < TOLERANCE * 10.0
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


def test_kat_imaginary_rotating_frame_lattice():
    grid = ts.Lattice2D(300, 20.0, angular_velocity=0.7)
    state = ts.GaussianState(grid, 1.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0), 1.0, 100.0, 0.7)
    solver = ts.Solver(grid, state, ham, 1e-4)
    n0 = solver.get_squared_norm()
    solver.evolve(1000, True)
    # the reference test states 4.89895, but the reference itself gives
    # 4.901807766935512 on this setup (its 5th Hamiltonian argument became
    # the LHY coupling after that constant was recorded); pin the reference run
    assert abs(4.901807766935512 - solver.get_total_energy()) < 1e-8
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


def test_rotating_frame_with_rotation_active():
    """Omega = 0.7 in the Hamiltonian itself: energy and norm conserved in real time."""
    grid = ts.Lattice2D(200, 20.0, angular_velocity=0.7)
    state = ts.GaussianState(grid, 1.0, 1.0, 1.0, 0.0)
    ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0), 1.0, 50.0, 0.0, 0.7)
    solver = ts.Solver(grid, state, ham, 1e-4)
    e0, n0 = solver.get_total_energy(), solver.get_squared_norm()
    solver.evolve(500)
    assert abs(e0 - solver.get_total_energy()) < TOLERANCE * 10.0
    assert abs(n0 - solver.get_squared_norm()) < NORM_TOLERANCE


def test_fp32_storage_against_fp64_plain_method():
    """FP32 storage on the plain-method configuration: norm and energy within 1e-5."""
    out = {}
    for kt in ("gpu", "gpu_fp32"):
        grid = ts.Lattice2D(256, 20.0)
        state = ts.GaussianState(grid, 1.0, 1.0, 1.0, 0.0)
        ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 1.0, 1.0))
        solver = ts.Solver(grid, state, ham, 1e-4, kernel_type=kt)
        solver.evolve(1000)
        out[kt] = (solver.get_total_energy(), solver.get_squared_norm(), state.get_state())
    e64, n64, p64 = out["gpu"]
    e32, n32, p32 = out["gpu_fp32"]
    assert abs(e32 - e64) / abs(e64) <= 1e-5
    assert abs(n32 - n64) / abs(n64) <= 1e-5
    assert np.abs(p32 - p64).max() <= 1e-4


@pytest.mark.parametrize("periodic,omega", [(False, 0.0), (True, 0.7)], ids=["closed", "periodic_rot"])
def test_fp32_storage_at_large_pair_angle(periodic, omega):
    """A fine grid (pair angle dt / (4 m dx^2) = 0.52 rad, as in the 8192^2
    precision configuration): a fixed float coefficient pair would drift the
    norm and the phase every step; the per-step coefficient schedule keeps
    FP32 within 1e-5 of FP64 in norm and energy over 2000 steps."""
    out = {}
    for kt in ("gpu", "gpu_fp32"):
        grid = ts.Lattice2D(256, 1.25, periodic_x_axis=periodic, periodic_y_axis=periodic,
                            angular_velocity=omega)
        state = ts.GaussianState(grid, 40.0, 40.0, 0.05, 0.0)
        state.imprint(lambda x, y: np.exp(3j * x))
        ham = ts.Hamiltonian(grid, ts.HarmonicPotential(grid, 4.0, 4.0), 1.0, 20.0, 0.0, omega)
        solver = ts.Solver(grid, state, ham, 5e-5, kernel_type=kt)
        solver.evolve(2000)
        out[kt] = (solver.get_total_energy(), solver.get_squared_norm(), state.get_state())
    e64, n64, p64 = out["gpu"]
    e32, n32, p32 = out["gpu_fp32"]
    assert abs(n32 - n64) / abs(n64) <= 1e-5
    assert abs(e32 - e64) / abs(e64) <= 1e-5
    assert np.linalg.norm(p32 - p64) / np.linalg.norm(p64) <= 1e-4


def test_device_pointer_calls_follow_the_torch_stream():
    """set_state_device / get_state_device on tensors that torch writes and
    reads on its own (non-default) stream, without a synchronisation in
    between: the handle's stream waits for torch's work before the copy in,
    and torch's stream waits for the copy out."""
    import torch
    from trottersuzuki_b200 import Kernel
    from helpers import desc_from_params, seeded_case
    lat, psi0, V = seeded_case(96, 10.0, 80, (False, False))
    p = lat.params(1e-3, False, 1.0, 1.0, 0.0, 0.0)
    s = torch.cuda.Stream()
    H, W = psi0.shape
    with Kernel(desc_from_params(p)) as k, torch.cuda.stream(s):
        src = torch.tensor(psi0, dtype=torch.complex128, device="cuda")
        # a long chain of kernels on torch's stream ends in the state to upload
        big = torch.rand(4096, 4096, dtype=torch.float64, device="cuda")
        for _ in range(20):
            big = big @ big * 1e-4
        src = src + 0.0 * big[:H, :W]
        k.set_state_device(src.data_ptr(), W)
        out = torch.empty_like(src)
        k.get_state_device(out.data_ptr(), W)
        res = (out - src).abs().max()
        assert float(res.item()) == 0.0
