"""Ground-state convergence of the GPE imaginary-time configuration against the
reference's own CPU path.

The configuration: 2D GPE in imaginary time, closed boundaries, harmonic trap
omega = (1, 1.5), g = 100, side length 24, normalised Gaussian (sigma 2) times
(1 + 0.01 u) with u seeded uniform, dt = 1e-4, renormalised every step, 20000
steps.  The B200 path runs it at full size in the benchmark; here the same
setup runs on a 512 x 512 lattice through the drop-in Solver on the GPU and
through the compiled reference CPUBlock (oracle/_ref, its unmodified sources,
Solver::evolve of src/solver.cpp:150-242), and the total energies of the
final states (src/solver.cpp:244-564) agree to 1e-10 relative.
"""
import math
import os
import sys

import numpy as np
import pytest

import tsref

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

N, LENGTH, OMEGA, G, DT, STEPS = 512, 24.0, (1.0, 1.5), 100.0, 1e-4, 20000
SEED = 20240601


def _initial_state(W, H, dx, dy):
    x = (np.arange(W) + 0.5) * dx - W * dx * 0.5
    y = (np.arange(H) + 0.5) * dy - H * dy * 0.5
    X, Y = np.meshgrid(x, y)
    w = 0.25  # omega = 1 / sigma^2, sigma = 2
    psi = np.sqrt(w / math.pi) * np.exp(-(w * X * X + w * Y * Y) * 0.5)
    rng = np.random.Generator(np.random.PCG64(SEED))
    psi = psi * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, psi.shape))
    psi = psi / math.sqrt(np.sum(psi * psi) * dx * dy)
    return psi.astype(np.complex128)


@pytest.fixture(scope="module")
def reference_run():
    """The reference CPUBlock (-O2 parity build, all host threads) on the setup."""
    import trottersuzuki_b200 as ts
    grid = ts.Lattice2D(N, LENGTH)
    psi0 = _initial_state(grid.dim_x, grid.dim_y, grid.delta_x, grid.delta_y)
    cfg = tsref.make_config(N, LENGTH, harmonic=(OMEGA[0], OMEGA[1], 1.0, 0.0, 0.0),
                            coupling=G, delta_t=DT, segments=((STEPS, True),),
                            omp_threads=os.cpu_count() or 1)
    psi_ref, res = tsref.run(cfg, psi0, None)
    return psi0, psi_ref, res


@pytest.mark.skipif(not tsref.available(), reason="compiled reference (oracle/_ref) not built")
@pytest.mark.parametrize("kernel_type,tol_e", [("gpu", 1e-10), ("gpu_fp32", 1e-5)])
def test_ground_state_energy_matches_reference_cpu(reference_run, kernel_type, tol_e):
    import trottersuzuki_b200 as ts
    psi0, psi_ref, res = reference_run
    grid = ts.Lattice2D(N, LENGTH)

    state = ts.State(grid)
    state.init_state_matrix(psi0.real, psi0.imag)
    pot = ts.HarmonicPotential(grid, OMEGA[0], OMEGA[1])
    ham = ts.Hamiltonian(grid, pot, 1.0, G)
    solver = ts.Solver(grid, state, ham, DT, kernel_type=kernel_type)
    solver.evolve(STEPS, True)
    e = solver.get_total_energy()
    norm = solver.get_squared_norm()

    rel = abs(e - res.total_energy) / abs(res.total_energy)
    print(f"{kernel_type}: E = {e!r}, reference E = {res.total_energy!r}, rel {rel:.2e}",
          file=sys.stderr)
    assert rel <= tol_e
    assert abs(norm - res.squared_norm) <= 1e-12
    if kernel_type == "gpu":
        assert np.abs(state.get_state() - psi_ref).max() <= 1e-10
