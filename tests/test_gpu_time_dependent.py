"""Time-dependent potentials V(x, y, t).

The reference's Python Solver re-tabulates exp(-i dt V(x, y, t)) on the host
before every real-time step and runs each step as its own evolve call
(classes_extension.py:360-366, 388-403), so step i uses V(t0 + i dt) and no
step refreshes the halo.  Checked here: that host path (Potential.init_potential
with a 3-argument function), DevicePotential (V and its table made on the
device every step, ts_b200_set_potential_device), and the C-ABI call itself,
against the oracle stepping one evolve per step with the same tables.
"""
import math

import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, seeded_case

pytestmark = pytest.mark.gpu

DT = 1e-3
G = 1.5


def moving_trap(x, y, t):
    """A harmonic trap whose centre oscillates along x; numpy or torch arrays."""
    return 0.5 * ((x - 0.8 * math.sin(30.0 * t)) ** 2 + 1.3 * y ** 2)


def moving_trap_torch(x, y, t):
    """moving_trap with t a tensor of step times (DevicePotential time_batch mode)."""
    import torch
    return 0.5 * ((x - 0.8 * torch.sin(30.0 * t)) ** 2 + 1.3 * y ** 2)


def _objects(kind, kernel_type, N=96, L=10.0, periodic=(False, False)):
    import trottersuzuki_b200 as ts
    lat, psi0, _ = seeded_case(N, L, None, periodic, 0.0, seed=3)
    grid = ts.Lattice2D(N, L, periodic_x_axis=periodic[0], periodic_y_axis=periodic[1])
    state = ts.State(grid)
    state.init_state_matrix(psi0.real, psi0.imag)
    if kind == "host":
        pot = ts.Potential(grid)
        pot.init_potential(moving_trap)
    elif kind == "device":
        pot = ts.DevicePotential(grid, moving_trap)
    elif kind == "device_batch":
        pot = ts.DevicePotential(grid, moving_trap_torch, time_batch=5)
    else:  # the static matrix V(x, y, 0)
        X, Y = lat.coordinates()
        pot = ts.Potential(grid, moving_trap(X, Y, 0.0))
    ham = ts.Hamiltonian(grid, pot, 1.0, G)
    solver = ts.Solver(grid, state, ham, DT, kernel_type=kernel_type)
    return lat, psi0, state, solver, (grid, pot, ham)


def oracle_steps(lat, psi0, n, t0=0.0):
    p = lat.params(DT, False, 1.0, G, 0.0, 0.0)
    X, Y = lat.coordinates()
    psi = psi0
    for i in range(n):
        tr, ti = O.exp_table(moving_trap(X, Y, t0 + i * DT), DT, False)
        psi = O.evolve(p, psi, tr, ti, 1)
    return psi


PERIODIC = [(False, False), (True, True)]


@pytest.mark.parametrize("periodic", PERIODIC, ids=["closed", "periodic"])
@pytest.mark.parametrize("kind", ["host", "device", "device_batch"])
def test_time_dependent_potential_matches_oracle(kind, periodic):
    lat, psi0, state, solver, keep = _objects(kind, "gpu", periodic=periodic)
    solver.evolve(7)
    solver.evolve(5)
    assert abs(solver.current_evolution_time - 12 * DT) < 1e-15
    ref = oracle_steps(lat, psi0, 12)
    err = np.abs(state.get_state() - ref).max()
    assert err <= 1e-10, f"{kind}: {err:.3e}"
    # the potential really moved: a static V(t = 0) run ends elsewhere
    X, Y = lat.coordinates()
    tr, ti = O.exp_table(moving_trap(X, Y, 0.0), DT, False)
    static = psi0
    for _ in range(12):
        static = O.evolve(lat.params(DT, False, 1.0, G, 0.0, 0.0), static, tr, ti, 1)
    assert np.abs(static - ref).max() > 1e3 * err + 1e-9


@pytest.mark.parametrize("kind", ["device", "device_batch"])
@pytest.mark.parametrize("kernel_type,tol", [("gpu", 1e-12), ("gpu_fp32", 2e-6)])
def test_device_potential_matches_host_path(kernel_type, tol, kind):
    _, _, s_host, host, keep1 = _objects("host", kernel_type)
    _, _, s_dev, dev, keep2 = _objects(kind, kernel_type)
    for n in (9, 1, 6, -3, 2):  # -3: no copy back, as the C++ evolve
        host.evolve(n)
        dev.evolve(n)
    a, b = s_dev.get_state(), s_host.get_state()
    assert np.abs(a - b).max() <= tol * np.abs(b).max()
    # energies use V at t = 0 on both paths, as the reference's do
    for x, y in zip(dev._energies(), host._energies()):
        assert abs(x - y) <= max(tol, 1e-12) * max(1.0, abs(y))


def test_device_potential_imaginary_time_is_static():
    """Imaginary time ignores the time dependence (classes_extension.py:389-392)."""
    lat, _, s_dev, dev, keep1 = _objects("device", "gpu")
    _, _, s_ref, ref, keep2 = _objects("static", "gpu")
    dev.evolve(20, True)
    ref.evolve(20, True)
    a, b = s_dev.get_state(), s_ref.get_state()
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    # and real time after imaginary time rebuilds the real-time kernel
    dev.evolve(4)
    want = oracle_steps(lat, a, 4, t0=20 * DT)
    assert np.abs(s_dev.get_state() - want).max() <= 1e-10


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_c_abi_table_from_device_potential(imag, precision):
    """ts_b200_set_potential_device == ts_b200_set_exp_potential of the host table."""
    import torch
    from trottersuzuki_b200 import Kernel
    lat, psi0, V = seeded_case(70, 9.0, 53, (False, True), 0.0, seed=5)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(DT, imag, 1.0, G, 0.0, 0.0, norm0=n0)
    tr, ti = O.exp_table(V, DT, imag)
    Vd = torch.zeros((V.shape[0], V.shape[1] + 6), dtype=torch.float64, device="cuda")
    Vd[:, :V.shape[1]] = torch.from_numpy(V)  # pitch > width
    out = []
    for mode in ("host", "device"):
        with Kernel(desc_from_params(p, precision)) as k:
            k.set_state(psi0)
            if mode == "host":
                k.set_exp_potential(tr, ti)
            else:
                torch.cuda.synchronize()
                k.set_potential_device(Vd.data_ptr(), Vd.shape[1], DT)
            k.evolve(10)
            out.append(k.get_state())
    tol = 1e-13 if precision == 0 else 1e-6
    assert np.abs(out[0] - out[1]).max() <= tol * np.abs(out[0]).max()


# (N, Ny, periodic, lhy): even tile widths take the step that forms the
# table's entries from the potential rows itself, the odd one the table pass
SEQUENCE_CASES = [(64, 48, (True, False), 0.0), (64, 64, (False, False), 0.3),
                  (61, 47, (False, False), 0.3)]


@pytest.mark.parametrize("case", SEQUENCE_CASES, ids=["periodic_x", "lhy", "odd_width"])
@pytest.mark.parametrize("exchange", [False, True])
def test_c_abi_potential_sequence_is_the_per_step_loop(exchange, case):
    """ts_b200_evolve_potentials == per step: set_potential_device, step,
    bit for bit (the fused path forms the same table entries)."""
    import torch
    from trottersuzuki_b200 import Kernel
    N, Ny, periodic, lhy = case
    lat, psi0, V = seeded_case(N, 8.0, Ny, periodic, 0.0, seed=8)
    p = lat.params(DT, False, 1.0, G, lhy, 0.0)
    X, Y = lat.coordinates()
    n = 6
    Vs = torch.from_numpy(np.stack([moving_trap(X, Y, i * DT) for i in range(n)])).cuda()
    slab = Vs.shape[1] * Vs.shape[2]
    out = []
    for mode in ("loop", "sequence"):
        with Kernel(desc_from_params(p)) as k:
            k.set_state(psi0)
            torch.cuda.synchronize()
            if mode == "loop":
                for i in range(n):
                    k.set_potential_device(Vs[i].data_ptr(), Vs.shape[2], DT)
                    k.step(exchange)
            else:
                k.evolve_potentials(Vs.data_ptr(), Vs.shape[2], slab, n, DT, exchange)
            out.append(k.get_state())
            # the table left for later steps is the last potential's either way
            k.step(False)
            out.append(k.get_state())
    assert np.array_equal(out[0], out[2])
    assert np.array_equal(out[1], out[3])


def test_c_abi_rejects_bad_potential_arguments():
    from trottersuzuki_b200 import B200Error, Kernel
    lat, psi0, V = seeded_case(32, 5.0, None, (False, False), 0.0)
    p = lat.params(DT, False, 1.0, 0.0, 0.0, 0.0)
    with Kernel(desc_from_params(p)) as k:
        with pytest.raises(B200Error):
            k.set_potential_device(0, 32, DT)  # null pointer
        with pytest.raises(B200Error):
            k.set_potential_device(16, 31, DT)  # pitch below the tile width
        with pytest.raises(B200Error):
            k.set_potential_device(16, 32, 0.0)  # delta_t must be positive
        with pytest.raises(B200Error):
            k.evolve_potentials(16, 32, 31 * 32, 2, DT)  # slab below one tile
        with pytest.raises(B200Error):
            k.evolve_potentials(16, 32, 32 * 32, -1, DT)  # negative count


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_device_table_values(imag):
    """The table itself, read back through one step with the kinetic pair
    rotations set to the identity and no nonlinearity: psi = 1 becomes the
    table (real time: cos(dt V) - i sin(dt V), the small-angle series below
    |dt V| = 1/16 and sincos above; imaginary time: exp(-dt V)), within 2 ulp
    of numpy's values."""
    import torch
    from trottersuzuki_b200 import Kernel
    lat, _, _ = seeded_case(256, 10.0, 8, (False, False), 0.0)
    p = lat.params(DT, imag, 1.0, 0.0, 0.0, 0.0, norm0=1.0)
    p.aH = p.aV = 1.0
    p.bH = p.bV = 0.0
    # angles dt V from -0.2 to 0.2 (both sides of the series threshold), a
    # few exact zeros and tiny values
    ang = np.linspace(-0.2, 0.2, lat.shape[0] * lat.shape[1]).reshape(lat.shape)
    ang[0, :4] = [0.0, 1e-300, -3e-9, 0.0625]
    V = ang / DT
    with Kernel(desc_from_params(p)) as k:
        k.set_state(np.ones(lat.shape, np.complex128))
        Vd = torch.from_numpy(np.ascontiguousarray(V)).cuda()
        torch.cuda.synchronize()
        k.set_potential_device(Vd.data_ptr(), V.shape[1], DT)
        k.evolve(1)
        got = k.get_state()
    a = DT * V  # the angle the kernel forms, dt * V rounded as on the device
    ys, xs = slice(p.iy0, p.iy1), slice(p.ix0, p.ix1)
    got = got[ys, xs]
    eps = np.finfo(np.float64).eps
    if imag:
        # imaginary time renormalises: compare up to the common scale
        want = np.exp(-a[ys, xs])
        r = got.real / want
        assert np.abs(got.imag).max() == 0.0
        assert np.abs(r / r.mean() - 1.0).max() <= 4 * eps
    else:
        want = np.cos(a[ys, xs]) - 1j * np.sin(a[ys, xs])
        assert np.abs(got.real - want.real).max() <= 2 * eps
        assert np.all(np.abs(got.imag - want.imag) <= 2 * eps * np.abs(want.imag) + 1e-320)
