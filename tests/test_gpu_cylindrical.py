"""Cylindrical lattices on the GPU (radial kinetic sweeps fused into the step,
the mirrored axis column fused into the store) against the reference's
cylindrical Solver (golden fixtures under tests/golden/cyl/) and the oracle."""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, energy_params
from test_oracle_cyl import cyl_names, load_cyl, oracle_cyl

pytestmark = pytest.mark.gpu


def run_kernel(lat, meta, z, precision=0):
    from trottersuzuki_b200 import Kernel
    psi = z["psi0"]
    Vt = z["V"] + lat.azimuthal(meta["l"])
    k, n0, prev = None, 0.0, None
    for it, imag in meta["segments"]:
        if k is None or imag != prev:
            if imag:
                n0 = O.expectations(lat, psi)["norm2"] if k is None else k.squared_norm()
            p = lat.params(meta["dt"], imag, 1.0, meta["g"], 0.0, 0.0, norm0=n0,
                           angular_momentum=meta["l"])
            if k is not None:
                psi = k.get_state()
                k.close()
            k = Kernel(desc_from_params(p, precision))
            k.set_state(psi)
            k.set_exp_potential(*O.exp_table(Vt, meta["dt"], imag))
        k.evolve(it)
        prev = imag
    return k, Vt


@pytest.mark.parametrize("name", cyl_names())
def test_cylindrical_matches_reference_fixture(name):
    lat, meta, z = load_cyl(name)
    k, Vt = run_kernel(lat, meta, z)
    assert np.abs(k.get_state() - z["psi"]).max() <= 1e-10
    e = k.energies(Vt, energy_params(lat, 1.0, meta["g"]))
    got = np.array([e[n] for n in ("total", "kinetic", "potential", "rotational", "intra", "lhy",
                                   "norm2")])
    assert np.allclose(got, z["energies"], rtol=1e-10, atol=1e-12), (got, z["energies"])
    k.close()


@pytest.mark.parametrize("name", ["cyl_real_l0", "cyl_imag_l1"])
def test_cylindrical_fp32_storage(name):
    lat, meta, z = load_cyl(name)
    k, _ = run_kernel(lat, meta, z, precision=1)
    assert np.abs(k.get_state() - z["psi"]).max() <= 2e-5 * np.abs(z["psi"]).max()
    k.close()


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_wide_cylindrical_tile_matches_oracle(imag):
    """A tile wider than one strip of the kernel (and than one cache block of
    the reference, whose block edges leave a 1e-14 trace there): GPU against
    the oracle's whole-tile sweeps, odd angular momentum (mirror sign -1)."""
    from trottersuzuki_b200 import Kernel
    lat = O.Lattice(300, 20.0, 64, 8.0, cylindrical=True)
    X, Y = lat.coordinates()
    rng = np.random.default_rng(11)
    psi0 = X * np.exp(-(X ** 2 / 8.0 + Y ** 2) / 2.0) * (1 + 0.01 * rng.uniform(-1, 1, lat.shape))
    psi0 = psi0 * np.exp(0.3j * Y)
    Vt = 0.5 * (X ** 2 + Y ** 2) + lat.azimuthal(3)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(2e-3, imag, 1.0, 5.0, 0.0, 0.0, norm0=n0, angular_momentum=3)
    tr, ti = O.exp_table(Vt, 2e-3, imag)
    with Kernel(desc_from_params(p)) as k:
        k.set_state(psi0)
        k.set_exp_potential(tr, ti)
        k.evolve(23)
        got = k.get_state()
    ref = O.evolve(p, psi0, tr, ti, 23)
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    if imag:
        assert np.array_equal(got[:, 0], -got[:, 1])  # the axis column mirrors column 1


def test_cylindrical_rejects_rotation_and_radial_periodicity():
    from trottersuzuki_b200 import B200Error, Kernel
    lat = O.Lattice(40, 8.0, cylindrical=True)
    p = lat.params(1e-3)
    d = desc_from_params(p)
    d.periodic_x = 1
    with pytest.raises(B200Error):
        Kernel(d)
    d = desc_from_params(p)
    d.alpha_x = d.alpha_y = 0.1
    with pytest.raises(B200Error):
        Kernel(d)


@pytest.mark.parametrize("name", cyl_names())
def test_drop_in_cylindrical_solver(name):
    """Lattice2D(..., coordinate_system="cylindrical"), State(grid, l) and the
    Solver: the azimuthal term enters the table and the energies."""
    import trottersuzuki_b200 as ts
    lat, meta, z = load_cyl(name)
    N, L, Ny, Ly, py = meta["lat"]
    grid = ts.Lattice2D(N, L, Ny, Ly, periodic_y_axis=py, coordinate_system="cylindrical")
    state = ts.State(grid, meta["l"])
    state.init_state_matrix(z["psi0"].real, z["psi0"].imag)
    pot = ts.Potential(grid, z["V"])
    ham = ts.Hamiltonian(grid, pot, 1.0, meta["g"])
    solver = ts.Solver(grid, state, ham, meta["dt"])
    for it, imag in meta["segments"]:
        solver.evolve(it, imag)
    assert np.abs(state.get_state() - z["psi"]).max() <= 1e-10
    got = solver._energies()
    assert np.allclose(got, z["energies"], rtol=1e-10, atol=1e-12), (got, z["energies"])


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("g,l", [(0.0, 0), (40.0, 1), (25.0, 2)])
def test_cylindrical_look_ahead_walk_matches_checked_walk(imag, walk, g, l):
    """The look-ahead walk on a cylindrical lattice (radial sweeps around the
    potential stage, 8 halo columns, the mirrored axis column at the store):
    the checked walk's bits in real time, its result to 1e-13 in imaginary
    time, the oracle at the parity bar; a tall ragged tile in several
    segments and strips, two evolve calls."""
    from trottersuzuki_b200 import Kernel
    lat = O.Lattice(150, 8.0, 133, 10.0, cylindrical=True)
    X, Y = lat.coordinates()
    rng = np.random.default_rng(7 + l)
    psi0 = np.exp(-((X - 2.0) ** 2 + Y ** 2) / 3.0) * (1 + 0.05 * rng.uniform(-1, 1, lat.shape))
    psi0 = psi0 * np.exp(0.3j * Y)
    V = 0.5 * (X ** 2 + Y ** 2) + lat.azimuthal(l)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(1e-3, imag, 1.0, g, 0.0, 0.0, norm0=n0, angular_momentum=l)
    tr, ti = O.exp_table(V, 1e-3, imag)
    ref = O.evolve(p, O.evolve(p, psi0, tr, ti, 6), tr, ti, 5)
    out = {}
    for wk in (walk, 0):
        with Kernel(desc_from_params(p)) as k:
            k.set_walk(wk)
            k.set_launch(segment_rows=24)
            assert k.launch_shape()["walk"] == wk
            k.set_state(psi0)
            k.set_exp_potential(tr, ti)
            k.evolve(6)
            k.evolve(5)
            out[wk] = k.get_state()
    got, old = out[walk], out[0]
    assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()
    if imag:
        assert np.abs(got - old).max() <= 1e-13 * np.abs(old).max()
    else:
        assert np.array_equal(got, old)
