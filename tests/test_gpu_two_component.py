"""Two components on the GPU (ts_b200_pair_*) against the reference's
two-state Solver (golden fixtures under tests/golden/two/) and the oracle.

One evolve() call of the reference's two-component Solver is a Rabi half step
followed by the loop (src/solver.cpp:172-230); here that is pair.rabi(0.5)
then pair.evolve(n).  The species' tiles keep their own states, tables and
step constants; the cross energies come from the pair.
"""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, energy_params
from test_oracle_two import load_two, oracle_two, two_names

pytestmark = pytest.mark.gpu


def run_pair(lat, meta, z, precision=0, segments=None, walk=None, seg_rows=0):
    from trottersuzuki_b200 import Kernel, Pair
    dt, imag = meta["dt"], meta["segments"][0][1]
    a0, b0 = z["psi0_a"], z["psi0_b"]
    na = O.expectations(lat, a0)["norm2"] if imag else 0.0
    nb = O.expectations(lat, b0)["norm2"] if imag else 0.0
    pa = lat.params(dt, imag, 1.0, meta["g"], 0.0, 0.0, norm0=na)
    pb = lat.params(dt, imag, meta["mass_b"], meta["g_b"], 0.0, 0.0, norm0=nb)
    ka, kb = Kernel(desc_from_params(pa, precision)), Kernel(desc_from_params(pb, precision))
    for k in (ka, kb):
        if walk is not None:
            k.set_walk(walk)
        if seg_rows:
            k.set_launch(segment_rows=seg_rows)
    ka.set_state(a0)
    kb.set_state(b0)
    ka.set_exp_potential(*O.exp_table(z["Va"], dt, imag))
    kb.set_exp_potential(*O.exp_table(z["Vb"], dt, imag))
    pair = Pair(ka, kb, meta["g_ab"], meta["omega"][0], meta["omega"][1], dt)
    for it, seg_imag in (segments or meta["segments"]):
        assert seg_imag == imag
        pair.rabi(0.5)
        pair.evolve(it)
    return ka, kb, pair


def gpu_energies(lat, meta, z, ka, kb, pair):
    ea = ka.energies(z["Va"], energy_params(lat, 1.0, meta["g"]))
    eb = kb.energies(z["Vb"], energy_params(lat, meta["mass_b"], meta["g_b"]))
    inter, rabi = pair.cross_energies()
    total = sum(e[k] for e in (ea, eb) for k in ("kinetic", "potential", "intra", "rotational"))
    total += inter + rabi
    return np.array([total, ea["kinetic"], eb["kinetic"], ea["potential"], eb["potential"],
                     ea["rotational"], eb["rotational"], ea["intra"], eb["intra"], inter, rabi,
                     ea["norm2"], eb["norm2"]])


@pytest.mark.parametrize("name", two_names())
def test_pair_matches_reference_fixture(name):
    lat, meta, z = load_two(name)
    ka, kb, pair = run_pair(lat, meta, z)
    a, b = ka.get_state(), kb.get_state()
    assert np.abs(a - z["psi_a"]).max() <= 1e-10
    assert np.abs(b - z["psi_b"]).max() <= 1e-10
    e = gpu_energies(lat, meta, z, ka, kb, pair)
    assert np.allclose(e, z["energies"], rtol=1e-10, atol=1e-12), (e, z["energies"])
    pair.close()


@pytest.mark.parametrize("name", ["two_real_rabi", "two_imag_rabi"])
def test_pair_fp32_storage(name):
    lat, meta, z = load_two(name)
    ka, kb, pair = run_pair(lat, meta, z, precision=1)
    a, b = ka.get_state(), kb.get_state()
    for got, want in ((a, z["psi_a"]), (b, z["psi_b"])):
        assert np.abs(got - want).max() <= 2e-5 * np.abs(want).max()
    e = gpu_energies(lat, meta, z, ka, kb, pair)
    assert np.allclose(e, z["energies"], rtol=2e-5, atol=1e-9)
    pair.close()


def test_pair_longer_run_matches_oracle():
    """Many steps, odd step counts per call (buffer parities of both species)."""
    lat, meta, z = load_two("two_imag_rabi")
    segs = [(33, True), (8, True)]
    ka, kb, pair = run_pair(lat, meta, z, segments=segs)
    ref_a, ref_b, _ = oracle_two(lat, dict(meta, segments=segs), z)
    assert np.abs(ka.get_state() - ref_a).max() <= 1e-10
    assert np.abs(kb.get_state() - ref_b).max() <= 1e-10
    pair.close()


def test_pair_rules():
    from trottersuzuki_b200 import B200Error, Kernel, Pair
    lat, meta, z = load_two("two_real_rabi")
    p = lat.params(1e-3, False, 1.0, 1.0, 0.0, 0.0)
    ka, kb = Kernel(desc_from_params(p)), Kernel(desc_from_params(p))
    for k, s in ((ka, z["psi0_a"]), (kb, z["psi0_b"])):
        k.set_state(s)
        k.set_exp_potential(*O.exp_table(z["Va"], 1e-3, False))
    with pytest.raises(B200Error):
        Pair(ka, ka, 1.0, 0.0, 0.0, 1e-3)  # the same tile twice
    other = O.Lattice(32, 8.0)
    kc = Kernel(desc_from_params(other.params(1e-3, False)))
    with pytest.raises(B200Error):
        Pair(ka, kc, 1.0, 0.0, 0.0, 1e-3)  # different geometry
    pair = Pair(ka, kb, 1.0, 2.0, 0.0, 1e-3)
    with pytest.raises(B200Error):
        ka.evolve(1)  # a paired tile steps only through the pair
    with pytest.raises(B200Error):
        Pair(ka, kc, 1.0, 0.0, 0.0, 1e-3)  # already paired
    pair.evolve(3)
    pair.close()
    # unpaired, each tile steps alone again and matches a fresh single tile
    psi = ka.get_state()
    ka.evolve(5)
    with Kernel(desc_from_params(p)) as k1:
        k1.set_state(psi)
        k1.set_exp_potential(*O.exp_table(z["Va"], 1e-3, False))
        k1.evolve(5)
        assert np.array_equal(k1.get_state(), ka.get_state())


# ------------------------------------------------------- the drop-in Solver
def _drop_in(name, kernel_type="gpu"):
    import trottersuzuki_b200 as ts
    lat, meta, z = load_two(name)
    N, L, Ny, px, py = meta["lat"]
    grid = ts.Lattice2D(N, L, Ny, None, periodic_x_axis=px, periodic_y_axis=py)
    sa, sb = ts.State(grid), ts.State(grid)
    sa.init_state_matrix(z["psi0_a"].real, z["psi0_a"].imag)
    sb.init_state_matrix(z["psi0_b"].real, z["psi0_b"].imag)
    pa, pb = ts.Potential(grid, z["Va"]), ts.Potential(grid, z["Vb"])
    ham = ts.Hamiltonian2Component(grid, pa, pb, 1.0, meta["mass_b"], meta["g"], meta["g_ab"],
                                   meta["g_b"], *meta["omega"])
    solver = ts.Solver(grid, sa, ham, meta["dt"], State2=sb, kernel_type=kernel_type)
    return meta, z, solver, (sa, sb), (grid, pa, pb, ham)


@pytest.mark.parametrize("name", two_names())
def test_drop_in_two_component_solver(name):
    meta, z, solver, (sa, sb), keep = _drop_in(name)
    for it, imag in meta["segments"]:
        solver.evolve(it, imag)
    assert np.abs(sa.get_state() - z["psi_a"]).max() <= 1e-10
    assert np.abs(sb.get_state() - z["psi_b"]).max() <= 1e-10
    got = [solver.get_total_energy(), solver.get_kinetic_energy(1), solver.get_kinetic_energy(2),
           solver.get_potential_energy(1), solver.get_potential_energy(2),
           solver.get_rotational_energy(1), solver.get_rotational_energy(2),
           solver.get_intra_species_energy(1), solver.get_intra_species_energy(2),
           solver.get_inter_species_energy(), solver.get_rabi_energy(),
           solver.get_squared_norm(1), solver.get_squared_norm(2)]
    assert np.allclose(got, z["energies"], rtol=1e-10, atol=1e-12), (got, z["energies"])
    assert abs(solver.get_squared_norm() - z["energies"][11] - z["energies"][12]) < 1e-12


@pytest.mark.parametrize("kernel_type", ["gpu", "gpu_fp32"])
def test_kat_mixed_bec(kernel_type):
    """test/kerneltest.cpp:177-235 through the Python drop-in."""
    import math

    import trottersuzuki_b200 as ts
    for imag in (False, True):
        grid = ts.Lattice2D(250, 100.0)
        s1 = ts.GaussianState(grid, 1.0)
        s2 = ts.State(grid)
        pot = ts.HarmonicPotential(grid, 1.0, 1.0)
        ham = ts.Hamiltonian2Component(grid, pot, pot, 1.0, 1.0, 0.0, 0.0, 0.0,
                                       2.0 * math.pi / 10.0)
        solver = ts.Solver(grid, s1, ham, 1e-3, State2=s2, kernel_type=kernel_type)
        # the second species starts empty: the initial energy is 0/0 (NaN),
        # in the reference too, so only the norms are compared
        n0 = solver.get_squared_norm(1) + solver.get_squared_norm(2)
        n01, n02 = s1.get_squared_norm(), s2.get_squared_norm()
        solver.evolve(1000 if imag else 5000, imag)
        assert math.isfinite(solver.get_total_energy())
        assert abs(n0 - solver.get_squared_norm()) < 1e-5
        if imag:
            assert abs(0.915292 - s1.get_squared_norm()) < 1e-5
            assert abs(0.084708 - s2.get_squared_norm()) < 1e-5
        else:
            assert abs(n01 - s2.get_squared_norm()) < 1e-5
            assert abs(n02 - s1.get_squared_norm()) < 1e-5


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_pair_with_an_empty_species_matches_oracle(imag):
    import math

    from test_oracle_two import empty_species_case
    from trottersuzuki_b200 import Kernel, Pair
    lat, a, b, V = empty_species_case()
    om, dt = 2 * math.pi / 10, 1e-3
    norms = (O.expectations(lat, a)["norm2"], 0.0) if imag else (0.0, 0.0)
    p_a = lat.params(dt, imag, norm0=norms[0])
    p_b = lat.params(dt, imag, norm0=0.0)
    table = O.exp_table(V, dt, imag)
    ka, kb = Kernel(desc_from_params(p_a)), Kernel(desc_from_params(p_b))
    ka.set_state(a)
    kb.set_state(b)
    ka.set_exp_potential(*table)
    kb.set_exp_potential(*table)
    pair = Pair(ka, kb, 0.0, om, 0.0, dt)
    pair.rabi(0.5)
    pair.evolve(150)
    oa, ob, _ = O.evolve2(lat.params(dt, imag), lat.params(dt, imag), 0.0, om, 0.0, dt, a, b,
                          table, table, 150, norms, sum(norms))
    assert np.abs(ka.get_state() - oa).max() <= 1e-10
    assert np.abs(kb.get_state() - ob).max() <= 1e-10
    pair.close()


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("name", ["two_real_rabi", "two_imag_rabi"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_pair_look_ahead_walk_matches_checked_walk(name, walk, precision):
    """Both species on the look-ahead walk (the other species' rows in the
    ring, the Rabi rotation at load in real time, the joint normalisation in
    the last block) against the checked walk: its bits in real time, its
    result to rounding in imaginary time; short segments so that every tile
    has several, odd step counts per call."""
    lat, meta, z = load_two(name)
    imag = meta["segments"][0][1]
    segs = [(7, imag), (4, imag)]
    out = {}
    for wk in (walk, 0):
        ka, kb, pair = run_pair(lat, meta, z, precision=precision, segments=segs, walk=wk,
                                seg_rows=10)
        assert ka.launch_shape()["walk"] == wk
        out[wk] = (ka.get_state(), kb.get_state())
        pair.close()
    for got, old in zip(out[walk], out[0]):
        if imag:
            tol = 1e-13 if precision == 0 else 1e-6
            assert np.abs(got - old).max() <= tol * np.abs(old).max()
        else:
            assert np.array_equal(got, old)
