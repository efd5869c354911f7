"""Pin the oracle restatement (oracle/ts_oracle.c) to the reference.

1. Golden fixtures (tests/golden/*.npz, produced by the reference itself via
   tests/golden/gen_golden.py) must be reproduced bit for bit.
2. When the compiled reference is present (oracle/_ref), seeded cases are run
   on both and must agree bit for bit.
3. The reference's own known-answer tests (test/kerneltest.cpp:7-175) hold on
   the oracle with the reference's tolerances (test/kerneltest.h:8-9).
"""
import numpy as np
import pytest

import oracle as O
import tsref
from helpers import golden_names, load_golden, oracle_run_golden, seeded_case

TOLERANCE = 1e-3       # test/kerneltest.h:8
NORM_TOLERANCE = 1e-5  # test/kerneltest.h:9


@pytest.mark.parametrize("name", golden_names())
def test_oracle_reproduces_golden_fixture(name):
    g = load_golden(name)
    psi = oracle_run_golden(g)
    assert np.array_equal(psi, g["psi"]), np.abs(psi - g["psi"]).max()
    m = g["meta"]
    e = O.energies(g["lat"], psi, g["V"], 1.0, m["g"], m["lhy"], m["omega"])
    ref = g["energies"]
    got = [e["total"], e["kinetic"], e["potential"], e["rotational"], e["intra"], e["lhy"],
           e["norm2"]]
    assert np.array_equal(np.array(got), ref), (got, ref)
    if not g["lat"].one_d:
        x = O.expectations(g["lat"], psi)
        xr = g["expectations"]
        got = [x[k] for k in ("norm2", "mean_x", "mean_xx", "mean_y", "mean_yy", "mean_px",
                              "mean_pxpx", "mean_py", "mean_pypy", "mean_lz")]
        assert np.array_equal(np.array(got), xr), (got, xr)


LIVE = [
    (64, 10.0, None, (False, False), 0.0, 0.0, 0.0, False),
    (61, 10.0, 47, (False, False), 0.0, 4.0, 0.2, False),
    (64, 10.0, None, (True, True), 0.0, 1.0, 0.0, True),
    (64, 10.0, None, (True, False), 0.0, 0.0, 0.0, False),
    (64, 10.0, None, (False, False), 0.7, 3.0, 0.0, False),
    (300, 20.0, None, (False, False), 0.7, 2.0, 0.0, True),
    (160, 10.0, None, (True, True), 0.0, 0.0, 0.0, False),
]


@pytest.mark.skipif(not tsref.available(), reason="compiled reference not built")
@pytest.mark.parametrize("case", LIVE)
def test_oracle_matches_compiled_reference(case):
    N, L, Ny, per, omega, g, lhy, imag = case
    lat, psi0, V = seeded_case(N, L, Ny, per, omega, seed=N)
    steps = 6
    cfg = tsref.make_config(N, L, Ny, None, per[0], per[1], omega, coupling=g, lhy_coupling=lhy,
                            angular_velocity=omega, delta_t=1e-3, segments=((steps, imag),))
    ref, res = tsref.run(cfg, psi0, V)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(1e-3, imag, 1.0, g, lhy, omega, norm0=n0)
    tr, ti = O.exp_table(V, 1e-3, imag)
    psi = O.evolve(p, psi0, tr, ti, steps)
    assert np.array_equal(psi, ref)
    e = O.energies(lat, psi, V, 1.0, g, lhy, omega)
    assert e["total"] == res.total_energy


@pytest.mark.skipif(not tsref.available(), reason="compiled reference not built")
def test_reference_defect_width_248_is_not_restated():
    """Tile widths 128+120q leave columns [124, 244) unwritten in the reference's
    cache blocking (src/cpukernel.cpp:111,151); the restatement computes them."""
    lat = O.Lattice(248, 20.0)
    psi0 = O.gaussian(lat, 1.0, 1.0, 1.0, 0.0)
    V = lat.harmonic(1.0, 1.0)
    cfg = tsref.make_config(248, 20.0, segments=((1, False),))
    ref, _ = tsref.run(cfg, psi0, V)
    assert np.abs(ref[:, 124:244]).max() == 0.0
    p = lat.params(1e-4, False)
    tr, ti = O.exp_table(V, 1e-4, False)
    psi = O.evolve(p, psi0, tr, ti, 1)
    assert np.abs(psi[:, 124:244]).max() > 0.1
    # elsewhere the two agree
    assert np.array_equal(psi[:, :124], ref[:, :124])


# ------------------------------------------- reference KATs on the oracle
def _solve(lat, psi0, V, dt, steps, imag, g=0.0, lhy=0.0, omega=0.0):
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(dt, imag, 1.0, g, lhy, omega, norm0=n0)
    tr, ti = O.exp_table(V, dt, imag)
    return O.evolve(p, psi0, tr, ti, steps)


def test_kat_free_particle():
    """test/kerneltest.cpp:7-27: periodic 250^2, L=100, plane wave, 100 steps."""
    lat = O.Lattice(250, 100.0, None, None, True, True)
    psi0 = O.exponential(lat)
    V = np.zeros(lat.shape)
    e0 = O.energies(lat, psi0, V)
    psi = _solve(lat, psi0, V, 5e-3, 100, False)
    e1 = O.energies(lat, psi, V)
    assert abs(e0["total"] - e1["total"]) < TOLERANCE
    assert abs(e0["norm2"] - e1["norm2"]) < NORM_TOLERANCE


def test_kat_imaginary_harmonic_oscillator():
    """test/kerneltest.cpp:52-73: ground state energy 1.00001 after 1000 imaginary steps."""
    lat = O.Lattice(250, 100.0)
    psi0 = O.gaussian(lat, 0.5)
    V = lat.harmonic(1.0, 1.0)
    n0 = O.energies(lat, psi0, V)["norm2"]
    psi = _solve(lat, psi0, V, 5e-3, 1000, True)
    e = O.energies(lat, psi, V)
    assert abs(1.00001 - e["total"]) < TOLERANCE
    assert abs(n0 - e["norm2"]) < NORM_TOLERANCE


def test_kat_imaginary_intra_particle_interaction():
    """test/kerneltest.cpp:101-125: g=10, E = 1.59273, <x^2> = 0.768148."""
    lat = O.Lattice(250, 100.0)
    psi0 = O.gaussian(lat, 1.0)
    V = lat.harmonic(1.0, 1.0)
    psi = _solve(lat, psi0, V, 1e-3, 1000, True, g=10.0)
    e = O.energies(lat, psi, V, 1.0, 10.0)
    x = O.expectations(lat, psi)
    assert abs(1.59273 - e["total"]) < TOLERANCE
    assert abs(0.768148 - x["mean_xx"]) < TOLERANCE


@pytest.mark.parametrize("g,lhy", [(0.0, 0.0), (3.0, 0.0), (3.0, 0.8)])
def test_cpu_adjoint_matches_finite_differences(g, lhy):
    """The CPU FP64 adjoint (the check of the B200 adjoint) against central
    differences of the oracle forward pass, for L = sum_{x>0} |psi(T)|^2 dA."""
    lat = O.Lattice(24, 6.0, 20, None)
    rng = np.random.default_rng(1)
    X, _ = lat.coordinates()
    psi0 = O.gaussian(lat, 1.0, 1.0, -0.5, 0.0) * np.exp(2j * X)
    V = lat.harmonic(1.0, 1.0) + 0.2 * rng.uniform(-1, 1, lat.shape)
    dt, steps = 1e-2, 30
    p = lat.params(dt, False, 1.0, g, lhy, 0.0)
    dA = lat.delta_x * lat.delta_y
    mask = X > 0

    def loss(Vh, ph):
        tr, ti = O.exp_table(Vh, dt, False)
        psi = O.evolve(p, ph, tr, ti, steps)
        return float((np.abs(psi) ** 2 * mask).sum() * dA), psi

    _, psi_t = loss(V, psi0)
    tr, ti = O.exp_table(V, dt, False)
    gv, gp = O.adjoint_real(p, tr, ti, dt, psi0, steps, 2 * dA * mask * psi_t)
    h = 1e-5
    sites = [(10, 12), (5, 3), (15, 20), (9, 8), (3, 17)]
    fd = []
    for y, x in sites:
        e = np.zeros_like(V)
        e[y, x] = h
        fd.append(((loss(V + e, psi0)[0] - loss(V - e, psi0)[0]) / (2 * h),
                   (loss(V, psi0 + e)[0] - loss(V, psi0 - e)[0]) / (2 * h),
                   (loss(V, psi0 + 1j * e)[0] - loss(V, psi0 - 1j * e)[0]) / (2 * h)))
    fd = np.array(fd)
    ys, xs = zip(*sites)
    for col, adj in ((0, gv[ys, xs]), (1, gp.real[ys, xs]), (2, gp.imag[ys, xs])):
        assert np.abs(adj - fd[:, col]).max() <= 1e-6 * np.abs(fd[:, col]).max()


@pytest.mark.parametrize("g,lhy", [(0.0, 0.0), (3.0, 0.0), (3.0, 0.8)])
def test_cpu_imag_adjoint_matches_finite_differences(g, lhy):
    """The CPU FP64 imaginary-time adjoint (renormalisation after every step
    to the initial norm) against central differences of the oracle's
    imaginary-time evolution, for L = sum_{x>0} |psi(T)|^2 dA; the initial
    norm moves with psi0 as in Solver::evolve (src/solver.cpp:155)."""
    lat = O.Lattice(24, 6.0, 20, None)
    rng = np.random.default_rng(2)
    X, _ = lat.coordinates()
    psi0 = (O.gaussian(lat, 1.0, 1.0, -0.5, 0.3) * (1 + 0.3 * rng.uniform(-1, 1, lat.shape))
            * np.exp(0.7j * X))
    V = lat.harmonic(1.0, 1.0) + 0.2 * rng.uniform(-1, 1, lat.shape)
    dt, steps = 1e-2, 30
    dA = lat.delta_x * lat.delta_y
    mask = X > 0

    def loss(Vh, ph):
        n0 = O.expectations(lat, ph)["norm2"]
        p = lat.params(dt, True, 1.0, g, lhy, 0.0, norm0=n0)
        tr, ti = O.exp_table(Vh, dt, True)
        psi = O.evolve(p, ph, tr, ti, steps)
        return float((np.abs(psi) ** 2 * mask).sum() * dA), psi

    _, psi_t = loss(V, psi0)
    p = lat.params(dt, True, 1.0, g, lhy, 0.0, norm0=O.expectations(lat, psi0)["norm2"])
    tr, _ = O.exp_table(V, dt, True)
    gv, gp = O.adjoint_imag(p, tr, dt, psi0, steps, 2 * dA * mask * psi_t)
    h = 1e-5
    sites = [(10, 12), (5, 3), (15, 20), (9, 8), (3, 17)]
    fd = []
    for y, x in sites:
        e = np.zeros_like(V)
        e[y, x] = h
        fd.append(((loss(V + e, psi0)[0] - loss(V - e, psi0)[0]) / (2 * h),
                   (loss(V, psi0 + e)[0] - loss(V, psi0 - e)[0]) / (2 * h),
                   (loss(V, psi0 + 1j * e)[0] - loss(V, psi0 - 1j * e)[0]) / (2 * h)))
    fd = np.array(fd)
    ys, xs = zip(*sites)
    for col, adj in ((0, gv[ys, xs]), (1, gp.real[ys, xs]), (2, gp.imag[ys, xs])):
        assert np.abs(adj - fd[:, col]).max() <= 1e-6 * np.abs(fd[:, col]).max()
