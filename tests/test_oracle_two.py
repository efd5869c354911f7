"""Two-component oracle (Hamiltonian2Component path) pinned to the reference.

The fixtures under tests/golden/two/ are outputs of the reference's own CPU
implementation (tests/golden/gen_golden.py): two states evolved together
with intra- and inter-species couplings, different masses and a Rabi
coupling, in real and imaginary time (src/solver.cpp:172-230,
src/cpukernel.cpp:274-392,581-667, src/cpucartesian.cpp:73-126,264-290).
"""
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
TWO = os.path.join(HERE, "golden", "two")


def two_names():
    return sorted(f[:-4] for f in os.listdir(TWO) if f.endswith(".npz"))


def load_two(name):
    z = np.load(os.path.join(TWO, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    N, L, Ny, px, py = meta["lat"]
    lat = O.Lattice(N, L, Ny, None, px, py, 0.0)
    return lat, meta, {k: z[k] for k in z.files if k != "meta"}


def oracle_two(lat, meta, z):
    """The fixture's evolve() calls through the oracle; returns (a, b, energies)."""
    a, b = z["psi0_a"], z["psi0_b"]
    dt, ga, gb, gab = meta["dt"], meta["g"], meta["g_b"], meta["g_ab"]
    om_r, om_i = meta["omega"]
    norms, tot, prev = (0.0, 0.0), None, None
    for it, imag in meta["segments"]:
        if imag and prev is not True:  # kernel (re)built: norms from the states
            norms = (O.expectations(lat, a)["norm2"], O.expectations(lat, b)["norm2"])
            tot = norms[0] + norms[1]
        pa = lat.params(dt, imag, 1.0, ga, 0.0, 0.0)
        pb = lat.params(dt, imag, meta["mass_b"], gb, 0.0, 0.0)
        ta = O.exp_table(z["Va"], dt, imag)
        tb = O.exp_table(z["Vb"], dt, imag)
        a, b, norms = O.evolve2(pa, pb, gab * dt, om_r, om_i, dt, a, b, ta, tb, it, norms,
                                tot if tot is not None else 0.0)
        prev = imag
    ea = O.energies(lat, a, z["Va"], 1.0, ga)
    eb = O.energies(lat, b, z["Vb"], meta["mass_b"], gb)
    inter, rabi = O.cross_energies(lat, a, b, gab, om_r, om_i)
    total = (ea["kinetic"] + ea["potential"] + ea["intra"] + ea["rotational"] + eb["kinetic"] +
             eb["potential"] + eb["intra"] + eb["rotational"] + inter + rabi)
    e = np.array([total, ea["kinetic"], eb["kinetic"], ea["potential"], eb["potential"],
                  ea["rotational"], eb["rotational"], ea["intra"], eb["intra"], inter, rabi,
                  ea["norm2"], eb["norm2"]])
    return a, b, e


@pytest.mark.parametrize("name", two_names())
def test_oracle_reproduces_two_component_fixture(name):
    lat, meta, z = load_two(name)
    a, b, e = oracle_two(lat, meta, z)
    assert np.abs(a - z["psi_a"]).max() <= 1e-12
    assert np.abs(b - z["psi_b"]).max() <= 1e-12
    assert np.allclose(e, z["energies"], rtol=1e-11, atol=1e-13), (e, z["energies"])


def test_rabi_alone_is_unitary_in_real_time():
    lat = O.Lattice(24, 6.0)
    rng = np.random.default_rng(4)
    a = rng.normal(size=lat.shape) + 1j * rng.normal(size=lat.shape)
    b = rng.normal(size=lat.shape) + 1j * rng.normal(size=lat.shape)
    p = lat.params(1e-3, False)
    a2, b2 = O.rabi(p, 3.0, 1.0, 1.0, 0.05, a, b)
    n0 = np.abs(a) ** 2 + np.abs(b) ** 2
    assert np.allclose(np.abs(a2) ** 2 + np.abs(b2) ** 2, n0, rtol=1e-13)
    assert np.abs(a2 - a).max() > 1e-3


def empty_species_case(n=48, L=20.0):
    """The reference's mixed-BEC scenario (test/kerneltest.cpp:177-235) on a
    small lattice: a Gaussian first species, an empty second one, Rabi
    coupling 2 pi / 10."""
    lat = O.Lattice(n, L)
    X, Y = lat.coordinates()
    a = np.exp(-(X ** 2 + Y ** 2) / 2.0) + 0j
    a = a / np.sqrt(np.sum(np.abs(a) ** 2) * lat.delta_x * lat.delta_y)
    b = np.zeros_like(a)
    V = 0.5 * (X ** 2 + Y ** 2)
    return lat, a, b, V


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_oracle_matches_reference_with_an_empty_species(imag):
    """The species that starts empty is renormalised once the joint
    normalisation gives it a share (its kept norm starts at 0)."""
    import math

    import tsref
    if not tsref.available():
        pytest.skip("compiled reference not built")
    lat, a, b, V = empty_species_case()
    om = 2 * math.pi / 10
    cfg = tsref.make_config(lat.dim_x, 20.0, harmonic=None, delta_t=1e-3,
                            segments=((150, imag),), omp_threads=1)
    ra, rb, res = tsref.run2(cfg, tsref.Config2(1.0, 0.0, 0.0, om, 0.0), a, b, V, V)
    pa = lat.params(1e-3, imag)
    norms = (O.expectations(lat, a)["norm2"], 0.0) if imag else (0.0, 0.0)
    oa, ob, _ = O.evolve2(pa, pa, 0.0, om, 0.0, 1e-3, a, b, O.exp_table(V, 1e-3, imag),
                          O.exp_table(V, 1e-3, imag), 150, norms, sum(norms))
    assert np.abs(oa - ra).max() <= 1e-12
    assert np.abs(ob - rb).max() <= 1e-12
