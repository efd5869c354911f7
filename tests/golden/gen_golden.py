"""Generate the golden fixtures in this folder by running the reference itself.

The reference's own CPU implementation (trotter-suzuki-mpi 1.6.2, compiled
from its sources by oracle/build_ref.sh into oracle/_ref/libtsref.so) evolves
seeded inputs; each case stores the inputs (initial tile, potential V), the
parameters and the reference's outputs (final tile, energies, expectation
values) as a compressed .npz.  The reference ships no golden vectors of its
own; these fixtures pin both the oracle restatement and the B200 kernel.

    python tests/golden/gen_golden.py        (needs oracle/_ref, i.e. the reference sources)

Two-component cases (Hamiltonian2Component, the two-state Solver) go to two/,
cylindrical lattices (the radial kinetic term, the azimuthal potential, the
mirrored axis column) to cyl/.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))

import oracle as O  # noqa: E402
import tsref  # noqa: E402

# name: lattice (N, L, Ny, periodic_x, periodic_y, omega, one_d), physics, evolve segments
CASES = {
    "closed_real": dict(lat=(64, 10.0, None, False, False, 0.0, False), g=0.0, lhy=0.0,
                        omega=0.0, dt=1e-3, segments=[(50, False)]),
    "gpe_lhy_real": dict(lat=(48, 8.0, None, False, False, 0.0, False), g=5.0, lhy=0.3,
                         omega=0.0, dt=1e-3, segments=[(30, False)]),
    "gpe_imag": dict(lat=(48, 8.0, None, False, False, 0.0, False), g=5.0, lhy=0.0, omega=0.0,
                     dt=1e-3, segments=[(40, True)]),
    "periodic_real": dict(lat=(40, 8.0, 36, True, True, 0.0, False), g=1.0, lhy=0.0, omega=0.0,
                          dt=1e-3, segments=[(30, False)]),
    "periodic_x_real": dict(lat=(40, 8.0, None, True, False, 0.0, False), g=0.0, lhy=0.0,
                            omega=0.0, dt=1e-3, segments=[(20, False)]),
    "rotation_real": dict(lat=(50, 8.0, None, False, False, 0.7, False), g=3.0, lhy=0.0,
                          omega=0.7, dt=1e-3, segments=[(20, False)]),
    "rotation_imag": dict(lat=(50, 8.0, None, False, False, 0.7, False), g=0.0, lhy=0.0,
                          omega=0.7, dt=1e-3, segments=[(20, True)]),
    "ragged_real": dict(lat=(37, 6.0, 29, False, False, 0.0, False), g=2.0, lhy=0.0, omega=0.0,
                        dt=1e-3, segments=[(25, False)]),
    "multi_call_periodic": dict(lat=(32, 6.0, None, True, True, 0.0, False), g=1.0, lhy=0.0,
                                omega=0.0, dt=1e-3, segments=[(7, False), (5, False)]),
    "chain_1d": dict(lat=(96, 12.0, None, False, False, 0.0, True), g=1.0, lhy=0.0, omega=0.0,
                     dt=1e-3, segments=[(40, False)]),
}


def inputs(case, seed):
    N, L, Ny, px, py, omega, one_d = case["lat"]
    lat = O.Lattice(N, L, Ny, None, px, py, omega, one_d=one_d)
    rng = np.random.default_rng(seed)
    X, Y = lat.coordinates()
    psi0 = np.exp(-((X - 0.4) ** 2 + (Y + 0.3) ** 2) / 2.0) * np.exp(1j * 0.5 * X)
    psi0 = psi0 * (1 + 0.02 * rng.uniform(-1, 1, lat.shape))
    psi0 = psi0 / np.sqrt(np.sum(np.abs(psi0) ** 2) * lat.delta_x * lat.delta_y)
    V = 0.5 * (X ** 2 + 1.3 * Y ** 2) + 0.1 * rng.uniform(-1, 1, lat.shape)
    return lat, psi0, V


# Two components (files under two/): lattice (N, L, Ny, periodic_x, periodic_y),
# g_a, g_b, g_ab, mass_b, Rabi omega = (omega_r, omega_i), evolve segments.
CASES2 = {
    "two_real_rabi": dict(lat=(40, 8.0, None, False, False), g=2.0, g_b=1.0, g_ab=1.5,
                          mass_b=1.5, omega=(3.0, 1.0), dt=1e-3, segments=[(15, False), (6, False)]),
    "two_imag_rabi": dict(lat=(40, 8.0, None, False, False), g=2.0, g_b=1.0, g_ab=1.5,
                          mass_b=1.5, omega=(3.0, 1.0), dt=1e-3, segments=[(20, True)]),
    "two_imag_norabi": dict(lat=(36, 8.0, 30, False, False), g=4.0, g_b=2.0, g_ab=3.0,
                            mass_b=1.0, omega=(0.0, 0.0), dt=1e-3, segments=[(20, True)]),
    "two_periodic_real": dict(lat=(36, 8.0, 32, True, True), g=1.0, g_b=2.0, g_ab=0.5,
                              mass_b=0.8, omega=(2.0, 0.0), dt=1e-3, segments=[(10, False)]),
}


def inputs2(case, seed):
    N, L, Ny, px, py = case["lat"]
    lat = O.Lattice(N, L, Ny, None, px, py, 0.0)
    rng = np.random.default_rng(seed)
    X, Y = lat.coordinates()
    dxdy = lat.delta_x * lat.delta_y
    a = np.exp(-((X - 0.4) ** 2 + (Y + 0.3) ** 2) / 2.0) * np.exp(1j * 0.5 * X)
    a = a * (1 + 0.02 * rng.uniform(-1, 1, lat.shape))
    a = a / np.sqrt(np.sum(np.abs(a) ** 2) * dxdy)
    b = np.exp(-((X + 0.5) ** 2 + (Y - 0.2) ** 2) / 1.5) * np.exp(-1j * 0.3 * Y)
    b = b * (1 + 0.02 * rng.uniform(-1, 1, lat.shape))
    b = 0.7 * b / np.sqrt(np.sum(np.abs(b) ** 2) * dxdy)
    Va = 0.5 * (X ** 2 + 1.3 * Y ** 2) + 0.1 * rng.uniform(-1, 1, lat.shape)
    Vb = 0.5 * (1.2 * (X - 0.3) ** 2 + Y ** 2) + 0.1 * rng.uniform(-1, 1, lat.shape)
    return lat, a, b, Va, Vb


def main2():
    os.makedirs(os.path.join(HERE, "two"), exist_ok=True)
    for i, (name, case) in enumerate(sorted(CASES2.items())):
        lat, a, b, Va, Vb = inputs2(case, seed=2000 + i)
        N, L, Ny, px, py = case["lat"]
        cfg = tsref.make_config(N, L, Ny, None, px, py, 0.0, harmonic=None, coupling=case["g"],
                                delta_t=case["dt"], segments=case["segments"], omp_threads=1)
        c2 = tsref.Config2(case["mass_b"], case["g_b"], case["g_ab"], *case["omega"])
        pa, pb, res = tsref.run2(cfg, c2, a, b, Va, Vb)
        meta = dict(case, name=name)
        np.savez_compressed(
            os.path.join(HERE, "two", name + ".npz"), psi0_a=a, psi0_b=b, Va=Va, Vb=Vb,
            psi_a=pa, psi_b=pb,
            energies=np.array([res.total_energy, *res.kinetic, *res.potential, *res.rotational,
                               *res.intra, res.inter_species, res.rabi, *res.squared_norm]),
            meta=json.dumps(meta))
        print(f"{name}: tile {pa.shape}, E = {res.total_energy:.15g}")


# Cylindrical lattices (files under cyl/): the radial axis is x; tiles at most
# 128 columns wide (one cache block of the reference).  lattice (N, L, Ny, Ly,
# periodic_y), angular momentum l, g, evolve segments.
CASES_CYL = {
    "cyl_real_l0": dict(lat=(60, 10.0, 48, 8.0, False), l=0, g=2.0, dt=1e-3,
                        segments=[(25, False)]),
    "cyl_imag_l1": dict(lat=(60, 10.0, 48, 8.0, False), l=1, g=1.0, dt=1e-3,
                        segments=[(30, True)]),
    "cyl_real_l2_two_calls": dict(lat=(50, 8.0, 40, 6.0, False), l=2, g=0.0, dt=1e-3,
                                  segments=[(10, False), (7, False)]),
    "cyl_periodic_y_imag": dict(lat=(40, 8.0, 36, 6.0, True), l=0, g=3.0, dt=1e-3,
                                segments=[(20, True)]),
}


def main_cyl():
    os.makedirs(os.path.join(HERE, "cyl"), exist_ok=True)
    for i, (name, case) in enumerate(sorted(CASES_CYL.items())):
        N, L, Ny, Ly, py = case["lat"]
        lat = O.Lattice(N, L, Ny, Ly, False, py, cylindrical=True)
        rng = np.random.default_rng(3000 + i)
        X, Y = lat.coordinates()
        psi0 = (X ** case["l"]) * np.exp(-(X ** 2 + (Y - 0.3) ** 2) / 2.0) * np.exp(0.2j * Y)
        psi0 = psi0 * (1 + 0.02 * rng.uniform(-1, 1, lat.shape))
        V = 0.5 * (X ** 2 + 1.3 * Y ** 2) + 0.1 * rng.uniform(-1, 1, lat.shape)
        cfg = tsref.make_config(N, L, Ny, Ly, False, py, 0.0, harmonic=None, coupling=case["g"],
                                delta_t=case["dt"], segments=case["segments"], omp_threads=1,
                                cylindrical=True, angular_momentum=case["l"])
        psi, res = tsref.run(cfg, psi0, V)
        meta = dict(case, name=name)
        np.savez_compressed(
            os.path.join(HERE, "cyl", name + ".npz"), psi0=psi0, V=V, psi=psi,
            energies=np.array([res.total_energy, res.kinetic_energy, res.potential_energy,
                               res.rotational_energy, res.intra_energy, res.lhy_energy,
                               res.squared_norm]),
            meta=json.dumps(meta))
        print(f"{name}: tile {psi.shape}, E = {res.total_energy:.15g}")


def main():
    if not tsref.available():
        raise SystemExit("oracle/_ref/libtsref.so is missing: run oracle/build_ref.sh first")
    for i, (name, case) in enumerate(sorted(CASES.items())):
        lat, psi0, V = inputs(case, seed=1000 + i)
        N, L, Ny, px, py, omega, one_d = case["lat"]
        cfg = tsref.make_config(N, L, 0 if one_d else Ny, None, px, py, omega, harmonic=None,
                                coupling=case["g"], lhy_coupling=case["lhy"],
                                angular_velocity=case["omega"], delta_t=case["dt"],
                                segments=case["segments"], omp_threads=1)
        psi, res = tsref.run(cfg, psi0, V)
        meta = dict(case, name=name)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), psi0=psi0, V=V, psi=psi,
            energies=np.array([res.total_energy, res.kinetic_energy, res.potential_energy,
                               res.rotational_energy, res.intra_energy, res.lhy_energy,
                               res.squared_norm]),
            expectations=np.array([res.state_norm, res.mean_x, res.mean_xx, res.mean_y,
                                   res.mean_yy, res.mean_px, res.mean_pxpx, res.mean_py,
                                   res.mean_pypy, res.mean_lz]),
            meta=json.dumps(meta))
        print(f"{name}: tile {psi.shape}, E = {res.total_energy:.15g}")
    main2()
    main_cyl()


if __name__ == "__main__":
    main()
