"""Cylindrical lattices in the oracle, pinned to the reference.

Fixtures under tests/golden/cyl/ are outputs of the reference's own CPU path
on cylindrical Lattice2D tiles (tests/golden/gen_golden.py): the radial
kinetic sweeps (src/cpucylindrical.cpp:4-81), the azimuthal term
l^2 / (2 m r^2) in the potential (src/solver.cpp:85-95, src/model.cpp:967-971),
the mirrored axis column in imaginary time (src/cpukernel.cpp:669-689), and
the cylindrical energy region and norm (src/solver.cpp:301,336,561).
"""
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
CYL = os.path.join(HERE, "golden", "cyl")


def cyl_names():
    return sorted(f[:-4] for f in os.listdir(CYL) if f.endswith(".npz"))


def load_cyl(name):
    z = np.load(os.path.join(CYL, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    N, L, Ny, Ly, py = meta["lat"]
    lat = O.Lattice(N, L, Ny, Ly, False, py, cylindrical=True)
    return lat, meta, {k: z[k] for k in z.files if k != "meta"}


def oracle_cyl(lat, meta, z):
    """The fixture's evolve() calls through the oracle; returns (psi, energies)."""
    psi = z["psi0"]
    Vt = z["V"] + lat.azimuthal(meta["l"])
    n0, prev = 0.0, None
    for it, imag in meta["segments"]:
        if imag and prev is not True:
            n0 = O.expectations(lat, psi)["norm2"]
        p = lat.params(meta["dt"], imag, 1.0, meta["g"], 0.0, 0.0, norm0=n0,
                       angular_momentum=meta["l"])
        tr, ti = O.exp_table(Vt, meta["dt"], imag)
        psi = O.evolve(p, psi, tr, ti, it)
        prev = imag
    e = O.energies(lat, psi, Vt, 1.0, meta["g"])
    return psi, np.array([e[k] for k in ("total", "kinetic", "potential", "rotational", "intra",
                                          "lhy", "norm2")])


@pytest.mark.parametrize("name", cyl_names())
def test_oracle_reproduces_cylindrical_fixture(name):
    lat, meta, z = load_cyl(name)
    psi, e = oracle_cyl(lat, meta, z)
    assert np.abs(psi - z["psi"]).max() <= 1e-13
    assert np.allclose(e, z["energies"], rtol=1e-12, atol=1e-14), (e, z["energies"])


def test_cylindrical_geometry():
    """One more column (r = -dx/2), dx = L / (N + 0.5), inner region from column 1."""
    lat = O.Lattice(60, 10.0, 48, 8.0, cylindrical=True)
    assert lat.shape == (48, 61)
    assert lat.delta_x == 10.0 / 60.5
    assert lat.inner()[0] == 1
    X, _ = lat.coordinates()
    assert X[0, 0] == -0.5 * lat.delta_x and X[0, 1] == 0.5 * lat.delta_x


def test_host_cylindrical_lattice_matches_oracle_geometry():
    """The drop-in Lattice2D / Lattice1D with coordinate_system="cylindrical"
    (no GPU needed) against the oracle's restatement of src/model.cpp:32-158."""
    import trottersuzuki_b200 as ts
    for args in ((60, 10.0, 48, 8.0, False), (40, 8.0, 36, 6.0, True)):
        N, L, Ny, Ly, py = args
        g = ts.Lattice2D(N, L, Ny, Ly, periodic_y_axis=py, coordinate_system="cylindrical")
        lat = O.Lattice(N, L, Ny, Ly, False, py, cylindrical=True)
        assert (g.dim_y, g.dim_x) == lat.shape
        assert g.delta_x == lat.delta_x and g.delta_y == lat.delta_y
        assert g.inner_start_x - g.start_x == lat.inner()[0]
        X, Y = lat.coordinates()
        assert ts.map_lattice_to_coordinate_space(g, 0, 3) == (X[3, 0], Y[3, 0])
    g1 = ts.Lattice1D(50, 6.0, coordinate_system="cylindrical")
    assert g1.dim_x == 51 and g1.delta_x == 6.0 / 50.5
