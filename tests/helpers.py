"""Shared test helpers: seeded inputs and oracle <-> C-ABI descriptor glue."""
import numpy as np

import oracle as O
from trottersuzuki_b200 import _capi


def desc_from_params(p, precision=_capi.FP64):
    """C-ABI descriptor carrying exactly the oracle's step constants."""
    d = _capi.Desc()
    d.dim_x, d.dim_y = p.W, p.H
    d.inner_x0, d.inner_x1, d.inner_y0, d.inner_y1 = p.ix0, p.ix1, p.iy0, p.iy1
    d.halo_x, d.halo_y = p.halo_x, p.halo_y
    d.periodic_x, d.periodic_y = p.periodic_x, p.periodic_y
    d.imag_time = p.imag_time
    d.precision = precision
    d.a_h, d.b_h, d.a_v, d.b_v = p.aH, p.bH, p.aV, p.bV
    d.coupling, d.lhy_coupling = p.coupling, p.lhy_coupling
    d.alpha_x, d.alpha_y = p.alpha_x, p.alpha_y
    d.rot_offset_x, d.rot_offset_y = float(p.rot_off_x), float(p.rot_off_y)
    d.delta_x, d.delta_y = p.delta_x, p.delta_y
    d.norm0 = p.norm0
    d.cylindrical = p.cylindrical
    d.kin_radial = p.kin_radial
    d.angular_momentum = 0 if p.mirror_sign >= 0 else 1  # only its parity enters
    return d


def energy_params(lat, mass=1.0, coupling=0.0, lhy=0.0, omega=0.0):
    e = _capi.EnergyParams()
    e.mass, e.coupling, e.lhy_coupling, e.angular_velocity = mass, coupling, lhy, omega
    e.start_x, e.start_y = lat.start_x, lat.start_y
    e.global_no_halo_dim_x = lat.global_no_halo_dim_x
    e.global_no_halo_dim_y = lat.global_no_halo_dim_y
    e.length_x, e.length_y = lat.length_x, lat.length_y
    return e


def seeded_case(N, L, Ny=None, periodic=(False, False), omega=0.0, seed=0, momentum=0.3):
    """Lattice, initial state and potential used by the parity tests."""
    lat = O.Lattice(N, L, Ny, None, periodic[0], periodic[1], omega)
    rng = np.random.default_rng(seed)
    X, _ = lat.coordinates()
    psi0 = (O.gaussian(lat, 1.0, 1.0, 0.5, -0.3) * (1 + 0.01 * rng.uniform(-1, 1, lat.shape))
            * np.exp(1j * momentum * X))
    V = lat.harmonic(1.0, 1.3) + 0.1 * rng.uniform(-1, 1, lat.shape)
    return lat, psi0, V


# ---------------------------------------------------------------- fixtures
import json  # noqa: E402
import os  # noqa: E402

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    N, L, Ny, px, py, omega, one_d = meta["lat"]
    lat = O.Lattice(N, L, Ny, None, px, py, omega, one_d=one_d)
    return dict(lat=lat, psi0=z["psi0"], V=z["V"], psi=z["psi"], energies=z["energies"],
                expectations=z["expectations"], meta=meta)


def oracle_run_golden(g):
    """Evolve a golden case with the oracle, segment by segment like Solver::evolve."""
    meta, lat = g["meta"], g["lat"]
    psi = g["psi0"].copy()
    prev_imag = None
    n0 = 0.0
    for it, imag in meta["segments"]:
        if imag and prev_imag is not True:
            n0 = O.expectations(lat, psi)["norm2"]
        p = lat.params(meta["dt"], imag, 1.0, meta["g"], meta["lhy"], meta["omega"], norm0=n0)
        tr, ti = O.exp_table(g["V"], meta["dt"], imag)
        psi = O.evolve(p, psi, tr, ti, it)
        prev_imag = imag
    return psi
