"""Parity of the B200 step kernel (through the C ABI) against the oracle.

The oracle (oracle/ts_oracle.c) is pinned bit-exactly to the compiled
reference CPUBlock in tests/test_oracle_pin.py.  Bar: max |psi_gpu - psi_ref|
<= 1e-10 over the whole tile after the stated number of steps (FP64), with
FMA contraction on the GPU and none in the oracle as the only difference.
"""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, energy_params, seeded_case

pytestmark = pytest.mark.gpu

TOL_PSI = 1e-10

# (N, L, Ny, periodic, omega, g, lhy, imag, dt, steps)
CASES = [
    ("closed", 64, 10.0, None, (False, False), 0.0, 0.0, 0.0, False, 1e-3, 20),
    ("gpe_lhy", 64, 10.0, None, (False, False), 0.0, 5.0, 0.3, False, 1e-3, 20),
    ("imag_gpe", 64, 10.0, None, (False, False), 0.0, 5.0, 0.0, True, 1e-3, 20),
    ("ragged", 61, 10.0, 47, (False, False), 0.0, 0.0, 0.0, False, 1e-3, 20),
    ("periodic", 64, 10.0, None, (True, True), 0.0, 0.0, 0.0, False, 1e-3, 20),
    ("periodic_x", 64, 10.0, None, (True, False), 0.0, 0.0, 0.0, False, 1e-3, 20),
    ("periodic_y", 64, 10.0, None, (False, True), 0.0, 0.0, 0.0, False, 1e-3, 20),
    ("rotation", 64, 10.0, None, (False, False), 0.7, 3.0, 0.0, False, 1e-3, 20),
    ("rotation_imag", 64, 10.0, None, (False, False), 0.7, 0.0, 0.0, True, 1e-3, 20),
    ("wide", 200, 10.0, None, (False, False), 0.0, 2.0, 0.0, False, 1e-3, 10),
    ("rotation_300", 300, 20.0, None, (False, False), 0.7, 2.0, 0.0, False, 1e-3, 5),
    ("periodic_rotation", 64, 10.0, None, (True, True), 0.5, 0.0, 0.0, False, 1e-3, 10),
    ("periodic_odd", 63, 10.0, 45, (True, True), 0.0, 1.0, 0.0, False, 1e-3, 12),
    ("tall", 40, 10.0, 700, (False, False), 0.0, 1.0, 0.0, False, 1e-3, 8),
    ("wide_imag_periodic", 530, 20.0, 96, (True, True), 0.0, 4.0, 0.2, True, 1e-3, 6),
    ("tiny", 3, 1.0, 2, (False, False), 0.0, 1.0, 0.0, False, 1e-3, 5),
]


def run_oracle(lat, psi0, V, dt, imag, g, lhy, omega, steps):
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(dt, imag, 1.0, g, lhy, omega, norm0=n0)
    tr, ti = O.exp_table(V, dt, imag)
    return p, tr, ti, O.evolve(p, psi0, tr, ti, steps)


def run_gpu(p, psi0, tr, ti, steps, precision=0, launch=None, split=None):
    from trottersuzuki_b200 import Kernel
    with Kernel(desc_from_params(p, precision)) as k:
        if launch:
            k.set_launch(**launch)
        k.set_state(psi0)
        k.set_exp_potential(tr, ti)
        if split:
            for s in split:
                k.evolve(s)
        else:
            k.evolve(steps)
        return k.get_state()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_fp64_matches_oracle(case):
    _, N, L, Ny, per, omega, g, lhy, imag, dt, steps = case
    lat, psi0, V = seeded_case(N, L, Ny, per, omega)
    p, tr, ti, ref = run_oracle(lat, psi0, V, dt, imag, g, lhy, omega, steps)
    got = run_gpu(p, psi0, tr, ti, steps)
    err = np.abs(got - ref).max()
    assert err <= TOL_PSI, f"max|dpsi| = {err:.3e}"


@pytest.mark.parametrize("launch", [
    dict(cells_per_lane=2, segment_rows=16),
    dict(cells_per_lane=4, segment_rows=40),
    dict(cells_per_lane=2, segment_rows=7, warps_per_block=1, ring_depth=4),
    dict(cells_per_lane=4, segment_rows=256, warps_per_block=2, ring_depth=12),
])
def test_launch_shape_does_not_change_result(launch):
    """Every cell gets the same operations whatever the strip/segment cut: bitwise equal."""
    lat, psi0, V = seeded_case(333, 12.0, 290, (False, False))
    p, tr, ti, _ = run_oracle(lat, psi0, V, 1e-3, False, 3.0, 0.0, 0.0, 0)
    base = run_gpu(p, psi0, tr, ti, 9)
    other = run_gpu(p, psi0, tr, ti, 9, launch=launch)
    assert np.array_equal(base, other)


def test_multi_call_evolve_matches_oracle():
    """Consecutive evolve() calls keep the halo of the last step (reference semantics)."""
    lat, psi0, V = seeded_case(64, 10.0, None, (True, True))
    p = lat.params(1e-3, False, 1.0, 1.0, 0.0, 0.0)
    tr, ti = O.exp_table(V, 1e-3, False)
    ref = O.evolve(p, O.evolve(p, psi0, tr, ti, 7), tr, ti, 5)
    got = run_gpu(p, psi0, tr, ti, 12, split=(7, 5))
    assert np.abs(got - ref).max() <= TOL_PSI


def test_graph_replay_long_run_matches_oracle():
    """100 steps: exercises the CUDA-graph replay path (32-step graphs)."""
    lat, psi0, V = seeded_case(96, 10.0, 80, (True, False))
    p, tr, ti, ref = run_oracle(lat, psi0, V, 1e-3, False, 2.0, 0.0, 0.0, 100)
    got = run_gpu(p, psi0, tr, ti, 100)
    assert np.abs(got - ref).max() <= TOL_PSI


def test_config1_plain_method():
    """256^2, L=20, closed, HO omega=1, Gaussian at (1,0), dt=1e-4, 1000 real-time steps."""
    from trottersuzuki_b200 import Kernel
    lat = O.Lattice(256, 20.0)
    psi0 = O.gaussian(lat, 1.0, 1.0, 1.0, 0.0)
    V = lat.harmonic(1.0, 1.0)
    p = lat.params(1e-4, False)
    tr, ti = O.exp_table(V, 1e-4, False)
    ref = O.evolve(p, psi0, tr, ti, 1000)
    e_ref = O.energies(lat, ref, V)
    with Kernel(desc_from_params(p)) as k:
        k.set_state(psi0)
        k.set_exp_potential(tr, ti)
        k.evolve(1000)
        got = k.get_state()
        e = k.energies(V, energy_params(lat))
        n = k.squared_norm()
    assert np.abs(got - ref).max() <= TOL_PSI
    for key in ("total", "kinetic", "potential", "norm2"):
        assert abs(e[key] - e_ref[key]) <= 1e-10 * max(1.0, abs(e_ref[key])), key
    assert abs(n - O.squared_norm(p, ref)) <= 1e-12


@pytest.mark.parametrize("case", ["closed", "rotation", "periodic_odd", "wide_imag_periodic"])
def test_energies_and_expectations_match_oracle(case):
    from trottersuzuki_b200 import Kernel
    c = [c for c in CASES if c[0] == case][0]
    _, N, L, Ny, per, omega, g, lhy, imag, dt, steps = c
    lat, psi0, V = seeded_case(N, L, Ny, per, omega)
    p, tr, ti, ref = run_oracle(lat, psi0, V, dt, imag, g, lhy, omega, steps)
    with Kernel(desc_from_params(p)) as k:
        k.set_state(psi0)
        k.set_exp_potential(tr, ti)
        k.evolve(steps)
        e = k.energies(V, energy_params(lat, 1.0, g, lhy, omega))
        x = k.expectations(energy_params(lat))
    e_ref = O.energies(lat, ref, V, 1.0, g, lhy, omega)
    x_ref = O.expectations(lat, ref)
    for key, v in e_ref.items():
        assert abs(e[key] - v) <= 1e-9 * max(1.0, abs(v)), (key, e[key], v)
    for key, v in x_ref.items():
        assert abs(x[key] - v) <= 1e-9 * max(1.0, abs(v)), (key, x[key], v)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_autotune_keeps_state_and_results(imag):
    """ts_b200_autotune times shapes on the current state without changing it;
    afterwards the evolution equals the untuned one (bitwise in real time; in
    imaginary time the norm is summed over a different grid: 1e-13)."""
    from trottersuzuki_b200 import Kernel
    lat, psi0, V = seeded_case(300, 12.0, 260, (False, False))
    p, tr, ti, _ = run_oracle(lat, psi0, V, 1e-3, imag, 3.0, 0.0, 0.0, 0)
    res = []
    for tune in (False, True):
        with Kernel(desc_from_params(p)) as k:
            k.set_state(psi0)
            k.set_exp_potential(tr, ti)
            k.evolve(3)
            if tune:
                before = k.get_state()
                shape = k.autotune(2)
                assert shape["blocks"] >= 1
                assert np.array_equal(k.get_state(), before)
            k.evolve(17)
            res.append(k.get_state())
    if imag:
        assert np.abs(res[0] - res[1]).max() <= 1e-13 * np.abs(res[0]).max()
    else:
        assert np.array_equal(res[0], res[1])
