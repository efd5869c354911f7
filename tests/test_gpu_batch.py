"""Batched evolution (ts_b200_batch_*): many tiles of uneven sizes, one launch per step.

A batched step runs exactly the per-tile arithmetic of the single-tile kernel,
so in real time the batch must reproduce per-tile evolve() calls bit for bit,
whatever the batch's tile shape.  In imaginary time the per-tile norm is
summed in a different order (per task, then per tile), so the renormalised
states agree to rounding (1e-12 relative) instead.
"""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, seeded_case

pytestmark = pytest.mark.gpu

# (name, N, L, Ny, periodic, g, lhy)
TILES = [
    ("closed", 64, 10.0, None, (False, False), 2.0, 0.0),
    ("ragged", 61, 10.0, 47, (False, False), 0.0, 0.0),
    ("periodic", 64, 10.0, None, (True, True), 1.0, 0.0),
    ("periodic_x", 50, 8.0, 40, (True, False), 3.0, 0.0),
    ("wide", 200, 12.0, 30, (False, False), 5.0, 0.3),
    ("tall", 40, 10.0, 300, (False, False), 1.0, 0.0),
    ("tiny", 3, 1.0, 2, (False, False), 0.0, 0.0),
]


def make_tiles(imag=False, precision=0, dt=1e-3, seed0=10, tiles=TILES):
    from trottersuzuki_b200 import Kernel
    out = []
    for j, (name, N, L, Ny, per, g, lhy) in enumerate(tiles):
        lat, psi0, V = seeded_case(N, L, Ny, per, 0.0, seed=seed0 + j)
        n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
        p = lat.params(dt, imag, 1.0, g, lhy, 0.0, norm0=n0)
        tr, ti = O.exp_table(V, dt, imag)
        k = Kernel(desc_from_params(p, precision))
        k.set_state(psi0)
        k.set_exp_potential(tr, ti)
        out.append(dict(name=name, k=k, p=p, psi0=psi0, tr=tr, ti=ti))
    return out


def individual(tiles, splits, precision=0):
    """The same tiles evolved one by one (fresh handles, same inputs)."""
    from trottersuzuki_b200 import Kernel
    res = []
    for t in tiles:
        with Kernel(desc_from_params(t["p"], precision)) as k:
            k.set_state(t["psi0"])
            k.set_exp_potential(t["tr"], t["ti"])
            for n in splits:
                k.evolve(n)
            res.append(k.get_state())
    return res


def close_all(tiles):
    for t in tiles:
        t["k"].close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_real_time_batch_is_bitwise_per_tile(precision):
    from trottersuzuki_b200 import Batch
    tiles = make_tiles(False, precision)
    splits = [37, 6]  # graph run + direct steps, odd count (buffer parity flips)
    with Batch([t["k"] for t in tiles]) as b:
        for n in splits:
            b.evolve(n)
        b.synchronize()
        got = [t["k"].get_state() for t in tiles]
    ref = individual(tiles, splits, precision)
    for t, g, r in zip(tiles, got, ref):
        assert np.array_equal(g, r), f"{t['name']}: max|d| = {np.abs(g - r).max():.3e}"
    close_all(tiles)


def test_real_time_batch_matches_oracle():
    from trottersuzuki_b200 import Batch
    tiles = make_tiles(False, 0)
    steps = 20
    with Batch([t["k"] for t in tiles]) as b:
        b.evolve(steps)
        for t in tiles:
            ref = O.evolve(t["p"], t["psi0"], t["tr"], t["ti"], steps)
            err = np.abs(t["k"].get_state() - ref).max()
            assert err <= 1e-10, f"{t['name']}: {err:.3e}"
    close_all(tiles)


def test_imaginary_time_batch():
    from trottersuzuki_b200 import Batch
    tiles = make_tiles(True, 0)
    splits = [35, 4]
    with Batch([t["k"] for t in tiles]) as b:
        for n in splits:
            b.evolve(n)
        got = [t["k"].get_state() for t in tiles]
        norms = [t["k"].squared_norm() for t in tiles]
    ref = individual(tiles, splits, 0)
    for t, g, r, n in zip(tiles, got, ref, norms):
        scale = np.abs(r).max()
        assert np.abs(g - r).max() <= 1e-12 * scale, t["name"]
        oracle = t["psi0"]
        for n_steps in splits:  # the last step of each evolve() skips the halo refresh
            oracle = O.evolve(t["p"], oracle, t["tr"], t["ti"], n_steps)
        assert np.abs(g - oracle).max() <= 1e-10, t["name"]
        assert abs(n - t["p"].norm0) <= 1e-9 * t["p"].norm0, t["name"]
    close_all(tiles)


def test_autotune_keeps_state_and_results():
    from trottersuzuki_b200 import Batch
    tiles = make_tiles(False, 0)
    before = [t["k"].get_state() for t in tiles]
    with Batch([t["k"] for t in tiles]) as b:
        shape = b.autotune(trial_steps=2, use_cache=False)
        assert shape["segment_rows"] in (16, 32, 64, 96, 128, 192, 256)
        assert shape["warps_per_block"] in (2, 4)
        after = [t["k"].get_state() for t in tiles]
        for x, y in zip(before, after):
            assert np.array_equal(x, y)
        assert b.autotune(trial_steps=2, use_cache=True) == shape
        b.evolve(9)
        got = [t["k"].get_state() for t in tiles]
    ref = individual(tiles, [9], 0)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
    close_all(tiles)


@pytest.mark.parametrize("seg,warps", [(2, 1), (10, 2), (128, 4)])
def test_batch_shape_does_not_change_result(seg, warps):
    from trottersuzuki_b200 import Batch
    tiles = make_tiles(False, 0)
    with Batch([t["k"] for t in tiles]) as b:
        b.set_launch(segment_rows=seg, warps_per_block=warps)
        info = b.launch_shape()
        assert info["segment_rows"] == seg + (seg & 1)
        b.evolve(11)
        got = [t["k"].get_state() for t in tiles]
    ref = individual(tiles, [11], 0)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
    close_all(tiles)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
def test_batch_walks_agree(precision, imag):
    """The batch runs its tiles' row walk: the look-ahead walk by default, the
    checked walk when the tiles are set to it; both give the same bits in real
    time and agree to rounding in imaginary time."""
    from trottersuzuki_b200 import Batch
    got = {}
    for walk in (2, 0):
        tiles = make_tiles(imag, precision)
        for t in tiles:
            t["k"].set_walk(walk)
        with Batch([t["k"] for t in tiles]) as b:
            b.set_launch(segment_rows=24, warps_per_block=2)
            assert b.launch_shape()["walk"] == walk
            for n in (33, 5):
                b.evolve(n)
            b.synchronize()
            got[walk] = [t["k"].get_state() for t in tiles]
        close_all(tiles)
    for t, x, y in zip(make_tiles(imag, precision), got[2], got[0]):
        if imag:
            tol = 1e-12 if precision == 0 else 1e-6
            assert np.abs(x - y).max() <= tol * np.abs(y).max(), t["name"]
        else:
            assert np.array_equal(x, y), f"{t['name']}: max|d| = {np.abs(x - y).max():.3e}"
        t["k"].close()


def test_batch_rejects_mixed_or_unsupported_tiles():
    from trottersuzuki_b200 import B200Error, Batch, Kernel
    t64 = make_tiles(False, 0, tiles=TILES[:1])
    t32 = make_tiles(False, 1, tiles=TILES[:1])
    with pytest.raises(B200Error):
        Batch([t64[0]["k"], t32[0]["k"]])
    with pytest.raises(B200Error):
        Batch([t64[0]["k"], t64[0]["k"]])
    lat, psi0, V = seeded_case(64, 10.0, None, (False, False), 0.7)
    p = lat.params(1e-3, False, 1.0, 0.0, 0.0, 0.7)
    with Kernel(desc_from_params(p)) as kr:
        with pytest.raises(B200Error):
            Batch([kr])
    close_all(t64)
    close_all(t32)


def _solver(ts, N, L, omega, g, centre, width, kernel_type="gpu"):
    grid = ts.Lattice2D(N, L)
    state = ts.GaussianState(grid, 1.0 / width ** 2, 1.0 / width ** 2, centre[0], centre[1])
    pot = ts.HarmonicPotential(grid, omega, omega)
    ham = ts.Hamiltonian(grid, pot, 1.0, g)
    return ts.Solver(grid, state, ham, 1e-4, kernel_type=kernel_type), state


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_solver_batch_matches_solver_loop(imag):
    """The drop-in level: SolverBatch(solvers).evolve(T) == for s: s.evolve(T)."""
    import trottersuzuki_b200 as ts
    cfg = [(128, 20.0, 1.0, 50.0, (0.5, -1.0), 1.0), (192, 20.0, 1.7, 0.0, (-1.5, 0.3), 0.7),
           (96, 20.0, 0.6, 150.0, (0.0, 1.2), 1.8)]
    batch = [_solver(ts, *c) for c in cfg]
    loop = [_solver(ts, *c) for c in cfg]
    sb = ts.SolverBatch([s for s, _ in batch], imag_time=imag)
    sb.autotune(trial_steps=1)
    sb.evolve(70)
    for (s1, st1), (s2, st2) in zip(batch, loop):
        s2.evolve(70, imag)
        a = np.asarray(st1.get_particle_density())
        b = np.asarray(st2.get_particle_density())
        if imag:
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
            assert abs(s1.get_total_energy() - s2.get_total_energy()) <= 1e-11 * abs(s2.get_total_energy())
        else:
            assert np.array_equal(a, b)
            assert s1.get_total_energy() == s2.get_total_energy()
    sb.close()
