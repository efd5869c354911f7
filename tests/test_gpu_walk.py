"""The look-ahead row walk of the fused step against the oracle and against
the checked walk.

Both walks perform the same operations per cell (the same pair forms,
potential row and fused multiply-adds), so in real time they agree bit for
bit, whatever the launch shape; in imaginary time the squared norm is summed
over a different grid of blocks, so the renormalisation factor may differ in
its last bits (1e-13).  The oracle bar is the FP64 parity bar, 1e-10.
"""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, seeded_case

pytestmark = pytest.mark.gpu

TOL_PSI = 1e-10


def _oracle(lat, psi0, V, dt, imag, g, lhy, steps):
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(dt, imag, 1.0, g, lhy, 0.0, norm0=n0)
    tr, ti = O.exp_table(V, dt, imag)
    return p, tr, ti, O.evolve(p, psi0, tr, ti, steps)


def _gpu(p, psi0, tr, ti, steps, walk, launch=None, precision=0, split=None):
    from trottersuzuki_b200 import Kernel
    with Kernel(desc_from_params(p, precision)) as k:
        k.set_walk(walk)
        if launch:
            k.set_launch(**launch)
        shape = k.launch_shape()
        k.set_state(psi0)
        k.set_exp_potential(tr, ti)
        for s in (split or [steps]):
            k.evolve(s)
        return k.get_state(), shape


# name, N, L, Ny, periodic, g, lhy, imag, steps
CASES = [
    ("closed_real", 64, 10.0, None, (False, False), 0.0, 0.0, False, 20),
    ("gpe_lhy_real", 64, 10.0, None, (False, False), 5.0, 0.3, False, 20),
    ("gpe_imag", 64, 10.0, None, (False, False), 5.0, 0.0, True, 20),
    ("ragged", 61, 10.0, 47, (False, False), 1.0, 0.0, False, 20),
    ("periodic", 64, 10.0, None, (True, True), 2.0, 0.0, False, 20),
    ("periodic_x_imag", 64, 10.0, None, (True, False), 2.0, 0.0, True, 12),
    ("periodic_odd", 63, 10.0, 45, (True, True), 1.0, 0.0, False, 12),
    ("tall", 40, 10.0, 700, (False, False), 1.0, 0.0, False, 8),
    ("wide_imag_periodic", 530, 20.0, 96, (True, True), 4.0, 0.2, True, 6),
    ("tiny", 3, 1.0, 2, (False, False), 1.0, 0.0, False, 5),
    ("one_row", 50, 5.0, 1, (False, False), 1.0, 0.0, False, 5),
    ("short_rows", 200, 10.0, 9, (False, False), 1.0, 0.0, True, 7),
]


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_look_ahead_walk_matches_oracle_and_checked_walk(case, walk):
    _, N, L, Ny, per, g, lhy, imag, steps = case
    lat, psi0, V = seeded_case(N, L, Ny, per)
    p, tr, ti, ref = _oracle(lat, psi0, V, 1e-3, imag, g, lhy, steps)
    got, shape = _gpu(p, psi0, tr, ti, steps, walk=walk)
    assert shape["walk"] == walk
    assert np.abs(got - ref).max() <= TOL_PSI
    old, shape0 = _gpu(p, psi0, tr, ti, steps, walk=0)
    assert shape0["walk"] == 0
    if imag:
        assert np.abs(got - old).max() <= 1e-13 * np.abs(old).max()
    else:
        assert np.array_equal(got, old)


@pytest.mark.parametrize("launch", [
    dict(cells_per_lane=2, segment_rows=16),
    dict(cells_per_lane=4, segment_rows=40),
    dict(cells_per_lane=2, segment_rows=7, warps_per_block=1),
    dict(cells_per_lane=4, segment_rows=256, warps_per_block=8),
    dict(cells_per_lane=2, segment_rows=2, warps_per_block=8),
    dict(cells_per_lane=2, segment_rows=300, warps_per_block=2),
])
@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("walk", [1, 2])
def test_look_ahead_walk_launch_shapes(launch, imag, walk):
    """Any strip/segment cut of the look-ahead walk gives the checked walk's
    bits (real time) and the oracle's result at the parity bar."""
    lat, psi0, V = seeded_case(333, 12.0, 290, (False, False))
    p, tr, ti, ref = _oracle(lat, psi0, V, 1e-3, imag, 3.0, 0.0, 9)
    got, shape = _gpu(p, psi0, tr, ti, 9, walk=walk, launch=launch, split=[4, 5])
    rows = walk if launch["cells_per_lane"] == 2 else 1
    assert shape["walk"] == rows and shape["segment_rows"] % 2 == 0
    assert np.abs(got - ref).max() <= TOL_PSI
    if not imag:
        old, _ = _gpu(p, psi0, tr, ti, 9, walk=0, split=[4, 5])
        assert np.array_equal(got, old)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("seg", [10, 12, 14])
def test_many_segments_odd_height(imag, walk, seg):
    """Many segments on 301 rows with a short last segment (segment rows 10:
    31 segments, the last of 1 row; 12: 26 segments, the last of 1 row; 14:
    22 segments, the last of 7 rows), ragged columns (233 = 4 x 56 + 9): the
    checked walk's bits in real time, the oracle's result always."""
    lat, psi0, V = seeded_case(233, 12.0, 301, (False, False))
    p, tr, ti, ref = _oracle(lat, psi0, V, 1e-3, imag, 3.0, 0.2, 7)
    got, shape = _gpu(p, psi0, tr, ti, 7, walk=walk,
                      launch=dict(cells_per_lane=2, segment_rows=seg), split=[3, 4])
    assert shape["segments"] == -(-301 // seg)
    assert np.abs(got - ref).max() <= TOL_PSI
    if not imag:
        old, _ = _gpu(p, psi0, tr, ti, 7, walk=0, split=[3, 4])
        assert np.array_equal(got, old)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("cells,walk", [(2, 1), (2, 2), (4, 1)])
def test_look_ahead_walk_fp32(imag, cells, walk):
    """FP32 storage through the look-ahead walk: the checked walk's bits in
    real time (the same float arithmetic per cell), the FP32 bar against the
    FP64 oracle."""
    from trottersuzuki_b200 import _capi
    lat, psi0, V = seeded_case(257, 12.0, 203, (False, False))
    p, tr, ti, ref = _oracle(lat, psi0, V, 1e-3, imag, 3.0, 0.0, 15)
    launch = dict(cells_per_lane=cells, segment_rows=24)
    got, shape = _gpu(p, psi0, tr, ti, 15, walk=walk, launch=launch, precision=_capi.FP32)
    assert shape["walk"] == walk
    assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max()
    old, _ = _gpu(p, psi0, tr, ti, 15, walk=0, launch=launch, precision=_capi.FP32)
    if imag:
        assert np.abs(got - old).max() <= 1e-6 * np.abs(old).max()
    else:
        assert np.array_equal(got, old)


# rotating frame: name, N, Ny, periodic, g, lhy, omega, imag, steps
ROT_CASES = [
    ("rot_real", 64, None, (False, False), 1.0, 0.0, 0.7, False, 20),
    ("rot_imag", 64, None, (False, False), 5.0, 0.0, 0.7, True, 20),
    ("rot_lhy_real", 72, 60, (False, False), 3.0, 0.2, 0.4, False, 15),
    ("rot_periodic", 64, None, (True, True), 2.0, 0.0, 0.5, False, 12),
    ("rot_periodic_imag", 80, 64, (True, True), 2.0, 0.0, 0.5, True, 12),
    ("rot_ragged", 61, 47, (False, False), 1.0, 0.0, 0.9, False, 14),
    ("rot_short", 50, 9, (False, False), 1.0, 0.0, 0.6, True, 7),
]


def _rot_oracle(case, split):
    """The oracle over the same evolve() calls (a periodic tile skips its halo
    refresh after the last step of each call)."""
    _, N, Ny, per, g, lhy, omega, imag, steps = case
    lat, psi0, V = seeded_case(N, 10.0, Ny, per, omega=omega)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(1e-3, imag, 1.0, g, lhy, omega, norm0=n0)
    tr, ti = O.exp_table(V, 1e-3, imag)
    ref = psi0
    for n in split:
        ref = O.evolve(p, ref, tr, ti, n)
    return lat, psi0, p, tr, ti, ref


@pytest.mark.parametrize("walk", [1, 2])
@pytest.mark.parametrize("case", ROT_CASES, ids=[c[0] for c in ROT_CASES])
def test_rotating_frame_look_ahead_walk(case, walk):
    """The rotating frame's look-ahead walk (8-row window, row and column
    rotation sweeps, their identity across the tile edges) against the oracle
    and the checked walk."""
    steps = case[-1]
    imag = case[7]
    split = [steps // 2, steps - steps // 2]
    lat, psi0, p, tr, ti, ref = _rot_oracle(case, split)
    got, shape = _gpu(p, psi0, tr, ti, steps, walk=walk, split=split)
    assert shape["walk"] == walk and shape["ring_depth"] == 8
    assert np.abs(got - ref).max() <= TOL_PSI * max(1.0, np.abs(ref).max())
    old, shape0 = _gpu(p, psi0, tr, ti, steps, walk=0, split=split)
    assert shape0["walk"] == 0
    if imag:
        assert np.abs(got - old).max() <= 1e-13 * np.abs(old).max()
    else:
        assert np.array_equal(got, old)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
@pytest.mark.parametrize("seg", [8, 14, 40])
def test_rotating_frame_segments_and_fp32(imag, seg):
    """Segment cuts of the rotating-frame walk (301 rows, ragged columns) in
    both precisions: the checked walk's bits in real time."""
    from trottersuzuki_b200 import _capi
    lat, psi0, V = seeded_case(233, 12.0, 301, (False, False), omega=0.5)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(1e-3, imag, 1.0, 3.0, 0.0, 0.5, norm0=n0)
    tr, ti = O.exp_table(V, 1e-3, imag)
    ref = O.evolve(p, psi0, tr, ti, 7)
    for prec, cells, tol in ((_capi.FP64, 2, TOL_PSI), (_capi.FP32, 2, 2e-5), (_capi.FP32, 4, 2e-5)):
        launch = dict(cells_per_lane=cells, segment_rows=seg)
        got, shape = _gpu(p, psi0, tr, ti, 7, walk=2, launch=launch, precision=prec, split=[3, 4])
        assert shape["walk"] == 2 and shape["cells_per_lane"] == cells
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max()
        # the checked walk (2 cells per lane in a rotating frame)
        old, _ = _gpu(p, psi0, tr, ti, 7, walk=0, launch=dict(cells_per_lane=2, segment_rows=seg),
                      precision=prec, split=[3, 4])
        if imag:
            assert np.abs(got - old).max() <= (1e-13 if prec == _capi.FP64 else 1e-6) * np.abs(old).max()
        else:
            assert np.array_equal(got, old)
