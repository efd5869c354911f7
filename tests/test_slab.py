"""One lattice split into slabs of rows across ranks (trottersuzuki_b200.slab):
the reference's MPI tiles (src/common.cpp:83-102) and halo exchange
(src/cpukernel.cpp:717-747), here over torch.distributed with gloo on the CPU
and the oracle as each rank's tile.  The slabs' inner rows must reproduce the
whole lattice evolved as one tile: bit for bit in real time, to rounding in
imaginary time (the norm is summed in another order)."""
import json
import os
import socket

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (N, Ny, periodic_y, imag, g, calls)
CASES = [(32, 40, False, False, 2.0, (5, 4)), (32, 36, True, False, 1.0, (6, 3)),
         (28, 44, False, True, 3.0, (7, 2)), (30, 33, True, True, 0.0, (4, 5))]


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def whole_lattice(case):
    import oracle as O
    N, Ny, py, imag, g, calls = case
    lat = O.Lattice(N, 8.0, Ny, 8.0, False, py)
    X, Y = lat.coordinates()
    rng = np.random.default_rng(N + Ny)
    psi0 = np.exp(-((X - 0.5) ** 2 + (Y + 0.4) ** 2) / 2.0) * np.exp(0.4j * X)
    psi0 = psi0 * (1 + 0.02 * rng.uniform(-1, 1, lat.shape))
    V = 0.5 * (X ** 2 + 1.3 * Y ** 2)
    return lat, psi0, V


class OracleTile:
    """A slab's tile stepped by the oracle (closed in y), for the CPU test."""

    def __init__(self, lat, layout, psi_global, V_global, case):
        import oracle as O
        import torch
        self.O, self.torch = O, torch
        N, Ny, py, imag, g, calls = case
        # tile rows of the global tile (global tile row = global row + halo if periodic)
        off = lat.halo_y if py else 0
        rows = slice(layout.start + off, layout.end + off)
        self.psi = np.array(psi_global[rows], dtype=np.complex128, order="C")
        self.tr, self.ti = O.exp_table(V_global[rows], 1e-3, imag)
        p = lat.params(1e-3, imag, 1.0, g, 0.0, 0.0)
        p.H = layout.rows
        p.iy0, p.iy1 = layout.inner_rows()
        p.periodic_y = 0
        self.p = p
        self.imag = imag
        self.norm0 = None

    def step(self):
        re = np.ascontiguousarray(self.psi.real)
        im = np.ascontiguousarray(self.psi.imag)
        self.O.lib().tso_full_step(self.O.C.byref(self.p), re.ctypes.data, im.ctypes.data,
                                   self.tr.ctypes.data, self.ti.ctypes.data)
        self.psi[...] = re + 1j * im

    def rows(self, row0, nrows):
        return self.torch.from_numpy(self.psi.view(np.float64)[row0:row0 + nrows]).reshape(-1)

    def last_norm(self):
        n = self.O.squared_norm(self.p, self.psi)
        self._t = self.torch.tensor([n], dtype=self.torch.float64)
        return self._t

    def renormalize_from(self, t):
        self.psi /= np.sqrt(float(t[0]) / self.norm0)


def _rank_main(rank, world, port, case_idx, out_dir):
    import datetime

    import torch.distributed as dist
    import sys
    sys.path.insert(0, os.path.join(REPO, "trotter-suzuki-mpi_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    from trottersuzuki_b200.slab import Slab, SlabLayout
    case = CASES[case_idx]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lat, psi0, V = whole_lattice(case)
        N, Ny, py, imag, g, calls = case
        layout = SlabLayout(Ny, lat.halo_y, py, rank, world)
        tile = OracleTile(lat, layout, psi0, V, case)
        tile.norm0 = O.expectations(lat, psi0)["norm2"]
        slab = Slab(tile, layout, dist, imag_time=imag)
        for n in calls:
            slab.evolve(n)
        a, b = layout.inner_rows()
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), tile.psi[a:b])
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"inner_start": layout.inner_start, "inner_end": layout.inner_end}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case_idx", range(len(CASES)))
def test_slabs_over_gloo_reproduce_the_whole_lattice(case_idx, world, tmp_path):
    import torch.multiprocessing as mp

    import oracle as O
    case = CASES[case_idx]
    mp.start_processes(_rank_main, args=(world, free_port(), case_idx, str(tmp_path)),
                       nprocs=world, join=True, start_method="spawn")
    lat, psi0, V = whole_lattice(case)
    N, Ny, py, imag, g, calls = case
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(1e-3, imag, 1.0, g, 0.0, 0.0, norm0=n0)
    tr, ti = O.exp_table(V, 1e-3, imag)
    ref = psi0
    for n in calls:
        ref = O.evolve(p, ref, tr, ti, n)
    off = lat.halo_y if py else 0
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy")
        meta = json.loads((tmp_path / f"rank{r}.json").read_text())
        want = ref[meta["inner_start"] + off:meta["inner_end"] + off]
        if imag:
            assert np.abs(got - want).max() <= 1e-13 * np.abs(ref).max()
        else:
            assert np.array_equal(got, want), r


def test_layout_matches_the_reference_borders():
    """Tile rows per rank as src/common.cpp:83-102 computes them."""
    from trottersuzuki_b200.slab import SlabLayout, calculate_borders
    assert calculate_borders(0, 3, 100, 4, False, 34) == (0, 38, 0, 34)
    assert calculate_borders(1, 3, 100, 4, False) == (30, 72, 34, 68)
    assert calculate_borders(2, 3, 100, 4, False) == (64, 100, 68, 100)
    assert calculate_borders(0, 3, 100, 4, True) == (-4, 38, 0, 34)
    assert calculate_borders(2, 3, 100, 4, True) == (64, 104, 68, 100)
    # slabs: an even number of rows per rank (44 rows over 3 ranks: 16, not 15)
    assert SlabLayout(44, 4, False, 1, 3).inner_start == 16
    top = SlabLayout(100, 4, False, 0, 3)
    assert top.up is None and top.down == 1
    sends, recvs = SlabLayout(100, 4, True, 2, 3).messages()
    assert sends == [(32, 4, 0, 1), (4, 4, 1, 2)] and recvs == [(0, 4, 1, 1), (36, 4, 0, 2)]
    # after the last step of a call the wrap (rank 2 -> 0) is skipped
    sends, recvs = SlabLayout(100, 4, True, 2, 3).messages(final=True)
    assert sends == [(4, 4, 1, 2)] and recvs == [(0, 4, 1, 1)]


# ---- the library's slab plan (ts_b200_slab_messages / ts_b200_slab_windows):
# host functions, no device needed

LAYOUTS = [(ny, h, per, world) for ny in (40, 41, 100, 333) for h in (4, 8)
           for per in (False, True) for world in (1, 2, 3, 5)]


def _layouts():
    from trottersuzuki_b200.slab import SlabLayout
    for ny, h, per, world in LAYOUTS:
        for rank in range(world):
            try:
                yield SlabLayout(ny, h, per, rank, world)
            except ValueError:
                continue


def test_library_messages_match_the_layout():
    """The messages the native engine posts are the layout's (the reference's
    exchange, src/cpukernel.cpp:717-747), in the same order, final or not."""
    from trottersuzuki_b200.slab import slab_messages
    n = 0
    for lay in _layouts():
        for final in (False, True):
            assert slab_messages(lay, final) == lay.messages(final), (lay.ny, lay.rank, final)
            n += 1
    assert n > 100


def test_split_windows_cover_the_slab():
    """Edge bands hold every row sent to a neighbour, the interior reads no
    halo row (its walk reaches `reach` rows past its window), the windows
    start on even rows and together cover the tile once."""
    from trottersuzuki_b200.slab import split_windows
    n_split = 0
    for lay in _layouts():
        a, b = lay.inner_rows()
        for reach in (4, 6):
            if reach > lay.halo:
                continue
            edge, inner, split = split_windows(lay.rows, a, b, lay.halo, reach,
                                               lay.up is not None, lay.down is not None)
            if not split:
                continue
            n_split += 1
            wins = [w for w in edge if w[1] > w[0]] + [inner]
            covered = sorted(r for w in wins for r in range(*w))
            assert covered == list(range(lay.rows))
            assert all(w[0] % 2 == 0 for w in wins)
            sends, _ = lay.messages()
            for row, cnt, _, _ in sends:
                assert any(w[0] <= row and row + cnt <= w[1] for w in edge)
            # halo rows exist on the sides with a neighbour
            assert lay.up is None or inner[0] - reach >= a
            assert lay.down is None or inner[1] + reach <= b
    assert n_split > 50


def _plan_rank(rank, world, port, out_dir):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.join(REPO, "trotter-suzuki-mpi_b200"))
    from trottersuzuki_b200.slab import SlabLayout, slab_messages
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {}
        for ny, per in ((100, True), (100, False), (41, True)):
            lay = SlabLayout(ny, 4, per, rank, world)
            plans = [None] * world
            mine = {f: slab_messages(lay, f) for f in (False, True)}
            dist.all_gather_object(plans, mine)
            # every span sent to a peer meets a receive of that peer from this
            # rank, in the same position of the per-peer order (NCCL matches
            # sends and receives between two ranks in posting order)
            ok = True
            for f in (False, True):
                for p in range(world):
                    to_p = [(c, tag) for _, c, peer, tag in plans[rank][f][0] if peer == p]
                    p_from_me = [(c, tag) for _, c, peer, tag in plans[p][f][1] if peer == rank]
                    ok = ok and to_p == p_from_me
            res[f"{ny}-{per}"] = ok
        with open(os.path.join(out_dir, f"plan{rank}.json"), "w") as fh:
            json.dump(res, fh)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_library_messages_pair_up_across_ranks(world, tmp_path):
    """Over gloo ranks: each rank's sends to a peer and that peer's receives
    from it agree in number, size, tag and order (so NCCL's in-order matching
    pairs them), on every step and on the last step of a call."""
    import torch.multiprocessing as mp
    mp.start_processes(_plan_rank, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        res = json.loads((tmp_path / f"plan{r}.json").read_text())
        assert all(res.values()), (r, res)
