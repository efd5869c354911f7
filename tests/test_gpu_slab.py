"""Slabs of one lattice as B200 tiles (trottersuzuki_b200.slab.KernelTile),
here all on the one GPU of the test box with the exchange done in-process:
the same layout and messages as Slab.evolve sends between ranks, the rows
copied between the tiles' device spans, the norm summed on the device.  The
slabs reproduce the whole lattice evolved as one tile (bit for bit in real
time)."""
import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params
from test_slab import CASES, whole_lattice

pytestmark = pytest.mark.gpu


def run_slabs(case, world):
    import torch
    from trottersuzuki_b200 import Kernel
    from trottersuzuki_b200.slab import KernelTile, SlabLayout
    lat, psi0, V = whole_lattice(case)
    N, Ny, py, imag, g, calls = case
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    off = lat.halo_y if py else 0
    stream = torch.cuda.Stream()
    lays, tiles, kernels = [], [], []
    for r in range(world):
        lay = SlabLayout(Ny, lat.halo_y, py, r, world)
        p = lat.params(1e-3, imag, 1.0, g, 0.0, 0.0, norm0=n0)
        p.H = lay.rows
        p.iy0, p.iy1 = lay.inner_rows()
        p.periodic_y = 0
        rows = slice(lay.start + off, lay.end + off)
        k = Kernel(desc_from_params(p))
        k.set_state(np.ascontiguousarray(psi0[rows]))
        tr, ti = O.exp_table(V[rows], 1e-3, imag)
        k.set_exp_potential(tr, ti)
        lays.append(lay)
        kernels.append(k)
        tiles.append(KernelTile(k, stream))
    with torch.cuda.stream(stream):
        for n in calls:
            for i in range(n):
                for t in tiles:
                    t.step()
                if imag:
                    norms = [t.last_norm() for t in tiles]
                    total = torch.stack([x[0] for x in norms]).sum().reshape(1)
                    for t in tiles:
                        t.renormalize_from(total)
                final = i == n - 1
                sent = {}
                for r, (lay, t) in enumerate(zip(lays, tiles)):
                    for row, cnt, peer, tag in lay.messages(final)[0]:
                        sent[(r, peer, tag)] = t.rows(row, cnt).clone()
                for r, (lay, t) in enumerate(zip(lays, tiles)):
                    for row, cnt, src, tag in lay.messages(final)[1]:
                        t.rows(row, cnt).copy_(sent[(src, r, tag)])
    torch.cuda.synchronize()
    p = lat.params(1e-3, imag, 1.0, g, 0.0, 0.0, norm0=n0)
    tr, ti = O.exp_table(V, 1e-3, imag)
    ref = psi0
    for n in calls:
        ref = O.evolve(p, ref, tr, ti, n)
    out = []
    for lay, k in zip(lays, kernels):
        a, b = lay.inner_rows()
        out.append((k.get_state()[a:b], ref[lay.inner_start + off:lay.inner_end + off]))
        k.close()
    return out, ref


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case_idx", range(len(CASES)))
def test_kernel_slabs_reproduce_the_whole_lattice(case_idx, world):
    case = CASES[case_idx]
    out, ref = run_slabs(case, world)
    for got, want in out:
        assert np.abs(got - want).max() <= 1e-10 * np.abs(ref).max()


# ---- slabs driven by the library (trottersuzuki_b200.slab.NativeSlabs):
# edge bands and interior on two streams, the exchange and the norm issued
# on the streams, graphs for runs of 16 steps

def _lattice(N, Ny, px, py, omega=0.0):
    lat = O.Lattice(N, 8.0, Ny, 8.0, px, py, omega)
    X, Y = lat.coordinates()
    rng = np.random.default_rng(N * 7 + Ny)
    psi0 = np.exp(-((X - 0.5) ** 2 + (Y + 0.4) ** 2) / 2.0) * np.exp(0.4j * X)
    psi0 = psi0 * (1 + 0.02 * rng.uniform(-1, 1, lat.shape))
    V = 0.5 * (X ** 2 + 1.3 * Y ** 2)
    return lat, psi0, V


def _kernel(p, psi, V, dt, imag, precision):
    from trottersuzuki_b200 import Kernel
    k = Kernel(desc_from_params(p, precision))
    k.set_state(np.ascontiguousarray(psi))
    tr, ti = O.exp_table(V, dt, imag)
    k.set_exp_potential(tr, ti)
    return k


def _slab_kernels(lat, psi0, V, world, dt, imag, g, omega, n0, precision):
    from trottersuzuki_b200.slab import SlabLayout
    off = lat.halo_y if lat.periodic_y else 0
    lays, ks = [], []
    for r in range(world):
        lay = SlabLayout(lat.global_no_halo_dim_y, lat.halo_y, lat.periodic_y, r, world)
        p = lat.params(dt, imag, 1.0, g, 0.0, omega, norm0=n0)
        p.H = lay.rows
        p.iy0, p.iy1 = lay.inner_rows()
        p.periodic_y = 0
        p.rot_off_y += lay.start + off  # the slab's first row in the lattice's rows
        rows = slice(lay.start + off, lay.end + off)
        lays.append(lay)
        ks.append(_kernel(p, psi0[rows], V[rows], dt, imag, precision))
    return lays, ks


def _inner(lat, lays, ks):
    """The slabs' inner rows as the lattice's tile rows (halo rows of a
    periodic lattice left out)."""
    parts = []
    for lay, k in zip(lays, ks):
        a, b = lay.inner_rows()
        parts.append(k.get_state()[a:b])
    return np.concatenate(parts, axis=0)


def _compare_native(lat, psi0, V, world, calls, imag=False, g=2.0, omega=0.0, split=True,
                    precision=None):
    from trottersuzuki_b200 import _capi
    from trottersuzuki_b200.slab import NativeSlabs
    precision = _capi.FP64 if precision is None else precision
    dt = 1e-3
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    lays, ks = _slab_kernels(lat, psi0, V, world, dt, imag, g, omega, n0, precision)
    with NativeSlabs.local(ks, lays) as s:
        s.set_split(split)
        plans = [s.plan(i) for i in range(world)]
        for n in calls:
            s.evolve(n)
        got = _inner(lat, lays, ks)
    for k in ks:
        k.close()
    whole = _kernel(lat.params(dt, imag, 1.0, g, 0.0, omega, norm0=n0), psi0, V, dt, imag,
                    precision)
    for n in calls:
        whole.evolve(n)
    off = lat.halo_y if lat.periodic_y else 0
    want = whole.get_state()[off:off + lat.global_no_halo_dim_y]
    whole.close()
    return got, want, plans


@pytest.mark.parametrize("split", [True, False], ids=["split", "one_launch"])
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("case_idx", range(len(CASES)))
def test_native_slabs_reproduce_the_whole_tile(case_idx, world, split):
    """Slabs in one process, exchanged by the library: the whole tile's bits
    in real time (every cell takes the same arithmetic), its result to
    rounding in imaginary time (the norm is summed in another order), and
    the oracle's at the parity bar."""
    N, Ny, py, imag, g, calls = CASES[case_idx]
    lat, psi0, V = _lattice(N, Ny, False, py)
    got, want, plans = _compare_native(lat, psi0, V, world, calls, imag=imag, g=g, split=split)
    # (slabs with a short interior step in one launch even when split)
    assert split or not any(p[2] for p in plans)
    if imag:
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    else:
        assert np.array_equal(got, want)
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    p = lat.params(1e-3, imag, 1.0, g, 0.0, 0.0, norm0=n0)
    tr, ti = O.exp_table(V, 1e-3, imag)
    ref = psi0
    for n in calls:
        ref = O.evolve(p, ref, tr, ti, n)
    off = lat.halo_y if py else 0
    assert np.abs(got - ref[off:off + Ny]).max() <= 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_native_slabs_in_graphs(imag):
    """Long calls replay the 16-step graphs (37 steps: 2 graphs, 4 direct
    steps and the final one); a tall lattice in 4 slabs, periodic in y."""
    lat, psi0, V = _lattice(64, 160, False, True)
    got, want, plans = _compare_native(lat, psi0, V, 4, (37, 20), imag=imag, g=3.0)
    assert all(p[2] for p in plans)
    if imag:
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_native_slabs_rotating_frame(imag):
    """Rotating frame (halo 8 rows, the checked walk reaching 6 rows past its
    window) and the rows' rotation coefficients at the slab's offset."""
    lat, psi0, V = _lattice(48, 96, False, False, omega=0.6)
    got, want, plans = _compare_native(lat, psi0, V, 3, (9, 18), imag=imag, g=1.0, omega=0.6)
    assert all(p[2] for p in plans)
    if imag:
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_native_slabs_fp32(imag):
    """Single precision: in real time the per-step kinetic coefficients
    advance once per step of a split step (the second of its two launches to
    finish moves the schedule on), so the slabs keep the whole tile's bits."""
    from trottersuzuki_b200 import _capi
    lat, psi0, V = _lattice(72, 120, False, True)
    got, want, _ = _compare_native(lat, psi0, V, 3, (21, 17), imag=imag, g=2.0,
                                   precision=_capi.FP32)
    if imag:
        assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
    else:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("py", [True, False], ids=["periodic_y", "closed_y"])
def test_native_slabs_periodic_x(py, world):
    """Periodic in x: each slab refreshes the x halo of the rows whose
    lattice rows the whole tile refreshes, received halo rows included, after
    the exchange (the interior then waits for the end of the previous step);
    the whole tile's bits, halo columns included."""
    lat, psi0, V = _lattice(40, 64, True, py)
    got, want, _ = _compare_native(lat, psi0, V, world, (6, 19), g=1.5)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("imag", [False, True], ids=["real", "imag"])
def test_native_slab_over_nccl_one_rank(imag):
    """The NCCL transport on the one GPU of the box: one rank holding the
    whole periodic lattice as a slab that is its own upper and lower
    neighbour (ncclSend/ncclRecv to itself, a one-rank ncclAllReduce of the
    norm), against the whole tile with its periodic halo kernel."""
    import datetime
    import socket

    import torch.distributed as dist
    from trottersuzuki_b200 import _capi
    from trottersuzuki_b200.slab import NativeSlabs, SlabLayout
    lat, psi0, V = _lattice(56, 72, False, True)
    dt, g = 1e-3, 2.0
    n0 = O.expectations(lat, psi0)["norm2"] if imag else 0.0
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        lay = SlabLayout(72, lat.halo_y, True, 0, 1)
        assert lay.up == 0 and lay.down == 0
        p = lat.params(dt, imag, 1.0, g, 0.0, 0.0, norm0=n0)
        p.iy0, p.iy1 = lay.inner_rows()
        p.periodic_y = 0
        k = _kernel(p, psi0, V, dt, imag, _capi.FP64)
        with NativeSlabs.nccl(k, lay, dist) as s:
            edge, inner, split, _ = s.plan()
            assert split and edge[1][1] == lay.rows
            for n in (5, 33, 2):
                s.evolve(n)
            a, b = lay.inner_rows()
            got = k.get_state()[a:b]
        k.close()
    finally:
        dist.destroy_process_group()
    whole = _kernel(lat.params(dt, imag, 1.0, g, 0.0, 0.0, norm0=n0), psi0, V, dt, imag,
                    _capi.FP64)
    for n in (5, 33, 2):
        whole.evolve(n)
    want = whole.get_state()[lat.halo_y:lat.halo_y + 72]
    whole.close()
    if imag:
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    else:
        assert np.array_equal(got, want)
