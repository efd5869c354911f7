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
