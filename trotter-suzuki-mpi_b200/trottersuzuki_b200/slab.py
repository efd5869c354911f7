"""One lattice over several ranks: slabs of rows, one per rank.

The reference splits a lattice over MPI ranks (Lattice2D on MPI_Cart_create,
tile borders src/common.cpp:83-102) and, after every step but the last of an
evolve() call, sends each neighbour the halo_y rows next to its border
(src/cpukernel.cpp:717-747, CPUBlock::finish_halo_exchange); the imaginary-
time renormalisation sums the squared norm over the ranks
(src/cpukernel.cpp:537-546).  Here the ranks are stacked along y, the
reference's layout with mpi_dims = (ranks, 1).  Each rank's slab is a tile
with its own halo rows, evolved by its own fused step; the halo rows travel
as contiguous device spans with torch.distributed point-to-point operations
(NCCL between GPUs, gloo on the CPU), and the norm is all-reduced on the
device before the deferred renormalisation is set from it.

The exchange does not depend on what a tile is: `Slab` drives any object with
step(), rows(row0, nrows) (a writable 1D tensor view of those rows),
last_norm() (a 1-element float64 tensor view) and renormalize_from(t).
`KernelTile` is the GPU tile; the tests drive the same exchange over the
oracle on the CPU.
"""
import contextlib
import ctypes as C
import math

from ._capi import check, lib


def calculate_borders(coord, dims, length, halo, periodic, inner=None):
    """(start, end, inner_start, inner_end) of rank `coord` of `dims` along an
    axis of `length` cells (src/common.cpp:83-102); `inner` overrides the
    rows per rank, ceil(length / dims)."""
    if inner is None:
        inner = int(math.ceil(float(length) / float(dims)))
    inner_start = coord * inner
    if periodic:
        start = inner_start - halo
    else:
        start = 0 if coord == 0 else inner_start - halo
    end = inner_start + inner + halo
    if end > length:
        end = length + halo if periodic else length
    if periodic:
        inner_end = end - halo
    else:
        inner_end = end if end == length else end - halo
    return start, end, inner_start, inner_end


class SlabLayout:
    """Rows of rank `rank` of `world` over a lattice of `ny` rows.

    Each rank owns ceil(ny / world) rows rounded up to an even number: the
    checkerboard of the pair sweeps follows the tile's own row index, so a
    slab has to start on an even lattice row to sweep the same pairs as the
    whole lattice (the reference's MPI tiles start wherever ceil(ny / ranks)
    puts them, and an odd start shifts their checkerboard)."""

    def __init__(self, ny, halo_y, periodic_y, rank, world):
        if world < 2:
            raise ValueError("a slab layout needs at least two ranks")
        if halo_y % 2:
            raise ValueError("the halo must be even")
        self.ny, self.halo, self.periodic = ny, halo_y, bool(periodic_y)
        self.rank, self.world = rank, world
        inner = int(math.ceil(float(ny) / float(world)))
        inner += inner & 1
        if inner * (world - 1) >= ny:
            raise ValueError("too few rows for this many ranks")
        self.start, self.end, self.inner_start, self.inner_end = calculate_borders(
            rank, world, ny, halo_y, periodic_y, inner)
        if self.inner_end - self.inner_start < halo_y:
            raise ValueError("each rank needs at least halo_y inner rows")
        self.rows = self.end - self.start
        # neighbours along y (MPI_Cart_shift(cartcomm, 0, 1, &UP, &DOWN))
        self.up = rank - 1 if rank > 0 else (world - 1 if periodic_y else None)
        self.down = rank + 1 if rank < world - 1 else (0 if periodic_y else None)

    def inner_rows(self):
        """Tile-local [first, last) of the rows this rank owns."""
        return self.inner_start - self.start, self.inner_end - self.start

    def messages(self, final=False):
        """(sends, recvs): (tile row, rows, peer, tag).  As the reference:
        the last halo rows of the inner region go down into the lower
        neighbour's top halo (tag 1), the rows from halo_y on go up into the
        upper neighbour's bottom halo (tag 2).  final: the step is the last of
        an evolve() call, after which a single tile skips its periodic halo
        copy (src/solver.cpp:203-209): the messages across the periodic wrap
        are left out, those between slabs (inside the lattice) are not."""
        h, lo = self.halo, self.inner_end - self.start
        last = self.world - 1
        down_ok = self.down is not None and not (final and self.rank == last)
        up_ok = self.up is not None and not (final and self.rank == 0)
        sends, recvs = [], []
        if down_ok:
            sends.append((lo - h, h, self.down, 1))
        if up_ok:
            sends.append((h, h, self.up, 2))
        if up_ok:
            recvs.append((0, h, self.up, 1))
        if down_ok:
            recvs.append((lo, h, self.down, 2))
        return sends, recvs


def exchange(tile, layout, dist, group=None, final=False):
    """One halo exchange of `tile` with its neighbours (all ranks call it)."""
    sends, recvs = layout.messages(final)
    ops = [dist.P2POp(dist.isend, tile.rows(r, n), peer, group, tag)
           for r, n, peer, tag in sends]
    ops += [dist.P2POp(dist.irecv, tile.rows(r, n), peer, group, tag)
            for r, n, peer, tag in recvs]
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class Slab:
    """A tile that is one slab of a lattice split across the ranks of `dist`
    (torch.distributed, initialised).  evolve(n) runs the reference's loop:
    n steps, the norm summed over the ranks in imaginary time, the halo rows
    exchanged after every step.  Between slabs the exchange follows the last
    step of a call too: the reference's MPI run skips it there, and a second
    evolve() call then starts from stale halo rows, so that its slabs drift
    from the single-tile result; here the slabs reproduce the single tile."""

    def __init__(self, tile, layout, dist, imag_time=False, group=None):
        self.tile, self.layout, self.dist, self.group = tile, layout, dist, group
        self.imag_time = bool(imag_time)

    def evolve(self, iterations):
        n = int(iterations)
        # the tile's stream is the current one, so that the collectives order
        # against its steps
        with getattr(self.tile, "context", contextlib.nullcontext)():
            for i in range(n):
                self.tile.step()
                if self.imag_time:
                    t = self.tile.last_norm()
                    self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
                    self.tile.renormalize_from(t)
                exchange(self.tile, self.layout, self.dist, self.group, final=i == n - 1)


class _DeviceSpan:
    """A raw device span as a 1D tensor-compatible object (no copy)."""

    def __init__(self, ptr, nbytes, typestr="|u1", itemsize=1):
        self.__cuda_array_interface__ = {
            "shape": (nbytes // itemsize,), "typestr": typestr, "data": (ptr, False),
            "version": 3, "strides": None}


class KernelTile:
    """A Kernel (one slab's tile, closed in y: the neighbours supply the halo
    rows) on this rank's GPU, its work queued on `stream` (a torch stream)."""

    def __init__(self, kernel, stream):
        import torch
        self.torch = torch
        self.k = kernel
        self.stream = stream
        check(lib().ts_b200_set_stream(kernel.handle, C.c_void_p(stream.cuda_stream)),
              kernel.handle)

    def context(self):
        return self.torch.cuda.stream(self.stream)

    def step(self):
        check(lib().ts_b200_step(self.k.handle, 0), self.k.handle)

    def rows(self, row0, nrows):
        ptr, nbytes = C.c_void_p(), C.c_size_t()
        check(lib().ts_b200_rows(self.k.handle, int(row0), int(nrows), C.byref(ptr),
                                 C.byref(nbytes)), self.k.handle)
        return self.torch.as_tensor(_DeviceSpan(ptr.value, nbytes.value),
                                    device=self.torch.device("cuda",
                                                             self.torch.cuda.current_device()))

    def last_norm(self):
        ptr = C.c_void_p()
        check(lib().ts_b200_last_norm(self.k.handle, C.byref(ptr)), self.k.handle)
        return self.torch.as_tensor(_DeviceSpan(ptr.value, 8, "<f8", 8),
                                    device=self.torch.device("cuda",
                                                             self.torch.cuda.current_device()))

    def renormalize_from(self, t):
        check(lib().ts_b200_renormalize_from(self.k.handle, C.c_void_p(t.data_ptr())),
              self.k.handle)
