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

`NativeSlabs` runs the same layout inside the library (ts_b200_slabs_*):
each step as the slab's edge bands and its interior on two streams, the
halo rows over NCCL (one slab per rank) or by device copies (slabs of one
process), the norm summed on the device, all issued on the streams without
a host round trip per step and replayed from CUDA graphs.
"""
import contextlib
import ctypes as C
import math

from ._capi import SlabLink, check, lib


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
        if world < 1 or not 0 <= rank < world:
            raise ValueError("rank outside the world")
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
        if self.down is not None and self.end - self.inner_end != halo_y:
            # the borders reach the lattice's end before the last rank (too
            # many ranks for the rows): the slabs would overlap
            raise ValueError("too few rows for this many ranks")

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


def xhalo_rows(layout):
    """Tile rows [r0, r1) of a slab whose periodic x halo is refreshed after
    a step: those whose lattice row the whole tile refreshes.  The whole
    tile refreshes its rows [inner_y0, inner_y0 + dim_y - 2 halo_y)
    (src/cpukernel.cpp:706-716): for a lattice periodic in y every lattice
    row (its y-halo rows then copy refreshed rows), for a closed one the
    lattice rows below ny - 2 halo_y."""
    if layout.periodic:
        return 0, layout.rows
    return 0, max(0, min(layout.rows, layout.ny - 2 * layout.halo - layout.start))


def slab_link(layout):
    """The C-ABI link of a layout: its neighbours (-1: none), the links that
    cross the lattice's periodic wrap (rank 0 upwards, the last rank
    downwards) and the rows whose periodic x halo the slab refreshes."""
    up = -1 if layout.up is None else int(layout.up)
    down = -1 if layout.down is None else int(layout.down)
    return SlabLink(up, down, int(up >= 0 and layout.periodic and layout.rank == 0),
                    int(down >= 0 and layout.periodic and layout.rank == layout.world - 1),
                    *xhalo_rows(layout))


def split_windows(rows, inner_y0, inner_y1, halo, reach, has_up, has_down):
    """Row windows of a slab's split step (ts_b200_slab_windows, host only):
    (edge windows [(a0, a1), (b0, b1)], interior (i0, i1), split)."""
    out = (C.c_int32 * 8)()
    check(lib().ts_b200_slab_windows(int(rows), int(inner_y0), int(inner_y1), int(halo),
                                     int(reach), int(bool(has_up)), int(bool(has_down)), out))
    v = list(out)
    return [(v[0], v[1]), (v[2], v[3])], (v[4], v[5]), bool(v[6])


def slab_messages(layout, final=False):
    """(sends, recvs) of the library's exchange for `layout`, in the form of
    SlabLayout.messages (tile row, rows, peer, tag): ts_b200_slab_messages."""
    a, b = layout.inner_rows()
    out = (C.c_int32 * 16)()
    link = slab_link(layout)
    n = lib().ts_b200_slab_messages(a, b, layout.halo, C.byref(link), int(bool(final)), out)
    if n < 0:
        raise ValueError("invalid slab")
    v = list(out)
    sends, recvs = [], []
    for i in range(n):
        peer, row, tag, send = v[4 * i:4 * i + 4]
        (sends if send else recvs).append((row, layout.halo, peer, tag))
    return sends, recvs


class NativeSlabs:
    """Slabs of one lattice driven by the library.

    local(kernels, layouts): every slab in this process, on one GPU; the
    halo rows move by device copies.  nccl(kernel, layout, dist): one slab
    per rank of `dist` (torch.distributed, initialised); the ranks build an
    NCCL communicator of their own (the id travels over `dist`) and exchange
    halo rows with ncclSend/ncclRecv on the slab's streams.  Each kernel is a
    Kernel whose descriptor is its slab's tile (closed in y, inner rows of the
    layout, the whole lattice's norm0 in imaginary time)."""

    def __init__(self, ptr, keep):
        self._ptr = ptr
        self._keep = keep

    @classmethod
    def local(cls, kernels, layouts):
        n = len(kernels)
        handles = (C.c_void_p * n)(*[k.handle for k in kernels])
        links = (SlabLink * n)(*[slab_link(lay) for lay in layouts])
        ptr = C.c_void_p()
        check(lib().ts_b200_slabs_create_local(C.byref(ptr), handles, links, n), kernels[0].handle)
        return cls(ptr, list(kernels))

    @classmethod
    def nccl(cls, kernel, layout, dist=None, group=None):
        """dist may be None for a one-rank layout (its own neighbour across
        the periodic wrap)."""
        buf = (C.c_ubyte * 128)()
        if dist is None:
            if layout.world != 1:
                raise ValueError("several ranks need torch.distributed to share the NCCL id")
            check(lib().ts_b200_nccl_unique_id(buf, 128))
            uid = buf
        else:
            if dist.get_rank(group) == 0:
                check(lib().ts_b200_nccl_unique_id(buf, 128))
            obj = [bytes(buf)]
            src = 0 if group is None else dist.get_global_rank(group, 0)
            dist.broadcast_object_list(obj, src=src, group=group)
            uid = (C.c_ubyte * 128).from_buffer_copy(obj[0])
        link = slab_link(layout)
        ptr = C.c_void_p()
        check(lib().ts_b200_slabs_create_nccl(C.byref(ptr), kernel.handle, C.byref(link), uid, 128,
                                              int(layout.world), int(layout.rank)), kernel.handle)
        return cls(ptr, [kernel])

    def set_split(self, on):
        check(lib().ts_b200_slabs_set_split(self._ptr, int(bool(on))), slabs=self._ptr)

    def plan(self, tile=0):
        """(edge windows, interior window, split, kernel launches per step)."""
        out = (C.c_int32 * 8)()
        check(lib().ts_b200_slabs_plan(self._ptr, int(tile), out), slabs=self._ptr)
        v = list(out)
        return [(v[0], v[1]), (v[2], v[3])], (v[4], v[5]), bool(v[6]), v[7]

    def evolve(self, iterations):
        check(lib().ts_b200_slabs_evolve(self._ptr, int(iterations)), slabs=self._ptr)

    def close(self):
        if self._ptr:
            lib().ts_b200_slabs_destroy(self._ptr)
            self._ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
