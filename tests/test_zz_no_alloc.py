"""ts_b200_squared_norm_noalloc: the squared norm of a device tile the caller
owns, computed without any device allocation (for callers whose device memory
belongs to another allocator or a fixed pool, or that must not allocate --
and so synchronise the device -- after start-up).  Checked through the C ABI
against the allocating entry point (ts_b200_squared_norm) and the oracle's
squared norm on two calls in a row, on a pitched tile and a non-default
stream, and on narrow tiles that fill the whole static scratch (16384 rows,
so the kernel's grid-stride row loop runs); collected last so that a run
stopping at the first failure has run everything else first."""
import ctypes as C

import numpy as np
import pytest

import oracle as O
from helpers import desc_from_params, seeded_case

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # the FP64 reduction tolerance used for the norm elsewhere in the tests


def _device_tile(psi, torch, dtype):
    t = torch.from_numpy(np.ascontiguousarray(psi.astype(dtype))).cuda()
    return t


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_norm_matches_allocating_entry_point(precision):
    import torch
    from trottersuzuki_b200 import Kernel, _capi
    L = _capi.lib()
    lat, psi0, V = seeded_case(200, 10.0, 150, (True, True))
    p = lat.params(1e-3, False)
    with Kernel(desc_from_params(p, precision)) as k:
        k.set_state(psi0)
        ref = k.squared_norm()
    dtype = np.complex128 if precision == 0 else np.complex64
    tile = _device_tile(psi0, torch, dtype)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    ix0, ix1, iy0, iy1 = lat.inner()
    for call in range(2):
        out.zero_()
        st = L.ts_b200_squared_norm_noalloc(
            C.c_void_p(tile.data_ptr()), precision, lat.dim_x, lat.dim_x, lat.dim_y, ix0, ix1,
            iy0, iy1, lat.delta_x, lat.delta_y, C.c_void_p(out.data_ptr()), None)
        assert st == 0, (call, st)
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= REL_TOL * abs(ref), (call, got, ref)


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_norm_pitched_tile_on_a_stream_matches_oracle(precision):
    """Rows padded to a pitch wider than the tile, the call queued on a
    non-default stream, two calls in a row: the oracle's squared norm of the
    same values (src/cpukernel.cpp:526-549)."""
    import torch
    from trottersuzuki_b200 import _capi
    L = _capi.lib()
    lat, psi0, V = seeded_case(131, 10.0, 97, (True, False))
    p = lat.params(1e-3, False)
    dtype = np.complex128 if precision == 0 else np.complex64
    vals = psi0.astype(dtype)
    ref = O.squared_norm(p, vals.astype(np.complex128))
    pitch = lat.dim_x + 13
    host = np.zeros((lat.dim_y, pitch), dtype)
    host[:, :lat.dim_x] = vals
    host[:, lat.dim_x:] = 1e3  # padding that must not enter the sum
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        tile = torch.from_numpy(host).cuda()
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    ix0, ix1, iy0, iy1 = lat.inner()
    for call in range(2):
        st = L.ts_b200_squared_norm_noalloc(
            C.c_void_p(tile.data_ptr()), precision, pitch, lat.dim_x, lat.dim_y, ix0, ix1, iy0,
            iy1, lat.delta_x, lat.delta_y, C.c_void_p(out.data_ptr()),
            C.c_void_p(stream.cuda_stream))
        assert st == 0, (call, st)
        stream.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= REL_TOL * abs(ref), (call, got, ref)


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_norm_fills_the_whole_scratch(precision):
    """16384 x 8 tile: as many rows as the scratch holds, more rows than the
    1184-block grid has warps, so each warp walks several rows.  Compared with
    a numpy FP64 sum of the same values."""
    import torch
    from trottersuzuki_b200 import _capi
    L = _capi.lib()
    rng = np.random.default_rng(7)
    H, W = 16384, 8
    dtype = np.complex128 if precision == 0 else np.complex64
    vals = (rng.standard_normal((H, W)) + 1j * rng.standard_normal((H, W))).astype(dtype)
    v64 = vals.astype(np.complex128)
    ref = float(np.sum(v64.real ** 2 + v64.imag ** 2)) * 0.5 * 0.25
    tile = torch.from_numpy(vals).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for call in range(2):
        out.fill_(-1.0)
        st = L.ts_b200_squared_norm_noalloc(C.c_void_p(tile.data_ptr()), precision, W, W, H, 0,
                                            W, 0, H, 0.5, 0.25, C.c_void_p(out.data_ptr()), None)
        assert st == 0, (call, st)
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= REL_TOL * abs(ref), (call, got, ref)


def test_noalloc_norm_rejects_tiles_beyond_its_scratch():
    import torch
    from trottersuzuki_b200 import _capi
    L = _capi.lib()
    tile = torch.zeros((16385, 4), dtype=torch.complex128, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = L.ts_b200_squared_norm_noalloc(C.c_void_p(tile.data_ptr()), 0, 4, 4, 16385, 0, 4, 0,
                                        16385, 1.0, 1.0, C.c_void_p(out.data_ptr()), None)
    assert st == 4  # TS_B200_UNSUPPORTED: more rows than the static scratch holds
