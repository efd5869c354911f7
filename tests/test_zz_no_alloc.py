"""ts_b200_squared_norm_noalloc: the squared norm of a device tile the caller
owns, computed without any device allocation (for callers whose device memory
belongs to another allocator or a fixed pool, or that must not allocate --
and so synchronise the device -- after start-up).  Checked through the C ABI
against the allocating entry point (ts_b200_squared_norm) on two calls in a
row; collected last so that a run stopping at the first failure has run
everything else first."""
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


def test_noalloc_norm_rejects_tiles_beyond_its_scratch():
    import torch
    from trottersuzuki_b200 import _capi
    L = _capi.lib()
    tile = torch.zeros((16385, 4), dtype=torch.complex128, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = L.ts_b200_squared_norm_noalloc(C.c_void_p(tile.data_ptr()), 0, 4, 4, 16385, 0, 4, 0,
                                        16385, 1.0, 1.0, C.c_void_p(out.data_ptr()), None)
    assert st == 4  # TS_B200_UNSUPPORTED: more rows than the static scratch holds
