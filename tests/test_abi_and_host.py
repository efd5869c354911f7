"""CPU checks of the boundary and the host layer (no GPU needed).

- libtsb200.so / libtrottersuzuki_b200.so load and export every function that
  include/ts_b200.h and include/ts_host.h declare.
- Without a device the C ABI returns TS_B200_NO_DEVICE instead of crashing.
- The C++ host layer's lattice geometry and analytic initial states are
  identical to the reference's (compared with the compiled reference).
- Unknown kernel types are rejected like the reference's "Unknown kernel".
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import tsref
from trottersuzuki_b200 import _capi, api

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    text = open(os.path.join(REPO, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w[\w\s\*]*?\b(ts(?:_b200|h)_\w+)\s*\(",
                                 text, flags=re.M)))


def exported(path):
    lib = C.CDLL(path)
    return lib


def test_cuda_library_exports_every_declared_symbol():
    names = declared_functions("ts_b200.h")
    assert len(names) >= 20
    lib = exported(_capi.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(_capi.SIGNATURES), set(names) ^ set(_capi.SIGNATURES)


def test_host_library_exports_every_declared_symbol():
    names = declared_functions("ts_host.h")
    assert len(names) >= 20
    lib = exported(api.HOST_LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_create_without_device_fails_cleanly():
    d = _capi.Desc()
    d.dim_x = d.dim_y = 8
    d.inner_x1 = d.inner_y1 = 8
    h = C.c_void_p()
    st = _capi.lib().ts_b200_create(C.byref(d), C.byref(h))
    assert st == 6 and not h.value  # TS_B200_NO_DEVICE


def test_invalid_descriptor_is_rejected():
    d = _capi.Desc()
    d.dim_x, d.dim_y = 8, 8
    d.inner_x0, d.inner_x1, d.inner_y0, d.inner_y1 = 0, 9, 0, 8  # inner wider than the tile
    h = C.c_void_p()
    assert _capi.lib().ts_b200_create(C.byref(d), C.byref(h)) == 1  # TS_B200_INVALID_ARGUMENT


GEOMETRY = [
    (256, 20.0, None, False, False, 0.0),
    (250, 100.0, None, True, True, 0.0),
    (61, 10.0, 47, True, False, 0.0),
    (64, 10.0, 33, False, True, 0.0),
    (300, 20.0, None, False, False, 0.7),
    (64, 10.0, None, True, True, 0.5),
]


@pytest.mark.skipif(not tsref.available(), reason="compiled reference not built")
@pytest.mark.parametrize("case", GEOMETRY)
def test_lattice_geometry_matches_reference(case):
    N, L, Ny, px, py, om = case
    g = api.Lattice2D(N, L, Ny, None, px, py, om)
    r = tsref.geometry(tsref.make_config(N, L, Ny, None, px, py, om))
    for f in ("dim_x", "dim_y", "halo_x", "halo_y", "start_x", "start_y", "inner_start_x",
              "inner_start_y", "inner_end_x", "inner_end_y"):
        assert getattr(g, f) == getattr(r, f), f
    assert g.delta_x == r.delta_x and g.delta_y == r.delta_y


@pytest.mark.skipif(not tsref.available(), reason="compiled reference not built")
@pytest.mark.parametrize("kind", ["gaussian", "exponential"])
@pytest.mark.parametrize("case", GEOMETRY[:4])
def test_initial_states_match_reference(kind, case):
    N, L, Ny, px, py, om = case
    g = api.Lattice2D(N, L, Ny, None, px, py, om)
    if kind == "gaussian":
        s = api.GaussianState(g, 0.8, 1.3, 0.4, -0.2, 1.7, 0.3)
        cfg = tsref.make_config(N, L, Ny, None, px, py, om, gaussian=(0.8, 1.3, 0.4, -0.2, 1.7, 0.3),
                                harmonic="none", segments=())
    else:
        s = api.ExponentialState(g, 2, 1, 1.5, 0.2)
        cfg = tsref.make_config(N, L, Ny, None, px, py, om, exponential=(2, 1, 1.5, 0.2),
                                harmonic="none", segments=())
    ref, _ = tsref.run(cfg)
    assert np.array_equal(s.get_state(), ref)


def test_unknown_kernel_type_raises_like_the_reference():
    g = api.Lattice2D(16, 4.0)
    s = api.GaussianState(g, 1.0)
    h = api.Hamiltonian(g, api.HarmonicPotential(g, 1.0, 1.0))
    solver = api.Solver(g, s, h, 1e-3, kernel_type="cpu")
    with pytest.raises(RuntimeError, match="Unknown kernel"):
        solver.evolve(1)


def test_two_component_host_objects():
    """Two-state Solver construction (no GPU needed): a Hamiltonian2Component
    is required, and the CPU kernel type is refused as for one component."""
    g = api.Lattice2D(16, 4.0)
    s1, s2 = api.GaussianState(g, 1.0), api.State(g)
    pot = api.HarmonicPotential(g, 1.0, 1.0)
    h2 = api.Hamiltonian2Component(g, pot, None, 1.0, 1.2, 2.0, 1.0, 3.0, 0.5, 0.0)
    assert h2.potential_b is pot and h2.mass_b == 1.2
    with pytest.raises(RuntimeError, match="Hamiltonian2Component"):
        api.Solver(g, s1, api.Hamiltonian(g, pot), 1e-3, State2=s2)
    solver = api.Solver(g, s1, h2, 1e-3, State2=s2, kernel_type="cpu")
    with pytest.raises(RuntimeError, match="Unknown kernel"):
        solver.evolve(1)
