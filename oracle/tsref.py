"""ctypes binding of the reference's own CPU implementation (test infrastructure).

oracle/build_ref.sh compiles the reference's unmodified C++ sources with
oracle/ref_driver.cpp into oracle/_ref/libtsref.so (parity flavour, -O2),
libtsref_fast.so (the reference's -Ofast flags) and libtsref_gpu.so (with the
reference's CUDA kernel, kernel_gpu=True).  Only tests/, the golden fixture
generator and bench.py's reference legs use this module.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


class Config(C.Structure):
    _fields_ = [
        ("dim_x", C.c_int), ("dim_y", C.c_int),
        ("length_x", C.c_double), ("length_y", C.c_double),
        ("periodic_x", C.c_int), ("periodic_y", C.c_int),
        ("lattice_angular_velocity", C.c_double),
        ("init_kind", C.c_int),
        ("g_omega_x", C.c_double), ("g_omega_y", C.c_double), ("g_mean_x", C.c_double),
        ("g_mean_y", C.c_double), ("g_norm", C.c_double), ("g_phase", C.c_double),
        ("e_nx", C.c_int), ("e_ny", C.c_int),
        ("pot_kind", C.c_int),
        ("h_omega_x", C.c_double), ("h_omega_y", C.c_double), ("h_mass", C.c_double),
        ("h_mean_x", C.c_double), ("h_mean_y", C.c_double),
        ("mass", C.c_double), ("coupling", C.c_double), ("lhy_coupling", C.c_double),
        ("angular_velocity", C.c_double), ("rot_coord_x", C.c_double), ("rot_coord_y", C.c_double),
        ("force_rotation_periodic", C.c_int),
        ("delta_t", C.c_double),
        ("n_segments", C.c_int),
        ("seg_iterations", C.c_int * 8),
        ("seg_imag", C.c_int * 8),
        ("omp_threads", C.c_int),
        ("kernel_gpu", C.c_int),
        ("cylindrical", C.c_int), ("angular_momentum", C.c_int),
    ]


class Result(C.Structure):
    _fields_ = [
        ("dim_x", C.c_int), ("dim_y", C.c_int), ("halo_x", C.c_int), ("halo_y", C.c_int),
        ("start_x", C.c_int), ("start_y", C.c_int),
        ("inner_start_x", C.c_int), ("inner_start_y", C.c_int),
        ("inner_end_x", C.c_int), ("inner_end_y", C.c_int),
        ("delta_x", C.c_double), ("delta_y", C.c_double),
        ("total_energy", C.c_double), ("kinetic_energy", C.c_double),
        ("potential_energy", C.c_double), ("rotational_energy", C.c_double),
        ("intra_energy", C.c_double), ("lhy_energy", C.c_double), ("squared_norm", C.c_double),
        ("mean_x", C.c_double), ("mean_xx", C.c_double), ("mean_y", C.c_double),
        ("mean_yy", C.c_double), ("mean_px", C.c_double), ("mean_pxpx", C.c_double),
        ("mean_py", C.c_double), ("mean_pypy", C.c_double), ("mean_lz", C.c_double),
        ("state_norm", C.c_double),
        ("initial_total_energy", C.c_double), ("initial_squared_norm", C.c_double),
        ("seconds", C.c_double),
        ("seg_seconds", C.c_double * 8),
    ]


class Config2(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("mass_b", "coupling_b", "coupling_ab", "omega_r", "omega_i")]


class Result2(C.Structure):
    _fields_ = [
        ("total_energy", C.c_double),
        ("kinetic", C.c_double * 2), ("potential", C.c_double * 2),
        ("rotational", C.c_double * 2), ("intra", C.c_double * 2),
        ("inter_species", C.c_double), ("rabi", C.c_double),
        ("squared_norm", C.c_double * 2),
        ("seconds", C.c_double), ("seg_seconds", C.c_double * 8),
    ]


_libs = {}


_NAMES = {"parity": "libtsref.so", "fast": "libtsref_fast.so", "gpu": "libtsref_gpu.so",
          "b200": "libtsref_b200.so"}


def available(flavour="parity"):
    return os.path.exists(os.path.join(REF_DIR, _NAMES[flavour]))


def _lib(flavour="parity"):
    if flavour not in _libs:
        lib = C.CDLL(os.path.join(REF_DIR, _NAMES[flavour]))
        lib.tsref_run.argtypes = [C.POINTER(Config), C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.POINTER(Result)]
        lib.tsref_run.restype = C.c_int
        lib.tsref_geometry.argtypes = [C.POINTER(Config), C.POINTER(Result)]
        lib.tsref_geometry.restype = C.c_int
        lib.tsref_last_error.restype = C.c_char_p
        lib.tsref_run2.argtypes = [C.POINTER(Config), C.POINTER(Config2)] + [C.c_void_p] * 6 + \
            [C.POINTER(Result2)]
        lib.tsref_run2.restype = C.c_int
        lib.tsref_state_io.argtypes = [C.POINTER(Config), C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_char_p, C.c_int]
        lib.tsref_state_io.restype = C.c_int
        _libs[flavour] = lib
    return _libs[flavour]


def make_config(dim_x, length_x, dim_y=None, length_y=None, periodic_x=False, periodic_y=False,
                lattice_angular_velocity=None, *, gaussian=None, exponential=None,
                harmonic=None, mass=1.0, coupling=0.0, lhy_coupling=0.0, angular_velocity=0.0,
                rot_coord=(0.0, 0.0), force_rotation_periodic=False, delta_t=1e-4,
                segments=((1, False),), omp_threads=1, kernel_gpu=False, cylindrical=False,
                angular_momentum=0):
    """Build a Config.  dim_y == 0 selects a 1D lattice.

    gaussian = (omega_x, omega_y, mean_x, mean_y, norm, phase) -> GaussianState;
    exponential = (n_x, n_y, norm, phase) -> ExponentialState; neither -> arrays given.
    harmonic = (omega_x, omega_y, mass, mean_x, mean_y) -> HarmonicPotential;
    harmonic == "none" -> no potential; None -> matrix given.
    """
    c = Config()
    c.dim_x = dim_x
    c.dim_y = dim_x if dim_y is None else dim_y
    c.length_x = length_x
    c.length_y = length_x if length_y is None else length_y
    c.periodic_x = int(periodic_x)
    c.periodic_y = int(periodic_y)
    c.lattice_angular_velocity = (angular_velocity if lattice_angular_velocity is None
                                  else lattice_angular_velocity)
    if gaussian is not None:
        c.init_kind = 1
        (c.g_omega_x, c.g_omega_y, c.g_mean_x, c.g_mean_y, c.g_norm, c.g_phase) = gaussian
    elif exponential is not None:
        c.init_kind = 2
        c.e_nx, c.e_ny, c.g_norm, c.g_phase = exponential
    else:
        c.init_kind = 0
    if harmonic is None:
        c.pot_kind = 0
    elif harmonic == "none":
        c.pot_kind = 2
    else:
        c.pot_kind = 1
        (c.h_omega_x, c.h_omega_y, c.h_mass, c.h_mean_x, c.h_mean_y) = harmonic
    c.mass = mass
    c.coupling = coupling
    c.lhy_coupling = lhy_coupling
    c.angular_velocity = angular_velocity
    c.rot_coord_x, c.rot_coord_y = rot_coord
    c.force_rotation_periodic = int(force_rotation_periodic)
    c.delta_t = delta_t
    if len(segments) > 8:
        raise ValueError("at most 8 evolve() segments")
    c.n_segments = len(segments)
    for i, (it, imag) in enumerate(segments):
        c.seg_iterations[i] = int(it)
        c.seg_imag[i] = int(bool(imag))
    c.omp_threads = omp_threads
    c.kernel_gpu = int(bool(kernel_gpu))
    c.cylindrical = int(bool(cylindrical))
    c.angular_momentum = int(angular_momentum)
    return c


def geometry(cfg, flavour="parity"):
    res = Result()
    if _lib(flavour).tsref_geometry(C.byref(cfg), C.byref(res)) != 0:
        raise RuntimeError(_lib(flavour).tsref_last_error().decode())
    return res


def run(cfg, psi=None, potential=None, flavour="parity"):
    """Run the reference.  Returns (psi tile as complex128 [dim_y, dim_x], Result)."""
    geo = geometry(cfg, flavour)
    shape = (geo.dim_y, geo.dim_x)
    re = np.zeros(shape, np.float64)
    im = np.zeros(shape, np.float64)
    if psi is not None:
        re[...] = np.real(psi)
        im[...] = np.imag(psi)
    pot = np.ascontiguousarray(potential if potential is not None else np.zeros(shape), np.float64)
    res = Result()
    rc = _lib(flavour).tsref_run(C.byref(cfg), re.ctypes.data, im.ctypes.data, pot.ctypes.data,
                                 C.byref(res))
    if rc != 0:
        raise RuntimeError(_lib(flavour).tsref_last_error().decode())
    return re + 1j * im, res


def run2(cfg, c2, psi_a, psi_b, pot_a, pot_b, flavour="parity"):
    """Two components (arrays and matrix potentials for both): returns
    (psi_a, psi_b, Result2)."""
    geo = geometry(cfg, flavour)
    shape = (geo.dim_y, geo.dim_x)
    arrs = []
    for psi in (psi_a, psi_b):
        re = np.ascontiguousarray(np.real(psi), np.float64).reshape(shape).copy()
        im = np.ascontiguousarray(np.imag(psi), np.float64).reshape(shape).copy()
        arrs += [re, im]
    va = np.ascontiguousarray(pot_a, np.float64)
    vb = np.ascontiguousarray(pot_b, np.float64)
    res = Result2()
    rc = _lib(flavour).tsref_run2(C.byref(cfg), C.byref(c2), *[a.ctypes.data for a in arrs],
                                  va.ctypes.data, vb.ctypes.data, C.byref(res))
    if rc != 0:
        raise RuntimeError(_lib(flavour).tsref_last_error().decode())
    return arrs[0] + 1j * arrs[1], arrs[2] + 1j * arrs[3], res


def write_state(cfg, psi, kind, name, flavour="parity"):
    """The reference writes the tile psi (kind 0 state, 1 density, 2 phase)."""
    re = np.ascontiguousarray(np.real(psi), np.float64).copy()
    im = np.ascontiguousarray(np.imag(psi), np.float64).copy()
    if _lib(flavour).tsref_state_io(C.byref(cfg), re.ctypes.data, im.ctypes.data, int(kind),
                                    str(name).encode(), 0) != 0:
        raise RuntimeError(_lib(flavour).tsref_last_error().decode())


def load_state(cfg, name, flavour="parity"):
    """The reference reads a state file into a fresh tile."""
    geo = geometry(cfg, flavour)
    re = np.zeros((geo.dim_y, geo.dim_x))
    im = np.zeros((geo.dim_y, geo.dim_x))
    if _lib(flavour).tsref_state_io(C.byref(cfg), re.ctypes.data, im.ctypes.data, 0,
                                    str(name).encode(), 1) != 0:
        raise RuntimeError(_lib(flavour).tsref_last_error().decode())
    return re + 1j * im

