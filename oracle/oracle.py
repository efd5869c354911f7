"""ctypes binding of the C restatement in oracle/ts_oracle.c (test infrastructure).

The restatement is the checker for the B200 kernels: tests/ and
__graft_entry__.smoke() call it on the same seeded inputs as the CUDA path,
bench.py times it as the CPU baseline when the compiled reference is absent.
Nothing in the product imports this module.

Geometry and set-up helpers below restate, in numpy with the same operation
order, the reference's lattice geometry (src/common.cpp:83-102,
src/model.cpp:103-158), coordinates (src/common.cpp:45-65), GaussianState
(src/model.cpp:692-714) and HarmonicPotential (src/model.cpp:920-926).
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libts_oracle.so")


class Params(C.Structure):
    _fields_ = [
        ("W", C.c_int), ("H", C.c_int),
        ("ix0", C.c_int), ("ix1", C.c_int), ("iy0", C.c_int), ("iy1", C.c_int),
        ("periodic_x", C.c_int), ("periodic_y", C.c_int),
        ("halo_x", C.c_int), ("halo_y", C.c_int),
        ("imag_time", C.c_int),
        ("aH", C.c_double), ("bH", C.c_double), ("aV", C.c_double), ("bV", C.c_double),
        ("coupling", C.c_double), ("lhy_coupling", C.c_double),
        ("alpha_x", C.c_double), ("alpha_y", C.c_double),
        ("rot_off_x", C.c_int), ("rot_off_y", C.c_int),
        ("delta_x", C.c_double), ("delta_y", C.c_double),
        ("norm0", C.c_double),
        ("cylindrical", C.c_int), ("kin_radial", C.c_double), ("mirror_sign", C.c_int),
    ]


class Geometry(C.Structure):
    _fields_ = [
        ("W", C.c_int), ("H", C.c_int), ("ix0", C.c_int), ("ix1", C.c_int),
        ("iy0", C.c_int), ("iy1", C.c_int),
        ("start_x", C.c_int), ("start_y", C.c_int),
        ("global_no_halo_dim_x", C.c_int), ("global_no_halo_dim_y", C.c_int),
        ("delta_x", C.c_double), ("delta_y", C.c_double),
        ("length_x", C.c_double), ("length_y", C.c_double),
        ("cylindrical", C.c_int),
    ]


class Energies(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("total", "kinetic", "potential", "rotational", "intra", "lhy", "norm2")]


class Expectations(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("norm2", "mean_x", "mean_xx", "mean_y", "mean_yy", "mean_px", "mean_pxpx",
                 "mean_py", "mean_pypy", "mean_lz")]


def build():
    """Compile the restatement (gcc, no FMA contraction)."""
    src = os.path.join(HERE, "ts_oracle.c")
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-std=c99",
                           src, "-o", tmp, "-lm"])
    os.replace(tmp, LIB_PATH)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.c_void_p
        L.tso_init_constants.argtypes = [C.POINTER(Params)] + [C.c_double] * 7
        L.tso_exp_table.argtypes = [C.c_int, C.c_double, dp, C.c_size_t, dp, dp]
        L.tso_full_step.argtypes = [C.POINTER(Params), dp, dp, dp, dp]
        L.tso_halo_exchange.argtypes = [C.POINTER(Params), dp, dp]
        L.tso_squared_norm.argtypes = [C.POINTER(Params), dp, dp]
        L.tso_squared_norm.restype = C.c_double
        L.tso_evolve.argtypes = [C.POINTER(Params), dp, dp, dp, dp, C.c_int]
        L.tso_energies.argtypes = [C.POINTER(Geometry), dp, dp, dp, C.c_double, C.c_double,
                                   C.c_double, C.c_double, C.POINTER(Energies)]
        L.tso_expectations.argtypes = [C.POINTER(Geometry), dp, dp, C.POINTER(Expectations)]
        L.tso_adjoint_real.argtypes = [C.POINTER(Params), dp, dp, C.c_double, dp, dp, C.c_int,
                                       dp, dp, dp, dp, dp]
        L.tso_adjoint_real.restype = C.c_int
        L.tso_adjoint_imag.argtypes = [C.POINTER(Params), dp, C.c_double, dp, dp, C.c_int,
                                       dp, dp, dp, dp, dp]
        L.tso_adjoint_imag.restype = C.c_int
        L.tso_full_step2.argtypes = [C.POINTER(Params), C.c_double, dp, dp, dp, dp, dp, dp]
        L.tso_rabi.argtypes = [C.POINTER(Params), C.c_double, C.c_double, C.c_double,
                               C.c_double, dp, dp, dp, dp]
        L.tso_evolve2.argtypes = [C.POINTER(Params), C.POINTER(Params)] + [C.c_double] * 4 + \
            [dp, C.c_double] + [dp] * 8 + [C.c_int, C.c_int]
        L.tso_evolve2.restype = C.c_int
        L.tso_cross_energies.argtypes = [C.POINTER(Geometry), dp, dp, dp, dp, C.c_double,
                                         C.c_double, C.c_double, dp, dp]
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# Reference geometry, restated (single process).
# --------------------------------------------------------------------------
def calculate_borders(length, halo, periodic):
    """src/common.cpp:83-102 with one process (coord 0, dim 1)."""
    inner = int(math.ceil(float(length) / 1.0))
    inner_start = 0
    start = inner_start - halo if periodic else 0
    end = inner_start + (inner + halo)
    if end > length:
        end = length + halo if periodic else length
    inner_end = end - halo if periodic else (end if end == length else end - halo)
    return start, end, inner_start, inner_end


class Lattice:
    """Geometry of a reference Lattice2D / Lattice1D tile (src/model.cpp:32-158)."""

    def __init__(self, dim_x, length_x, dim_y=None, length_y=None, periodic_x=False,
                 periodic_y=False, angular_velocity=0.0, one_d=False, cylindrical=False):
        """cylindrical: the radial axis is x (src/model.cpp:107-158): one more
        column (r = -dx/2, the mirror of r = dx/2), dx = L / (N + 1 - 0.5),
        the inner region starting at column 1."""
        if cylindrical:
            if periodic_x:
                raise ValueError("no periodic boundary on the radial axis")
            dim_x += 1
        self.cylindrical = bool(cylindrical)
        if one_d:
            dim_y, length_y = 1, 0.0
            self.delta_x = length_x / float(dim_x)
            self.delta_y = 1.0
            self.halo_x, self.halo_y = 4, 0
            periodic_y = False
        else:
            dim_y = (dim_x - (1 if cylindrical else 0)) if dim_y is None else dim_y
            length_y = length_x if length_y is None else length_y
            self.delta_x = (length_x / (float(dim_x) - 0.5) if cylindrical
                            else length_x / float(dim_x))
            self.delta_y = length_y / float(dim_y)
            self.halo_x = self.halo_y = 4 if angular_velocity == 0.0 else 8
        self.one_d = one_d
        self.length_x, self.length_y = length_x, length_y
        self.periodic_x, self.periodic_y = bool(periodic_x), bool(periodic_y)
        self.global_no_halo_dim_x, self.global_no_halo_dim_y = dim_x, dim_y
        self.start_x, self.end_x, self.inner_start_x, self.inner_end_x = calculate_borders(
            dim_x, self.halo_x, periodic_x)
        if one_d:
            self.start_y, self.end_y, self.inner_start_y, self.inner_end_y = 0, 1, 0, 1
        else:
            self.start_y, self.end_y, self.inner_start_y, self.inner_end_y = calculate_borders(
                dim_y, self.halo_y, periodic_y)
        if cylindrical:
            self.inner_start_x += 1
        self.dim_x = self.end_x - self.start_x
        self.dim_y = self.end_y - self.start_y

    @property
    def shape(self):
        return (self.dim_y, self.dim_x)

    def inner(self):
        return (self.inner_start_x - self.start_x, self.inner_end_x - self.start_x,
                self.inner_start_y - self.start_y, self.inner_end_y - self.start_y)

    def geometry(self):
        g = Geometry()
        g.W, g.H = self.dim_x, self.dim_y
        g.ix0, g.ix1, g.iy0, g.iy1 = self.inner()
        g.start_x, g.start_y = self.start_x, self.start_y
        g.global_no_halo_dim_x = self.global_no_halo_dim_x
        g.global_no_halo_dim_y = self.global_no_halo_dim_y
        g.delta_x, g.delta_y = self.delta_x, self.delta_y
        g.length_x, g.length_y = self.length_x, self.length_y
        g.cylindrical = int(self.cylindrical)
        return g

    def coordinates(self):
        """(x, y) arrays of shape (dim_y, dim_x), src/common.cpp:45-65."""
        xi = np.arange(self.dim_x, dtype=np.float64)
        yi = np.arange(self.dim_y, dtype=np.float64)
        if self.cylindrical:  # src/common.cpp:66-81
            idx = self.start_x * self.delta_x + xi * self.delta_x - 0.5 * self.delta_x
            idy = self.start_y * self.delta_y + 0.5 * self.delta_y + yi * self.delta_y
            y_c = self.global_no_halo_dim_y * self.delta_y * 0.5
            idy = np.where(idy - y_c < -self.length_y * 0.5, idy + self.length_y, idy)
            idy = np.where(idy - y_c > self.length_y * 0.5, idy - self.length_y, idy)
            X = np.broadcast_to(idx[None, :], self.shape)
            Y = np.broadcast_to((idy - y_c)[:, None], self.shape)
            return np.ascontiguousarray(X), np.ascontiguousarray(Y)
        idx = self.start_x * self.delta_x + 0.5 * self.delta_x + xi * self.delta_x
        idy = self.start_y * self.delta_y + 0.5 * self.delta_y + yi * self.delta_y
        x_c = self.global_no_halo_dim_x * self.delta_x * 0.5
        y_c = self.global_no_halo_dim_y * self.delta_y * 0.5
        idx = np.where(idx - x_c < -self.length_x * 0.5, idx + self.length_x, idx)
        idx = np.where(idx - x_c > self.length_x * 0.5, idx - self.length_x, idx)
        idy = np.where(idy - y_c < -self.length_y * 0.5, idy + self.length_y, idy)
        idy = np.where(idy - y_c > self.length_y * 0.5, idy - self.length_y, idy)
        X = np.broadcast_to((idx - x_c)[None, :], self.shape)
        Y = np.broadcast_to((idy - y_c)[:, None], self.shape)
        return np.ascontiguousarray(X), np.ascontiguousarray(Y)

    def azimuthal(self, angular_momentum, mass=1.0):
        """l^2 / (2 m r^2) over the tile (src/model.cpp:967-971), cylindrical."""
        X, _ = self.coordinates()
        return (angular_momentum * angular_momentum) / (2. * mass * X * X)

    def harmonic(self, omega_x, omega_y, mass=1.0, mean_x=0.0, mean_y=0.0):
        """HarmonicPotential::get_value over the tile (src/model.cpp:920-926)."""
        X, Y = self.coordinates()
        xr = X - mean_x
        yr = Y - mean_y
        return 0.5 * mass * (omega_x * omega_x * xr * xr + omega_y * omega_y * yr * yr)

    def params(self, delta_t, imag_time=False, mass=1.0, coupling=0.0, lhy=0.0,
               angular_velocity=0.0, rot_coord=(0.0, 0.0), norm0=0.0, angular_momentum=0):
        p = Params()
        p.W, p.H = self.dim_x, self.dim_y
        p.ix0, p.ix1, p.iy0, p.iy1 = self.inner()
        p.periodic_x, p.periodic_y = int(self.periodic_x), int(self.periodic_y)
        p.halo_x, p.halo_y = self.halo_x, self.halo_y
        p.imag_time = int(imag_time)
        lib().tso_init_constants(C.byref(p), delta_t, mass, coupling, lhy, angular_velocity,
                                 self.delta_x, self.delta_y)
        # Hamiltonian rotation centre in lattice units (src/model.cpp:950-956)
        rcx = (self.global_no_halo_dim_x) * 0.5 + rot_coord[0] / self.delta_x
        rcy = (self.global_no_halo_dim_y) * 0.5 + rot_coord[1] / self.delta_y
        p.rot_off_x = int(self.start_x - rcx)
        p.rot_off_y = int(self.start_y - rcy)
        p.norm0 = norm0
        if self.cylindrical:  # src/cpukernel.cpp:200-210,669-689
            p.cylindrical = 1
            p.kin_radial = delta_t / (8. * mass * self.delta_x * self.delta_x)
            p.mirror_sign = 1 if angular_momentum % 2 == 0 else -1
        return p


def _ptr(a):
    return a.ctypes.data


def exp_table(V, delta_t, imag_time):
    V = np.ascontiguousarray(V, np.float64)
    re = np.empty_like(V)
    im = np.empty_like(V)
    lib().tso_exp_table(int(imag_time), delta_t, _ptr(V), V.size, _ptr(re), _ptr(im))
    return re, im


def evolve(params, psi, pot_re, pot_im, iterations):
    """Evolve a tile in place semantics; returns the new complex tile."""
    re = np.ascontiguousarray(np.real(psi), np.float64).copy()
    im = np.ascontiguousarray(np.imag(psi), np.float64).copy()
    pr = np.ascontiguousarray(pot_re, np.float64)
    pi = np.ascontiguousarray(pot_im, np.float64)
    lib().tso_evolve(C.byref(params), _ptr(re), _ptr(im), _ptr(pr), _ptr(pi), int(iterations))
    return re + 1j * im


def _soa(psi):
    return (np.ascontiguousarray(np.real(psi), np.float64).copy(),
            np.ascontiguousarray(np.imag(psi), np.float64).copy())


def evolve2(pa, pb, coupling_ab, omega_r, omega_i, delta_t, psi_a, psi_b, table_a, table_b,
            iterations, norms=(0.0, 0.0), tot_norm=None, rabi_first_half=True):
    """`iterations` steps of the two-component loop (src/solver.cpp:172-230).
    pa.coupling / pb.coupling are g_a dt / g_b dt, coupling_ab is g_ab dt;
    norms are the per-component norms kept in imaginary time.  Returns
    (psi_a, psi_b, norms)."""
    ar, ai = _soa(psi_a)
    br, bi = _soa(psi_b)
    tar, tai = (np.ascontiguousarray(t, np.float64) for t in table_a)
    tbr, tbi = (np.ascontiguousarray(t, np.float64) for t in table_b)
    nrm = np.array(norms, np.float64)
    tot = float(nrm.sum()) if tot_norm is None else float(tot_norm)
    rc = lib().tso_evolve2(C.byref(pa), C.byref(pb), coupling_ab, omega_r, omega_i, delta_t,
                           _ptr(nrm), tot, _ptr(ar), _ptr(ai), _ptr(br), _ptr(bi), _ptr(tar),
                           _ptr(tai), _ptr(tbr), _ptr(tbi), int(iterations),
                           int(bool(rabi_first_half)))
    if rc != 0:
        raise MemoryError("tso_evolve2")
    return ar + 1j * ai, br + 1j * bi, (float(nrm[0]), float(nrm[1]))


def rabi(params, omega_r, omega_i, var, delta_t, psi_a, psi_b):
    ar, ai = _soa(psi_a)
    br, bi = _soa(psi_b)
    lib().tso_rabi(C.byref(params), omega_r, omega_i, var, delta_t, _ptr(ar), _ptr(ai), _ptr(br),
                   _ptr(bi))
    return ar + 1j * ai, br + 1j * bi


def cross_energies(lattice, psi_a, psi_b, coupling_ab, omega_r, omega_i):
    """(inter-species, Rabi) energies of src/solver.cpp:340-353,549-550."""
    ar, ai = _soa(psi_a)
    br, bi = _soa(psi_b)
    inter, rab = C.c_double(), C.c_double()
    g = lattice.geometry()
    lib().tso_cross_energies(C.byref(g), _ptr(ar), _ptr(ai), _ptr(br), _ptr(bi), coupling_ab,
                             omega_r, omega_i, C.byref(inter), C.byref(rab))
    return inter.value, rab.value


def squared_norm(params, psi):
    re = np.ascontiguousarray(np.real(psi), np.float64)
    im = np.ascontiguousarray(np.imag(psi), np.float64)
    return lib().tso_squared_norm(C.byref(params), _ptr(re), _ptr(im))


def energies(lattice, psi, V, mass=1.0, coupling=0.0, lhy=0.0, omega=0.0):
    re = np.ascontiguousarray(np.real(psi), np.float64)
    im = np.ascontiguousarray(np.imag(psi), np.float64)
    V = np.ascontiguousarray(V, np.float64)
    out = Energies()
    g = lattice.geometry()
    lib().tso_energies(C.byref(g), _ptr(re), _ptr(im), _ptr(V), mass, coupling, lhy, omega,
                       C.byref(out))
    return {n: getattr(out, n) for n, _ in Energies._fields_}


def expectations(lattice, psi):
    re = np.ascontiguousarray(np.real(psi), np.float64)
    im = np.ascontiguousarray(np.imag(psi), np.float64)
    out = Expectations()
    g = lattice.geometry()
    lib().tso_expectations(C.byref(g), _ptr(re), _ptr(im), C.byref(out))
    return {n: getattr(out, n) for n, _ in Expectations._fields_}


def gaussian(lattice, omega_x, omega_y=-1.0, mean_x=0.0, mean_y=0.0, norm=1.0, phase=0.0):
    """GaussianState values over the tile (src/model.cpp:692-714).

    std::pow(v, 2.0) is evaluated as v*v by glibc for an exact exponent of 2.
    """
    if omega_y == -1.0:
        omega_y = omega_x
    X, Y = lattice.coordinates()
    amp = math.sqrt(norm * math.sqrt(omega_x * omega_y) / math.pi)
    dx = X - mean_x
    dy = Y - mean_y
    val = amp * np.exp(-(omega_x * (dx * dx) + omega_y * (dy * dy)) * 0.5)
    return val * complex(math.cos(phase), math.sin(phase))


def exponential(lattice, n_x=1, n_y=1, norm=1.0, phase=0.0):
    """ExponentialState values over the tile (src/model.cpp:653-672)."""
    X, Y = lattice.coordinates()
    lx = lattice.global_no_halo_dim_x * lattice.delta_x
    ly = lattice.global_no_halo_dim_y * lattice.delta_y
    amp = math.sqrt(norm / (lx * ly)) * complex(math.cos(phase), math.sin(phase))
    arg = 2 * math.pi * float(n_x) / lx * X + 2 * math.pi * float(n_y) / ly * Y
    return amp * (np.cos(arg) + 1j * np.sin(arg))


def adjoint_real(p, tab_re, tab_im, delta_t, psi0, steps, lam_t):
    """Reverse mode of `steps` closed real-time steps (CPU FP64 check of the B200
    adjoint; oracle/ts_oracle.c tso_adjoint_real).  lam_t = dL/dre + i dL/dim at
    psi(T); returns (dL/dV, dL/dpsi0) with the same convention."""
    shape = (p.H, p.W)
    a = lambda z: np.ascontiguousarray(z, np.float64)
    r0, i0 = a(np.real(psi0)), a(np.imag(psi0))
    lr, li = a(np.real(lam_t)), a(np.imag(lam_t))
    tr, ti = a(tab_re), a(tab_im)
    gv = np.zeros(shape)
    gr = np.zeros(shape)
    gi = np.zeros(shape)
    rc = lib().tso_adjoint_real(C.byref(p), tr.ctypes.data, ti.ctypes.data, float(delta_t),
                                r0.ctypes.data, i0.ctypes.data, int(steps), lr.ctypes.data,
                                li.ctypes.data, gv.ctypes.data, gr.ctypes.data, gi.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"tso_adjoint_real: status {rc}")
    return gv, gr + 1j * gi


def adjoint_imag(p, tab_re, delta_t, psi0, steps, lam_t):
    """Reverse mode of `steps` closed imaginary-time steps with renormalisation
    to norm0 = N(psi0) (CPU FP64 check of the B200 imaginary-time adjoint;
    oracle/ts_oracle.c tso_adjoint_imag).  lam_t = dL/dre + i dL/dim at psi(T);
    returns (dL/dV, dL/dpsi0)."""
    shape = (p.H, p.W)
    a = lambda z: np.ascontiguousarray(z, np.float64)
    r0, i0 = a(np.real(psi0)), a(np.imag(psi0))
    lr, li = a(np.real(lam_t)), a(np.imag(lam_t))
    tr = a(tab_re)
    gv = np.zeros(shape)
    gr = np.zeros(shape)
    gi = np.zeros(shape)
    rc = lib().tso_adjoint_imag(C.byref(p), tr.ctypes.data, float(delta_t), r0.ctypes.data,
                                i0.ctypes.data, int(steps), lr.ctypes.data, li.ctypes.data,
                                gv.ctypes.data, gr.ctypes.data, gi.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"tso_adjoint_imag: status {rc}")
    return gv, gr + 1j * gi
