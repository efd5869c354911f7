"""Python API mirroring the reference's `trottersuzuki` package.

Same class and method names as trotter-suzuki-mpi 1.6.2's Python binding
(src/Python/trottersuzuki/__init__.py:8-19, classes_extension.py:14-403),
backed by the C++ host layer (include/ts_host.h) and the B200 kernel.

    import trottersuzuki_b200 as ts
    grid = ts.Lattice2D(256, 20.)
    state = ts.GaussianState(grid, 1., mean_x=1.)
    pot = ts.HarmonicPotential(grid, 1., 1.)
    ham = ts.Hamiltonian(grid, pot)
    solver = ts.Solver(grid, state, ham, 1e-4)      # kernel_type="gpu"
    solver.evolve(1000)
    print(solver.get_total_energy())

kernel_type "gpu" (or "b200") stores psi in FP64; "gpu_fp32" stores psi and
the exponential table in FP32 (norms and energies stay FP64).
"""
import ctypes as C
import inspect
import os

import numpy as np

from . import _capi

HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB_PATH = os.path.join(HERE, "libtrottersuzuki_b200.so")


class _Info(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "dim_x", "dim_y", "global_no_halo_dim_x", "global_no_halo_dim_y", "start_x", "start_y",
        "end_x", "end_y", "inner_start_x", "inner_start_y", "inner_end_x", "inner_end_y",
        "halo_x", "halo_y", "periodic_x", "periodic_y")] + [
        (n, C.c_double) for n in ("length_x", "length_y", "delta_x", "delta_y")]


_host = None


def host():
    """Load the C++ host layer (it loads libtsb200.so); raise if not built."""
    global _host
    if _host is None:
        _capi.lib()  # the CUDA library first, with its own error message
        if not os.path.exists(HOST_LIB_PATH):
            raise ImportError(f"{HOST_LIB_PATH} is missing: build the extension first")
        L = C.CDLL(HOST_LIB_PATH)
        vp, d, i = C.c_void_p, C.c_double, C.c_int
        P = C.POINTER
        sig = {
            "tsh_last_error": (C.c_char_p, []),
            "tsh_lattice2d_new": (i, [i, d, i, d, i, i, d, P(vp)]),
            "tsh_lattice1d_new": (i, [i, d, i, P(vp)]),
            "tsh_lattice2d_new_cs": (i, [i, d, i, d, i, i, d, C.c_char_p, P(vp)]),
            "tsh_lattice1d_new_cs": (i, [i, d, i, C.c_char_p, P(vp)]),
            "tsh_state_new_l": (i, [vp, i, P(vp)]),
            "tsh_state_write": (i, [vp, i, C.c_char_p]),
            "tsh_state_loadtxt": (i, [vp, C.c_char_p]),
            "tsh_lattice_info_get": (i, [vp, P(_Info)]),
            "tsh_lattice_free": (i, [vp]),
            "tsh_state_new": (i, [vp, P(vp)]),
            "tsh_gaussian_state_new": (i, [vp, d, d, d, d, d, d, P(vp)]),
            "tsh_exponential_state_new": (i, [vp, i, i, d, d, P(vp)]),
            "tsh_sinusoid_state_new": (i, [vp, i, i, d, d, P(vp)]),
            "tsh_state_arrays": (i, [vp, P(P(d)), P(P(d))]),
            "tsh_state_touch": (i, [vp]),
            "tsh_state_expectations": (i, [vp, P(d)]),
            "tsh_state_free": (i, [vp]),
            "tsh_potential_matrix_new": (i, [vp, vp, P(vp)]),
            "tsh_harmonic_potential_new": (i, [vp, d, d, d, d, d, P(vp)]),
            "tsh_potential_free": (i, [vp]),
            "tsh_hamiltonian_new": (i, [vp, vp, d, d, d, d, d, d, P(vp)]),
            "tsh_hamiltonian_free": (i, [vp]),
            "tsh_solver_new": (i, [vp, vp, vp, d, C.c_char_p, P(vp)]),
            "tsh_solver2_new": (i, [vp, vp, vp, vp, d, C.c_char_p, P(vp)]),
            "tsh_solver_energies2": (i, [vp, P(d)]),
            "tsh_hamiltonian2_new": (i, [vp, vp, vp] + [d] * 10 + [P(vp)]),
            "tsh_solver_evolve": (i, [vp, i, i]),
            "tsh_solver_prepare": (i, [vp, i]),
            "tsh_solver_energies": (i, [vp, P(d)]),
            "tsh_solver_set_exp_potential": (i, [vp, vp, vp, i, i]),
            "tsh_solver_update_parameters": (i, [vp]),
            "tsh_solver_kernel_handle": (i, [vp, P(vp)]),
            "tsh_solver_free": (i, [vp]),
            "tsh_make_desc": (i, [vp, vp, d, d, i, i, P(_capi.Desc)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _host = L
    return _host


def _chk(rc):
    if rc != 0:
        # the reference raises std::runtime_error through my_abort
        raise RuntimeError(host().tsh_last_error().decode())


def _new(fn, *args):
    out = C.c_void_p()
    _chk(fn(*args, C.byref(out)))
    return out


class _Handle:
    _free = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and self._free and host is not None:
            try:
                getattr(host(), self._free)(h)
            except Exception:
                pass


# ---------------------------------------------------------------- lattices
class Lattice(_Handle):
    _free = "tsh_lattice_free"

    def _load(self):
        info = _Info()
        _chk(host().tsh_lattice_info_get(self._h, C.byref(info)))
        for name, _ in _Info._fields_:
            setattr(self, name, getattr(info, name))
        self.periods = [self.periodic_y, self.periodic_x]

    def get_x_axis(self):
        """Cell-centred x coordinates of the lattice (no halo)."""
        return (np.arange(self.global_no_halo_dim_x) - self.global_no_halo_dim_x * 0.5 + 0.5) \
            * self.delta_x

    def get_y_axis(self):
        return (np.arange(self.global_no_halo_dim_y) - self.global_no_halo_dim_y * 0.5 + 0.5) \
            * self.delta_y


class Lattice1D(Lattice):
    def __init__(self, dim_x, length_x, periodic_x_axis=False, coordinate_system="cartesian"):
        self._h = _new(host().tsh_lattice1d_new_cs, int(dim_x), float(length_x),
                       int(bool(periodic_x_axis)), coordinate_system.encode())
        self.coordinate_system = coordinate_system
        self._load()


class Lattice2D(Lattice):
    def __init__(self, dim_x, length_x, dim_y=None, length_y=None, periodic_x_axis=False,
                 periodic_y_axis=False, angular_velocity=0., coordinate_system="cartesian"):
        dim_y = dim_x if dim_y is None else dim_y
        length_y = length_x if length_y is None else length_y
        self._h = _new(host().tsh_lattice2d_new_cs, int(dim_x), float(length_x), int(dim_y),
                       float(length_y), int(bool(periodic_x_axis)), int(bool(periodic_y_axis)),
                       float(angular_velocity), coordinate_system.encode())
        self.coordinate_system = coordinate_system
        self._load()


def map_lattice_to_coordinate_space(grid, x, y=0):
    """Cell-centre coordinates of tile cell (x, y) (src/common.cpp:45-81); on a
    cylindrical lattice x is the radius, -dx/2 at column 0."""
    if getattr(grid, "coordinate_system", "cartesian") == "cylindrical":
        idy = grid.start_y * grid.delta_y + 0.5 * grid.delta_y + y * grid.delta_y
        y_c = grid.global_no_halo_dim_y * grid.delta_y * 0.5
        if idy - y_c < -grid.length_y * 0.5:
            idy += grid.length_y
        if idy - y_c > grid.length_y * 0.5:
            idy -= grid.length_y
        return grid.start_x * grid.delta_x + x * grid.delta_x - 0.5 * grid.delta_x, idy - y_c
    idx = grid.start_x * grid.delta_x + 0.5 * grid.delta_x + x * grid.delta_x
    x_c = grid.global_no_halo_dim_x * grid.delta_x * 0.5
    if idx - x_c < -grid.length_x * 0.5:
        idx += grid.length_x
    if idx - x_c > grid.length_x * 0.5:
        idx -= grid.length_x
    idy = grid.start_y * grid.delta_y + 0.5 * grid.delta_y + y * grid.delta_y
    y_c = grid.global_no_halo_dim_y * grid.delta_y * 0.5
    if idy - y_c < -grid.length_y * 0.5:
        idy += grid.length_y
    if idy - y_c > grid.length_y * 0.5:
        idy -= grid.length_y
    return idx - x_c, idy - y_c


def _coordinate_grid(grid):
    xs = np.array([map_lattice_to_coordinate_space(grid, x, 0)[0] for x in range(grid.dim_x)])
    ys = np.array([map_lattice_to_coordinate_space(grid, 0, y)[1] for y in range(grid.dim_y)])
    return np.broadcast_to(xs[None, :], (grid.dim_y, grid.dim_x)), \
        np.broadcast_to(ys[:, None], (grid.dim_y, grid.dim_x))


def _eval_on_grid(grid, fn, nargs_extra=()):
    """Evaluate fn(x, y, *extra) (or fn(x) on a 1D lattice) on every tile cell."""
    X, Y = _coordinate_grid(grid)
    try:
        nparam = len(inspect.signature(fn).parameters)
    except (TypeError, ValueError):
        nparam = 2
    args = (X,) if nparam == 1 else (X, Y) + tuple(nargs_extra)
    try:
        v = np.asarray(fn(*args))
        if v.shape == X.shape:
            return v
    except Exception:
        pass
    out = np.empty(X.shape, dtype=np.result_type(fn(*(a[0, 0] for a in args[:2]),
                                                    *args[2:]), np.float64))
    for j in range(X.shape[0]):
        for i in range(X.shape[1]):
            out[j, i] = fn(*(a[j, i] for a in args[:2]), *args[2:]) if nparam != 1 \
                else fn(X[j, i])
    return out


# ------------------------------------------------------------------- states
class State(_Handle):
    _free = "tsh_state_free"

    def __init__(self, grid, angular_momentum=0):
        self.grid = grid
        self.angular_momentum = angular_momentum
        self._h = _new(host().tsh_state_new_l, grid._h, int(angular_momentum))

    def _arrays(self):
        re = C.POINTER(C.c_double)()
        im = C.POINTER(C.c_double)()
        _chk(host().tsh_state_arrays(self._h, C.byref(re), C.byref(im)))
        shape = (self.grid.dim_y, self.grid.dim_x)
        return (np.ctypeslib.as_array(re, shape=shape), np.ctypeslib.as_array(im, shape=shape))

    @property
    def p_real(self):
        """Real part of the tile (a view into the C++ State)."""
        return self._arrays()[0]

    @property
    def p_imag(self):
        return self._arrays()[1]

    def get_state(self):
        """The tile as a complex128 array of shape (dim_y, dim_x)."""
        re, im = self._arrays()
        return re + 1j * im

    def init_state_matrix(self, real, imag):
        re, im = self._arrays()
        re[...] = np.asarray(real, np.float64).reshape(re.shape)
        im[...] = np.asarray(imag, np.float64).reshape(im.shape)
        _chk(host().tsh_state_touch(self._h))

    def init_state(self, state_function):
        v = _eval_on_grid(self.grid, state_function).astype(np.complex128)
        self.init_state_matrix(v.real, v.imag)

    def imprint(self, function):
        v = _eval_on_grid(self.grid, function).astype(np.complex128)
        psi = self.get_state() * v
        self.init_state_matrix(psi.real, psi.imag)

    def _inner(self, a):
        g = self.grid
        return a[g.inner_start_y - g.start_y:g.inner_end_y - g.start_y,
                 g.inner_start_x - g.start_x:g.inner_end_x - g.start_x]

    def write_to_file(self, filename):
        """The state as text, "(re,im) " per cell (src/model.cpp:636-638)."""
        _chk(host().tsh_state_write(self._h, 0, str(filename).encode()))

    def write_particle_density(self, fileprefix):
        _chk(host().tsh_state_write(self._h, 1, str(fileprefix).encode()))

    def write_phase(self, fileprefix):
        _chk(host().tsh_state_write(self._h, 2, str(fileprefix).encode()))

    def loadtxt(self, filename):
        """Read a state written by write_to_file (src/model.cpp:254-322)."""
        _chk(host().tsh_state_loadtxt(self._h, str(filename).encode()))
        _chk(host().tsh_state_touch(self._h))

    def get_particle_density(self):
        re, im = self._arrays()
        return self._inner(re * re + im * im)

    def get_phase(self):
        re, im = self._arrays()
        n = np.sqrt(re * re + im * im)
        with np.errstate(invalid="ignore", divide="ignore"):
            ph = np.where(n == 0, 0.0, np.arccos(np.where(n == 0, 1.0, re / n))
                          * ((im >= 0).astype(float) - (im < 0).astype(float)))
        return self._inner(ph)

    def _expect(self):
        out = (C.c_double * 10)()
        _chk(host().tsh_state_expectations(self._h, out))
        return list(out)

    def get_squared_norm(self):
        return self._expect()[0]

    def get_mean_x(self):
        return self._expect()[1]

    def get_mean_xx(self):
        return self._expect()[2]

    def get_mean_y(self):
        return self._expect()[3]

    def get_mean_yy(self):
        return self._expect()[4]

    def get_mean_px(self):
        return self._expect()[5]

    def get_mean_pxpx(self):
        return self._expect()[6]

    def get_mean_py(self):
        return self._expect()[7]

    def get_mean_pypy(self):
        return self._expect()[8]

    def get_mean_angular_momentum(self):
        return self._expect()[9]

    def get_expected_value(self, operator):
        names = {"X": 1, "X^2": 2, "Y": 3, "Y^2": 4, "P_x": 5, "P_x^2": 6, "P_y": 7,
                 "P_y^2": 8, "L_z": 9}
        if operator not in names:
            return float("nan")
        return self._expect()[names[operator]]


class GaussianState(State):
    def __init__(self, grid, omega_x, omega_y=-1., mean_x=0., mean_y=0., norm=1., phase=0.):
        self.grid = grid
        self.angular_momentum = 0
        self._h = _new(host().tsh_gaussian_state_new, grid._h, float(omega_x), float(omega_y),
                       float(mean_x), float(mean_y), float(norm), float(phase))


class ExponentialState(State):
    def __init__(self, grid, n_x=1, n_y=1, norm=1., phase=0.):
        self.grid = grid
        self.angular_momentum = 0
        self._h = _new(host().tsh_exponential_state_new, grid._h, int(n_x), int(n_y),
                       float(norm), float(phase))


class SinusoidState(State):
    def __init__(self, grid, n_x=1, n_y=1, norm=1., phase=0.):
        self.grid = grid
        self.angular_momentum = 0
        self._h = _new(host().tsh_sinusoid_state_new, grid._h, int(n_x), int(n_y),
                       float(norm), float(phase))


# --------------------------------------------------------------- potentials
class Potential(_Handle):
    """External potential given as a matrix or a function V(x, y) / V(x, y, t)."""
    _free = "tsh_potential_free"

    def __init__(self, grid, matrix=None):
        self.grid = grid
        self.updated_potential_matrix = False
        self.pot_function = None
        self.init_potential_matrix(np.zeros((grid.dim_y, grid.dim_x)) if matrix is None
                                   else matrix)

    def init_potential_matrix(self, matrix):
        m = np.ascontiguousarray(matrix, np.float64).reshape(self.grid.dim_y, self.grid.dim_x)
        old = getattr(self, "_h", None)
        self._h = _new(host().tsh_potential_matrix_new, self.grid._h, m.ctypes.data)
        if old:
            host().tsh_potential_free(old)
        self.potential_matrix = m

    def init_potential(self, pot_function):
        try:
            nparam = len(inspect.signature(pot_function).parameters)
        except (TypeError, ValueError):
            nparam = 2
        if nparam == 3:
            self.updated_potential_matrix = True
            self.pot_function = pot_function
            self.init_potential_matrix(_eval_on_grid(self.grid, pot_function, (0.0,)))
        else:
            self.init_potential_matrix(_eval_on_grid(self.grid, pot_function))

    def exponential_update(self, delta_t, t):
        """exp(-i dt V(x, y, t)) over the tile (classes_extension.py:360-366)."""
        V = _eval_on_grid(self.grid, self.pot_function, (t,))
        return np.exp(-1j * delta_t * V)


class DevicePotential(Potential):
    """A time-dependent potential V(x, y, t) evaluated on the GPU.

    No counterpart in the reference, where a Python V(x, y, t) is tabulated
    on the host and uploaded before every step (classes_extension.py:360-366,
    388-403).  Here pot_function(X, Y, t) receives the tile's coordinates
    (the points of map_lattice_to_coordinate_space) as float64 CUDA tensors,
    X a 1 x dim_x row and Y a dim_y x 1 column that broadcast against each
    other, and a Python float t; it returns V as a tensor broadcastable to
    dim_y x dim_x.  Broadcast coordinates keep the terms that depend on x or
    on y alone as vectors, so only the final combination costs a pass over
    the tile.  The exponential table is
    then built on the device (ts_b200_set_potential_device), so a real-time
    step moves nothing between host and device.  The time schedule is the
    reference's: step i of an evolve() call uses V(t0 + i dt).  As in the
    reference, energies use V at t = 0 and imaginary-time evolution uses
    V(x, y, 0) throughout.

    time_batch = B > 0 evaluates B steps' potentials in one call: t is then
    a B x 1 x 1 float64 CUDA tensor of step times (write pot_function with
    torch operations, e.g. torch.sin(t)), the result is B x dim_y x dim_x,
    and the B steps run from one library call (ts_b200_evolve_potentials),
    which takes the per-step Python work off the critical path.  B tiles
    of doubles are held on the device meanwhile.
    """

    def __init__(self, grid, pot_function, device="cuda", time_batch=0):
        import torch
        self.grid = grid
        self.pot_function = pot_function
        self.time_batch = int(time_batch)
        self.updated_potential_matrix = True
        X, Y = _coordinate_grid(grid)
        self._X = torch.tensor(np.ascontiguousarray(X[:1, :]), dtype=torch.float64,
                               device=device)
        self._Y = torch.tensor(np.ascontiguousarray(Y[:, :1]), dtype=torch.float64,
                               device=device)
        self.shape = (grid.dim_y, grid.dim_x)
        self.init_potential_matrix(self.device_values(0.0).cpu().numpy())

    def device_values(self, t):
        """V(x, y, t) over the tile: a contiguous dim_y x dim_x float64 tensor
        on the device."""
        if self.time_batch:
            return self.device_values_batch([float(t)])[0]
        import torch
        v = torch.as_tensor(self.pot_function(self._X, self._Y, float(t)),
                            dtype=torch.float64, device=self._X.device)
        return v.expand(self.shape).contiguous()

    def device_values_batch(self, times):
        """V at each of `times` (time_batch mode): len(times) x dim_y x dim_x."""
        import torch
        # from pinned memory, so the copy does not wait for the queued steps
        tt = torch.tensor(times, dtype=torch.float64).pin_memory().to(self._X.device,
                                                                       non_blocking=True)
        v = torch.as_tensor(self.pot_function(self._X, self._Y, tt.view(-1, 1, 1)),
                            dtype=torch.float64, device=self._X.device)
        return v.expand((len(times),) + self.shape).contiguous()

    def exponential_update(self, delta_t, t):
        return np.exp(-1j * delta_t * self.device_values(t).cpu().numpy())


class HarmonicPotential(Potential):
    def __init__(self, grid, omegax, omegay, mass=1., mean_x=0., mean_y=0.):
        self.grid = grid
        self.updated_potential_matrix = False
        self.pot_function = None
        self._h = _new(host().tsh_harmonic_potential_new, grid._h, float(omegax),
                       float(omegay), float(mass), float(mean_x), float(mean_y))


class Hamiltonian(_Handle):
    _free = "tsh_hamiltonian_free"

    def __init__(self, grid, potential=None, mass=1., coupling_a=0., LeeHuangYang_coupling_a=0.,
                 angular_velocity=0., rot_coord_x=0., rot_coord_y=0.):
        self.grid = grid
        self.potential = potential
        self.mass = mass
        self.coupling_a = coupling_a
        self.LeeHuangYang_coupling_a = LeeHuangYang_coupling_a
        self.angular_velocity = angular_velocity
        self._h = _new(host().tsh_hamiltonian_new, grid._h,
                       potential._h if potential is not None else None, float(mass),
                       float(coupling_a), float(LeeHuangYang_coupling_a),
                       float(angular_velocity), float(rot_coord_x), float(rot_coord_y))


class Hamiltonian2Component(Hamiltonian):
    """Two species (src/trottersuzuki.h:455-497): masses, intra-species
    couplings g_a and g_b, inter-species g_ab and the Rabi coupling
    omega = omega_r + i omega_i; potential_b defaults to potential."""

    def __init__(self, grid, potential=None, potential_b=None, mass=1., mass_b=1.,
                 coupling_a=0., coupling_ab=0., coupling_b=0., omega_r=0., omega_i=0.,
                 angular_velocity=0., rot_coord_x=0., rot_coord_y=0.):
        self.grid = grid
        self.potential = potential
        self.potential_b = potential_b if potential_b is not None else potential
        self.mass, self.mass_b = mass, mass_b
        self.coupling_a, self.coupling_ab, self.coupling_b = coupling_a, coupling_ab, coupling_b
        self.omega_r, self.omega_i = omega_r, omega_i
        self.LeeHuangYang_coupling_a = 0.
        self.angular_velocity = angular_velocity
        self._h = _new(host().tsh_hamiltonian2_new, grid._h,
                       potential._h if potential is not None else None,
                       potential_b._h if potential_b is not None else None, float(mass),
                       float(mass_b), float(coupling_a), float(coupling_ab), float(coupling_b),
                       float(omega_r), float(omega_i), float(angular_velocity),
                       float(rot_coord_x), float(rot_coord_y))


# ------------------------------------------------------------------ solver
class Solver(_Handle):
    _free = "tsh_solver_free"

    def __init__(self, Lattice, State, Hamiltonian, delta_t, Potential=None, State2=None,
                 Potential2=None, kernel_type="gpu"):
        self.grid, self.state, self.hamiltonian = Lattice, State, Hamiltonian
        self.state2 = State2
        self.delta_t = delta_t
        self.potential = Potential if Potential is not None else Hamiltonian.potential
        self.kernel_type = kernel_type
        self.current_evolution_time = 0.0
        if State2 is None:
            self._h = _new(host().tsh_solver_new, Lattice._h, State._h, Hamiltonian._h,
                           float(delta_t), kernel_type.encode())
        else:
            if not isinstance(Hamiltonian, Hamiltonian2Component):
                raise RuntimeError("two states need a Hamiltonian2Component")
            self.potential2 = Potential2 if Potential2 is not None else self.potential
            self._h = _new(host().tsh_solver2_new, Lattice._h, State._h, State2._h,
                           Hamiltonian._h, float(delta_t), kernel_type.encode())

    def evolve(self, iterations, imag_time=False):
        pot = self.potential
        if self.state2 is not None:
            # two components: time-dependent potentials are re-tabulated by the
            # C++ Solver (src/solver.cpp:186-199)
            _chk(host().tsh_solver_evolve(self._h, int(iterations), int(bool(imag_time))))
            self.current_evolution_time += self.delta_t * abs(int(iterations))
            return
        if pot is None or not getattr(pot, "updated_potential_matrix", False) or imag_time:
            _chk(host().tsh_solver_evolve(self._h, int(iterations), int(bool(imag_time))))
            self.current_evolution_time += self.delta_t * abs(int(iterations))
            return
        # time-dependent Python potential: re-tabulate before every step
        # (classes_extension.py:388-403); iterations < 0 leaves the result
        # on the device, as the C++ evolve does
        n, copy_back = abs(int(iterations)), int(iterations) > 0
        if isinstance(pot, DevicePotential):
            self._evolve_device_potential(pot, n, copy_back)
            return
        for i in range(n):
            e = pot.exponential_update(self.delta_t, self.current_evolution_time)
            re = np.ascontiguousarray(e.real).ravel()
            im = np.ascontiguousarray(e.imag).ravel()
            _chk(host().tsh_solver_set_exp_potential(self._h, re.ctypes.data, im.ctypes.data,
                                                     re.size, 0))
            last = i == n - 1 and copy_back
            _chk(host().tsh_solver_evolve(self._h, 1 if last else -1, 0))
            self.current_evolution_time += self.delta_t

    def _evolve_device_potential(self, pot, iterations, copy_back=True):
        """The loop above with V(x, y, t) and its table made on the device:
        per step (or per time_batch steps), pot_function on a side stream,
        then the table kernel and one step per potential (no halo refresh, as
        each per-step evolve call of the reference loop ends its own
        iterations)."""
        import torch
        if iterations <= 0:
            return
        _chk(host().tsh_solver_prepare(self._h, 0))
        k = self.kernel_handle()
        lib = _capi.lib()
        # one side stream per solver, so the caching allocator reuses the
        # potential buffers of earlier calls
        stream = getattr(self, "_potential_stream", None)
        if stream is None or stream.device != pot._X.device:
            stream = self._potential_stream = torch.cuda.Stream(device=pot._X.device)
        stream.wait_stream(torch.cuda.current_stream(pot._X.device))
        _capi.check(lib.ts_b200_set_stream(k, C.c_void_p(stream.cuda_stream)), k)
        dt = float(self.delta_t)
        try:
            with torch.cuda.stream(stream):
                done = 0
                while done < iterations:
                    # the host path's times: t advanced by repeated addition
                    b = min(max(pot.time_batch, 1), iterations - done)
                    times = []
                    for _ in range(b):
                        times.append(self.current_evolution_time)
                        self.current_evolution_time += dt
                    if pot.time_batch:
                        V = pot.device_values_batch(times)
                    else:
                        V = pot.device_values(times[0])
                    W = V.shape[-1]
                    _capi.check(lib.ts_b200_evolve_potentials(
                        k, C.c_void_p(V.data_ptr()), W, W * V.shape[-2], b, dt, 0), k)
                    done += b
            stream.synchronize()
        finally:
            lib.ts_b200_set_stream(k, None)
        if copy_back:
            _chk(host().tsh_solver_evolve(self._h, 0, 0))  # copies the tile into the State

    def update_parameters(self):
        _chk(host().tsh_solver_update_parameters(self._h))

    def _energies(self):
        out = (C.c_double * 7)()
        _chk(host().tsh_solver_energies(self._h, out))
        return list(out)

    def _energies2(self):
        out = (C.c_double * 13)()
        _chk(host().tsh_solver_energies2(self._h, out))
        return list(out)

    def _pick(self, which, single_index, first):
        """which: 1 first species, 2 second, 3 total (src/solver.cpp:572-594)."""
        if self.state2 is None:
            if which == 2:
                print("The system has only one component. No input have to be given")
                return 0.0
            return self._energies()[single_index]
        e = self._energies2()
        a, b = e[first], e[first + 1]
        return {1: a, 2: b, 3: a + b}.get(int(which), 0.0)

    def get_total_energy(self):
        return self._energies2()[0] if self.state2 is not None else self._energies()[0]

    def get_kinetic_energy(self, which=3):
        return self._pick(which, 1, 1)

    def get_potential_energy(self, which=3):
        return self._pick(which, 2, 3)

    def get_rotational_energy(self, which=3):
        return self._pick(which, 3, 5)

    def get_intra_species_energy(self, which=3):
        return self._pick(which, 4, 7)

    def get_LeeHuangYang_energy(self):
        return 0.0 if self.state2 is not None else self._energies()[5]

    def get_inter_species_energy(self):
        if self.state2 is None:
            print("The system has only one component")
            return 0.0
        return self._energies2()[9]

    def get_rabi_energy(self):
        if self.state2 is None:
            print("The system has only one component")
            return 0.0
        return self._energies2()[10]

    def get_squared_norm(self, which=3):
        return self._pick(which, 6, 11)

    def kernel_handle(self):
        """The C-ABI handle (ts_b200_kernel*) of the current kernel, or None."""
        out = C.c_void_p()
        _chk(host().tsh_solver_kernel_handle(self._h, C.byref(out)))
        return out.value


def make_desc(grid, hamiltonian, delta_t, imag_time=False, norm=0.0, precision=0):
    """The C-ABI step descriptor (include/ts_b200.h) of a lattice and Hamiltonian,
    with the reference CPUBlock's constants (src/cpukernel.cpp:172-272)."""
    out = _capi.Desc()
    _chk(host().tsh_make_desc(grid._h, hamiltonian._h, float(delta_t), float(norm),
                              int(bool(imag_time)), int(precision), C.byref(out)))
    return out


class SolverBatch:
    """Evolve many Solvers together: one persistent launch per Trotter step.

    No counterpart in the reference, where each Solver evolves on its own; a
    loop of solver.evolve(T) calls becomes SolverBatch(solvers).evolve(T).
    The solvers must share kernel_type and have no rotating frame and no
    time-dependent potential.  Each solver's kernel is built (or rebuilt for
    the time mode) here, from its current State; evolve() leaves the results
    in the solvers' States, as Solver.evolve does.
    """

    def __init__(self, solvers, imag_time=False):
        from .kernel import Batch
        self.solvers = list(solvers)
        self.imag_time = bool(imag_time)
        for s in self.solvers:
            s.evolve(0, self.imag_time)  # (re)builds the kernel from the State, no step
        self.batch = Batch([s.kernel_handle() for s in self.solvers])

    def autotune(self, trial_steps=3, use_cache=True):
        return self.batch.autotune(trial_steps, use_cache)

    def evolve(self, iterations, copy_back=True):
        """iterations Trotter steps of every solver; with copy_back the States
        receive the results (else they stay on the device until the next
        Solver call that reads them)."""
        n = int(iterations)
        self.batch.evolve(n)
        for s in self.solvers:
            s.current_evolution_time += s.delta_t * n
            if copy_back:
                s.evolve(0, self.imag_time)  # copies the tile back into the State
        if not copy_back:
            self.batch.synchronize()

    def close(self):
        self.batch.close()
