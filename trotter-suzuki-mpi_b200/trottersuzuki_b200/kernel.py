"""Python handle over the C ABI: one B200 kernel per lattice tile.

This is the low-level object the Python Solver uses, the analogue of the
reference's ITrotterKernel (src/trottersuzuki.h:502-520).  Host arrays are
numpy complex128 tiles of shape (dim_y, dim_x) in the reference's tile layout.
"""
import ctypes as C

import numpy as np

from . import _capi
from ._capi import Desc, EnergyParams, EnergyResult, ExpectationResult, LaunchShape, check, lib

FP64 = _capi.FP64
FP32 = _capi.FP32


def _soa(psi):
    re = np.ascontiguousarray(np.real(psi), dtype=np.float64)
    im = np.ascontiguousarray(np.imag(psi), dtype=np.float64)
    return re, im


def _torch_stream():
    """torch's current CUDA stream (a cudaStream_t address) when torch is in
    use with CUDA initialised, else None."""
    import sys
    torch = sys.modules.get("torch")
    if torch is None or not torch.cuda.is_initialized():
        return None
    return torch.cuda.current_stream().cuda_stream


class Kernel:
    """A tile resident on the GPU plus its exponential table.

    desc: a _capi.Desc with the tile geometry and the step constants.
    """

    def __init__(self, desc):
        self.desc = desc
        self._h = C.c_void_p()
        check(lib().ts_b200_create(C.byref(desc), C.byref(self._h)))
        self.shape = (desc.dim_y, desc.dim_x)

    # -- lifetime -------------------------------------------------------
    def close(self):
        if self._h:
            lib().ts_b200_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def _check(self, status):
        check(status, self._h)

    # -- data movement ------------------------------------------------------
    def set_state(self, psi):
        psi = np.asarray(psi)
        if psi.shape != self.shape:
            raise ValueError(f"state shape {psi.shape} != tile {self.shape}")
        re, im = _soa(psi)
        self._check(lib().ts_b200_set_state(self._h, re.ctypes.data, im.ctypes.data,
                                            self.shape[1]))

    def set_exp_potential(self, pot_re, pot_im=None):
        pr = np.ascontiguousarray(pot_re, dtype=np.float64)
        if pr.shape != self.shape:
            raise ValueError("table shape mismatch")
        pi = None if pot_im is None else np.ascontiguousarray(pot_im, dtype=np.float64)
        self._check(lib().ts_b200_set_exp_potential(
            self._h, pr.ctypes.data, None if pi is None else pi.ctypes.data, self.shape[1]))

    def get_state(self, x=0, y=0, width=None, height=None):
        width = self.shape[1] - x if width is None else width
        height = self.shape[0] - y if height is None else height
        re = np.empty((height, width), np.float64)
        im = np.empty((height, width), np.float64)
        self._check(lib().ts_b200_get_sample(self._h, width, x, y, width, height,
                                             re.ctypes.data, im.ctypes.data))
        return re + 1j * im

    # The *_device calls read or write memory the caller produced or consumes
    # on torch's current stream: they are ordered after it (the handle's
    # stream waits for it) and, for reads back, before what torch queues next.
    def _after_torch(self):
        s = _torch_stream()
        if s is not None:
            self._check(lib().ts_b200_stream_wait(self._h, C.c_void_p(s)))

    def _before_torch(self):
        s = _torch_stream()
        if s is not None:
            self._check(lib().ts_b200_stream_signal(self._h, C.c_void_p(s)))

    def set_state_device(self, ptr, pitch):
        self._after_torch()
        self._check(lib().ts_b200_set_state_device(self._h, C.c_void_p(ptr), pitch))

    def get_state_device(self, ptr, pitch):
        self._after_torch()
        self._check(lib().ts_b200_get_state_device(self._h, C.c_void_p(ptr), pitch))
        self._before_torch()

    def set_exp_potential_device(self, ptr, pitch):
        self._after_torch()
        self._check(lib().ts_b200_set_exp_potential_device(self._h, C.c_void_p(ptr), pitch))

    def set_potential_device(self, ptr, pitch, delta_t):
        """The table exp(-i dt V) (exp(-dt V) in imaginary time) built on the
        device from V: dim_y rows of float64 at `ptr`, row pitch `pitch`."""
        self._after_torch()
        self._check(lib().ts_b200_set_potential_device(self._h, C.c_void_p(ptr), pitch,
                                                       float(delta_t)))

    def evolve_potentials(self, ptr, pitch, slab, count, delta_t, exchange=False):
        """`count` steps, step i with the potential at ptr + i * slab doubles
        (each dim_y rows of row pitch `pitch`) tabulated on the device."""
        self._check(lib().ts_b200_evolve_potentials(self._h, C.c_void_p(ptr), pitch, slab,
                                                    int(count), float(delta_t),
                                                    int(bool(exchange))))

    # -- evolution ---------------------------------------------------------
    def step(self, exchange=True):
        self._check(lib().ts_b200_step(self._h, int(bool(exchange))))

    def evolve(self, iterations):
        self._check(lib().ts_b200_evolve(self._h, int(iterations)))

    def synchronize(self):
        self._check(lib().ts_b200_synchronize(self._h))

    def set_stream(self, stream_ptr):
        self._check(lib().ts_b200_set_stream(self._h, C.c_void_p(stream_ptr)))

    # -- reductions --------------------------------------------------------
    def squared_norm(self):
        out = C.c_double()
        self._check(lib().ts_b200_squared_norm(self._h, C.byref(out)))
        return out.value

    def energies(self, potential, params):
        """potential: tile of V values or None (reuse); params: EnergyParams."""
        V = None if potential is None else np.ascontiguousarray(potential, np.float64)
        out = EnergyResult()
        self._check(lib().ts_b200_energies(self._h, None if V is None else V.ctypes.data,
                                           C.byref(params), C.byref(out)))
        return {n: getattr(out, n) for n, _ in EnergyResult._fields_}

    def expectations(self, params):
        out = ExpectationResult()
        self._check(lib().ts_b200_expectations(self._h, C.byref(params), C.byref(out)))
        return {n: getattr(out, n) for n, _ in ExpectationResult._fields_}

    # -- launch shape ------------------------------------------------------
    def launch_shape(self):
        s = LaunchShape()
        self._check(lib().ts_b200_launch_info(self._h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in LaunchShape._fields_}

    def autotune(self, trial_steps=3):
        """Pick the fastest balanced launch shape (state unchanged)."""
        self._check(lib().ts_b200_autotune(self._h, int(trial_steps)))
        return self.launch_shape()

    def set_launch(self, cells_per_lane=0, segment_rows=0, warps_per_block=0, ring_depth=0):
        self._check(lib().ts_b200_set_launch(self._h, cells_per_lane, segment_rows,
                                             warps_per_block, ring_depth))

    def set_walk(self, walk):
        """2: look-ahead row walk, two rows per iteration (default where the variant
        has one), 1: the same with one row per iteration, 0: checked walk."""
        self._check(lib().ts_b200_set_walk(self._h, int(walk)))


class Batch:
    """Many tiles advanced together, one persistent launch per Trotter step.

    kernels: Kernel objects (or raw ts_b200_kernel* handles, as
    Solver.kernel_handle() returns) of the same precision and time mode, no
    rotating frame.  The batch borrows their device state: set states and
    read results through the tiles' own calls; they must outlive the batch.
    """

    def __init__(self, kernels):
        self.kernels = list(kernels)

        def raw(k):  # a Kernel, a c_void_p or an integer ts_b200_kernel* address
            if hasattr(k, "handle"):
                return k.handle.value
            return k.value if isinstance(k, C.c_void_p) else int(k)
        arr = (C.c_void_p * len(self.kernels))(*[raw(k) for k in self.kernels])
        self._b = C.c_void_p()
        check(lib().ts_b200_batch_create(arr, len(self.kernels), C.byref(self._b)))

    def close(self):
        if self._b:
            lib().ts_b200_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.kernels)

    def _check(self, status):
        check(status, batch=self._b)

    def evolve(self, iterations):
        self._check(lib().ts_b200_batch_evolve(self._b, int(iterations)))

    def synchronize(self):
        self._check(lib().ts_b200_batch_synchronize(self._b))

    def set_stream(self, stream_ptr):
        self._check(lib().ts_b200_batch_set_stream(self._b, C.c_void_p(stream_ptr)))

    def set_launch(self, segment_rows=0, warps_per_block=0):
        self._check(lib().ts_b200_batch_set_launch(self._b, segment_rows, warps_per_block))

    def autotune(self, trial_steps=3, use_cache=True):
        self._check(lib().ts_b200_batch_autotune(self._b, int(trial_steps), int(bool(use_cache))))
        return self.launch_shape()

    def launch_shape(self):
        s = LaunchShape()
        self._check(lib().ts_b200_batch_launch_info(self._b, C.byref(s)))
        return {n: getattr(s, n) for n, _ in LaunchShape._fields_}


def launch_count():
    """Kernel launches made by this process through the library."""
    return int(lib().ts_b200_launch_count())


def version():
    return lib().ts_b200_version().decode()


class Pair:
    """Two species (two Kernel tiles of the same geometry) evolved together:
    the reference's two-component kernel and loop (ts_b200_pair_* of
    include/ts_b200.h).  coupling_ab is g_ab; omega = (omega_r, omega_i) the
    Rabi coupling.  While paired the tiles step only through the pair."""

    def __init__(self, a, b, coupling_ab, omega_r, omega_i, delta_t):
        self.a, self.b = a, b
        self._p = C.c_void_p()

        def raw(k):
            return k.handle if hasattr(k, "handle") else C.c_void_p(int(k))
        check(lib().ts_b200_pair_create(raw(a), raw(b), float(coupling_ab), float(omega_r),
                                        float(omega_i), float(delta_t), C.byref(self._p)),
              raw(a))

    def _check(self, status):
        check(status, pair=self._p)

    def rabi(self, var):
        self._check(lib().ts_b200_pair_rabi(self._p, float(var)))

    def evolve(self, iterations):
        self._check(lib().ts_b200_pair_evolve(self._p, int(iterations)))

    def cross_energies(self):
        inter, rabi = C.c_double(), C.c_double()
        self._check(lib().ts_b200_pair_cross_energies(self._p, C.byref(inter), C.byref(rabi)))
        return inter.value, rabi.value

    def close(self):
        if self._p:
            lib().ts_b200_pair_destroy(self._p)
            self._p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
