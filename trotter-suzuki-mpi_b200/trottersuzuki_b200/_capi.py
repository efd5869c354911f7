"""ctypes declarations of the C ABI in include/ts_b200.h.

The shared library libtsb200.so is built in-tree next to this file
(`python -m trottersuzuki_b200.build` or `__graft_entry__.build()`).  There is
no fallback: if the library is missing or no CUDA device is present, calls
raise.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_NAME = "libtsb200.so"
LIB_PATH = os.path.join(HERE, LIB_NAME)

OK = 0
STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
    4: "unsupported configuration", 5: "device wait timed out", 6: "no CUDA device",
}
FP64, FP32 = 0, 1


class Desc(C.Structure):
    _fields_ = [
        ("dim_x", C.c_int32), ("dim_y", C.c_int32),
        ("inner_x0", C.c_int32), ("inner_x1", C.c_int32),
        ("inner_y0", C.c_int32), ("inner_y1", C.c_int32),
        ("halo_x", C.c_int32), ("halo_y", C.c_int32),
        ("periodic_x", C.c_int32), ("periodic_y", C.c_int32),
        ("imag_time", C.c_int32), ("precision", C.c_int32),
        ("a_h", C.c_double), ("b_h", C.c_double), ("a_v", C.c_double), ("b_v", C.c_double),
        ("coupling", C.c_double), ("lhy_coupling", C.c_double),
        ("alpha_x", C.c_double), ("alpha_y", C.c_double),
        ("rot_offset_x", C.c_double), ("rot_offset_y", C.c_double),
        ("delta_x", C.c_double), ("delta_y", C.c_double),
        ("norm0", C.c_double),
        ("cylindrical", C.c_int32), ("angular_momentum", C.c_int32),
        ("kin_radial", C.c_double),
    ]


class EnergyParams(C.Structure):
    _fields_ = [
        ("mass", C.c_double), ("coupling", C.c_double), ("lhy_coupling", C.c_double),
        ("angular_velocity", C.c_double),
        ("start_x", C.c_int32), ("start_y", C.c_int32),
        ("global_no_halo_dim_x", C.c_int32), ("global_no_halo_dim_y", C.c_int32),
        ("length_x", C.c_double), ("length_y", C.c_double),
    ]


class EnergyResult(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("total", "kinetic", "potential", "rotational", "intra", "lhy", "norm2")]


class ExpectationResult(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("norm2", "mean_x", "mean_xx", "mean_y", "mean_yy", "mean_px", "mean_pxpx",
                 "mean_py", "mean_pypy", "mean_lz")]


class LaunchShape(C.Structure):
    _fields_ = [
        ("cells_per_lane", C.c_int32), ("segment_rows", C.c_int32),
        ("warps_per_block", C.c_int32), ("ring_depth", C.c_int32),
        ("strips", C.c_int32), ("segments", C.c_int32), ("blocks", C.c_int32),
        ("threads", C.c_int32), ("smem_bytes", C.c_int64),
        ("walk", C.c_int32), ("reserved", C.c_int32),
    ]


class SlabLink(C.Structure):
    _fields_ = [("up", C.c_int32), ("down", C.c_int32),
                ("up_wraps", C.c_int32), ("down_wraps", C.c_int32),
                ("xhalo_row0", C.c_int32), ("xhalo_row1", C.c_int32)]


# name -> (restype, argtypes); every symbol declared in include/ts_b200.h
_VP, _SZ, _DP, _I = C.c_void_p, C.c_size_t, C.c_void_p, C.c_int
SIGNATURES = {
    "ts_b200_create": (_I, [C.POINTER(Desc), C.POINTER(_VP)]),
    "ts_b200_destroy": (_I, [_VP]),
    "ts_b200_set_state": (_I, [_VP, _DP, _DP, _SZ]),
    "ts_b200_set_exp_potential": (_I, [_VP, _DP, _DP, _SZ]),
    "ts_b200_step": (_I, [_VP, _I]),
    "ts_b200_evolve": (_I, [_VP, _I]),
    "ts_b200_halo_exchange": (_I, [_VP]),
    "ts_b200_get_sample": (_I, [_VP, _SZ, _SZ, _SZ, _SZ, _SZ, _DP, _DP]),
    "ts_b200_squared_norm": (_I, [_VP, C.POINTER(C.c_double)]),
    "ts_b200_energies": (_I, [_VP, _DP, C.POINTER(EnergyParams), C.POINTER(EnergyResult)]),
    "ts_b200_expectations": (_I, [_VP, C.POINTER(EnergyParams), C.POINTER(ExpectationResult)]),
    "ts_b200_squared_norm_noalloc": (_I, [_VP, _I, _SZ, _I, _I, _I, _I, _I, _I, C.c_double,
                                          C.c_double, _VP, _VP]),
    "ts_b200_set_state_device": (_I, [_VP, _VP, _SZ]),
    "ts_b200_get_state_device": (_I, [_VP, _VP, _SZ]),
    "ts_b200_set_exp_potential_device": (_I, [_VP, _VP, _SZ]),
    "ts_b200_set_potential_device": (_I, [_VP, _VP, _SZ, C.c_double]),
    "ts_b200_evolve_potentials": (_I, [_VP, _VP, _SZ, _SZ, C.c_int, C.c_double, C.c_int]),
    "ts_b200_set_stream": (_I, [_VP, _VP]),
    "ts_b200_stream_wait": (_I, [_VP, _VP]),
    "ts_b200_stream_signal": (_I, [_VP, _VP]),
    "ts_b200_rows": (_I, [_VP, C.c_int, C.c_int, C.POINTER(_VP), C.POINTER(_SZ)]),
    "ts_b200_last_norm": (_I, [_VP, C.POINTER(_VP)]),
    "ts_b200_renormalize_from": (_I, [_VP, _VP]),
    "ts_b200_slab_windows": (_I, [_I, _I, _I, _I, _I, _I, _I, C.POINTER(C.c_int32)]),
    "ts_b200_slab_messages": (_I, [_I, _I, _I, C.POINTER(SlabLink), _I, C.POINTER(C.c_int32)]),
    "ts_b200_nccl_unique_id": (_I, [_VP, _SZ]),
    "ts_b200_slabs_create_local": (_I, [C.POINTER(_VP), C.POINTER(_VP), C.POINTER(SlabLink), _I]),
    "ts_b200_slabs_create_nccl": (_I, [C.POINTER(_VP), _VP, C.POINTER(SlabLink), _VP, _SZ, _I,
                                       _I]),
    "ts_b200_slabs_set_split": (_I, [_VP, _I]),
    "ts_b200_slabs_plan": (_I, [_VP, _I, C.POINTER(C.c_int32)]),
    "ts_b200_slabs_evolve": (_I, [_VP, _I]),
    "ts_b200_slabs_last_error": (C.c_char_p, [_VP]),
    "ts_b200_slabs_destroy": (_I, [_VP]),
    "ts_b200_pair_create": (_I, [_VP, _VP, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.POINTER(_VP)]),
    "ts_b200_pair_rabi": (_I, [_VP, C.c_double]),
    "ts_b200_pair_evolve": (_I, [_VP, C.c_int]),
    "ts_b200_pair_steps": (_I, [_VP, C.c_int, C.c_int]),
    "ts_b200_pair_step_species": (_I, [_VP, C.c_int]),
    "ts_b200_pair_normalize": (_I, [_VP]),
    "ts_b200_pair_cross_energies": (_I, [_VP, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "ts_b200_pair_last_error": (C.c_char_p, [_VP]),
    "ts_b200_pair_destroy": (_I, [_VP]),
    "ts_b200_synchronize": (_I, [_VP]),
    "ts_b200_launch_info": (_I, [_VP, C.POINTER(LaunchShape)]),
    "ts_b200_set_launch": (_I, [_VP, _I, _I, _I, _I]),
    "ts_b200_autotune": (_I, [_VP, _I]),
    "ts_b200_set_walk": (_I, [_VP, _I]),
    "ts_b200_set_overlap": (_I, [_VP, _I]),
    "ts_b200_batch_create": (_I, [C.POINTER(_VP), _I, C.POINTER(_VP)]),
    "ts_b200_batch_destroy": (None, [_VP]),
    "ts_b200_batch_size": (_I, [_VP]),
    "ts_b200_batch_evolve": (_I, [_VP, _I]),
    "ts_b200_batch_synchronize": (_I, [_VP]),
    "ts_b200_batch_set_stream": (_I, [_VP, _VP]),
    "ts_b200_batch_set_launch": (_I, [_VP, _I, _I]),
    "ts_b200_batch_autotune": (_I, [_VP, _I, _I]),
    "ts_b200_batch_launch_info": (_I, [_VP, C.POINTER(LaunchShape)]),
    "ts_b200_batch_last_error": (C.c_char_p, [_VP]),
    "ts_b200_adjoint_create": (_I, [C.POINTER(Desc), C.c_double, _I, _I, C.POINTER(_VP)]),
    "ts_b200_adjoint_destroy": (None, [_VP]),
    "ts_b200_adjoint_set_stream": (_I, [_VP, _VP]),
    "ts_b200_adjoint_set_segments": (_I, [_VP, _I, _I]),
    "ts_b200_adjoint_forward": (_I, [_VP, _VP, _VP, _VP]),
    "ts_b200_adjoint_backward": (_I, [_VP, _VP, _VP, _VP]),
    "ts_b200_adjoint_synchronize": (_I, [_VP]),
    "ts_b200_adjoint_last_error": (C.c_char_p, [_VP]),
    "ts_b200_host_alloc": (_I, [C.POINTER(_VP), _SZ]),
    "ts_b200_host_free": (_I, [_VP]),
    "ts_b200_last_error": (C.c_char_p, [_VP]),
    "ts_b200_status_string": (C.c_char_p, [_I]),
    "ts_b200_version": (C.c_char_p, []),
    "ts_b200_launch_count": (C.c_uint64, []),
}

_lib = None


class B200Error(RuntimeError):
    """A C-ABI call returned a non-zero status (mirrors the reference's my_abort)."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS.get(status, 'status %d' % status)}: {message}")
        self.status = status


def lib():
    """Load libtsb200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build the CUDA extension first "
                "(python -c 'import __graft_entry__ as g; g.build()')")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, handle=None, batch=None, adjoint=None, pair=None, slabs=None):
    if status != OK:
        if slabs:
            msg = lib().ts_b200_slabs_last_error(slabs).decode()
        elif pair:
            msg = lib().ts_b200_pair_last_error(pair).decode()
        elif adjoint:
            msg = lib().ts_b200_adjoint_last_error(adjoint).decode()
        elif batch:
            msg = lib().ts_b200_batch_last_error(batch).decode()
        else:
            msg = lib().ts_b200_last_error(handle).decode() if handle else ""
        raise B200Error(status, msg or STATUS.get(status, ""))
