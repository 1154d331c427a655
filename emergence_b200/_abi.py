"""ctypes declarations of the C ABI in include/emergence_b200.h.

The library is the in-tree ``libemergence_b200.so`` built by
``emergence_b200/build.py``. There is no fallback: if the library is missing,
every solver call raises ``RuntimeError``.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libemergence_b200.so")
LIB_PATH_BC = os.path.join(HERE, "libemergence_b200_bc.so")

EMG_OK = 0
STATUS_NAMES = {
    1: "EMG_ERR_INVALID",
    2: "EMG_ERR_CUDA",
    3: "EMG_ERR_DT_COLLAPSED",
    4: "EMG_ERR_INADMISSIBLE",
    5: "EMG_ERR_UNFILLABLE",
    6: "EMG_ERR_BOUNDS",
    7: "EMG_ERR_NO_DEVICE",
    8: "EMG_ERR_TIMEOUT",
}


class EmgEos(C.Structure):
    _fields_ = [("gamma", C.c_double), ("p_inf", C.c_double), ("b", C.c_double), ("q", C.c_double), ("cv", C.c_double)]


class EmgMesh(C.Structure):
    _fields_ = [("n", C.c_int64 * 3), ("lo", C.c_double * 3), ("dx", C.c_double * 3), ("ng", C.c_int64)]


class EmgBc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("state", C.c_double * 5)]


class EmgBc7(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("state", C.c_double * 7)]


class EmgFiveSystem(C.Structure):
    _fields_ = [("eos", EmgEos * 2), ("kapila", C.c_int32), ("reserved", C.c_int32)]


class EmgAmrConfig(C.Structure):
    _fields_ = [("b", C.c_int64), ("levels", C.c_int64), ("eps", C.c_double), ("regrid_every", C.c_int64),
                ("base_blocks", C.c_int64 * 3), ("ghosts", C.c_int64)]


# void (*)(void* ctx, const double* x, int64_t n, double* w)
INIT_FN = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.POINTER(C.c_double))

class EmgOpts(C.Structure):
    _fields_ = [("cfl", C.c_double), ("tol", C.c_double), ("mode", C.c_int32), ("positivity", C.c_int32),
                ("precision", C.c_int32), ("flags", C.c_int32)]


EMG_K_COUNT = 5
KERNEL_KINDS = ("ghost", "axis0", "axis1", "axis2", "cfl")

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_U64 = C.POINTER(C.c_uint64)

# name -> (restype, argtypes)
SIGNATURES = {
    "emg_last_error": (C.c_char_p, []),
    "emg_version": (C.c_char_p, []),
    "emg_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "emg_state_hash": (C.c_int, [C.POINTER(EmgMesh), _D, C.c_size_t, _U64]),
    "emg_uniform_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc), C.POINTER(EmgOpts),
                                     _D, C.c_size_t, C.POINTER(_P)]),
    "emg_uniform_destroy": (C.c_int, [_P]),
    "emg_release_memory": (C.c_int, []),
    "emg_five_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgFiveSystem), C.POINTER(EmgBc7), C.POINTER(EmgOpts),
                                  _D, C.c_size_t, C.POINTER(_P)]),
    "emg_five_destroy": (C.c_int, [_P]),
    "emg_five_step": (C.c_int, [_P, C.c_double]),
    "emg_five_dt_cfl": (C.c_int, [_P, _D]),
    "emg_five_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emg_five_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_five_counters": (C.c_int, [_P, _U64]),
    "emg_five_totals": (C.c_int, [_P, _D]),
    "emg_five_get_time": (C.c_int, [_P, _D]),
    "emg_five_launch_count": (C.c_int, [_P, _U64]),
    "emg_five_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "emg_uniform_step": (C.c_int, [_P, C.c_double]),
    "emg_uniform_dt_cfl": (C.c_int, [_P, _D]),
    "emg_uniform_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emg_uniform_advance": (C.c_int, [_P, C.c_uint64, C.c_double, _U64]),
    "emg_uniform_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_uniform_upload": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_uniform_totals": (C.c_int, [_P, _D]),
    "emg_uniform_counters": (C.c_int, [_P, _U64]),
    "emg_uniform_get_time": (C.c_int, [_P, _D]),
    "emg_uniform_set_time": (C.c_int, [_P, C.c_double]),
    "emg_uniform_synchronize": (C.c_int, [_P]),
    "emg_uniform_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "emg_uniform_set_profiling": (C.c_int, [_P, C.c_int]),
    "emg_uniform_kernel_times": (C.c_int, [_P, _D, _U64]),
    "emg_uniform_launch_count": (C.c_int, [_P, _U64]),
    "emg_uniform_features": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "emg_uniform_step_noalloc": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc),
                                           C.POINTER(EmgOpts), C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    "emg_batch1d_create": (C.c_int, [C.POINTER(EmgEos), C.POINTER(EmgOpts), C.POINTER(EmgBc), C.c_size_t,
                                     C.POINTER(C.c_int64), _D, _D, C.POINTER(_P)]),
    "emg_batch1d_destroy": (C.c_int, [_P]),
    "emg_batch1d_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emg_batch1d_download": (C.c_int, [_P, _D]),
    "emg_batch1d_status": (C.c_int, [_P, _D, _U64]),
    "emg_batch1d_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "emg_batch1d_record": (C.c_int, [_P, C.c_double, C.c_uint64, _U64]),
    "emg_batch1d_objective": (C.c_int, [_P, C.c_int, C.c_double, C.c_double, _D]),
    "emg_batch1d_backward": (C.c_int, [_P, C.c_double, _D, _D]),
    "emg_batch1d_adjoint_times": (C.c_int, [_P, _D]),
    "emg_amr_create": (C.c_int, [C.POINTER(EmgAmrConfig), C.POINTER(EmgEos), _D, _D, C.POINTER(EmgBc),
                                 C.POINTER(EmgOpts), INIT_FN, C.c_void_p, C.POINTER(_P)]),
    "emg_amr_create_from_blocks": (C.c_int, [C.POINTER(EmgAmrConfig), C.POINTER(EmgEos), _D, _D, C.POINTER(EmgBc),
                                             C.POINTER(EmgOpts), C.POINTER(C.c_int64), C.c_size_t, _D, C.POINTER(_P)]),
    "emg_amr_destroy": (C.c_int, [_P]),
    "emg_amr_step": (C.c_int, [_P, C.c_double]),
    "emg_amr_dt_cfl": (C.c_int, [_P, _D]),
    "emg_amr_step_subcycled": (C.c_int, [_P, C.c_double]),
    "emg_amr_dt_cfl_subcycled": (C.c_int, [_P, _D]),
    "emg_amr_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emg_amr_regrid": (C.c_int, [_P]),
    "emg_amr_block_count": (C.c_int, [_P, _U64, _U64]),
    "emg_amr_structure": (C.c_int, [_P, C.POINTER(C.c_int64), C.c_size_t]),
    "emg_amr_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_amr_create_five": (C.c_int, [C.POINTER(EmgAmrConfig), C.POINTER(EmgFiveSystem), _D, _D, C.POINTER(EmgBc7),
                                      C.POINTER(EmgOpts), INIT_FN, C.c_void_p, C.POINTER(_P)]),
    "emg_amr_create_five_from_blocks": (C.c_int, [C.POINTER(EmgAmrConfig), C.POINTER(EmgFiveSystem), _D, _D,
                                                  C.POINTER(EmgBc7), C.POINTER(EmgOpts), C.POINTER(C.c_int64),
                                                  C.c_size_t, _D, C.POINTER(_P)]),
    "emg_amr_nv": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "emg_amr_totals": (C.c_int, [_P, _D]),
    "emg_amr_counters": (C.c_int, [_P, _U64]),
    "emg_amr_get_time": (C.c_int, [_P, _D]),
    "emg_amr_steps": (C.c_int, [_P, _U64]),
    "emg_amr_synchronize": (C.c_int, [_P]),
    "emg_amr_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "emg_amr_phase_times": (C.c_int, [_P, _D]),
    "emg_amr_launch_count": (C.c_int, [_P, _U64]),
    "emg_adjoint_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc), C.POINTER(EmgOpts), _D,
                                     C.c_size_t, C.POINTER(_P)]),
    "emg_adjoint_destroy": (C.c_int, [_P]),
    "emg_adjoint_set_initial": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_adjoint_forward": (C.c_int, [_P, C.c_uint64, C.c_double, C.c_uint64, _U64]),
    "emg_adjoint_forward_dts": (C.c_int, [_P, _D, C.c_uint64, C.c_uint64]),
    "emg_adjoint_dts": (C.c_int, [_P, _D, C.c_size_t, _U64]),
    "emg_adjoint_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_adjoint_objective": (C.c_int, [_P, C.c_int, _D, _D, _D]),
    "emg_adjoint_seed": (C.c_int, [_P, _D, C.c_size_t]),
    "emg_adjoint_backward": (C.c_int, [_P, _D, _D, _D]),
    "emg_adjoint_step_vjp": (C.c_int, [_P, _D, C.c_size_t, C.c_double, _D, _D, _D]),
    "emg_adjoint_times": (C.c_int, [_P, _D]),
    "emg_adjoint_stream": (C.c_int, [_P, C.POINTER(_P)]),
}

_lib = None


def lib_path():
    """The product library, or its bounds-check build when the environment
    sets EMG_BOUNDS_CHECK=1 (index checks that report EMG_ERR_BOUNDS)."""
    return LIB_PATH_BC if os.environ.get("EMG_BOUNDS_CHECK") == "1" else LIB_PATH


def lib():
    """Load the in-tree CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise RuntimeError(
                f"{os.path.basename(path)} is missing: build it with `python -m emergence_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class EmgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(code):
    if code != EMG_OK:
        msg = lib().emg_last_error()
        raise EmgError(code, msg.decode() if msg else "")
    return code
