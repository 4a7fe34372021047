"""ctypes binding of the native library (``pptk_b200/_lib/libpptkg.so``).

The library is the only compute path: there is no CPU fallback.  If it is
missing or fails to load, every entry point raises ``NativeLibraryError``.
"""
import ctypes
import os
import threading

import numpy as np

# PPTKG_LIBRARY selects another build of the library (the bounds-checked
# diagnostic build, libpptkg_checked.so)
LIB_PATH = os.environ.get("PPTKG_LIBRARY") or os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib",
                                                            "libpptkg.so")

OK, E_INVALID, E_TYPE, E_CUDA, E_RANGE, E_DEVICE, E_UNSUPPORTED = range(7)
MEM_HOST, MEM_DEVICE = 0, 1
PREC_AUTO, PREC_FP32, PREC_FP64 = 0, 1, 2

DTYPE_CODES = {
    np.dtype(np.float32): 0, np.dtype(np.float64): 1,
    np.dtype(np.int8): 2, np.dtype(np.int16): 3, np.dtype(np.int32): 4, np.dtype(np.int64): 5,
    np.dtype(np.uint8): 6, np.dtype(np.uint16): 7, np.dtype(np.uint32): 8, np.dtype(np.uint64): 9,
}
CODE_DTYPES = {v: k for k, v in DTYPE_CODES.items()}


class NativeLibraryError(RuntimeError):
    """The CUDA library could not be loaded."""


class PptkgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_vp, _i64, _int, _dbl, _flt = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_float
_pvp = ctypes.POINTER(ctypes.c_void_p)
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pint = ctypes.POINTER(ctypes.c_int)

SIGNATURES = {
    "pptkg_version": [],
    "pptkg_bounds_checked": [],
    "pptkg_last_error": [ctypes.c_char_p, ctypes.c_size_t],
    "pptkg_tree_build": [_vp, _i64, _int, _int, _int, _int, _dbl, _vp, _pvp],
    "pptkg_tree_free": [_vp],
    "pptkg_tree_info": [_vp, _pi64, _pi64, _pint, _pint, _pi64, _pint],
    "pptkg_tree_reverse_indices": [_vp, _vp, _int, _vp],
    "pptkg_tree_ref_nodes": [_vp, _vp, _i64, _pi64],
    "pptkg_tree_set_bucket": [_vp, _int, _vp],
    "pptkg_knn": [_vp, _vp, _i64, _int, _int, _int, _dbl, _vp, _vp, _vp],
    "pptkg_knn_self": [_vp, _vp, _i64, _int, _int, _dbl, _vp, _vp, _vp],
    "pptkg_rnear_count": [_vp, _vp, _vp, _i64, _int, _int, _dbl, _vp, _pi64, _vp],
    "pptkg_rnear_fill": [_vp, _vp, _vp, _i64, _int, _int, _dbl, _vp, _vp, _vp],
    "pptkg_estimate_normals": [_vp, _i64, _int, _int, _int, _flt, _vp, _i64, _int, _int, _vp, _vp, _vp, _vp],
    "pptkg_tree_normals": [_vp, _vp, _i64, _int, _int, _flt, _int, _int, _vp, _vp, _vp, _vp],
    "pptkg_eigh3": [_vp, _i64, _int, _int, _vp, _vp, _int, _vp],
    "pptkg_nbhd_covariance": [_vp, _i64, _int, _int, _vp, _vp, _i64, _vp, _vp],
    "pptkg_forest_build": [_vp, _i64, _int, _int, _int, _vp, _int, _int, _dbl, _vp, _pvp],
    "pptkg_forest_info": [_vp, _pint, _vp],
    "pptkg_forest_ref_nodes": [_vp, _int, _vp, _i64, _pi64],
    "pptkg_forest_knn": [_vp, _int, _dbl, _int, _int, _vp, _vp, _vp],
    "pptkg_forest_normals": [_vp, _int, _flt, _int, _int, _int, _vp, _vp, _vp, _vp],
    "pptkg_forest_knn_normals": [_vp, _int, _flt, _int, _int, _int, _vp, _vp, _vp, _vp, _vp, _vp],
    "pptkg_forest_capture_ready": [_vp, _vp],
    "pptkg_forest_rebuild": [_vp, _vp, _vp],
    "pptkg_tree_normals_noalloc": [_vp, _vp, _i64, _int, _flt, _int, _int, _vp, _vp, _vp, _vp],
    "pptkg_multi_knn": [_vp, _int, _vp, _vp, _int, _int, _int, _dbl, _vp, _vp, _vp],
    "pptkg_multi_normals": [_vp, _int, _vp, _vp, _int, _int, _flt, _int, _int, _vp, _vp, _vp, _vp],
    "pptkg_profile_enable": [_int],
    "pptkg_profile_get": [ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), _pi64],
    "pptkg_tune_set": [ctypes.c_char_p, _i64],
    "pptkg_tune_get": [ctypes.c_char_p, _pi64],
    "pptkg_set_status_sink": [_vp],
    "pptkg_tree_save": [_vp, _vp, _i64, _pi64],
    "pptkg_tree_load": [_vp, _i64, _vp, _pvp],
}

_lib = None
_lock = threading.Lock()


def lib():
    """The loaded library; raises NativeLibraryError when it is unavailable."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise NativeLibraryError(
                        f"{LIB_PATH} is missing: build it with `python -m pptk_b200._build` "
                        "(there is no CPU fallback)")
                try:
                    handle = ctypes.CDLL(LIB_PATH)
                except OSError as e:
                    raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
                for name, args in SIGNATURES.items():
                    fn = getattr(handle, name)
                    fn.argtypes = args
                    fn.restype = ctypes.c_int
                handle.pptkg_launch_count.argtypes = []
                handle.pptkg_launch_count.restype = ctypes.c_int64
                _lib = handle
    return _lib


def last_error():
    buf = ctypes.create_string_buffer(2048)
    code = lib().pptkg_last_error(buf, len(buf))
    return code, buf.value.decode(errors="replace")


_EXC = {
    E_INVALID: ValueError,
    E_TYPE: TypeError,
    E_RANGE: RuntimeError,
    E_UNSUPPORTED: NotImplementedError,
}


def check(status, where=""):
    """Raises the Python exception that matches a C ABI status."""
    if status == OK:
        return
    code, msg = last_error()
    exc = _EXC.get(status)
    text = f"{where}: {msg}" if where else msg
    if exc is None:
        raise PptkgError(status, text)
    raise exc(text)


def call(name, *args, where=None):
    check(getattr(lib(), name)(*args), where or name)


# ------------------------------------------------------------- arrays ------
def is_torch_cuda(x):
    mod = type(x).__module__
    if not mod.startswith("torch"):
        return False
    import torch
    return isinstance(x, torch.Tensor) and x.is_cuda


def torch_stream(device=None):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(a):
    """Address of a numpy array or torch tensor (None passes through)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return ctypes.c_void_p(a.ctypes.data)
    return ctypes.c_void_p(a.data_ptr())


def tune_set(name, value):
    """Sets a process-wide tuning knob of the native library (pptkg_tune_set)."""
    call("pptkg_tune_set", name.encode(), int(value))


def tune_get(name):
    v = ctypes.c_int64()
    call("pptkg_tune_get", name.encode(), ctypes.byref(v))
    return v.value
