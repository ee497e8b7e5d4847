"""ctypes binding of libfastesp_b200.so (the C ABI declared in include/fastesp_b200.h).

The library is loaded from the package directory.  There is no fallback: if the
shared object is missing or does not load, every call raises
:class:`NativeLibraryError` -- the ESP path has no CPU implementation.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfastesp_b200.so"
NCLASS = 9

FE_OK = 0
RULES = {"numpy": 0, "native": 1}


class NativeLibraryError(RuntimeError):
    pass


class FeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fastesp_b200 error {code}: {msg}")
        self.code = code


class FeBasis(C.Structure):
    _fields_ = [("n_func", C.c_int), ("n_prim", C.c_int), ("n_atoms", C.c_int),
                ("fn_atom", C.c_void_p), ("fn_nprim", C.c_void_p), ("fn_off", C.c_void_p),
                ("fn_lx", C.c_void_p), ("fn_ly", C.c_void_p), ("fn_lz", C.c_void_p),
                ("fn_shell", C.c_void_p), ("fc", C.c_void_p), ("pexp", C.c_void_p),
                ("pcoef", C.c_void_p), ("Z", C.c_void_p), ("xyz", C.c_void_p)]


class FeSizes(C.Structure):
    _fields_ = [("plan_bytes", C.c_size_t), ("table_bytes", C.c_size_t),
                ("build_ws_bytes", C.c_size_t), ("n_shell", C.c_int),
                ("n_shell_pair", C.c_int), ("n_work", C.c_int), ("cap", C.c_int * NCLASS)]


class FeTableInfo(C.Structure):
    _fields_ = [("count", C.c_int * NCLASS), ("n_pairs", C.c_int), ("n_atoms", C.c_int),
                ("sum_rule", C.c_double), ("tol", C.c_double), ("rule", C.c_int),
                ("has_f32", C.c_int), ("n_warp_screen", C.c_int)]


class FeBatchMol(C.Structure):
    _fields_ = [("d_table", C.c_void_p), ("d_pts", C.c_void_p), ("d_out", C.c_void_p),
                ("n_pts", C.c_int), ("reserved", C.c_int)]


class FeBatchShape(C.Structure):
    _fields_ = [("points_per_thread", C.c_int), ("waves", C.c_int), ("stage_bytes", C.c_int)]


_P = C.c_void_p
_SIGS = {
    "fe_version": (C.c_int, []),
    "fe_last_error": (C.c_char_p, []),
    "fe_status": (C.c_int, [C.POINTER(C.c_uint), C.c_int]),
    "fe_plan_create": (C.c_int, [C.POINTER(FeBasis), C.POINTER(_P)]),
    "fe_plan_destroy": (None, [_P]),
    "fe_plan_sizes": (C.c_int, [_P, C.POINTER(FeSizes)]),
    "fe_plan_upload": (C.c_int, [_P, _P, _P]),
    "fe_table_build": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_double, C.c_int, _P, _P,
                                 C.c_size_t, _P]),
    "fe_build_ws_bytes": (C.c_size_t, [_P, C.c_int]),
    "fe_table_bytes": (C.c_size_t, [C.POINTER(C.c_int), C.c_int]),
    "fe_table_offsets": (C.c_int, [C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_size_t),
                                   C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "fe_table_init": (C.c_int, [_P, C.POINTER(C.c_int), C.c_int, _P, _P, _P]),
    "fe_table_make_f32": (C.c_int, [_P, _P]),
    "fe_table_info_get": (C.c_int, [_P, C.POINTER(FeTableInfo), _P]),
    "fe_eval_ws_bytes": (C.c_size_t, [C.c_int]),
    "fe_point_order_bytes": (C.c_size_t, [C.c_int]),
    "fe_eval_ws_bytes_mixed": (C.c_size_t, [C.c_int, C.POINTER(C.c_int)]),
    "fe_esp_fp64": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "fe_electron_fp64": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "fe_nuclear_fp64": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_size_t, _P]),
    "fe_electron_classes": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_size_t, C.c_int,
                                      C.c_double, C.c_int, C.c_int, _P, _P]),
    "fe_esp_mixed": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_size_t, C.c_double, _P, _P]),
    "fe_electron_mixed": (C.c_int, [_P, _P, C.c_int, _P, _P, C.c_size_t, C.c_double, _P, _P]),
    "fe_boys_fp64": (C.c_int, [_P, C.c_int, C.c_int, _P, _P]),
    "fe_peak_run": (C.c_int, [C.c_int, C.c_longlong, C.c_int, _P, _P]),
    "fe_wait_selftest": (C.c_int, [C.c_longlong, _P, _P]),
    "fe_esp_fp64_noalloc": (C.c_int, [_P, _P, C.c_int, _P, _P]),
    "fe_noalloc_scratch_bytes": (C.c_size_t, []),
    "fe_field_ws_bytes": (C.c_size_t, [C.c_int]),
    "fe_esp_field_fp64": (C.c_int, [_P, _P, C.c_int, _P, _P, _P, _P, C.c_size_t, _P]),
    "fe_adjoint_ws_bytes": (C.c_size_t, [_P, C.c_int]),
    "fe_esp_adjoint": (C.c_int, [_P, _P, _P, _P, C.c_int, _P, _P, _P, _P, C.c_size_t, _P]),
    "fe_batch_create": (C.c_int, [C.POINTER(FeBatchMol), C.c_int, C.POINTER(FeBatchShape),
                                  C.POINTER(_P), _P]),
    "fe_batch_destroy": (None, [_P]),
    "fe_batch_sizes": (C.c_int, [_P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                 C.POINTER(C.c_int)]),
    "fe_batch_upload": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "fe_batch_run": (C.c_int, [_P, _P, _P, C.c_size_t, _P]),
    "fe_points_ws_bytes": (C.c_size_t, [C.c_longlong]),
    "fe_surface_points": (C.c_int, [_P, _P, C.c_int, _P, C.c_longlong, C.c_double, _P,
                                    C.c_longlong, _P, _P, C.c_size_t, _P]),
    "fe_grid_points": (C.c_int, [_P, C.c_int, C.c_double, _P, C.c_longlong, _P,
                                 C.c_longlong, C.c_longlong, C.c_longlong,
                                 _P, C.c_longlong, _P, _P, C.c_size_t, _P]),
}

_lock = threading.Lock()
_lib = None


def lib():
    """The loaded library; raises NativeLibraryError if it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise NativeLibraryError(
                    f"{LIB_PATH} is missing; build it with `python -m fastesp_b200.build`")
            try:
                h = C.CDLL(str(LIB_PATH))
            except OSError as e:
                raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
            for name, (res, args) in _SIGS.items():
                fn = getattr(h, name)
                fn.restype = res
                fn.argtypes = args
            _lib = h
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != FE_OK:
        raise FeError(rc, lib().fe_last_error().decode(errors="replace"))


def status(clear: bool = True) -> int:
    bits = C.c_uint(0)
    check(lib().fe_status(C.byref(bits), int(clear)))
    return int(bits.value)


def ptr(t) -> int:
    """Device (or host) address of a torch tensor / numpy array."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def stream_ptr(stream=None) -> int:
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return s.cuda_stream


def ws_bytes(n_pts: int, precision: str = "fp64", caps=None) -> int:
    """Evaluation workspace bytes (``caps``: per-class pair bounds, mixed only),
    with room for the evaluators' spatial point order."""
    L = lib()
    if precision == "fp64":
        return int(L.fe_eval_ws_bytes(int(n_pts))) + int(L.fe_point_order_bytes(int(n_pts)))
    cap = (C.c_int * NCLASS)(*[int(c) for c in caps])
    return int(L.fe_eval_ws_bytes_mixed(int(n_pts), cap))
