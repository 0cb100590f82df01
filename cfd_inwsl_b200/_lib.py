"""ctypes binding of libcfdgpu.so (include/cfdgpu.h).

The library is the only compute path: if it is missing or cannot be loaded,
every entry point raises. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libcfdgpu.so"

CFD_OK = 0
ERRORS = {
    -1: "CFD_ERR_CONFIG",
    -2: "CFD_ERR_CUDA",
    -3: "CFD_ERR_NONFINITE",
    -4: "CFD_ERR_NEGATIVE_STATE",
    -5: "CFD_ERR_TIMEOUT",
    -6: "CFD_ERR_UNSUPPORTED",
    -7: "CFD_ERR_NOMEM",
}


class CfdError(RuntimeError):
    def __init__(self, code: int, msg: str = ""):
        self.code = code
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")


class CfdConfig(C.Structure):
    _fields_ = [
        ("dim", C.c_int),
        ("n", C.c_int * 3),
        ("h", C.c_double * 3),
        ("x0", C.c_double * 3),
        ("n_ghost", C.c_int),
        ("gamma", C.c_double),
        ("inter_method", C.c_int),
        ("flux_method", C.c_int),
        ("diff_method", C.c_int),
        ("precision", C.c_int),
        ("strict", C.c_int),
        ("bc", (C.c_int * 2) * 3),
        ("device", C.c_int),
        ("seg_len", C.c_int * 3),
        ("source_type", C.c_int),
        ("positivity", C.c_int),
    ]


_lib = None

# name -> (restype, argtypes)
_PROTOS = {
    "cfd_config_default": (None, [C.POINTER(CfdConfig)]),
    "cfd_create": (C.c_int, [C.POINTER(CfdConfig), C.POINTER(C.c_void_p)]),
    "cfd_destroy": (None, [C.c_void_p]),
    "cfd_last_error": (C.c_char_p, [C.c_void_p]),
    "cfd_set_line_bc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_longlong, C.c_int,
                                  C.c_void_p]),
    "cfd_upload_cons": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_download_cons": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_download_prim": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_rhs": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p]),
    "cfd_max_dt": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_double)]),
    "cfd_rk3_step": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "cfd_run": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_double),
                          C.POINTER(C.c_int), C.c_void_p, C.c_void_p]),
    "cfd_step_host": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                                C.POINTER(C.c_double)]),
    "cfd_device_state": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_longlong),
                                   C.POINTER(C.c_void_p)]),
    "cfd_set_state_device": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_eval_inter5": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "cfd_check_division": (C.c_int, [C.c_longlong, C.c_ulonglong, C.POINTER(C.c_ulonglong)]),
    "cfd_fp64_peak_probe": (C.c_int, [C.c_longlong, C.c_void_p, C.POINTER(C.c_double)]),
    "cfd_eval_flux": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "cfd_version": (C.c_char_p, []),
    "cfd_batch_create": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cfd_batch_destroy": (None, [C.c_void_p]),
    "cfd_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "cfd_batch_case": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cfd_batch_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_batch_launch_count": (C.c_ulonglong, [C.c_void_p]),
    "cfd_batch_run": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "cfd_batch_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "cfd_batch_set_tiling": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]),
    "cfd_accuracy_test": (C.c_int, [C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p]),
    "cfd_eval_face": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p]),
    "cfd_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_launch_count": (C.c_ulonglong, [C.c_void_p]),
    "cfd_sweep": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_double]),
    "cfd_rhs_noalloc": (C.c_int, [C.POINTER(CfdConfig), C.c_void_p, C.c_void_p, C.c_double, C.c_void_p]),
    "cfd_rhs_vjp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "cfd_adjoint_record": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int]),
    "cfd_run_fixed": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int]),
    "cfd_adjoint_reverse": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "cfd_enable_halo": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_longlong)]),
    "cfd_stage_state": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "cfd_loop_begin": (C.c_int, [C.c_void_p, C.c_double, C.c_double]),
    "cfd_reduction_words": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "cfd_loop_step_begin": (C.c_int, [C.c_void_p]),
    "cfd_loop_stage": (C.c_int, [C.c_void_p, C.c_int]),
    "cfd_loop_step_end": (C.c_int, [C.c_void_p]),
    "cfd_loop_end": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    "cfd_rk3_stage": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double]),
    "cfd_max_wave_speeds": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfd_save_checkpoint": (C.c_int, [C.c_void_p, C.c_char_p, C.c_double, C.c_longlong]),
    "cfd_load_checkpoint": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
}


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load libcfdgpu.so (raises if it is absent: there is no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m cfd_inwsl_b200.build_ext`")
    lib = C.CDLL(str(p))
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(_PROTOS)


def check(rc: int, handle=None) -> None:
    if rc != CFD_OK:
        msg = ""
        if handle is not None:
            m = load().cfd_last_error(handle)
            msg = m.decode() if m else ""
        raise CfdError(rc, msg)


def ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def eval_inter5(inter_method: int, q: np.ndarray, strict: bool = True) -> np.ndarray:
    """Device interpolator on rows of q (n x 5)."""
    q = np.ascontiguousarray(q, dtype=np.float64)
    n = q.shape[0]
    out = np.empty(n)
    check(load().cfd_eval_inter5(inter_method, int(strict), ptr(q), n, ptr(out)))
    return out


def eval_flux(dim: int, ax: int, flux_method: int, lr: np.ndarray, strict: bool = True) -> np.ndarray:
    """Device Riemann flux on rows of lr (n x 2*nvar: left prim | right prim)."""
    lr = np.ascontiguousarray(lr, dtype=np.float64)
    nv = dim + 2
    n = lr.shape[0]
    out = np.empty((n, nv))
    check(load().cfd_eval_flux(dim, ax, flux_method, int(strict), ptr(lr), n, ptr(out)))
    return out


def eval_face(dim: int, ax: int, inter_method: int, prims6: np.ndarray, precision: int = 0) -> np.ndarray:
    """Device face reconstruction of n six-cell stencils (n x 6 x nvar prims) -> n x 2*nvar."""
    prims6 = np.ascontiguousarray(prims6, dtype=np.float64)
    n = prims6.shape[0]
    out = np.empty((n, 2 * (dim + 2)))
    check(load().cfd_eval_face(dim, ax, inter_method, precision, ptr(prims6), n, ptr(out)))
    return out


def accuracy_derivative(inter_method: int, q_with_ghosts: np.ndarray, h: float) -> np.ndarray:
    """Device d q / d x of the AccuracyTest composition (see cfd_accuracy_test)."""
    q = np.ascontiguousarray(q_with_ghosts, dtype=np.float64)
    n = q.size - 8
    out = np.empty(n)
    check(load().cfd_accuracy_test(inter_method, n, float(h), ptr(q), ptr(out)))
    return out
