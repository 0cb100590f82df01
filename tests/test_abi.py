"""The C-ABI library loads and exports every entry point include/cfdgpu.h declares (CPU only)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from cfd_inwsl_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "cfdgpu.h"


def declared_functions():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(cfd_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_expected_entry_points():
    names = declared_functions()
    for must in ("cfd_create", "cfd_destroy", "cfd_rhs", "cfd_rk3_step", "cfd_max_dt", "cfd_run",
                 "cfd_upload_cons", "cfd_download_cons", "cfd_set_line_bc", "cfd_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def _cfg(**kw):
    lib = _lib.load()
    cfg = _lib.CfdConfig()
    lib.cfd_config_default(C.byref(cfg))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return lib, cfg


@pytest.mark.parametrize("field,value,code", [
    ("n_ghost", 3, -6), ("gamma", 1.3, -6), ("diff_method", 1, -6), ("diff_method", 2, -6), ("diff_method", 0, -6),
    ("precision", 7, -1),
    ("dim", 4, -1), ("inter_method", 99, -6), ("flux_method", 5, -1),
])
def test_config_validation_without_gpu(field, value, code):
    lib, cfg = _cfg(**{field: value})
    h = C.c_void_p()
    assert lib.cfd_create(C.byref(cfg), C.byref(h)) == code
    assert not h.value


def test_trad6_needs_five_ghosts_and_fp64():
    """TRAD6 (diff_method 1) with n_ghost 4 or the mixed form is refused before
    any device call; with n_ghost 5 in FP64 it passes validation (and then
    needs a device)."""
    lib, cfg = _cfg(diff_method=1, n_ghost=5, precision=1)
    h = C.c_void_p()
    assert lib.cfd_create(C.byref(cfg), C.byref(h)) == -6
    lib, cfg = _cfg(diff_method=3, n_ghost=5)
    assert lib.cfd_create(C.byref(cfg), C.byref(h)) == -6


def test_small_grid_rejected():
    lib, cfg = _cfg()
    cfg.n[0] = 4
    h = C.c_void_p()
    assert lib.cfd_create(C.byref(cfg), C.byref(h)) == -1


def test_version_string():
    assert b"sm_100a" in _lib.load().cfd_version()
