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


@pytest.mark.parametrize("dim,d,value", [
    (2, 1, 101),  # CFD_BND_HALO: wired by cfd_enable_halo only
    (2, 0, 3),    # DIRICLET: needs ghost values per line
    (2, 1, 0),    # TYPENULL: static data as well
    (2, 0, 57),   # not a BndType
    (2, 0, 2),    # SYMMETRY1D outside 1D leaves the pressure ghost undefined
    (2, 1, 12),   # SYMMETRYZ in 2D
    (3, 2, 8),    # DoubleMachUp is a 2D boundary
    (1, 0, 11),   # SYMMETRYY in 1D
])
def test_config_boundary_types_rejected_without_gpu(dim, d, value):
    """cfg->bc may only hold types the configuration can wire by itself; the
    rest is refused with CFD_ERR_CONFIG before any device call, by cfd_create
    and by the allocation-free entry point (dummy pointers: nothing is read)."""
    lib, cfg = _cfg(dim=dim)
    for k in range(3):
        cfg.n[k] = 16 if k < dim else 1
    cfg.bc[d][1] = value
    h = C.c_void_p()
    assert lib.cfd_create(C.byref(cfg), C.byref(h)) == -1
    assert not h.value
    dummy = C.c_void_p(0x1000)
    assert lib.cfd_rhs_noalloc(C.byref(cfg), dummy, dummy, C.c_double(0.0), None) == -1


def test_valid_boundary_types_pass_validation_without_gpu():
    """Accepted types get past validation and fail only at the first CUDA call
    here (no device): CFD_ERR_CUDA, not CFD_ERR_CONFIG."""
    if _lib_has_gpu():
        pytest.skip("a device is present")
    for dim, types in ((1, [2, 7]), (2, [1, 7, 10, 11, 8, 100]), (3, [12, 10, 11, 100])):
        lib, cfg = _cfg(dim=dim)
        for k in range(3):
            cfg.n[k] = 16 if k < dim else 1
        for t in types:
            for d in range(dim):
                if t == 8 and d != 1:
                    continue
                cfg.bc[d][0] = t
                h = C.c_void_p()
                assert lib.cfd_create(C.byref(cfg), C.byref(h)) == -2, (dim, d, t)
                cfg.bc[d][0] = 7


def _lib_has_gpu():
    from tests.conftest import gpu_available
    return gpu_available()


def test_make_config_refuses_static_types_without_per_line_wiring():
    from cfd_inwsl_b200 import zone
    info = zone.Info()
    info.dim = 2
    info.iMax = [17, 17, 1]
    with pytest.raises(ValueError):
        zone.make_config(info, bc=[[zone.BndType.DIRICLET] * 2, [7, 7], [7, 7]])
    info.nCase = 3  # RTI: the Dirichlet rows are wired line by line after cfd_create
    cfg = zone.make_config(info)
    assert list(cfg.bc[1]) == [int(zone.BndType.SUPERSONICOUTLET)] * 2
