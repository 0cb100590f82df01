"""ORACLE / TEST INFRASTRUCTURE ONLY.

ctypes wrapper of oracle/_ref/libcongfd_ref.so: the reference zone_FD solver
compiled unmodified from its own sources (zone_FD/src/src/*.cpp) by
oracle/Makefile, plus the C harness in oracle/ref_capi.cpp. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may use this module;
the product path never does.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libcongfd_ref.so"


class RefCfg(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int * 3), ("zone", C.c_double * 6), ("inter_method", C.c_int),
                ("flux_method", C.c_int), ("n_case", C.c_int), ("cfl", C.c_double), ("source_type", C.c_int),
                ("diff_method", C.c_int)]


_lib = None


def available() -> bool:
    return REF_LIB.exists()


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle` where the reference sources are present")
        lib = C.CDLL(str(REF_LIB))
        vp = C.c_void_p
        d = C.c_double
        protos = {
            "ref_create": (vp, [C.POINTER(RefCfg)]),
            "ref_destroy": (None, [vp]),
            "ref_ncells": (C.c_int, [vp]),
            "ref_nvar": (C.c_int, [vp]),
            "ref_h": (d, [vp, C.c_int]),
            "ref_time": (d, [vp]),
            "ref_set_time": (None, [vp, d]),
            "ref_set_cons": (None, [vp, vp]),
            "ref_get_cons": (None, [vp, vp]),
            "ref_get_prim": (None, [vp, vp]),
            "ref_rhs": (None, [vp, vp]),
            "ref_max_dt": (d, [vp]),
            "ref_rk3": (None, [vp, d]),
            "ref_rho_linf": (d, [vp]),
            "ref_run": (C.c_int, [vp, C.c_int, d, C.c_int, vp, vp]),
            "ref_set_line_bc": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp]),
            "ref_inter5": (d, [C.c_int, vp]),
            "ref_flux2d": (None, [C.c_int, vp, C.c_int, vp]),
            "ref_flux1d": (None, [C.c_int, vp, vp]),
            "ref_set_threads": (None, [C.c_int]),
            "ref_recon_face": (C.c_int, [C.c_int, C.c_int, C.c_int, vp, vp]),
        }
        for name, (res, args) in protos.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float64
    return C.c_void_p(a.ctypes.data)


class RefSolver:
    """The reference BlockSolver driven through the harness.

    dim/n: grid (cells); zone: Info::calZone; n_case selects the reference's
    initial state and boundary wiring (Initializer); periodic=True rewires every
    line end to a true wrap (PERIODIC1D with i0/offset pointing at the far end).
    """

    def __init__(self, dim, n, zone, inter_method=2, flux_method=0, n_case=0, cfl=0.5, periodic=False, threads=None,
                 source_type=0, diff_method=3):
        self.lib = load()
        if threads is not None:
            self.lib.ref_set_threads(int(threads))
        n3 = list(n) + [1] * (3 - len(n))
        cfg = RefCfg(dim, (C.c_int * 3)(*n3), (C.c_double * 6)(*zone), inter_method, flux_method, n_case, cfl,
                     source_type, diff_method)
        self.h = self.lib.ref_create(C.byref(cfg))
        self.ng = 5 if diff_method == 1 else 4  # Info::nGhostCell (info.cpp:7-22)
        self.dim = dim
        self.n = n3
        self.ncell = self.lib.ref_ncells(self.h)
        self.nvar = self.lib.ref_nvar(self.h)
        if periodic:
            self.wire_periodic()

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def wire_periodic(self):
        nx, ny = self.n[0], self.n[1]
        if self.dim == 1:
            self.lib.ref_set_line_bc(self.h, 1, 0, 0, 0, 1, nx - 1, -1, None)
            self.lib.ref_set_line_bc(self.h, 1, 0, 0, 1, 1, 0, 1, None)
            return
        for j in range(ny):
            self.lib.ref_set_line_bc(self.h, 1, j, 0, 0, 1, j * nx + nx - 1, -1, None)
            self.lib.ref_set_line_bc(self.h, 1, j, 0, 1, 1, j * nx, 1, None)
        for i in range(nx):
            self.lib.ref_set_line_bc(self.h, 2, i, 0, 0, 1, i + (ny - 1) * nx, -nx, None)
            self.lib.ref_set_line_bc(self.h, 2, i, 0, 1, 1, i, nx, None)

    def set_line_bc(self, idim, i, j, side, typ, i0, offset, values=None):
        v = None if values is None else np.ascontiguousarray(np.broadcast_to(np.asarray(values, float), (self.ng, self.nvar)))
        rc = self.lib.ref_set_line_bc(self.h, idim, i, j, side, int(typ), int(i0), int(offset),
                                      _p(v) if v is not None else None)
        assert rc == 0

    @property
    def cons(self) -> np.ndarray:
        a = np.empty((self.ncell, self.nvar))
        self.lib.ref_get_cons(self.h, _p(a))
        return a

    @cons.setter
    def cons(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64).reshape(self.ncell, self.nvar)
        self.lib.ref_set_cons(self.h, _p(a))

    @property
    def prim(self) -> np.ndarray:
        a = np.empty((self.ncell, self.nvar))
        self.lib.ref_get_prim(self.h, _p(a))
        return a

    @property
    def t(self) -> float:
        return self.lib.ref_time(self.h)

    @t.setter
    def t(self, v):
        self.lib.ref_set_time(self.h, float(v))

    def rhs(self) -> np.ndarray:
        a = np.empty((self.ncell, self.nvar))
        self.lib.ref_rhs(self.h, _p(a))
        return a

    def max_dt(self) -> float:
        return self.lib.ref_max_dt(self.h)

    def solve(self, dt: float) -> float:
        self.lib.ref_rk3(self.h, float(dt))
        return self.lib.ref_rho_linf(self.h)

    def run(self, end_step: int, output_dt: float, max_steps: int = 1 << 22):
        dts = np.zeros(max_steps)
        lin = np.zeros(max_steps)
        k = self.lib.ref_run(self.h, end_step, output_dt, max_steps, _p(dts), _p(lin))
        return dts[:k], lin[:k]


def ref_inter5(inter_method: int, q: np.ndarray) -> np.ndarray:
    lib = load()
    q = np.ascontiguousarray(q, dtype=np.float64)
    return np.array([lib.ref_inter5(inter_method, C.c_void_p(q[i].ctypes.data)) for i in range(q.shape[0])])


def ref_flux(dim: int, ax: int, flux_method: int, lr: np.ndarray) -> np.ndarray:
    lib = load()
    lr = np.ascontiguousarray(lr, dtype=np.float64)
    nv = dim + 2
    out = np.empty((lr.shape[0], nv))
    for i in range(lr.shape[0]):
        row = np.ascontiguousarray(lr[i])
        o = np.empty(nv)
        if dim == 1:
            lib.ref_flux1d(flux_method, _p(row), _p(o))
        else:
            lib.ref_flux2d(flux_method, _p(row), int(ax == 1), _p(o))
        out[i] = o
    return out


def ref_recon_face(inter_method: int, dim: int, normal_y: int, prims6: np.ndarray) -> np.ndarray:
    """The reference's reconI on n six-cell stencils (n x 6 x nvar) -> n x 2 nvar."""
    lib = load()
    prims6 = np.ascontiguousarray(prims6, dtype=np.float64)
    nv = dim + 2
    out = np.empty((prims6.shape[0], 2 * nv))
    for i in range(prims6.shape[0]):
        o = np.empty(2 * nv)
        assert lib.ref_recon_face(inter_method, dim, normal_y, _p(np.ascontiguousarray(prims6[i])), _p(o)) == 0
        out[i] = o
    return out


# ---------------------------------------------------------------- C restatement
ORC_LIB = HERE / "_ref" / "libcfd_oracle.so"
ORC_OUTLET, ORC_SYMMETRY, ORC_WRAP, ORC_MIRRORCOPY = 7, 10, 100, 1
# InterMethod -> (family, constant), as the library's selector maps it
ORC_FAMILY = {2: (0, 0.0), 3: (1, 0.0), 11: (2, 1e-5), 12: (2, 1e-4), 13: (2, 1e-7), 22: (2, 1e-5),
              23: (2, 1e-10), 35: (2, 1e-5), 8: (3, 0.15704178024750198), 37: (3, 0.15704178024750198),
              9: (3, 0.23050581003334941), 10: (3, 0.072892337360747711), 15: (4, 0.0)}


class OrcCfg(C.Structure):
    _fields_ = [("dim", C.c_int), ("n", C.c_int * 3), ("h", C.c_double), ("fam", C.c_int), ("icst", C.c_double),
                ("flux", C.c_int), ("bc", (C.c_int * 2) * 3), ("threads", C.c_int), ("diff", C.c_int),
                ("posl", C.c_int)]


_orc = None


def orc_load() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORC_LIB.exists():
            raise RuntimeError(f"{ORC_LIB} missing: run `make -C oracle`")
        lib = C.CDLL(str(ORC_LIB))
        vp = C.c_void_p
        lib.orc_rhs.argtypes = [C.POINTER(OrcCfg), vp, vp]
        lib.orc_rhs.restype = None
        lib.orc_max_dt.argtypes = [C.POINTER(OrcCfg), vp, C.c_double]
        lib.orc_max_dt.restype = C.c_double
        lib.orc_rk3.argtypes = [C.POINTER(OrcCfg), vp, C.c_double]
        lib.orc_rk3.restype = C.c_double
        lib.orc_inter5.argtypes = [C.c_int, C.c_double, vp]
        lib.orc_inter5.restype = C.c_double
        _orc = lib
    return _orc


class OracleC:
    """The plain-C restatement (1D/2D/3D) on a uniform grid with per-side BC kinds."""

    def __init__(self, dim, n, h, inter_method=2, flux_method=0, bc=None, threads=0, trad6=False, positivity=False):
        self.lib = orc_load()
        fam, icst = ORC_FAMILY[inter_method]
        n3 = list(n) + [1] * (3 - len(n))
        bcs = bc if bc is not None else [[ORC_OUTLET] * 2] * 3
        arr = ((C.c_int * 2) * 3)(*[(C.c_int * 2)(*bcs[d]) for d in range(3)])
        self.cfg = OrcCfg(dim, (C.c_int * 3)(*n3), h, fam, icst, flux_method, arr, threads, int(bool(trad6)),
                          int(bool(positivity)))
        self.nvar = dim + 2
        self.ncell = n3[0] * n3[1] * n3[2]
        self.cons = None

    def rhs(self, cons=None) -> np.ndarray:
        u = np.ascontiguousarray(self.cons if cons is None else cons, dtype=np.float64)
        out = np.empty((self.ncell, self.nvar))
        self.lib.orc_rhs(C.byref(self.cfg), _p(u), _p(out))
        return out

    def max_dt(self, cfl) -> float:
        return self.lib.orc_max_dt(C.byref(self.cfg), _p(np.ascontiguousarray(self.cons)), cfl)

    def solve(self, dt) -> float:
        self.cons = np.ascontiguousarray(self.cons, dtype=np.float64).copy()
        return self.lib.orc_rk3(C.byref(self.cfg), _p(self.cons), float(dt))
