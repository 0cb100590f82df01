"""Python mirror of the zone_FD solver interface over the GPU library.

Names follow the reference so that code written against it reads the same:

  * ``InterMethod``, ``FluxMethod``, ``DiffMethod``, ``BndType``, ``EquationType``
    mirror the enums of zone_FD/src/include/macro.hpp:33-90 (same values);
  * ``Info`` mirrors zone_FD/src/include/info.hpp (fields, ``icMax``, ``geth``,
    ``nPrim``, ``nGhostCell``);
  * ``BlockSolver`` mirrors zone_FD/src/include/blockSolver.hpp: ``solve``,
    ``RK3_SSP``, ``getTimeIntervalExplicit``, ``stepsLoopCFL``, ``timesteps``,
    with the state in the reference's AoS ``Data`` layout (``cons``/``prim``/``rhs``
    numpy arrays of shape (ncell, nvar)).

The boundary wiring follows Initializer::initBnds (initializer.cpp:743-870)
for the Euler cases; initial states are supplied by the caller (``set_cons``)
or by :func:`sod_1d` for the Sod case of Initializer::solInit
(initializer.cpp:87-109). Every computation runs in libcfdgpu.so.
"""
from __future__ import annotations

import ctypes as C
import enum
import math

import numpy as np

from . import _lib


class BndType(enum.IntEnum):  # macro.hpp:33-34
    TYPENULL = 0
    PERIODIC1D = 1
    SYMMETRY1D = 2
    DIRICLET = 3
    DIRICLET_SODL = 4
    DIRICLET_SODR = 5
    FLUXGHOST = 6
    SUPERSONICOUTLET = 7
    DoubleMachUp = 8
    ARDBND = 9
    SYMMETRYX = 10
    SYMMETRYY = 11
    SYMMETRYZ = 12          # extension: 3D mirror in z
    PERIODIC_WRAP = 100     # extension: PERIODIC1D wired as a true wrap


class InterMethod(enum.IntEnum):  # macro.hpp:37-78
    FIRSTORDER = 0
    MUSCL = 1
    WCNS5 = 2
    WCNSZ5 = 3
    WCNS5Char = 4
    WCNSZ5Char = 5
    WCNS5CONG = 6
    TCNSCongA = 7
    WCNS5CONGZ = 8
    WCNS5CONGZCT4 = 9
    WCNS5CONGZCT7 = 10
    TCNS5 = 11
    TCNS5CT4 = 12
    TCNS5CT7 = 13
    LINEAR5 = 14
    MUCSLIN5 = 15
    INTERMAX = 16
    whfTCNSN = 17
    whfTCNSNA = 18
    whfTCNSNAS = 19
    whfTCNSNS = 20
    whfTCNSNLAD = 21
    congTCNS5CT5 = 22
    congTCNS5CT10 = 23
    whfAITCNSNS = 24
    whfAITCNSNA = 25
    whfAITCNSNAS_1 = 26
    whfAITCNSNAS_2 = 27
    whfAITCNSNLADS = 28
    whfAITCNSNAZS = 29
    whfAITCNSNmyASF002_1 = 30
    whfAITCNSNmyASF002_2 = 31
    whfAITCNSNmyASF002_ai1 = 32
    whfzycTCNSNmyASF002_1 = 33
    whfCOMPARE = 34
    new_TCNS5 = 35
    new_WHFTCNSA = 36
    new_WCNS5CONGZ = 37
    new_WHFTCNSASF203_NoS = 38
    new_WHFTCNSASF202_NoS = 39


class DiffMethod(enum.IntEnum):  # macro.hpp:82
    HDS6 = 0
    TRAD6 = 1
    TRAD2 = 2
    MND6 = 3


class EquationType(enum.IntEnum):  # macro.hpp:84
    LINEARCONV1D = 0
    BURGERS1D = 1
    EULER = 2
    ACCURACYTEST = 3


class SourceType(enum.IntEnum):  # macro.hpp:90
    SOURCENULL = 0
    GRAVITY = 1


class FluxMethod(enum.IntEnum):  # macro.hpp:86
    HLLC = 0
    ROE = 1


GAMMA = 1.4  # macro.hpp:28


class Info:
    """Mirror of the reference's Info (info.hpp:4-66) with its defaults."""

    def __init__(self):
        self.spMethod = InterMethod.WCNS5
        self.eqType = EquationType.EULER
        self.nCase = 2
        self.t = 0.0
        self.dt = 0.0001
        self.step = 0
        self.endStep = 25000
        self.outputInterval = 100
        self.outputDt = 0.01
        self.outputT = 0.0
        self.CFL = 0.5
        self.diffMethod = DiffMethod.MND6
        self.interMethod = InterMethod.WCNS5
        self.fluxMethod = FluxMethod.ROE
        self.sourceType = SourceType.SOURCENULL
        self.iMax = [201, 201, 2]
        self.calZone = [0.0, 0.3, 0.0, 0.3, 0.0, 2.0]
        self.constH = True
        self.dim = self.getDim()
        # GPU-only knobs (no counterpart in the reference)
        self.strict = False     # bitwise-parity build of the kernels
        self.precision = 0      # 0: FP64, 1: mixed FP32 reconstruction / FP64 state (CFD_PREC_MIXED)
        self.device = 0
        self.seg_len = [0, 0, 0]
        self.positivity = 0     # 1: the 1D positivity limiter on 2D/3D face states (cfd_config.positivity)

    def getDim(self) -> int:  # info.cpp:103-114
        return sum(1 for i in range(3) if self.iMax[i] > 2)

    def icMax(self) -> list[int]:  # info.cpp:117-129
        return [1 if self.iMax[i] < 2 else self.iMax[i] - 1 for i in range(3)]

    def geth(self, idim: int) -> float:  # info.cpp:359-365 with constH (initializer.cpp:604-609)
        if self.constH:
            return (self.calZone[1] - self.calZone[0]) / (self.iMax[0] - 1)
        return (self.calZone[2 * idim + 1] - self.calZone[2 * idim]) / (self.iMax[idim] - 1)

    def nPrim(self) -> int:
        return {1: 3, 2: 4, 3: 5}[self.dim]

    nCons = nPrim

    def nGhostCell(self) -> int:  # info.cpp:7-22 (spMethod WCNS5)
        return {DiffMethod.MND6: 4, DiffMethod.TRAD6: 5, DiffMethod.HDS6: 3}.get(DiffMethod(self.diffMethod), 0)


# BndTypes whose OneDBnd::update is a no-op (the ghosts keep static data set by
# OneDBnd::setValue): cfd_config.bc cannot wire them by itself.
STATIC_BND_TYPES = frozenset({BndType.TYPENULL, BndType.DIRICLET, BndType.DIRICLET_SODL, BndType.DIRICLET_SODR,
                              BndType.FLUXGHOST, BndType.ARDBND})


def default_bc_types(info: Info) -> list[list[int]]:
    """Per direction/side BndType of Initializer::initBnds for Euler
    (initializer.cpp:775-811): outlets by default, mirrors for nCase 2,
    SYMMETRYX/DIRICLET for nCase 3 (RTI), PERIODIC1D for nCase 6."""
    bc = [[BndType.SUPERSONICOUTLET] * 2 for _ in range(3)]
    if info.dim == 1:
        if info.nCase == 4:
            bc[0] = [BndType.SYMMETRY1D] * 2
    else:
        if info.nCase == 2:
            bc[0] = [BndType.SYMMETRYX] * 2
            bc[1] = [BndType.SYMMETRYY] * 2
        elif info.nCase == 3:
            bc[0] = [BndType.SYMMETRYX] * 2
            bc[1] = [BndType.DIRICLET] * 2
        elif info.nCase == 6:
            bc = [[BndType.PERIODIC1D] * 2 for _ in range(3)]
    return bc


def make_config(info: Info, bc=None, periodic: bool = False) -> _lib.CfdConfig:
    """cfd_config from an Info, with the Initializer::initBnds boundary types
    unless bc ([[lo, hi], ...]) or periodic=True overrides them."""
    lib = _lib.load()
    n = info.icMax()
    cfg = _lib.CfdConfig()
    lib.cfd_config_default(C.byref(cfg))
    cfg.dim = info.dim
    for d in range(3):
        cfg.n[d] = n[d] if d < info.dim else 1
        cfg.h[d] = info.geth(d)
        cfg.x0[d] = info.calZone[2 * d]
        cfg.seg_len[d] = int(info.seg_len[d])
    cfg.inter_method = int(info.interMethod)
    cfg.flux_method = int(info.fluxMethod)
    cfg.diff_method = int(info.diffMethod)
    cfg.n_ghost = info.nGhostCell()
    cfg.strict = int(bool(info.strict))
    cfg.precision = int(getattr(info, "precision", 0))
    cfg.device = int(info.device)
    cfg.source_type = int(getattr(info, "sourceType", 0))
    cfg.positivity = int(getattr(info, "positivity", 0))
    types = bc if bc is not None else default_bc_types(info)
    if periodic:
        types = [[BndType.PERIODIC_WRAP] * 2 for _ in range(3)]
    # sides of a named case whose lines wire_case_bnds sets one by one
    per_line = bc is None and not periodic and info.dim == 2 and info.nCase in (3, 4)
    for d in range(3):
        for s in range(2):
            t = int(types[d][s])
            if d < info.dim and t in STATIC_BND_TYPES:
                if not per_line:
                    raise ValueError(f"boundary type {BndType(t).name} (direction {d}, side {s}) needs ghost "
                                     "values per line: wire it with set_line_bc")
                # provisional wiring of cfd_create; wire_case_bnds replaces every line of this side
                t = int(BndType.SUPERSONICOUTLET)
            cfg.bc[d][s] = t
    return cfg


def _set_line_bc(lib, h, nvar, idim, i, j, side, bnd_type, i0=0, offset=0, ghost_prim=None, nghost=4):
    gp = None
    if ghost_prim is not None:
        gp = np.ascontiguousarray(np.broadcast_to(np.asarray(ghost_prim, dtype=np.float64), (nghost, nvar)))
    _lib.check(lib.cfd_set_line_bc(h, idim, i, j, side, int(bnd_type), int(i0), int(offset),
                                   _lib.ptr(gp) if gp is not None else None), h)


def wire_case_bnds(lib, h, info: Info):
    """The per-line boundary wiring Initializer::initBnds gives a named 2D case
    beyond its per-direction types: the RTI Dirichlet values (nCase 3,
    initializer.cpp:831-861) and Initializer::initDoubleMachBnds (nCase 4,
    initializer.cpp:880-943)."""
    if info.dim != 2 or info.nCase not in (3, 4):
        return
    n = info.icMax()
    nx, ny = n[0], n[1]
    nv = info.nPrim()
    ng = info.nGhostCell()
    if info.nCase == 3:
        for i in range(nx):
            _set_line_bc(lib, h, nv, 2, i, 0, 0, BndType.DIRICLET, i, nx, [2.0, 0, 0, 1.0], nghost=ng)
            _set_line_bc(lib, h, nv, 2, i, 0, 1, BndType.DIRICLET, i + (ny - 1) * nx, -nx, [1.0, 0, 0, 2.5],
                         nghost=ng)
        return
    post = [8.0, 8.25 * math.cos(math.pi / 6), -8.25 * math.sin(math.pi / 6), 116.5]
    hx = info.geth(0)
    for j in range(ny):
        _set_line_bc(lib, h, nv, 1, j, 0, 0, BndType.DIRICLET, j * nx, 1, post, nghost=ng)
        _set_line_bc(lib, h, nv, 1, j, 0, 1, BndType.SUPERSONICOUTLET, j * nx + nx - 1, -1, nghost=ng)
    for i in range(nx):
        x = info.calZone[0] + (i + 0.5) * hx  # Block::coorCel as initializer.cpp:677 fills it
        if x < 1.0 / 6.0:
            _set_line_bc(lib, h, nv, 2, i, 0, 0, BndType.DIRICLET, i, nx, post, nghost=ng)
        else:
            _set_line_bc(lib, h, nv, 2, i, 0, 0, BndType.SYMMETRYY, i, nx, nghost=ng)
        _set_line_bc(lib, h, nv, 2, i, 0, 1, BndType.DoubleMachUp, i + (ny - 1) * nx, -nx, nghost=ng)


class BlockSolver:
    """GPU counterpart of BlockSolver (blockSolver.hpp:7-57) for the Euler path.

    ``bc`` overrides the per-direction boundary types ([[lo, hi], ...]);
    ``periodic=True`` wires every direction as a true periodic wrap.
    """

    def __init__(self, info: Info, bc=None, periodic: bool = False):
        self.info = info
        self.lib = _lib.load()
        self.dim = info.dim
        self.nvar = info.nPrim()
        self.n = info.icMax()
        self.ncell = self.n[0] * self.n[1] * self.n[2]
        self.timesteps = 0
        cfg = make_config(info, bc, periodic)
        self.cfg = cfg
        h = C.c_void_p()
        rc = self.lib.cfd_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise _lib.CfdError(rc, "cfd_create")
        self.h = h
        if bc is None and not periodic:
            wire_case_bnds(self.lib, self.h, info)

    # --- lifetime
    def close(self):
        if getattr(self, "h", None):
            self.lib.cfd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- boundary wiring
    def set_line_bc(self, idim: int, i: int, j: int, side: int, bnd_type: int, i0: int = 0, offset: int = 0,
                    ghost_prim=None):
        """Mirror of OneDBnd::setUpdate/setValue for one line end (idim 1-based)."""
        _set_line_bc(self.lib, self.h, self.nvar, idim, i, j, side, bnd_type, i0, offset, ghost_prim,
                     self.info.nGhostCell())

    # --- state access (reference AoS layout)
    def set_cons(self, cons: np.ndarray):
        a = np.ascontiguousarray(cons, dtype=np.float64).reshape(self.ncell, self.nvar)
        _lib.check(self.lib.cfd_upload_cons(self.h, _lib.ptr(a)), self.h)

    @property
    def cons(self) -> np.ndarray:
        out = np.empty((self.ncell, self.nvar))
        _lib.check(self.lib.cfd_download_cons(self.h, _lib.ptr(out)), self.h)
        return out

    @property
    def prim(self) -> np.ndarray:
        out = np.empty((self.ncell, self.nvar))
        _lib.check(self.lib.cfd_download_prim(self.h, _lib.ptr(out)), self.h)
        return out

    def rhsSolve(self) -> np.ndarray:
        """One RHS evaluation at info.t (RK3_SSP's per-stage body)."""
        out = np.empty((self.ncell, self.nvar))
        _lib.check(self.lib.cfd_rhs(self.h, float(self.info.t), _lib.ptr(out)), self.h)
        return out

    # --- time stepping
    def getTimeIntervalExplicit(self) -> float:
        dt = C.c_double()
        _lib.check(self.lib.cfd_max_dt(self.h, float(self.info.CFL), C.byref(dt)), self.h)
        return dt.value

    def RK3_SSP(self, dt: float) -> float:
        """One SSP-RK3 step; returns max |R_rho| of the last stage. Leaves info.t
        where the reference's RK3_SSP leaves it (t + dt - dt/2 - dt/2)."""
        linf = C.c_double()
        _lib.check(self.lib.cfd_rk3_step(self.h, float(dt), float(self.info.t), C.byref(linf)), self.h)
        self.info.t = ((self.info.t + dt) - dt / 2) - dt / 2
        return linf.value

    def solve(self, dt: float) -> float:
        linf = self.RK3_SSP(dt)
        self.info.t += dt
        return linf

    def stepsLoopCFL(self, max_steps: int = 1 << 30, record: bool = False):
        """BlockSolver::stepsLoopCFL (blockSolver.cpp:170-235) without output files:
        steps until info.step reaches info.endStep. Returns (dts, linfs) if record."""
        info = self.info
        dts, linfs = [], []
        k = 0
        while info.step < info.endStep and k < max_steps:
            dt = self.getTimeIntervalExplicit()
            if info.outputT + dt > info.outputDt:
                dt = info.outputDt - info.outputT
                info.outputT = 0.0
                info.step += 1
            else:
                info.outputT += dt
            linf = self.solve(dt)
            self.timesteps += 1
            k += 1
            if record:
                dts.append(dt)
                linfs.append(linf)
        return (np.array(dts), np.array(linfs)) if record else None

    # --- checkpoint / restart (cfd_save_checkpoint / cfd_load_checkpoint)
    def save_checkpoint(self, path) -> None:
        """Write the state with info.t and info.step."""
        _lib.check(self.lib.cfd_save_checkpoint(self.h, str(path).encode(), float(self.info.t), int(self.info.step)),
                   self.h)

    def load_checkpoint(self, path) -> None:
        """Read a state written by save_checkpoint; restores info.t and info.step."""
        t, step = C.c_double(), C.c_longlong()
        _lib.check(self.lib.cfd_load_checkpoint(self.h, str(path).encode(), C.byref(t), C.byref(step)), self.h)
        self.info.t = t.value
        self.info.step = step.value

    # --- discrete adjoint (no counterpart in the reference)
    def rhs_vjp(self, mu: np.ndarray) -> np.ndarray:
        """(dR/dU)^T mu at the current state (cfd_rhs_vjp); mu, result: AoS (ncell, nvar)."""
        m = np.ascontiguousarray(mu, dtype=np.float64).reshape(self.ncell, self.nvar)
        out = np.empty_like(m)
        _lib.check(self.lib.cfd_rhs_vjp(self.h, _lib.ptr(m), _lib.ptr(out)), self.h)
        return out

    def adjoint_record(self, dt: float, nsteps: int, ckpt_every: int = 20):
        """Forward run of nsteps frozen-dt RK3 steps with checkpoints (cfd_adjoint_record)."""
        _lib.check(self.lib.cfd_adjoint_record(self.h, float(dt), int(nsteps), int(ckpt_every)), self.h)

    def adjoint_reverse(self, dJ_dUN: np.ndarray) -> np.ndarray:
        """dJ/dU^0 from dJ/dU^N of the recorded run (cfd_adjoint_reverse)."""
        g = np.ascontiguousarray(dJ_dUN, dtype=np.float64).reshape(self.ncell, self.nvar)
        out = np.empty_like(g)
        _lib.check(self.lib.cfd_adjoint_reverse(self.h, _lib.ptr(g), _lib.ptr(out)), self.h)
        return out

    def run_device(self, max_steps: int = 1 << 30):
        """Device-resident stepsLoopCFL (cfd_run): returns (dts, linfs)."""
        info = self.info
        t = C.c_double(info.t)
        ns = C.c_int()
        cap = min(max_steps, 1 << 22)
        dts = np.zeros(cap)
        lin = np.zeros(cap)
        rc = self.lib.cfd_run(self.h, float(info.CFL), int(info.endStep - info.step), float(info.outputDt), cap,
                              C.byref(t), C.byref(ns), _lib.ptr(dts), _lib.ptr(lin))
        _lib.check(rc, self.h)
        info.t = t.value
        self.timesteps += ns.value
        return dts[: ns.value], lin[: ns.value]


class BlockBatch:
    """Many independent BlockSolver cases advanced together (cfd_batch_*).

    infos: one Info per case (same dim, scheme, flux, flavour, precision);
    grids, spacings and boundaries may differ."""

    def __init__(self, infos, bc=None, periodic: bool = False):
        self.lib = _lib.load()
        self.infos = list(infos)
        n = len(self.infos)
        cfgs = (_lib.CfdConfig * n)()
        for i, info in enumerate(self.infos):
            cfgs[i] = make_config(info, bc, periodic)
        h = C.c_void_p()
        rc = self.lib.cfd_batch_create(cfgs, n, C.byref(h))
        if rc != 0:
            raise _lib.CfdError(rc, "cfd_batch_create")
        self.h = h
        self.ncases = n
        self.cases = []
        for i in range(n):
            ch = C.c_void_p()
            _lib.check(self.lib.cfd_batch_case(self.h, i, C.byref(ch)))
            self.cases.append(ch)
            if bc is None and not periodic:
                wire_case_bnds(self.lib, ch, self.infos[i])

    def close(self):
        if getattr(self, "h", None):
            self.lib.cfd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _shape(self, i):
        info = self.infos[i]
        n = info.icMax()
        return n[0] * n[1] * n[2], info.nPrim()

    def set_line_bc(self, case: int, idim: int, i: int, j: int, side: int, bnd_type: int, i0: int = 0,
                    offset: int = 0, ghost_prim=None):
        """BlockSolver.set_line_bc on one case of the batch."""
        _set_line_bc(self.lib, self.cases[case], self._shape(case)[1], idim, i, j, side, bnd_type, i0, offset,
                     ghost_prim, self.infos[case].nGhostCell())

    def set_cons(self, i, cons):
        nc, nv = self._shape(i)
        a = np.ascontiguousarray(cons, dtype=np.float64).reshape(nc, nv)
        _lib.check(self.lib.cfd_upload_cons(self.cases[i], _lib.ptr(a)), self.cases[i])

    def cons(self, i) -> np.ndarray:
        nc, nv = self._shape(i)
        out = np.empty((nc, nv))
        _lib.check(self.lib.cfd_download_cons(self.cases[i], _lib.ptr(out)), self.cases[i])
        return out

    def run(self, output_dt, end_step: int = 1, max_steps: int = 1 << 30, cfl: float = None):
        """Advance every case (stepsLoopCFL per case); returns (t, nsteps) arrays."""
        od = np.ascontiguousarray(np.broadcast_to(np.asarray(output_dt, dtype=np.float64), (self.ncases,)))
        t = np.ascontiguousarray([info.t for info in self.infos], dtype=np.float64)
        ns = np.zeros(self.ncases, dtype=np.int32)
        cfl = self.infos[0].CFL if cfl is None else cfl
        rc = self.lib.cfd_batch_run(self.h, float(cfl), int(end_step), _lib.ptr(od), int(max_steps), _lib.ptr(t),
                                    _lib.ptr(ns))
        if rc != 0:
            m = self.lib.cfd_batch_last_error(self.h)
            raise _lib.CfdError(rc, m.decode() if m else "")
        for info, tt in zip(self.infos, t):
            info.t = float(tt)
        return t, ns

    def set_tiling(self, idim: int, shape: int = 0, segments: int = 1, one_cta: bool = False):
        """cfd_batch_set_tiling for the sweeps along idim (1-based)."""
        rc = self.lib.cfd_batch_set_tiling(self.h, int(idim), int(shape), int(segments), int(bool(one_cta)))
        if rc != 0:
            m = self.lib.cfd_batch_last_error(self.h)
            raise _lib.CfdError(rc, m.decode() if m else "")

    def autotune(self) -> list[dict]:
        """cfd_batch_autotune: per direction, the tiling it chose and the
        chosen first-stage sweep's time."""
        dim = self.infos[0].dim
        choice = np.zeros(9, dtype=np.int32)
        ms = np.zeros(3)
        rc = self.lib.cfd_batch_autotune(self.h, _lib.ptr(choice), _lib.ptr(ms))
        if rc != 0:
            m = self.lib.cfd_batch_last_error(self.h)
            raise _lib.CfdError(rc, m.decode() if m else "")
        return [{"shape": int(choice[3 * d]), "segments_per_line": int(choice[3 * d + 1]),
                 "one_cta_per_sm": bool(choice[3 * d + 2]), "sweep_ms": float(ms[d])} for d in range(dim)]


def sod_1d(info: Info) -> np.ndarray:
    """Sod initial state of Initializer::solInit (initializer.cpp:87-109):
    (1, 0, 1) for x < 0, (0.125, 0, 0.1) otherwise, cell centres
    calZone[0] + (i + 1/2) h. Returns cons (ncell, 3)."""
    n = info.icMax()[0]
    h = info.geth(0)
    out = np.empty((n, 3))
    gamma = 1.4
    for i in range(n):
        x = info.calZone[0] + (i + 0.5) * h
        if x < 0:
            out[i] = (1.0, 0.0, 1.0 / (gamma - 1) * 1)
        else:
            out[i] = (0.125, 0.0, 1.0 / (gamma - 1) * 0.1)
    return out


def prim_to_cons(prim: np.ndarray) -> np.ndarray:
    """(rho, u[, v[, w]], p) -> (rho, rho u, ..., rho E) with E = p/(gamma-1)/rho + |u|^2/2."""
    prim = np.asarray(prim, dtype=np.float64)
    nv = prim.shape[-1]
    r = prim[..., 0]
    vel = prim[..., 1:nv - 1]
    p = prim[..., nv - 1]
    out = np.empty_like(prim)
    out[..., 0] = r
    out[..., 1:nv - 1] = r[..., None] * vel
    out[..., nv - 1] = p / (GAMMA - 1) + 0.5 * r * np.sum(vel * vel, axis=-1)
    return out



# --------------------------------------------------------------------- checkpoint files
CKPT_HEADER = np.dtype([("magic", "S8"), ("version", "<u4"), ("dim", "<u4"), ("n", "<i8", 3), ("nvar", "<u4"),
                        ("inter_method", "<i4"), ("flux_method", "<i4"), ("pad", "<i4"), ("gamma", "<f8"),
                        ("h", "<f8", 3), ("t", "<f8"), ("step", "<i8")])


def _fnv1a(data: bytes, h: int = 14695981039346656037) -> int:
    a = np.frombuffer(data, dtype=np.uint8)
    for b in a.tolist():
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def read_checkpoint(path, verify: bool = True):
    """(header dict, cons (ncell, nvar)) of a checkpoint file; raises ValueError
    on a bad magic, version or size, and (verify=True) a bad checksum. The
    checksum runs byte by byte in Python: pass verify=False for large files
    (cfd_load_checkpoint always verifies)."""
    raw = open(path, "rb").read()
    if len(raw) < CKPT_HEADER.itemsize + 8:
        raise ValueError("truncated checkpoint")
    hd = np.frombuffer(raw[:CKPT_HEADER.itemsize], dtype=CKPT_HEADER)[0]
    if hd["magic"] != b"CFDGPUCK" or hd["version"] != 1:
        raise ValueError("not a version-1 checkpoint")
    n = [int(x) for x in hd["n"]]
    count = n[0] * n[1] * n[2] * int(hd["nvar"])
    end = CKPT_HEADER.itemsize + 8 * count
    if len(raw) != end + 8:
        raise ValueError("checkpoint size does not match its header")
    stored = int(np.frombuffer(raw[end:end + 8], dtype="<u8")[0])
    if verify and _fnv1a(raw[:end]) != stored:
        raise ValueError("checkpoint checksum mismatch")
    cons = np.frombuffer(raw[CKPT_HEADER.itemsize:end], dtype="<f8").reshape(-1, int(hd["nvar"])).copy()
    meta = {k: hd[k] for k in CKPT_HEADER.names if k not in ("magic", "pad")}
    return meta, cons


def write_checkpoint(path, info: Info, cons: np.ndarray) -> None:
    """The file cfd_save_checkpoint writes, from the host (same layout and checksum)."""
    hd = np.zeros((), dtype=CKPT_HEADER)
    hd["magic"] = b"CFDGPUCK"
    hd["version"] = 1
    hd["dim"] = info.dim
    n = info.icMax()
    hd["n"] = [n[d] if d < info.dim else 1 for d in range(3)]
    hd["nvar"] = info.nPrim()
    hd["inter_method"] = int(info.interMethod)
    hd["flux_method"] = int(info.fluxMethod)
    hd["gamma"] = 1.4
    hd["h"] = [info.geth(d) for d in range(3)]
    hd["t"] = info.t
    hd["step"] = info.step
    body = hd.tobytes() + np.ascontiguousarray(cons, dtype="<f8").tobytes()
    with open(path, "wb") as f:
        f.write(body + np.array([_fnv1a(body)], dtype="<u8").tobytes())
