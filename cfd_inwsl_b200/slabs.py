"""One grid over several GPUs: slab decomposition along the last direction.

The reference runs one block on one host (BlockSolver, blockSolver.hpp:7-57);
this module splits that block into slabs along y (2D) or z (3D), one handle
per slab, and exchanges the four boundary rows (planes) of every stage's input
state between neighbouring slabs before the stage, which is exactly the data
the reference's ghost fill (Bnds::update, bnds.cpp:23-27) would read from the
neighbouring cells of the undivided block. Results are bit for bit those of
the undivided block (strict flavour) because every ghost is an exact copy.

Two ways to run the slabs:
  * SlabGrid: every slab in this process (one GPU, or one device per slab);
    halos are device-to-device copies.
  * SlabRank: one slab per process, launched with torch.distributed (NCCL on
    GPUs, gloo for the CPU tests of the exchange); halos travel by
    point-to-point send/recv, and dt takes the maximum wave speeds over ranks.

Only per-direction boundary types are supported (a `bc` list or periodic=True):
the named cases' per-line wiring (RTI, double Mach) addresses global cells.
"""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np

from . import _lib, zone

GHOST = 4


def slab_rows(n: int, parts: int) -> list[tuple[int, int]]:
    """Contiguous row ranges [r0, r1) of n rows over `parts` slabs, sizes as even as possible."""
    base, extra = divmod(n, parts)
    out, r = [], 0
    for k in range(parts):
        m = base + (1 if k < extra else 0)
        out.append((r, r + m))
        r += m
    return out


def neighbours(k: int, parts: int, periodic: bool) -> tuple[int | None, int | None]:
    """Low and high neighbour slab of slab k (None: physical boundary)."""
    lo = k - 1 if k > 0 else (parts - 1 if periodic else None)
    hi = k + 1 if k < parts - 1 else (0 if periodic else None)
    return lo, hi


class _DevArray:
    """A device buffer of this library seen by torch without a copy."""

    def __init__(self, ptr: int, shape, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _tensor(ptr: int, shape, device, typestr: str = "<f8"):
    import torch
    return torch.as_tensor(_DevArray(ptr, shape, typestr), device=device)


class Slab:
    """One slab's handle: rows [r0, r1) of the last direction of a global grid."""

    def __init__(self, info: zone.Info, rows: tuple[int, int], halo_sides, bc=None, periodic: bool = False,
                 device: int = 0):
        self.global_info = info
        d = info.dim - 1
        self.r0, self.r1 = rows
        if self.r1 - self.r0 < GHOST + 1:
            raise ValueError("a slab needs at least 5 rows")
        loc = copy.deepcopy(info)
        h = info.geth(d)
        loc.iMax = list(info.iMax)
        loc.iMax[d] = self.r1 - self.r0 + 1
        z0 = info.calZone[2 * d]
        loc.calZone = list(info.calZone)
        loc.calZone[2 * d] = z0 + self.r0 * h
        loc.calZone[2 * d + 1] = z0 + self.r1 * h
        loc.device = device
        types = ([[zone.BndType.PERIODIC_WRAP] * 2 for _ in range(3)] if periodic
                 else [list(x) for x in (bc if bc is not None else zone.default_bc_types(info))])
        for side in (0, 1):
            if halo_sides[side]:
                types[d][side] = zone.BndType.SUPERSONICOUTLET  # rewired as halo below
        self.solver = zone.BlockSolver(loc, bc=types)
        self.lib = self.solver.lib
        self.device = device
        n = loc.icMax()
        self.nvar = loc.nPrim()
        self.nrows = n[d]
        self.rowlen = self.solver.ncell // self.nrows
        self.halo = [None, None]
        for side in (0, 1):
            if halo_sides[side]:
                ptr, cnt = C.c_void_p(), C.c_longlong()
                _lib.check(self.lib.cfd_enable_halo(self.solver.h, side, C.byref(ptr), C.byref(cnt)), self.solver.h)
                assert cnt.value == self.nvar * GHOST * self.rowlen
                self.halo[side] = _tensor(ptr.value, (self.nvar, GHOST, self.rowlen), f"cuda:{device}")

    def stage_state(self, stage: int):
        ptr = C.c_void_p()
        _lib.check(self.lib.cfd_stage_state(self.solver.h, stage, C.byref(ptr)), self.solver.h)
        return _tensor(ptr.value, (self.nvar, self.nrows, self.rowlen), f"cuda:{self.device}")

    def set_stream(self, stream):
        _lib.check(self.lib.cfd_set_stream(self.solver.h, C.c_void_p(stream.cuda_stream)), self.solver.h)

    def reduction_words(self):
        """The 4 reduction words (max |R_rho|, wave speed per direction) as an
        int64 device tensor: IEEE bit patterns of non-negative doubles, ordered
        like the integers, so a MAX all-reduce gives the global maxima."""
        ptr = C.c_void_p()
        _lib.check(self.lib.cfd_reduction_words(self.solver.h, C.byref(ptr)), self.solver.h)
        return _tensor(ptr.value, (4,), f"cuda:{self.device}", "<i8")

    def wave_speeds(self) -> np.ndarray:
        lam = np.zeros(3)
        _lib.check(self.lib.cfd_max_wave_speeds(self.solver.h, _lib.ptr(lam)), self.solver.h)
        return lam

    def stage(self, stage: int, dt: float, t: float):
        _lib.check(self.lib.cfd_rk3_stage(self.solver.h, stage, float(dt), float(t)), self.solver.h)


def words_from_wave_speeds(lam) -> np.ndarray:
    """Non-negative doubles as the int64 reduction words the library keeps
    (their IEEE bit patterns, which order like the integers)."""
    a = np.ascontiguousarray(np.asarray(lam, dtype=np.float64))
    if np.any(np.signbit(a)) or np.any(np.isnan(a)):
        raise ValueError("reduction words hold non-negative, non-NaN doubles")
    return a.view(np.int64).copy()


def wave_speeds_from_words(words) -> np.ndarray:
    """Inverse of words_from_wave_speeds."""
    return np.ascontiguousarray(np.asarray(words, dtype=np.int64)).view(np.float64).copy()


def allreduce_max_words(dist, group, words):
    """Global maxima of every rank's reduction words ([0] max |R_rho|, [1..3]
    max (c + |u_d|) / h_d), in place: a MAX all-reduce of the int64 bit
    patterns is the maximum of the doubles they encode."""
    dist.all_reduce(words, op=dist.ReduceOp.MAX, group=group)
    return words


def dt_from_words(words, dim: int, cfl: float) -> float:
    """The step the device's step control takes from the (reduced) words:
    CFL / sum_d lambda_d (getTimeIntervalExplicit, blockSolver.cpp:318-349)."""
    return dt_from_wave_speeds(wave_speeds_from_words(words)[1:1 + dim], dim, cfl)


def dt_from_wave_speeds(lam, dim: int, cfl: float) -> float:
    """getTimeIntervalExplicit's CFL / sum_d max (c + |u_d|) / h_d, summed in direction order."""
    total = 0.0
    for d in range(dim):
        total += float(lam[d])
    return cfl / total


class SlabGrid:
    """All slabs of one grid in this process; halos by device copies."""

    def __init__(self, info: zone.Info, parts: int, bc=None, periodic: bool = False, devices=None):
        self.info = info
        d = info.dim - 1
        self.d = d
        self.parts = parts
        per_dir = periodic or (bc is not None and bc[d][0] == zone.BndType.PERIODIC_WRAP)
        self.periodic_last = per_dir
        self.rows = slab_rows(info.icMax()[d], parts)
        devices = devices or [info.device] * parts
        self.nb = [neighbours(k, parts, per_dir) for k in range(parts)]
        self.slabs = [Slab(info, self.rows[k], (self.nb[k][0] is not None, self.nb[k][1] is not None), bc, periodic,
                           devices[k]) for k in range(parts)]
        import torch
        # one stream per device for the stages and the halo copies: stream order
        # makes every copy see the finished previous stage (the legacy default
        # stream would not order against the library's non-blocking streams)
        self.streams = {dev: torch.cuda.Stream(device=dev) for dev in set(devices)}
        for s in self.slabs:
            s.set_stream(self.streams[s.device])

    def set_cons(self, cons: np.ndarray):
        """Global AoS state (ncell, nvar) -> every slab's rows."""
        nv = self.info.nPrim()
        g = np.ascontiguousarray(cons).reshape(-1, self.slabs[0].rowlen, nv)
        for s, (r0, r1) in zip(self.slabs, self.rows):
            s.solver.set_cons(g[r0:r1].reshape(-1, nv))

    @property
    def cons(self) -> np.ndarray:
        return np.concatenate([s.solver.cons for s in self.slabs], 0)

    def exchange(self, stage: int):
        import torch
        states = [s.stage_state(stage) for s in self.slabs]
        for k, s in enumerate(self.slabs):
            lo, hi = self.nb[k]
            with torch.cuda.stream(self.streams[s.device]):
                if lo is not None:
                    s.halo[0].copy_(states[lo][:, -GHOST:, :])
                if hi is not None:
                    s.halo[1].copy_(states[hi][:, :GHOST, :])
        if len(self.streams) > 1:  # slabs on several devices: copies may cross streams
            for st in self.streams.values():
                st.synchronize()

    def max_dt(self, cfl: float) -> float:
        lam = np.max([s.wave_speeds() for s in self.slabs], axis=0)
        return dt_from_wave_speeds(lam, self.info.dim, cfl)

    def step(self, dt: float, t: float = 0.0):
        for stage in (1, 2, 3):
            self.exchange(stage)
            for s in self.slabs:
                s.stage(stage, dt, t)


class SlabRank:
    """This process's slab of a grid split over the ranks of a torch.distributed group."""

    def __init__(self, info: zone.Info, bc=None, periodic: bool = False, group=None, device: int = 0):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.info = info
        d = info.dim - 1
        per_dir = periodic or (bc is not None and bc[d][0] == zone.BndType.PERIODIC_WRAP)
        self.rows = slab_rows(info.icMax()[d], self.world)
        self.nb = neighbours(self.rank, self.world, per_dir)
        halo_sides = (self.nb[0] is not None, self.nb[1] is not None)
        self.slab = Slab(info, self.rows[self.rank], halo_sides, bc, periodic, device)
        import torch
        # the stages and NCCL's point-to-point calls share one stream (NCCL
        # orders its work after the current stream, set around each exchange)
        self.stream = torch.cuda.Stream(device=device)
        self.slab.set_stream(self.stream)

    def set_cons(self, cons: np.ndarray):
        """This rank's rows of the global AoS state."""
        nv = self.info.nPrim()
        g = np.ascontiguousarray(cons).reshape(-1, self.slab.rowlen, nv)
        r0, r1 = self.rows[self.rank]
        self.slab.solver.set_cons(g[r0:r1].reshape(-1, nv))

    def exchange(self, stage: int):
        import torch
        with torch.cuda.stream(self.stream):
            exchange_rows(self.dist, self.group, self.rank, self.nb, self.slab.stage_state(stage), self.slab.halo)

    def max_dt(self, cfl: float) -> float:
        import torch
        with torch.cuda.stream(self.stream):
            lam = torch.tensor(self.slab.wave_speeds(), dtype=torch.float64, device=f"cuda:{self.slab.device}")
            self.dist.all_reduce(lam, op=self.dist.ReduceOp.MAX, group=self.group)
            # read back on the same stream: a copy on torch's default stream
            # would not wait for the reduction (the streams are non-blocking)
            lam_host = lam.cpu().numpy()
        return dt_from_wave_speeds(lam_host, self.info.dim, cfl)

    def step(self, dt: float, t: float = 0.0):
        for stage in (1, 2, 3):
            self.exchange(stage)
            self.slab.stage(stage, dt, t)

    def run_device(self, steps: int, cfl: float, t: float = 0.0) -> tuple[float, int]:
        """`steps` CFL steps with dt kept on the device: per step a MAX
        all-reduce of the reduction words, then the three stages each after
        its halo exchange, all enqueued on the slab's stream with no host
        round trip (cfd_loop_*). Returns the end time and the steps taken."""
        import torch
        lib, h = self.slab.lib, self.slab.solver.h
        with torch.cuda.stream(self.stream):
            _lib.check(lib.cfd_loop_begin(h, float(cfl), float(t)), h)
            words = self.slab.reduction_words()
            for _ in range(steps):
                allreduce_max_words(self.dist, self.group, words)
                _lib.check(lib.cfd_loop_step_begin(h), h)
                for stage in (1, 2, 3):
                    exchange_rows(self.dist, self.group, self.rank, self.nb, self.slab.stage_state(stage),
                                  self.slab.halo)
                    _lib.check(lib.cfd_loop_stage(h, stage), h)
                _lib.check(lib.cfd_loop_step_end(h), h)
            t_out, n = C.c_double(), C.c_int()
            _lib.check(lib.cfd_loop_end(h, C.byref(t_out), C.byref(n)), h)
        return t_out.value, n.value


def exchange_rows(dist, group, rank, nb, state, halo):
    """Send this slab's first / last GHOST rows of `state` ([var][row][line]) to
    its low / high neighbour and receive theirs into halo[0] / halo[1].

    The order of the point-to-point operations is the same on every rank:
    send high rows, receive into the low halo, send low rows, receive into the
    high halo. When both neighbours are the same rank (two periodic slabs), the
    two messages between a pair then match in order: my high rows become its
    low halo, my low rows its high halo."""
    lo, hi = nb
    if lo == rank and hi == rank:  # one periodic slab: its own rows
        halo[0].copy_(state[:, -GHOST:, :])
        halo[1].copy_(state[:, :GHOST, :])
        return
    ops = []
    if hi is not None:
        ops.append(dist.P2POp(dist.isend, state[:, -GHOST:, :].contiguous(), hi, group))
    if lo is not None:
        ops.append(dist.P2POp(dist.irecv, halo[0], lo, group))
    if lo is not None:
        ops.append(dist.P2POp(dist.isend, state[:, :GHOST, :].contiguous(), lo, group))
    if hi is not None:
        ops.append(dist.P2POp(dist.irecv, halo[1], hi, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
