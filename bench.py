"""Benchmark of the zone_FD RHS + SSP-RK3 path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One step = one SSP-RK3 step (three RHS evaluations, stage combinations and the
CFL time step) over the whole grid. Metric: cell-steps/s (cells x RK3 steps
per second), whole job. Default workload: the 2D isentropic vortex at 2048^2
(periodic [0,10]^2, TENO5 = TCNS5 + Roe, CFL 0.4, FP64), the largest grid of
the vortex refinement study; synthetic initial data with the configuration's
analytic field.

  value   device-resident stepping (state in HBM, dt on the device), timed
          with CUDA events on the stream the kernels run on, max over ranks;
  e2e     the same through the C ABI with host buffers: every step uploads the
          state from pinned host memory, steps, and downloads the state and
          the log values (dt, rhoLinf);
  roofline  the dominant kernel (the stage-closing sweep, which carries the
          stage's compulsory traffic: read U^k and U^0, write U^(k+1));
  cpu_baseline  the reference CPU solver (compiled from its own sources) on a
          bounded sample of the same workload, on this host's cores.

--impl reference runs only the reference CPU solver on the same workload.
For --gpus N > 1 (one process per GPU under torchrun) the ranks share one
periodic grid split into slabs along the last direction, each rank an n^dim
tile (weak scaling): before every RK stage neighbouring slabs exchange their
four boundary rows by NCCL point-to-point, and every step takes dt from a MAX
all-reduce of the ranks' wave speeds; value = all ranks' cell-steps / max rank
time.
"""
from __future__ import annotations

import argparse
import copy
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (dim, n, zone, inter_method, flux, cfl, description)
    "vortex2048": (2, 2048, 10.0, 11, 1, 0.4,
                   "2D isentropic vortex 2048^2, periodic [0,10]^2, TENO5 (TCNS5) + Roe, SSP-RK3, CFL 0.4, FP64"),
    "vortex1024": (2, 1024, 10.0, 11, 1, 0.4,
                   "2D isentropic vortex 1024^2, periodic [0,10]^2, TENO5 (TCNS5) + Roe, SSP-RK3, CFL 0.4, FP64"),
    "tgv256": (3, 256, 2 * np.pi, 2, 0, 0.5,
               "3D Taylor-Green vortex 256^3, periodic [0,2pi]^3, WCNS5 + HLLC, SSP-RK3, CFL 0.5, FP64"),
}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except (ValueError, KeyError, TypeError):
            pass
    return 6650.0, "fallback"


def initial_state(dim, n, L):
    from cfd_inwsl_b200.cases import isentropic_vortex, tgv_state
    if dim == 2:
        c, h = isentropic_vortex(n, L=L)
    else:
        c, h = tgv_state(n)
    return np.ascontiguousarray(c), h


# --------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, val in zip(names, parts[3:7]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------- reference arm
def usable_cores() -> int:
    """Cores this process may run on: the affinity mask, capped by a cgroup CPU
    quota (OpenMP oversubscription of a quota makes the reference crawl)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        q = Path("/sys/fs/cgroup/cpu.max").read_text().split()
        if q[0] != "max":
            n = min(n, max(1, int(float(q[0]) / float(q[1]))))
    except Exception:
        pass
    return max(1, n)


def reference_throughput(dim, n, L, im, fm, cfl, budget_s=12.0, max_steps=50):
    """The reference zone_FD CPU solver (oracle/_ref/libcongfd_ref.so, compiled
    from its own sources) on the same configuration, full RK3 steps including
    its CFL step, OpenMP over the usable host cores.

    Sample grid: 1024^2 for the 2D configurations. The reference's own CFL step
    reserves nVer doubles per cell in Block::getCellInterval (block.cpp:135-144);
    from 2049^2 vertices on that is a 33.6 MB allocation per cell, above glibc's
    mmap threshold, and the CFL step alone then takes minutes (247 s on 8 threads
    measured here, against 1.9 s for the RK3 step). Its per-cell cost is flat
    from 1024^2 to 1448^2, so the 1024^2 sample stands for the workload without
    that allocator pathology inflating the GPU/CPU ratio."""
    from oracle.refsolver import OracleC, RefSolver, ORC_WRAP
    threads = usable_cores()
    if dim == 2:
        kind = "reference"
        ns = min(n, 1024)
        c, h = initial_state(dim, ns, L)
        r = RefSolver(2, [ns, ns], [0, L, 0, L, 0, 0], inter_method=im, flux_method=fm, n_case=0, cfl=cfl,
                      periodic=True, threads=threads)
        r.cons = c
        step = lambda: r.solve(r.max_dt())  # noqa: E731
        what = "the reference solver (zone_FD sources, oracle/_ref/libcongfd_ref.so)"
    else:
        # the reference has no 3D Euler path: time the project's C restatement
        kind = "port"
        ns = min(n, 128)
        c, h = initial_state(dim, ns, L)
        o = OracleC(3, [ns, ns, ns], h, im, fm, bc=[[ORC_WRAP] * 2] * 3, threads=threads)
        o.cons = c
        step = lambda: o.solve(o.max_dt(cfl))  # noqa: E731
        what = "the project's C restatement (oracle/cfd_oracle.c; the reference has no 3D path)"
    t0 = time.perf_counter()
    step()  # warm-up
    warm = time.perf_counter() - t0
    k = 0
    t0 = time.perf_counter()
    while k < max_steps and (k < 2 or time.perf_counter() - t0 < budget_s):
        step()
        k += 1
    el = time.perf_counter() - t0
    ncell = ns ** dim
    return {"value": ncell * k / el, "unit": "cell-steps/s", "cores": threads, "kind": kind,
            "sample": f"{k} full RK3 steps (CFL step included; after 1 warm-up step of {warm:.1f} s) of the same "
                      f"configuration on a {ns}^{dim} grid, {el:.1f} s, {what}, OpenMP threads = {threads} "
                      f"(os.cpu_count() = {os.cpu_count()})"}


def vortex_accuracy(n, L, im, fm, cfl, device, t_end=2.0):
    """L1 density error against the exact translated vortex at t_end, FP64 and
    mixed, on an n^2 grid of the benchmark configuration."""
    from cfd_inwsl_b200 import cases, zone
    out = {"grid": n, "t": t_end}
    for key, prec in (("fp64", 0), ("mixed", 1)):
        info = zone.Info()
        info.dim = 2
        info.iMax = [n + 1, n + 1, 1]
        info.calZone = [0, L, 0, L, 0, 0]
        info.interMethod = im
        info.fluxMethod = fm
        info.CFL = cfl
        info.precision = prec
        info.device = device
        info.endStep = 1
        info.outputDt = t_end
        s = zone.BlockSolver(info, periodic=True)
        c, _ = cases.isentropic_vortex(n, L=L)
        s.set_cons(c)
        s.run_device()
        exact, _ = cases.isentropic_vortex(n, t=t_end, L=L)
        out[key] = float(np.abs(s.cons[:, 0] - exact[:, 0]).mean())
        s.close()
    out["ratio_mixed_over_fp64"] = out["mixed"] / out["fp64"]
    return out


def adjoint_cost(device, stream, n=256, nsteps=400, ckpt=20, seed=0):
    """Adjoint configuration: 256^2 periodic [0,1]^2, rho = 1 + drho (seeded
    Gaussian-filtered noise, correlation length 0.05, RMS 1e-2), p = 1/gamma,
    (u, v) = (0.5, 0.3), WCNS5 + Roe, nsteps (400) frozen-dt RK3 steps (dt from CFL 0.5 at
    t = 0), checkpoints every 20 steps, J = sum of rho^2 over 64 seeded probe
    cells. Times, with CUDA events on the handle's stream: the forward steps,
    cfd_adjoint_record (forward with checkpoints) and cfd_adjoint_reverse
    (segment recomputation + transposed stage Jacobians)."""
    import torch
    from cfd_inwsl_b200 import _lib, zone
    from cfd_inwsl_b200.cases import adjoint_problem
    cons, probes = adjoint_problem(n, seed)
    info = zone.Info()
    info.dim = 2
    info.iMax = [n + 1, n + 1, 1]
    info.calZone = [0, 1, 0, 1, 0, 0]
    info.interMethod = 2
    info.fluxMethod = 1
    info.CFL = 0.5
    info.device = device
    s = zone.BlockSolver(info, periodic=True)
    _lib.check(s.lib.cfd_set_stream(s.h, C.c_void_p(stream.cuda_stream)), s.h)
    s.set_cons(cons)
    dt = s.getTimeIntervalExplicit()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def forward():
        for _ in range(nsteps):
            _lib.check(s.lib.cfd_rk3_step(s.h, dt, 0.0, None), s.h)

    s.set_cons(cons)
    forward()  # warm-up
    s.set_cons(cons)
    fwd_ms = timed(forward)
    s.set_cons(cons)
    s.adjoint_record(dt, nsteps, ckpt)  # warm-up: buffers, module loading
    UN = s.cons
    seed_g = np.zeros_like(UN)
    seed_g[probes, 0] = 2 * UN[probes, 0]
    s.adjoint_reverse(seed_g)
    s.set_cons(cons)
    rec_ms = timed(lambda: s.adjoint_record(dt, nsteps, ckpt))
    out = {}
    rev_ms = timed(lambda: out.setdefault("g", s.adjoint_reverse(seed_g)))
    J = float(np.sum(UN[probes, 0] ** 2))
    s.close()
    return {"config": f"{n}^2 periodic, WCNS5 + Roe, {nsteps} frozen-dt RK3 steps, checkpoints every {ckpt}, "
                      "J = sum of rho^2 over 64 probes",
            "forward_ms": fwd_ms, "record_ms": rec_ms, "reverse_ms": rev_ms,
            "reverse_over_forward": rev_ms / fwd_ms, "record_plus_reverse_over_forward": (rec_ms + rev_ms) / fwd_ms,
            # the record pass is itself a forward run (graph-replayed, plus the
            # checkpoint copies): the reverse pass against the fastest forward
            "reverse_over_record": rev_ms / rec_ms,
            "forward": f"{nsteps} cfd_rk3_step calls (the per-step API, one host sync each)",
            "J": J, "grad_l2": float(np.linalg.norm(out["g"]))}


def batch_throughput(device, stream, ncases=256, steps=20, seed=0):
    """Batched configuration: 256 independent 2D Riemann problems on [0,1]^2,
    N = round(2^U(7,10)) cells per side (seeded), quadrant states rho ~
    U[0.1,2], p ~ U[0.05,2], u, v ~ U[-1,1], WCNS5 + HLLC, CFL 0.5, per-case dt,
    transmissive boundaries, advanced together in one persistent launch per
    sweep. Timed: `steps` steps of every case (cfd_batch_run with max_steps),
    CUDA events on the batch's stream, after 3 warm-up steps."""
    import torch
    from cfd_inwsl_b200 import _lib, cases, zone
    rng = np.random.default_rng(seed)
    sizes = [int(round(2 ** rng.uniform(7, 10))) for _ in range(ncases)]
    infos = []
    for n in sizes:
        info = zone.Info()
        info.dim = 2
        info.iMax = [n + 1, n + 1, 1]
        info.calZone = [0, 1, 0, 1, 0, 0]
        info.interMethod = 2
        info.fluxMethod = 0
        info.CFL = 0.5
        info.nCase = 0
        info.device = device
        infos.append(info)
    b = zone.BlockBatch(infos)
    _lib.check(b.lib.cfd_batch_set_stream(b.h, C.c_void_p(stream.cuda_stream)))
    for i, n in enumerate(sizes):
        b.set_cons(i, cases.riemann_quadrants(n, rng))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_run():
        b.run(0.25, end_step=1, max_steps=3)  # warm-up (graph capture after a tiling change)
        torch.cuda.synchronize()
        e0.record(stream)
        _, ns = b.run(0.25, end_step=1, max_steps=steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), float(sum(n * n * int(k) for n, k in zip(sizes, ns)))

    ms0, cs0 = timed_run()  # the default tiling: whole lines, single-grid tile shapes
    tiling = b.autotune()
    ms, cell_steps = timed_run()
    b.close()
    return {"config": f"{ncases} cases, N = round(2^U(7,10)) (seeded, {min(sizes)}..{max(sizes)}), "
                      "WCNS5 + HLLC, CFL 0.5, transmissive, per-case dt",
            "cells": int(sum(n * n for n in sizes)), "steps_per_case": steps, "ms": ms,
            "value": cell_steps / (ms / 1e3), "unit": "cell-steps/s",
            "autotuned_tiling": tiling, "default_tiling_value": cs0 / (ms0 / 1e3)}


def tgv_history(device, stream, n=256, steps=100, every=10):
    """3D Taylor-Green configuration: [0,2pi]^3 periodic, n^3 cells, WCNS5 +
    HLLC, CFL 0.5, `steps` RK3 steps in FP64 and in the mixed form. Times the
    steps (device loop, CUDA events on the handle's stream, outside the
    kinetic-energy reads) and records the kinetic energy sum rho |u|^2 / 2 h^3
    every `every` steps, computed on the device from the state buffer."""
    import torch
    from cfd_inwsl_b200 import _lib, zone
    from cfd_inwsl_b200.cases import tgv_state
    c, h = tgv_state(n)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"config": f"{n}^3 periodic [0,2pi]^3, WCNS5 + HLLC, CFL 0.5, {steps} steps", "steps": steps}
    for key, prec in (("fp64", 0), ("mixed", 1)):
        info = zone.Info()
        info.dim = 3
        info.iMax = [n + 1] * 3
        info.calZone = [0, 2 * np.pi] * 3
        info.interMethod = 2
        info.fluxMethod = 0
        info.CFL = 0.5
        info.precision = prec
        info.device = device
        s = zone.BlockSolver(info, periodic=True)
        _lib.check(s.lib.cfd_set_stream(s.h, C.c_void_p(stream.cuda_stream)), s.h)
        s.set_cons(c)

        def ke():
            ptr = C.c_void_p()
            _lib.check(s.lib.cfd_stage_state(s.h, 1, C.byref(ptr)), s.h)
            from cfd_inwsl_b200.slabs import _tensor
            u = _tensor(ptr.value, (5, n ** 3), f"cuda:{device}")
            with torch.cuda.stream(stream):
                k = (0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]).sum() * h ** 3
                return float(k.item())  # on the stream that computed it

        t = C.c_double(0.0)
        ns = C.c_int(0)
        hist, ms = [ke()], 0.0
        for _ in range(steps // every):
            torch.cuda.synchronize()
            e0.record(stream)
            _lib.check(s.lib.cfd_run(s.h, 0.5, 1, 1e300, every, C.byref(t), C.byref(ns), None, None), s.h)
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            hist.append(ke())
        s.close()
        out[key] = {"value": n ** 3 * steps / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms / steps,
                    "t_end": t.value, "kinetic_energy": hist}
    ref = np.array(out["fp64"]["kinetic_energy"])
    out["mixed"]["ke_max_rel_dev_vs_fp64"] = float(np.max(np.abs(np.array(out["mixed"]["kinetic_energy"]) - ref) /
                                                          ref))
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


# --------------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import torch
    from cfd_inwsl_b200 import _lib, zone

    dim, n, L, im, fm, cfl, desc = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    info = zone.Info()
    info.dim = dim
    info.iMax = [n + 1] * dim + [1] * (3 - dim)
    info.calZone = [0, L, 0, L, 0, L]
    info.interMethod = im
    info.fluxMethod = fm
    info.CFL = cfl
    info.device = local_rank
    info.strict = False
    info.precision = 1 if args.precision == "mixed" else 0
    c, h = initial_state(dim, n, L)
    slab = None
    if world > 1 or args.force_slabs:
        # one grid over the ranks: slabs along the last direction (each rank an
        # n^dim tile of a periodic grid n^(dim-1) x (n * world)), halos by NCCL
        from cfd_inwsl_b200 import slabs
        ginfo = copy.deepcopy(info)
        ginfo.iMax[dim - 1] = n * world + 1
        ginfo.calZone[2 * (dim - 1) + 1] = L * world
        slab = slabs.SlabRank(ginfo, periodic=True, device=local_rank)
        solver = slab.slab.solver
        stream = slab.stream
    else:
        solver = zone.BlockSolver(info, periodic=True)
        stream = torch.cuda.Stream(device=dev)
        _lib.check(solver.lib.cfd_set_stream(solver.h, C.c_void_p(stream.cuda_stream)), solver.h)
    lib = solver.lib
    ncell = solver.ncell

    tbuf = C.c_double(0.0)
    nsteps = C.c_int(0)

    def run(k):
        if slab is not None:
            _, taken = slab.run_device(k, cfl)
            assert taken == k
            return
        _lib.check(lib.cfd_run(solver.h, cfl, 1, 1e300, k, C.byref(tbuf), C.byref(nsteps), None, None), solver.h)
        assert nsteps.value == k

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- value: device-resident steps
    solver.set_cons(c)
    run(args.warmup)
    torch.cuda.synchronize()
    l0 = lib.cfd_launch_count(solver.h)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0.record(stream)
    run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    launches = lib.cfd_launch_count(solver.h) - l0
    value = world * ncell * args.steps / (ms / 1e3)

    # ---- roofline of the stage-closing sweep (last direction, RK epilogue)
    reps = 20
    for _ in range(3):
        _lib.check(lib.cfd_sweep(solver.h, dim, 2, 0.0), solver.h)
    torch.cuda.synchronize()
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    k0.record(stream)
    for _ in range(reps):
        _lib.check(lib.cfd_sweep(solver.h, dim, 2, 0.0), solver.h)
    k1.record(stream)
    torch.cuda.synchronize()
    kern_ms = k0.elapsed_time(k1) / reps
    # first sweep for the launch share
    k0.record(stream)
    for _ in range(reps):
        _lib.check(lib.cfd_sweep(solver.h, 1, 0, 0.0), solver.h)
    k1.record(stream)
    torch.cuda.synchronize()
    kern0_ms = k0.elapsed_time(k1) / reps
    bytes_per_cell = 3 * (dim + 2) * 8  # read U^k, read U^0, write U^(k+1)
    alg_bytes = bytes_per_cell * ncell
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = None
    fp64 = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        t = json.loads(tp.read_text()).get(args.workload)
        if t:
            traffic = t.get("bytes_per_launch")
            ops = t.get("fp64_ops_per_face")
            if ops and args.precision == "fp64":
                # the path's binding roof: FP64 arithmetic (counted instructions
                # per face from ncu, times the faces of one launch, over the
                # live kernel time), against B200's nominal FP64 vector peak
                tflops = ops["flops"] * ncell / (kern_ms / 1e3) / 1e12
                fp64 = {"achieved_tflops": tflops, "peak_tflops": 37.0, "peak_source": "nominal (B200 datasheet)",
                        "frac": tflops / 37.0, "flops_per_face": ops["flops"], "count_source": ops["source"]}

    # ---- e2e through the C ABI with host buffers
    e2e_steps = max(2, min(args.steps // 10, 10))
    host = torch.empty(ncell * (dim + 2), dtype=torch.float64, pin_memory=True).numpy()
    host[:] = c.reshape(-1)
    hp = _lib.ptr(host)
    dts = np.zeros(1)
    lin = np.zeros(1)
    def e2e_step():
        _lib.check(lib.cfd_upload_cons(solver.h, hp), solver.h)
        if slab is not None:
            slab.run_device(1, cfl)
        else:
            _lib.check(lib.cfd_run(solver.h, cfl, 1, 1e300, 1, C.byref(tbuf), C.byref(nsteps), _lib.ptr(dts),
                                   _lib.ptr(lin)), solver.h)
        _lib.check(lib.cfd_download_cons(solver.h, hp), solver.h)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    e2e_value = world * ncell * e2e_steps / (e2e_ms / 1e3)
    state_bytes = ncell * (dim + 2) * 8

    # ---- the mixed FP32/FP64 form on the same workload, and both forms' accuracy
    mixed = None
    if not args.no_mixed and args.precision == "fp64" and world == 1:
        info_m = zone.Info()
        for k, v in vars(info).items():
            setattr(info_m, k, v)
        info_m.precision = 1
        sm = zone.BlockSolver(info_m, periodic=True)
        _lib.check(lib.cfd_set_stream(sm.h, C.c_void_p(stream.cuda_stream)), sm.h)
        sm.set_cons(c)
        tm = C.c_double(0.0)
        nm = C.c_int(0)
        _lib.check(lib.cfd_run(sm.h, cfl, 1, 1e300, args.warmup, C.byref(tm), C.byref(nm), None, None), sm.h)
        torch.cuda.synchronize()
        e0.record(stream)
        _lib.check(lib.cfd_run(sm.h, cfl, 1, 1e300, args.steps, C.byref(tm), C.byref(nm), None, None), sm.h)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_m = max_over_ranks(e0.elapsed_time(e1))
        sm.close()
        value_m = world * ncell * args.steps / (ms_m / 1e3)
        mixed = {"value": value_m, "unit": "cell-steps/s", "ms_per_step": ms_m / args.steps,
                 "speedup_vs_fp64": value_m / value}
        if dim == 2 and rank == 0:
            mixed["l1_rho_vs_exact"] = vortex_accuracy(args.accuracy_grid, L, im, fm, cfl, local_rank)

    adjoint = None
    if not args.no_adjoint and world == 1:
        adjoint = adjoint_cost(local_rank, stream, nsteps=args.adjoint_steps)
    batch = None
    if not args.no_batch and world == 1:
        batch = batch_throughput(local_rank, stream)
    tgv = None
    if not args.no_tgv and world == 1 and dim == 2:
        tgv = tgv_history(local_rank, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_throughput(dim, n, L, im, fm, cfl, budget_s=args.cpu_budget)

    result = {
        "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64 state, f32 reconstruction",
        "data": "synthetic (analytic initial field of the configuration)",
        "config": {"workload": desc, "grid": [n] * dim, "cells": ncell, "inter_method": im,
                   "flux_method": "Roe" if fm else "HLLC", "cfl": cfl, "flavour": "fast (FMA, 1e-12 parity)",
                   "l2": "inputs larger than L2: 3 state arrays + RHS of %.0f MB each" % (state_bytes / 1e6),
                   "parallelism": (f"{world} slabs along the last direction, one per GPU, 4-row halos "
                                   "exchanged by NCCL before every stage, dt from the ranks' maximum wave speeds")
                                  if slab is not None else "single GPU",
                   "global_grid": [n] * (dim - 1) + [n * world],
                   "cell_stages_per_s": 3 * value},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_source": peak_kind,
                     "kernel": f"sweep along axis {dim - 1} with the RK stage epilogue",
                     "kernel_ms": kern_ms, "first_sweep_ms": kern0_ms,
                     "algorithmic_bytes_per_cell": bytes_per_cell,
                     "note": "FP64-arithmetic bound path; the HBM fraction is low by construction",
                     "fp64": fp64},
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes + 16, "steps": e2e_steps,
                "path": ("cfd_upload_cons + one step (" + ("stages with halo exchanges" if slab is not None
                                                         else "cfd_run") + ") + cfd_download_cons per step, pinned host buffer")},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    if mixed is not None:
        result["mixed"] = mixed
    if adjoint is not None:
        result["adjoint"] = adjoint
    if batch is not None:
        result["batch"] = batch
    if tgv is not None:
        result["tgv"] = tgv
    if cpu is not None:
        result["cpu_baseline"] = cpu
    solver.close()
    return result


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="vortex2048", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-tgv", action="store_true", help="skip the 3D Taylor-Green throughput and energy history")
    ap.add_argument("--force-slabs", action="store_true",
                    help="run the multi-GPU slab path (halo exchange) even on one GPU (one periodic slab)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="form of the timed steps (mixed: CFD_PREC_MIXED)")
    ap.add_argument("--accuracy-grid", type=int, default=512)
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint cost measurement and print its dict (for profiling the adjoint kernels)")
    ap.add_argument("--adjoint-steps", type=int, default=400, help="RK3 steps of the adjoint measurement")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.adjoint_only:
        import torch
        torch.cuda.set_device(0)
        r = adjoint_cost(0, torch.cuda.Stream(), nsteps=args.adjoint_steps)
        print(json.dumps({"adjoint": r}), flush=True)
        return 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        dim, n, L, im, fm, cfl, desc = WORKLOADS[args.workload]
        r = reference_throughput(dim, n, L, im, fm, cfl, budget_s=args.cpu_budget)
        out = {"impl": "reference", "metric": "cell-steps/s", "value": r["value"], "unit": "cell-steps/s",
               "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": desc, "grid": [n] * dim},
               "cpu_baseline": {"value": r["value"], "unit": r["unit"], "cores": r["cores"], "kind": r["kind"],
                                "sample": r["sample"]},
               "e2e": {"value": r["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out), flush=True)
        return 0

    distributed = world > 1 or args.force_slabs
    if distributed:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29511")
        os.environ.setdefault("RANK", str(rank))
        os.environ.setdefault("WORLD_SIZE", str(world))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    res = run_ours(args, rank, world, local_rank)
    if distributed:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(res), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
