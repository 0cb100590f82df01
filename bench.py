"""Benchmark of the zone_FD RHS + SSP-RK3 path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

One step = one SSP-RK3 step (three RHS evaluations, stage combinations and the
CFL time step) over the whole grid. Metric: cell-steps/s (cells x RK3 steps
per second), whole job. Default workload: the 2D isentropic vortex at 2048^2
(periodic [0,10]^2, TENO5 = TCNS5 + Roe, CFL 0.4, FP64), the largest grid of
the vortex refinement study; synthetic initial data with the configuration's
analytic field. The timed steps use the strict flavour, whose results equal
the reference solver's bit for bit (the fast flavour, FMA-contracted, is
timed beside it).

  value   device-resident stepping (state in HBM, dt on the device), timed
          with CUDA events on the stream the kernels run on, max over ranks;
  e2e     the same through the C ABI with host buffers: every step is one
          cfd_step_host call that uploads the state from pinned host memory,
          takes one CFL step and downloads the new state, the copies
          overlapped with the step's sweeps (slabs: upload, step, download);
  roofline  the dominant kernel (the stage-closing sweep, which carries the
          stage's compulsory traffic: read U^k and U^0, write U^(k+1)), with
          its FP64 throughput against a DFMA peak measured in the same run;
  cpu_baseline  the reference CPU solver (compiled from its own sources) on the
          same grid, RK3 steps of one fixed dt, on this host's cores.

--impl reference runs only the reference CPU solver on the same workload.
For --gpus N > 1 (one process per GPU under torchrun) the ranks share one
periodic grid split into slabs along the last direction, each rank an n^dim
tile (weak scaling): before every RK stage neighbouring slabs exchange their
four boundary rows by NCCL point-to-point, and every step takes dt from a MAX
all-reduce of the ranks' wave speeds; value = all ranks' cell-steps / max rank
time. The batch block then runs the 256 independent cases as replicas, split
over the ranks by cost (no exchange).
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

GAMMA = 1.4
WORKLOADS = {
    # name: (dim, n, zone, inter_method, flux, cfl, description)
    "vortex2048": (2, 2048, 10.0, 11, 1, 0.4,
                   "2D isentropic vortex 2048^2, periodic [0,10]^2, TENO5 (TCNS5) + Roe, SSP-RK3, CFL 0.4, FP64"),
    "vortex1024": (2, 1024, 10.0, 11, 1, 0.4,
                   "2D isentropic vortex 1024^2, periodic [0,10]^2, TENO5 (TCNS5) + Roe, SSP-RK3, CFL 0.4, FP64"),
    "tgv256": (3, 256, 2 * np.pi, 2, 0, 0.5,
               "3D Taylor-Green vortex 256^3, periodic [0,2pi]^3, WCNS5 + HLLC, SSP-RK3, CFL 0.5, FP64"),
    "tgv128": (3, 128, 2 * np.pi, 2, 0, 0.5,
               "3D Taylor-Green vortex 128^3, periodic [0,2pi]^3, WCNS5 + HLLC, SSP-RK3, CFL 0.5, FP64"),
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


def kernel_counts(workload, flavour):
    """Per-launch DRAM traffic and FP64 operations per face of the
    stage-closing sweep, from ncu captures (profiles/traffic.json)."""
    tp = ROOT / "profiles" / "traffic.json"
    if not tp.exists():
        return {}
    try:
        return json.loads(tp.read_text()).get(workload, {}).get(flavour, {}) or {}
    except ValueError:
        return {}


def initial_state(dim, n, L):
    from cfd_inwsl_b200.cases import isentropic_vortex, tgv_state
    if dim == 2:
        c, h = isentropic_vortex(n, L=L)
    else:
        c, h = tgv_state(n)
    return np.ascontiguousarray(c), h


def cfl_dt(cons, dim, h, cfl):
    """getTimeIntervalExplicit's step (blockSolver.cpp:318-349) in numpy:
    CFL / sum_d max_cells (c + |u_d|) / h."""
    rho = cons[:, 0]
    vel = cons[:, 1:1 + dim] / rho[:, None]
    p = (GAMMA - 1) * (cons[:, -1] - 0.5 * rho * np.sum(vel * vel, axis=1))
    c = np.sqrt(GAMMA * p / rho)
    lam = 0.0
    for d in range(dim):
        lam += float(np.max((c + np.abs(vel[:, d])) / h))
    return cfl / lam


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



def reference_rk3(dim, n, L, im, fm, cfl, steps, budget_s=20.0):
    """The reference zone_FD CPU solver (oracle/_ref/libcongfd_ref.so, compiled
    from its own sources) on the benchmark grid itself: BlockSolver::RK3_SSP
    steps of one fixed dt (the CFL step of the initial state), OpenMP over the
    usable host cores; up to `steps` timed steps after one warm-up step, fewer
    when they would exceed budget_s.

    The reference's CFL step is left out of the timed steps: its
    Block::getCellInterval reserves nVer doubles per cell (block.cpp:135-144),
    which from 2049^2 vertices is a 33.6 MB allocation per cell and makes one
    CFL step take about a minute on 16 cores; its per-cell cost is about 1% of
    the RK3 step below that size, so leaving it out favours the reference.
    3D: the reference has no 3D Euler path; the project's C restatement
    (oracle/cfd_oracle.c) stands in, labelled kind "port"."""
    from oracle.refsolver import ORC_WRAP, OracleC, RefSolver
    threads = usable_cores()
    c, h = initial_state(dim, n, L)
    dt = cfl_dt(c, dim, h, cfl)
    if dim == 2:
        kind = "reference"
        r = RefSolver(2, [n, n], [0, L, 0, L, 0, 0], inter_method=im, flux_method=fm, n_case=0, cfl=cfl,
                      periodic=True, threads=threads)
        r.cons = c
        step = lambda: r.solve(dt)  # noqa: E731
        what = "the reference solver (zone_FD sources, oracle/_ref/libcongfd_ref.so), BlockSolver::RK3_SSP"
    else:
        kind = "port"
        o = OracleC(3, [n] * 3, h, im, fm, bc=[[ORC_WRAP] * 2] * 3, threads=threads)
        o.cons = c
        step = lambda: o.solve(dt)  # noqa: E731
        what = "the project's C restatement (oracle/cfd_oracle.c; the reference has no 3D path)"
    t0 = time.perf_counter()
    step()  # warm-up: first touch of the solver's arrays
    warm = time.perf_counter() - t0
    k = 0
    t0 = time.perf_counter()
    while k < max(1, steps) and (k < 2 or time.perf_counter() - t0 < budget_s):
        step()
        k += 1
    el = time.perf_counter() - t0
    ncell = n ** dim
    return {"value": ncell * k / el, "unit": "cell-steps/s", "cores": threads, "kind": kind,
            "sample": f"{k} RK3 steps of one fixed dt (the CFL step of the initial state; after 1 warm-up step of "
                      f"{warm:.1f} s) on the benchmark's own {n}^{dim} grid, {el:.1f} s, {what}, OpenMP threads = "
                      f"{threads} (os.cpu_count() = {os.cpu_count()})"}


def reference_full_steps(n, L, im, fm, cfl, budget_s=8.0, max_steps=20):
    """The reference's own stepping (RK3 step plus its CFL step) on an n^2
    sample of the vortex configuration, for comparison with reference_rk3."""
    from oracle.refsolver import RefSolver
    threads = usable_cores()
    c, _ = initial_state(2, n, L)
    r = RefSolver(2, [n, n], [0, L, 0, L, 0, 0], inter_method=im, flux_method=fm, n_case=0, cfl=cfl, periodic=True,
                  threads=threads)
    r.cons = c
    r.solve(r.max_dt())
    k, t0 = 0, time.perf_counter()
    while k < max_steps and (k < 2 or time.perf_counter() - t0 < budget_s):
        r.solve(r.max_dt())
        k += 1
    el = time.perf_counter() - t0
    return {"value": n * n * k / el, "unit": "cell-steps/s", "cores": threads,
            "sample": f"{k} full steps (CFL step + RK3_SSP) on {n}^2, {el:.1f} s"}



# --------------------------------------------------------------------- our arm: helpers
def make_solver(dim, n, L, im, fm, cfl, device, stream, strict=True, precision=0):
    from cfd_inwsl_b200 import _lib, zone
    info = zone.Info()
    info.dim = dim
    info.iMax = [n + 1] * dim + [1] * (3 - dim)
    info.calZone = [0, L, 0, L, 0, L]
    info.interMethod = im
    info.fluxMethod = fm
    info.CFL = cfl
    info.device = device
    info.strict = strict
    info.precision = precision
    s = zone.BlockSolver(info, periodic=True)
    _lib.check(s.lib.cfd_set_stream(s.h, C.c_void_p(stream.cuda_stream)), s.h)
    return s


def device_steps(s, stream, k, cfl, warmup=3):
    """ms per step of the device-resident loop (cfd_run), CUDA events on the stream."""
    import torch
    from cfd_inwsl_b200 import _lib
    t, ns = C.c_double(0.0), C.c_int(0)

    def run(m):
        _lib.check(s.lib.cfd_run(s.h, cfl, 1, 1e300, m, C.byref(t), C.byref(ns), None, None), s.h)

    run(warmup)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run(k)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / k


def sweep_ms(s, stream, idim, mode, reps=20):
    """Average launch time of one sweep (cfd_sweep: mode 0 writes the RHS, mode
    2 is the stage-closing sweep with the RK epilogue), CUDA events."""
    import torch
    from cfd_inwsl_b200 import _lib
    for _ in range(3):
        _lib.check(s.lib.cfd_sweep(s.h, idim, mode, 0.0), s.h)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        _lib.check(s.lib.cfd_sweep(s.h, idim, mode, 0.0), s.h)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def fp64_peak(stream, iters=4096, reps=3):
    """Measured FP64 throughput of the device: the library's DFMA probe (eight
    independent DFMA chains per thread on every SM), best of `reps`."""
    import torch
    from cfd_inwsl_b200 import _lib
    lib = _lib.load()
    flops = C.c_double(0.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(reps + 1):
        e0.record(stream)
        _lib.check(lib.cfd_fp64_peak_probe(iters, C.c_void_p(stream.cuda_stream), C.byref(flops)))
        e1.record(stream)
        torch.cuda.synchronize()
        best = max(best, flops.value / (e0.elapsed_time(e1) / 1e3) / 1e12)
    return best


def roofline_of(ncell, dim, kern_ms, counts, peak_tflops, faces=None):
    """HBM roofline of the stage-closing sweep (algorithmic bytes: read U^k and
    U^0, write U^(k+1)) and its FP64 throughput from the counted operations
    per face (2 per DFMA, 1 per DADD / DMUL) against the measured DFMA peak."""
    hbm, hbm_kind = measured_peaks()
    bytes_per_cell = 3 * (dim + 2) * 8
    achieved = bytes_per_cell * ncell / (kern_ms / 1e3) / 1e9
    traffic = counts.get("bytes_per_launch")
    if traffic is not None and counts.get("cells") and counts["cells"] != ncell:
        traffic = traffic * ncell / counts["cells"]  # captured on a smaller grid: scaled by cells
    out = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
           "traffic": traffic, "peak_source": hbm_kind, "kernel_ms": kern_ms,
           "algorithmic_bytes_per_cell": bytes_per_cell,
           "note": "FP64-arithmetic bound path; the HBM fraction is low by construction (see fp64)"}
    ops = counts.get("fp64_per_face")
    if ops:
        nf = faces if faces is not None else ncell
        tflops = ops["flops"] * nf / (kern_ms / 1e3) / 1e12
        out["fp64"] = {"achieved_tflops": tflops, "peak_tflops": peak_tflops,
                       "peak_source": "measured in this run (cfd_fp64_peak_probe: DFMA chains on every SM)",
                       "frac": tflops / peak_tflops, "flops_per_face": ops["flops"],
                       "count_source": ops.get("source", "ncu")}
    return out


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
    cells. Times, with CUDA events on the handle's stream: the forward run
    (cfd_run_fixed: the same frozen-dt steps replayed from graphs of 20 steps),
    cfd_adjoint_record (the forward with checkpoints) and cfd_adjoint_reverse
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
        _lib.check(s.lib.cfd_run_fixed(s.h, dt, nsteps, ckpt), s.h)

    s.set_cons(cons)
    forward()  # warm-up: graph capture
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
            "forward": f"cfd_run_fixed: {nsteps} frozen-dt steps replayed from CUDA graphs of {ckpt} steps "
                       "(the record pass without its checkpoint copies)",
            "J": J, "grad_l2": float(np.linalg.norm(out["g"]))}


def batch_throughput(device, stream, ncases=256, steps=20, seed=0, full_run=True, subset=None):
    """Batched configuration: 256 independent 2D Riemann problems on [0,1]^2,
    N = round(2^U(7,10)) cells per side (seeded), quadrant states rho ~
    U[0.1,2], p ~ U[0.05,2], u, v ~ U[-1,1], WCNS5 + HLLC, CFL 0.5, per-case dt,
    transmissive boundaries, advanced together in one persistent launch per
    sweep (fast flavour; the strict flavour equals the reference case by case).
    Timed with CUDA events on the batch's stream: `steps` steps of every case
    with the default tiling and after cfd_batch_autotune, then (full_run) the
    whole configuration, every case to t = 0.25. subset: the indices of the
    cases this rank runs (replicas over GPUs), default all."""
    import torch
    from cfd_inwsl_b200 import _lib, cases, zone
    sizes, prims = cases.riemann_batch(ncases, seed)
    if subset is not None:
        sizes = [sizes[i] for i in subset]
        prims = [prims[i] for i in subset]
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

    def reset():
        for i, (n, P) in enumerate(zip(sizes, prims)):
            b.set_cons(i, cases.quadrant_state(P, n))
            b.infos[i].t = 0.0

    reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_run(max_steps):
        torch.cuda.synchronize()
        e0.record(stream)
        _, ns = b.run(0.25, end_step=1, max_steps=max_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), float(sum(n * n * int(k) for n, k in zip(sizes, ns))), ns

    b.run(0.25, end_step=1, max_steps=3)  # warm-up (graph capture)
    ms0, cs0, _ = timed_run(steps)  # the default tiling: whole lines, single-grid tile shapes
    tiling = b.autotune()
    b.run(0.25, end_step=1, max_steps=3)  # warm-up after the tiling change
    ms, cell_steps, _ = timed_run(steps)
    out = {"config": f"{ncases} cases, N = round(2^U(7,10)) (seeded, {min(sizes)}..{max(sizes)}), "
                     "WCNS5 + HLLC, CFL 0.5, transmissive, per-case dt, fast flavour",
           "cells": int(sum(n * n for n in sizes)), "steps_per_case": steps, "ms": ms, "cell_steps": cell_steps,
           "value": cell_steps / (ms / 1e3), "unit": "cell-steps/s",
           "autotuned_tiling": tiling, "default_tiling_value": cs0 / (ms0 / 1e3)}
    if full_run:
        reset()
        ms_f, cs_f, ns_f = timed_run(1 << 30)
        out["to_t_end"] = {"t_end": 0.25, "ms": ms_f, "cell_steps": cs_f, "value": cs_f / (ms_f / 1e3),
                           "steps_min": int(np.min(ns_f)), "steps_max": int(np.max(ns_f)),
                           "steps_total": int(np.sum(ns_f))}
    b.close()
    return out


def tgv_block(device, stream, sizes=(128, 256, 384), steps=100, every=10, peak_tflops=None):
    """3D Taylor-Green configuration: [0,2pi]^3 periodic, WCNS5 + HLLC, CFL
    0.5. Per grid size: device-resident steps in the strict flavour (the
    reference's roundings) and the fast flavour (fewer steps at 384^3); at
    256^3 also the mixed form, the kinetic-energy history sum rho |u|^2 / 2 h^3
    every `every` steps (on the device, outside the timed steps) of strict and
    mixed, the roofline of the stage-closing z sweep, and the C restatement as
    the CPU baseline."""
    import torch
    from cfd_inwsl_b200 import _lib
    from cfd_inwsl_b200.cases import tgv_state
    L = 2 * np.pi
    out = {"config": "periodic [0,2pi]^3, WCNS5 + HLLC, SSP-RK3, CFL 0.5", "sizes": {}}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for n in sizes:
        c, h = tgv_state(n)
        k = steps if n <= 256 else 40
        row = {"steps": k}
        for key, strict, prec in (("strict", True, 0), ("fast", False, 0), ("mixed", False, 1)):
            if key == "mixed" and n != 256:
                continue
            s = make_solver(3, n, L, 2, 0, 0.5, device, stream, strict=strict, precision=prec)
            s.set_cons(c)
            if n == 256 and key in ("strict", "mixed"):
                def ke():
                    ptr = C.c_void_p()
                    _lib.check(s.lib.cfd_stage_state(s.h, 1, C.byref(ptr)), s.h)
                    from cfd_inwsl_b200.slabs import _tensor
                    u = _tensor(ptr.value, (5, n ** 3), f"cuda:{device}")
                    with torch.cuda.stream(stream):
                        return float(((0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]).sum() * h ** 3).item())
                t, ns = C.c_double(0.0), C.c_int(0)
                hist, ms = [ke()], 0.0
                for _ in range(steps // every):
                    torch.cuda.synchronize()
                    e0.record(stream)
                    _lib.check(s.lib.cfd_run(s.h, 0.5, 1, 1e300, every, C.byref(t), C.byref(ns), None, None), s.h)
                    e1.record(stream)
                    torch.cuda.synchronize()
                    ms += e0.elapsed_time(e1)
                    hist.append(ke())
                ms_step = ms / steps
                row[key] = {"value": n ** 3 / (ms_step / 1e3), "ms_per_step": ms_step, "t_end": t.value,
                            "kinetic_energy": hist}
                if key == "strict":
                    kern = sweep_ms(s, stream, 3, 2)
                    row["roofline"] = roofline_of(n ** 3, 3, kern, kernel_counts(f"tgv{n}", "strict"), peak_tflops)
                    row["roofline"]["kernel"] = "strict z sweep with the RK stage epilogue"
                    row["roofline"]["x_y_sweep_ms"] = [sweep_ms(s, stream, 1, 0), sweep_ms(s, stream, 2, 0)]
            else:
                ms_step = device_steps(s, stream, k, 0.5)
                row[key] = {"value": n ** 3 / (ms_step / 1e3), "ms_per_step": ms_step}
            s.close()
        row["fast"]["speedup_vs_strict"] = row["fast"]["value"] / row["strict"]["value"]
        if "mixed" in row:
            row["mixed"]["speedup_vs_strict"] = row["mixed"]["value"] / row["strict"]["value"]
            row["mixed"]["speedup_vs_fast"] = row["mixed"]["value"] / row["fast"]["value"]
            ref = np.array(row["strict"]["kinetic_energy"])
            row["mixed"]["ke_max_rel_dev_vs_strict"] = float(np.max(np.abs(np.array(row["mixed"]["kinetic_energy"]) - ref) / ref))
        out["sizes"][str(n)] = row
    return out


# --------------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import torch
    from cfd_inwsl_b200 import _lib, zone

    dim, n, L, im, fm, cfl, desc = WORKLOADS[args.workload]
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    strict = args.flavour == "strict"
    info = zone.Info()
    info.dim = dim
    info.iMax = [n + 1] * dim + [1] * (3 - dim)
    info.calZone = [0, L, 0, L, 0, L]
    info.interMethod = im
    info.fluxMethod = fm
    info.CFL = cfl
    info.device = local_rank
    info.strict = strict
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
    peak_tflops = fp64_peak(stream)
    kern_ms = sweep_ms(solver, stream, dim, 2)
    kern0_ms = sweep_ms(solver, stream, 1, 0)
    roofline = roofline_of(ncell, dim, kern_ms, kernel_counts(args.workload, args.flavour), peak_tflops)
    roofline["kernel"] = f"{args.flavour} sweep along axis {dim - 1} with the RK stage epilogue"
    roofline["first_sweep_ms"] = kern0_ms

    # ---- e2e through the C ABI with host buffers
    e2e_steps = max(2, min(args.steps // 10, 10))
    host = torch.empty(ncell * (dim + 2), dtype=torch.float64, pin_memory=True).numpy()
    host[:] = c.reshape(-1)
    hp = _lib.ptr(host)
    dtb = C.c_double(0.0)

    def e2e_step():
        if slab is not None:
            _lib.check(lib.cfd_upload_cons(solver.h, hp), solver.h)
            slab.run_device(1, cfl)
            _lib.check(lib.cfd_download_cons(solver.h, hp), solver.h)
        else:
            # one call: upload, CFL step and download of the host state, the
            # copies overlapped with the step's first and last sweeps
            _lib.check(lib.cfd_step_host(solver.h, cfl, 1e300, hp, hp, C.byref(tbuf), C.byref(dtb)), solver.h)

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

    # ---- the other FP64 flavour and the mixed form on the same workload
    others = {}
    if world == 1 and args.precision == "fp64":
        other = "fast" if strict else "strict"
        so = make_solver(dim, n, L, im, fm, cfl, local_rank, stream, strict=not strict)
        so.set_cons(c)
        ms_o = device_steps(so, stream, args.steps, cfl, warmup=args.warmup)
        counts_o = kernel_counts(args.workload, other)
        k_o = sweep_ms(so, stream, dim, 2)
        others[other] = {"value": ncell / (ms_o / 1e3), "unit": "cell-steps/s", "ms_per_step": ms_o,
                         "speedup_vs_" + args.flavour: ms / args.steps / ms_o,
                         "roofline": roofline_of(ncell, dim, k_o, counts_o, peak_tflops)}
        so.close()
        if not args.no_mixed:
            sm = make_solver(dim, n, L, im, fm, cfl, local_rank, stream, strict=False, precision=1)
            sm.set_cons(c)
            ms_m = device_steps(sm, stream, args.steps, cfl, warmup=args.warmup)
            sm.close()
            fast_ms = ms_o if other == "fast" else ms / args.steps
            strict_ms = ms / args.steps if strict else ms_o
            mixed = {"value": ncell / (ms_m / 1e3), "unit": "cell-steps/s", "ms_per_step": ms_m,
                     "speedup_vs_strict_fp64": strict_ms / ms_m, "speedup_vs_fast_fp64": fast_ms / ms_m}
            if dim == 2:
                mixed["l1_rho_vs_exact"] = vortex_accuracy(args.accuracy_grid, L, im, fm, cfl, local_rank)
            others["mixed"] = mixed

    adjoint = None
    if not args.no_adjoint and world == 1:
        adjoint = adjoint_cost(local_rank, stream, nsteps=args.adjoint_steps)
    batch = None
    if not args.no_batch and world == 1:
        batch = batch_throughput(local_rank, stream, full_run=args.batch_full)
    elif not args.no_batch:
        # replicas: the 256 cases split over the ranks by cost (N^3), no
        # exchange; time = the slowest rank's, value = all ranks' cell-steps
        from cfd_inwsl_b200 import cases as _cases
        from cfd_inwsl_b200.replicas import case_cost, partition_by_cost
        sizes_all, _ = _cases.riemann_batch(256, 0)
        shares = partition_by_cost([case_cost(n) for n in sizes_all], world)
        mine = batch_throughput(local_rank, stream, full_run=False, subset=shares[rank])
        ms_b = max_over_ranks(mine["ms"])
        import torch.distributed as dist
        tot = torch.tensor([mine["cell_steps"]], dtype=torch.float64, device=dev)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
        batch = {"config": mine["config"].replace(f"{len(shares[rank])} cases", "256 cases"),
                 "parallelism": f"replicas: cases split over {world} ranks by cost N^3 (LPT), no exchange",
                 "cases_per_rank": [len(sh) for sh in shares], "steps_per_case": mine["steps_per_case"],
                 "ms": ms_b, "value": float(tot.item()) / (ms_b / 1e3), "unit": "cell-steps/s",
                 "scaling": "strong"}
    tgv = None
    if not args.no_tgv and world == 1 and dim == 2:
        tgv = tgv_block(local_rank, stream, peak_tflops=peak_tflops)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = reference_rk3(dim, n, L, im, fm, cfl, steps=args.steps, budget_s=args.cpu_budget)
        if dim == 2:
            cpu["full_steps_1024"] = reference_full_steps(min(n, 1024), L, im, fm, cfl)
        if tgv is not None:
            tgv["cpu_baseline"] = reference_rk3(3, 64, 2 * np.pi, 2, 0, 0.5, steps=20, budget_s=8.0)

    result = {
        "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f64 state, f32 reconstruction",
        "data": "synthetic (analytic initial field of the configuration)",
        "config": {"workload": desc, "grid": [n] * dim, "cells": ncell, "inter_method": im,
                   "flux_method": "Roe" if fm else "HLLC", "cfl": cfl,
                   "flavour": ("strict: the reference's operation order and roundings, bit for bit"
                               if strict else "fast: FMA contraction and shared reciprocals"),
                   "l2": "inputs larger than L2: 3 state arrays + RHS of %.0f MB each" % (state_bytes / 1e6),
                   "parallelism": (f"{world} slabs along the last direction, one per GPU, 4-row halos "
                                   "exchanged by NCCL before every stage, dt from the ranks' maximum wave speeds")
                                  if slab is not None else "single GPU",
                   "global_grid": [n] * (dim - 1) + [n * world],
                   "cell_stages_per_s": 3 * value},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes, "steps": e2e_steps,
                "path": ("cfd_upload_cons + one step (stages with halo exchanges) + cfd_download_cons per step, "
                         "pinned host buffer" if slab is not None else
                         "cfd_step_host per step: the host state (pinned) uploaded, one CFL step, the new state "
                         "downloaded into the same buffer; the copies run in 8 chunks overlapped with the "
                         "step's first and last sweeps")},
        "gpu_launches": int(launches),
        "clocks": clk,
    }
    result.update(others)
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
    ap.add_argument("--flavour", default="strict", choices=["strict", "fast"],
                    help="FP64 arithmetic of the timed steps: strict (the reference's roundings, bit for bit) or "
                         "fast (FMA contraction and shared reciprocals)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--batch-full", action="store_true",
                    help="also run the whole batched configuration to t = 0.25 (about 2.5 minutes)")
    ap.add_argument("--no-tgv", action="store_true", help="skip the 3D Taylor-Green block")
    ap.add_argument("--force-slabs", action="store_true",
                    help="run the multi-GPU slab path (halo exchange) even on one GPU (one periodic slab)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="form of the timed steps (mixed: CFD_PREC_MIXED, fast flavour)")
    ap.add_argument("--accuracy-grid", type=int, default=512)
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint cost measurement and print its dict (for profiling the adjoint kernels)")
    ap.add_argument("--adjoint-steps", type=int, default=400, help="RK3 steps of the adjoint measurement")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.precision == "mixed":
        args.flavour = "fast"  # the mixed form is built on the fast flavour
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
        r = reference_rk3(dim, n, L, im, fm, cfl, steps=args.steps, budget_s=args.cpu_budget)
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
