"""Generate the golden fixtures under tests/golden from the reference itself.

    python tests/golden/make_golden.py            (needs oracle/_ref/libcongfd_ref.so
                                                   and the reference checkout for the log file)

Every value here is produced by the reference zone_FD code compiled from its
own sources (oracle/Makefile -> oracle/_ref/libcongfd_ref.so), or read from a
file the reference repository commits:

  sod_congtcns5ct5_101.json  per-step dt / rhoLinf of the reference's committed
                             run log zone_FD/cases/"Sod - congTCNS5CT5 - 101.txt"
                             (two identical appended runs of 86 steps)
  order_congfd.json          CongFD1.0/order.txt (AccuracyTest convergence orders)
  kat_inter5.npz             interpolator outputs (interScheme.hpp) on random and
                             adversarial stencils, per selector entry
  kat_flux.npz               HLLC / Roe face fluxes (fluxSchemes.hpp) 1D and 2D
  rhs_2d.npz                 one RHS, one CFL step and one RK3 step of small 2D
                             grids (random quadrants, smooth periodic field)
  sod_400.npz                1D Sod, 400 cells, WCNS5 + HLLC, CFL 0.5, t = 0.2
  kat_face.npz               one-face characteristic reconstructions (reconI,
                             reconstructor5order.hpp:233-429), 1D and 2D, both normals
  rhs_trad6.npz              one RHS, one CFL step and one RK3 step with the TRAD6
                             difference (Info::diffMethod = TRAD6, 5 ghosts), 1D and 2D

    python tests/golden/make_golden.py rhs_trad6   (one fixture only)
"""
from __future__ import annotations

import json
import os
import re
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle.refsolver import RefSolver, ref_flux, ref_inter5, ref_recon_face  # noqa: E402

REF_ROOT = Path(os.environ.get("CFD_REFERENCE_ROOT", "/root/reference"))
INTER_METHODS = [2, 3, 8, 9, 10, 11, 12, 13, 15, 22, 23, 35, 37]
GAMMA = 1.4


def prim_to_cons(prim):
    prim = np.asarray(prim, float)
    nv = prim.shape[-1]
    out = np.empty_like(prim)
    out[..., 0] = prim[..., 0]
    out[..., 1:nv - 1] = prim[..., :1] * prim[..., 1:nv - 1]
    out[..., nv - 1] = prim[..., nv - 1] / (GAMMA - 1) + 0.5 * prim[..., 0] * np.sum(prim[..., 1:nv - 1] ** 2, -1)
    return out


def quadrant_state(n, rng):
    P = np.array([[rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.05, 2)]
                  for _ in range(4)])
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    q = (X >= 0.5).astype(int) + 2 * (Y >= 0.5).astype(int)
    return prim_to_cons(P[q].reshape(-1, 4))


def smooth_state(n, rng):
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    a, b = rng.uniform(0.05, 0.3, 2)
    rho = 1 + a * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    u = 0.5 + b * np.sin(2 * np.pi * Y)
    v = 0.3 - b * np.cos(2 * np.pi * X)
    p = 1 + 0.1 * np.cos(2 * np.pi * (X + Y))
    return prim_to_cons(np.stack([rho, u, v, p], -1).reshape(-1, 4))


def sod_log():
    path = REF_ROOT / "zone_FD" / "cases" / "Sod - congTCNS5CT5 - 101.txt"
    rows = []
    for line in path.read_text().strip().splitlines():
        t = float(re.search(r"time = ([\d.]+)", line).group(1))
        dt = float(re.search(r"dt=([\d.]+)", line).group(1))
        lin = float(re.search(r"rhoLinf = ([\d.]+)", line).group(1))
        rows.append([t, dt, lin])
    return {
        "source": "zone_FD/cases/Sod - congTCNS5CT5 - 101.txt (reference run log)",
        "config": {"dim": 1, "cells": 100, "calZone": [-0.5, 0.5], "nCase": 0, "interMethod": 22,
                   "fluxMethod": "HLLC", "CFL": 0.5, "outputDt": 0.1, "endStep": 2},
        "format": "time (4 decimals), dt (10 decimals), rhoLinf (4 decimals) per RK3 step",
        "rows": rows,
    }


def order_txt():
    rows = []
    for line in (REF_ROOT / "CongFD1.0" / "order.txt").read_text().strip().splitlines()[1:]:
        rows.append([float(x) for x in line.split()])
    return {"source": "CongFD1.0/order.txt (AccuracyTest, TCNS5 face interpolation + MND6)",
            "columns": ["h", "L1order", "L2order", "Linforder"], "rows": rows}


def kat_inter5(rng):
    q = rng.normal(size=(200, 5)) * rng.choice([1e-3, 1, 1e3], size=(200, 1))
    adv = np.array([
        [1, 1, 1, 1, 1], [0, 0, 0, 0, 0], [0, 0, 1, 1, 1], [1, 1, 1, 0, 0], [1, 0, 1, 0, 1],
        [1e-12, 0, -1e-12, 0, 1e-12], [1, 2, 3, 4, 5], [5, 4, 3, 2, 1], [1, 1, 1, 1, 2], [2, 1, 1, 1, 1],
        [0, 1, 0, 1, 0], [1, 1, 2, 2, 2], [-1, -1, 1, 1, 1], [1e8, 1e8, -1e8, -1e8, 1e8], [3, 3, 3, 3, 3.0000001],
    ], float)
    q = np.concatenate([q, adv])
    out = {"q": q}
    for m in INTER_METHODS:
        out[f"m{m}"] = ref_inter5(m, q)
    return out


def kat_flux(rng):
    out = {}
    n = 200
    for dim in (1, 2):
        nv = dim + 2
        L = np.empty((n, nv))
        R = np.empty((n, nv))
        for S in (L, R):
            S[:, 0] = rng.uniform(0.05, 3, n)
            S[:, 1:nv - 1] = rng.uniform(-2, 2, (n, nv - 2))
            S[:, nv - 1] = rng.uniform(0.02, 3, n)
        R[:20] = L[:20]  # contact / equal states
        lr = np.concatenate([L, R], 1)
        out[f"lr{dim}d"] = lr
        for fm in (0, 1):
            for ax in range(dim):
                out[f"f{dim}d_fm{fm}_ax{ax}"] = ref_flux(dim, ax, fm, lr)
    return out


def rhs_2d(rng):
    out = {}
    cases = [("quad", 20, 2, 0, 0, False), ("quad", 20, 11, 1, 0, False), ("quad", 20, 8, 0, 2, False),
             ("quad", 20, 3, 1, 6, False), ("smooth", 24, 35, 1, 0, True), ("smooth", 24, 2, 0, 0, True),
             ("quad", 20, 15, 0, 0, False), ("quad", 20, 13, 1, 0, False)]
    meta = []
    for k, (kind, n, im, fm, ncase, periodic) in enumerate(cases):
        cons = quadrant_state(n, rng) if kind == "quad" else smooth_state(n, rng)
        r = RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=im, flux_method=fm, n_case=ncase, cfl=0.5,
                      periodic=periodic)
        r.cons = cons
        rhs = r.rhs()
        dt = r.max_dt()
        linf = r.solve(dt)
        out[f"c{k}_cons"] = cons
        out[f"c{k}_rhs"] = rhs
        out[f"c{k}_step"] = r.cons
        out[f"c{k}_dt"] = np.array([dt, linf])
        meta.append([k, n, im, fm, ncase, int(periodic)])
        r.close()
    out["meta"] = np.array(meta)
    return out


def sod_400():
    r = RefSolver(1, [400], [-0.5, 0.5, 0, 0, 0, 0], inter_method=2, flux_method=0, n_case=0, cfl=0.5)
    cons0 = r.cons
    dts, lin = r.run(1, 0.2)
    return {"cons0": cons0, "cons": r.cons, "dts": dts, "linf": lin}


def kat_face(rng):
    out = {}
    n = 120
    for dim in (1, 2):
        nv = dim + 2
        P = np.empty((n, 6, nv))
        P[..., 0] = rng.uniform(0.1, 2.0, (n, 6))
        P[..., 1:nv - 1] = rng.uniform(-1.5, 1.5, (n, 6, nv - 2))
        P[..., nv - 1] = rng.uniform(0.05, 2.0, (n, 6))
        # smooth stencils, shocked stencils and near-vacuum stencils
        x = np.linspace(0, 1, 6)
        P[:30] = P[:30, :1] + 0.05 * x[None, :, None] * P[:30, 1:2]
        P[30:40, 3:, 0] *= 8.0
        P[40:45, :, nv - 1] *= 1e-6
        out[f"p{dim}d"] = P
        for im in (2, 3, 11, 8, 15):
            for ny in range(dim):
                out[f"f{dim}d_m{im}_n{ny}"] = ref_recon_face(im, dim, ny, P)
    return out


def line_state(n, rng):
    """Three constant 1D regions (random prim) on n cells."""
    P = np.array([[rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(0.05, 2)] for _ in range(3)])
    q = np.minimum((np.arange(n) * 3) // n, 2)
    return prim_to_cons(P[q])


def rhs_trad6(rng):
    """TRAD6 (ExplicitDif6, differ.cpp:23-52) through the reference's own solver."""
    out = {}
    cases = [(1, "line", 40, 2, 0, 0, False), (1, "line", 40, 11, 1, 0, False), (1, "line", 40, 8, 0, 4, False),
             (1, "line", 40, 3, 1, 0, True), (2, "quad", 16, 2, 0, 0, False), (2, "quad", 16, 11, 1, 2, False),
             (2, "quad", 16, 8, 0, 6, False), (2, "smooth", 16, 35, 1, 0, True), (2, "quad", 16, 15, 1, 0, False),
             (2, "smooth", 16, 3, 0, 0, True)]
    meta = []
    for k, (dim, kind, n, im, fm, ncase, periodic) in enumerate(cases):
        if kind == "line":
            cons = line_state(n, rng)
            shape, zone = [n], [0, 1, 0, 0, 0, 0]
        else:
            cons = quadrant_state(n, rng) if kind == "quad" else smooth_state(n, rng)
            shape, zone = [n, n], [0, 1, 0, 1, 0, 0]
        r = RefSolver(dim, shape, zone, inter_method=im, flux_method=fm, n_case=ncase, cfl=0.5, periodic=periodic,
                      diff_method=1)
        r.cons = cons
        rhs = r.rhs()
        dt = r.max_dt()
        linf = r.solve(dt)
        out[f"c{k}_cons"] = cons
        out[f"c{k}_rhs"] = rhs
        out[f"c{k}_step"] = r.cons
        out[f"c{k}_dt"] = np.array([dt, linf])
        meta.append([k, dim, n, im, fm, ncase, int(periodic)])
        r.close()
    out["meta"] = np.array(meta)
    return out


def main():
    if sys.argv[1:] == ["rhs_trad6"]:
        np.savez_compressed(HERE / "rhs_trad6.npz", **rhs_trad6(np.random.default_rng(606)))
        return
    rng = np.random.default_rng(20261203)
    (HERE / "sod_congtcns5ct5_101.json").write_text(json.dumps(sod_log(), indent=0))
    (HERE / "order_congfd.json").write_text(json.dumps(order_txt(), indent=1))
    np.savez_compressed(HERE / "kat_inter5.npz", **kat_inter5(rng))
    np.savez_compressed(HERE / "kat_flux.npz", **kat_flux(rng))
    np.savez_compressed(HERE / "rhs_2d.npz", **rhs_2d(rng))
    np.savez_compressed(HERE / "sod_400.npz", **sod_400())
    np.savez_compressed(HERE / "kat_face.npz", **kat_face(np.random.default_rng(77)))
    np.savez_compressed(HERE / "rhs_trad6.npz", **rhs_trad6(np.random.default_rng(606)))
    for p in sorted(HERE.glob("*")):
        if p.suffix in (".npz", ".json"):
            print(p.name, p.stat().st_size)


if __name__ == "__main__":
    main()
