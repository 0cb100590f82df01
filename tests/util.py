"""Shared helpers for the parity tests: build matching GPU and reference solvers."""
from __future__ import annotations

import numpy as np

from cfd_inwsl_b200 import zone

GAMMA = 1.4


def make_info(dim, n, zone_=None, im=2, fm=0, strict=False, ncase=0, cfl=0.5, seg_len=(0, 0, 0), precision=0):
    info = zone.Info()
    info.dim = dim
    n3 = list(n) + [1] * (3 - len(n))
    info.iMax = [k + 1 if k > 1 else 1 for k in n3]
    info.calZone = list(zone_) if zone_ is not None else [0, 1, 0, 1, 0, 1]
    info.interMethod = im
    info.fluxMethod = fm
    info.strict = strict
    info.nCase = ncase
    info.CFL = cfl
    info.seg_len = list(seg_len)
    info.precision = precision
    return info


def gpu_solver(dim, n, zone_=None, im=2, fm=0, strict=False, ncase=0, periodic=False, bc=None, cfl=0.5,
               seg_len=(0, 0, 0), precision=0):
    info = make_info(dim, n, zone_, im, fm, strict, ncase, cfl, seg_len, precision)
    return zone.BlockSolver(info, bc=bc, periodic=periodic)


def quadrant_state(n, rng):
    P = np.array([[rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.05, 2)]
                  for _ in range(4)])
    ny = n if np.isscalar(n) else n[1]
    nx = n if np.isscalar(n) else n[0]
    X, Y = np.meshgrid((np.arange(nx) + 0.5) / nx, (np.arange(ny) + 0.5) / ny)
    q = (X >= 0.5).astype(int) + 2 * (Y >= 0.5).astype(int)
    return zone.prim_to_cons(P[q].reshape(-1, 4))


def smooth_state_3d(n, rng, w=True):
    nx, ny, nz = n
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    z = (np.arange(nz) + 0.5) / nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    a = rng.uniform(0.1, 0.3)
    rho = 1 + a * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y) * np.cos(2 * np.pi * Z)
    u = 0.4 + 0.2 * np.sin(2 * np.pi * (Y + Z))
    v = -0.3 + 0.2 * np.cos(2 * np.pi * (X + Z))
    ww = (0.2 * np.sin(2 * np.pi * (X - Y))) if w else np.zeros_like(X)
    p = 1 + 0.2 * np.cos(2 * np.pi * (X + Y + Z))
    return zone.prim_to_cons(np.stack([rho, u, v, ww, p], -1).reshape(-1, 5))


from cfd_inwsl_b200.cases import isentropic_vortex, tgv_state  # noqa: E402,F401


def rel_linf(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
