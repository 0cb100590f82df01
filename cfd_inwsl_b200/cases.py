"""Initial states of the benchmark configurations (host-side case setup).

The reference builds its initial states in Initializer::solInit
(zone_FD/src/src/initializer.cpp:9-566); the configurations below are not in
its case library, so they are set up here from their analytic definitions and
handed to BlockSolver.set_cons like any other initial state.
"""
from __future__ import annotations

import numpy as np

from .zone import GAMMA, prim_to_cons


def isentropic_vortex(n, t=0.0, L=10.0, beta=5.0):
    """Isentropic vortex of strength beta centred at (5,5) + (1,1) t on the
    periodic box [0,L]^2 with freestream (rho,u,v,p) = (1,1,1,1). Returns the
    cell-centred cons (n*n, 4) and h = L/n."""
    h = L / n
    x = (np.arange(n) + 0.5) * h
    X, Y = np.meshgrid(x, x)
    xc = (5.0 + t) % L
    yc = (5.0 + t) % L
    dx = (X - xc + L / 2) % L - L / 2
    dy = (Y - yc + L / 2) % L - L / 2
    r2 = dx * dx + dy * dy
    f = beta / (2 * np.pi) * np.exp(0.5 * (1 - r2))
    u = 1 - f * dy
    v = 1 + f * dx
    T = 1 - (GAMMA - 1) * beta ** 2 / (8 * GAMMA * np.pi ** 2) * np.exp(1 - r2)
    rho = T ** (1 / (GAMMA - 1))
    p = rho ** GAMMA
    return prim_to_cons(np.stack([rho, u, v, p], -1).reshape(-1, 4)), h


def tgv_state(n):
    """Compressible Taylor-Green vortex on the periodic box [0,2pi]^3:
    rho = 1, u = sin x cos y cos z, v = -cos x sin y cos z, w = 0,
    p = 100/1.4 + (cos 2x + cos 2y)(cos 2z + 2)/16. Returns cons (n^3, 5), h."""
    h = 2 * np.pi / n
    x = (np.arange(n) + 0.5) * h
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    p = 100 / 1.4 + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2) / 16
    prim = np.stack([np.ones_like(X), u, v, np.zeros_like(X), p], -1).reshape(-1, 5)
    return prim_to_cons(prim), h


def quadrant_prims(rng):
    """The four quadrant states (rho, u, v, p) of one seeded Riemann problem:
    rho ~ U[0.1,2], u, v ~ U[-1,1], p ~ U[0.05,2] (quadrants in the order
    lower-left, lower-right, upper-left, upper-right)."""
    return np.array([[rng.uniform(0.1, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(0.05, 2)]
                     for _ in range(4)])


def quadrant_state(P, n):
    """Cell-centred cons (n*n, 4) of the quadrant states P on [0,1]^2 split at (0.5, 0.5)."""
    X, Y = np.meshgrid((np.arange(n) + 0.5) / n, (np.arange(n) + 0.5) / n)
    q = (X >= 0.5).astype(int) + 2 * (Y >= 0.5).astype(int)
    return prim_to_cons(np.asarray(P)[q].reshape(-1, 4))


def riemann_quadrants(n, rng):
    """Four-quadrant 2D Riemann state on [0,1]^2 split at (0.5, 0.5): each
    quadrant's rho ~ U[0.1,2], u, v ~ U[-1,1], p ~ U[0.05,2]."""
    return quadrant_state(quadrant_prims(rng), n)


def riemann_batch(ncases=256, seed=0):
    """The batched configuration's cases: grid sizes N = round(2^U(7,10)) and
    quadrant states, drawn in this order from one seeded generator (sizes
    first, then each case's four states). Returns (sizes, prims)."""
    rng = np.random.default_rng(seed)
    sizes = [int(round(2 ** rng.uniform(7, 10))) for _ in range(ncases)]
    prims = [quadrant_prims(rng) for _ in sizes]
    return sizes, prims


def adjoint_problem(n=256, seed=0, nprobe=64):
    """Adjoint configuration on the periodic [0,1]^2, n^2 cells: rho = 1 + drho
    with drho seeded Gaussian noise periodically filtered to correlation length
    0.05 and scaled to RMS 1e-2, p = 1/gamma, (u, v) = (0.5, 0.3). Returns the
    AoS cons and nprobe seeded probe cells (the objective is the sum of rho^2
    over them)."""
    rng = np.random.default_rng(seed)
    k = np.fft.fftfreq(n, d=1.0 / n)
    KX, KY = np.meshgrid(k, k)
    noise = rng.normal(size=(n, n))
    filt = np.exp(-0.5 * (2 * np.pi * 0.05) ** 2 * (KX ** 2 + KY ** 2))
    drho = np.real(np.fft.ifft2(np.fft.fft2(noise) * filt))
    drho *= 1e-2 / np.sqrt(np.mean(drho ** 2))
    rho = 1.0 + drho.reshape(-1)
    cons = np.stack([rho, 0.5 * rho, 0.3 * rho, (1 / GAMMA) / (GAMMA - 1) + 0.5 * rho * (0.25 + 0.09)], -1)
    probes = rng.choice(n * n, nprobe, replace=False)
    return cons, probes


def kinetic_energy(cons, h):
    """sum over cells of rho |u|^2 / 2 h^3 (AoS 3D cons)."""
    c = np.asarray(cons)
    return float(np.sum(0.5 * (c[:, 1] ** 2 + c[:, 2] ** 2 + c[:, 3] ** 2) / c[:, 0]) * h ** 3)
