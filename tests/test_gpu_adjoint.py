"""Discrete adjoint (cfd_rhs_vjp, cfd_adjoint_record / cfd_adjoint_reverse)
against central finite differences.

The adjoint differentiates the 2D WCNS5 + Roe + MND6 path on periodic grids.
Checks, along seeded random directions d of the state:
  * one RHS: mu . (R(U + eps d) - R(U - eps d)) / (2 eps) = (J^T mu) . d
  * N frozen-dt SSP-RK3 steps, J = sum over probe cells of rho^2 at step N:
    (J(U0 + eps d) - J(U0 - eps d)) / (2 eps) = (dJ/dU0) . d,
    with the forward of the finite differences run by this library and, for
    the pin to the reference, by the reference solver itself (RefSolver).
Tolerance: 1e-6 relative. The finite differences are Richardson-extrapolated
central differences with steps of 2e-7 and 1e-7 of the state: WCNS5's weights
gamma_k / (1e-6 + beta_k)^2 vary on the scale of their 1e-6 wherever a
characteristic field is nearly constant (beta_k ~ 1e-6 or below, as for the
acoustic fields of a density perturbation at uniform pressure), so plain
central differences with steps of 1e-5 or 1e-6 carry truncation errors of
1e-4 to 1e-5 there, not the adjoint.
"""
import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, zone
from tests.util import make_info

pytestmark = pytest.mark.gpu
TOL = 1e-6


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def smooth_periodic(nx, ny, rng, amp=0.05):
    """rho = 1 + delta rho, p = 1/gamma, (u, v) = (0.5, 0.3): the adjoint configuration's shape."""
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    d = np.zeros_like(X)
    for _ in range(4):
        kx, ky = rng.integers(1, 4, 2)
        d += rng.normal() * np.sin(2 * np.pi * (kx * X + ky * Y) + rng.uniform(0, 2 * np.pi))
    rho = 1 + amp * d / np.abs(d).max()
    prim = np.stack([rho, 0.5 + 0 * X, 0.3 + 0 * X, 1 / 1.4 + 0 * X], -1).reshape(-1, 4)
    return zone.prim_to_cons(prim)


def richardson(fun, eps=2e-7):
    """(4 D(eps/2) - D(eps)) / 3 with D(e) = (fun(e) - fun(-e)) / (2 e)."""
    d1 = (fun(eps) - fun(-eps)) / (2 * eps)
    d2 = (fun(eps / 2) - fun(-eps / 2)) / eps
    return (4 * d2 - d1) / 3


def solver(nx, ny, strict=False, im=2, fm=1):
    info = make_info(2, [nx, ny], [0, 1, 0, ny / nx, 0, 0], im=im, fm=fm, strict=strict)
    return zone.BlockSolver(info, periodic=True)


def test_rhs_vjp_matches_finite_differences():
    rng = np.random.default_rng(11)
    nx, ny = 40, 24
    s = solver(nx, ny)
    U = smooth_periodic(nx, ny, rng)
    mu = rng.normal(size=U.shape)
    s.set_cons(U)
    lam = s.rhs_vjp(mu)
    def mu_R(U1):
        s.set_cons(U1)
        return float(np.sum(mu * s.rhsSolve()))

    for _ in range(3):
        d = rng.normal(size=U.shape) * np.abs(U)
        fd = richardson(lambda e: mu_R(U + e * d))
        ad = np.sum(lam * d)
        assert abs(fd - ad) <= TOL * max(abs(fd), abs(ad)), (fd, ad)


def test_rhs_vjp_per_cell_against_finite_differences():
    """Single-cell directions: each entry of J^T mu on a small grid."""
    rng = np.random.default_rng(3)
    nx, ny = 12, 10
    s = solver(nx, ny)
    U = smooth_periodic(nx, ny, rng, amp=0.3)
    mu = rng.normal(size=U.shape)
    s.set_cons(U)
    lam = s.rhs_vjp(mu)
    def mu_R(U1):
        s.set_cons(U1)
        return float(np.sum(mu * s.rhsSolve()))

    for cell in rng.choice(nx * ny, 6, replace=False):
        for v in range(4):
            d = np.zeros_like(U)
            d[cell, v] = max(abs(U[cell, v]), 1.0)
            fd = richardson(lambda e: mu_R(U + e * d)) / d[cell, v]
            assert abs(fd - lam[cell, v]) <= 1e-6 * max(abs(fd), 1e-2 * np.abs(lam).max()), (cell, v, fd, lam[cell, v])


def objective(U, probes):
    return float(np.sum(U[probes, 0] ** 2))


def seed(U, probes):
    g = np.zeros_like(U)
    g[probes, 0] = 2 * U[probes, 0]
    return g


def forward(s, U0, dt, n):
    s.set_cons(U0)
    for _ in range(n):
        s.RK3_SSP(dt)
    return s.cons


@pytest.mark.parametrize("nsteps,ckpt", [(12, 5), (7, 7), (6, 1)])
def test_adjoint_matches_finite_differences(nsteps, ckpt):
    rng = np.random.default_rng(100 + nsteps)
    nx, ny = 32, 28
    s = solver(nx, ny)
    U0 = smooth_periodic(nx, ny, rng, amp=0.1)
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    probes = rng.choice(nx * ny, 16, replace=False)
    s.adjoint_record(dt, nsteps, ckpt)
    UN = s.cons
    np.testing.assert_allclose(UN, forward(solver(nx, ny), U0, dt, nsteps), rtol=0, atol=1e-13)
    g = s.adjoint_reverse(seed(UN, probes))
    f = solver(nx, ny)
    for _ in range(3):
        d = rng.normal(size=U0.shape) * np.abs(U0)
        fd = richardson(lambda e: objective(forward(f, U0 + e * d, dt, nsteps), probes))
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= TOL * max(abs(fd), abs(ad)), (fd, ad)


def test_adjoint_pinned_by_reference_forward(ref):
    """dJ/dU0 . d against central differences of the reference solver's own
    RK3_SSP steps (zone_FD compiled from its sources), WCNS5 + Roe, periodic."""
    rng = np.random.default_rng(7)
    nx = ny = 24
    s = solver(nx, ny)
    U0 = smooth_periodic(nx, ny, rng, amp=0.1)
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    nsteps = 8
    probes = rng.choice(nx * ny, 12, replace=False)
    s.adjoint_record(dt, nsteps, 3)
    g = s.adjoint_reverse(seed(s.cons, probes))
    r = ref.RefSolver(2, [nx, ny], [0, 1, 0, 1, 0, 0], inter_method=2, flux_method=1, n_case=0, periodic=True)

    def ref_J(U):
        r.cons = U
        for _ in range(nsteps):
            r.solve(dt)
        return objective(r.cons, probes)

    for _ in range(2):
        d = rng.normal(size=U0.shape) * np.abs(U0)
        fd = richardson(lambda e: ref_J(U0 + e * d))
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= TOL * max(abs(fd), abs(ad)), (fd, ad)


def test_adjoint_rejects_unsupported_configurations():
    s = solver(16, 16, im=11, fm=1)  # TENO: not differentiated
    with pytest.raises(_lib.CfdError) as e:
        s.rhs_vjp(np.zeros((256, 4)))
    assert e.value.code == -6
    info = make_info(2, [16, 16], im=2, fm=1)
    o = zone.BlockSolver(info)  # outlet boundaries
    with pytest.raises(_lib.CfdError) as e:
        o.adjoint_record(1e-3, 2, 1)
    assert e.value.code == -6
    p = solver(16, 16)
    with pytest.raises(_lib.CfdError) as e:
        p.adjoint_reverse(np.zeros((256, 4)))
    assert e.value.code == -1
