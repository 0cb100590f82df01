"""Discrete adjoint (cfd_rhs_vjp, cfd_adjoint_record / cfd_adjoint_reverse)
against central finite differences.

The adjoint differentiates the 2D WCNS5 / TENO + Roe + MND6 path on periodic
grids (TENO with its cut-off decisions frozen).
Checks, along seeded random directions d of the state:
  * one RHS: mu . (R(U + eps d) - R(U - eps d)) / (2 eps) = (J^T mu) . d
  * N frozen-dt SSP-RK3 steps, J = sum over probe cells of rho^2 at step N:
    (J(U0 + eps d) - J(U0 - eps d)) / (2 eps) = (dJ/dU0) . d,
    with the forward of the finite differences run by this library and, for
    the pin to the reference, by the reference solver itself (RefSolver).
Tolerance: 1e-6 relative. For WCNS5 the finite differences are Richardson-extrapolated
central differences with steps of 2e-7 and 1e-7 of the state: WCNS5's weights
gamma_k / (1e-6 + beta_k)^2 vary on the scale of their 1e-6 wherever a
characteristic field is nearly constant (beta_k ~ 1e-6 or below, as for the
acoustic fields of a density perturbation at uniform pressure), so plain
central differences with steps of 1e-5 or 1e-6 carry truncation errors of
1e-4 to 1e-5 there, not the adjoint.

TENO's forward map is only piecewise smooth: a cut-off decision flips where a
stencil's measure crosses the cut-off, and a finite difference whose step
crosses one sees a jump. On states whose characteristic fields all vary
(excited_periodic) the decisions are robust to steps of 2e-8 of the state but
not to 2e-7, so TENO is checked with plain central differences of step 2e-8
(rounding noise ~1e-8 relative); a direction whose differences at 2e-8 and
1e-8 disagree (a decision within the step of its boundary) is set aside and
another drawn. States with a characteristic field constant
up to rounding (a pure density perturbation) leave that field's TENO
decisions to rounding noise; the map is not differentiable there along
directions that excite the field.
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


def excited_periodic(nx, ny, rng, amp=0.1):
    """Smooth periodic rho, u, v and p (every characteristic field varies)."""
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)

    def f():
        return sum(rng.normal() * np.sin(2 * np.pi * (rng.integers(1, 4) * X + rng.integers(1, 4) * Y) +
                                         rng.uniform(0, 2 * np.pi)) for _ in range(3)) / 3

    prim = np.stack([1 + amp * f(), 0.5 + amp * f(), 0.3 + amp * f(), 1 / 1.4 + amp * f()], -1).reshape(-1, 4)
    return zone.prim_to_cons(prim)


def central(fun, eps=2e-8):
    """Central difference at eps, or None when the one at eps / 2 disagrees
    with it (a cut-off decision flips within the step)."""
    d1 = (fun(eps) - fun(-eps)) / (2 * eps)
    d2 = (fun(eps / 2) - fun(-eps / 2)) / eps
    return d1 if abs(d1 - d2) <= 2e-7 * max(abs(d1), abs(d2)) else None


def check_directions(g, U0, rng, diff, J_of, need=3, tries=10):
    """dJ/dU0 . d against diff(J) along seeded directions d ~ N(0, |U0|)."""
    done = 0
    for _ in range(tries):
        d = rng.normal(size=U0.shape) * np.abs(U0)
        fd = diff(lambda e: J_of(U0 + e * d))
        if fd is None:
            continue
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= TOL * max(abs(fd), abs(ad)), (fd, ad)
        done += 1
        if done == need:
            return
    assert done == need, f"only {done} of {need} directions free of cut-off flips"


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


@pytest.mark.parametrize("nsteps,ckpt,im", [(12, 5, 2), (7, 7, 2), (6, 1, 2), (12, 5, 11), (7, 3, 8), (6, 2, 13)])
def test_adjoint_matches_finite_differences(nsteps, ckpt, im):
    """im 2: WCNS5; 11 / 13: TENO-Z (cut-off 1e-5 / 1e-7); 8: TENO-Cong. TENO's
    cut-off is frozen in the adjoint; the finite differences see the same
    selection as long as no decision sits within the step of its boundary."""
    rng = np.random.default_rng(100 + nsteps + im)
    nx, ny = 32, 28
    s = solver(nx, ny, im=im)
    U0 = smooth_periodic(nx, ny, rng, amp=0.1) if im == 2 else excited_periodic(nx, ny, rng)
    diff = richardson if im == 2 else central
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    probes = rng.choice(nx * ny, 16, replace=False)
    s.adjoint_record(dt, nsteps, ckpt)
    UN = s.cons
    np.testing.assert_allclose(UN, forward(solver(nx, ny, im=im), U0, dt, nsteps), rtol=0, atol=1e-13)
    g = s.adjoint_reverse(seed(UN, probes))
    f = solver(nx, ny, im=im)
    check_directions(g, U0, rng, diff, lambda U: objective(forward(f, U, dt, nsteps), probes))


@pytest.mark.parametrize("nsteps,ckpt", [(12, 5), (10, 5), (4, 6)])
def test_reverse_twice_after_one_record(nsteps, ckpt):
    """The record pass keeps its last segment's stage states for the first
    reverse pass, which then skips recomputing that segment; a second reverse
    pass recomputes it from the checkpoint. Both give the same gradient, bit
    for bit (full and partial last segments, one segment)."""
    rng = np.random.default_rng(31 + nsteps)
    nx, ny = 32, 28
    s = solver(nx, ny)
    U0 = smooth_periodic(nx, ny, rng, amp=0.1)
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    probes = rng.choice(nx * ny, 16, replace=False)
    s.adjoint_record(dt, nsteps, ckpt)
    sd = seed(s.cons, probes)
    g1 = s.adjoint_reverse(sd)
    g2 = s.adjoint_reverse(sd)
    np.testing.assert_array_equal(g1, g2)


@pytest.mark.parametrize("im", [2, 11])
def test_adjoint_pinned_by_reference_forward(ref, im):
    """dJ/dU0 . d against central differences of the reference solver's own
    RK3_SSP steps (zone_FD compiled from its sources), WCNS5 or TENO5 (cut-off
    frozen) + Roe, periodic."""
    rng = np.random.default_rng(7 + im)
    nx = ny = 24 if im == 2 else 32  # (24^2 TENO: one decision within 1e-8 of its boundary for every direction)
    s = solver(nx, ny, im=im)
    U0 = smooth_periodic(nx, ny, rng, amp=0.1) if im == 2 else excited_periodic(nx, ny, rng)
    diff = richardson if im == 2 else central
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    nsteps = 8
    probes = rng.choice(nx * ny, 12, replace=False)
    s.adjoint_record(dt, nsteps, 3)
    g = s.adjoint_reverse(seed(s.cons, probes))
    r = ref.RefSolver(2, [nx, ny], [0, 1, 0, 1, 0, 0], inter_method=im, flux_method=1, n_case=0, periodic=True)

    def ref_J(U):
        r.cons = U
        for _ in range(nsteps):
            r.solve(dt)
        return objective(r.cons, probes)

    check_directions(g, U0, rng, diff, ref_J, need=2)


def test_autograd_function_wrapper():
    """The adjoint through torch.autograd (test harness wrapper): J computed
    by torch from U^N, J.backward() gives dJ/dU0 = cfd_adjoint_reverse(dJ/dU^N)."""
    import torch
    from tests.adjoint_autograd import RK3Frozen
    rng = np.random.default_rng(19)
    nx, ny = 24, 20
    s = solver(nx, ny)
    U0 = smooth_periodic(nx, ny, rng, amp=0.1)
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    probes = rng.choice(nx * ny, 10, replace=False)
    U0_t = torch.tensor(U0, requires_grad=True)
    UN = RK3Frozen.apply(U0_t, s, dt, 9, 4)
    J = (UN[torch.as_tensor(probes), 0] ** 2).sum()
    J.backward()
    assert abs(J.item() - objective(forward(solver(nx, ny), U0, dt, 9), probes)) <= 1e-13 * J.item()
    s2 = solver(nx, ny)
    s2.set_cons(U0)
    s2.adjoint_record(dt, 9, 4)
    np.testing.assert_array_equal(U0_t.grad.numpy(), s2.adjoint_reverse(seed(s2.cons, probes)))
    d = rng.normal(size=U0.shape) * np.abs(U0)
    f = solver(nx, ny)
    fd = richardson(lambda e: objective(forward(f, U0 + e * d, dt, 9), probes))
    ad = float(np.sum(U0_t.grad.numpy() * d))
    assert abs(fd - ad) <= TOL * max(abs(fd), abs(ad)), (fd, ad)


def test_adjoint_full_configuration_32_directions():
    """The adjoint configuration itself: 256^2 periodic, WCNS5 + Roe, 400
    frozen-dt RK3 steps, checkpoints every 20, J = sum of rho^2 over 64 seeded
    probes, against central differences (Richardson, module docstring, density
    step 1e-6) along 32 seeded directions of the initial density at fixed
    velocity and pressure."""
    from cfd_inwsl_b200.cases import adjoint_problem
    n, nsteps = 256, 400
    U0, probes = adjoint_problem(n, seed=0)
    info = make_info(2, [n, n], [0, 1, 0, 1, 0, 0], im=2, fm=1)
    s = zone.BlockSolver(info, periodic=True)
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    s.adjoint_record(dt, nsteps, 20)
    g = s.adjoint_reverse(seed(s.cons, probes))
    f = zone.BlockSolver(info, periodic=True)
    rng = np.random.default_rng(32)
    u, v = U0[:, 1] / U0[:, 0], U0[:, 2] / U0[:, 0]
    worst = 0.0
    for _ in range(32):
        dr = rng.normal(size=n * n)
        d = np.stack([dr, u * dr, v * dr, 0.5 * (u * u + v * v) * dr], -1)  # d cons / d rho at fixed u, v, p
        fd = richardson(lambda e: objective(forward(f, U0 + e * d, dt, nsteps), probes), eps=1e-6)
        ad = float(np.sum(g * d))
        worst = max(worst, abs(fd - ad) / max(abs(fd), abs(ad)))
    assert worst <= TOL, worst


def test_adjoint_rejects_unsupported_configurations():
    s = solver(16, 16, im=3, fm=1)  # WENO-Z: not differentiated
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


def test_adjoint_full_configuration_against_reference_solver_fd(ref):
    """The adjoint configuration (256^2 periodic, WCNS5 + Roe, 400 frozen-dt
    RK3 steps, checkpoints every 20, J = sum of rho^2 over 64 seeded probes)
    against finite differences of the reference solver's own RK3_SSP steps
    (zone_FD compiled from its sources), along 3 seeded directions of the
    initial density at fixed velocity and pressure (Richardson central
    differences, density step 1e-6), to 1e-6 relative."""
    from cfd_inwsl_b200.cases import adjoint_problem
    n, nsteps = 256, 400
    U0, probes = adjoint_problem(n, seed=0)
    info = make_info(2, [n, n], [0, 1, 0, 1, 0, 0], im=2, fm=1)
    s = zone.BlockSolver(info, periodic=True)
    s.set_cons(U0)
    dt = s.getTimeIntervalExplicit()
    s.adjoint_record(dt, nsteps, 20)
    g = s.adjoint_reverse(seed(s.cons, probes))
    s.close()
    r = ref.RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=2, flux_method=1, n_case=0, periodic=True)

    def ref_J(U):
        r.cons = U
        for _ in range(nsteps):
            r.solve(dt)
        return objective(r.cons, probes)

    rng = np.random.default_rng(33)
    u, v = U0[:, 1] / U0[:, 0], U0[:, 2] / U0[:, 0]
    for _ in range(3):
        dr = rng.normal(size=n * n)
        d = np.stack([dr, u * dr, v * dr, 0.5 * (u * u + v * v) * dr], -1)
        fd = richardson(lambda e: ref_J(U0 + e * d), eps=1e-6)
        ad = float(np.sum(g * d))
        assert abs(fd - ad) <= TOL * max(abs(fd), abs(ad)), (fd, ad)
    r.close()
