"""3D Taylor-Green vortex (the throughput configuration, scaled down to 32^3):
the kinetic-energy history sum rho |u|^2 / 2 h^3 of every step, FP64 strict
against the C restatement (bit for bit: state and energy), and the mixed form
against FP64 on the same dt sequence."""
import numpy as np
import pytest

from cfd_inwsl_b200 import cases
from tests.util import gpu_solver

pytestmark = pytest.mark.gpu
N, STEPS = 32, 20


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def history(solver_or_oracle, dts, h):
    ke = [cases.kinetic_energy(solver_or_oracle.cons, h)]
    for dt in dts:
        solver_or_oracle.solve(dt)
        ke.append(cases.kinetic_energy(solver_or_oracle.cons, h))
    return np.array(ke)


def test_tgv_energy_history_against_c_oracle():
    from oracle.refsolver import ORC_WRAP, OracleC
    c, h = cases.tgv_state(N)
    zone_ = [0, 2 * np.pi, 0, 2 * np.pi, 0, 2 * np.pi]
    s = gpu_solver(3, [N] * 3, zone_, im=2, fm=0, strict=True, periodic=True)
    o = OracleC(3, [N] * 3, s.info.geth(0), 2, 0, bc=[[ORC_WRAP] * 2] * 3)
    s.set_cons(c)
    o.cons = c
    ke_o, ke_g = [cases.kinetic_energy(c, h)], [cases.kinetic_energy(c, h)]
    for _ in range(STEPS):
        dt = o.max_dt(0.5)
        assert s.getTimeIntervalExplicit() == dt
        o.solve(dt)
        s.solve(dt)
        ke_o.append(cases.kinetic_energy(o.cons, h))
        ke_g.append(cases.kinetic_energy(s.cons, h))
    np.testing.assert_array_equal(s.cons, o.cons)
    assert ke_g == ke_o
    assert ke_g[-1] < ke_g[0]  # the scheme dissipates kinetic energy


def test_tgv_mixed_energy_history_close_to_fp64():
    """Mixed form: kinetic energy within 1e-9 relative of FP64 at every step
    (the dt sequence of the FP64 run for both)."""
    c, h = cases.tgv_state(N)
    zone_ = [0, 2 * np.pi, 0, 2 * np.pi, 0, 2 * np.pi]
    s64 = gpu_solver(3, [N] * 3, zone_, im=2, fm=0, periodic=True)
    s32 = gpu_solver(3, [N] * 3, zone_, im=2, fm=0, periodic=True, precision=1)
    s64.set_cons(c)
    s32.set_cons(c)
    dts = []
    for _ in range(STEPS):
        dt = s64.getTimeIntervalExplicit()
        s64.solve(dt)
        dts.append(dt)
    s64.set_cons(c)
    k64 = history(s64, dts, h)
    k32 = history(s32, dts, h)
    dev = np.max(np.abs(k32 - k64) / k64)
    print("max relative KE deviation, mixed vs FP64:", dev)
    assert dev < 1e-9


def test_tgv_64_energy_history_100_steps():
    """The throughput configuration's physics at 64^3: 100 CFL steps (CFL 0.5,
    WCNS5 + HLLC). The strict flavour's dt, state and kinetic-energy history
    equal the C restatement's bit for bit at every step; the fast flavour,
    taking its own dt, stays within 1e-10 relative L-inf of the strict state
    after the 100 steps (the WCNS5 weights are continuous: FMA rounding cannot
    switch a stencil)."""
    from oracle.refsolver import ORC_WRAP, OracleC
    from tests.util import rel_linf
    n, steps = 64, 100
    c, h = cases.tgv_state(n)
    zone_ = [0, 2 * np.pi, 0, 2 * np.pi, 0, 2 * np.pi]
    s = gpu_solver(3, [n] * 3, zone_, im=2, fm=0, strict=True, periodic=True)
    f = gpu_solver(3, [n] * 3, zone_, im=2, fm=0, strict=False, periodic=True)
    o = OracleC(3, [n] * 3, s.info.geth(0), 2, 0, bc=[[ORC_WRAP] * 2] * 3)
    s.set_cons(c)
    f.set_cons(c)
    o.cons = c
    ke_o, ke_g = [cases.kinetic_energy(c, h)], [cases.kinetic_energy(c, h)]
    for _ in range(steps):
        dt = o.max_dt(0.5)
        assert s.getTimeIntervalExplicit() == dt
        o.solve(dt)
        s.solve(dt)
        f.solve(f.getTimeIntervalExplicit())
        ke_o.append(cases.kinetic_energy(o.cons, h))
        ke_g.append(cases.kinetic_energy(s.cons, h))
    np.testing.assert_array_equal(s.cons, o.cons)
    assert ke_g == ke_o
    assert rel_linf(f.cons, s.cons) <= 1e-10
    for x in (s, f):
        x.close()
