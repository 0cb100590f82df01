"""The C restatement oracle pinned against the reference's golden outputs (CPU only).

Fixtures come from tests/golden/make_golden.py (the reference compiled from its
own sources, and logs the reference repository commits).
"""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle.refsolver import ORC_MIRRORCOPY, ORC_OUTLET, ORC_SYMMETRY, ORC_WRAP, OracleC, orc_load

GOLD = Path(__file__).resolve().parent / "golden"

BC_OF_CASE = {0: [[ORC_OUTLET] * 2] * 3, 2: [[ORC_SYMMETRY] * 2] * 3, 6: [[ORC_MIRRORCOPY] * 2] * 3}


@pytest.fixture(scope="module")
def orc():
    try:
        return orc_load()
    except RuntimeError as e:
        pytest.skip(str(e))


def test_inter5_kat_bitwise(orc):
    from oracle.refsolver import ORC_FAMILY
    import ctypes as C
    g = np.load(GOLD / "kat_inter5.npz")
    q = g["q"]
    for key in g.files:
        if not key.startswith("m"):
            continue
        m = int(key[1:])
        fam, c = ORC_FAMILY[m]
        out = np.array([orc.orc_inter5(fam, c, C.c_void_p(np.ascontiguousarray(row).ctypes.data)) for row in q])
        np.testing.assert_array_equal(out, g[key], err_msg=f"interMethod {m}")


def test_rhs_and_step_2d_bitwise(orc):
    g = np.load(GOLD / "rhs_2d.npz")
    for k, n, im, fm, ncase, periodic in g["meta"]:
        bc = [[ORC_WRAP] * 2] * 3 if periodic else BC_OF_CASE[int(ncase)]
        o = OracleC(2, [n, n], 1.0 / n, int(im), int(fm), bc=bc)
        o.cons = g[f"c{k}_cons"]
        np.testing.assert_array_equal(o.rhs(), g[f"c{k}_rhs"], err_msg=f"case {k}")
        dt, linf = g[f"c{k}_dt"]
        assert o.max_dt(0.5) == dt
        assert o.solve(dt) == linf
        np.testing.assert_array_equal(o.cons, g[f"c{k}_step"])


def run_cfl(o, cfl, end_step, output_dt, max_steps=100000):
    """BlockSolver::stepsLoopCFL restated around the oracle (blockSolver.cpp:170-235)."""
    step, outT, dts, lin = 0, 0.0, [], []
    while step < end_step and len(dts) < max_steps:
        dt = o.max_dt(cfl)
        if outT + dt > output_dt:
            dt = output_dt - outT
            outT = 0.0
            step += 1
        else:
            outT += dt
        lin.append(o.solve(dt))
        dts.append(dt)
    return np.array(dts), np.array(lin)


def test_sod_400_bitwise(orc):
    g = np.load(GOLD / "sod_400.npz")
    o = OracleC(1, [400], 1.0 / 400, 2, 0)
    o.cons = g["cons0"]
    dts, lin = run_cfl(o, 0.5, 1, 0.2)
    np.testing.assert_array_equal(dts, g["dts"])
    np.testing.assert_array_equal(lin, g["linf"])
    np.testing.assert_array_equal(o.cons, g["cons"])


def test_reference_sod_log(orc):
    """Reproduces the reference's committed run log (dt to 10, rhoLinf to 4 decimals)."""
    log = json.loads((GOLD / "sod_congtcns5ct5_101.json").read_text())
    rows = np.array(log["rows"])
    assert len(rows) == 172
    n = 100
    h = 1.0 / n
    x = -0.5 + (np.arange(n) + 0.5) * h
    cons = np.where(x[:, None] < 0, [1.0, 0.0, 1.0 / 0.4], [0.125, 0.0, 1.0 / 0.4 * 0.1])
    o = OracleC(1, [n], h, 22, 0)
    o.cons = np.ascontiguousarray(cons)
    dts, lin = run_cfl(o, 0.5, 2, 0.1)
    assert len(dts) == 86
    for half in (rows[:86], rows[86:]):
        assert np.all(np.round(dts, 10) == half[:, 1])
        assert np.all(np.round(lin, 4) == half[:, 2])


def test_z_invariance_3d(orc):
    """3D restatement on a z-invariant field with w = 0 reproduces the 2D path."""
    rng = np.random.default_rng(3)
    n, nz = 16, 8
    x = (np.arange(n) + 0.5) / n
    X, Y = np.meshgrid(x, x)
    prim2 = np.stack([1 + 0.2 * np.sin(2 * np.pi * X), 0.4 + 0.1 * np.cos(2 * np.pi * Y),
                      -0.2 + 0.1 * np.sin(2 * np.pi * (X + Y)), 1 + 0.1 * rng.random(X.shape)], -1).reshape(-1, 4)
    from tests.golden.make_golden import prim_to_cons
    c2 = prim_to_cons(prim2)
    prim3 = np.zeros((nz, n * n, 5))
    prim3[:, :, 0] = prim2[:, 0]
    prim3[:, :, 1] = prim2[:, 1]
    prim3[:, :, 2] = prim2[:, 2]
    prim3[:, :, 4] = prim2[:, 3]
    c3 = prim_to_cons(prim3.reshape(-1, 5))
    for im, fm in ((2, 0), (11, 1)):
        o2 = OracleC(2, [n, n], 1.0 / n, im, fm, bc=[[ORC_WRAP] * 2] * 3)
        o3 = OracleC(3, [n, n, nz], 1.0 / n, im, fm, bc=[[ORC_WRAP] * 2] * 3)
        r2 = o2.rhs(c2)
        r3 = o3.rhs(np.ascontiguousarray(c3)).reshape(nz, n * n, 5)
        for k in range(nz):
            np.testing.assert_allclose(r3[k][:, [0, 1, 2, 4]], r2, rtol=0, atol=1e-12 * np.abs(r2).max())
            assert np.abs(r3[k][:, 3]).max() <= 1e-14 * np.abs(r2).max()


def test_reference_cross_check_random(orc, ref):
    """C oracle vs the compiled reference on fresh random 2D states (all selector entries)."""
    from tests.golden.make_golden import INTER_METHODS, quadrant_state
    rng = np.random.default_rng(7)
    for im in INTER_METHODS:
        for fm in (0, 1):
            n = 12
            c = quadrant_state(n, rng)
            r = ref.RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=im, flux_method=fm, n_case=0)
            r.cons = c
            o = OracleC(2, [n, n], 1.0 / n, im, fm)
            np.testing.assert_array_equal(o.rhs(c), r.rhs())


def test_trad6_bitwise(orc):
    """TRAD6 (ExplicitDif6, 5 ghosts): the C restatement against the reference's
    own RHS, CFL step and RK3 step, 1D and 2D (tests/golden/rhs_trad6.npz)."""
    g = np.load(GOLD / "rhs_trad6.npz")
    bc_1d = {0: [[ORC_OUTLET] * 2] * 3, 4: [[ORC_SYMMETRY] * 2] * 3}
    for k, dim, n, im, fm, ncase, periodic in g["meta"]:
        if periodic:
            bc = [[ORC_WRAP] * 2] * 3
        else:
            bc = bc_1d[int(ncase)] if dim == 1 else BC_OF_CASE[int(ncase)]
        shape = [n] if dim == 1 else [n, n]
        o = OracleC(int(dim), shape, 1.0 / n, int(im), int(fm), bc=bc, trad6=True)
        o.cons = g[f"c{k}_cons"]
        np.testing.assert_array_equal(o.rhs(), g[f"c{k}_rhs"], err_msg=f"case {k}")
        dt, linf = g[f"c{k}_dt"]
        assert o.max_dt(0.5) == dt
        assert o.solve(dt) == linf
        np.testing.assert_array_equal(o.cons, g[f"c{k}_step"], err_msg=f"case {k}")
