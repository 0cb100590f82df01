"""The TRAD6 difference (ExplicitDif6, zone_FD/src/src/differ.cpp:23-52) on the
GPU: Info::diffMethod = TRAD6, five ghost cells per line end (info.cpp:7-22),
n + 5 faces per line and no node fluxes (SolverType::initDiffer,
solverType.cpp:657-681).

Strict flavour: bit for bit against the reference's own RHS, CFL step and RK3
steps (committed fixtures tests/golden/rhs_trad6.npz, and the compiled
reference for multi-step runs and the named cases); 3D against the C
restatement. Fast flavour: within 1e-12 relative L-inf after one step.
"""
from pathlib import Path

import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, zone
from tests.util import make_info, quadrant_state, rel_linf, smooth_state_3d

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
TOL = 1e-12


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def trad6_solver(dim, n, zone_=None, im=2, fm=0, strict=True, ncase=0, periodic=False, bc=None, seg_len=(0, 0, 0),
                 cfl=0.5):
    info = make_info(dim, n, zone_, im, fm, strict, ncase, cfl, seg_len)
    info.diffMethod = zone.DiffMethod.TRAD6
    return zone.BlockSolver(info, bc=bc, periodic=periodic)


@pytest.mark.parametrize("strict", [True, False])
def test_trad6_golden(strict):
    g = np.load(GOLD / "rhs_trad6.npz")
    for k, dim, n, im, fm, ncase, periodic in g["meta"]:
        shape = [n] if dim == 1 else [n, n]
        zone_ = [0, 1, 0, 0, 0, 0] if dim == 1 else [0, 1, 0, 1, 0, 0]
        s = trad6_solver(int(dim), shape, zone_, int(im), int(fm), strict, int(ncase), bool(periodic))
        s.set_cons(g[f"c{k}_cons"])
        rhs = s.rhsSolve()
        dt_ref, linf_ref = g[f"c{k}_dt"]
        dt = s.getTimeIntervalExplicit()
        linf = s.solve(dt_ref)
        if strict:
            np.testing.assert_array_equal(rhs, g[f"c{k}_rhs"], err_msg=f"case {k}")
            assert dt == dt_ref and linf == linf_ref, k
            np.testing.assert_array_equal(s.cons, g[f"c{k}_step"], err_msg=f"case {k}")
        else:
            assert rel_linf(rhs, g[f"c{k}_rhs"]) < TOL, k
            assert rel_linf(s.cons, g[f"c{k}_step"]) < TOL, k
        s.close()


@pytest.mark.parametrize("im,fm", [(2, 0), (11, 1), (8, 1), (22, 0)])
def test_trad6_random_quadrants_vs_reference(ref, im, fm):
    """Ten RK3 steps with odd sizes and short segments (chunk and segment
    boundaries inside the five-face carry-over)."""
    rng = np.random.default_rng(im * 10 + fm)
    nx, ny = 37, 29
    c = quadrant_state((nx, ny), rng)
    r = ref.RefSolver(2, [nx, ny], [0, 1, 0, 1, 0, 0], inter_method=im, flux_method=fm, n_case=2, diff_method=1)
    r.cons = c
    want = r.rhs()
    for seg in ((0, 0, 0), (8, 8, 0), (5, 7, 0)):
        s = trad6_solver(2, [nx, ny], [0, 1, 0, 1, 0, 0], im, fm, True, 2, seg_len=seg)
        s.set_cons(c)
        np.testing.assert_array_equal(s.rhsSolve(), want, err_msg=str(seg))
        s.close()
    s = trad6_solver(2, [nx, ny], [0, 1, 0, 1, 0, 0], im, fm, True, 2)
    s.set_cons(c)
    for _ in range(10):
        dt = r.max_dt()
        assert s.getTimeIntervalExplicit() == dt
        r.solve(dt)
        s.solve(dt)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_trad6_sod_device_loop(ref):
    """1D Sod (the reference's nCase 0 state) through the device-resident loop."""
    r = ref.RefSolver(1, [200], [-0.5, 0.5, 0, 0, 0, 0], inter_method=11, flux_method=0, n_case=0, diff_method=1)
    s = trad6_solver(1, [200], [-0.5, 0.5, 0, 0, 0, 0], im=11, fm=0)
    s.set_cons(r.cons)
    rd, rl = r.run(1, 0.05)
    s.info.endStep = 1
    s.info.outputDt = 0.05
    dts, lin = s.run_device()
    np.testing.assert_array_equal(dts, rd)
    np.testing.assert_array_equal(lin, rl)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_trad6_rti_dirichlet_rows(ref):
    """RTI (nCase 3): five Dirichlet ghost rows and the gravity source."""
    n, zone_ = [16, 64], [0, 0.25, 0, 1, 0, 0]
    r = ref.RefSolver(2, n, zone_, inter_method=2, flux_method=1, n_case=3, source_type=1, diff_method=1)
    info = make_info(2, n, zone_, im=2, fm=1, strict=True, ncase=3)
    info.diffMethod = zone.DiffMethod.TRAD6
    info.sourceType = zone.SourceType.GRAVITY
    s = zone.BlockSolver(info)
    s.set_cons(r.cons)
    np.testing.assert_array_equal(s.rhsSolve(), r.rhs())
    for _ in range(4):
        dt = r.max_dt()
        r.solve(dt)
        s.solve(dt)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_trad6_double_mach(ref):
    """Double Mach reflection: the moving DoubleMachUp ghosts at k = 0..4. With
    TRAD6 (no node-flux dissipation) the reference's first RK3 step of this
    case already produces NaNs; the GPU step reports the same as
    CFD_ERR_NONFINITE."""
    n, zone_ = [64, 16], [0, 4, 0, 1, 0, 0]
    r = ref.RefSolver(2, n, zone_, inter_method=11, flux_method=0, n_case=4, diff_method=1)
    s = trad6_solver(2, n, zone_, im=11, fm=0, ncase=4)
    s.set_cons(r.cons)
    for t in (0.05, 0.0):
        r.t = t
        s.info.t = t
        np.testing.assert_array_equal(s.rhsSolve(), r.rhs())
    dt = r.max_dt()
    assert s.getTimeIntervalExplicit() == dt
    r.solve(dt)
    assert not np.isfinite(r.cons).all()
    with pytest.raises(_lib.CfdError) as e:
        s.solve(dt)
    assert e.value.code == -3  # CFD_ERR_NONFINITE


@pytest.mark.parametrize("im,fm", [(2, 0), (11, 1)])
def test_trad6_3d_against_c_oracle(im, fm):
    from oracle.refsolver import ORC_OUTLET, ORC_SYMMETRY, ORC_WRAP, OracleC
    rng = np.random.default_rng(im + 3)
    n = (11, 9, 13)
    c = smooth_state_3d(n, rng)
    zone_ = [0, 1.1, 0, 1, 0, 1]
    bcs = ([[ORC_WRAP] * 2] * 3, [[ORC_OUTLET, ORC_SYMMETRY], [ORC_SYMMETRY, ORC_OUTLET], [ORC_SYMMETRY] * 2])
    gpu_bc = (None, [[zone.BndType.SUPERSONICOUTLET, zone.BndType.SYMMETRYX],
                     [zone.BndType.SYMMETRYY, zone.BndType.SUPERSONICOUTLET], [zone.BndType.SYMMETRYZ] * 2])
    for bo, bg in zip(bcs, gpu_bc):
        s = trad6_solver(3, list(n), zone_, im, fm, True, periodic=bg is None, bc=bg)
        o = OracleC(3, list(n), s.info.geth(0), im, fm, bc=bo, trad6=True)
        o.cons = c
        s.set_cons(c)
        np.testing.assert_array_equal(s.rhsSolve(), o.rhs())
        dt = o.max_dt(0.5)
        assert s.getTimeIntervalExplicit() == dt
        assert s.solve(dt) == o.solve(dt)
        np.testing.assert_array_equal(s.cons, o.cons)
        s.close()


def test_trad6_conserves_on_a_periodic_grid():
    """Telescoping faces: the TRAD6 RHS of a periodic grid sums to zero."""
    rng = np.random.default_rng(1)
    s = trad6_solver(2, [64, 48], [0, 1, 0, 1, 0, 0], im=11, fm=1, strict=False, periodic=True)
    s.set_cons(quadrant_state((64, 48), rng))
    r = s.rhsSolve()
    assert np.abs(r.sum(0)).max() <= 1e-10 * np.abs(r).sum(0).max()


def test_trad6_unsupported_combinations():
    info = make_info(2, [16, 16], im=2, fm=1)
    info.diffMethod = zone.DiffMethod.TRAD6
    info.precision = 1
    with pytest.raises(_lib.CfdError):
        zone.BlockSolver(info)  # mixed form: MND6 only
    info.precision = 0
    cfg = zone.make_config(info)
    cfg.n_ghost = 4  # TRAD6 needs Info::nGhostCell() == 5
    lib = _lib.load()
    import ctypes as C
    h = C.c_void_p()
    assert lib.cfd_create(C.byref(cfg), C.byref(h)) == -6
    with pytest.raises(_lib.CfdError):
        zone.BlockBatch([info, info])  # the batched kernel is MND6 only
    s = zone.BlockSolver(info, periodic=True)
    ptr, cnt = C.c_void_p(), C.c_longlong()
    assert lib.cfd_enable_halo(s.h, 0, C.byref(ptr), C.byref(cnt)) == -6  # halos carry 4 rows
