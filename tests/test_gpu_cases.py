"""The reference's named 2D cases that add a source term or time-dependent
boundaries, on the GPU against the reference itself:

  nCase 3  Rayleigh-Taylor instability (initializer.cpp:396-420 state,
           initializer.cpp:796-861 SYMMETRYX / Dirichlet wiring) with the
           gravity source (sourceTerm.cpp:3-20), Info::sourceType = GRAVITY
  nCase 4  double Mach reflection (initializer.cpp:436-462 state,
           Initializer::initDoubleMachBnds initializer.cpp:880-943: Dirichlet
           inflow, outlet, Dirichlet / SYMMETRYY floor split at x = 1/6 and the
           time-dependent DoubleMachUp top, oneDBnd.cpp)

The initial states come from the reference's own Initializer; the strict
flavour must match bit for bit (RHS, CFL dt, RK3 steps and the device loop),
the fast flavour within 1e-12 relative L-inf after one step.
"""
import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, zone
from tests.util import make_info, rel_linf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


RTI = dict(n=[16, 64], zone_=[0, 0.25, 0, 1, 0, 0], ncase=3)
DMR = dict(n=[64, 16], zone_=[0, 4, 0, 1, 0, 0], ncase=4)


def _pair(ref, case, im, fm, strict, gravity):
    r = ref.RefSolver(2, case["n"], case["zone_"], inter_method=im, flux_method=fm, n_case=case["ncase"],
                      cfl=0.5, source_type=1 if gravity else 0)
    info = make_info(2, case["n"], case["zone_"], im=im, fm=fm, strict=strict, ncase=case["ncase"], cfl=0.5)
    if gravity:
        info.sourceType = zone.SourceType.GRAVITY
    s = zone.BlockSolver(info)
    s.set_cons(r.cons)
    return r, s


@pytest.mark.parametrize("im,fm", [(2, 1), (11, 0), (8, 1)])
def test_rti_gravity_bitwise(ref, im, fm):
    r, s = _pair(ref, RTI, im, fm, True, True)
    np.testing.assert_array_equal(s.rhsSolve(), r.rhs())
    for _ in range(5):
        dt = r.max_dt()
        assert s.getTimeIntervalExplicit() == dt
        r.solve(dt)
        s.solve(dt)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_rti_gravity_changes_the_rhs(ref):
    """The source is really applied: rhs(rho v) differs from the source-free
    RHS by exactly -rho (up to the rounding of one subtraction)."""
    r, s = _pair(ref, RTI, 2, 1, True, True)
    r0, s0 = _pair(ref, RTI, 2, 1, True, False)
    g, f = s.rhsSolve(), s0.rhsSolve()
    rho = r.cons[:, 0]
    np.testing.assert_allclose(f[:, 2] - g[:, 2], rho, rtol=1e-12, atol=1e-12)
    np.testing.assert_array_equal(g[:, :2], f[:, :2])
    np.testing.assert_array_equal(f, r0.rhs())


def test_rti_device_loop_bitwise(ref):
    r, s = _pair(ref, RTI, 2, 1, True, True)
    rd, rl = r.run(2, 0.02)
    s.info.endStep = 2
    s.info.outputDt = 0.02
    dts, lin = s.run_device()
    np.testing.assert_array_equal(dts, rd)
    np.testing.assert_array_equal(lin, rl)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_rti_fast_flavour(ref):
    r, s = _pair(ref, RTI, 2, 1, False, True)
    dt = r.max_dt()
    r.solve(dt)
    s.solve(dt)
    assert rel_linf(s.cons, r.cons) < 1e-12


@pytest.mark.parametrize("im,fm", [(2, 0), (11, 1), (35, 0)])
def test_double_mach_bitwise(ref, im, fm):
    r, s = _pair(ref, DMR, im, fm, True, False)
    np.testing.assert_array_equal(s.rhsSolve(), r.rhs())
    # the top boundary moves with the shock: compare at a later time too
    r.t = 0.05
    s.info.t = 0.05
    np.testing.assert_array_equal(s.rhsSolve(), r.rhs())
    r.t = 0.0
    s.info.t = 0.0
    for _ in range(6):
        dt = r.max_dt()
        assert s.getTimeIntervalExplicit() == dt
        r.solve(dt)
        s.solve(dt)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_double_mach_device_loop_bitwise(ref):
    r, s = _pair(ref, DMR, 11, 0, True, False)
    rd, rl = r.run(1, 0.02)
    s.info.endStep = 1
    s.info.outputDt = 0.02
    dts, lin = s.run_device()
    assert len(dts) > 10
    np.testing.assert_array_equal(dts, rd)
    np.testing.assert_array_equal(lin, rl)
    np.testing.assert_array_equal(s.cons, r.cons)


def test_gravity_in_batch_matches_single_case(ref):
    """Batched mode applies each case's source: RTI cases of two sizes."""
    infos, singles = [], []
    for n in ([16, 64], [12, 48]):
        case = dict(RTI, n=n)
        r, s = _pair(ref, case, 2, 1, True, True)
        singles.append((r, s))
        info = make_info(2, n, RTI["zone_"], im=2, fm=1, strict=True, ncase=3, cfl=0.5)
        info.sourceType = zone.SourceType.GRAVITY
        infos.append(info)
    b = zone.BlockBatch(infos)  # wires each case's RTI Dirichlet ends, as BlockSolver does
    for i, (r, _) in enumerate(singles):
        b.set_cons(i, r.cons)
    b.run(0.01, end_step=1)
    for i, (r, _) in enumerate(singles):
        r.run(1, 0.01)
        np.testing.assert_array_equal(b.cons(i), r.cons)


def test_noalloc_gravity_matches_handle():
    """cfd_rhs_noalloc honours source_type like the handle path (outlet walls)."""
    import ctypes as C
    import torch
    info = make_info(2, [40, 24], [0, 1, 0, 0.6, 0, 0], im=2, fm=0, strict=True, ncase=0)
    info.sourceType = zone.SourceType.GRAVITY
    s = zone.BlockSolver(info)
    rng = np.random.default_rng(3)
    prim = np.column_stack([rng.uniform(0.5, 2, 960), rng.uniform(-1, 1, (960, 2)), rng.uniform(0.5, 2, 960)])
    cons = zone.prim_to_cons(prim)
    s.set_cons(cons)
    want = s.rhsSolve()
    cfg = zone.make_config(info)
    lib = _lib.load()
    u = torch.tensor(cons.T.copy(), device="cuda")
    out = torch.empty_like(u)
    torch.cuda.synchronize()
    rc = lib.cfd_rhs_noalloc(C.byref(cfg), C.c_void_p(u.data_ptr()), C.c_void_p(out.data_ptr()), 0.0, None)
    assert rc == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().T, want)
