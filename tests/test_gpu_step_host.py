"""cfd_step_host (one CFL step from a host state to a host state, the copies
overlapped with the sweeps) against cfd_upload_cons + cfd_run (one step) +
cfd_download_cons. Both run the same kernels on the same data, the first in
chunks along the last dimension, so states, dt and t agree bit for bit: grids
whose chunks end ragged, 2D and 3D, strict, fast and mixed, the gravity source
(nCase 3), the time-dependent DoubleMachUp boundary (nCase 4), outlets, a
last chunk shorter than a segment's ghost cells, an in-place buffer, and a
grid small enough to take the unchunked path."""
import ctypes as C

import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, cases, zone
from tests.util import gpu_solver, make_info, smooth_state_3d

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def host_step(s, cons, cfl, t, out=None):
    a = np.ascontiguousarray(cons, dtype=np.float64)
    o = np.empty_like(a) if out is None else out
    tt, dt = C.c_double(t), C.c_double(0.0)
    _lib.check(s.lib.cfd_step_host(s.h, cfl, 1e300, _lib.ptr(a), _lib.ptr(o), C.byref(tt), C.byref(dt)), s.h)
    return o, tt.value, dt.value


def plain_step(s, cons, cfl, t):
    s.set_cons(cons)
    tt, ns, dts = C.c_double(t), C.c_int(0), np.zeros(1)
    _lib.check(s.lib.cfd_run(s.h, cfl, 1, 1e300, 1, C.byref(tt), C.byref(ns), _lib.ptr(dts), None), s.h)
    assert ns.value == 1
    return s.cons, tt.value, dts[0]


def compare(make, cons, cfl, steps=3, t0=0.0, in_place=False):
    a, b = make(), make()
    ua, ub, ta, tb = cons.copy(), cons.copy(), t0, t0
    for _ in range(steps):
        if in_place:
            _, ta, da = host_step(a, ua, cfl, ta, out=ua)
        else:
            ua, ta, da = host_step(a, ua, cfl, ta)
        ub, tb, db = plain_step(b, ub, cfl, tb)
        assert da == db and ta == tb
        np.testing.assert_array_equal(ua.view(np.uint64), ub.view(np.uint64))
    a.close()
    b.close()


def smooth_2d(nx, ny, rng):
    """A smooth periodic state with a seeded amplitude."""
    x = (np.arange(nx) + 0.5) / nx
    y = (np.arange(ny) + 0.5) / ny
    X, Y = np.meshgrid(x, y)
    a = rng.uniform(0.1, 0.3)
    rho = 1 + a * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    u = 0.5 + 0.1 * np.cos(2 * np.pi * Y)
    v = -0.3 + 0.1 * np.sin(2 * np.pi * X)
    p = 1 + 0.1 * np.cos(2 * np.pi * (X + Y))
    return zone.prim_to_cons(np.stack([rho, u, v, p], -1).reshape(-1, 4))


@pytest.mark.parametrize("flavour", ["strict", "fast", "mixed"])
def test_teno_roe_2d(flavour):
    nx, ny = 130, 200  # 7 upload chunks of 32 rows (the last of 8), 9 segments of 24 rows
    c = smooth_2d(nx, ny, np.random.default_rng(5))
    make = lambda: gpu_solver(2, [nx, ny], [0, 10, 0, 10, 0, 0], im=11, fm=1, periodic=True, cfl=0.4,
                              strict=flavour == "strict", precision=1 if flavour == "mixed" else 0,
                              seg_len=(0, 24, 0))
    compare(make, c, 0.4)


def test_short_last_chunk_and_outlets():
    """194 rows: the last upload chunk holds 2 rows, fewer than a segment's
    ghost cells, so stage 1's last sweep waits for the whole upload (periodic
    wrap); then the same grid with outlets from the configuration, whose
    ghosts come from the line's own cells."""
    nx, ny = 100, 194
    c = smooth_2d(nx, ny, np.random.default_rng(11))
    for periodic in (True, False):
        make = lambda: gpu_solver(2, [nx, ny], im=11, fm=1, periodic=periodic, cfl=0.4, strict=True,
                                  seg_len=(0, 16, 0))
        compare(make, c, 0.4)


def test_default_segments_2d_in_place():
    n = 256
    c, _ = cases.isentropic_vortex(n)
    make = lambda: gpu_solver(2, [n, n], [0, 10, 0, 10, 0, 0], im=11, fm=1, periodic=True, cfl=0.4, strict=True)
    compare(make, c, 0.4, in_place=True)


@pytest.mark.parametrize("strict", [True, False])
def test_3d(strict):
    n = (40, 36, 70)  # 3 upload chunks of planes, 5 segments of 16
    c = smooth_state_3d(n, np.random.default_rng(3))
    make = lambda: gpu_solver(3, list(n), im=2, fm=0, periodic=True, strict=strict, seg_len=(0, 0, 16))
    compare(make, c, 0.5, steps=2)


def test_small_grid_takes_the_plain_path():
    rng = np.random.default_rng(9)
    c = smooth_2d(40, 40, rng)
    make = lambda: gpu_solver(2, [40, 40], im=2, fm=1, periodic=True, strict=True)
    compare(make, c, 0.5)


def test_gravity_source_rti(ref):
    n, zone_ = [32, 128], [0, 0.25, 0, 1, 0, 0]
    r = ref.RefSolver(2, n, zone_, inter_method=2, flux_method=1, n_case=3, cfl=0.5, source_type=1)
    c = r.cons
    r.close()

    def make():
        info = make_info(2, n, zone_, im=2, fm=1, strict=True, ncase=3, cfl=0.5, seg_len=(0, 16, 0))
        info.sourceType = zone.SourceType.GRAVITY
        return zone.BlockSolver(info)

    compare(make, c, 0.5)


def test_double_mach_time_dependent_boundary(ref):
    n, zone_ = [256, 64], [0, 4, 0, 1, 0, 0]
    r = ref.RefSolver(2, n, zone_, inter_method=2, flux_method=0, n_case=4, cfl=0.5)
    c = r.cons
    r.close()
    make = lambda: zone.BlockSolver(make_info(2, n, zone_, im=2, fm=0, strict=True, ncase=4, cfl=0.5,
                                              seg_len=(0, 8, 0)))
    compare(make, c, 0.5, steps=3, t0=0.01)


def test_slab_handle_is_refused():
    """A handle with slab halos needs an exchange between stages, which the
    host step does not do: refused before any work, the state untouched."""
    rng = np.random.default_rng(2)
    c = smooth_2d(64, 96, rng)
    s = gpu_solver(2, [64, 96], im=2, fm=1, periodic=True, strict=True)
    s.set_cons(c)
    buf, cnt = C.c_void_p(), C.c_longlong(0)
    _lib.check(s.lib.cfd_enable_halo(s.h, 0, C.byref(buf), C.byref(cnt)), s.h)
    out = np.zeros_like(c)
    tt, dt = C.c_double(0.0), C.c_double(0.0)
    rc = s.lib.cfd_step_host(s.h, 0.5, 1e300, _lib.ptr(c), _lib.ptr(out), C.byref(tt), C.byref(dt))
    assert rc == -6 and tt.value == 0.0
    assert not out.any()
    s.close()


@pytest.mark.parametrize("periodic", [True, False])
def test_trad6_five_ghosts(periodic):
    """The TRAD6 difference reads five cells beyond a segment's ends; the
    host step's early stage-1 sweep waits for them (periodic wrap and
    outlets)."""
    nx, ny = 96, 160
    c = smooth_2d(nx, ny, np.random.default_rng(21))

    def make():
        info = make_info(2, [nx, ny], im=2, fm=0, strict=True, cfl=0.5, seg_len=(0, 16, 0))
        info.diffMethod = zone.DiffMethod.TRAD6
        return zone.BlockSolver(info, periodic=periodic)

    compare(make, c, 0.5)
