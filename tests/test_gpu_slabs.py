"""Slab decomposition (cfd_inwsl_b200.slabs) on one GPU: every slab in one
process, halos by device copies, against the undivided grid. The strict
flavour must match bit for bit (every ghost is an exact copy of the
neighbouring slab's cell); the fast flavour within 1e-13 relative."""
import ctypes as C

import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, slabs, zone
from tests.util import make_info, quadrant_state, rel_linf, smooth_state_3d

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def run_both(info, cons, parts, steps, bc=None, periodic=False):
    whole = zone.BlockSolver(info, bc=bc, periodic=periodic)
    whole.set_cons(cons)
    grid = slabs.SlabGrid(info, parts, bc=bc, periodic=periodic)
    grid.set_cons(cons)
    np.testing.assert_array_equal(grid.cons, cons)
    for _ in range(steps):
        dt = whole.getTimeIntervalExplicit()
        assert grid.max_dt(info.CFL) == dt
        whole.RK3_SSP(dt)
        grid.step(dt)
    return whole.cons, grid.cons


@pytest.mark.parametrize("parts", [2, 3])
def test_periodic_2d_slabs_bitwise(parts):
    rng = np.random.default_rng(parts)
    nx, ny = 48, 36
    info = make_info(2, [nx, ny], [0, 1, 0, 0.75, 0, 0], im=11, fm=1, strict=True)
    from cfd_inwsl_b200.cases import isentropic_vortex
    c = isentropic_vortex(nx, L=1.0)[0][: nx * ny]  # a smooth periodic-in-x field, cut in y
    c = c + 0.0 * rng.normal(size=c.shape)
    w, g = run_both(info, c, parts, 4, periodic=True)
    np.testing.assert_array_equal(g, w)


def test_outlet_2d_uneven_slabs_bitwise():
    rng = np.random.default_rng(5)
    nx, ny = 40, 50  # 50 rows over 4 slabs: 13, 13, 12, 12
    info = make_info(2, [nx, ny], [0, 1, 0, 1.25, 0, 0], im=2, fm=0, strict=True)
    c = quadrant_state((nx, ny), rng)
    bc = [[zone.BndType.SUPERSONICOUTLET] * 2, [zone.BndType.SUPERSONICOUTLET] * 2,
          [zone.BndType.SUPERSONICOUTLET] * 2]
    w, g = run_both(info, c, 4, 5, bc=bc)
    np.testing.assert_array_equal(g, w)


def test_3d_periodic_slabs_bitwise():
    rng = np.random.default_rng(9)
    n = [20, 16, 24]
    info = make_info(3, n, [0, 1, 0, 0.8, 0, 1.2], im=2, fm=0, strict=True)
    c = smooth_state_3d(n, rng)
    w, g = run_both(info, c, 2, 3, periodic=True)
    np.testing.assert_array_equal(g, w)


def test_fast_flavour_slabs():
    rng = np.random.default_rng(2)
    nx, ny = 64, 60
    info = make_info(2, [nx, ny], [0, 1, 0, 60 / 64, 0, 0], im=11, fm=1, strict=False)
    c = quadrant_state((nx, ny), rng)
    w, g = run_both(info, c, 3, 4, periodic=True)
    assert rel_linf(g, w) < 1e-13


def test_slab_rank_one_process_matches_whole_grid():
    """SlabRank (the multi-GPU path of bench.py) as one NCCL rank: one periodic
    slab, its halo exchange a copy of its own rows and dt from the all-reduced
    wave speeds read back on the slab's stream. Bit for bit against the
    undivided grid, dt included, on a grid large enough that a read-back
    racing the reduction would see stale values."""
    import socket
    import torch.distributed as dist
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        n = 512
        info = make_info(2, [n, n], [0, 10, 0, 10, 0, 0], im=11, fm=1, strict=True, cfl=0.4)
        from cfd_inwsl_b200.cases import isentropic_vortex
        c = isentropic_vortex(n)[0]
        whole = zone.BlockSolver(info, periodic=True)
        whole.set_cons(c)
        rank = slabs.SlabRank(info, periodic=True)
        rank.set_cons(c)
        for _ in range(5):
            dt = whole.getTimeIntervalExplicit()
            assert rank.max_dt(info.CFL) == dt
            whole.RK3_SSP(dt)
            rank.step(dt)
        np.testing.assert_array_equal(rank.slab.solver.cons, whole.cons)
        # the device-controlled form (dt reduced and kept on the device)
        # against the undivided grid's device loop
        tw, nw = C.c_double(0.0), C.c_int(0)
        _lib.check(whole.lib.cfd_run(whole.h, info.CFL, 1, 1e300, 6, C.byref(tw), C.byref(nw), None, None), whole.h)
        tr, nr = rank.run_device(6, info.CFL)
        assert nr == nw.value == 6 and tr == tw.value
        np.testing.assert_array_equal(rank.slab.solver.cons, whole.cons)
    finally:
        dist.destroy_process_group()
