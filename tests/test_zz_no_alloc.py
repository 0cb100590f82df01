"""The allocation-free RHS entry point against the handle-based one.

cfd_rhs_noalloc serves callers that cannot allocate device memory (code running
inside another framework's memory pool, or a program that reserved the whole
device up front): the caller owns the input and output buffers, and the
library's only scratch is a fixed file-scope device array. Here the caller's
buffers are torch tensors; the result must equal cfd_rhs on the same state
(bit for bit in the strict flavour, 1e-12 relative otherwise), on two calls in a
row with different grids, schemes and boundaries.
"""
import ctypes as C

import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, cases
from tests.util import gpu_solver, rel_linf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def _noalloc_rhs(solver, cons_aos, t=0.0):
    """Runs cfd_rhs_noalloc on torch-owned device buffers with the solver's config."""
    import torch
    nv = solver.nvar
    dev = torch.device("cuda", 0)
    cons = torch.from_numpy(np.ascontiguousarray(cons_aos.T)).to(dev)  # SoA [var][cell]
    rhs = torch.full_like(cons, float("nan"))
    stream = torch.cuda.current_stream(dev)
    rc = solver.lib.cfd_rhs_noalloc(C.byref(solver.cfg), C.c_void_p(cons.data_ptr()), C.c_void_p(rhs.data_ptr()),
                                    float(t), C.c_void_p(stream.cuda_stream))
    assert rc == 0, rc
    torch.cuda.synchronize(dev)
    out = rhs.cpu().numpy().T.copy()
    assert out.shape == (solver.ncell, nv)
    return out


@pytest.mark.parametrize("strict", [True, False])
def test_noalloc_rhs_matches_cfd_rhs_twice(strict):
    rng = np.random.default_rng(2024)
    # call 1: 2D Riemann quadrants, WCNS5 + HLLC, supersonic outlets
    n = 64
    c1 = cases.riemann_quadrants(n, rng)
    s1 = gpu_solver(2, [n, n], im=2, fm=0, strict=strict)
    s1.set_cons(c1)
    want1 = s1.rhsSolve()
    got1 = _noalloc_rhs(s1, c1)
    # call 2: a different grid, TENO5 + Roe, periodic wrap in both directions
    c2, _ = cases.isentropic_vortex(48, L=10.0)
    s2 = gpu_solver(2, [48, 48], [0, 10, 0, 10, 0, 0], im=11, fm=1, strict=strict, periodic=True)
    s2.set_cons(c2)
    want2 = s2.rhsSolve()
    got2 = _noalloc_rhs(s2, c2)
    for got, want in ((got1, want1), (got2, want2)):
        assert np.all(np.isfinite(got))
        if strict:
            np.testing.assert_array_equal(got, want)
        else:
            assert rel_linf(got, want) < 1e-12
    s1.close()
    s2.close()


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = _lib.load()
    cfg = _lib.CfdConfig()
    lib.cfd_config_default(C.byref(cfg))
    cfg.n[0] = cfg.n[1] = 8192  # 2 * (8192 + 8192) line ends > 16384
    cfg.h[0] = cfg.h[1] = 1.0 / 8192
    dummy = C.c_void_p(1)
    assert lib.cfd_rhs_noalloc(C.byref(cfg), dummy, dummy, 0.0, None) == -1


@pytest.mark.parametrize("strict", [True, False])
def test_noalloc_rhs_3d_and_gravity(strict):
    """Two more calls in a row: a 3D grid with mirror and outlet sides (three
    directions of line ends in the one scratch table), then the 2D gravity
    source with mirror walls in x and y."""
    from cfd_inwsl_b200 import zone
    from tests.util import make_info, smooth_state_3d
    rng = np.random.default_rng(77)
    n3 = [16, 12, 10]
    c3 = smooth_state_3d(n3, rng)
    bc3 = [[zone.BndType.SYMMETRYX, zone.BndType.SUPERSONICOUTLET],
           [zone.BndType.SUPERSONICOUTLET, zone.BndType.SYMMETRYY],
           [zone.BndType.SYMMETRYZ, zone.BndType.PERIODIC1D]]
    s3 = gpu_solver(3, n3, im=11, fm=0, strict=strict, bc=bc3)
    s3.set_cons(c3)
    want3 = s3.rhsSolve()
    got3 = _noalloc_rhs(s3, c3)
    info = make_info(2, [40, 24], [0, 1, 0, 0.6, 0, 0], im=2, fm=1, strict=strict)
    info.sourceType = zone.SourceType.GRAVITY
    s2 = zone.BlockSolver(info, bc=[[zone.BndType.SYMMETRYX] * 2, [zone.BndType.SYMMETRYY] * 2, [7, 7]])
    prim = np.column_stack([rng.uniform(0.5, 2, 960), rng.uniform(-1, 1, (960, 2)), rng.uniform(0.5, 2, 960)])
    c2 = zone.prim_to_cons(prim)
    s2.set_cons(c2)
    want2 = s2.rhsSolve()
    got2 = _noalloc_rhs(s2, c2)
    for got, want in ((got3, want3), (got2, want2)):
        assert np.all(np.isfinite(got))
        if strict:
            np.testing.assert_array_equal(got, want)
        else:
            assert rel_linf(got, want) < 1e-12
    s3.close()
    s2.close()
