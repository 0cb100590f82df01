"""The TENO-A/AS research variants on the GPU against the reference.

Variants whose decision uses only + - * / floor min max match the reference
bit for bit (pointwise and in strict-flavour runs). Variants that call pow()
round it as CUDA's libdevice does, within a few ulps of the host libm; a
decision can then differ only where a measure sits on its cut-off, so those
are held to a small fraction of differing pointwise values and to L1
closeness of whole runs."""
import numpy as np
import pytest

from cfd_inwsl_b200 import _lib
from tests.test_research_host import RESEARCH, stencils
from tests.util import gpu_solver, quadrant_state

pytestmark = pytest.mark.gpu
NO_POW = {18, 30, 31, 32, 33, 34, 36, 38, 39}


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


@pytest.mark.parametrize("method", sorted(m for m in RESEARCH if m != 1010))
def test_research_pointwise(ref, method):
    q = stencils()
    got = _lib.eval_inter5(method, q)
    want = ref.ref_inter5(method, q)
    if method in NO_POW:
        np.testing.assert_array_equal(got, want)
    else:
        assert np.mean(got != want) < 0.01


@pytest.mark.parametrize("method", [18, 34, 38])
def test_research_runs_bitwise(ref, method):
    rng = np.random.default_rng(method)
    n = 40
    c = quadrant_state(n, rng)
    r = ref.RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=method, flux_method=1, n_case=0)
    r.cons = c
    s = gpu_solver(2, [n, n], im=method, fm=1, strict=True)
    s.set_cons(c)
    for _ in range(6):
        dt = r.max_dt()
        assert s.getTimeIntervalExplicit() == dt
        r.solve(dt)
        s.solve(dt)
    np.testing.assert_array_equal(s.cons, r.cons)


@pytest.mark.parametrize("method", [17, 25, 28])
def test_research_runs_close(ref, method):
    rng = np.random.default_rng(method)
    n = 40
    c = quadrant_state(n, rng)
    r = ref.RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=method, flux_method=0, n_case=0)
    r.cons = c
    s = gpu_solver(2, [n, n], im=method, fm=0, strict=True)
    s.set_cons(c)
    for _ in range(6):
        dt = r.max_dt()
        r.solve(dt)
        s.solve(dt)
    assert np.abs(s.cons - r.cons).mean() / np.abs(r.cons).mean() < 1e-6


def test_congaa_in_1d(ref):
    """Entry 10 (WCNS5CONGZCT7) is Teno5_CongAA in 1D (solverType.cpp:248-250)."""
    from cfd_inwsl_b200 import zone
    r = ref.RefSolver(1, [200], [-0.5, 0.5, 0, 0, 0, 0], inter_method=10, flux_method=0, n_case=0)
    s = gpu_solver(1, [200], [-0.5, 0.5, 0, 0, 0, 0], im=10, fm=0, strict=True)
    s.set_cons(r.cons)
    for _ in range(20):
        dt = r.max_dt()
        r.solve(dt)
        s.solve(dt)
    assert np.abs(s.cons - r.cons).mean() / np.abs(r.cons).mean() < 1e-6
