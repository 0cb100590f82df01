"""Batched mode (scaled down): independent 2D Riemann
problems of uneven grid sizes in one persistent launch per sweep, each with
its own dt and output clipping, against the reference solver case by case."""
import numpy as np
import pytest

from cfd_inwsl_b200 import cases, zone
from tests.util import make_info, rel_linf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def batch_setup(sizes, strict, seed=0):
    rng = np.random.default_rng(seed)
    infos, states = [], []
    for n in sizes:
        info = make_info(2, [n, n], [0, 1, 0, 1, 0, 0], im=2, fm=0, strict=strict, ncase=0, cfl=0.5)
        infos.append(info)
        states.append(cases.riemann_quadrants(n, rng))
    b = zone.BlockBatch(infos)
    for i, c in enumerate(states):
        b.set_cons(i, c)
    return b, states


@pytest.mark.parametrize("strict", [True, False])
def test_batch_matches_reference_case_by_case(ref, strict):
    sizes = [16, 40, 24, 64, 33, 17, 96, 48, 20, 72]
    t_end = [0.02 + 0.01 * (i % 3) for i in range(len(sizes))]
    b, states = batch_setup(sizes, strict)
    t, ns = b.run(t_end)
    for i, n in enumerate(sizes):
        r = ref.RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=2, flux_method=0, n_case=0, cfl=0.5)
        r.cons = states[i]
        dts, _ = r.run(1, t_end[i])
        assert ns[i] == len(dts), (i, ns[i], len(dts))
        assert abs(t[i] - r.t) <= 1e-15
        if strict:
            np.testing.assert_array_equal(b.cons(i), r.cons, err_msg=f"case {i}")
        else:
            assert rel_linf(b.cons(i), r.cons) < 1e-10, i
    b.close()


def test_batch_equals_single_case_path():
    """Every case of a batch equals the single-case path on the same state
    (fast flavour, step limit instead of output clipping)."""
    sizes = [128, 200, 160]
    b, states = batch_setup(sizes, False, seed=3)
    t, ns = b.run(1e9, max_steps=7)
    assert list(ns) == [7, 7, 7]
    for i, n in enumerate(sizes):
        info = make_info(2, [n, n], [0, 1, 0, 1, 0, 0], im=2, fm=0, strict=False, ncase=0, cfl=0.5)
        s = zone.BlockSolver(info)
        s.set_cons(states[i])
        s.info.endStep = 10 ** 6
        s.info.outputDt = 1e9
        s.run_device(max_steps=7)
        # segment boundaries differ (whole lines in the batch), so a face may be
        # formed by a different inlined copy of the same code: FMA rounding only
        assert rel_linf(b.cons(i), s.cons) < 1e-13, i
        s.close()
    b.close()


@pytest.mark.parametrize("strict", [True, False])
def test_every_tiling_gives_the_same_bits(strict):
    """Tile shapes, segments per line and persistent grid sizes only change
    which CTA computes a face: every tiling gives the default's bits."""
    sizes = [40, 64, 33, 130, 17]
    base, _ = batch_setup(sizes, strict, seed=5)
    base.run(1e9, max_steps=5)
    want = [base.cons(i) for i in range(len(sizes))]
    base.close()
    for shape in (0, 1):
        for seg in (1, 2, 3):
            for one in (False, True):
                b, _ = batch_setup(sizes, strict, seed=5)
                for idim in (1, 2):
                    b.set_tiling(idim, shape, seg, one)
                b.run(1e9, max_steps=5)
                for i in range(len(sizes)):
                    np.testing.assert_array_equal(b.cons(i), want[i], err_msg=f"{shape} {seg} {one} case {i}")
                b.close()


def test_autotune_keeps_results(ref):
    """cfd_batch_autotune picks a tiling per direction; the run after it is
    still the reference's, bit for bit (strict flavour)."""
    sizes = [48, 100, 30, 70]
    b, states = batch_setup(sizes, True, seed=9)
    choice = b.autotune()
    assert len(choice) == 2 and all(c["sweep_ms"] > 0 for c in choice)
    t, ns = b.run(0.03)
    for i, n in enumerate(sizes):
        r = ref.RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=2, flux_method=0, n_case=0, cfl=0.5)
        r.cons = states[i]
        dts, _ = r.run(1, 0.03)
        assert ns[i] == len(dts)
        np.testing.assert_array_equal(b.cons(i), r.cons, err_msg=f"case {i}")
    b.close()
