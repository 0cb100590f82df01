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


# ----------------------------------------------------------------- the batched configuration at its own scale
def _ref_case_digest(args):
    """Reference solver (one OpenMP thread) on one case of the batched
    configuration; returns (case, steps, t, sha256 of the final cons bytes)."""
    import hashlib

    from cfd_inwsl_b200 import cases as cs
    from oracle.refsolver import RefSolver
    i, n, P, t_end, max_steps = args
    r = RefSolver(2, [n, n], [0, 1, 0, 1, 0, 0], inter_method=2, flux_method=0, n_case=0, cfl=0.5, threads=1)
    r.cons = cs.quadrant_state(P, n)
    dts, _ = r.run(1, t_end, max_steps=max_steps)
    out = (i, len(dts), r.t, hashlib.sha256(np.ascontiguousarray(r.cons).tobytes()).hexdigest())
    r.close()
    return out


def _digest(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _run_reference_cases(jobs):
    """Reference runs in a spawn pool (one single-threaded solver per core),
    largest first."""
    import multiprocessing as mp
    import os
    jobs = sorted(jobs, key=lambda j: -j[1])
    ctx = mp.get_context("spawn")
    with ctx.Pool(max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        return {r[0]: r[1:] for r in pool.imap_unordered(_ref_case_digest, jobs)}


def _same_run(got, want):
    """Same step count and state bits; the end times within 1e-15 (as the
    case-by-case test above compares them)."""
    return got[0] == want[0] and abs(got[1] - want[1]) <= 1e-15 and got[2] == want[2]


def _batch_of(sizes, prims, strict):
    infos = [make_info(2, [n, n], [0, 1, 0, 1, 0, 0], im=2, fm=0, strict=strict, ncase=0, cfl=0.5) for n in sizes]
    b = zone.BlockBatch(infos)
    for i, (n, P) in enumerate(zip(sizes, prims)):
        b.set_cons(i, cases.quadrant_state(P, n))
    return b


def test_batched_configuration_first_10_steps_every_case(ref):
    """All 256 cases of the batched configuration (N = round(2^U(7,10)),
    seeded quadrant states, WCNS5 + HLLC, CFL 0.5, per-case dt) advanced 10
    steps together in the strict flavour: every case equals the reference
    solver's 10 steps bit for bit (step count, time and state)."""
    sizes, prims = cases.riemann_batch(256, seed=0)
    b = _batch_of(sizes, prims, strict=True)
    t, ns = b.run(0.25, end_step=1, max_steps=10)
    got = {i: (int(ns[i]), float(t[i]), _digest(b.cons(i))) for i in range(len(sizes))}
    b.close()
    want = _run_reference_cases([(i, n, prims[i], 0.25, 10) for i, n in enumerate(sizes)])
    bad = [i for i in range(len(sizes)) if not _same_run(got[i], want[i])]
    assert not bad, [(i, sizes[i], got[i][:2], want[i][:2]) for i in bad[:5]]


def test_batched_configuration_smallest_16_to_the_end(ref):
    """The 16 smallest cases of the batched configuration run to t = 0.25 in
    one batch (strict flavour), each equal to the reference solver's whole run."""
    sizes, prims = cases.riemann_batch(256, seed=0)
    idx = sorted(range(len(sizes)), key=lambda i: sizes[i])[:16]
    b = _batch_of([sizes[i] for i in idx], [prims[i] for i in idx], strict=True)
    t, ns = b.run(0.25)
    got = {k: (int(ns[k]), float(t[k]), _digest(b.cons(k))) for k in range(len(idx))}
    b.close()
    want = _run_reference_cases([(k, sizes[i], prims[i], 0.25, 1 << 20) for k, i in enumerate(idx)])
    for k in range(len(idx)):
        assert _same_run(got[k], want[k]), (k, sizes[idx[k]], got[k][:2], want[k][:2])
