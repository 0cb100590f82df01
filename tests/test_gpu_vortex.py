"""Isentropic vortex refinement study (the benchmark configuration): periodic
[0,10]^2, freestream (1,1,1,1), strength 5, TENO5 (TCNS5) + Roe, SSP-RK3, CFL
0.4, t = 2.

  * the strict flavour (the benchmark's timed flavour) equals the reference
    CPU solver bit for bit over the whole run, 64^2 to 512^2 (1024^2 with
    CFD_LONG_TESTS=1: about ten minutes of reference CPU time);
  * its L1 density error against the exact translated vortex falls at fourth
    to fifth order to 512^2 and reaches the periodic box's floor (about 1e-10,
    the infinite-plane vortex's tail at the edge) at 1024^2 and 2048^2;
  * the fast flavour (FMA contraction) differs from it because ulp-level
    differences flip TENO cut-off decisions; the deviation is reported and
    bounded far below the discretisation error;
  * the mixed form stays within 2x of the FP64 error on every grid.
"""
import os

import numpy as np
import pytest

from cfd_inwsl_b200 import cases
from tests.util import gpu_solver, rel_linf

pytestmark = pytest.mark.gpu
T_END = 2.0


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def run_gpu(n, precision=0, strict=True):
    c, _ = cases.isentropic_vortex(n)
    s = gpu_solver(2, [n, n], [0, 10, 0, 10, 0, 0], im=11, fm=1, periodic=True, cfl=0.4, precision=precision,
                   strict=strict and precision == 0)
    s.set_cons(c)
    s.info.endStep = 1
    s.info.outputDt = T_END
    dts, _ = s.run_device()
    out = s.cons
    s.close()
    return out, len(dts)


def run_ref(ref, n):
    c, _ = cases.isentropic_vortex(n)
    r = ref.RefSolver(2, [n, n], [0, 10, 0, 10, 0, 0], inter_method=11, flux_method=1, n_case=0, cfl=0.4,
                      periodic=True)
    r.cons = c
    dts, _ = r.run(1, T_END)
    out = r.cons
    r.close()
    return out, len(dts)


def l1_rho(cons, n):
    exact, _ = cases.isentropic_vortex(n, t=T_END)
    return np.abs(cons[:, 0] - exact[:, 0]).mean()


@pytest.fixture(scope="module")
def study():
    res = {}
    for n in (64, 128, 256, 512):
        cs, steps = run_gpu(n)
        cf, _ = run_gpu(n, strict=False)
        cmx, _ = run_gpu(n, precision=1)
        res[n] = {"strict": cs, "fast": cf, "steps": steps, "l1": l1_rho(cs, n), "l1_fast": l1_rho(cf, n),
                  "l1_mixed": l1_rho(cmx, n)}
    return res


def test_convergence_order(study):
    ns = sorted(study)
    e = [study[n]["l1"] for n in ns]
    orders = [np.log(e[i] / e[i + 1]) / np.log(2) for i in range(len(e) - 1)]
    print("vortex L1(rho), strict FP64:", dict(zip(ns, e)), "orders:", orders)
    assert all(o > 4.0 for o in orders), orders


def test_refinement_at_1024_and_2048(study):
    """1024^2 and 2048^2 (the benchmark grid) against the exact vortex. The
    translated vortex is the solution on the infinite plane; on the periodic
    box its tail (about 5e-6 in velocity at the box edge) makes it exact only
    to about 1e-10 in L1, the floor the scheme reaches from 1024^2 on
    (measured: 7.2e-10 at 512^2, 1.2e-10 at 1024^2, 2.9e-10 at 2048^2).
    Both stay below the 512^2 error and at that floor."""
    e = {512: study[512]["l1"]}
    for n in (1024, 2048):
        c, _ = run_gpu(n)
        e[n] = l1_rho(c, n)
    print("vortex L1(rho), strict FP64:", e)
    assert e[1024] < e[512] and e[2048] < e[512], e
    assert e[1024] < 5e-10 and e[2048] < 5e-10, e


@pytest.mark.parametrize("n", [64, 128, 256, 512])
def test_strict_flavour_is_the_reference_over_whole_runs(ref, study, n):
    """The timed flavour to t = 2: the reference solver's step count and state,
    bit for bit."""
    want, steps = run_ref(ref, n)
    assert steps == study[n]["steps"]
    np.testing.assert_array_equal(study[n]["strict"], want)


@pytest.mark.skipif(os.environ.get("CFD_LONG_TESTS") != "1", reason="about ten minutes of reference CPU time")
def test_strict_flavour_is_the_reference_at_1024(ref):
    got, steps = run_gpu(1024)
    want, steps_ref = run_ref(ref, 1024)
    assert steps == steps_ref
    np.testing.assert_array_equal(got, want)


def test_fast_flavour_deviation(study):
    """FMA contraction moves values by ulps; where a TENO stencil's measure
    sits at the cut-off that flips the selection, and in this under-resolved
    vortex the differences then grow over the run (measured rel L-inf against
    the reference: 6e-6 at 64^2, 4e-9 at 128^2, below 1e-11 at 256^2 and
    512^2). Bounded here at 1e-5 relative, two orders below the L1
    discretisation error of the coarsest grid."""
    for n in sorted(study):
        dev = rel_linf(study[n]["fast"], study[n]["strict"])
        print(f"n={n}: fast vs strict rel L-inf {dev:.3e}; L1 strict {study[n]['l1']:.3e} fast "
              f"{study[n]['l1_fast']:.3e}")
        assert dev < 1e-5, (n, dev)
        assert abs(study[n]["l1_fast"] - study[n]["l1"]) < 1e-2 * study[n]["l1"], n


def test_mixed_within_2x_of_fp64(study):
    for n in sorted(study):
        e64, emx = study[n]["l1"], study[n]["l1_mixed"]
        print(f"n={n}: L1 fp64 {e64:.3e} mixed {emx:.3e} ratio {emx / e64:.3f}")
        assert emx <= 2.0 * e64, (n, e64, emx)
