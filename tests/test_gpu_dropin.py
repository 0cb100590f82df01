"""The drop-in itself: the reference's own BlockSolver, patched as
INTEGRATION.md describes (RK3_SSP and getTimeIntervalExplicit call the GPU
library through include/cfdgpu.h) and compiled with the unmodified reference
sources into oracle/_ref/libcongfd_dropin.so (oracle/Makefile, target
dropin). Its own driver, BlockSolver::stepsLoopCFL (blockSolver.cpp:170-235),
runs the named cases of the reference's Initializer; the final state must equal
the unpatched reference solver's, bit for bit (the patch sets the strict
flavour).

The run goes to a child process: the patched and the unpatched reference
libraries define the same C++ symbols, and stepsLoopCFL writes its log file
into the working directory (a temporary one here)."""
import ctypes as C
import multiprocessing as mp
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
DROPIN = ROOT / "oracle" / "_ref" / "libcongfd_dropin.so"


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    if not DROPIN.exists():
        pytest.skip("drop-in build absent (make -C oracle dropin, where the reference checkout is present)")


def _dropin_child(args):
    import os
    dim, n, zone_, im, fm, ncase, cfl, src, t_end, workdir = args
    os.chdir(workdir)
    lib = C.CDLL(str(DROPIN))
    lib.dropin_run.restype = C.c_int
    lib.dropin_run.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int,
                               C.c_double, C.c_void_p, C.POINTER(C.c_longlong)]
    n3 = (C.c_int * 3)(*(list(n) + [1] * (3 - len(n))))
    z = (C.c_double * 6)(*zone_)
    ncell = int(np.prod(n))
    out = np.empty((ncell, dim + 2))
    steps = C.c_longlong(0)
    rc = lib.dropin_run(dim, C.cast(n3, C.c_void_p), C.cast(z, C.c_void_p), im, fm, ncase, cfl, src, t_end,
                        out.ctypes.data, C.byref(steps))
    return rc, out, steps.value


def run_dropin(tmp_path, *args):
    ctx = mp.get_context("spawn")
    with ctx.Pool(1) as pool:
        return pool.apply(_dropin_child, (args + (str(tmp_path),),))


@pytest.mark.parametrize("case", ["sod", "riemann2d", "doublemach", "rti"])
def test_patched_reference_driver_matches_reference(ref, tmp_path, case):
    # (dim, cells, calZone, InterMethod, FluxMethod, nCase, CFL, SourceType, t_end)
    cfgs = {
        "sod": (1, [400], [-0.5, 0.5, 0, 0, 0, 0], 2, 0, 0, 0.5, 0, 0.2),              # Initializer nCase 0, 1D
        "riemann2d": (2, [64, 64], [0, 1, 0, 1, 0, 0], 11, 1, 0, 0.5, 0, 0.05),        # nCase 0, 2D, TENO5 + Roe
        "doublemach": (2, [96, 24], [0, 4, 0, 1, 0, 0], 2, 0, 4, 0.5, 0, 0.02),        # nCase 4: per-line wiring
        "rti": (2, [16, 64], [0, 0.25, 0, 1, 0, 0], 2, 0, 3, 0.5, 1, 0.05),           # nCase 3 with gravity
    }
    dim, n, zone_, im, fm, ncase, cfl, src, t_end = cfgs[case]
    rc, got, steps = run_dropin(tmp_path, dim, n, zone_, im, fm, ncase, cfl, src, t_end)
    assert rc == 0
    r = ref.RefSolver(dim, n, zone_, inter_method=im, flux_method=fm, n_case=ncase, cfl=cfl, source_type=src)
    dts, _ = r.run(1, t_end)
    assert steps == len(dts)
    np.testing.assert_array_equal(got, r.cons)
    r.close()
