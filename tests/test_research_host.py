"""The TENO-A/AS research variants of the interpolator selector on the CPU.

The device code's research_flag (cfd_inwsl_b200/csrc/euler_math.cuh) is
compiled for the host (tests/inter5_host.cu) and evaluated with the host libm,
against the reference's own interpolators (interScheme.hpp, compiled from its
sources into oracle/_ref/libcongfd_ref.so): bit for bit on random, scaled and
adversarial stencils, every variant. On the GPU the pow() calls of some
variants round differently (tests/test_gpu_parity.py)."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]

# InterMethod -> ResearchVariant (the map of cfd_inwsl_b200/csrc/api.cu); 1010 = 1D WCNS5CONGZCT7
RESEARCH = {17: 0, 18: 1, 19: 2, 20: 3, 21: 4, 24: 5, 25: 6, 26: 7, 27: 8, 28: 9, 29: 10, 30: 11, 31: 12, 32: 13,
            33: 14, 34: 15, 36: 16, 38: 17, 39: 18, 1010: 19}


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    out = tmp_path_factory.mktemp("inter5") / "libinter5h.so"
    subprocess.run([nvcc, "-O2", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC", "-shared",
                    "-I", str(ROOT / "cfd_inwsl_b200" / "csrc"), str(ROOT / "tests" / "inter5_host.cu"),
                    "-o", str(out)], check=True, capture_output=True)
    return C.CDLL(str(out))


def stencils():
    rng = np.random.default_rng(12)
    q = rng.normal(size=(3000, 5)) * rng.choice([1e-4, 1e-2, 1, 1e2], size=(3000, 1))
    smooth = np.cumsum(rng.normal(size=(500, 5)) * 1e-3, 1) + rng.normal(size=(500, 1))
    steps = np.where(rng.random((500, 5)) < 0.3, 1.0, 0.0).cumsum(1) * rng.normal(size=(500, 1))
    adv = np.array([[1, 1, 1, 1, 1], [0, 0, 0, 0, 0], [0, 0, 1, 1, 1], [1, 1, 1, 0, 0], [1, 0, 1, 0, 1],
                    [1, 2, 3, 4, 5], [1, 1, 2, 2, 2], [3, 3, 3, 3, 3.0000001]], float)
    return np.ascontiguousarray(np.concatenate([q, smooth, steps, adv]))


@pytest.mark.parametrize("method", sorted(RESEARCH))
def test_research_variant_bitwise_on_host(ref, host, method):
    q = stencils()
    out = np.empty(len(q))
    host.h_research_inter5(RESEARCH[method], q.ctypes.data_as(C.c_void_p), len(q), out.ctypes.data_as(C.c_void_p))
    want = ref.ref_inter5(method, q)
    np.testing.assert_array_equal(out, want)
