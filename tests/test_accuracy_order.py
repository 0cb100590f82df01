"""Order of accuracy of the face interpolation + MND6 difference against the
reference's AccuracyTest (CongFD1.0/AccuracyTest.cpp, committed orders in
CongFD1.0/order.txt: L1 order 4.94-4.98 for h = 0.2 ... 0.04)."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

from tests import accuracy

GOLD = Path(__file__).resolve().parent / "golden"


def oracle_derivative(q, h):
    """MND6 of TCNS5 face values, restated with the oracle's interpolator
    (differ.cpp:54-103, w = 3/2, -3/10, 1/30)."""
    from oracle.refsolver import ORC_FAMILY, orc_load
    lib = orc_load()
    fam, c = ORC_FAMILY[11]
    n = q.size - 8
    gq = lambda k: q[k + 4]  # noqa: E731
    face = lambda k: lib.orc_inter5(fam, c, C.c_void_p(np.ascontiguousarray(  # noqa: E731
        [gq(k - 2), gq(k - 1), gq(k), gq(k + 1), gq(k + 2)]).ctypes.data))
    w0, w1, w2 = 3.0 / 2.0, -3.0 / 10.0, 1.0 / 30.0
    out = np.empty(n)
    for i in range(n):
        out[i] = (w1 * (gq(i + 1) - gq(i - 1)) + w0 * (face(i) - face(i - 1)) + w2 * (face(i + 1) - face(i - 2))) / h
    return out


def reference_orders():
    rows = json.loads((GOLD / "order_congfd.json").read_text())["rows"]
    return np.array([r[1] for r in rows[:5]])


def test_oracle_reproduces_reference_order():
    try:
        from oracle.refsolver import orc_load
        orc_load()
    except RuntimeError as e:
        pytest.skip(str(e))
    hs = accuracy.HS
    l1 = [accuracy.errors(oracle_derivative, h)[0] for h in hs]
    ords = accuracy.orders(l1, hs)[:5]
    assert np.all(np.abs(np.array(ords) - reference_orders()) < 0.1), ords
    assert all(4.8 < o < 5.2 for o in ords)


@pytest.mark.gpu
def test_gpu_order_and_bitwise_derivative():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")
    from cfd_inwsl_b200 import _lib
    dev = lambda q, h: _lib.accuracy_derivative(11, q, h)  # noqa: E731
    hs = accuracy.HS
    for h in hs:
        n, q, _ = accuracy.samples(h)
        np.testing.assert_array_equal(dev(q, h), oracle_derivative(q, h))
    l1 = [accuracy.errors(dev, h)[0] for h in hs]
    ords = accuracy.orders(l1, hs)[:5]
    assert np.all(np.abs(np.array(ords) - reference_orders()) < 0.1), ords
