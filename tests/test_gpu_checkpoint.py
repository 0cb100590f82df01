"""Checkpoint / restart through the C ABI (cfd_save_checkpoint,
cfd_load_checkpoint): the file the library writes is the documented format,
a restarted run continues bit for bit, and damaged files are refused."""
import numpy as np
import pytest

from cfd_inwsl_b200 import _lib, zone
from tests.util import gpu_solver, quadrant_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from tests.conftest import gpu_available
    if not gpu_available():
        pytest.skip("no CUDA device")


def test_restart_continues_bitwise(tmp_path):
    rng = np.random.default_rng(4)
    n = 40
    c = quadrant_state(n, rng)
    a = gpu_solver(2, [n, n], im=11, fm=1, strict=True)
    a.set_cons(c)
    for _ in range(10):
        a.solve(a.getTimeIntervalExplicit())
    b = gpu_solver(2, [n, n], im=11, fm=1, strict=True)
    b.set_cons(c)
    for _ in range(5):
        b.solve(b.getTimeIntervalExplicit())
    b.info.step = 5
    p = tmp_path / "mid.ckpt"
    b.save_checkpoint(p)
    meta, cons = zone.read_checkpoint(p)
    np.testing.assert_array_equal(cons, b.cons)
    assert meta["t"] == b.info.t and meta["step"] == 5
    r = gpu_solver(2, [n, n], im=11, fm=1, strict=True)
    r.load_checkpoint(p)
    assert r.info.t == b.info.t and r.info.step == 5
    for _ in range(5):
        r.solve(r.getTimeIntervalExplicit())
    np.testing.assert_array_equal(r.cons, a.cons)
    assert r.info.t == a.info.t


def test_host_written_file_loads(tmp_path):
    info = gpu_solver(1, [64]).info
    cons = zone.sod_1d(info)
    info.t, info.step = 0.5, 3
    p = tmp_path / "host.ckpt"
    zone.write_checkpoint(p, info, cons)
    s = gpu_solver(1, [64])
    s.load_checkpoint(p)
    np.testing.assert_array_equal(s.cons, cons)
    assert s.info.t == 0.5 and s.info.step == 3


def test_damaged_or_mismatched_files_refused(tmp_path):
    s = gpu_solver(2, [16, 16])
    s.set_cons(quadrant_state(16, np.random.default_rng(0)))
    p = tmp_path / "x.ckpt"
    s.save_checkpoint(p)
    raw = bytearray(p.read_bytes())
    raw[150] ^= 4
    q = tmp_path / "bad.ckpt"
    q.write_bytes(bytes(raw))
    with pytest.raises(_lib.CfdError) as e:
        s.load_checkpoint(q)
    assert e.value.code == -1 and "checksum" in str(e.value)
    other = gpu_solver(2, [16, 12])
    with pytest.raises(_lib.CfdError) as e:
        other.load_checkpoint(p)
    assert "shape" in str(e.value)
