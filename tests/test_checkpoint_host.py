"""Checkpoint file format on CPU: the host writer and reader of
cfd_inwsl_b200.zone (the layout cfd_save_checkpoint / cfd_load_checkpoint use)."""
import numpy as np
import pytest

from cfd_inwsl_b200 import zone
from tests.util import make_info


def test_round_trip(tmp_path):
    info = make_info(2, [12, 9], im=11, fm=1)
    info.t, info.step = 0.125, 7
    cons = np.random.default_rng(0).normal(size=(108, 4))
    p = tmp_path / "a.ckpt"
    zone.write_checkpoint(p, info, cons)
    meta, got = zone.read_checkpoint(p)
    np.testing.assert_array_equal(got, cons)
    assert meta["t"] == 0.125 and meta["step"] == 7 and list(meta["n"]) == [12, 9, 1] and meta["nvar"] == 4
    assert meta["inter_method"] == 11 and meta["flux_method"] == 1
    assert p.stat().st_size == 104 + 8 * 108 * 4 + 8


def test_corruption_and_truncation_detected(tmp_path):
    info = make_info(1, [20])
    cons = np.random.default_rng(1).normal(size=(20, 3))
    p = tmp_path / "b.ckpt"
    zone.write_checkpoint(p, info, cons)
    raw = bytearray(p.read_bytes())
    raw[200] ^= 1
    q = tmp_path / "c.ckpt"
    q.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        zone.read_checkpoint(q)
    q.write_bytes(p.read_bytes()[:-9])
    with pytest.raises(ValueError):
        zone.read_checkpoint(q)
    raw = bytearray(p.read_bytes())
    raw[0:8] = b"NOTACKPT"
    q.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="version-1"):
        zone.read_checkpoint(q)
