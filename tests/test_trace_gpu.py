"""The per-scene block trace (steel_trace / steel_trace_read): every prepare and solve block of a
traced frame leaves its start, end and SM; turning the trace on changes no result bit; scene groups
(parallel launch sequences) record into the same per-scene slots."""
import numpy as np
import pytest

from steel_webgpu_b200 import pack
from steel_webgpu_b200._lib import SteelError
from steel_webgpu_b200.sim import Batch
from tests import scenes

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def _check_records(rec, n):
    p, s = rec["prepare"], rec["solve"]
    assert p.shape == (n, 3) and s.shape == (n, 3)
    for r in (p, s):
        assert (r[:, 0] > 0).all() and (r[:, 1] >= r[:, 0]).all()
        assert (r[:, 2] >= 0).all() and (r[:, 2] < 1024).all()
    # One stream: the last prepare launch ends before the last solve launch starts.
    assert p[:, 1].max() <= s[:, 0].min()


def test_trace_records_every_block_and_changes_no_result(steel):
    pks = [pack(sc) for sc in scenes.small_batch(seed=5, n=6)]
    plain = Batch(pks)
    plain.step(3)
    ref = [plain.poses(i) for i in range(len(pks))]
    plain.close()
    b = Batch(pks)
    with pytest.raises(SteelError):
        b.trace_read()  # off by default
    b.trace(True)
    b.step(3)
    for i in range(len(pks)):
        assert np.array_equal(_bits(b.poses(i)), _bits(ref[i]))
    _check_records(b.trace_read(), len(pks))
    b.trace(False)
    b.step(1)
    b.close()


def test_trace_with_scene_groups(steel):
    pks = [pack(sc) for sc in scenes.small_batch(seed=9, n=8)] * 20  # 160 scenes > 148 SMs
    plain = Batch(pks)
    plain.step(2)
    ref = [plain.poses(i) for i in (0, 7, 80, 159)]
    plain.close()
    b = Batch(pks)
    b.set_tiles(64, 0, 0, 2)
    b.trace(True)
    b.step(2)
    for k, i in enumerate((0, 7, 80, 159)):
        assert np.array_equal(_bits(b.poses(i)), _bits(ref[k]))
    rec = b.trace_read()
    assert (rec["prepare"][:, 0] > 0).all() and (rec["solve"][:, 1] >= rec["solve"][:, 0]).all()
    b.close()
