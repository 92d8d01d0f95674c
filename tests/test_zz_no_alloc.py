"""steel_sort_contacts_noalloc, the contact sort that allocates no device memory, against the
batch path's sort (steel_collide + steel_read_contacts).

The sorted records of two scenes are shuffled on the host, uploaded to caller-owned device
buffers and sorted again by the no-alloc entry point, twice in a row on the same static scratch
(the larger scene first, so stale keys of the first call would show in the second). Contact
order is integer work: the outputs must match the batch path's bit for bit.
"""
import ctypes

import numpy as np
import pytest

from steel_webgpu_b200 import _lib, pack
from steel_webgpu_b200.sim import Batch
from tests import scenes

pytestmark = pytest.mark.gpu


def _flat(rec, smu):
    """steel_read_contacts layout: n records of 5 vec4, then n shape-mu vec4."""
    return np.concatenate([rec.reshape(-1), smu.reshape(-1)]).astype(np.float32)


def _shuffled(rec, smu, rng):
    perm = rng.permutation(rec.shape[0])
    return _flat(rec[perm], smu[perm])


def _sort_noalloc(flat, n, torch):
    L = _lib.load()
    raw = torch.from_numpy(flat).to("cuda:0")
    out = torch.full_like(raw, float("nan"))
    torch.cuda.synchronize()
    rc = L.steel_sort_contacts_noalloc(ctypes.c_void_p(raw.data_ptr()), n, ctypes.c_void_p(out.data_ptr()), None)
    _lib.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_sort_matches_batch_sort_twice(steel):
    import torch
    torch.cuda.init()
    torch.cuda.set_device(0)
    pks = [pack(scenes.hull_bin()), pack(scenes.boxes())]
    g = Batch(pks)
    g.step(40)
    g.collide()
    refs = [g.contacts(0), g.contacts(1)]
    counts = [r[0].shape[0] for r in refs]
    assert min(counts) > 0 and counts[0] != counts[1], counts
    rng = np.random.default_rng(2024)
    for scene in sorted((0, 1), key=lambda s: -counts[s]):
        rec, smu = refs[scene]
        n = rec.shape[0]
        # Keys (pair, feature, point bits) are distinct, so the order is independent of the raw order.
        m = rec[:, 2, :].astype(np.int64)
        bits = rec[:, 0, :].view(np.uint32)
        assert len({(tuple(a), tuple(b)) for a, b in zip(m, bits)}) == n
        got = _sort_noalloc(_shuffled(rec, smu, rng), n, torch)
        assert np.array_equal(got.view(np.uint32), _flat(rec, smu).view(np.uint32)), f"scene {scene} order differs"
    g.close()


def test_noalloc_sort_rejects_oversize(steel):
    L = _lib.load()
    limit = 65536
    rc = L.steel_sort_contacts_noalloc(None, limit + 1, None, None)
    assert rc == 3
    assert b"65536" in L.steel_last_error()
