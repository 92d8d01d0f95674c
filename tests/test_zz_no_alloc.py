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


def _mix32(x):
    x = x.astype(np.uint64)
    m = np.uint64(0xFFFFFFFF)
    x ^= x >> np.uint64(16)
    x = (x * np.uint64(0x7FEB352D)) & m
    x ^= x >> np.uint64(15)
    x = (x * np.uint64(0x846CA68B)) & m
    x ^= x >> np.uint64(16)
    return x


def _expected_order(rec):
    """The canonical order restated on the host: (pair, feature, point-bit hash, raw index), the key
    of wgsl.js:3906-3918."""
    m = rec[:, 2, :]
    pair = ((m[:, 0].astype(np.int64) + 1) | ((m[:, 1].astype(np.int64) + 1) << 16)) & 0xFFFFFFFF
    feat = (m[:, 2].astype(np.int64) | (m[:, 3].astype(np.int64) << 16)) & 0xFFFFFFFF
    p = rec[:, 0, :].view(np.uint32).astype(np.uint64)
    bits = _mix32(_mix32(_mix32(p[:, 0]) ^ p[:, 1]) ^ p[:, 2]) ^ p[:, 3]
    idx = np.arange(rec.shape[0])
    return np.lexsort((idx, bits, feat, pair))


def _synthetic_records(n, rng):
    """n raw records with few distinct (pair, feature) keys, so the point-bit hash decides most of
    the order, and groups of records that share the whole key (position and shape words) but differ
    elsewhere, so the raw index decides between them."""
    rec = rng.uniform(-1, 1, (n, 5, 4)).astype(np.float32)
    rec[:, 2, 0] = rng.integers(0, 300, n)
    rec[:, 2, 1] = rec[:, 2, 0] + rng.integers(1, 4, n)
    rec[:, 2, 2] = rng.integers(0, 3, n)
    rec[:, 2, 3] = rng.integers(0, 2, n)
    dup = rng.choice(n, n // 8, replace=False)
    src = rng.choice(n, n // 8)
    rec[dup, 0, :] = rec[src, 0, :]
    rec[dup, 2, :] = rec[src, 2, :]
    smu = rng.uniform(0, 1, (n, 4)).astype(np.float32)
    return rec, smu


def test_noalloc_sort_sizes_in_a_row(steel):
    """Synthetic raw records at the maximum size, then smaller sizes that are not powers of two
    (the shared-memory path at 1025, the static array above it), one call after another on one
    stream over the same static array: each output equals the host's lexicographic order."""
    import torch
    torch.cuda.init()
    torch.cuda.set_device(0)
    rng = np.random.default_rng(7)
    for n in (65536, 40001, 1025, 2049, 65536):
        rec, smu = _synthetic_records(n, rng)
        order = _expected_order(rec)
        got = _sort_noalloc(_flat(rec, smu), n, torch)
        assert np.array_equal(got.view(np.uint32), _flat(rec[order], smu[order]).view(np.uint32)), f"n={n}"


def test_noalloc_sort_rejects_oversize(steel):
    L = _lib.load()
    limit = 65536
    rc = L.steel_sort_contacts_noalloc(None, limit + 1, None, None)
    assert rc == 3
    assert b"65536" in L.steel_last_error()


def test_noalloc_sort_rejects_bad_buffers(steel):
    """Misaligned, overlapping and host-only buffers are refused before anything is launched."""
    import torch
    L = _lib.load()
    buf = torch.zeros(24 * 64 + 8, dtype=torch.float32, device="cuda:0")
    p = buf.data_ptr()
    assert L.steel_sort_contacts_noalloc(ctypes.c_void_p(p + 4), 32, ctypes.c_void_p(p + 24 * 4 * 32 + 64), None) == 1
    assert b"aligned" in L.steel_last_error()
    assert L.steel_sort_contacts_noalloc(ctypes.c_void_p(p), 32, ctypes.c_void_p(p + 16 * 8), None) == 1
    assert b"overlap" in L.steel_last_error()
    host = np.zeros(24 * 32, dtype=np.float32)
    assert L.steel_sort_contacts_noalloc(ctypes.c_void_p(host.ctypes.data), 32, ctypes.c_void_p(p), None) == 1
    torch.cuda.synchronize()
