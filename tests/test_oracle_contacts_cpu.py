"""Known geometric answers for the oracle's narrowphase (CPU): contact points, normals and signed
distances of shape pairs whose contact is analytic.

A contact record holds the point halfway between the two surfaces, the signed distance phi
(negative in penetration) and the unit normal from the lower-indexed body to the higher (the
ground, body -1, first), as the reference's emit writes them (wgsl.js:269-307). Sphere pairs
(the primitive routines of narrow_pair), faces resting on the plane (plane contacts), a
face-to-face box pair (the SAT manifold clipped to the overlap rectangle), crossed box edges (the
SAT edge query) and a capsule on the plane (segment against plane) are checked against their
closed forms; boxes apart by more than the speculative margin make no contact.
"""
import math

import numpy as np

from steel_webgpu_b200 import SceneBuilder, pack


def _contacts(oracle_lib, scene):
    pk = pack(scene)
    o = oracle_lib.OracleSim(pk)
    o.collide()
    n = int(o.read("collide_counts", np.uint32)[1])
    rec = o.read("contacts")[:n * 20].reshape(n, 5, 4).astype(np.float64)
    # (point, phi, normal, body a, body b), in a fixed order for comparison
    out = [(tuple(r[0, :3]), r[0, 3], tuple(r[1, :3]), int(r[2, 0]), int(r[2, 1])) for r in rec]
    return sorted(out, key=lambda c: (round(c[0][0], 6), round(c[0][1], 6), round(c[0][2], 6)))


def _check(got, expected, tol=1e-6):
    assert len(got) == len(expected)
    expected = sorted(expected, key=lambda c: (round(c[0][0], 6), round(c[0][1], 6), round(c[0][2], 6)))
    for (p, phi, n, a, b), (pe, phie, ne, ae, be) in zip(got, expected):
        np.testing.assert_allclose(p, pe, atol=tol)
        assert abs(phi - phie) < tol
        np.testing.assert_allclose(n, ne, atol=tol)
        assert (a, b) == (ae, be)


def test_sphere_pair(oracle_lib):
    b = SceneBuilder(fps=240, gravity=(0.0, 0.0, 0.0))
    s = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1])
    b.add_shape_sphere(s, radius=0.1)
    t = b.add_body(xform=[0.12, 0.16, 1.0, 0, 0, 0, 1])
    b.add_shape_sphere(t, radius=0.15)
    # centres 0.2 apart along (0.6, 0.8): phi = 0.2 - 0.25; halfway between the surface points
    # 0.1 and 0.05 along the normal
    _check(_contacts(oracle_lib, b.finalize()), [((0.045, 0.06, 1.0), -0.05, (0.6, 0.8, 0.0), 0, 1)])


def test_sphere_on_plane(oracle_lib):
    b = SceneBuilder(fps=240)
    b.add_ground_plane()
    s = b.add_body(xform=[0.3, 0.2, 0.08, 0, 0, 0, 1])
    b.add_shape_sphere(s, radius=0.1)
    _check(_contacts(oracle_lib, b.finalize()), [((0.3, 0.2, -0.01), -0.02, (0.0, 0.0, 1.0), -1, 0)])


def test_turned_box_on_plane(oracle_lib):
    b = SceneBuilder(fps=240, box_hulls="direct")
    b.add_ground_plane()
    turn = math.pi / 4
    s = b.add_body(xform=[0.1, 0.0, 0.09, 0.0, 0.0, math.sin(turn / 2), math.cos(turn / 2)])
    b.add_shape_box(s, hx=0.2, hy=0.15, hz=0.1)
    c, sn = math.cos(turn), math.sin(turn)
    corners = [(0.1 + x * c - y * sn, x * sn + y * c, -0.005) for x in (-0.2, 0.2) for y in (-0.15, 0.15)]
    _check(_contacts(oracle_lib, b.finalize()), [(p, -0.01, (0.0, 0.0, 1.0), -1, 0) for p in corners], tol=2e-6)


def test_stacked_boxes_clip_to_the_overlap(oracle_lib):
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    s = b.add_body(xform=[0.0, 0.0, 1.0, 0, 0, 0, 1])
    b.add_shape_box(s, hx=0.2, hy=0.2, hz=0.1)
    t = b.add_body(xform=[0.1, 0.05, 1.19, 0, 0, 0, 1])
    b.add_shape_box(t, hx=0.15, hy=0.1, hz=0.1)
    # faces 0.01 into each other at z = 1.1 / 1.09; the overlap of [-0.2, 0.2]^2 and
    # [-0.05, 0.25] x [-0.05, 0.15]
    corners = [(x, y, 1.095) for x in (-0.05, 0.2) for y in (-0.05, 0.15)]
    _check(_contacts(oracle_lib, b.finalize()), [(p, -0.01, (0.0, 0.0, 1.0), 0, 1) for p in corners])


def test_crossed_box_edges(oracle_lib):
    """Two long boxes turned 45 degrees about x and about y: their edges cross, one contact on the
    normal x cross y (the SAT edge-edge case)."""
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    h, c = math.sin(math.pi / 8), math.cos(math.pi / 8)
    s = b.add_body(xform=[0.0, 0.0, 1.0, h, 0.0, 0.0, c])
    b.add_shape_box(s, hx=0.5, hy=0.1, hz=0.1)
    t = b.add_body(xform=[0.0, 0.0, 1.27, 0.0, h, 0.0, c])
    b.add_shape_box(t, hx=0.1, hy=0.5, hz=0.1)
    ridge = 0.1 * math.sqrt(2.0)  # each edge's height from its box centre
    _check(_contacts(oracle_lib, b.finalize()), [((0.0, 0.0, 1.135), 0.27 - 2.0 * ridge, (0.0, 0.0, 1.0), 0, 1)])


def test_capsule_lying_on_plane(oracle_lib):
    b = SceneBuilder(fps=240)
    b.add_ground_plane()
    s = b.add_body(xform=[0.0, 0.0, 0.045, 0.0, math.sin(math.pi / 4), 0.0, math.cos(math.pi / 4)])
    b.add_shape_capsule(s, radius=0.05, half_height=0.2)
    ends = [(x, 0.0, -0.0025) for x in (-0.2, 0.2)]
    _check(_contacts(oracle_lib, b.finalize()), [(p, -0.005, (0.0, 0.0, 1.0), -1, 0) for p in ends])


def test_separated_boxes_make_no_contact(oracle_lib):
    b = SceneBuilder(fps=240, box_hulls="direct", gravity=(0.0, 0.0, 0.0))
    for x in (0.0, 0.5):
        s = b.add_body(xform=[x, 0.0, 1.0, 0, 0, 0, 1])
        b.add_shape_box(s, hx=0.1, hy=0.1, hz=0.1)
    assert _contacts(oracle_lib, b.finalize()) == []


def test_sorted_contacts_are_a_permutation_in_key_order(oracle_lib):
    """The canonical sort (wgsl.js:3899-3982) on a pile of hulls, boxes and capsules: the sorted
    records are the raw records permuted, in nondecreasing (body pair, feature) order."""
    from tests import scenes
    pk = pack(scenes.hull_bin())
    o = oracle_lib.OracleSim(pk)
    o.step(40)
    o.collide()
    n = int(o.read("collide_counts", np.uint32)[1])
    assert n > 100
    raw = o.read("craw")[:n * 20].reshape(n, 20)
    srt = o.read("contacts")[:n * 20].reshape(n, 20)
    as_rows = lambda a: sorted(map(bytes, a.view(np.uint32)))  # noqa: E731
    assert as_rows(raw) == as_rows(srt)
    m = srt.reshape(n, 5, 4)[:, 2, :].astype(np.int64)
    pair = (m[:, 0] + 1) | ((m[:, 1] + 1) << 16)
    feat = m[:, 2] | (m[:, 3] << 16)
    key = pair * (1 << 32) + feat
    assert np.all(np.diff(key) >= 0)


def test_colors_are_first_fit_in_row_order(oracle_lib):
    """The row coloring (first_free_color and its serial pass, wgsl.js:1233-1267) restated over the
    oracle's rows of a pile: every row takes the lowest color that no earlier row on either of its
    bodies holds (the overflow color when all are taken), so no color holds two rows of a body."""
    from tests import scenes
    pk = pack(scenes.hull_bin())
    C = pk.C
    o = oracle_lib.OracleSim(pk)
    o.step(40)
    sch = o.read("sched", np.uint32).astype(np.int64)
    nu = int(sch[C["S_META"]])
    total = int(sch[C["S_USTART"] + nu])
    ncol = C["NCOL"]
    assert total > 100
    used: dict = {}
    colors = set()
    for r in range(total):
        key = int(sch[C["S_UKEY"] + sch[C["S_RUNIT"] + r]])
        bodies = [x for x in ((key & 0xFFFF) - 1, (key >> 16) - 1) if x >= 0]
        taken = set().union(*(used.get(x, set()) for x in bodies))
        expected = next((k for k in range(ncol) if k not in taken), ncol)
        assert int(sch[C["S_PCOL"] + r]) == expected, f"row {r}"
        if expected < ncol:
            for x in bodies:
                used.setdefault(x, set()).add(expected)
        colors.add(expected)
    assert len(colors) > 3


def test_sort_is_independent_of_the_raw_order(oracle_lib):
    """The canonical order does not depend on the order the narrowphase emitted the contacts in
    (wgsl.js:3895-3898; the CUDA narrowphase emits them in a different order, by atomics): the raw
    records of a pile, reversed and shuffled, sort to the same records bit for bit."""
    from tests import scenes
    pk = pack(scenes.hull_bin())
    maxc = pk.C["MAXC"]
    o = oracle_lib.OracleSim(pk)
    o.step(40)
    o.collide()
    n = int(o.read("collide_counts", np.uint32)[1])
    assert n > 100
    raw = o.read("craw").reshape(-1, 4)
    rec, smu = raw[:n * 5].reshape(n, 5, 4).copy(), raw[maxc * 5:maxc * 5 + n].copy()
    want = o.read("contacts").view(np.uint32).copy()
    for perm in (np.arange(n)[::-1], np.random.default_rng(9).permutation(n)):
        o.write("craw", 0, rec[perm].reshape(-1))
        o.write("craw", maxc * 5 * 4, smu[perm].reshape(-1))
        o.sort_raw(n)
        got = o.read("contacts").view(np.uint32)
        assert np.array_equal(got[:n * 20], want[:n * 20])
        assert np.array_equal(got[maxc * 20:maxc * 20 + n * 4], want[maxc * 20:maxc * 20 + n * 4])
