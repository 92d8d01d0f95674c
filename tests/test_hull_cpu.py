"""The C++ quickhull (steel_convex_hull, host only) against the Python builder's convex_hull
(builder.js:61-173): the same vertices, faces (vertex order included) and planes, bit for bit, on
random clouds, the analytic shapes' sample points (coplanar faces merged, symmetric ties),
lattices full of coplanar and collinear points, duplicates and signed zeros; the same errors."""
import math
import time

import numpy as np
import pytest

from steel_webgpu_b200 import synth
from steel_webgpu_b200._lib import SteelError
from steel_webgpu_b200.builder import GT, SceneBuilder, convex_hull, convex_hull_native, shape_points


def _same(points):
    a = convex_hull(points)
    b = convex_hull_native(points)
    assert a == b
    return a


def test_random_clouds(steel):
    rng = np.random.default_rng(11)
    for _ in range(200):
        _same(synth._ellipsoid_points(rng, int(rng.integers(4, 97))))
    for _ in range(50):
        _same(rng.normal(size=(int(rng.integers(4, 200)), 3)).tolist())


def test_analytic_shapes(steel):
    for g in ("BOX", "CYLINDER", "CAPSULE", "SPHERE", "CONE", "ELLIPSOID"):
        if g not in GT or len(shape_points(GT[g], [0.1, 0.2, 0.3])) < 4:
            continue  # types without sample points (their hulls come from elsewhere)
        for size in ([0.1, 0.2, 0.3], [0.05, 0.05, 0.05], [1.0, 0.5, 0.25]):
            h = _same(shape_points(GT[g], size))
            assert len(h["faces"]) >= 4


def test_lattices_duplicates_and_signed_zeros(steel):
    grid = [[x, y, z] for x in (-1.0, 0.0, 1.0) for y in (-1.0, 0.0, 1.0) for z in (-1.0, 0.0, 1.0)]
    h = _same(grid)
    assert len(h["verts"]) == 8 and len(h["faces"]) == 6  # interior and mid-edge points dropped
    _same(grid + grid[::-1])
    _same([[0.0, 0.0, 0.0], [-0.0, 0.0, -0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0], [0.25, 0.25, 0.25]])
    rng = np.random.default_rng(5)
    pts = (rng.integers(-3, 4, size=(300, 3)) * 0.1).tolist()  # many coplanar, collinear and equal points
    _same(pts)


@pytest.mark.parametrize("pts,msg", [
    ([[0, 0, 0], [1, 0, 0], [0, 1, 0]], "at least 4 distinct"),
    ([[0, 0, 0], [1, 1, 1], [2, 2, 2], [3, 3, 3], [1, 1, 1]], "collinear"),
    ([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0.5, 0.2, 0.0]], "coplanar"),
])
def test_errors(pts, msg, steel):
    with pytest.raises(ValueError, match=msg):
        convex_hull(pts)
    with pytest.raises(SteelError, match=msg):
        convex_hull_native(pts)


def test_builder_option_and_speed(steel):
    rng = np.random.default_rng(3)
    clouds = [synth._ellipsoid_points(rng, int(rng.integers(8, 33))) for _ in range(100)]
    t0 = time.perf_counter()
    py = [convex_hull(c) for c in clouds]
    t1 = time.perf_counter()
    nat = [convex_hull_native(c) for c in clouds]
    t2 = time.perf_counter()
    assert py == nat
    assert (t2 - t1) < (t1 - t0)  # the native hull is the faster one (about 10x here)
    a, b = SceneBuilder(), SceneBuilder(native_hulls=True)
    for sb in (a, b):
        body = sb.add_body(mass=1.0)
        sb.add_shape_convex_hull(body, vertices=clouds[0])
        sb.add_shape(body, GT["CAPSULE"], [0.03, 0.1, 0.0])
    assert [s["hull"] for s in a.shapes] == [s["hull"] for s in b.shapes]
    assert math.isfinite(b.shapes[0]["hull"]["faces"][0]["d"])
