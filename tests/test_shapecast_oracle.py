"""The oracle's intersectsSphere (MeshBVH.js:796-809, sphereIntersectTriangle
src/math/MathUtilities.js:167-201) and intersectsBox (MeshBVH.js:780-792, OrientedBox.js:78-260),
pinned by the reference's known answers (test/ShapeCasts.test.js:565-604, :606-696) and by
brute-force equivalences: the BVH answer must equal "some triangle of the mesh is within r of the
centre" / "some triangle passes the oriented box's separating-axis test", triangle by triangle."""
import math

import numpy as np

from obb_util import brute_force, compose, quaternion_xyz, random_boxes, record


def test_intersects_sphere_known_answers(pkg, orc):
    geo = pkg.sphere(1, 50, 50)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=0)
    spheres = np.array([[0, 1, 0, 0.01],      # touching the surface at the pole
                        [0, 0, 0, 0.9],       # inside the mesh, not reaching it
                        [0, 2.01, 0, 0.9]],   # outside
                       dtype=np.float32)
    assert list(o.intersects_sphere(spheres)) == [True, False, False]


def test_intersects_sphere_equals_brute_force(pkg, orc):
    geo = pkg.torus_knot(10, 3, 60, 12)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=2)
    idx = np.empty(geo.index.size, dtype=np.uint32)
    orc.lib().orc_copy_index(o.h, idx.ctypes.data)
    tri = geo.position[idx.astype(np.int64).reshape(-1, 3)].astype(np.float64)
    rng = np.random.default_rng(5)
    lo, hi = geo.position.min(0) - 3, geo.position.max(0) + 3
    c = lo + rng.random((400, 3)) * (hi - lo)
    r = rng.uniform(0.05, 3.0, 400)
    spheres = np.concatenate([c, r[:, None]], 1).astype(np.float32)
    got = o.intersects_sphere(spheres)
    for i in range(spheres.shape[0]):
        p = spheres[i, :3].astype(np.float64)
        rad = float(spheres[i, 3])
        d = min(orc.point_triangle_distance(p, *t) for t in tri)
        if abs(d - rad) <= 1e-9 * max(rad, 1.0):
            continue                                  # on the boundary: either answer
        assert got[i] == (d <= rad), (i, d, rad)
    assert 0 < got.sum() < spheres.shape[0]


def test_intersects_box_known_answers(pkg, orc):
    """test/ShapeCasts.test.js:606-696: a 50 x 50 unit sphere, boxes rotated by Euler (pi/4, pi/4, 0)."""
    geo = pkg.sphere(1, 50, 50)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=0)
    q = quaternion_xyz(math.pi / 4, math.pi / 4, 0)
    cases = [((-1, -1, -1), (1, 1, 1), (0, 3, 0), False),       # outside
             ((-1, -1, -1), (1, 1, 1), (0, 2, 0), True),        # one corner inside
             ((-10, -10, -10), (10, 10, 10), (0, 0, 0), True),  # encloses the mesh
             ((-.5, -.5, -.5), (.5, .5, .5), (0, 0, 0), False),  # inside the mesh, not touching it
             ((-10, 0, -10), (10, 10, 10), (0, 0, 0), True)]    # cuts it with one side
    boxes = np.stack([record(mn, mx, compose(pos, q)) for mn, mx, pos, _ in cases])
    assert list(o.intersects_box(boxes)) == [c[3] for c in cases]


def test_intersects_box_equals_brute_force(pkg, orc):
    geo = pkg.torus_knot(10, 3, 60, 12)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=2)
    idx = np.empty(geo.index.size, dtype=np.uint32)
    orc.lib().orc_copy_index(o.h, idx.ctypes.data)
    tri = geo.position[idx.astype(np.int64).reshape(-1, 3)].astype(np.float64)
    rng = np.random.default_rng(11)
    boxes = np.concatenate([random_boxes(rng, 150, np.zeros(3), 14.0),
                            random_boxes(rng, 50, np.zeros(3), 14.0, shear=True)])
    got = o.intersects_box(boxes)
    checked = 0
    for i in range(boxes.shape[0]):
        meets, gap = brute_force(tri, boxes[i])
        if gap.min() < 1e-9:
            continue                                  # some triangle touches the box: either answer
        assert got[i] == meets.any(), i
        checked += 1
    assert checked > 150 and 0 < got.sum() < boxes.shape[0]


def test_sphere_triangles_equal_brute_force(pkg, orc):
    """Triangles within a sphere through shapecast's CONTAINED path (shapecast.js:111-117): the
    collected set equals every triangle whose closest point lies within r, each once; large
    spheres hand whole subtrees over as CONTAINED ranges."""
    geo = pkg.torus_knot(10, 3, 60, 12)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=2)
    idx = np.empty(geo.index.size, dtype=np.uint32)
    orc.lib().orc_copy_index(o.h, idx.ctypes.data)
    tri = geo.position[idx.astype(np.int64).reshape(-1, 3)].astype(np.float64)
    rng = np.random.default_rng(13)
    lo, hi = geo.position.min(0), geo.position.max(0)
    c = lo + rng.random((300, 3)) * (hi - lo)
    r = np.exp(rng.uniform(np.log(0.3), np.log(12.0), 300))
    spheres = np.concatenate([c, r[:, None]], 1).astype(np.float32)
    counts, faces = o.sphere_triangles(spheres, cap=tri.shape[0])
    big = 0
    for i in range(spheres.shape[0]):
        p, rad = spheres[i, :3].astype(np.float64), float(spheres[i, 3])
        d = np.array([orc.point_triangle_distance(p, *t) for t in tri])
        got = faces[i, :counts[i]]
        assert np.unique(got).size == got.size
        want = np.nonzero(d <= rad)[0]
        sure_in = np.nonzero(d <= rad * (1 - 1e-9))[0]
        sure_out = np.nonzero(d > rad * (1 + 1e-9))[0]
        assert np.isin(sure_in, got).all() and not np.isin(sure_out, got).any(), i
        big += counts[i] > 200
    assert big > 20 and (counts == 0).sum() > 0
