"""The oracle's intersectsSphere (MeshBVH.js:796-809, sphereIntersectTriangle
src/math/MathUtilities.js:167-201), pinned by the reference's known answers
(test/ShapeCasts.test.js:565-604) and by a brute-force equivalence: the BVH answer must equal
"some triangle of the mesh is within r of the centre", evaluated triangle by triangle."""
import numpy as np


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
