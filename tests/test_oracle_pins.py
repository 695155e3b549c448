"""The oracle pinned against the known answers and properties the reference's own tests hold.

Reference tests (three-mesh-bvh 0.9.14, test/):
  Utils.geometryUtils.test.js:6-90    degenerate triangle raycastFirst(DoubleSide) known answer
  ShapeCasts.test.js:700-754          closestPointToPoint on SphereGeometry(1, 200, 200)
  ShapeCasts.test.js:872-930          all-hits / first-hit counts on TorusGeometry(5, 5, 40, 10)
  RandomRaycasts.test.js:179-208      BVH raycast == brute force, strategy x indirect x groups
  repro/RaycastsRepro.test.js:10-16   fixed LCG seed pairs (test/utils.js:6-23, m = 2e31)
"""
import math

import numpy as np
import pytest


def test_degenerate_triangle_known_answer(orc):
    hit = orc.ray_triangle([0, 0, 1], [0, 0, -1], [2, 0, 0], [0, 0, 0], [1, np.float32(1e-15), 0], side=2)
    assert hit is not None
    assert hit["face_index"] == 0
    assert hit["distance"] == 1.0
    assert list(hit["point"]) == [0.0, 0.0, 0.0]
    assert list(hit["barycoord"]) == [0.0, 0.0, 0.0]        # getBarycoord's zero-denominator result
    assert list(hit["normal"]) == [0.0, 0.0, -1.0]
    assert list(hit["face"]) == [0, 1, 2]
    # FrontSide culls it (the normal faces away from the ray)
    assert orc.ray_triangle([0, 0, 1], [0, 0, -1], [2, 0, 0], [0, 0, 0], [1, np.float32(1e-15), 0], side=0) is None


def test_sphere_distance_known_answers(pkg, orc):
    geo = pkg.sphere(1, 200, 200)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=0)
    res = o.closest_point(np.array([[0, 0, 0], [0, 1, 0]], dtype=np.float32))
    assert 1 - 0.001 <= res["distance"][0] <= 1
    assert res["distance"][1] == 0.0
    rng = np.random.default_rng(7)
    v = rng.uniform(-0.5, 0.5, size=(100, 3))
    length = rng.uniform(0, 3, size=100)
    pts = (v / np.linalg.norm(v, axis=1, keepdims=True) * length[:, None]).astype(np.float32)
    res = o.closest_point(pts)
    expected = np.abs(1 - np.linalg.norm(pts.astype(np.float64), axis=1))
    assert np.all(np.abs(res["distance"] - expected) <= 0.001)


def test_horn_torus_hit_counts(pkg, orc):
    geo = pkg.torus(5, 5, 40, 10)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=0)
    ray = np.array([[0, 0, -10, 0, 0, 1]], dtype=np.float32)
    counts, hits = o.raycast_all(ray)
    assert counts[0] == 10
    bc, _ = o.brute_raycast_all(ray)
    assert bc[0] == 10
    first = o.raycast_first(ray)[0]
    assert first["face_index"] >= 0 and first["distance"] == hits[0, :10]["distance"].min()


def _random_case(pkg, orc, strategy, indirect, grouped, seed, n_rays=100, near=0.0, far=math.inf):
    geo = pkg.torus(1, 1, 40, 10)
    if grouped:
        size = geo.index.size // 10
        for g in range(10):
            geo.add_group(g * size, size, 0)
    o = orc.OracleBVH.build(geo.position, geo.index, groups=geo.groups, strategy=strategy, indirect=indirect)
    rng = np.random.default_rng(seed)
    origin = rng.uniform(-5, 5, size=(n_rays, 3))
    target = rng.uniform(-1, 1, size=(n_rays, 3))
    d = target - origin
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([origin, d], 1).astype(np.float32)
    counts, hits = o.raycast_all(rays, near=near, far=far)
    bcounts, bhits = o.brute_raycast_all(rays, near=near, far=far)
    first = o.raycast_first(rays, near=near, far=far)
    return counts, hits, bcounts, bhits, first


@pytest.mark.parametrize("strategy", [0, 1, 2])
@pytest.mark.parametrize("indirect", [False, True])
@pytest.mark.parametrize("grouped", [False, True])
@pytest.mark.parametrize("near,far", [(0.0, math.inf), (6.0, math.inf), (0.0, 7.0), (6.0, 7.0)])
def test_bvh_equals_brute_force(pkg, orc, strategy, indirect, grouped, near, far):
    counts, hits, bcounts, bhits, first = _random_case(pkg, orc, strategy, indirect, grouped,
                                                       seed=strategy * 8 + indirect * 4 + grouped, near=near, far=far)
    assert np.array_equal(counts, bcounts)
    for i in range(counts.shape[0]):
        k = counts[i]
        assert sorted(hits[i, :k]["face_index"]) == sorted(bhits[i, :k]["face_index"])
        if k:
            assert first[i]["distance"] == hits[i, :k]["distance"].min()
        else:
            assert first[i]["face_index"] == -1


class _Lcg:
    """test/utils.js:6-23 (note m = 2e31, not 2**31)."""

    def __init__(self, seed):
        self.s = float(seed)

    def __call__(self):
        self.s = math.fmod(1103515245 * self.s + 12345, 2e31)
        return self.s / 2e31


@pytest.mark.parametrize("strategy,seed", [(1, 4697211981), (1, 1592666709), (2, 8903271423)])
@pytest.mark.parametrize("indirect", [False, True])
def test_repro_seeds(pkg, orc, strategy, seed, indirect):
    rnd = _Lcg(seed)
    rnd()
    o_ = np.array([rnd() * 10, rnd() * 10, rnd() * 10])
    d = -o_ / np.linalg.norm(o_)
    ray = np.array([[*o_, *d]], dtype=np.float32)
    geo = pkg.torus(1, 1, 40, 10)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=strategy, indirect=indirect)
    counts, hits = o.raycast_all(ray)
    bcounts, bhits = o.brute_raycast_all(ray)
    assert counts[0] == bcounts[0]
    assert sorted(hits[0, :counts[0]]["face_index"]) == sorted(bhits[0, :counts[0]]["face_index"])


def test_closest_point_equals_brute_force(pkg, orc):
    geo = pkg.torus_knot(10, 3, 64, 16)
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=2)
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 10)
    res = o.closest_point(pts)
    tri = geo.position[geo.index.astype(np.int64)].reshape(-1, 3, 3).astype(np.float64)
    for i in range(0, pts.shape[0], 37):
        best = min(np.sum((orc.closest_point_triangle(pts[i], *t) - pts[i]) ** 2) for t in tri)
        assert res["distance"][i] == pytest.approx(math.sqrt(best), rel=1e-12, abs=1e-12)


def test_box_group_sides_known_answer(pkg, orc):
    """ShapeCasts.test.js:931-979: a unit box, one group per face, per-group material sides."""
    geo = pkg.box()
    o = orc.OracleBVH.build(geo.position, geo.index, strategy=0)
    o.set_materials(geo.groups, [1, 0, 1, 0, 1, 0])        # Back, Front, Back, Front, Back, Front
    ray = np.array([[0, 0.25, -10, 0, 0, 1]], dtype=np.float32)
    counts, hits = o.raycast_all(ray)
    assert counts[0] == 2
    o.set_materials(geo.groups, [0, 0, 0, 0, 1, 1])        # Front x4, Back, Back
    first = o.raycast_first(ray)[0]
    assert first["point"][2] == 0.5
    assert first["material_index"] == 4


def test_box_group_gap_is_never_hit(pkg, orc):
    """ShapeCasts.test.js:981-1003: triangles in no group are not in the BVH."""
    geo = pkg.box()
    geo.groups = []
    geo.add_group(0, 6, 0)
    geo.add_group(12, 24, 1)
    o = orc.OracleBVH.build(geo.position, geo.index, groups=geo.groups, strategy=0)
    counts, _ = o.raycast_all(np.array([[-2, 0, 0, 1, 0, 0]], dtype=np.float32))
    assert counts[0] == 0
