"""GPU intersectsSphere (bvhc_intersects_sphere) and intersectsBox (bvhc_intersects_box) against
the oracle, and the reference's known answers (test/ShapeCasts.test.js:565-696) through the MeshBVH
mirror; Intersection attribute fields (uv, normal) interpolated at the hits (bvhc_hit_interpolate)."""
import math

import numpy as np
import pytest

from obb_util import compose, quaternion_xyz, random_boxes, record

pytestmark = pytest.mark.gpu


def test_intersects_sphere_known_answers_gpu(pkg, cuda):
    geo = pkg.sphere(1, 50, 50)
    bvh = pkg.MeshBVH(geo, {"verbose": False})
    assert bvh.intersectsSphere(((0, 1, 0), 0.01)) is True
    assert bvh.intersectsSphere(((0, 0, 0), 0.9)) is False
    assert bvh.intersectsSphere(((0, 2.01, 0), 0.9)) is False


@pytest.mark.parametrize("indirect", [False, True])
def test_intersects_sphere_matches_oracle(pkg, orc, cuda, indirect):
    import torch

    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=3)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "indirect": indirect})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
    rng = np.random.default_rng(17)
    lo, hi = geo.position.min(0) - 4, geo.position.max(0) + 4
    n = 200_000
    c = lo + rng.random((n, 3)) * (hi - lo)
    r = np.exp(rng.uniform(np.log(0.01), np.log(6.0), n))
    spheres = np.concatenate([c, r[:, None]], 1).astype(np.float32)
    # spheres that just touch a vertex (the boundary): the GPU must not miss a touching triangle
    v = geo.position[rng.choice(geo.position.shape[0], 2000, replace=False)]
    touch = np.concatenate([v + np.float32(0.5), np.full((2000, 1), np.float32(0.5 * np.sqrt(3) + 1e-3))], 1)
    spheres = np.concatenate([spheres, touch.astype(np.float32)])
    exp = ref.intersects_sphere(spheres)
    got = bvh.intersects_sphere_batch(spheres)
    dev = bvh.intersects_sphere_batch(torch.from_numpy(spheres).to(cuda)).cpu().numpy().astype(bool)
    bvh.synchronize()
    assert np.array_equal(got, dev)
    bad = np.nonzero(got != exp)[0]
    # a disagreement is allowed only on the boundary: the nearest triangle within 1e-6 relative of r
    tri = geo.position[geo.index.astype(np.int64).reshape(-1, 3)].astype(np.float64)
    for i in bad[:50]:
        p = spheres[i, :3].astype(np.float64)
        rad = float(spheres[i, 3])
        cp = ref.closest_point(spheres[i:i + 1, :3])
        d = float(cp["distance"][0])
        assert abs(d - rad) <= 1e-6 * max(rad, 1.0), (i, d, rad, got[i], exp[i])
    assert bad.size <= 5, bad.size
    assert 0.05 < exp.mean() < 0.95


def test_hit_attribute_interpolation(pkg, cuda):
    """uv and normal at the hit point (ThreeRayIntersectUtilities.js:59-117): the barycentric
    combination of the hit triangle's vertex attributes, the normal turned against the ray."""
    import torch

    geo = pkg.torus_knot(10, 3, 200, 40)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    rays = np.concatenate([pkg.rays_camera(96, 96), pkg.rays_sphere_to_box(5000, seed=2)])
    hits = bvh.raycast_first_batch(rays, 2)                 # double sided: back faces too
    hit = hits["face_index"] != 0xFFFFFFFF
    assert hit.sum() > 2000
    tri = geo.index.astype(np.int64).reshape(-1, 3)[np.where(hit, hits["face_index"], 0)]
    w = hits["barycoord"].astype(np.float64)[..., None]
    exp_uv = (w * geo.uv[tri].astype(np.float64)).sum(1)
    exp_n = (w * geo.normal[tri].astype(np.float64)).sum(1)
    flip = (exp_n * rays[:, 3:]).sum(1) > 0
    exp_n[flip] *= -1
    uv = bvh.hit_interpolate(hits, geo.uv)
    nrm = bvh.hit_interpolate(hits, geo.normal, rays)
    assert np.abs(uv[hit] - exp_uv[hit]).max() <= 1e-5
    assert np.abs(nrm[hit] - exp_n[hit]).max() <= 1e-5
    assert not uv[~hit].any() and not nrm[~hit].any()
    d_hits = bvh.raycast_first_batch(torch.from_numpy(rays).to(cuda), 2)
    d_uv = bvh.hit_interpolate(d_hits, torch.from_numpy(geo.uv).to(cuda))
    bvh.synchronize()
    assert np.array_equal(d_uv.cpu().numpy(), uv)
    first = bvh.raycastFirst((rays[0, :3], rays[0, 3:]), 2)
    if first is not None:
        assert first.uv is not None and first.normal is not None
        assert float(np.dot(first.normal, rays[0, 3:])) <= 0


def test_intersects_box_known_answers_gpu(pkg, cuda):
    geo = pkg.sphere(1, 50, 50)
    bvh = pkg.MeshBVH(geo, {"verbose": False})
    q = quaternion_xyz(math.pi / 4, math.pi / 4, 0)
    assert bvh.intersectsBox(((-1, -1, -1), (1, 1, 1)), compose((0, 3, 0), q)) is False
    assert bvh.intersectsBox(((-1, -1, -1), (1, 1, 1)), compose((0, 2, 0), q)) is True
    assert bvh.intersectsBox(((-10, -10, -10), (10, 10, 10)), compose((0, 0, 0), q)) is True
    assert bvh.intersectsBox(((-.5, -.5, -.5), (.5, .5, .5)), compose((0, 0, 0), q)) is False
    assert bvh.intersectsBox(((-10, 0, -10), (10, 10, 10)), compose((0, 0, 0), q)) is True


def _touching_boxes(rng, geo, n):
    """Axis-aligned boxes (identity matrix) whose faces sit exactly on vertex coordinates: every
    decision there is an exact tie that the float-float margin hands to binary64."""
    v = geo.position[rng.integers(0, geo.position.shape[0], (n, 2))]
    lo, hi = np.minimum(v[:, 0], v[:, 1]), np.maximum(v[:, 0], v[:, 1])
    side = rng.integers(0, 3, n)
    far = geo.position.max(0) + 5
    hi2 = hi.copy()
    lo2 = lo.copy()
    # half the boxes end exactly at a vertex coordinate on one axis and extend away from the mesh
    for i in range(n // 2):
        lo2[i, side[i]] = hi[i, side[i]]
        hi2[i, side[i]] = far[side[i]]
    eye = np.eye(4).reshape(-1)
    return np.stack([record(lo2[i], hi2[i], eye) for i in range(n)])


def _projective(rng, n, spread):
    out = random_boxes(rng, n, np.zeros(3), spread)
    out[:, 8 + 3] = rng.uniform(-0.01, 0.01, n)   # e[3]: a perspective term (non-affine)
    out[:, 8 + 15] = rng.uniform(0.9, 1.1, n)
    return out


@pytest.mark.parametrize("indirect", [False, True])
def test_intersects_box_matches_oracle(pkg, orc, cuda, indirect):
    import torch

    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=3)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "indirect": indirect})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
    rng = np.random.default_rng(23)
    boxes = np.concatenate([random_boxes(rng, 20_000, np.zeros(3), 16.0),
                            random_boxes(rng, 4_000, np.zeros(3), 16.0, shear=True),
                            _projective(rng, 1_000, 16.0),
                            _touching_boxes(rng, geo, 4_000)])
    want = ref.intersects_box(boxes)
    got = bvh.intersects_box_batch(boxes)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, (bad[:10], boxes[bad[:2]])
    assert 0.05 < want.mean() < 0.95
    d = torch.from_numpy(boxes).to(cuda)
    dev = bvh.intersects_box_batch(d)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy().astype(bool), got)
    bvh.dispose()


def test_intersects_box_lattice_ties(pkg, orc, cuda):
    """Unit cubes on an integer lattice and integer-aligned boxes: faces coincide exactly."""
    cube = pkg.box()
    pos, idx, k = [], [], 0
    for x in range(5):
        for y in range(5):
            for z in range(5):
                pos.append(cube.position + np.array([x, y, z], np.float32) * 2)
                idx.append(cube.index.astype(np.int64) + k)
                k += cube.position.shape[0]
    geo = pkg.Geometry(np.concatenate(pos), np.concatenate(idx).astype(np.uint32))
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, None, geo.position)
    rng = np.random.default_rng(29)
    n = 5000
    lo = rng.integers(-2, 10, (n, 3)).astype(np.float32) - 0.5 * rng.integers(0, 2, (n, 3))
    hi = lo + rng.integers(0, 3, (n, 3)).astype(np.float32) * 0.5
    eye = np.eye(4).reshape(-1)
    boxes = np.stack([record(lo[i], hi[i], eye) for i in range(n)])
    want = ref.intersects_box(boxes)
    got = bvh.intersects_box_batch(boxes)
    assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
    assert 0.05 < want.mean() < 0.95
    bvh.dispose()


def _near_plane_boxes(rng, geo, n):
    """Rotated boxes resting on a triangle's plane: the box's bottom face is parallel to the
    triangle, offset along its normal by +-1e-5 .. 0 of the mesh scale, box rotated about the normal
    and slid so a vertex or an edge is near its rim.  Decisions there sit on the normal and
    cross-product axes' margins."""
    pos, tri = geo.position.astype(np.float64), geo.index.reshape(-1, 3)
    scale = np.abs(pos).max()
    out = np.zeros((n, 24), np.float32)
    for i in range(n):
        a, b, c = pos[tri[rng.integers(0, tri.shape[0])]]
        nrm = np.cross(b - a, c - a)
        nrm /= np.linalg.norm(nrm)
        u = (b - a) / np.linalg.norm(b - a)
        ang = rng.uniform(0, 2 * np.pi)
        u = u * np.cos(ang) + np.cross(nrm, u) * np.sin(ang)
        nrm = nrm * rng.choice([-1.0, 1.0])
        w = np.cross(nrm, u)
        h = rng.uniform(0.002, 0.05)
        delta = rng.choice([-1e-5, -1e-6, -1e-7, 0.0, 1e-7, 1e-6, 1e-5]) * scale
        anchor = (a, (a + b) / 2, (a + b + c) / 3)[rng.integers(0, 3)]
        m = np.eye(4)
        m[:3, 0], m[:3, 1], m[:3, 2] = u, w, nrm
        m[:3, 3] = anchor + nrm * delta + (u * rng.uniform(-h, h) + w * rng.uniform(-h, h)) * rng.integers(0, 2)
        out[i] = record(np.array([-h, -h, 0.0]), np.array([h, h, 2 * h]), m.T.reshape(-1))
    return out


def test_intersects_box_near_contact(pkg, orc, cuda):
    """Rotated boxes within 1e-5 of the mesh scale of a triangle's plane: the float32 and
    float-float tiers must hand every close call on; results identical to the oracle."""
    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=3)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, None, geo.position)
    boxes = _near_plane_boxes(np.random.default_rng(37), geo, 20_000)
    want = ref.intersects_box(boxes)
    got = bvh.intersects_box_batch(boxes)
    bad = np.nonzero(got != want)[0]
    assert bad.size == 0, (bad[:10], boxes[bad[:2]])
    assert 0.05 < want.mean() < 0.95
    bvh.dispose()


@pytest.mark.parametrize("indirect", [False, True])
def test_sphere_triangles_match_oracle(pkg, orc, cuda, indirect):
    """Triangles within spheres through shapecast's CONTAINED path: the same faceIndex sequence as
    the oracle (traversal order), counts identical; spheres from tiny to enclosing whole subtrees."""
    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=3)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "indirect": indirect})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
    rng = np.random.default_rng(31)
    lo, hi = geo.position.min(0), geo.position.max(0)
    n = 20_000
    c = lo + rng.random((n, 3)) * (hi - lo)
    r = np.exp(rng.uniform(np.log(0.05), np.log(8.0), n))
    spheres = np.concatenate([c, r[:, None]], 1).astype(np.float32)
    cap = 512
    counts, faces = bvh.sphere_triangles_batch(spheres, cap=cap)
    ec, ef = ref.sphere_triangles(spheres, cap=cap)
    diff = np.nonzero(counts.astype(np.int64) != ec)[0]
    # a triangle exactly at the radius (the float-float triangle predicate against the float64 one)
    assert diff.size <= max(2, n // 5000), diff[:10]
    same = np.setdiff1d(np.arange(n), diff)
    k = np.minimum(ec[same], cap)
    for i, kk in zip(same, k):
        assert np.array_equal(faces[i, :kk].astype(np.int64), ef[i, :kk]), i
    assert (ec > cap).sum() > 0 and (ec == 0).sum() > 0
    c0, _ = bvh.sphere_triangles_batch(spheres, cap=0)
    assert np.array_equal(c0, counts)
    bvh.dispose()
