"""GPU parity: libbvhcuda's kernels, called through the C ABI, against the oracle on the same
serialized BVHs and the same float32 inputs (tolerances in tests/parity.py)."""
import math

import numpy as np
import pytest

from parity import check_all, check_closest, check_first, tie_exempt

pytestmark = pytest.mark.gpu

ZERO = dict(hitmiss=0, face=0, distance=0, point=0, barycoord=0)


def _assert_first_ok(rep):
    bad = {k: rep[k] for k in ZERO if rep[k]}
    assert not bad, rep


def _oracle_for(orc, bvh, geo):
    return orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)


@pytest.fixture(scope="module")
def knot80k(pkg, orc, cuda):
    geo = pkg.torus_knot(10, 3, 400, 100)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "maxLeafSize": 10, "maxDepth": 40})
    return geo, bvh, _oracle_for(orc, bvh, geo)


@pytest.mark.parametrize("side", [0, 1, 2])
def test_raycast_first_knot80k(pkg, knot80k, side):
    geo, bvh, ref = knot80k
    rays = pkg.rays_sphere_to_box(200_000 if side == 0 else 50_000, seed=0)
    got = bvh.raycast_first_batch(rays, side)
    exp = ref.raycast_first(rays, side)
    ac, ah = ref.raycast_all(rays, side, cap=64)
    rep = check_first(got, exp, tie_exempt(ac, ah))
    _assert_first_ok(rep)
    assert rep["hits"] > rays.shape[0] // 10


def test_raycast_all_knot80k(pkg, knot80k):
    geo, bvh, ref = knot80k
    rays = pkg.rays_sphere_to_box(50_000, seed=5)
    for side in (0, 2):
        counts, hits = bvh.raycast_batch(rays, side, cap=64)
        ec, eh = ref.raycast_all(rays, side, cap=64)
        rep = check_all(counts, hits, ec, eh)
        assert rep["count"] == 0 and rep["set"] == 0 and rep["distance"] == 0, rep


def test_closest_point_knot80k(pkg, orc, knot80k):
    geo, bvh, ref = knot80k
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 40)
    got = bvh.closest_point_batch(pts, 0.0, 5.0)
    exp = ref.closest_point(pts, 0.0, 5.0)

    def tri_distance(i, face):
        t = geo.triangle(face)
        q = orc.closest_point_triangle(pts[i].astype(np.float64), *t)
        return float(np.linalg.norm(q - pts[i].astype(np.float64)))

    rep = check_closest(got, exp, tri_distance)
    assert rep["null"] == 0 and rep["distance"] == 0 and rep["face"] == 0, rep


def test_closest_point_min_threshold_and_unbounded(pkg, knot80k):
    geo, bvh, ref = knot80k
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 16)
    for lo, hi in ((0.0, math.inf), (0.5, 3.0)):
        got = bvh.closest_point_batch(pts, lo, hi)
        exp = ref.closest_point(pts, lo, hi)
        rep = check_closest(got, exp)
        assert rep["null"] == 0, rep
        if lo == 0.0:
            assert rep["distance"] == 0, rep


@pytest.mark.parametrize("strategy", [0, 1, 2])
@pytest.mark.parametrize("indirect", [False, True])
@pytest.mark.parametrize("grouped", [False, True])
def test_random_torus_matrix(pkg, orc, cuda, strategy, indirect, grouped):
    """RandomRaycasts.test.js:32-38 matrix, with near/far in {0, 6} x {inf, 7}."""
    geo = pkg.torus(1, 1, 40, 10)
    if grouped:
        size = geo.index.size // 10
        for g in range(10):
            geo.add_group(g * size, size, 0)
    bvh = pkg.MeshBVH(geo, {"strategy": strategy, "indirect": indirect})
    ref = _oracle_for(orc, bvh, geo)
    rng = np.random.default_rng(100 + strategy * 4 + indirect * 2 + grouped)
    o = rng.uniform(-5, 5, size=(2000, 3))
    d = rng.uniform(-1, 1, size=(2000, 3)) - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    for near, far in ((0.0, math.inf), (6.0, math.inf), (0.0, 7.0), (6.0, 7.0)):
        got = bvh.raycast_first_batch(rays, 0, near, far)
        exp = ref.raycast_first(rays, 0, near, far)
        ac, ah = ref.raycast_all(rays, 0, near, far)
        _assert_first_ok(check_first(got, exp, tie_exempt(ac, ah)))
        counts, hits = bvh.raycast_batch(rays, 0, near, far)
        rep = check_all(counts, hits, ac, ah)
        assert rep["count"] == 0 and rep["set"] == 0, rep
    bvh.dispose()


def test_degenerate_triangle_gpu(pkg, cuda):
    pos = np.array([[2, 0, 0], [0, 0, 0], [1, 1e-15, 0]], dtype=np.float32)
    geo = pkg.Geometry(pos, None)
    bvh = pkg.MeshBVH(geo)
    hit = bvh.raycastFirst(((0, 0, 1), (0, 0, -1)), pkg.DoubleSide)
    assert hit is not None
    assert hit.faceIndex == 0 and hit.distance == 1.0
    assert list(hit.point) == [0.0, 0.0, 0.0]
    assert list(hit.barycoord) == [0.0, 0.0, 0.0]
    assert (hit.face.a, hit.face.b, hit.face.c) == (0, 1, 2)
    assert list(hit.face.normal) == [0.0, 0.0, -1.0]
    assert bvh.raycastFirst(((0, 0, 1), (0, 0, -1)), pkg.FrontSide) is None


def test_sliver_triangles_barycoords(pkg, orc, cuda):
    """Hit records on sliver triangles (apex 2^-30 .. 2^-12 of the base length off the base line):
    the degenerate-triangle test is settled in float32 only when the triangle is clearly not
    degenerate (apex at 2^-16 and wider here) and in float-float otherwise, and the records (the
    zero barycentrics of the degenerate ones included) match the oracle's."""
    heights = [2.0 ** -30, 2.0 ** -28, 2.0 ** -20, 2.0 ** -18, 2.0 ** -17, 2.0 ** -16, 2.0 ** -15, 2.0 ** -12]
    pos, rays = [], []
    for k, h in enumerate(heights):
        x = 10.0 * k
        pos += [[x, 0.0, 0.0], [x + 2.0, 0.0, 0.0], [x + 1.0, h, 0.0]]
        for fx, fy in ((1.0, 0.5), (0.75, 0.25), (1.25, 0.25), (1.0, 0.875)):
            rays.append([x + fx, h * fy, 5.0, 0.0, 0.0, -1.0])
    geo = pkg.Geometry(np.array(pos, dtype=np.float32), None)
    bvh = pkg.MeshBVH(geo)
    ref = _oracle_for(orc, bvh, geo)
    rays = np.array(rays, dtype=np.float32)
    got = bvh.raycast_first_batch(rays, pkg.DoubleSide)
    exp = ref.raycast_first(rays, pkg.DoubleSide)
    ac, ah = ref.raycast_all(rays, pkg.DoubleSide)
    _assert_first_ok(check_first(got, exp, tie_exempt(ac, ah)))
    hit = exp["face_index"] != 0xFFFFFFFF
    assert hit.sum() >= 20
    zero = (exp["barycoord"] == 0).all(1)
    assert zero[hit].any() and (~zero[hit]).any()   # both degenerate and ordinary slivers are hit
    bvh.dispose()


def test_sphere_distance_gpu(pkg, cuda):
    geo = pkg.sphere(1, 200, 200)
    bvh = pkg.MeshBVH(geo, {"verbose": False})
    t = bvh.closestPointToPoint((0, 0, 0))
    assert 1 - 0.001 <= t.distance <= 1
    assert bvh.closestPointToPoint((0, 1, 0)).distance == 0
    rng = np.random.default_rng(11)
    for _ in range(100):
        v = rng.uniform(-0.5, 0.5, 3)
        length = rng.uniform(0, 3)
        v = v / np.linalg.norm(v) * length
        t = bvh.closestPointToPoint(v)
        assert abs(t.distance - abs(1 - length)) <= 0.001 + 1e-6


def test_horn_torus_hits_gpu(pkg, cuda):
    geo = pkg.torus(5, 5, 40, 10)
    bvh = pkg.MeshBVH(geo)
    hits = bvh.raycast(((0, 0, -10), (0, 0, 1)))
    assert len(hits) == 10
    first = bvh.raycastFirst(((0, 0, -10), (0, 0, 1)))
    assert first is not None and first.distance == min(h.distance for h in hits)


def test_noisy_knot_incoherent_and_camera(pkg, orc, cuda):
    geo = pkg.torus_knot(10, 3, 500, 125, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = _oracle_for(orc, bvh, geo)
    for rays in (pkg.rays_incoherent(200_000, seed=1), pkg.rays_camera(320, 320)):
        got = bvh.raycast_first_batch(rays)
        exp = ref.raycast_first(rays)
        ac, ah = ref.raycast_all(rays, cap=64)
        _assert_first_ok(check_first(got, exp, tie_exempt(ac, ah)))
        counts, hits = bvh.raycast_batch(rays[:50_000], cap=64)
        rep = check_all(counts, hits, ac[:50_000], ah[:50_000])
        assert rep["count"] == 0 and rep["set"] == 0, rep


def test_device_buffers_match_host(pkg, knot80k, cuda):
    import torch

    geo, bvh, ref = knot80k
    rays = pkg.rays_sphere_to_box(100_000, seed=3)
    host = bvh.raycast_first_batch(rays)
    dev = bvh.raycast_first_batch(torch.from_numpy(rays).to(cuda))
    bvh.synchronize()
    got = dev.cpu().numpy().view(np.uint8).reshape(-1).view(host.dtype)
    assert np.array_equal(got.view(np.uint8), host.view(np.uint8))
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 20)
    h2 = bvh.closest_point_batch(pts, 0.0, 5.0)
    d2 = bvh.closest_point_batch(torch.from_numpy(pts).to(cuda), 0.0, 5.0)
    bvh.synchronize()
    assert np.array_equal(d2.cpu().numpy().view(np.uint8).reshape(-1), h2.view(np.uint8))


def test_box_group_sides_gpu(pkg, cuda):
    """ShapeCasts.test.js:931-979 on the GPU: material-array raycast and raycastFirst."""
    geo = pkg.box()
    bvh = pkg.MeshBVH(geo)
    ray = ((0, 0.25, -10), (0, 0, 1))
    hits = bvh.raycast(ray, [1, 0, 1, 0, 1, 0])
    assert len(hits) == 2
    first = bvh.raycastFirst(ray, [0, 0, 0, 0, 1, 1])
    assert first is not None and first.point[2] == 0.5 and first.face.materialIndex == 4
    gap = pkg.box()
    gap.groups = []
    gap.add_group(0, 6, 0)
    gap.add_group(12, 24, 1)
    bvh2 = pkg.MeshBVH(gap)
    assert bvh2.raycast(((-2, 0, 0), (1, 0, 0))) == []


def test_material_array_random_parity(pkg, orc, cuda):
    geo = pkg.torus_knot(10, 3, 120, 24)
    n = geo.index.size
    step = (n // 3 // 7) * 3
    for g in range(7):
        geo.add_group(g * step, step if g < 6 else math.inf, g % 4)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = _oracle_for(orc, bvh, geo)
    sides = [0, 1, 2]                  # material 3 is past the array: FrontSide
    ref.set_materials(geo.groups, sides)
    rays = pkg.rays_sphere_to_box(20_000, seed=9)
    got = bvh.raycast_first_batch(rays, sides)
    exp = ref.raycast_first(rays)
    ac, ah = ref.raycast_all(rays, cap=64)
    _assert_first_ok(check_first(got, exp, tie_exempt(ac, ah)))
    counts, hits = bvh.raycast_batch(rays, sides, cap=64)
    rep = check_all(counts, hits, ac, ah)
    assert rep["count"] == 0 and rep["set"] == 0, rep


@pytest.mark.parametrize("persistent,order,refill,occupancy,compact,sort",
                         [(0, 0, 16, 0, 0, 0), (0, 1, 16, 0, 0, 0), (1, 0, 1, 0, 0, 0), (1, 1, 16, 1, 0, 0),
                          (1, 1, 32, 2, 0, 0), (1, 0, 24, 2, 0, 0), (1, 1, 8, 2, 1, 0), (1, 0, 16, 1, 1, 0),
                          (2, 0, 16, 0, 0, 0), (2, 1, 16, 0, 0, 0), (2, 0, 16, 0, 1, 0), (1, 1, 32, 2, 1, 1),
                          (1, 1, 16, 1, 0, 2), (1, 0, 32, 2, 1, 3), (2, 0, 16, 0, 1, 1), (2, 1, 16, 0, 0, 2),
                          (2, 0, 16, 0, 1, 3)])
def test_traversal_variants_agree(pkg, orc, cuda, persistent, order, refill, occupancy, compact, sort):
    geo = pkg.torus_knot(10, 3, 500, 125, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = _oracle_for(orc, bvh, geo)
    bvh.set_traversal(persistent, order, refill, occupancy, compact, sort)
    assert bvh.get_traversal() == dict(persistent=persistent, order=order, refill=refill, occupancy=occupancy,
                                       compact=compact, sort=sort, closest=0, wide=0, all=0, tile=0,
                                       block=0, stack=0, tile_rows=0)
    rays = np.concatenate([pkg.rays_incoherent(100_000, seed=4), pkg.rays_camera(256, 256),
                           pkg.rays_sphere_to_box(50_000, seed=6)])
    for side in (0, 2):
        got = bvh.raycast_first_batch(rays, side)
        exp = ref.raycast_first(rays, side)
        ac, ah = ref.raycast_all(rays, side, cap=64)
        _assert_first_ok(check_first(got, exp, tie_exempt(ac, ah)))
    near_far = bvh.raycast_first_batch(rays, 0, 30.0, 45.0)
    exp = ref.raycast_first(rays, 0, 30.0, 45.0)
    ac, ah = ref.raycast_all(rays, 0, 30.0, 45.0, cap=64)
    _assert_first_ok(check_first(near_far, exp, tie_exempt(ac, ah)))
    bvh.dispose()


def test_pipelined_host_path_matches_device(pkg, knot80k, cuda):
    """Host batches above one chunk (2^20 rays) run chunk-pipelined over two streams."""
    import torch

    geo, bvh, ref = knot80k
    rays = pkg.rays_sphere_to_box(3_000_000 + 1234, seed=12)
    pinned = torch.from_numpy(rays).pin_memory()
    # the compacting and ordering variants keep one queue (and sort scratch) per pipeline slot
    for persistent, compact, sort in ((1, 0, 0), (1, 1, 0), (1, 1, 3), (2, 0, 1)):
        bvh.set_traversal(persistent, 1, 16, 2, compact, sort)
        host = bvh.raycast_first_batch(pinned.numpy())
        dev = bvh.raycast_first_batch(torch.from_numpy(rays).to(cuda))
        bvh.synchronize()
        assert np.array_equal(dev.cpu().numpy().view(np.uint8).reshape(-1), host.view(np.uint8).reshape(-1))
        sub = slice(0, 20_000)
        exp = ref.raycast_first(rays[sub])
        ac, ah = ref.raycast_all(rays[sub], cap=64)
        _assert_first_ok(check_first(host[sub], exp, tie_exempt(ac, ah)))
    bvh.set_traversal(1, 1, 16, 0, 0)


@pytest.mark.parametrize("leaf", [1, 3, 4])
def test_split_leaf_layouts_agree(pkg, orc, cuda, leaf):
    """Device leaves split to at most `leaf` triangles: every query kind still matches the oracle
    (which keeps the reference's leaves), and the reference layout comes back with leaf size 0."""
    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=1)
    n = geo.index.size
    step = (n // 3 // 5) * 3
    for g in range(5):
        geo.add_group(g * step, step if g < 4 else math.inf, g % 3)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = _oracle_for(orc, bvh, geo)
    base_nodes = bvh.mesh_info()["node_records"]
    bvh.set_leaf_size(leaf)
    assert bvh.get_leaf_size() == leaf
    assert bvh.mesh_info()["node_records"] > base_nodes
    rays = np.concatenate([pkg.rays_incoherent(60_000, seed=4), pkg.rays_camera(160, 160),
                           pkg.rays_sphere_to_box(30_000, seed=6)])
    ac, ah = ref.raycast_all(rays, 0, cap=64)
    exp = ref.raycast_first(rays, 0)
    for cfg in ((0, 1, 16, 0, 0, 0), (1, 1, 32, 2, 1, 2), (2, 1, 16, 2, 1, 1), (2, 1, 16, 2, 1, 1, 0, 1)):
        bvh.set_traversal(*cfg)
        _assert_first_ok(check_first(bvh.raycast_first_batch(rays, 0), exp, tie_exempt(ac, ah)))
    counts, hits = bvh.raycast_batch(rays, 0, cap=64)
    rep = check_all(counts, hits, ac, ah)
    assert rep["count"] == 0 and rep["set"] == 0, rep
    sides = [0, 1, 2]
    ref.set_materials(geo.groups, sides)
    mexp = ref.raycast_first(rays)
    mac, mah = ref.raycast_all(rays, cap=64)
    _assert_first_ok(check_first(bvh.raycast_first_batch(rays, sides), mexp, tie_exempt(mac, mah)))
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 24)

    def tri_distance(i, face):
        t = geo.triangle(face)
        q = orc.closest_point_triangle(pts[i].astype(np.float64), *t)
        return float(np.linalg.norm(q - pts[i].astype(np.float64)))

    rep = check_closest(bvh.closest_point_batch(pts, 0.0, 5.0), ref.closest_point(pts, 0.0, 5.0), tri_distance)
    assert rep["null"] == 0 and rep["distance"] == 0 and rep["face"] == 0, rep
    bvh.set_leaf_size(0)
    assert bvh.mesh_info()["node_records"] == base_nodes
    _assert_first_ok(check_first(bvh.raycast_first_batch(rays, 0), exp, tie_exempt(ac, ah)))
    bvh.dispose()


@pytest.mark.parametrize("closest,occupancy,leaf", [(1, 0, 0), (1, 2, 0), (2, 0, 0), (2, 2, 0), (1, 0, 4), (3, 0, 0),
                                                    (4, 2, 2), (5, 1, 0), (6, 0, 0), (6, 2, 3)])
def test_closest_point_warp_cooperative(pkg, orc, knot80k, closest, occupancy, leaf):
    """The warp-cooperative closest-point kernels (input order and Morton-sorted queries, whole warps
    and 16- or 8-lane groups; with and without raycastFirst's split-leaf copy present, which closest
    point does not read) against the
    oracle: grid queries with maxThreshold 5 (nulls beyond it, and results beyond it from leaves
    whose box is within it), unbounded, and a sparse random set; minThreshold > 0 falls back to the
    per-query kernel and must match too."""
    geo, bvh, ref = knot80k
    bvh.set_leaf_size(leaf)
    bvh.set_traversal(1, 1, 16, occupancy, 0, 0, closest)
    rng = np.random.default_rng(21)
    lo, hi = geo.position.min(0), geo.position.max(0)
    sets = [pkg.grid_points(lo, hi, 40),
            (lo - 8 + rng.random((20_000, 3)) * (hi - lo + 16)).astype(np.float32)]

    def tri_distance(pts):
        def f(i, face):
            t = geo.triangle(face)
            q = orc.closest_point_triangle(pts[i].astype(np.float64), *t)
            return float(np.linalg.norm(q - pts[i].astype(np.float64)))
        return f

    for pts in sets:
        for lo_t, hi_t in ((0.0, 5.0), (0.0, math.inf), (0.5, 3.0)):
            got = bvh.closest_point_batch(pts, lo_t, hi_t)
            exp = ref.closest_point(pts, lo_t, hi_t)
            rep = check_closest(got, exp, tri_distance(pts))
            assert rep["null"] == 0 and rep["face"] == 0, (lo_t, hi_t, rep)
            if lo_t == 0.0:
                assert rep["distance"] == 0, (lo_t, hi_t, rep)
    bvh.set_traversal(1, 1, 16, 0, 0, 0, 0)
    bvh.set_leaf_size(0)


@pytest.mark.parametrize("leaf,occupancy,compact,sort", [(0, 0, 0, 0), (0, 2, 1, 1), (4, 1, 1, 2), (2, 2, 0, 0),
                                                         (3, 0, 1, 3)])
def test_wide_warp_cooperative_raycast_first(pkg, orc, cuda, leaf, occupancy, compact, sort):
    """raycastFirst over the four-child records (with the reference's or split leaves), against the
    oracle, including near/far limits and a double-sided pass; the records follow a refit."""
    geo = pkg.torus_knot(10, 3, 400, 80, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = _oracle_for(orc, bvh, geo)
    bvh.set_leaf_size(leaf)
    bvh.set_traversal(2, 1, 16, occupancy, compact, sort, 0, 1)
    assert bvh.get_traversal()["wide"] == 1
    rays = np.concatenate([pkg.rays_incoherent(60_000, seed=9), pkg.rays_camera(200, 200),
                           pkg.rays_sphere_to_box(30_000, seed=10)])
    for side, near, far in ((0, 0.0, math.inf), (2, 0.0, math.inf), (0, 30.0, 45.0)):
        got = bvh.raycast_first_batch(rays, side, near, far)
        exp = ref.raycast_first(rays, side, near, far)
        ac, ah = ref.raycast_all(rays, side, near, far, cap=64)
        _assert_first_ok(check_first(got, exp, tie_exempt(ac, ah)))
    pos = (geo.position * np.float32(1.25)).astype(np.float32)
    bvh.refit(pos)
    ref.refit(pos)
    got = bvh.raycast_first_batch(rays)
    ac, ah = ref.raycast_all(rays, cap=64)
    _assert_first_ok(check_first(got, ref.raycast_first(rays), tie_exempt(ac, ah)))
    bvh.dispose()


@pytest.mark.parametrize("closest,leaf", [(0, 0), (1, 0), (2, 0), (2, 4), (3, 0), (4, 0), (6, 0)])
def test_closest_point_host_pipeline(pkg, orc, knot80k, cuda, closest, leaf):
    """closestPointToPoint through host memory for more than one pipeline chunk (2.5M points: three
    1M-point chunks on three streams, the last one partial) gives the device-memory call's results,
    and a strided sample of them matches the oracle."""
    import torch

    geo, bvh, ref = knot80k
    bvh.set_leaf_size(leaf)
    bvh.set_traversal(1, 1, 16, 0, 0, 0, closest)
    rng = np.random.default_rng(23)
    lo, hi = geo.position.min(0), geo.position.max(0)
    pts = (lo - 2 + rng.random((2_500_000, 3)) * (hi - lo + 4)).astype(np.float32)
    host = bvh.closest_point_batch(pts, 0.0, 5.0)
    d = bvh.closest_point_batch(torch.from_numpy(pts).to(cuda), 0.0, 5.0)
    torch.cuda.synchronize()
    dev = d.cpu().numpy().view(np.uint8).reshape(-1)
    dev = np.frombuffer(dev.tobytes(), dtype=host.dtype)
    # byte-identical: exact distance ties go to the smaller faceIndex whatever the grouping of the
    # queries (chunks, Morton sort per chunk or over the whole call)
    assert np.array_equal(host.view(np.uint8), dev.view(np.uint8))

    def tri_distance(p):
        def f(i, face):
            q = orc.closest_point_triangle(p[i].astype(np.float64), *geo.triangle(face))
            return float(np.linalg.norm(q - p[i].astype(np.float64)))
        return f

    idx = np.arange(0, pts.shape[0], 97)
    exp = ref.closest_point(pts[idx], 0.0, 5.0)

    rep = check_closest(host[idx], exp, tri_distance(pts[idx]))
    assert rep["null"] == 0 and rep["face"] == 0 and rep["distance"] == 0, rep
    bvh.set_traversal(1, 1, 16, 0, 0, 0, 0)
    bvh.set_leaf_size(0)


def test_traversal_config_rejects_bad_fields(pkg, cuda):
    """Tile pitches that are not a positive multiple of 8 (of 16 for 2-row tiles), tile heights other
    than 2 / 4 / 8, block sizes other than 64 / 128 / 256, stacks other than 32 / 64 and
    closest-point kernels outside 0..6 are rejected."""
    geo = pkg.torus_knot(10, 3, 32, 8)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    for bad in (dict(tile=12), dict(tile=-8), dict(block=96), dict(stack=48), dict(stack=16), dict(tile_rows=3),
                dict(tile=24, tile_rows=2), dict(closest=7), dict(closest=-1)):
        with pytest.raises(pkg.BVHCError):
            bvh.set_traversal(2, 1, 16, 0, **bad)
    bvh.set_traversal(2, 1, 16, 2, tile=4096, block=256, stack=32, tile_rows=8, closest=6)
    assert bvh.get_traversal() == dict(persistent=2, order=1, refill=16, occupancy=2, compact=0, sort=0, closest=6,
                                       wide=0, all=0, tile=4096, block=256, stack=32, tile_rows=8)
    bvh.dispose()
