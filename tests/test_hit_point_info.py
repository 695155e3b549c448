"""getTriangleHitPointInfo (src/utils/TriangleUtilities.js:65-147): the oracle against known
answers worked out by hand, and bvhc_triangle_hit_point_info against the oracle on closest-point
results, off-plane points and degenerate triangles, through host and device memory."""
import math

import numpy as np
import pytest


def test_oracle_known_answers(orc):
    # right triangle in z = 0: a = (0,0,0), b = (1,0,0), c = (0,1,0)
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 0], [1, 1, 1], [2, 2, 2]], np.float32)
    index = np.array([0, 1, 2, 3, 4, 5], np.uint32)
    uv = np.array([[0, 0], [1, 0], [0, 1], [5, 5], [6, 6], [7, 7]], np.float32)
    pts = np.array([[0.25, 0.25, 0.0], [0.25, 0.25, 3.0], [1.0, 0.0, 0.0], [1.0, 1.0, 1.0]], np.float32)
    faces = np.array([0, 0, 0, 1])
    r = orc.triangle_hit_point_info(pts, faces, index, pos, uv, groups=[(0, 3, 7), (3, math.inf, 9)])
    assert list(r["a"]) == [0, 0, 0, 3] and list(r["b"]) == [1, 1, 1, 4] and list(r["c"]) == [2, 2, 2, 5]
    assert list(r["materialIndex"]) == [7, 7, 7, 9]
    # barycoord (w_a, w_b, w_c) of (0.25, 0.25): 0.5, 0.25, 0.25; an off-plane point projects
    np.testing.assert_allclose(r["barycoord"][0], [0.5, 0.25, 0.25], rtol=0, atol=1e-15)
    np.testing.assert_allclose(r["barycoord"][1], [0.5, 0.25, 0.25], rtol=0, atol=1e-15)
    np.testing.assert_allclose(r["barycoord"][2], [0.0, 1.0, 0.0], rtol=0, atol=1e-15)
    # (c - b) x (a - b) = (-1, 1, 0) x (-1, 0, 0) = (0, 0, 1)
    np.testing.assert_array_equal(r["normal"][0], [0.0, 0.0, 1.0])
    np.testing.assert_allclose(r["uv"][0], [0.25, 0.25], rtol=0, atol=1e-15)
    # the collinear triangle (0,0,0), (1,1,1), (2,2,2): zero barycoord, uv and normal
    np.testing.assert_array_equal(r["barycoord"][3], [0.0, 0.0, 0.0])
    np.testing.assert_array_equal(r["normal"][3], [0.0, 0.0, 0.0])
    np.testing.assert_array_equal(r["uv"][3], [0.0, 0.0])
    # no group holds the triangle: materialIndex 0; the first matching group wins
    r = orc.triangle_hit_point_info(pts[:1], [1], index, pos, None, groups=[(0, 3, 4)])
    assert r["materialIndex"][0] == 0 and r["uv"] is None
    r = orc.triangle_hit_point_info(pts[:1], [1], index, pos, None, groups=[(0, 6, 4), (3, 3, 8)])
    assert r["materialIndex"][0] == 4


def _hpi_dtype():
    return np.dtype([("a", np.uint32), ("b", np.uint32), ("c", np.uint32), ("material_index", np.uint32),
                     ("normal", np.float32, 3), ("barycoord", np.float32, 3), ("uv", np.float32, 2)])


def _compare(got, want):
    for k in ("a", "b", "c", "materialIndex"):
        assert np.array_equal(got[k].astype(np.int64), want[k]), k
    for k in ("normal", "barycoord", "uv"):
        if want[k] is None:
            assert got[k] is None
            continue
        # float32 rounding of the float64 result (barycoord against max(1, |ref|))
        err = np.abs(got[k].astype(np.float64) - want[k]) / np.maximum(1.0, np.abs(want[k]))
        assert err.max() <= 1e-5, (k, np.unravel_index(err.argmax(), err.shape))


@pytest.mark.gpu
def test_hit_point_info_matches_oracle(pkg, orc, cuda):
    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=5)
    rng = np.random.default_rng(41)
    geo.uv = rng.random((geo.position.shape[0], 2)).astype(np.float32)
    n_tri = geo.triangle_count
    third = 3 * (n_tri // 3)
    geo.groups = [(0, third, 2), (third, third, 5), (2 * third, math.inf, 1)]
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    lo, hi = geo.position.min(0), geo.position.max(0)
    q = (lo + rng.random((20_000, 3)) * (hi - lo)).astype(np.float32)
    res = bvh.closest_point_batch(q, 0.0, math.inf)
    pts = np.ascontiguousarray(res["point"], dtype=np.float32)
    faces = res["face_index"].astype(np.uint32)
    # plus random faces with points off their plane
    f2 = rng.integers(0, n_tri, 5000).astype(np.uint32)
    p2 = (lo + rng.random((5000, 3)) * (hi - lo)).astype(np.float32)
    pts, faces = np.concatenate([pts, p2]), np.concatenate([faces, f2])
    want = orc.triangle_hit_point_info(pts, faces, geo.index, geo.position, geo.uv, geo.groups)
    got = bvh.triangle_hit_point_info_batch(pts, faces)
    _compare(got, want)
    assert len(set(want["materialIndex"].tolist())) == 3
    single = bvh.getTriangleHitPointInfo(pts[0], int(faces[0]))
    assert single["face"]["a"] == int(want["a"][0])
    assert single["face"]["materialIndex"] == int(want["materialIndex"][0])
    np.testing.assert_allclose(single["barycoord"], want["barycoord"][0], rtol=0, atol=1e-5)

    # device memory through the C ABI
    import torch

    lib = pkg.lib()
    d_pts, d_faces = torch.from_numpy(pts).to(cuda), torch.from_numpy(faces.astype(np.int32)).to(cuda)
    d_pos, d_uv = torch.from_numpy(geo.position).to(cuda), torch.from_numpy(geo.uv).to(cuda)
    d_out = torch.empty((pts.shape[0], 12), dtype=torch.int32, device=cuda)   # 48-byte records
    grp = np.array([[s, -1 if math.isinf(c) else c, m] for s, c, m in geo.groups], np.int64).reshape(-1)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    st = lib.bvhc_triangle_hit_point_info(bvh._device_mesh(), d_pts.data_ptr(), d_faces.data_ptr(), pts.shape[0],
                                          d_pos.data_ptr(), 3, d_uv.data_ptr(), 2, geo.position.shape[0],
                                          grp.ctypes.data, len(geo.groups), d_out.data_ptr(), 1, stream)
    assert st == 0
    torch.cuda.synchronize()
    rec = d_out.cpu().numpy().view(_hpi_dtype()).reshape(-1)
    dev = {"a": rec["a"], "b": rec["b"], "c": rec["c"], "materialIndex": rec["material_index"],
           "normal": rec["normal"], "barycoord": rec["barycoord"], "uv": rec["uv"]}
    _compare(dev, want)
    bvh.dispose()


@pytest.mark.gpu
def test_hit_point_info_degenerate_and_errors(pkg, orc, cuda):
    from three_mesh_bvh_b200._native import BVHCError

    # a regular triangle, a collinear one and one with two equal vertices; no uv attribute
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 2], [2, 2, 3],
                    [0.1, 0.2, 0.3], [0.1, 0.2, 0.3], [1.0, 0.5, 0.25]], np.float32)
    geo = pkg.Geometry(pos, np.arange(9, dtype=np.uint32))
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    rng = np.random.default_rng(43)
    pts = rng.uniform(-1, 3, (300, 3)).astype(np.float32)
    faces = np.tile(np.arange(3, dtype=np.uint32), 100)
    want = orc.triangle_hit_point_info(pts, faces, geo.index, geo.position, None, geo.groups)
    got = bvh.triangle_hit_point_info_batch(pts, faces)
    _compare(got, want)
    assert np.all(want["barycoord"][faces == 1] == 0) and np.all(want["normal"][faces == 2] == 0)
    with pytest.raises(BVHCError):
        bvh.triangle_hit_point_info_batch(pts[:1], [3])
    bvh.dispose()
