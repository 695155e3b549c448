"""GPU refit (bvhc_mesh_refit) against the oracle's restatement of MeshBVH#refit: the read-back
serialized roots are byte-identical, and every query kind matches the oracle on the refit BVH."""
import math

import numpy as np
import pytest

from parity import check_all, check_closest, check_first, tie_exempt
from refit_util import validate_bounds

pytestmark = pytest.mark.gpu


def _oracle(orc, bvh, geo, roots=None):
    return orc.OracleBVH.from_serialized(roots or bvh._roots, geo.index, bvh._indirectBuffer, geo.position)


def _queries_match(pkg, orc, bvh, geo, ref):
    rays = np.concatenate([pkg.rays_sphere_to_box(40_000, seed=3), pkg.rays_camera(128, 128)])
    ac, ah = ref.raycast_all(rays, cap=64)
    check = check_first(bvh.raycast_first_batch(rays), ref.raycast_first(rays), tie_exempt(ac, ah))
    assert all(check[k] == 0 for k in ("hitmiss", "face", "distance", "point", "barycoord")), check
    counts, hits = bvh.raycast_batch(rays[:20_000], cap=64)
    rep = check_all(counts, hits, ac[:20_000], ah[:20_000])
    assert rep["count"] == 0 and rep["set"] == 0, rep
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 20)

    def tri_distance(i, face):
        t = geo.triangle(face)
        q = orc.closest_point_triangle(pts[i].astype(np.float64), *t)
        return float(np.linalg.norm(q - pts[i].astype(np.float64)))

    rep = check_closest(bvh.closest_point_batch(pts, 0.0, 2.0), ref.closest_point(pts, 0.0, 2.0), tri_distance)
    assert rep["null"] == 0 and rep["distance"] == 0 and rep["face"] == 0, rep


@pytest.mark.parametrize("indirect", [False, True])
def test_refit_matches_reference_rule(pkg, orc, cuda, indirect):
    geo = pkg.torus_knot(10, 3, 200, 40)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "indirect": indirect})
    ref = _oracle(orc, bvh, geo)
    rng = np.random.default_rng(7)
    # 1) every vertex moves
    pos = (geo.position + rng.normal(0, 0.05, geo.position.shape)).astype(np.float32)
    bvh.refit(pos)
    ref.refit(pos)
    assert bvh._roots == ref.roots()
    assert validate_bounds(bvh._roots, pos, geo.index, bvh._indirectBuffer)
    _queries_match(pkg, orc, bvh, geo, ref)
    # 2) a few vertices move: only their paths are rewritten (the reference's change rule)
    pos2 = pos.copy()
    pos2[rng.choice(pos.shape[0], 5, replace=False)] += np.float32(0.3)
    bvh.refit(pos2)
    ref.refit(pos2)
    assert bvh._roots == ref.roots()
    _queries_match(pkg, orc, bvh, geo, ref)
    # 3) nothing moves: nothing changes
    before = list(bvh._roots)
    bvh.refit(pos2)
    assert bvh._roots == before
    bvh.dispose()


def test_refit_from_device_positions_with_split_leaves_and_gradients(pkg, orc, cuda):
    """Device-memory positions; raycastFirst's split-leaf copy is refit too; the backward uses the
    refit vertices."""
    import torch

    geo = pkg.torus_knot(10, 3, 160, 32, noise_sigma=0.02, noise_seed=2)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = _oracle(orc, bvh, geo)
    bvh.set_leaf_size(3)
    bvh.set_traversal(2, 1, 16, 2, 1, 1)
    bvh._gradients_ready()   # the gradient vertex copy is taken now, from the old positions
    pos = (geo.position * np.float32(1.5) + np.float32(0.25)).astype(np.float32)
    bvh.refit(torch.from_numpy(pos).to(cuda))
    ref.refit(pos)
    assert bvh._roots == ref.roots()
    geo.position = pos
    _queries_match(pkg, orc, bvh, geo, ref)
    rays = pkg.rays_camera(64, 64, distance=55.0)
    d_rays = torch.from_numpy(rays).to(cuda)
    hits = bvh.raycast_first_batch(d_rays)
    g = torch.ones(rays.shape[0], dtype=torch.float32, device=cuda)
    gv, _, _ = bvh.raycast_first_backward(d_rays, hits, g)
    bvh.synchronize()
    rec = hits.cpu().numpy().view(np.uint8).reshape(-1).view(pkg.HIT_DTYPE)
    i = int(np.nonzero(rec["face_index"] != 0xFFFFFFFF)[0][0])
    f = int(rec["face_index"][i])
    ids = geo.index[3 * f:3 * f + 3].astype(np.int64)
    _, jac = orc.ray_triangle_jacobian(rays[i, :3], rays[i, 3:], *pos[ids].astype(np.float64))
    only = np.zeros(rays.shape[0], dtype=np.float32)
    only[i] = 1.0
    gv1, _, _ = bvh.raycast_first_backward(d_rays, hits, torch.from_numpy(only).to(cuda))
    bvh.synchronize()
    got = gv1.cpu().numpy()[ids].reshape(-1)
    assert np.abs(got - jac[0][:9]).max() <= 1e-3 * np.abs(jac[0][:9]).max()
    assert math.isfinite(float(gv.sum()))
    bvh.dispose()
