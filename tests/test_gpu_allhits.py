"""raycast (all hits) kernel variants against the oracle: the counts, and each ray's stored hits
in the reference's order (left child before right child), for one ray per thread, the
warp-cooperative form, and the warp-cooperative form over rays sorted by each ray key (direction,
entry point, entry point and direction)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant,occupancy", [(0, 0), (1, 0), (1, 2), (2, 2), (3, 2), (4, 0), (5, 0), (6, 0), (8, 0), (9, 0), (11, 0)])
def test_all_hits_variants_keep_reference_order(pkg, orc, cuda, variant, occupancy):
    import torch

    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=4)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
    bvh.set_traversal(1, 1, 16, occupancy, 0, 0, 0, 0, variant)
    assert bvh.get_traversal()["all"] == variant
    rays = np.concatenate([pkg.rays_camera(160, 160), pkg.rays_incoherent(40_000, seed=8),
                           pkg.rays_sphere_to_box(20_000, seed=9)])
    for side, near, far, cap in ((0, 0.0, math.inf, 64), (2, 0.0, math.inf, 8), (2, 30.0, 45.0, 64)):
        counts, hits = bvh.raycast_batch(rays, side, near, far, cap=cap)
        ec, eh = ref.raycast_all(rays, side, near, far, cap=cap)
        assert np.array_equal(counts.astype(np.int64), ec.astype(np.int64))
        stored = np.minimum(ec, cap)
        for i in np.nonzero(stored)[0]:
            k = int(stored[i])
            got_faces = hits[i, :k]["face_index"].astype(np.int64)
            assert np.array_equal(got_faces, eh[i, :k]["face_index"].astype(np.int64))
            d = np.abs(hits[i, :k]["distance"].astype(np.float64) - eh[i, :k]["distance"])
            assert (d <= 1e-5 * np.maximum(eh[i, :k]["distance"], 1e-3)).all()
    d_rays = torch.from_numpy(rays).to(cuda)
    dc, dh = bvh.raycast_batch(d_rays, 0, cap=64)
    bvh.synchronize()
    hc, hh = bvh.raycast_batch(rays, 0, cap=64)
    assert np.array_equal(dc.cpu().numpy(), hc)
    bvh.dispose()
