"""Batched meshes on the GPU: one persistent launch over many BVHs (a BatchedMesh's bounds trees,
ExtensionUtilities.js:216-268) against per-geometry oracles, the per-mesh launches and the CUDA
graph replay."""
import numpy as np
import pytest

from parity import check_first, tie_exempt

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene(pkg, orc, cuda):
    import torch

    from three_mesh_bvh_b200.batched import BatchedMeshBVH

    geoms, _, rays, off = pkg.batched_scene(n_geometries=24, tri_range=(200, 20_000), ray_range=(100, 5_000), seed=5)
    batch = BatchedMeshBVH(geoms, {"strategy": pkg.SAH}, threads=4)
    d_rays = torch.from_numpy(rays).to(cuda)
    return batch, rays, off, d_rays


def _oracle_mesh(orc, batch, k):
    r0 = sum(batch.roots_per_mesh[:k])
    roots = batch.roots[r0:r0 + batch.roots_per_mesh[k]]
    return orc.OracleBVH.from_serialized(roots, batch.index, None, batch.position)


def _hits(t):
    return t.cpu().numpy().view(np.uint8).reshape(-1).view(
        np.dtype([("face_index", "<u4"), ("distance", "<f4"), ("point", "<f4", 3), ("barycoord", "<f4", 3)]))


@pytest.mark.parametrize("cfg,leaf", [((1, 1, 16, 0, 0), 0), ((1, 0, 32, 1, 1), 0), ((0, 1, 16, 0, 0), 0),
                                      ((1, 1, 8, 2, 1), 0), ((1, 1, 32, 2, 1, 0, 0, 1), 0),
                                      ((1, 1, 16, 1, 0, 0, 0, 1), 0), ((1, 1, 16, 2, 1, 0, 0, 1), 4),
                                      ((1, 1, 16, 2, 1), 2)])
def test_batched_matches_oracle_per_geometry(orc, scene, cfg, leaf):
    """Each geometry's rays against its own oracle, for the persistent launch over child pairs and
    over four-child records (the 8th field, wide), with and without compaction, per ray, and on
    split-leaf layouts."""
    batch, rays, off, d_rays = scene
    batch.set_leaf_size(leaf)
    batch.set_traversal(*cfg)
    got = _hits(batch.raycast_first(d_rays, off))
    batch.synchronize()
    for k in range(batch.n_meshes):
        a, b = int(off[k]), int(off[k + 1])
        ref = _oracle_mesh(orc, batch, k)
        exp = ref.raycast_first(rays[a:b])
        ac, ah = ref.raycast_all(rays[a:b], cap=64)
        rep = check_first(got[a:b], exp, tie_exempt(ac, ah))
        bad = {x: rep[x] for x in ("hitmiss", "face", "distance", "point", "barycoord") if rep[x]}
        assert not bad, (k, rep)
    batch.set_leaf_size(0)


def test_per_mesh_launches_and_graph_agree(scene, cuda):
    import torch

    batch, rays, off, d_rays = scene
    batch.set_traversal(1, 1, 16, 0)
    one = _hits(batch.raycast_first(d_rays, off))
    per = _hits(batch.raycast_first_per_mesh(d_rays, off))
    out = torch.empty((rays.shape[0], 8), dtype=torch.float32, device=cuda)
    graph = batch.capture(d_rays, off, out)
    for _ in range(2):
        out.fill_(0)
        graph.launch(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(_hits(out).view(np.uint8), one.view(np.uint8))
    batch.synchronize()
    assert np.array_equal(per.view(np.uint8), one.view(np.uint8))
