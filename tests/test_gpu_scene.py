"""Instanced raycastFirst on the GPU (bvhc_scene_*: a tree over instance world boxes, each
instance's geometry tree walked in its local frame) against the oracle's restatement of the
BatchedMesh raycast with firstHitOnly.  Hit/miss, instance and faceIndex agree except for rays
that graze an edge (the local ray is rounded to float32 once; the reference keeps it in float64)
or whose two closest world hits are within 1e-6 relative; distances and points within 1e-5
relative, barycoords within 1e-4."""
import numpy as np
import pytest

from scene_util import instance_matrices, world_rays

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch(pkg, cuda):
    from three_mesh_bvh_b200.batched import BatchedMeshBVH

    geoms, _, _, _ = pkg.batched_scene(n_geometries=16, tri_range=(200, 20_000), seed=7, make_rays=False)
    return BatchedMeshBVH(geoms, {"strategy": pkg.SAH}, threads=4)


def _oracles(orc, batch):
    out, r0 = [], 0
    for k in range(batch.n_meshes):
        roots = batch.roots[r0:r0 + batch.roots_per_mesh[k]]
        r0 += batch.roots_per_mesh[k]
        out.append(orc.OracleBVH.from_serialized(roots, batch.index, None, batch.position))
    return out


def _compare(got, ginst, exp, einst):
    ok_edge = lambda h: h["barycoord"].min() < 1e-4
    bad = []
    for i in range(exp.shape[0]):
        e_hit, g_hit = einst[i] >= 0, ginst[i] != 0xFFFFFFFF
        if e_hit != g_hit:
            if not ((e_hit and ok_edge(exp[i])) or (g_hit and ok_edge(got[i]))):
                bad.append(("hitmiss", i))
            continue
        if not e_hit:
            continue
        d = float(exp[i]["distance"])
        if abs(got[i]["distance"] - d) > 1e-5 * d:
            bad.append(("distance", i))
            continue
        if int(ginst[i]) != int(einst[i]) or int(got[i]["face_index"]) != int(exp[i]["face_index"]):
            if not (ok_edge(exp[i]) or ok_edge(got[i]) or abs(got[i]["distance"] - d) <= 1e-6 * d):
                bad.append(("face", i))
            continue
        scale = max(np.abs(exp[i]["point"]).max(), d)
        if np.abs(got[i]["point"] - exp[i]["point"]).max() > 1e-5 * scale:
            bad.append(("point", i))
        if np.abs(got[i]["barycoord"] - exp[i]["barycoord"]).max() > 1e-4:
            bad.append(("barycoord", i))
    return bad


@pytest.mark.parametrize("n_inst,scaled", [(1, False), (200, False), (400, True)])
def test_scene_matches_oracle(pkg, orc, batch, cuda, n_inst, scaled):
    import torch

    rng = np.random.default_rng(50 + n_inst)
    geometry, mats = instance_matrices(rng, n_inst, batch.n_meshes, spread=150.0 if n_inst > 1 else 0.0,
                                       scaled=scaled)
    visible = (rng.random(n_inst) > 0.1).astype(np.uint8) if n_inst > 1 else None
    rays = world_rays(rng, 12_000) if n_inst > 1 else world_rays(rng, 12_000, radius=40.0, half=13.0)
    scene = batch.instances(geometry, mats, visible)
    got, ginst = scene.raycast_first(rays)
    exp, einst = orc.scene_raycast_first(_oracles(orc, batch), geometry, mats, rays, visible=visible)
    bad = _compare(got, ginst, exp, einst)
    assert not bad, bad[:10]
    assert (einst >= 0).mean() > 0.2
    # device buffers, every ray order and every kernel variant give the same records
    for variant in (0, 1, 2):
        scene.set_variant(variant)
        for order in (0, 1, 2, 3, 4):
            scene.set_order(order)
            dh, di = scene.raycast_first(torch.from_numpy(rays).to(cuda))
            torch.cuda.synchronize()
            assert np.array_equal(di.cpu().numpy().view(np.uint32), ginst), (variant, order)
            assert np.array_equal(dh.cpu().numpy().view(np.uint8).reshape(-1), got.view(np.uint8).reshape(-1)), (
                variant, order)
    with pytest.raises(pkg.BVHCError):
        scene.set_variant(3)
    scene.set_variant(0)
    scene.set_order(0)
    # the geometries on split leaves of at most 4 triangles (the first-hit query walks
    # raycastFirst's records): the oracle's records again
    batch.set_leaf_size(4)
    got4, ginst4 = scene.raycast_first(rays)
    batch.set_leaf_size(0)
    bad = _compare(got4, ginst4, exp, einst)
    assert not bad, bad[:10]
    scene.dispose()


def test_scene_near_far_and_update(pkg, orc, batch, cuda):
    rng = np.random.default_rng(77)
    geometry, mats = instance_matrices(rng, 120, batch.n_meshes, scaled=True)
    rays = world_rays(rng, 6_000)
    scene = batch.instances(geometry, mats)
    oracles = _oracles(orc, batch)
    for near, far in ((0.0, 350.0), (250.0, float("inf")), (200.0, 420.0)):
        got, ginst = scene.raycast_first(rays, near=near, far=far)
        exp, einst = orc.scene_raycast_first(oracles, geometry, mats, rays, near=near, far=far)
        bad = _compare(got, ginst, exp, einst)
        assert not bad, (near, far, bad[:10])
    # move every instance, hide a third of them
    geometry2, mats2 = instance_matrices(rng, 90, batch.n_meshes, scaled=True)
    vis2 = (np.arange(90) % 3 != 0).astype(np.uint8)
    scene.set_instances(geometry2, mats2, vis2)
    got, ginst = scene.raycast_first(rays)
    exp, einst = orc.scene_raycast_first(oracles, geometry2, mats2, rays, visible=vis2)
    assert not _compare(got, ginst, exp, einst)
    assert not np.isin(ginst[ginst != 0xFFFFFFFF], np.nonzero(vis2 == 0)[0]).any()
    scene.dispose()


def test_scene_rejects_bad_input(pkg, batch, cuda):
    bad = np.eye(4).reshape(-1).copy()
    bad[3] = 0.5  # a perspective row: not affine
    with pytest.raises(Exception):
        batch.instances([0], bad[None, :])
    with pytest.raises(Exception):
        batch.instances([batch.n_meshes], np.eye(4).reshape(1, -1))


def test_scene_many_overlapping_instances(pkg, orc, batch, cuda):
    """100 copies of one geometry at the same place, rays starting inside every instance box: more
    candidates than one listing round holds, all entered at distance 0, and equal hit distances,
    which the lowest instance index wins (the raycaster's stable sort)."""
    rng = np.random.default_rng(91)
    n = 100
    geometry = np.zeros(n, dtype=np.uint32)
    mats = np.tile(np.eye(4).reshape(-1), (n, 1))
    rays = world_rays(rng, 4_000, radius=2.0, half=12.0)
    scene = batch.instances(geometry, mats)
    got, ginst = scene.raycast_first(rays)
    exp, einst = orc.scene_raycast_first(_oracles(orc, batch), geometry, mats, rays)
    assert not _compare(got, ginst, exp, einst)
    hit = ginst != 0xFFFFFFFF
    assert hit.mean() > 0.3 and (ginst[hit] == 0).all()
    # hiding the first instances moves every hit to the first visible one
    vis = (np.arange(n) >= 37).astype(np.uint8)
    scene.set_instances(geometry, mats, vis)
    got2, ginst2 = scene.raycast_first(rays)
    assert (ginst2[hit] == 37).all() and (ginst2[~hit] == 0xFFFFFFFF).all()
    assert np.array_equal(got2["face_index"], got["face_index"])
    scene.dispose()


def test_scene_all_hits_match_oracle(pkg, orc, batch, cuda):
    rng = np.random.default_rng(61)
    geometry, mats = instance_matrices(rng, 150, batch.n_meshes, scaled=True)
    vis = (rng.random(150) > 0.1).astype(np.uint8)
    rays = world_rays(rng, 6_000)
    scene = batch.instances(geometry, mats, vis)
    cap = 12
    counts, hits, inst = scene.raycast(rays, cap=cap)
    ec, eh, ei = orc.scene_raycast_all(_oracles(orc, batch), geometry, mats, rays, visible=vis, cap=cap)
    bad = 0
    for i in range(rays.shape[0]):
        if counts[i] != ec[i]:
            k = min(int(max(counts[i], ec[i])), cap)
            edge = (eh[i, :min(int(ec[i]), cap)]["barycoord"].min(initial=1) < 1e-4 or
                    hits[i, :min(int(counts[i]), cap)]["barycoord"].min(initial=1) < 1e-4)
            bad += 0 if edge else 1
            continue
        k = min(int(counts[i]), cap)
        d = eh[i, :k]["distance"]
        assert np.all(np.abs(hits[i, :k]["distance"] - d) <= 1e-5 * d), i
        same = (inst[i, :k].astype(np.int64) == ei[i, :k]) & (hits[i, :k]["face_index"].astype(np.int64) ==
                                                               eh[i, :k]["face_index"])
        if not same.all():  # equal distances can swap two hits
            for q in np.nonzero(~same)[0]:
                dd = d[q]
                assert (np.abs(d - dd) <= 1e-6 * dd).sum() > 1 or eh[i, q]["barycoord"].min() < 1e-4, (i, q)
        assert np.all(inst[i, k:] == 0xFFFFFFFF)
    assert bad == 0
    assert (ec > 1).mean() > 0.1
    # counts only
    c0, _, _ = scene.raycast(rays, cap=0)
    assert np.array_equal(c0, counts)
    scene.dispose()


def test_scene_host_pipeline(pkg, batch, cuda):
    """World rays through host memory in more than one pipeline chunk (2.5M rays: three 1M-ray
    chunks on three streams, the last partial) give exactly the device-memory call's records."""
    import torch

    rng = np.random.default_rng(77)
    geometry, mats = instance_matrices(rng, 300, batch.n_meshes, spread=150.0)
    scene = batch.instances(geometry, mats)
    rays = world_rays(rng, 2_500_000)
    got, ginst = scene.raycast_first(rays)
    dh, di = scene.raycast_first(torch.from_numpy(rays).to(cuda))
    torch.cuda.synchronize()
    assert np.array_equal(di.cpu().numpy().view(np.uint32), ginst)
    assert np.array_equal(dh.cpu().numpy().view(np.uint8).reshape(-1), got.view(np.uint8).reshape(-1))
    assert (ginst != 0xFFFFFFFF).mean() > 0.2
    scene.dispose()
