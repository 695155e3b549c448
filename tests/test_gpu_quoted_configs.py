"""Parity on the workloads the benchmark numbers are quoted on, at their full sizes.

* The 2,000,000-triangle noisy torus knot (TorusKnot(10,3,2000,500) + N(0,0.02) along the tube
  normal, seed 1; SAH, maxLeafSize 10, maxDepth 40) with its two ray sets: 2^24 incoherent rays
  and a 4096^2 pinhole camera.  The engine traces each whole set, as the benchmark does (ray
  ordering and the warp-shared forms depend on the whole set's coherence); the oracle checks an
  evenly strided 2^18-ray sample of each set for every traversal variant the autotuner can pick,
  on every device leaf layout it tries, and the whole of both sets for the variant it picks.
* raycast (all hits, cap 64) on the same sets: every all-hits kernel, the stored hits of a strided
  2^18-ray sample of each set in the oracle's order (raycast.template.js:37-49).
* The 80,000-triangle knot (TorusKnot(10,3,400,100)) with its full 1,000,000-ray set (seed 0): every
  variant traces the whole set, a strided quarter is checked per variant and the whole set for
  the default variant and the host-memory path.
* closestPointToPoint on the 256^3 grid over that knot's box padded by 10%, maxThreshold 5: every
  kernel (and the tiled query orders) on the whole grid, byte-identical across them, a strided
  2^20-query sample against the oracle.

Tolerances are tests/parity.py's (faceIndex / hit-miss identical except 1e-6 t ties; distance,
point, barycentrics within 1e-5 relative; closest-point distance within 1e-5 relative).
"""
import math
import os

import numpy as np
import pytest

from parity import FIRST_KEYS, check_all, check_closest, check_first, first_parity, tie_exempt

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1
HIT = np.dtype([("face_index", "<u4"), ("distance", "<f4"), ("point", "<f4", 3), ("barycoord", "<f4", 3)])
CLOSEST = np.dtype([("face_index", "<u4"), ("distance", "<f4"), ("point", "<f4", 3)])
ALL_ROWS = np.dtype([("face_index", "<i4"), ("distance", "<f8")])


def _rows(t, dtype):
    """A torch tensor of fixed-size records on the device -> numpy structured rows on the host."""
    return np.frombuffer(t.contiguous().cpu().numpy().tobytes(), dtype=dtype)


def _zero(rep, keys=FIRST_KEYS):
    return {k: rep[k] for k in keys if rep[k]}


class SampleOracle:
    """The oracle's raycastFirst on a fixed ray sample, with tie exemptions computed once per ray
    on demand (only rays whose hit/miss or faceIndex differ need the all-hits row)."""

    def __init__(self, ref, rays):
        self.ref, self.rays = ref, np.ascontiguousarray(rays)
        self.exp = ref.raycast_first(self.rays, threads=THREADS)
        self.known = np.zeros(self.rays.shape[0], dtype=bool)
        self.exempt = np.zeros(self.rays.shape[0], dtype=bool)

    def check(self, got):
        with np.errstate(invalid="ignore"):
            gh, eh = got["face_index"] != 0xFFFFFFFF, self.exp["face_index"] >= 0
            differ = (gh != eh) | (gh & eh & (got["face_index"].astype(np.int64) != self.exp["face_index"]))
        need = np.nonzero(differ & ~self.known)[0]
        if need.size:
            ac, ah = self.ref.raycast_all(np.ascontiguousarray(self.rays[need]), cap=64, threads=THREADS)
            self.exempt[need] = tie_exempt(ac, ah)
            self.known[need] = True
        return check_first(got, self.exp, self.exempt)


# ------------------------------------------------------------------------------------------
# 2M-triangle knot, both ray sets
# ------------------------------------------------------------------------------------------

@pytest.fixture(scope="module")
def knot2m(pkg, orc, cuda):
    import torch

    geo = pkg.torus_knot(10, 3, 2000, 500, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "maxLeafSize": 10, "maxDepth": 40})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
    sets = {"incoherent": pkg.rays_incoherent(1 << 24, seed=1), "camera": pkg.rays_camera(4096, 4096)}
    dev = {k: torch.from_numpy(v).to(cuda) for k, v in sets.items()}
    stride = 64
    samples = {k: SampleOracle(ref, v[::stride]) for k, v in sets.items()}
    yield geo, bvh, ref, sets, dev, samples, stride
    bvh.dispose()


def _first_sample(bvh, d, stride):
    import torch

    out = bvh.raycast_first_batch(d)
    bvh.synchronize()
    idx = torch.arange(0, d.shape[0], stride, device=d.device)
    return _rows(out.index_select(0, idx), HIT)


def _stage2(cands):
    """The autotuner's stage-2 forms of its stage-1 candidates: threads per block 64 / 256 for the
    warp-cooperative form over child pairs, its tiled order's other tile heights (2, 8 rows), the
    persistent form's refill thresholds 8 / 24, and the 32-entry stack for both forms."""
    out = []
    for c in cands:
        if c[0] == 2 and not c[7]:
            out += [c[:10] + [64, 0, 0], c[:10] + [256, 32, 0], c[:10] + [0, 32, 0]]
            if c[9] and c[9] % 16 == 0:
                out += [c[:10] + [0, 32, 2], c[:10] + [0, 0, 8]]
        elif c[0] == 1:
            out += [c[:10] + [0, 32, 0], [c[0], c[1], 8] + c[3:10] + [0, 0, 0], [c[0], c[1], 24] + c[3:10] + [0, 32, 0]]
    return out


@pytest.mark.parametrize("leaf", [0, 2, 4])
def test_knot2m_first_hit_every_variant(knot2m, leaf):
    from three_mesh_bvh_b200 import autotune

    geo, bvh, ref, sets, dev, samples, stride = knot2m
    bvh.set_leaf_size(leaf)
    cands = autotune.candidates(tile_pitches=(4096, 2048))
    cands += _stage2([c for c in cands if c[3] == 2])
    bad = {}
    for cand in cands:
        bvh.set_traversal(*cand)
        for name, d in dev.items():
            rep = samples[name].check(_first_sample(bvh, d, stride))
            if _zero(rep):
                bad[(name, cand)] = rep
    bvh.set_leaf_size(0)
    assert not bad, bad
    for name, s in samples.items():
        assert (s.exp["face_index"] >= 0).sum() > (0.02 if name == "incoherent" else 0.3) * s.rays.shape[0]


def test_knot2m_first_hit_tuned_whole_sets(knot2m):
    """The autotuner's pick (as the benchmark runs it: leaf layouts 0, 2, 4; one variant per set),
    then every ray of both sets against the oracle."""
    from three_mesh_bvh_b200 import autotune

    geo, bvh, ref, sets, dev, samples, stride = knot2m
    res = autotune.tune_raycast_first_sets(bvh, list(dev.items()), leaf_sizes=[0, 2, 4], tag="parity-knot2M",
                                           tile_pitches=(4096,))
    for name, d in dev.items():
        bvh.set_traversal(*res["sets"][name]["best"])
        got = _rows(bvh.raycast_first_batch(d), HIT)
        bvh.synchronize()
        rep = first_parity(ref, sets[name], got, threads=THREADS)
        assert not _zero(rep), (name, res["leaf"], res["sets"][name]["best"], rep)
        assert rep["rays"] == sets[name].shape[0]
    bvh.set_leaf_size(0)


@pytest.fixture(scope="module")
def knot2m_all_rows(knot2m):
    """The oracle's all-hits rows (cap 64) for a strided 2^18-ray sample of each set."""
    geo, bvh, ref, sets, dev, samples, stride = knot2m
    rows = {}
    for name, r in sets.items():
        sub = np.ascontiguousarray(r[::64])
        counts = np.empty(sub.shape[0], dtype=np.int64)
        hits = np.empty((sub.shape[0], 64), dtype=ALL_ROWS)
        for c0 in range(0, sub.shape[0], 1 << 15):
            c, h = ref.raycast_all(sub[c0:c0 + (1 << 15)], cap=64, threads=THREADS)
            counts[c0:c0 + c.shape[0]] = c
            hits[c0:c0 + c.shape[0]]["face_index"] = h["face_index"]
            hits[c0:c0 + c.shape[0]]["distance"] = h["distance"]
        rows[name] = (counts, hits)
    return rows


@pytest.mark.parametrize("variant", list(range(13)) + ["1t"])
def test_knot2m_all_hits_every_variant(knot2m, knot2m_all_rows, cuda, variant):
    """Cap 64 (no ray of these sets has more front-face hits) and cap 2 (rays with more hits than
    the cap keep the first two of the reference's order)."""
    import torch

    geo, bvh, ref, sets, dev, samples, stride = knot2m
    bvh.set_leaf_size(0)
    if variant == "1t":   # the warp-cooperative kernel in tiled order (the camera's row pitch)
        bvh.set_traversal(1, 1, 16, 2, 0, 0, 0, 0, 1, 4096)
    else:
        bvh.set_traversal(1, 1, 16, 2, 0, 0, 0, 0, variant)
    for name, d in dev.items():
        ec, eh = knot2m_all_rows[name]
        idx = torch.arange(0, d.shape[0], 64, device=cuda)
        for cap in (64, 2):
            counts, hits = bvh.raycast_batch(d, cap=cap)
            bvh.synchronize()
            gc = counts.index_select(0, idx).cpu().numpy()
            gh = _rows(hits.index_select(0, idx), HIT).reshape(-1, cap)
            del counts, hits
            rep = check_all(gc, gh, ec, eh[:, :cap])
            assert rep["count"] == 0 and rep["set"] == 0 and rep["distance"] == 0, (name, variant, cap, rep)
            if name == "camera" and cap == 2:
                assert rep["over_cap"] > 1000, rep
    bvh.set_traversal(1, 1, 16, 0, 0, 0, 0, 0, 0)


# ------------------------------------------------------------------------------------------
# 80k-triangle knot: the full 1,000,000-ray set and the 256^3 closest-point grid
# ------------------------------------------------------------------------------------------

@pytest.fixture(scope="module")
def knot80k_full(pkg, orc, cuda):
    geo = pkg.torus_knot(10, 3, 400, 100)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH, "maxLeafSize": 10, "maxDepth": 40})
    ref = orc.OracleBVH.from_serialized(bvh._roots, geo.index, bvh._indirectBuffer, geo.position)
    yield geo, bvh, ref
    bvh.dispose()


def test_knot80k_million_rays_every_variant(knot80k_full, cuda):
    import torch

    from three_mesh_bvh_b200 import autotune

    geo, bvh, ref = knot80k_full
    rays = __import__("__graft_entry__").load_package().rays_sphere_to_box(1_000_000, seed=0)
    assert rays.shape[0] == 1_000_000
    oracle = SampleOracle(ref, rays)
    quarter = SampleOracle(ref, rays[::4])
    d = torch.from_numpy(rays).to(cuda)
    idx = torch.arange(0, d.shape[0], 4, device=cuda)
    bad = {}
    for leaf in (0, 2, 4):
        bvh.set_leaf_size(leaf)
        # tiled orders of any row pitch (a multiple of 8) are permutations: still every ray's own hit
        cands = autotune.candidates(tile_pitches=(8, 1000, 4096))
        for cand in cands + _stage2(cands):
            bvh.set_traversal(*cand)
            out = bvh.raycast_first_batch(d)
            bvh.synchronize()
            rep = quarter.check(_rows(out.index_select(0, idx), HIT))
            if _zero(rep):
                bad[(leaf, cand)] = rep
    bvh.set_leaf_size(0)
    bvh.set_traversal(1, 1, 16, 0, 0, 0, 0, 0, 0)
    rep = oracle.check(_rows(bvh.raycast_first_batch(d), HIT))
    assert not _zero(rep), rep
    # the host-memory path (chunked over streams) on the whole set
    host = bvh.raycast_first_batch(rays)
    rep = oracle.check(host)
    assert not bad, bad
    assert not _zero(rep), rep
    assert (oracle.exp["face_index"] >= 0).mean() > 0.2


def test_knot80k_closest_point_grid256(knot80k_full, orc, cuda):
    import torch

    geo, bvh, ref = knot80k_full
    pkg = __import__("__graft_entry__").load_package()
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 256)
    assert pts.shape[0] == 1 << 24
    d = torch.from_numpy(pts).to(cuda)
    results = {}
    forms = {0: {}, 1: {}, 2: {}, 3: {}, 4: {}, 5: {}, 6: {}, "1t2": dict(tile=256, tile_rows=2), "1t4": dict(tile=256),
             "1t8": dict(tile=256, tile_rows=8), "3t4": dict(tile=256), "3t8": dict(tile=256, tile_rows=8),
             "5t4": dict(tile=256)}
    for name, kw in forms.items():
        bvh.set_traversal(1, 1, 16, 2, 0, 0, int(str(name)[0]), **kw)
        results[name] = bvh.closest_point_batch(d, 0.0, 5.0).contiguous().view(torch.int32).clone()
        bvh.synchronize()
    # raycastFirst's split-leaf layouts leave closest point on the reference's leaves
    for leaf in (2, 4):
        bvh.set_leaf_size(leaf)
        for name in (2, "1t4"):
            bvh.set_traversal(1, 1, 16, 2, 0, 0, int(str(name)[0]), **forms[name])
            results[f"{name}@leaf{leaf}"] = bvh.closest_point_batch(d, 0.0, 5.0).contiguous().view(torch.int32).clone()
            bvh.synchronize()
    bvh.set_leaf_size(0)
    bvh.set_traversal(1, 1, 16, 0, 0, 0, 0)
    # every kernel and query order gives the same bytes on every query (exact distance ties go to
    # the smaller faceIndex, whatever the traversal order)
    for name in results:
        assert torch.equal(results[name], results[0]), name
    # results beyond maxThreshold: leaves whose box is within it but whose triangles are not
    dist = results[0].view(torch.float32)[:, 1]
    assert int(((dist > 5.0) & torch.isfinite(dist)).sum()) > 1000
    stride = 16
    idx = np.arange(0, pts.shape[0], stride)
    got = _rows(results[2][::stride], CLOSEST)
    exp = ref.closest_point(np.ascontiguousarray(pts[idx]), 0.0, 5.0, threads=THREADS)

    def tri_distance(i, face):
        q = orc.closest_point_triangle(pts[idx[i]].astype(np.float64), *geo.triangle(face))
        return float(np.linalg.norm(q - pts[idx[i]].astype(np.float64)))

    rep = check_closest(got, exp, tri_distance)
    assert rep["null"] == 0 and rep["distance"] == 0 and rep["face"] == 0, rep
    assert (exp["face_index"] >= 0).mean() > 0.1 and (exp["face_index"] < 0).mean() > 0.01
    assert math.isfinite(float(exp["distance"][exp["face_index"] >= 0].max()))
