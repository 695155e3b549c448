"""Parity checks of GPU results against the oracle, with the tolerances of the engine's contract:

* raycastFirst: hit/miss and faceIndex bit-identical, except rays whose two nearest reference
  hits lie within 1e-6 * t of each other (TIE_REL); distance within 1e-5 relative; point and
  barycoord within 1e-5 * max(1, |reference|) (components near zero make a pure relative test
  meaningless).
* raycast (all hits): identical uncapped counts, identical faceIndex sets for stored hits.
* closestPointToPoint: null results identical; distance within 1e-5 relative (1e-5 * 1e-3
  absolute floor for queries on the surface); faceIndex identical unless the GPU's triangle is
  at the same float64 distance within 1e-5 relative (a tie).
"""
import numpy as np

NO_HIT = 0xFFFFFFFF
TIE_REL = 1e-6
REL = 1e-5


def tie_exempt(all_counts, all_hits):
    """Rays whose two nearest reference hits lie within TIE_REL * t of each other."""
    n = all_counts.shape[0]
    ex = np.zeros(n, dtype=bool)
    d = np.where(np.arange(all_hits.shape[1])[None, :] < all_counts[:, None], all_hits["distance"], np.inf)
    d.sort(axis=1)
    if d.shape[1] >= 2:
        ex = np.isfinite(d[:, 1]) & (d[:, 1] - d[:, 0] <= TIE_REL * d[:, 0])
    return ex


@np.errstate(invalid="ignore")
def check_first(got, exp, exempt=None):
    """Returns a dict of mismatch counts (all zero when the parity bar is met)."""
    n = exp.shape[0]
    exempt = np.zeros(n, dtype=bool) if exempt is None else exempt
    gh = got["face_index"] != NO_HIT
    eh = exp["face_index"] >= 0
    hitmiss = (gh != eh) & ~exempt
    both = gh & eh
    face = both & (got["face_index"].astype(np.int64) != exp["face_index"]) & ~exempt
    ok = both & ~face & ~exempt
    dist = ok & (np.abs(got["distance"] - exp["distance"]) > REL * np.abs(exp["distance"]))
    pscale = np.maximum(1.0, np.linalg.norm(exp["point"], axis=1))
    point = ok & (np.abs(got["point"] - exp["point"]).max(1) > REL * pscale)
    bscale = np.maximum(1.0, np.abs(exp["barycoord"]))
    bary = ok & (np.abs(got["barycoord"] - exp["barycoord"]) > REL * bscale).any(1)
    return dict(hitmiss=int(hitmiss.sum()), face=int(face.sum()), distance=int(dist.sum()), point=int(point.sum()),
                barycoord=int(bary.sum()), exempt=int(exempt.sum()), hits=int(eh.sum()), rays=n)


def check_all(counts, hits, exp_counts, exp_hits):
    n = exp_counts.shape[0]
    cap = hits.shape[1]
    bad_count = int((counts.astype(np.int64) != exp_counts.astype(np.int64)).sum())
    bad_set = 0
    bad_dist = 0
    for i in np.nonzero(exp_counts > 0)[0]:
        k = min(int(exp_counts[i]), cap)
        kg = min(int(counts[i]), cap)
        gs = np.sort(hits[i, :kg]["face_index"].astype(np.int64))
        es = np.sort(exp_hits[i, :k]["face_index"])
        if not np.array_equal(gs, es):
            bad_set += 1
            continue
        og = np.argsort(hits[i, :kg]["face_index"].astype(np.int64), kind="stable")
        oe = np.argsort(exp_hits[i, :k]["face_index"], kind="stable")
        dg = hits[i, :kg]["distance"][og]
        de = exp_hits[i, :k]["distance"][oe]
        bad_dist += int((np.abs(dg - de) > REL * np.abs(de)).any())
    return dict(count=bad_count, set=bad_set, distance=bad_dist, rays=n)


@np.errstate(invalid="ignore")
def check_closest(got, exp, tri_distance=None):
    """tri_distance(i, face) -> float64 distance from query i to triangle `face` (tie check)."""
    gh = got["face_index"] != NO_HIT
    eh = exp["face_index"] >= 0
    null = int((gh != eh).sum())
    both = gh & eh
    ed = exp["distance"]
    dist = both & (np.abs(got["distance"] - ed) > REL * np.maximum(ed, 1e-3))
    face_diff = both & (got["face_index"].astype(np.int64) != exp["face_index"])
    face = 0
    for i in np.nonzero(face_diff)[0]:
        if tri_distance is None:
            face += 1
            continue
        alt = tri_distance(i, int(got["face_index"][i]))
        if abs(alt - ed[i]) > REL * max(ed[i], 1e-3):
            face += 1
    return dict(null=null, distance=int(dist.sum()), face=face, face_ties=int(face_diff.sum()) - face,
                queries=int(exp.shape[0]))
