"""Parity checks of GPU results against the oracle, with the tolerances of the engine's contract:

* raycastFirst: hit/miss and faceIndex bit-identical, except rays whose two nearest reference
  hits lie within 1e-6 * t of each other (TIE_REL); distance within 1e-5 relative; point and
  barycoord within 1e-5 * max(1, |reference|) (components near zero make a pure relative test
  meaningless).
* raycast (all hits): identical uncapped counts, and each ray's stored hits in the oracle's order
  (the reference's left-then-right DFS order, raycast.template.js:37-49): the same faceIndex
  sequence, which also decides which hits are kept when a ray has more than `cap`; distances
  within 1e-5 relative, position by position.
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


@np.errstate(invalid="ignore")
def check_all(counts, hits, exp_counts, exp_hits):
    """All-hits rows against the oracle's, in stored order.  `set` counts rays whose stored
    faceIndex sequence differs from the oracle's (a different order counts), `distance` rays whose
    distances differ beyond REL at some position."""
    n = exp_counts.shape[0]
    cap = hits.shape[1]
    ec = exp_counts.astype(np.int64)
    gc = counts.astype(np.int64)
    bad_count = int((gc != ec).sum())
    es, gs = np.minimum(ec, cap), np.minimum(gc, cap)
    pos = np.arange(cap)[None, :] < es[:, None]
    gf = hits["face_index"].astype(np.int64)
    if hits["face_index"].dtype == np.uint32:
        gf = np.where(gf == NO_HIT, -1, gf)
    ef = exp_hits["face_index"][:, :cap].astype(np.int64)
    seq = (es != gs) | (pos & (gf != ef)).any(1)
    de = exp_hits["distance"][:, :cap]
    dd = pos & (np.abs(hits["distance"].astype(np.float64) - de) > REL * np.abs(de))
    bad_dist = (~seq & dd.any(1))
    return dict(count=bad_count, set=int((seq & (ec > 0)).sum()), distance=int(bad_dist.sum()),
                over_cap=int((ec > cap).sum()), rays=n)


FIRST_KEYS = ("hitmiss", "face", "distance", "point", "barycoord")


def first_parity_chunk(ref, rays, got, exp, side=0, near=0.0, far=np.inf, threads=None):
    """check_first of the engine's rows `got` against the oracle's `exp` for the same rays; the
    oracle's all-hits rows (tie exemption) are computed only for the rays whose hit/miss or
    faceIndex differ."""
    with np.errstate(invalid="ignore"):
        gh, eh = got["face_index"] != NO_HIT, exp["face_index"] >= 0
        differ = (gh != eh) | (gh & eh & (got["face_index"].astype(np.int64) != exp["face_index"]))
    exempt = np.zeros(rays.shape[0], dtype=bool)
    idx = np.nonzero(differ)[0]
    if idx.size:
        ac, ah = ref.raycast_all(np.ascontiguousarray(rays[idx]), side, near, far, cap=64, threads=threads)
        exempt[idx] = tie_exempt(ac, ah)
    return check_first(got, exp, exempt)


def add_counts(tot, rep):
    for k, v in rep.items():
        tot[k] = tot.get(k, 0) + v
    return tot


def first_parity(ref, rays, got, side=0, near=0.0, far=np.inf, threads=None, chunk=1 << 21):
    """check_first over a large ray set in chunks (the oracle's raycastFirst per chunk).  `got` is
    the engine's bvhc_hit rows (HIT_DTYPE) for the same rays.  Returns summed counts."""
    tot = {}
    for c0 in range(0, rays.shape[0], chunk):
        sub = np.ascontiguousarray(rays[c0:c0 + chunk])
        exp = ref.raycast_first(sub, side, near, far, threads=threads)
        add_counts(tot, first_parity_chunk(ref, sub, got[c0:c0 + chunk], exp, side, near, far, threads))
    return tot


def all_parity(ref, rays, counts, hits, side=0, near=0.0, far=np.inf, threads=None, chunk=1 << 16):
    """check_all over a ray set in chunks (the oracle's all-hits rows, cap = hits.shape[1])."""
    cap = hits.shape[1]
    tot = dict(count=0, set=0, distance=0, over_cap=0, rays=0)
    for c0 in range(0, rays.shape[0], chunk):
        sub = np.ascontiguousarray(rays[c0:c0 + chunk])
        ec, eh = ref.raycast_all(sub, side, near, far, cap=cap, threads=threads)
        rep = check_all(counts[c0:c0 + chunk], hits[c0:c0 + chunk], ec, eh)
        for k in tot:
            tot[k] += rep[k]
    return tot


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
