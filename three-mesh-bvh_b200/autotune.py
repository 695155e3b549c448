"""Autotuner for the traversal kernels.

For a mesh and a representative ray batch already on the device, each candidate traversal
variant (persistent warps with lane refill, warp-cooperative traversal or one ray per thread,
child visiting order, refill threshold, register budget, compaction and ray-ordering key) is timed with CUDA events on the launching stream after a warm-up launch, and the
fastest is installed on the mesh.  Results are cached per (GPU name, triangle-count bucket,
workload tag), in memory and optionally in a JSON file, so a serving process tunes once per
mesh class.  Every variant returns the same hits (up to exact ties), so tuning never changes
results, only speed.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

# (persistent, order, refill, occupancy, compact, sort, closest, wide): one ray per thread;
# warp-cooperative traversal over child pairs (wide 0; order 0 / 1) or four-child records (wide 1);
# persistent warps with lane refill.  compact / sort select the root-box compaction pass and the
# Morton-key ray ordering (0 none, 1 direction, 2 entry point, 3 entry point + direction); closest
# is closestPointToPoint's kernel and is tuned separately (tune_closest_point).
_QUEUE = [(0, 0), (1, 0), (1, 1), (1, 2), (1, 3)]
CANDIDATES = [(0, 0, 16, 0, 0, 0, 0, 0), (0, 1, 16, 0, 0, 0, 0, 0)] + [
    (2, order, 16, occ, c, s, 0, 0) for order in (0, 1) for occ in (0, 1, 2) for c, s in _QUEUE] + [
    (2, 1, 16, occ, c, s, 0, 1) for occ in (0, 1, 2) for c, s in _QUEUE] + [
    (1, order, refill, occ, c, s, 0, 0) for order in (0, 1) for refill in (16, 32) for occ in (1, 2)
    for c, s in _QUEUE]

_cache: dict = {}


def _key(bvh, tag: str) -> str:
    import torch

    tris = bvh.mesh_info()["triangle_records"]
    bucket = int(math.log2(max(tris, 1)))
    return f"{torch.cuda.get_device_name()}|tri2^{bucket}|{tag}"


def tune_raycast_first(bvh, rays, side: int = 0, near: float = 0.0, far: float = math.inf, tag: str = "default",
                       reps: int = 3, cache_file: str | Path | None = None, candidates=CANDIDATES) -> dict:
    """Time every candidate on `rays` (torch CUDA tensor, n x 6) and install the fastest."""
    import torch

    key = _key(bvh, tag)
    if cache_file is not None and not _cache:
        p = Path(cache_file)
        if p.exists():
            _cache.update(json.loads(p.read_text()))
    if key in _cache:
        best = _cache[key]["best"]
        bvh.set_traversal(*best)
        return _cache[key]
    stream = torch.cuda.current_stream(rays.device)
    out = torch.empty((rays.shape[0], 8), dtype=torch.float32, device=rays.device)
    timings = {}
    for cand in candidates:
        bvh.set_traversal(*cand)
        bvh.raycast_first_batch(rays, side, near, far, out=out, stream=stream.cuda_stream)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            bvh.raycast_first_batch(rays, side, near, far, out=out, stream=stream.cuda_stream)
        end.record(stream)
        end.synchronize()
        timings[str(list(cand))] = start.elapsed_time(end) / reps
    bvh.synchronize(stream.cuda_stream)
    best = min(candidates, key=lambda c: timings[str(list(c))])
    bvh.set_traversal(*best)
    entry = {"best": list(best), "ms": timings[str(list(best))], "timings_ms": timings, "rays": int(rays.shape[0])}
    _cache[key] = entry
    if cache_file is not None:
        Path(cache_file).write_text(json.dumps(_cache, indent=1))
    return entry


def tune_raycast_all(bvh, rays, cap: int = 64, reps: int = 3, candidates=tuple(range(13))) -> dict:
    """Time raycast's (all hits) kernels (the `all` field: per ray, warp-cooperative,
    warp-cooperative over rays sorted by the direction / entry-point / entry-point-and-direction
    key, one ray per thread over the rays that enter the tree, in ray order or sorted by each key,
    and the same with persistent warps)
    on `rays` (torch CUDA tensor,
    n x 6), keeping the mesh's other traversal fields, and install the fastest."""
    import torch

    cur = bvh.get_traversal()
    stream = torch.cuda.current_stream(rays.device)
    out = (torch.empty(rays.shape[0], dtype=torch.int32, device=rays.device),
           torch.empty((rays.shape[0], cap, 8), dtype=torch.float32, device=rays.device))
    timings = {}
    for c in candidates:
        bvh.set_traversal(**{**cur, "all": c})
        bvh.raycast_batch(rays, cap=cap, stream=stream.cuda_stream, out=out)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            bvh.raycast_batch(rays, cap=cap, stream=stream.cuda_stream, out=out)
        end.record(stream)
        end.synchronize()
        timings[c] = start.elapsed_time(end) / reps
    bvh.synchronize(stream.cuda_stream)
    best = min(candidates, key=lambda c: timings[c])
    bvh.set_traversal(**{**cur, "all": best})
    return {"best": best, "timings_ms": {str(k): v for k, v in timings.items()}}


def tune_closest_point(bvh, points, min_t: float = 0.0, max_t: float = math.inf, reps: int = 3,
                       candidates=(0, 1, 2)) -> dict:
    """Time closestPointToPoint's kernels (the `closest` field: per query, warp-cooperative,
    warp-cooperative over Morton-sorted queries) on `points` (torch CUDA tensor, n x 3), keeping
    the mesh's other traversal fields, and install the fastest."""
    import torch

    cur = bvh.get_traversal()
    stream = torch.cuda.current_stream(points.device)
    out = torch.empty((points.shape[0], 5), dtype=torch.float32, device=points.device)
    timings = {}
    for c in candidates:
        bvh.set_traversal(**{**cur, "closest": c})
        bvh.closest_point_batch(points, min_t, max_t, out=out, stream=stream.cuda_stream)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            bvh.closest_point_batch(points, min_t, max_t, out=out, stream=stream.cuda_stream)
        end.record(stream)
        end.synchronize()
        timings[c] = start.elapsed_time(end) / reps
    bvh.synchronize(stream.cuda_stream)
    best = min(candidates, key=lambda c: timings[c])
    bvh.set_traversal(**{**cur, "closest": best})
    return {"best": best, "timings_ms": {str(k): v for k, v in timings.items()}}


def tune_raycast_first_sets(bvh, named_rays, leaf_sizes=(0,), tag: str = "default", **kw) -> dict:
    """Tune several ray sets that share one mesh: the device leaf layout (bvh.set_leaf_size; one
    layout serves every set) is chosen by the sum of the sets' best times, and each set keeps its
    own traversal variant for that layout.  named_rays: [(name, rays)].  Leaves the chosen layout
    installed and returns {"leaf": L, "sets": {name: entry}, "total_ms": {L: ms}}."""
    per_leaf, totals = {}, {}
    for leaf in leaf_sizes:
        bvh.set_leaf_size(leaf)
        per_leaf[leaf] = {name: tune_raycast_first(bvh, rays, tag=f"{tag}-{name}-leaf{leaf}", **kw)
                          for name, rays in named_rays}
        totals[leaf] = sum(e["ms"] for e in per_leaf[leaf].values())
    leaf = min(totals, key=totals.get)
    bvh.set_leaf_size(leaf)
    return {"leaf": leaf, "sets": per_leaf[leaf], "total_ms": {str(k): v for k, v in totals.items()}}
