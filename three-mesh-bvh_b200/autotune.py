"""Autotuner for the traversal kernels.

raycastFirst is tuned by the library itself (bvhc_mesh_autotune: CUDA events on the launching
stream, stage 1 over every candidate variant and device leaf layout, stage 2 over threads per
block and traversal stack depth); this module is a thin caller of it with a cache per (GPU name,
triangle-count bucket, workload tag), in memory and optionally in a JSON file, so a serving
process tunes once per mesh class.  closestPointToPoint's and raycast's (all hits) kernels are
tuned here with torch CUDA events.  Every variant returns the same hits (up to exact ties), so
tuning never changes results, only speed.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from pathlib import Path

from . import _native as N

# Traversal config fields in bvhc_traversal_config order (the positional order of
# MeshBVH.set_traversal).
FIELDS = [name for name, _ in N.BvhcTraversalConfig._fields_]

_cache: dict = {}


def _as_list(cfg) -> list:
    return [int(getattr(cfg, f)) for f in FIELDS]


def candidates(tile_pitches=()) -> list:
    """bvhc_mesh_autotune's stage-1 candidates (as set_traversal argument lists) for these tiled-order
    row pitches."""
    tiles = (C.c_int32 * max(1, len(tile_pitches)))(*tile_pitches)
    n = N.lib().bvhc_autotune_candidates(tiles, len(tile_pitches), None, 0)
    if n < 0:
        raise ValueError("invalid tile pitches")
    out = (N.BvhcTraversalConfig * n)()
    N.lib().bvhc_autotune_candidates(tiles, len(tile_pitches), out, n)
    return [_as_list(c) for c in out]


def _key(bvh, tag: str) -> str:
    import torch

    tris = bvh.mesh_info()["triangle_records"]
    bucket = int(math.log2(max(tris, 1)))
    return f"{torch.cuda.get_device_name()}|tri2^{bucket}|{tag}"


def tune_raycast_first_sets(bvh, named_rays, leaf_sizes=(0,), tag: str = "default", tile_pitches=(), reps: int = 3,
                            side: int = 0, near: float = 0.0, far: float = math.inf,
                            cache_file: str | Path | None = None) -> dict:
    """Tune several ray sets that share one mesh through bvhc_mesh_autotune: the device leaf layout
    (one serves every set) is chosen by the sum of the sets' best times, and each set keeps its own
    traversal variant.  named_rays: [(name, rays)] with rays torch CUDA tensors (n x 6).  Leaves the
    chosen layout installed and returns {"leaf": L, "sets": {name: {"best": cfg, "ms": ms}},
    "total_ms": {L: ms}}."""
    import torch

    key = _key(bvh, tag)
    if cache_file is not None and not _cache:
        p = Path(cache_file)
        if p.exists():
            _cache.update(json.loads(p.read_text()))
    if key in _cache:
        entry = _cache[key]
        bvh.set_leaf_size(entry["leaf"])
        bvh.set_traversal(*entry["sets"][named_rays[0][0]]["best"])
        return entry
    k = len(named_rays)
    dev = named_rays[0][1].device
    ptrs = (C.c_void_p * k)(*[r.data_ptr() for _, r in named_rays])
    counts = (C.c_uint64 * k)(*[r.shape[0] for _, r in named_rays])
    leaves = (C.c_int32 * max(1, len(leaf_sizes)))(*leaf_sizes)
    tiles = (C.c_int32 * max(1, len(tile_pitches)))(*tile_pitches)
    best = (N.BvhcTraversalConfig * k)()
    best_ms = (C.c_float * k)()
    leaf_out = C.c_int32()
    totals = (C.c_float * max(1, len(leaf_sizes)))()
    stream = torch.cuda.current_stream(dev).cuda_stream
    N.check(N.lib().bvhc_mesh_autotune(bvh._device_mesh(), k, ptrs, counts, int(side), float(near), float(far), leaves,
                                       len(leaf_sizes), tiles, len(tile_pitches), int(reps), stream, best, best_ms,
                                       C.byref(leaf_out), totals), "bvhc_mesh_autotune")
    entry = {"leaf": int(leaf_out.value),
             "sets": {name: {"best": _as_list(best[j]), "ms": float(best_ms[j])} for j, (name, _) in enumerate(named_rays)},
             "total_ms": {str(leaf): float(totals[j]) for j, leaf in enumerate(leaf_sizes)}}
    _cache[key] = entry
    if cache_file is not None:
        Path(cache_file).write_text(json.dumps(_cache, indent=1))
    return entry


def tune_raycast_first(bvh, rays, tag: str = "default", **kw) -> dict:
    """One ray set (torch CUDA tensor, n x 6) on the mesh's current leaf layout; installs the fastest
    variant and returns {"best": cfg, "ms": ms}."""
    res = tune_raycast_first_sets(bvh, [("rays", rays)], leaf_sizes=(bvh.get_leaf_size(),), tag=tag, **kw)
    return res["sets"]["rays"]


def tune_raycast_all(bvh, rays, cap: int = 64, reps: int = 3, candidates=tuple(range(13))) -> dict:
    """Time raycast's (all hits) kernels (the `all` field: per ray, warp-cooperative,
    warp-cooperative over rays sorted by the direction / entry-point / entry-point-and-direction
    key, one ray per thread over the rays that enter the tree, in ray order or sorted by each key,
    and the same with persistent warps) on `rays` (torch CUDA tensor, n x 6), keeping the mesh's
    other traversal fields, and install the fastest."""
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
                       candidates=(0, 1, 2, 3, 4, 5, 6), tile_pitches=()) -> dict:
    """Time closestPointToPoint's kernels (the `closest` field: per query; warp-cooperative in
    input order and over Morton-sorted queries, with whole warps (1, 2), 16-lane (3, 4) or 8-lane
    (5, 6) groups; and each input-order form reading the queries in tiled order for each row length
    in `tile_pitches`, e.g. a grid's, with 2-, 4- and 8-row tiles) on `points` (torch CUDA tensor,
    n x 3), keeping the mesh's other traversal fields, and install the fastest.
    Returns {"best": name, "setting": fields, "timings_ms": ...}."""
    import torch

    cur = bvh.get_traversal()
    settings = {str(c): {"closest": c, "tile": 0, "tile_rows": 0} for c in candidates}
    for pitch in tile_pitches:
        for c in (c for c in candidates if c % 2 == 1):
            for rows in (2, 4, 8):
                if pitch % (32 // rows) == 0:
                    settings[f"{c}t{rows}@{pitch}"] = {"closest": c, "tile": pitch, "tile_rows": rows}
    stream = torch.cuda.current_stream(points.device)
    out = torch.empty((points.shape[0], 5), dtype=torch.float32, device=points.device)
    timings = {}
    for name, kw in settings.items():
        bvh.set_traversal(**{**cur, **kw})
        bvh.closest_point_batch(points, min_t, max_t, out=out, stream=stream.cuda_stream)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(reps):
            bvh.closest_point_batch(points, min_t, max_t, out=out, stream=stream.cuda_stream)
        end.record(stream)
        end.synchronize()
        timings[name] = start.elapsed_time(end) / reps
    bvh.synchronize(stream.cuda_stream)
    best = min(timings, key=timings.get)
    bvh.set_traversal(**{**cur, **settings[best]})
    return {"best": best, "setting": settings[best], "timings_ms": timings}
