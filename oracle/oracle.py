"""ctypes wrapper of liboracle.so — TEST INFRASTRUCTURE ONLY.

The oracle is a float64 CPU restatement of three-mesh-bvh's build and query path (oracle.cpp).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the checker.
"""
from __future__ import annotations

import ctypes as C
import math
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

HIT_DTYPE = np.dtype([("face_index", "<i8"), ("distance", "<f8"), ("point", "<f8", 3), ("barycoord", "<f8", 3),
                      ("normal", "<f8", 3), ("face", "<i8", 3), ("material_index", "<i8")])
CP_DTYPE = np.dtype([("face_index", "<i8"), ("distance", "<f8"), ("point", "<f8", 3)])

_lib = None


def build() -> Path:
    src = HERE / "oracle.cpp"
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        P, I64, I = C.c_void_p, C.c_int64, C.c_int
        D = C.c_double
        L.orc_build.restype = P
        L.orc_build.argtypes = [P, I64, I, P, I64, I, P, I, I64, I64, I, I, I, I]
        L.orc_from_serialized.restype = P
        L.orc_from_serialized.argtypes = [P, P, I, P, I64, P, I64, P, I64, I]
        L.orc_free.argtypes = [P]
        L.orc_num_roots.argtypes = [P]
        L.orc_root_bytes.restype = I64
        L.orc_root_bytes.argtypes = [P, I]
        L.orc_copy_root.argtypes = [P, I, P]
        L.orc_index_elem_bytes.argtypes = [P]
        L.orc_index_count.restype = I64
        L.orc_index_count.argtypes = [P]
        L.orc_copy_index.argtypes = [P, P]
        L.orc_indirect_elem_bytes.argtypes = [P]
        L.orc_indirect_count.restype = I64
        L.orc_indirect_count.argtypes = [P]
        L.orc_copy_indirect.argtypes = [P, P]
        L.orc_raycast_first.argtypes = [P, P, I64, I, D, D, P, P, P, I]
        L.orc_raycast_all.argtypes = [P, P, I64, I, D, D, I, P, P, P, P, I]
        L.orc_closest_point.argtypes = [P, P, I64, D, D, P, P, P, I]
        L.orc_brute_raycast_all.argtypes = [P, P, I64, I, D, D, I, P, P, I]
        L.orc_ray_triangle.restype = I
        L.orc_ray_triangle.argtypes = [P, P, P, P, P, I, D, D, P]
        L.orc_closest_point_triangle.argtypes = [P, P, P, P, P]
        L.orc_stats.argtypes = [P, P]
        L.orc_set_materials.argtypes = [P, P, I, P, I]
        L.orc_ray_triangle_jacobian.argtypes = [P, P, P, P, P, P, P]
        L.orc_point_triangle_distance.restype = D
        L.orc_point_triangle_distance.argtypes = [P, P, P, P]
        L.orc_refit.argtypes = [P, P, I64, I]
        L.orc_intersects_sphere.argtypes = [P, P, I64, P, P, P, I]
        L.orc_intersects_box.argtypes = [P, P, I64, P, P, P, I]
        L.orc_sphere_triangles.argtypes = [P, P, I64, I, P, P, P, P, I]
        L.orc_scene_raycast_first.argtypes = [P, I, P, P, P, P, I64, I, D, D, P, P, I]
        L.orc_scene_raycast_all.argtypes = [P, I, P, P, P, P, I64, I, D, D, I, P, P, P, I]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data if a is not None else None


def _threads():
    import os
    return os.cpu_count() or 1


class OracleBVH:
    """A reference-semantics BVH: built by the restated builder, or adopted from serialized data."""

    def __init__(self, handle):
        self.h = handle

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    @classmethod
    def build(cls, position, index=None, groups=(), draw_range=(0, math.inf), strategy=2, max_depth=40,
              target_leaf=10, indirect=False):
        pos = np.ascontiguousarray(position, dtype=np.float32).reshape(-1, 3)
        idx = None if index is None else np.ascontiguousarray(index).astype(np.uint32)
        elem = 0 if index is None else np.asarray(index).dtype.itemsize
        g = np.array([[s, -1 if (isinstance(c, float) and math.isinf(c)) else c] for s, c, *_ in groups],
                     dtype=np.int64).reshape(-1)
        dc = -1 if math.isinf(draw_range[1]) else int(draw_range[1])
        h = lib().orc_build(_p(pos), pos.shape[0], 3, _p(idx), 0 if idx is None else idx.size, elem,
                            _p(g) if g.size else None, len(groups), int(draw_range[0]), dc, strategy, max_depth,
                            target_leaf, 1 if indirect else 0)
        if not h:
            raise RuntimeError("oracle build failed")
        return cls(h)

    @classmethod
    def from_serialized(cls, roots, index, indirect, position):
        pos = np.ascontiguousarray(position, dtype=np.float32).reshape(-1, 3)
        bufs = [np.frombuffer(bytes(r), dtype=np.uint8) for r in roots]
        ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
        sizes = (C.c_int64 * len(bufs))(*[b.size for b in bufs])
        idx = None if index is None else np.ascontiguousarray(index).astype(np.uint32)
        ind = None if indirect is None else np.ascontiguousarray(indirect).astype(np.uint32)
        h = lib().orc_from_serialized(ptrs, sizes, len(bufs), _p(idx), 0 if idx is None else idx.size, _p(ind),
                                      0 if ind is None else ind.size, _p(pos), pos.shape[0], 3)
        obj = cls(h)
        obj._keep = (bufs, idx, ind, pos)
        return obj

    def set_materials(self, groups, sides):
        """Material-array raycasts: groups [(start, count, materialIndex)], one side per material."""
        g = np.array([[s, -1 if (isinstance(c, float) and math.isinf(c)) else c, m] for s, c, m in groups],
                     dtype=np.int64).reshape(-1)
        sd = np.asarray(sides, dtype=np.int32)
        self._mat = (g, sd)
        lib().orc_set_materials(self.h, _p(g) if g.size else None, len(groups), _p(sd) if sd.size else None, sd.size)

    def intersects_sphere(self, spheres, threads=None, counters=False):
        """MeshBVH#intersectsSphere for each row (cx, cy, cz, radius) -> bool array."""
        sp = np.ascontiguousarray(spheres, dtype=np.float32).reshape(-1, 4)
        n = sp.shape[0]
        out = np.empty(n, dtype=np.uint8)
        nn = np.empty(n, dtype=np.int64) if counters else None
        nt = np.empty(n, dtype=np.int64) if counters else None
        lib().orc_intersects_sphere(self.h, _p(sp), n, _p(out), _p(nn), _p(nt), threads or _threads())
        return (out.astype(bool), nn, nt) if counters else out.astype(bool)

    def sphere_triangles(self, spheres, cap=256, threads=None, counters=False):
        """Triangles within each sphere (cx, cy, cz, r) through shapecast's CONTAINED path: counts
        and the first `cap` triangle indices in traversal order (-1 past the count); with counters,
        also the boxes read and the triangles tested one by one per sphere."""
        sp = np.ascontiguousarray(spheres, dtype=np.float32).reshape(-1, 4)
        n = sp.shape[0]
        counts = np.empty(n, dtype=np.int32)
        faces = np.empty((n, cap), dtype=np.int64)
        nn = np.empty(n, dtype=np.int64) if counters else None
        nt = np.empty(n, dtype=np.int64) if counters else None
        lib().orc_sphere_triangles(self.h, _p(sp), n, cap, _p(counts), _p(faces), _p(nn), _p(nt),
                                   threads or _threads())
        return (counts, faces, nn, nt) if counters else (counts, faces)

    def intersects_box(self, boxes, threads=None, counters=False):
        """MeshBVH#intersectsBox for each row of 24 float32 (min xyz, pad, max xyz, pad, the
        column-major box-to-mesh matrix) -> bool array."""
        bx = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 24)
        n = bx.shape[0]
        out = np.empty(n, dtype=np.uint8)
        nn = np.empty(n, dtype=np.int64) if counters else None
        nt = np.empty(n, dtype=np.int64) if counters else None
        lib().orc_intersects_box(self.h, _p(bx), n, _p(out), _p(nn), _p(nt), threads or _threads())
        return (out.astype(bool), nn, nt) if counters else out.astype(bool)

    def refit(self, position):
        """MeshBVH#refit() after the vertex positions changed to `position` (n x 3 float32)."""
        pos = np.ascontiguousarray(position, dtype=np.float32).reshape(-1, 3)
        lib().orc_refit(self.h, _p(pos), pos.shape[0], 3)

    def roots(self):
        L = lib()
        out = []
        for i in range(L.orc_num_roots(self.h)):
            b = np.empty(L.orc_root_bytes(self.h, i), dtype=np.uint8)
            L.orc_copy_root(self.h, i, _p(b))
            out.append(b.tobytes())
        return out

    def index(self):
        L = lib()
        eb = L.orc_index_elem_bytes(self.h)
        if eb == 0:
            return None
        a = np.empty(L.orc_index_count(self.h), dtype=np.uint32)
        L.orc_copy_index(self.h, _p(a))
        return a.astype(np.uint16 if eb == 2 else np.uint32)

    def indirect(self):
        L = lib()
        eb = L.orc_indirect_elem_bytes(self.h)
        if eb == 0:
            return None
        a = np.empty(L.orc_indirect_count(self.h), dtype=np.uint32)
        L.orc_copy_indirect(self.h, _p(a))
        return a.astype(np.uint16 if eb == 2 else np.uint32)

    def stats(self):
        s = np.zeros(4, dtype=np.int64)
        lib().orc_stats(self.h, _p(s))
        return dict(nodes=int(s[0]), leaves=int(s[1]), max_depth=int(s[2]), leaf_triangles=int(s[3]))

    def raycast_first(self, rays, side=0, near=0.0, far=math.inf, threads=None, counters=False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        out = np.empty(n, dtype=HIT_DTYPE)
        nn = np.empty(n, dtype=np.int64) if counters else None
        nt = np.empty(n, dtype=np.int64) if counters else None
        lib().orc_raycast_first(self.h, _p(rays), n, side, near, far, _p(out), _p(nn), _p(nt), threads or _threads())
        return (out, nn, nt) if counters else out

    def raycast_all(self, rays, side=0, near=0.0, far=math.inf, cap=64, threads=None, counters=False):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        counts = np.empty(n, dtype=np.int32)
        hits = np.empty((n, cap), dtype=HIT_DTYPE)
        nn = np.empty(n, dtype=np.int64) if counters else None
        nt = np.empty(n, dtype=np.int64) if counters else None
        lib().orc_raycast_all(self.h, _p(rays), n, side, near, far, cap, _p(counts), _p(hits), _p(nn), _p(nt),
                              threads or _threads())
        return (counts, hits, nn, nt) if counters else (counts, hits)

    def brute_raycast_all(self, rays, side=0, near=0.0, far=math.inf, cap=64, threads=None):
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        counts = np.empty(n, dtype=np.int32)
        hits = np.empty((n, cap), dtype=HIT_DTYPE)
        lib().orc_brute_raycast_all(self.h, _p(rays), n, side, near, far, cap, _p(counts), _p(hits),
                                    threads or _threads())
        return counts, hits

    def closest_point(self, points, min_t=0.0, max_t=math.inf, threads=None, counters=False):
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        n = pts.shape[0]
        out = np.empty(n, dtype=CP_DTYPE)
        nn = np.empty(n, dtype=np.int64) if counters else None
        nt = np.empty(n, dtype=np.int64) if counters else None
        lib().orc_closest_point(self.h, _p(pts), n, min_t, max_t, _p(out), _p(nn), _p(nt), threads or _threads())
        return (out, nn, nt) if counters else out


def ray_triangle(o, d, a, b, c, side=0, near=0.0, far=math.inf):
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (o, d, a, b, c)]
    out = np.zeros(1, dtype=HIT_DTYPE)
    hit = lib().orc_ray_triangle(*[_p(x) for x in arrs], side, near, far, _p(out))
    return out[0] if hit else None


def ray_triangle_jacobian(o, d, a, b, c):
    """(values, jacobian): values = (distance, t, wa, wb, wc) of the ray/triangle formula in float64,
    jacobian (5, 15) = their partials w.r.t. (a, b, c, o, d), from forward-mode dual numbers."""
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (o, d, a, b, c)]
    vals = np.zeros(5)
    jac = np.zeros((5, 15))
    lib().orc_ray_triangle_jacobian(*[_p(x) for x in arrs], _p(vals), _p(jac))
    return vals, jac


def point_triangle_distance(p, a, b, c):
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (p, a, b, c)]
    return lib().orc_point_triangle_distance(*[_p(x) for x in arrs])


def closest_point_triangle(p, a, b, c):
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (p, a, b, c)]
    out = np.zeros(3)
    lib().orc_closest_point_triangle(*[_p(x) for x in arrs], _p(out))
    return out


def scene_raycast_first(geoms, geometry, matrices, rays, visible=None, side=0, near=0.0, far=math.inf, threads=None):
    """Instanced raycastFirst (acceleratedBatchedMeshRaycast with firstHitOnly): geoms a list of
    OracleBVH (one per geometry), geometry the geometry of each instance, matrices (n x 16,
    column-major float64 world matrices), rays (m x 6 float32, world space).  Returns the world-space
    hits (HIT_DTYPE, barycoord and face_index local) and the hit instance (-1: none)."""
    gs = (C.c_void_p * len(geoms))(*[g.h for g in geoms])
    geo = np.ascontiguousarray(geometry, dtype=np.uint32)
    mats = np.ascontiguousarray(matrices, dtype=np.float64).reshape(-1, 16)
    vis = None if visible is None else np.ascontiguousarray(visible, dtype=np.uint8)
    r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
    out = np.empty(r.shape[0], dtype=HIT_DTYPE)
    inst = np.empty(r.shape[0], dtype=np.int64)
    lib().orc_scene_raycast_first(gs, mats.shape[0], _p(geo), _p(mats), _p(vis), _p(r), r.shape[0], side, near, far,
                                  _p(out), _p(inst), threads or _threads())
    return out, inst


def scene_raycast_all(geoms, geometry, matrices, rays, visible=None, side=0, near=0.0, far=math.inf, cap=64,
                      threads=None):
    """Instanced raycast (all hits): per ray the total count, and the first `cap` world-space hits
    by distance (stable: instance order, then DFS order) with their instances (-1 past the count)."""
    gs = (C.c_void_p * len(geoms))(*[g.h for g in geoms])
    geo = np.ascontiguousarray(geometry, dtype=np.uint32)
    mats = np.ascontiguousarray(matrices, dtype=np.float64).reshape(-1, 16)
    vis = None if visible is None else np.ascontiguousarray(visible, dtype=np.uint8)
    r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
    counts = np.empty(r.shape[0], dtype=np.int32)
    hits = np.empty((r.shape[0], cap), dtype=HIT_DTYPE)
    inst = np.empty((r.shape[0], cap), dtype=np.int64)
    lib().orc_scene_raycast_all(gs, mats.shape[0], _p(geo), _p(mats), _p(vis), _p(r), r.shape[0], side, near, far,
                                cap, _p(counts), _p(hits), _p(inst), threads or _threads())
    return counts, hits, inst


def triangle_hit_point_info(points, faces, index, position, uv=None, groups=()):
    """getTriangleHitPointInfo(point, geometry, triangleIndex) (src/utils/TriangleUtilities.js:65-147)
    in float64 for each (point, faceIndex) pair: dict of a, b, c, materialIndex (first group whose
    [start, start + count) holds 3 * triangle, else 0, :80-93), normal ((c - b) x (a - b) made unit,
    zeros when its squared length is 0), barycoord (dot-product solve with v0 = c - a, v1 = b - a,
    v2 = p - a; zeros when the Gram determinant is exactly 0), uv (barycentric weights on the uv
    attribute; zeros for a degenerate triangle; None without uv).  Evaluation order is left to
    right, as the reference's Vector3 arithmetic."""
    p = np.asarray(points, dtype=np.float32).astype(np.float64).reshape(-1, 3)
    f = np.asarray(faces, dtype=np.int64).reshape(-1)
    idx = (np.asarray(index, dtype=np.int64).reshape(-1, 3) if index is not None
           else np.arange(np.asarray(position).shape[0], dtype=np.int64).reshape(-1, 3))
    pos = np.asarray(position, dtype=np.float32).astype(np.float64).reshape(-1, 3)
    va, vb, vc = idx[f, 0], idx[f, 1], idx[f, 2]
    A, B, C = pos[va], pos[vb], pos[vc]

    def dot(x, y):
        return x[:, 0] * y[:, 0] + x[:, 1] * y[:, 1] + x[:, 2] * y[:, 2]

    def cross(x, y):
        return np.stack([x[:, 1] * y[:, 2] - x[:, 2] * y[:, 1], x[:, 2] * y[:, 0] - x[:, 0] * y[:, 2],
                         x[:, 0] * y[:, 1] - x[:, 1] * y[:, 0]], 1)

    v0, v1, v2 = C - A, B - A, p - A
    d00, d01, d02, d11, d12 = dot(v0, v0), dot(v0, v1), dot(v0, v2), dot(v1, v1), dot(v1, v2)
    denom = d00 * d11 - d01 * d01
    ok = denom != 0
    inv = np.where(ok, 1.0 / np.where(ok, denom, 1.0), 0.0)
    u = (d11 * d02 - d01 * d12) * inv
    v = (d00 * d12 - d01 * d02) * inv
    bary = np.where(ok[:, None], np.stack([1.0 - u - v, v, u], 1), 0.0)
    n = cross(C - B, A - B)
    l2 = dot(n, n)
    pos_l = l2 > 0
    normal = np.where(pos_l[:, None], n * (1.0 / np.sqrt(np.where(pos_l, l2, 1.0)))[:, None], 0.0)
    mat = np.zeros(f.shape[0], dtype=np.int64)
    found = np.zeros(f.shape[0], dtype=bool)
    first = 3 * f
    for start, count, material in groups:
        end = math.inf if count is None or count < 0 or math.isinf(count) else start + count
        hit = ~found & (first >= start) & (first < end)
        mat[hit] = material
        found |= hit
    out = {"a": va, "b": vb, "c": vc, "materialIndex": mat, "normal": normal, "barycoord": bary, "uv": None}
    if uv is not None:
        t = np.asarray(uv, dtype=np.float32).astype(np.float64).reshape(-1, 2)
        w = bary
        out["uv"] = np.where(ok[:, None], t[va] * w[:, 0:1] + t[vb] * w[:, 1:2] + t[vc] * w[:, 2:3], 0.0)
    return out
