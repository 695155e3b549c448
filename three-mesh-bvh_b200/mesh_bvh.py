"""`MeshBVH` — the reference's query interface, answered by the GPU engine.

Mirrors src/core/MeshBVH.js (three-mesh-bvh 0.9.14): the constructor builds a BVH over a
`Geometry` (reordering its index in place, as the reference does), `serialize` / `deserialize`
move the packed roots in and out, and `raycastFirst`, `raycast` and `closestPointToPoint` keep
the reference's argument meaning, defaults and null / empty results.  Every query runs on the
GPU through libbvhcuda; the batched forms (`raycast_first_batch`, ...) are the engine's
purpose and take whole arrays of rays or points, as numpy arrays (host) or torch CUDA tensors
(device-resident, enqueued on the current stream).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N
from .geometry import Geometry

FrontSide, BackSide, DoubleSide = N.FRONT_SIDE, N.BACK_SIDE, N.DOUBLE_SIDE
CENTER, AVERAGE, SAH = N.CENTER, N.AVERAGE, N.SAH
DEFAULT_OPTIONS = dict(strategy=CENTER, maxDepth=40, targetLeafSize=10, indirect=False, range=None,
                       setBoundingBox=True, verbose=True)   # Constants.js:74-85

HIT_DTYPE = np.dtype([("face_index", "<u4"), ("distance", "<f4"), ("point", "<f4", 3), ("barycoord", "<f4", 3)])
CLOSEST_DTYPE = np.dtype([("face_index", "<u4"), ("distance", "<f4"), ("point", "<f4", 3)])
assert HIT_DTYPE.itemsize == 32 and CLOSEST_DTYPE.itemsize == 20


@dataclass
class Face:
    a: int
    b: int
    c: int
    normal: np.ndarray
    materialIndex: int = 0


@dataclass
class Intersection:
    distance: float
    point: np.ndarray
    face: Face
    faceIndex: int
    barycoord: np.ndarray
    # vertex attributes at the hit point (ThreeRayIntersectUtilities.js:59-117), when the geometry
    # has them; `normal` faces against the ray
    uv: np.ndarray | None = None
    uv1: np.ndarray | None = None
    normal: np.ndarray | None = None


@dataclass
class HitPointInfo:
    point: np.ndarray = field(default_factory=lambda: np.zeros(3))
    distance: float = 0.0
    faceIndex: int = -1


def _side_of(material_or_side) -> int:
    """getSide (ThreeRayIntersectUtilities.js:147-151): a material's `side`, or the side itself."""
    side = getattr(material_or_side, "side", material_or_side)
    if side not in (FrontSide, BackSide, DoubleSide):
        raise ValueError(f"unsupported side {material_or_side!r}")
    return int(side)


def _material_sides(materials) -> np.ndarray | None:
    """An array of materials as `materialOrSide` (ThreeRayIntersectUtilities.js:170-205) -> int8
    side per material; None for a single material or side."""
    if isinstance(materials, (list, tuple)):
        return np.array([_side_of(m) for m in materials], dtype=np.int8)
    return None


# bvhc_hit_point_info as a numpy record
_HPI_DTYPE = np.dtype([("a", np.uint32), ("b", np.uint32), ("c", np.uint32), ("material_index", np.uint32),
                       ("normal", np.float32, 3), ("barycoord", np.float32, 3), ("uv", np.float32, 2)])


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class MeshBVH:
    """GPU-backed MeshBVH (src/core/MeshBVH.js:80-886)."""

    def __init__(self, geometry: Geometry, options: dict | None = None, *, device: int = 0, _skip_build=False):
        opts = dict(DEFAULT_OPTIONS)
        opts.update(options or {})
        if "maxLeafSize" in opts:       # BVH.js:76-84 deprecated alias
            opts["targetLeafSize"] = opts.pop("maxLeafSize")
        if "maxLeafTris" in opts:       # MeshBVH.js:262-270 deprecated alias
            opts["targetLeafSize"] = opts.pop("maxLeafTris")
        self.geometry = geometry
        self.device = device
        self._roots: list[bytes] = []
        self._indirectBuffer: np.ndarray | None = None
        self._mesh = None
        if not _skip_build:
            self._build(opts)

    # -- build -----------------------------------------------------------------------------
    def _build(self, opts):
        lib = N.lib()
        g = self.geometry
        pos = np.ascontiguousarray(g.position, dtype=np.float32)
        idx = g.index
        rng = opts.get("range")
        start, count = (rng if rng is not None else g.draw_range)
        count = -1 if count is None or (isinstance(count, float) and math.isinf(count)) else int(count)
        groups = np.array([[s, -1 if (isinstance(c, float) and math.isinf(c)) else int(c)] for s, c, *_ in g.groups],
                          dtype=np.int64).reshape(-1)
        out = C.c_void_p()
        args = (_ptr(pos), pos.shape[0], 3, _ptr(idx) if idx is not None else None,
                idx.dtype.itemsize if idx is not None else 0, idx.size if idx is not None else 0,
                _ptr(groups) if groups.size else None, len(g.groups), int(start), count,
                int(opts["strategy"]), int(opts["maxDepth"]), int(opts["targetLeafSize"]),
                1 if opts.get("indirect") else 0)
        if opts.get("deviceBuild"):
            # the same tree built on the GPU (SAH / CENTER), byte-identical serialized output
            st = lib.bvhc_build_device(*args, int(self.device), None, C.byref(out))
            N.check(st, "bvhc_build_device")
        else:
            st = lib.bvhc_build(*args, C.byref(out))
            N.check(st, "bvhc_build")
        try:
            self._adopt_serialized(out)
        finally:
            lib.bvhc_serialized_free(out)

    def _adopt_serialized(self, s):
        lib = N.lib()
        roots = []
        for i in range(lib.bvhc_serialized_root_count(s)):
            p, n = C.c_void_p(), C.c_uint64()
            N.check(lib.bvhc_serialized_root(s, i, C.byref(p), C.byref(n)), "bvhc_serialized_root")
            roots.append(C.string_at(p, n.value))
        self._roots = roots
        p, eb, n = C.c_void_p(), C.c_int(), C.c_uint64()
        N.check(lib.bvhc_serialized_index(s, C.byref(p), C.byref(eb), C.byref(n)), "bvhc_serialized_index")
        if eb.value:
            dt = np.uint16 if eb.value == 2 else np.uint32
            self.geometry.index = np.frombuffer(C.string_at(p, n.value * eb.value), dtype=dt).copy()
        N.check(lib.bvhc_serialized_indirect(s, C.byref(p), C.byref(eb), C.byref(n)), "bvhc_serialized_indirect")
        if eb.value:
            dt = np.uint16 if eb.value == 2 else np.uint32
            self._indirectBuffer = np.frombuffer(C.string_at(p, n.value * eb.value), dtype=dt).copy()

    @property
    def indirect(self) -> bool:
        return self._indirectBuffer is not None

    def resolveTriangleIndex(self, i: int) -> int:
        return int(self._indirectBuffer[i]) if self.indirect else int(i)

    # -- serialize / deserialize (MeshBVH.js:112-232) --------------------------------------
    @staticmethod
    def serialize(bvh: "MeshBVH", options: dict | None = None) -> dict:
        clone = (options or {}).get("cloneBuffers", True)
        idx = bvh.geometry.index
        return {
            "version": 1,
            "roots": [bytes(r) for r in bvh._roots] if clone else bvh._roots,
            "index": (idx.copy() if clone else idx) if idx is not None else None,
            "indirectBuffer": (bvh._indirectBuffer.copy() if clone else bvh._indirectBuffer)
            if bvh._indirectBuffer is not None else None,
        }

    @staticmethod
    def deserialize(data: dict, geometry: Geometry, options: dict | None = None, *, device: int = 0) -> "MeshBVH":
        opts = {"setIndex": True, **(options or {})}
        bvh = MeshBVH(geometry, device=device, _skip_build=True)
        bvh._version = int(data.get("version", 0) or 0)
        bvh._roots = [bytes(r) for r in data["roots"]]
        ind = data.get("indirectBuffer")
        bvh._indirectBuffer = None if ind is None else np.asarray(ind)
        if opts["setIndex"] and data.get("index") is not None:
            if geometry.index is None:
                geometry.index = np.asarray(data["index"])
            elif geometry.index is not data["index"]:
                geometry.index[:] = data["index"]
        return bvh

    # -- device mesh -----------------------------------------------------------------------
    def _device_mesh(self):
        if self._mesh is None:
            lib = N.lib()
            g = self.geometry
            pos = np.ascontiguousarray(g.position, dtype=np.float32)
            idx = g.index
            ind = self._indirectBuffer
            bufs = [np.frombuffer(r, dtype=np.uint8) for r in self._roots]
            ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
            sizes = (C.c_uint64 * len(bufs))(*[b.size for b in bufs])
            out = C.c_void_p()
            st = lib.bvhc_mesh_create(self.device, getattr(self, "_version", 1), ptrs, sizes, len(bufs),
                                      _ptr(idx) if idx is not None else None,
                                      idx.dtype.itemsize if idx is not None else 0,
                                      idx.size if idx is not None else 0,
                                      _ptr(ind) if ind is not None else None,
                                      ind.dtype.itemsize if ind is not None else 0,
                                      ind.size if ind is not None else 0, _ptr(pos), pos.shape[0], 3, C.byref(out))
            N.check(st, "bvhc_mesh_create")
            self._mesh = out
            if g.groups:
                grp = np.array([[st_, -1 if (isinstance(c, float) and math.isinf(c)) else int(c), mi]
                                for st_, c, mi in g.groups], dtype=np.int64).reshape(-1)
                N.check(lib.bvhc_mesh_set_groups(out, _ptr(grp), len(g.groups)), "bvhc_mesh_set_groups")
        return self._mesh

    def mesh_info(self) -> dict:
        info = N.BvhcMeshInfo()
        N.check(N.lib().bvhc_mesh_get_info(self._device_mesh(), C.byref(info)), "bvhc_mesh_get_info")
        return {k: getattr(info, k) for k, _ in N.BvhcMeshInfo._fields_}

    def set_traversal(self, persistent: int = 1, order: int = 1, refill: int = 16, occupancy: int = 0,
                      compact: int = 0, sort: int = 0, closest: int = 0, wide: int = 0, all: int = 0,
                      tile: int = 0, block: int = 0, stack: int = 0, tile_rows: int = 0) -> None:
        """Select the traversal variants (see bvhc_mesh_set_traversal)."""
        cfg = N.BvhcTraversalConfig(persistent, order, refill, occupancy, compact, sort, closest, wide, all, tile,
                                    block, stack, tile_rows)
        N.check(N.lib().bvhc_mesh_set_traversal(self._device_mesh(), C.byref(cfg)), "bvhc_mesh_set_traversal")

    def get_traversal(self) -> dict:
        cfg = N.BvhcTraversalConfig()
        N.check(N.lib().bvhc_mesh_get_traversal(self._device_mesh(), C.byref(cfg)), "bvhc_mesh_get_traversal")
        return {k: getattr(cfg, k) for k, _ in N.BvhcTraversalConfig._fields_}

    def refit(self, positions=None, stream=None, read_back: bool = True) -> None:
        """MeshBVH#refit() (MeshBVH.js:504-508) on the GPU after the vertices moved.  positions:
        None (the geometry's position array, host memory), a numpy array, or a torch CUDA tensor
        (n x 3, on the device; enqueued on `stream`).  With read_back the serialized roots are
        copied back (waiting for the device), so serialize() returns the refit boxes as the
        reference's would; without it a device-memory refit only enqueues."""
        lib, mesh = N.lib(), self._device_mesh()
        if positions is not None and self._is_torch(positions):
            import torch
            p = positions.contiguous()
            s = stream if stream is not None else torch.cuda.current_stream(p.device).cuda_stream
            N.check(lib.bvhc_mesh_refit(mesh, p.data_ptr(), p.shape[0], 3, N.MEM_DEVICE, s), "bvhc_mesh_refit")
            if read_back:
                N.check(lib.bvhc_mesh_synchronize(mesh, s), "bvhc_mesh_synchronize")
        else:
            pos = self.geometry.position if positions is None else positions
            pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
            if positions is not None:
                self.geometry.position = pos
            N.check(lib.bvhc_mesh_refit(mesh, _ptr(pos), pos.shape[0], 3, N.MEM_HOST, None), "bvhc_mesh_refit")
        if not read_back:
            return
        roots = []
        for r in range(lib.bvhc_mesh_root_count(mesh)):
            buf = np.empty(lib.bvhc_mesh_root_bytes(mesh, r), dtype=np.uint8)
            N.check(lib.bvhc_mesh_read_root(mesh, r, _ptr(buf), buf.size), "bvhc_mesh_read_root")
            roots.append(buf.tobytes())
        self._roots = roots

    def set_leaf_size(self, max_leaf: int) -> None:
        """Device leaf layout (see bvhc_mesh_set_leaf_size): split leaves above max_leaf triangles;
        0 restores the reference's leaves."""
        N.check(N.lib().bvhc_mesh_set_leaf_size(self._device_mesh(), int(max_leaf)), "bvhc_mesh_set_leaf_size")

    def get_leaf_size(self) -> int:
        return int(N.lib().bvhc_mesh_get_leaf_size(self._device_mesh()))

    def dispose(self):
        if self._mesh is not None:
            N.lib().bvhc_mesh_destroy(self._mesh)
            self._mesh = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass

    # -- batched queries -------------------------------------------------------------------
    @staticmethod
    def _is_torch(x):
        return type(x).__module__.startswith("torch")

    def raycast_first_batch(self, rays, side=FrontSide, near=0.0, far=math.inf, out=None, stream=None):
        """raycastFirst for every row of `rays` (n x 6 float32).  numpy in -> numpy HIT_DTYPE out;
        torch CUDA tensor in -> (n, 8) float32 tensor whose rows are bvhc_hit records."""
        lib, mesh = N.lib(), self._device_mesh()
        if self._is_torch(rays):
            import torch
            n = rays.shape[0]
            if out is None:
                out = torch.empty((n, 8), dtype=torch.float32, device=rays.device)
            s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
            N.check(lib.bvhc_raycast_first(mesh, rays.data_ptr(), n, _side_of(side), float(near), float(far),
                                           out.data_ptr(), N.MEM_DEVICE, s), "bvhc_raycast_first")
            return out
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        res = np.empty(rays.shape[0], dtype=HIT_DTYPE) if out is None else out
        mats = _material_sides(side)
        if mats is not None:
            N.check(lib.bvhc_raycast_first_materials(mesh, _ptr(rays), rays.shape[0], _ptr(mats) if mats.size else None,
                                                     mats.size, float(near), float(far), _ptr(res), N.MEM_HOST, None),
                    "bvhc_raycast_first_materials")
            return res
        N.check(lib.bvhc_raycast_first(mesh, _ptr(rays), rays.shape[0], _side_of(side), float(near), float(far),
                                       _ptr(res), N.MEM_HOST, None), "bvhc_raycast_first")
        return res

    def raycast_batch(self, rays, side=FrontSide, near=0.0, far=math.inf, cap=64, stream=None, out=None):
        """All hits for every ray: (counts[n] uncapped, hits[n, cap]) in the reference's DFS order.
        out: optional (counts, hits) torch tensors to fill (device calls)."""
        lib, mesh = N.lib(), self._device_mesh()
        if self._is_torch(rays):
            import torch
            n = rays.shape[0]
            if out is not None:
                counts, hits = out
            else:
                counts = torch.empty(n, dtype=torch.int32, device=rays.device)
                hits = torch.empty((n, cap, 8), dtype=torch.float32, device=rays.device)
            s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
            N.check(lib.bvhc_raycast(mesh, rays.data_ptr(), n, _side_of(side), float(near), float(far), cap,
                                     counts.data_ptr(), hits.data_ptr(), N.MEM_DEVICE, s), "bvhc_raycast")
            return counts, hits
        rays = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = rays.shape[0]
        counts = np.empty(n, dtype=np.uint32)
        hits = np.empty((n, cap), dtype=HIT_DTYPE)
        mats = _material_sides(side)
        if mats is not None:
            N.check(lib.bvhc_raycast_materials(mesh, _ptr(rays), n, _ptr(mats) if mats.size else None, mats.size,
                                               float(near), float(far), cap, _ptr(counts), _ptr(hits), N.MEM_HOST,
                                               None), "bvhc_raycast_materials")
            return counts, hits
        N.check(lib.bvhc_raycast(mesh, _ptr(rays), n, _side_of(side), float(near), float(far), cap, _ptr(counts),
                                 _ptr(hits), N.MEM_HOST, None), "bvhc_raycast")
        return counts, hits

    def closest_point_batch(self, points, min_threshold=0.0, max_threshold=math.inf, stream=None, out=None):
        """closestPointToPoint for every row of `points` (n x 3 float32)."""
        lib, mesh = N.lib(), self._device_mesh()
        if self._is_torch(points):
            import torch
            n = points.shape[0]
            if out is None:
                out = torch.empty((n, 5), dtype=torch.float32, device=points.device)
            s = stream if stream is not None else torch.cuda.current_stream(points.device).cuda_stream
            N.check(lib.bvhc_closest_point_to_point(mesh, points.data_ptr(), n, float(min_threshold),
                                                    float(max_threshold), out.data_ptr(), N.MEM_DEVICE, s),
                    "bvhc_closest_point_to_point")
            return out
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        res = np.empty(pts.shape[0], dtype=CLOSEST_DTYPE)
        N.check(lib.bvhc_closest_point_to_point(mesh, _ptr(pts), pts.shape[0], float(min_threshold),
                                                float(max_threshold), _ptr(res), N.MEM_HOST, None),
                "bvhc_closest_point_to_point")
        return res

    def synchronize(self, stream=None):
        N.check(N.lib().bvhc_mesh_synchronize(self._device_mesh(), stream), "bvhc_mesh_synchronize")

    # -- gradients (forward/backward pairs; torch CUDA tensors) -----------------------------
    def _gradients_ready(self):
        if not getattr(self, "_grad_ready", False):
            g = self.geometry
            pos = np.ascontiguousarray(g.position, dtype=np.float32)
            idx = g.index
            N.check(N.lib().bvhc_mesh_enable_gradients(self._device_mesh(), _ptr(idx) if idx is not None else None,
                                                        idx.dtype.itemsize if idx is not None else 0,
                                                        idx.size if idx is not None else 0, _ptr(pos), pos.shape[0], 3),
                    "bvhc_mesh_enable_gradients")
            self._grad_ready = True

    def raycast_first_backward(self, rays, hits, grad_distance=None, grad_barycoord=None, grad_vertices=None,
                               stream=None):
        """Backward of raycast_first_batch: dL/d(distance) (n) and/or dL/d(barycoord) (n, 3) ->
        (grad_vertices (n_verts, 3) accumulated, grad_origins (n, 3), grad_directions (n, 3))."""
        import torch

        self._gradients_ready()
        n = rays.shape[0]
        dev = rays.device
        if grad_vertices is None:
            grad_vertices = torch.zeros((self.geometry.position.shape[0], 3), dtype=torch.float32, device=dev)
        go = torch.empty((n, 3), dtype=torch.float32, device=dev)
        gd = torch.empty((n, 3), dtype=torch.float32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        N.check(N.lib().bvhc_raycast_first_backward(
            self._device_mesh(), rays.data_ptr(), hits.data_ptr(), n,
            grad_distance.data_ptr() if grad_distance is not None else None,
            grad_barycoord.data_ptr() if grad_barycoord is not None else None,
            grad_vertices.data_ptr(), go.data_ptr(), gd.data_ptr(), s), "bvhc_raycast_first_backward")
        return grad_vertices, go, gd

    def closest_point_backward(self, points, results, grad_distance, grad_vertices=None, stream=None):
        """Backward of closest_point_batch's distance -> (grad_vertices accumulated, grad_points)."""
        import torch

        self._gradients_ready()
        n = points.shape[0]
        dev = points.device
        if grad_vertices is None:
            grad_vertices = torch.zeros((self.geometry.position.shape[0], 3), dtype=torch.float32, device=dev)
        gp = torch.empty((n, 3), dtype=torch.float32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        N.check(N.lib().bvhc_closest_point_backward(self._device_mesh(), points.data_ptr(), results.data_ptr(), n,
                                                     grad_distance.data_ptr(), grad_vertices.data_ptr(),
                                                     gp.data_ptr(), s), "bvhc_closest_point_backward")
        return grad_vertices, gp

    # -- reference-shaped single queries (MeshBVH.js:532-577, 874-884) ---------------------
    def _material_index(self, face_index: int) -> int:
        first = 3 * face_index
        for start, count, mi in self.geometry.groups:
            if first >= start and (math.isinf(count) or first < start + count):
                return int(mi)
        return 0

    def _intersection(self, rec, materials=False, direction=None) -> Intersection:
        f = int(rec["face_index"])
        tri = self.geometry.triangle(f)
        base = 3 * f
        if self.geometry.index is not None:
            a, b, c = (int(v) for v in self.geometry.index[base:base + 3])
        else:
            a, b, c = base, base + 1, base + 2
        n = np.cross(tri[2] - tri[1], tri[0] - tri[1])       # Triangle.getNormal
        ln = float(np.dot(n, n))
        n = n / math.sqrt(ln) if ln > 0 else np.zeros(3)
        bary = np.array(rec["barycoord"], dtype=np.float64)
        g = self.geometry

        def interp(attr):                                     # Triangle.getInterpolation
            return None if attr is None else bary @ attr[[a, b, c]].astype(np.float64)

        normal = interp(g.normal)
        if normal is not None and direction is not None and float(np.dot(normal, direction)) > 0:
            normal = -normal
        return Intersection(distance=float(rec["distance"]), point=np.array(rec["point"], dtype=np.float64),
                            face=Face(a, b, c, n, self._material_index(f) if materials else 0), faceIndex=f,
                            barycoord=bary, uv=interp(g.uv), uv1=interp(g.uv1), normal=normal)

    @staticmethod
    def _ray_row(ray) -> np.ndarray:
        o, d = ray
        return np.array([[*o, *d]], dtype=np.float32)

    def raycastFirst(self, ray, materialOrSide=FrontSide, near=0.0, far=math.inf):
        """`ray` is (origin, direction).  Returns an Intersection or None."""
        rec = self.raycast_first_batch(self._ray_row(ray), materialOrSide, near, far)[0]
        if int(rec["face_index"]) == N.NO_HIT:
            return None
        mats = isinstance(materialOrSide, (list, tuple))
        return self._intersection(rec, mats, np.asarray(ray[1], dtype=np.float64))

    def raycast(self, ray, materialOrSide=FrontSide, near=0.0, far=math.inf, cap=1024):
        """All hits of one ray, unsorted (DFS order), as a list of Intersection."""
        counts, hits = self.raycast_batch(self._ray_row(ray), materialOrSide, near, far, cap=cap)
        mats = isinstance(materialOrSide, (list, tuple))
        d = np.asarray(ray[1], dtype=np.float64)
        return [self._intersection(hits[0, k], mats, d) for k in range(min(int(counts[0]), cap))]

    def closestPointToPoint(self, point, target: HitPointInfo | None = None, minThreshold=0.0,
                            maxThreshold=math.inf):
        rec = self.closest_point_batch(np.array([point], dtype=np.float32), minThreshold, maxThreshold)[0]
        if int(rec["face_index"]) == N.NO_HIT:
            return None
        target = target if target is not None else HitPointInfo()
        target.point = np.array(rec["point"], dtype=np.float64)
        target.distance = float(rec["distance"])
        target.faceIndex = int(rec["face_index"])
        return target

    def hit_interpolate(self, hits, attribute, rays=None, stream=None):
        """A vertex attribute (n_verts x k, k <= 4) at every hit of raycast_first_batch's records
        (Intersection.uv / uv1 / normal in batch form, bvhc_hit_interpolate); with `rays`, a
        3-component result pointing along its ray is negated (the reference's normal).  torch CUDA
        tensors -> (n, k) tensor enqueued on `stream`; numpy -> (n, k) array."""
        lib, mesh = N.lib(), self._device_mesh()
        if self._is_torch(hits):
            import torch
            attr = attribute.contiguous()
            n, k = hits.shape[0], attr.shape[1]
            out = torch.empty((n, k), dtype=torch.float32, device=hits.device)
            s = stream if stream is not None else torch.cuda.current_stream(hits.device).cuda_stream
            N.check(lib.bvhc_hit_interpolate(mesh, hits.data_ptr(), n, attr.data_ptr(), attr.shape[0], k, k,
                                             rays.data_ptr() if rays is not None else None, out.data_ptr(),
                                             N.MEM_DEVICE, s), "bvhc_hit_interpolate")
            return out
        h = np.ascontiguousarray(hits).view(np.uint8).reshape(-1)
        n = h.size // 32
        attr = np.ascontiguousarray(attribute, dtype=np.float32)
        attr = attr.reshape(attr.shape[0], -1)
        k = attr.shape[1]
        r = None if rays is None else np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        out = np.empty((n, k), dtype=np.float32)
        N.check(lib.bvhc_hit_interpolate(mesh, _ptr(h), n, _ptr(attr), attr.shape[0], k, k,
                                         _ptr(r) if r is not None else None, _ptr(out), N.MEM_HOST, None),
                "bvhc_hit_interpolate")
        return out

    def intersects_sphere_batch(self, spheres, stream=None):
        """intersectsSphere for every row (cx, cy, cz, radius) of `spheres`: numpy -> bool array;
        torch CUDA tensor (n x 4, float32) -> uint8 tensor, enqueued on `stream`."""
        lib, mesh = N.lib(), self._device_mesh()
        if self._is_torch(spheres):
            import torch
            sp = spheres.contiguous()
            out = torch.empty(sp.shape[0], dtype=torch.uint8, device=sp.device)
            s = stream if stream is not None else torch.cuda.current_stream(sp.device).cuda_stream
            N.check(lib.bvhc_intersects_sphere(mesh, sp.data_ptr(), sp.shape[0], out.data_ptr(), N.MEM_DEVICE, s),
                    "bvhc_intersects_sphere")
            return out
        sp = np.ascontiguousarray(spheres, dtype=np.float32).reshape(-1, 4)
        out = np.empty(sp.shape[0], dtype=np.uint8)
        N.check(lib.bvhc_intersects_sphere(mesh, _ptr(sp), sp.shape[0], _ptr(out), N.MEM_HOST, None),
                "bvhc_intersects_sphere")
        return out.astype(bool)

    def sphere_triangles_batch(self, spheres, cap: int = 256):
        """The triangles within each sphere (cx, cy, cz, r), collected through shapecast's CONTAINED
        path as in the reference's sculpting / selection use: numpy -> (counts, faces (n, cap)) with
        faceIndex values in traversal order, 0xFFFFFFFF past the count."""
        lib, mesh = N.lib(), self._device_mesh()
        sp = np.ascontiguousarray(spheres, dtype=np.float32).reshape(-1, 4)
        counts = np.empty(sp.shape[0], dtype=np.uint32)
        faces = np.empty((sp.shape[0], cap), dtype=np.uint32)
        N.check(lib.bvhc_sphere_triangles(mesh, _ptr(sp), sp.shape[0], cap, _ptr(counts), _ptr(faces), N.MEM_HOST,
                                          None), "bvhc_sphere_triangles")
        return counts, faces

    @staticmethod
    def box_records(box_min, box_max, box_to_mesh) -> np.ndarray:
        """Pack oriented boxes for intersects_box_batch: (n x 3) min, (n x 3) max and (n x 16)
        column-major box-to-mesh matrices (three.js Matrix4.elements) -> (n x 24) float32."""
        mn = np.asarray(box_min, dtype=np.float32).reshape(-1, 3)
        mx = np.asarray(box_max, dtype=np.float32).reshape(-1, 3)
        m = np.asarray(box_to_mesh, dtype=np.float32).reshape(-1, 16)
        n = max(mn.shape[0], mx.shape[0], m.shape[0])
        out = np.zeros((n, 24), dtype=np.float32)
        out[:, 0:3], out[:, 4:7], out[:, 8:24] = mn, mx, m
        return out

    def intersects_box_batch(self, boxes, stream=None):
        """intersectsBox for every row of `boxes` (n x 24, see box_records): numpy -> bool array;
        torch CUDA tensor (float32) -> uint8 tensor, enqueued on `stream`."""
        lib, mesh = N.lib(), self._device_mesh()
        if self._is_torch(boxes):
            import torch
            bx = boxes.contiguous()
            out = torch.empty(bx.shape[0], dtype=torch.uint8, device=bx.device)
            s = stream if stream is not None else torch.cuda.current_stream(bx.device).cuda_stream
            N.check(lib.bvhc_intersects_box(mesh, bx.data_ptr(), bx.shape[0], out.data_ptr(), N.MEM_DEVICE, s),
                    "bvhc_intersects_box")
            return out
        bx = np.ascontiguousarray(boxes, dtype=np.float32).reshape(-1, 24)
        out = np.empty(bx.shape[0], dtype=np.uint8)
        N.check(lib.bvhc_intersects_box(mesh, _ptr(bx), bx.shape[0], _ptr(out), N.MEM_HOST, None),
                "bvhc_intersects_box")
        return out.astype(bool)

    def intersectsBox(self, box, box_to_mesh) -> bool:
        """MeshBVH#intersectsBox (MeshBVH.js:780-792); box: (min, max) or an object with `min` and
        `max`; box_to_mesh: 16 column-major matrix elements (or an object with `elements`)."""
        mn, mx = (box.min, box.max) if hasattr(box, "min") else box
        el = getattr(box_to_mesh, "elements", box_to_mesh)
        return bool(self.intersects_box_batch(self.box_records(mn, mx, el))[0])

    def triangle_hit_point_info_batch(self, points, faces) -> dict:
        """getTriangleHitPointInfo (src/utils/TriangleUtilities.js:65-147) for every (point,
        faceIndex) pair over this BVH's geometry (its index, positions, uv and groups), e.g. on
        closestPointToPoint results: numpy -> dict of arrays a, b, c, materialIndex (n,), normal and
        barycoord (n, 3), uv (n, 2) or None without a uv attribute."""
        lib, mesh, g = N.lib(), self._device_mesh(), self.geometry
        pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
        fc = np.ascontiguousarray(faces, dtype=np.uint32).reshape(-1)
        if fc.shape[0] != pts.shape[0]:
            raise ValueError("points and faces differ in length")
        grp = np.array([[s0, -1 if math.isinf(c0) else c0, mi] for s0, c0, mi in g.groups],
                       dtype=np.int64).reshape(-1)
        uv = g.uv
        out = np.empty(pts.shape[0], dtype=_HPI_DTYPE)
        N.check(lib.bvhc_triangle_hit_point_info(mesh, _ptr(pts), _ptr(fc), pts.shape[0], _ptr(g.position), 3,
                                                 _ptr(uv) if uv is not None else None, 2, g.position.shape[0],
                                                 _ptr(grp) if grp.size else None, len(g.groups), _ptr(out),
                                                 N.MEM_HOST, None), "bvhc_triangle_hit_point_info")
        return {"a": out["a"], "b": out["b"], "c": out["c"], "materialIndex": out["material_index"],
                "normal": out["normal"], "barycoord": out["barycoord"],
                "uv": out["uv"] if uv is not None else None}

    def getTriangleHitPointInfo(self, point, triangleIndex: int, target: dict | None = None) -> dict:
        """getTriangleHitPointInfo(point, geometry, triangleIndex, target) on this BVH's geometry:
        {"face": {"a", "b", "c", "materialIndex", "normal"}, "uv", "barycoord"}; an existing
        `target` dict is filled in and returned."""
        r = self.triangle_hit_point_info_batch(np.asarray(point, dtype=np.float32).reshape(1, 3), [triangleIndex])
        face = {"a": int(r["a"][0]), "b": int(r["b"][0]), "c": int(r["c"][0]),
                "materialIndex": int(r["materialIndex"][0]), "normal": r["normal"][0].copy()}
        info = target if target is not None else {}
        info["face"] = face
        info["uv"] = r["uv"][0].copy() if r["uv"] is not None else None
        info["barycoord"] = r["barycoord"][0].copy()
        return info

    def intersectsSphere(self, sphere) -> bool:
        """MeshBVH#intersectsSphere (MeshBVH.js:796-809); sphere: (center, radius) or an object
        with `center` and `radius`."""
        center, radius = (sphere.center, sphere.radius) if hasattr(sphere, "center") else sphere
        row = np.array([[*center, radius]], dtype=np.float32)
        return bool(self.intersects_sphere_batch(row)[0])
