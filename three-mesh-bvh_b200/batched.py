"""Batched meshes: the bounds trees of a BatchedMesh served by one persistent GPU launch.

Mirrors `computeBatchedBoundsTree` (src/utils/ExtensionUtilities.js:216-268): one MeshBVH per
geometry over one shared index/position buffer, each built over its own draw range so that its
leaf offsets are absolute triangle indices of the shared index.  Each geometry's BVH is built on
its own (in parallel host threads; the build releases the GIL), then merged into the shared
buffers: vertex indices move by the geometry's first vertex and leaf offsets by its first
triangle (`shiftTriangleOffsets`, src/core/BVH.js:146-190).  The tree of every geometry is the one
a build over the shared geometry with `range` produces, because the build only sees the
triangles of the range, in the same order.

`raycast_first` replaces the per-instance serial loop of acceleratedBatchedMeshRaycast
(ExtensionUtilities.js:87-161) for rays already expressed in each geometry's local frame.
"""
from __future__ import annotations

import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _native as N
from .geometry import Geometry, index_dtype
from .mesh_bvh import FrontSide, MeshBVH, _side_of


def shift_triangle_offsets(root: bytes, offset: int) -> bytes:
    """Adds `offset` to every leaf's triangle offset of a serialized root (BVH.js:146-190)."""
    u32 = np.frombuffer(root, dtype=np.uint32).reshape(-1, 8).copy()
    leaf = (u32[:, 7] >> 16) == 0xFFFF
    u32[leaf, 6] += np.uint32(offset)
    return u32.tobytes()


class BatchedMeshBVH:
    def __init__(self, geometries: list[Geometry], options: dict | None = None, *, device: int = 0,
                 threads: int | None = None):
        self.device = device
        opts = dict(options or {})
        with ThreadPoolExecutor(max_workers=threads) as ex:
            bvhs = list(ex.map(lambda g: MeshBVH(g, opts, device=device), geometries))
        self.geometries = geometries
        vbase = np.cumsum([0] + [g.position.shape[0] for g in geometries])
        tbase = np.cumsum([0] + [g.triangle_count for g in geometries])
        self.vertex_base = vbase
        self.triangle_base = tbase
        self.position = np.ascontiguousarray(np.concatenate([g.position for g in geometries]), dtype=np.float32)
        dt = index_dtype(int(vbase[-1]))
        self.index = np.concatenate([g.index.astype(np.int64) + vbase[k] for k, g in enumerate(geometries)]).astype(dt)
        self.roots = []
        self.roots_per_mesh = []
        for k, b in enumerate(bvhs):
            rs = [shift_triangle_offsets(r, int(tbase[k])) for r in b._roots]
            self.roots.extend(rs)
            self.roots_per_mesh.append(len(rs))
            b.dispose()
        self._mesh = None
        self._graphs = []

    @property
    def n_meshes(self) -> int:
        return len(self.roots_per_mesh)

    def _device_mesh(self):
        if self._mesh is None:
            lib = N.lib()
            bufs = [np.frombuffer(r, dtype=np.uint8) for r in self.roots]
            ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
            sizes = (C.c_uint64 * len(bufs))(*[b.size for b in bufs])
            rpm = np.asarray(self.roots_per_mesh, dtype=np.int32)
            out = C.c_void_p()
            st = lib.bvhc_batch_create(self.device, self.n_meshes, rpm.ctypes.data, ptrs, sizes, self.index.ctypes.data,
                                       self.index.dtype.itemsize, self.index.size, self.position.ctypes.data,
                                       self.position.shape[0], 3, C.byref(out))
            N.check(st, "bvhc_batch_create")
            self._mesh = out
        return self._mesh

    def set_traversal(self, persistent=1, order=1, refill=16, occupancy=0, compact=0, sort=0, closest=0, wide=0,
                      all=0, tile=0, block=0, stack=0, tile_rows=0):
        cfg = N.BvhcTraversalConfig(persistent, order, refill, occupancy, compact, sort, closest, wide, all, tile,
                                    block, stack, tile_rows)
        N.check(N.lib().bvhc_mesh_set_traversal(self._device_mesh(), C.byref(cfg)), "bvhc_mesh_set_traversal")

    def set_leaf_size(self, max_leaf: int):
        """raycastFirst's device leaf layout for every geometry (bvhc_mesh_set_leaf_size): 0 keeps the
        reference's leaves, max_leaf > 0 splits larger leaves into exact-bounds subtrees."""
        N.check(N.lib().bvhc_mesh_set_leaf_size(self._device_mesh(), int(max_leaf)), "bvhc_mesh_set_leaf_size")

    def get_leaf_size(self) -> int:
        return int(N.lib().bvhc_mesh_get_leaf_size(self._device_mesh()))

    @staticmethod
    def _offsets(ray_offsets) -> np.ndarray:
        return np.ascontiguousarray(ray_offsets, dtype=np.uint64)

    def raycast_first(self, rays, ray_offsets, side=FrontSide, near=0.0, far=float("inf"), out=None, stream=None):
        """One persistent launch over every geometry's rays.  rays: torch CUDA tensor (n, 6) whose
        rows [ray_offsets[k], ray_offsets[k+1]) are geometry k's rays in its local frame; returns an
        (n, 8) float32 tensor of bvhc_hit records, faceIndex in the shared index."""
        import torch

        off = self._offsets(ray_offsets)
        if out is None:
            out = torch.empty((rays.shape[0], 8), dtype=torch.float32, device=rays.device)
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        N.check(N.lib().bvhc_batch_raycast_first(self._device_mesh(), rays.data_ptr(), off.ctypes.data,
                                                 _side_of(side), float(near), float(far), out.data_ptr(), s),
                "bvhc_batch_raycast_first")
        return out

    def raycast_first_per_mesh(self, rays, ray_offsets, side=FrontSide, near=0.0, far=float("inf"), out=None,
                               stream=None):
        """The same work as one launch per geometry (the comparison baseline)."""
        import torch

        off = self._offsets(ray_offsets)
        if out is None:
            out = torch.empty((rays.shape[0], 8), dtype=torch.float32, device=rays.device)
        s = stream if stream is not None else torch.cuda.current_stream(rays.device).cuda_stream
        N.check(N.lib().bvhc_batch_raycast_first_per_mesh(self._device_mesh(), rays.data_ptr(), off.ctypes.data,
                                                          _side_of(side), float(near), float(far), out.data_ptr(), s),
                "bvhc_batch_raycast_first_per_mesh")
        return out

    def capture(self, rays, ray_offsets, out, side=FrontSide, near=0.0, far=float("inf")):
        """CUDA graph of the batched launch on these fixed buffers; call .launch(stream) to replay."""
        off = self._offsets(ray_offsets)
        g = C.c_void_p()
        N.check(N.lib().bvhc_batch_graph_create(self._device_mesh(), rays.data_ptr(), off.ctypes.data, _side_of(side),
                                                float(near), float(far), out.data_ptr(), C.byref(g)),
                "bvhc_batch_graph_create")
        graph = _Graph(g)
        self._graphs.append(graph)
        return graph

    def synchronize(self, stream=None):
        N.check(N.lib().bvhc_mesh_synchronize(self._device_mesh(), stream), "bvhc_mesh_synchronize")

    def instances(self, geometry, matrices, visible=None) -> "InstancedScene":
        """The BatchedMesh's instances: instance j shows geometry[j] under the world matrix
        matrices[j] (16 column-major float64 elements: matrixWorld times the instance matrix);
        visible: per-instance flags (getVisibleAt), None for all."""
        return InstancedScene(self, geometry, matrices, visible)

    def dispose(self):
        for g in self._graphs:
            g.destroy()
        self._graphs = []
        if self._mesh is not None:
            N.lib().bvhc_mesh_destroy(self._mesh)
            self._mesh = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass


class _Graph:
    def __init__(self, handle):
        self.h = handle

    def launch(self, stream=None):
        N.check(N.lib().bvhc_graph_launch(self.h, stream), "bvhc_graph_launch")

    def destroy(self):
        if self.h:
            N.lib().bvhc_graph_destroy(self.h)
            self.h = None


class InstancedScene:
    """acceleratedBatchedMeshRaycast (ExtensionUtilities.js:87-161) with firstHitOnly on world
    rays: each visible instance's raycastFirst in its own frame, hits back in world space, the
    closest one kept, plus its instance (the Intersection's batchId)."""

    def __init__(self, batch: BatchedMeshBVH, geometry, matrices, visible=None):
        self.batch = batch  # the scene reads the batch's trees: keep it alive
        self.h = None
        out = C.c_void_p()
        g, m, v = self._arrays(geometry, matrices, visible)
        N.check(N.lib().bvhc_scene_create(batch._device_mesh(), g.size, g.ctypes.data, m.ctypes.data,
                                          None if v is None else v.ctypes.data, C.byref(out)), "bvhc_scene_create")
        self.h = out

    @staticmethod
    def _arrays(geometry, matrices, visible):
        g = np.ascontiguousarray(geometry, dtype=np.uint32).reshape(-1)
        m = np.ascontiguousarray(matrices, dtype=np.float64).reshape(-1, 16)
        if m.shape[0] != g.size:
            raise ValueError("one 16-element matrix per instance")
        v = None if visible is None else np.ascontiguousarray(visible, dtype=np.uint8).reshape(-1)
        return g, m, v

    def set_instances(self, geometry, matrices, visible=None):
        g, m, v = self._arrays(geometry, matrices, visible)
        N.check(N.lib().bvhc_scene_set_instances(self.h, g.size, g.ctypes.data, m.ctypes.data,
                                                 None if v is None else v.ctypes.data), "bvhc_scene_set_instances")

    def set_order(self, kind: int):
        """Traverse the rays in input order (0), sorted by a Morton key (1 direction, 2 entry point
        into the instances' box, 3 entry point and direction) or by the first instance they reach
        (4).  Results do not change."""
        N.check(N.lib().bvhc_scene_set_order(self.h, int(kind)), "bvhc_scene_set_order")

    def set_variant(self, variant: int):
        """raycastFirst kernel variant (bvhc_scene_set_variant): 0..2."""
        N.check(N.lib().bvhc_scene_set_variant(self.h, int(variant)), "bvhc_scene_set_variant")

    def raycast_first(self, rays, side=FrontSide, near=0.0, far=float("inf"), stream=None):
        """World rays (n x 6 float32): numpy -> (hits structured array, instance ids); torch CUDA
        tensor -> ((n, 8) float32 hit tensor, int32 instance tensor), enqueued on `stream`."""
        lib = N.lib()
        if hasattr(rays, "data_ptr"):
            import torch
            r = rays.contiguous()
            hits = torch.empty((r.shape[0], 8), dtype=torch.float32, device=r.device)
            inst = torch.empty(r.shape[0], dtype=torch.int32, device=r.device)
            s = stream if stream is not None else torch.cuda.current_stream(r.device).cuda_stream
            N.check(lib.bvhc_scene_raycast_first(self.h, r.data_ptr(), r.shape[0], _side_of(side), float(near),
                                                 float(far), hits.data_ptr(), inst.data_ptr(), N.MEM_DEVICE, s),
                    "bvhc_scene_raycast_first")
            return hits, inst
        from .mesh_bvh import HIT_DTYPE
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        hits = np.empty(r.shape[0], dtype=HIT_DTYPE)
        inst = np.empty(r.shape[0], dtype=np.uint32)
        N.check(lib.bvhc_scene_raycast_first(self.h, r.ctypes.data, r.shape[0], _side_of(side), float(near),
                                             float(far), hits.ctypes.data, inst.ctypes.data, N.MEM_HOST, None),
                "bvhc_scene_raycast_first")
        return hits, inst

    def raycast(self, rays, side=FrontSide, near=0.0, far=float("inf"), cap=64):
        """Every hit of every instance (no firstHitOnly), world space, sorted by distance: numpy
        rays -> (counts, hits (n, cap) structured, instances (n, cap))."""
        from .mesh_bvh import HIT_DTYPE
        r = np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)
        n = r.shape[0]
        counts = np.empty(n, dtype=np.uint32)
        hits = np.empty((n, cap), dtype=HIT_DTYPE)
        inst = np.empty((n, cap), dtype=np.uint32)
        N.check(N.lib().bvhc_scene_raycast(self.h, r.ctypes.data, n, _side_of(side), float(near), float(far), cap,
                                           counts.ctypes.data, hits.ctypes.data, inst.ctypes.data, N.MEM_HOST, None),
                "bvhc_scene_raycast")
        return counts, hits, inst

    def dispose(self):
        if self.h:
            N.lib().bvhc_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.dispose()
        except Exception:
            pass
