"""three-mesh-bvh B200 engine: GPU batches of raycastFirst / raycast / closestPointToPoint
against three-mesh-bvh's serialized MeshBVH, through the libbvhcuda C ABI."""
from ._native import BVHCError, NO_HIT, lib  # noqa: F401
from .geometry import (Geometry, batched_scene, box, grid_points, icosahedron, index_dtype,  # noqa: F401
                       rays_camera, rays_incoherent, rays_sphere_to_box, sphere, torus, torus_knot)
from .mesh_bvh import (AVERAGE, CENTER, CLOSEST_DTYPE, DEFAULT_OPTIONS, HIT_DTYPE, SAH, BackSide,  # noqa: F401
                       DoubleSide, FrontSide, HitPointInfo, Intersection, MeshBVH)
