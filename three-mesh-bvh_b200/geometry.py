"""Geometry containers and seeded synthetic inputs (meshes, rays, query grids).

`Geometry` carries what the reference reads from a three.js `BufferGeometry` on this path:
the float32 position attribute, the optional index (Uint16Array or Uint32Array, chosen the way
three.js sizes an index), the groups and the draw range.

The mesh generators build tessellated surfaces from their parametric definitions: a (p, q)
torus knot tube, a torus, a UV sphere and a subdivided icosahedron, with the same parameters
and triangle counts as the three.js generators of the same names (TorusKnotGeometry(10, 3,
400, 100) has 80,000 triangles and 401 x 101 vertices).  They are not bit-identical to three.js's
vertex positions: three.js is not available here, and nothing on the query path depends on it.
"""
from __future__ import annotations

import math
import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Geometry:
    position: np.ndarray                      # (n_verts, 3) float32
    index: np.ndarray | None = None           # uint16 / uint32, length multiple of 3
    groups: list = field(default_factory=list)  # [(start, count, materialIndex)] in index units
    draw_range: tuple = (0, math.inf)         # (start, count) in index units
    # optional vertex attributes reported on hits (Intersection.normal / uv / uv1)
    normal: np.ndarray | None = None          # (n_verts, 3) float32
    uv: np.ndarray | None = None              # (n_verts, 2) float32
    uv1: np.ndarray | None = None             # (n_verts, 2) float32

    def __post_init__(self):
        self.position = np.ascontiguousarray(self.position, dtype=np.float32).reshape(-1, 3)
        for name, k in (("normal", 3), ("uv", 2), ("uv1", 2)):
            a = getattr(self, name)
            if a is not None:
                setattr(self, name, np.ascontiguousarray(a, dtype=np.float32).reshape(-1, k))
        if self.index is not None:
            self.index = np.ascontiguousarray(self.index)
            if self.index.dtype not in (np.uint16, np.uint32):
                self.index = self.index.astype(index_dtype(int(self.index.max()) + 1 if self.index.size else 0))

    @property
    def triangle_count(self) -> int:
        n = self.index.size if self.index is not None else self.position.shape[0]
        return n // 3

    def add_group(self, start: int, count: float, material_index: int = 0) -> None:
        self.groups.append((int(start), count, int(material_index)))

    def clone(self) -> "Geometry":
        cp = (lambda a: None if a is None else a.copy())
        return Geometry(self.position.copy(), cp(self.index), list(self.groups), self.draw_range, cp(self.normal),
                        cp(self.uv), cp(self.uv1))

    def triangle(self, face_index: int) -> np.ndarray:
        """Vertices (3, 3) float64 of triangle `face_index` (through the index when present)."""
        base = 3 * int(face_index)
        ids = self.index[base:base + 3] if self.index is not None else np.arange(base, base + 3)
        return self.position[ids.astype(np.int64)].astype(np.float64)


def index_dtype(vertex_count: int):
    """three.js picks a Uint32 index when a vertex index exceeds 65535 (geometryUtils.js:15-27)."""
    return np.uint32 if vertex_count > 65535 else np.uint16


def _grid_index(rows: int, cols: int) -> np.ndarray:
    """Two triangles per quad of a (rows+1) x (cols+1) vertex grid, wound counter-clockwise when
    the first grid direction x second grid direction points along the surface normal."""
    i, j = np.meshgrid(np.arange(rows), np.arange(cols), indexing="ij")
    w = cols + 1
    a = i * w + j
    b = (i + 1) * w + j
    c = (i + 1) * w + j + 1
    d = i * w + j + 1
    tris = np.stack([np.stack([a, b, d], -1), np.stack([b, c, d], -1)], -2).reshape(-1, 3)
    return tris.reshape(-1)


def torus_knot(radius=1.0, tube=0.4, tubular_segments=64, radial_segments=8, p=2, q=3, noise_sigma=0.0,
               noise_seed=None) -> Geometry:
    """(p, q) torus-knot tube: centre curve c(s) = R/2 [(2 + cos(q s)) cos(p s), (2 + cos(q s)) sin(p s),
    sin(q s)], s in [0, 2 pi); circular cross-section of radius `tube` in the plane normal to c'(s).
    Optionally each vertex is displaced along its tube normal by N(0, noise_sigma) (seeded);
    seam duplicates share their displacement so the surface stays closed."""
    s = np.arange(tubular_segments + 1, dtype=np.float64) / tubular_segments * 2 * math.pi
    cq, sq, cp, sp = np.cos(q * s), np.sin(q * s), np.cos(p * s), np.sin(p * s)
    r = 2 + cq
    c = 0.5 * radius * np.stack([r * cp, r * sp, sq], -1)
    dc = 0.5 * radius * np.stack([-q * sq * cp - p * r * sp, -q * sq * sp + p * r * cp, q * cq], -1)
    t = dc / np.linalg.norm(dc, axis=-1, keepdims=True)
    ref = c - (c * t).sum(-1, keepdims=True) * t
    n = ref / np.linalg.norm(ref, axis=-1, keepdims=True)
    b = np.cross(t, n)
    v = np.arange(radial_segments + 1, dtype=np.float64) / radial_segments * 2 * math.pi
    cv, sv = np.cos(v)[None, :, None], np.sin(v)[None, :, None]
    normal = cv * n[:, None, :] + sv * b[:, None, :]          # outward tube normal, (T+1, R+1, 3)
    offset = np.full(normal.shape[:2], float(tube))
    if noise_sigma:
        rng = np.random.default_rng(noise_seed)
        base = rng.normal(0.0, noise_sigma, size=(tubular_segments, radial_segments))
        ii = np.arange(tubular_segments + 1) % tubular_segments
        jj = np.arange(radial_segments + 1) % radial_segments
        offset = offset + base[ii][:, jj]
    pos = c[:, None, :] + offset[..., None] * normal
    index = _grid_index(tubular_segments, radial_segments)
    # orient so that (b - a) x (c - a) points along the outward normal
    p0 = pos.reshape(-1, 3)
    tri = index[:3]
    nrm = np.cross(p0[tri[1]] - p0[tri[0]], p0[tri[2]] - p0[tri[0]])
    if np.dot(nrm, normal.reshape(-1, 3)[tri[0]]) < 0:
        index = index.reshape(-1, 3)[:, [0, 2, 1]].reshape(-1)
    n_verts = pos.shape[0] * pos.shape[1]
    uv = np.stack(np.meshgrid(np.arange(tubular_segments + 1) / tubular_segments,
                              np.arange(radial_segments + 1) / radial_segments, indexing="ij"), -1)
    return Geometry(p0.astype(np.float32), index.astype(index_dtype(n_verts)),
                    normal=normal.reshape(-1, 3).astype(np.float32), uv=uv.reshape(-1, 2).astype(np.float32))


def torus(radius=1.0, tube=0.4, radial_segments=12, tubular_segments=48) -> Geometry:
    """Torus about the z axis: (R + r cos v) (cos u, sin u) in xy, r sin v in z."""
    v = np.arange(radial_segments + 1, dtype=np.float64) / radial_segments * 2 * math.pi
    u = np.arange(tubular_segments + 1, dtype=np.float64) / tubular_segments * 2 * math.pi
    vv, uu = np.meshgrid(v, u, indexing="ij")
    x = (radius + tube * np.cos(vv)) * np.cos(uu)
    y = (radius + tube * np.cos(vv)) * np.sin(uu)
    z = tube * np.sin(vv)
    pos = np.stack([x, y, z], -1).reshape(-1, 3)
    index = _grid_index(radial_segments, tubular_segments)
    tri = index[:3]
    nrm = np.cross(pos[tri[1]] - pos[tri[0]], pos[tri[2]] - pos[tri[0]])
    centre = np.array([radius * math.cos(0.0), 0.0, 0.0])
    if np.dot(nrm, pos[tri[0]] - centre) < 0:
        index = index.reshape(-1, 3)[:, [0, 2, 1]].reshape(-1)
    return Geometry(pos.astype(np.float32), index.astype(index_dtype(pos.shape[0])))


def sphere(radius=1.0, width_segments=32, height_segments=16) -> Geometry:
    """UV sphere with poles at (0, +-radius, 0); the zero-area triangles at the poles are dropped."""
    phi = np.arange(width_segments + 1, dtype=np.float64) / width_segments * 2 * math.pi
    theta = np.arange(height_segments + 1, dtype=np.float64) / height_segments * math.pi
    th, ph = np.meshgrid(theta, phi, indexing="ij")
    x = -radius * np.cos(ph) * np.sin(th)
    y = radius * np.cos(th)
    z = radius * np.sin(ph) * np.sin(th)
    pos = np.stack([x, y, z], -1).reshape(-1, 3)
    w = width_segments + 1
    tris = []
    for iy in range(height_segments):
        for ix in range(width_segments):
            a = iy * w + ix + 1
            b = iy * w + ix
            c = (iy + 1) * w + ix
            d = (iy + 1) * w + ix + 1
            if iy != 0:
                tris.append((a, b, d))
            if iy != height_segments - 1:
                tris.append((b, c, d))
    index = np.array(tris, dtype=np.int64)
    nrm = np.cross(pos[index[:, 1]] - pos[index[:, 0]], pos[index[:, 2]] - pos[index[:, 0]])
    if np.mean((nrm * pos[index[:, 0]]).sum(-1)) < 0:
        index = index[:, [0, 2, 1]]
    return Geometry(pos.astype(np.float32), index.reshape(-1).astype(index_dtype(pos.shape[0])))


def icosahedron(radius=1.0, detail=0) -> Geometry:
    """Regular icosahedron with every face split into (detail + 1)^2 triangles, projected onto
    the sphere: 20 (detail + 1)^2 triangles, non-shared vertices per face."""
    t = (1 + math.sqrt(5)) / 2
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    n = detail + 1
    # barycentric lattice of one face
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = ii + jj <= n
    ii, jj = ii[keep], jj[keep]
    lid = -np.ones((n + 1, n + 1), dtype=np.int64)
    lid[ii, jj] = np.arange(ii.size)
    # lattice cells (i, j), i + j < n, row by row: the upward triangle, then the downward one
    # where it exists (i + j + 1 < n)
    ci, cj = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    cell = ci + cj < n
    ci, cj = ci[cell], cj[cell]
    up = np.stack([lid[ci, cj], lid[ci + 1, cj], lid[ci, cj + 1]], -1)
    has_down = ci + cj + 1 < n
    dn_i, dn_j = np.minimum(ci + 1, n), np.minimum(cj + 1, n)
    down = np.stack([lid[dn_i, cj], lid[dn_i, dn_j], lid[ci, dn_j]], -1)
    small = np.stack([up, down], 1)[np.stack([np.ones_like(has_down), has_down], 1)]
    pos, idx = [], []
    for k, (a, b, c) in enumerate(f):
        pts = v[a][None] + (ii[:, None] / n) * (v[b] - v[a])[None] + (jj[:, None] / n) * (v[c] - v[a])[None]
        pts = pts / np.linalg.norm(pts, axis=1, keepdims=True) * radius
        idx.append(small + k * ii.size)
        pos.append(pts)
    pos = np.concatenate(pos)
    idx = np.concatenate(idx)
    nrm = np.cross(pos[idx[:, 1]] - pos[idx[:, 0]], pos[idx[:, 2]] - pos[idx[:, 0]])
    flip = (nrm * pos[idx[:, 0]]).sum(-1) < 0
    idx[flip] = idx[flip][:, [0, 2, 1]]
    return Geometry(pos.astype(np.float32), idx.reshape(-1).astype(index_dtype(pos.shape[0])))


def box() -> Geometry:
    """Unit cube centred at the origin, faces ordered +x, -x, +y, -y, +z, -z, two triangles each,
    wound outward; one group per face (6 index entries each)."""
    faces = []
    for axis in range(3):
        for sign in (1.0, -1.0):
            u_ax, v_ax = (axis + 1) % 3, (axis + 2) % 3
            quad = []
            for (su, sv) in ((-0.5, -0.5), (0.5, -0.5), (0.5, 0.5), (-0.5, 0.5)):
                p = [0.0, 0.0, 0.0]
                p[axis] = 0.5 * sign
                p[u_ax] = su
                p[v_ax] = sv
                quad.append(p)
            quad = np.array(quad)
            tris = [(0, 1, 2), (0, 2, 3)]
            nrm = np.cross(quad[1] - quad[0], quad[2] - quad[0])
            if nrm[axis] * sign < 0:
                tris = [(0, 2, 1), (0, 3, 2)]
            faces.append((quad, tris))
    pos, idx = [], []
    for k, (quad, tris) in enumerate(faces):
        pos.append(quad)
        idx.extend([(a + 4 * k, b + 4 * k, c + 4 * k) for a, b, c in tris])
    g = Geometry(np.concatenate(pos).astype(np.float32), np.array(idx, dtype=np.uint16).reshape(-1))
    for k in range(6):
        g.add_group(6 * k, 6, k)
    return g


# ------------------------------------------------------------------------------------------
# Rays and query points (all float32, rows [ox, oy, oz, dx, dy, dz])
# ------------------------------------------------------------------------------------------

def _unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def rays_sphere_to_box(n, seed=0, radius=40.0, half=13.0) -> np.ndarray:
    """Origins uniform on a sphere of `radius`; each direction points at a uniform point in
    [-half, half]^3 and is normalised (the 1,000,000-ray set on the 80,000-triangle knot)."""
    rng = np.random.default_rng(seed)
    o = _unit(rng, n) * radius
    target = rng.uniform(-half, half, size=(n, 3))
    d = target - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


def rays_incoherent(n, seed=1, radius=40.0) -> np.ndarray:
    """Origins uniform on a sphere shell of `radius`, directions uniform on the unit sphere."""
    rng = np.random.default_rng(seed)
    o = _unit(rng, n) * radius
    d = _unit(rng, n)
    return np.concatenate([o, d], 1).astype(np.float32)


def rays_camera(width, height, distance=35.0, fov_deg=45.0) -> np.ndarray:
    """Pinhole camera at (0, 0, distance) looking at the origin (up +y), vertical FOV `fov_deg`,
    one ray through each pixel centre."""
    tan_half = math.tan(math.radians(fov_deg) / 2)
    aspect = width / height
    xs = ((np.arange(width) + 0.5) / width * 2 - 1) * tan_half * aspect
    ys = (1 - (np.arange(height) + 0.5) / height * 2) * tan_half
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    d = np.stack([xx, yy, -np.ones_like(xx)], -1).reshape(-1, 3)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    o = np.broadcast_to(np.array([0.0, 0.0, distance]), d.shape)
    return np.concatenate([o, d], 1).astype(np.float32)


def grid_points(lo, hi, res, pad=0.1) -> np.ndarray:
    """res^3 points spanning the box [lo, hi] enlarged by `pad` of its extent (half per side)."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    ext = hi - lo
    lo2, hi2 = lo - ext * pad / 2, hi + ext * pad / 2
    axes = [np.linspace(lo2[k], hi2[k], res) for k in range(3)]
    g = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    return g.astype(np.float32)


# ------------------------------------------------------------------------------------------
# Batched scene: many sub-geometries of very uneven size, each with its own rays
# ------------------------------------------------------------------------------------------

def batched_scene(n_geometries=1024, tri_range=(200, 200_000), ray_range=(1_000, 1_000_000), seed=2,
                  make_rays=True):
    """Sub-geometries alternating torus knots (radius 10, tube 3) and subdivided icosahedra
    (radius 10), triangle counts log-uniform in `tri_range`, each with a random rigid transform and
    a log-uniform number of rays in `ray_range` drawn as for the 80,000-triangle knot (origins on
    the r = 40 sphere, directions at uniform points of [-13, 13]^3) in its local frame.
    Returns (geometries, transforms (n, 4, 4), rays (sum, 6) float32 or None, ray_offsets)."""
    rng = np.random.default_rng(seed)
    lo_t, hi_t = tri_range
    lo_r, hi_r = ray_range
    tri_target = np.exp(rng.uniform(math.log(lo_t), math.log(hi_t), n_geometries))
    ray_counts = np.exp(rng.uniform(math.log(lo_r), math.log(hi_r), n_geometries)).astype(np.int64)
    def make(k):
        t = float(tri_target[k])
        if k % 2 == 0:
            radial = max(3, int(round(math.sqrt(t / 8))))
            tubular = max(3, int(round(t / (2 * radial))))
            return torus_knot(10, 3, tubular, radial)
        detail = max(0, int(round(math.sqrt(t / 20))) - 1)
        return icosahedron(10.0, detail)

    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
        geoms = list(ex.map(make, range(n_geometries)))
    transforms = np.zeros((n_geometries, 4, 4))
    for k in range(n_geometries):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        transforms[k, :3, :3] = rot
        transforms[k, :3, 3] = rng.uniform(-200, 200, 3)
        transforms[k, 3, 3] = 1
    offsets = np.concatenate([[0], np.cumsum(ray_counts)]).astype(np.uint64)
    rays = None
    if make_rays:
        rays = np.empty((int(offsets[-1]), 6), dtype=np.float32)

        def fill(k):   # each geometry's rays come from their own seed, so threads may fill them
            rays[int(offsets[k]):int(offsets[k + 1])] = rays_sphere_to_box(int(ray_counts[k]), seed=10_000 + k)

        with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 1)) as ex:
            list(ex.map(fill, range(n_geometries)))
    return geoms, transforms, rays, offsets
