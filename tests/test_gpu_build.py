"""Device SAH / CENTER build (bvhc_build_device) against the CPU build, whose output the builder
tests pin byte-for-byte to the oracle's restatement of the reference: every serialized root and the
reordered index (or indirect buffer) must be byte-identical.  The meshes cover the large-node
level kernels and the per-warp subtrees, bin-boundary and cost ties (integer lattices), planar
and degenerate nodes, duplicate and zero-area triangles, -0.0 coordinates, the small-count SAH
path (leaf sizes below 8), depth limits, groups / draw ranges (several roots), indirect builds and
non-indexed geometry."""
import math
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _serialized(pkg, geo, opts):
    bvh = pkg.MeshBVH(geo.clone(), opts)
    idx = None if bvh.geometry.index is None else bvh.geometry.index.copy()
    ind = None if bvh._indirectBuffer is None else bvh._indirectBuffer.copy()
    return list(bvh._roots), idx, ind


def _same_build(pkg, geo, **opts):
    base = {"strategy": pkg.SAH, "maxDepth": 40, "maxLeafSize": 10}
    base.update(opts)
    cpu = _serialized(pkg, geo, base)
    gpu = _serialized(pkg, geo, {**base, "deviceBuild": True})
    assert len(cpu[0]) == len(gpu[0])
    for r, (a, b) in enumerate(zip(cpu[0], gpu[0])):
        assert len(a) == len(b), (r, len(a), len(b))
        if a != b:
            wa, wb = np.frombuffer(a, np.uint32).reshape(-1, 8), np.frombuffer(b, np.uint32).reshape(-1, 8)
            bad = np.nonzero((wa != wb).any(axis=1))[0]
            raise AssertionError(f"root {r}: {bad.size} of {wa.shape[0]} nodes differ, first {bad[:5]}:\n"
                                 f"{wa[bad[:3]]}\n{wb[bad[:3]]}")
    for a, b in zip(cpu[1:], gpu[1:]):
        assert (a is None) == (b is None)
        if a is not None:
            assert a.dtype == b.dtype and np.array_equal(a, b)
    return cpu


def _lattice_cubes(pkg, n=6, spacing=2.0):
    cube = pkg.box()
    pos, idx = [], []
    k = 0
    for x in range(n):
        for y in range(n):
            for z in range(n):
                pos.append(cube.position + np.array([x, y, z], np.float32) * spacing)
                idx.append(cube.index.astype(np.int64) + k)
                k += cube.position.shape[0]
    return pkg.Geometry(np.concatenate(pos), np.concatenate(idx).astype(np.uint32))


def _plane_grid(pkg, n=120):
    ys, xs = np.meshgrid(np.arange(n + 1, dtype=np.float32), np.arange(n + 1, dtype=np.float32), indexing="ij")
    pos = np.stack([xs.ravel(), ys.ravel(), np.zeros(xs.size, np.float32)], axis=1)
    q = (np.arange(n)[:, None] * (n + 1) + np.arange(n)[None, :]).ravel()
    idx = np.stack([q, q + 1, q + n + 1, q + 1, q + n + 2, q + n + 1], axis=1).ravel().astype(np.uint32)
    return pkg.Geometry(pos, idx)


def _soup(pkg, n=20_000, seed=3):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-5, 5, (n, 1, 3)).astype(np.float32)
    tri = c + rng.normal(0, 0.3, (n, 3, 3)).astype(np.float32)
    tri[: n // 20] = tri[n // 20: n // 10]               # duplicate triangles
    tri[n // 10: n // 10 + 50] = tri[n // 10: n // 10 + 50, :1]  # zero-area (all vertices equal)
    tri[-200:, :, 2] = -0.0                                 # a -0.0 plane
    tri = np.round(tri * 8) / 8                             # many shared coordinates
    return pkg.Geometry(tri.reshape(-1, 3).astype(np.float32), None)


def test_torus_knot_k1(pkg, cuda):
    _same_build(pkg, pkg.torus_knot(10, 3, 400, 100))


def test_torus_knot_2m_and_speed(pkg, cuda):
    geo = pkg.torus_knot(10, 3, 2000, 500, noise_sigma=0.02, noise_seed=1)
    _same_build(pkg, geo)
    t0 = time.perf_counter()
    pkg.MeshBVH(geo.clone(), {"strategy": pkg.SAH, "deviceBuild": True})
    t_gpu = time.perf_counter() - t0
    t0 = time.perf_counter()
    pkg.MeshBVH(geo.clone(), {"strategy": pkg.SAH})
    t_cpu = time.perf_counter() - t0
    print(f"2M-triangle SAH build: device {t_gpu * 1e3:.1f} ms, CPU {t_cpu * 1e3:.1f} ms")


@pytest.mark.parametrize("strategy", ["SAH", "CENTER"])
def test_lattices_and_planes(pkg, cuda, strategy):
    s = getattr(pkg, strategy)
    _same_build(pkg, _lattice_cubes(pkg), strategy=s)
    _same_build(pkg, _plane_grid(pkg), strategy=s)
    _same_build(pkg, _soup(pkg), strategy=s)


@pytest.mark.parametrize("leaf,depth", [(1, 40), (3, 40), (5, 40), (7, 40), (10, 3), (10, 0), (2, 12)])
def test_leaf_sizes_and_depth_limits(pkg, cuda, leaf, depth):
    _same_build(pkg, pkg.torus_knot(10, 3, 64, 16), maxLeafSize=leaf, maxDepth=depth)
    _same_build(pkg, _soup(pkg, 3000, seed=leaf), maxLeafSize=leaf, maxDepth=depth)


@pytest.mark.parametrize("tris", [5, 1000, 1024, 1025, 2049, 5000])
def test_sizes_around_the_subtree_threshold(pkg, cuda, tris):
    _same_build(pkg, _soup(pkg, tris, seed=tris))


def test_groups_ranges_indirect_nonindexed(pkg, cuda):
    geo = pkg.torus_knot(10, 3, 300, 40)
    n = geo.index.size
    geo.groups = [(0, n // 3 - n // 3 % 3, 0), (n // 2 - n // 2 % 3, math.inf, 1)]
    _same_build(pkg, geo)
    _same_build(pkg, geo, indirect=True)
    g2 = pkg.torus_knot(10, 3, 300, 40)
    g2.draw_range = (3 * 500, 3 * 9000)
    _same_build(pkg, g2)
    _same_build(pkg, g2, indirect=True)
    _same_build(pkg, _soup(pkg, 8000), indirect=True)
    _same_build(pkg, _soup(pkg, 8000), strategy=pkg.CENTER, indirect=True)


def test_average_is_cpu_only(pkg, cuda):
    with pytest.raises(Exception):
        pkg.MeshBVH(pkg.torus_knot(10, 3, 64, 16), {"strategy": pkg.AVERAGE, "deviceBuild": True})
