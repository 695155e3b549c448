"""The library's CPU builder (bvhc_build) against the oracle's restatement of the reference build:
identical serialized roots, identical in-place index reorder, identical indirect buffer.

Covers the options matrix of test/utils.js:86-147 (strategy x indirect), groups and draw ranges
(test/ShapeCasts.test.js:981-1003, geometryUtils.js:60-159), maxDepth truncation, the Uint16 /
Uint32 index choice at 65535 vertices (test/MeshBVH.serialize.test.js:60-80) and non-indexed
geometry.
"""
import math

import numpy as np
import pytest


def _both(pkg, orc, geo, **opts):
    g1, g2 = geo.clone(), geo.clone()
    strategy = opts.get("strategy", 0)
    bvh = pkg.MeshBVH(g1, dict(opts))
    rng = opts.get("range")
    dr = rng if rng is not None else g2.draw_range
    o = orc.OracleBVH.build(g2.position, g2.index, groups=g2.groups, draw_range=dr, strategy=strategy,
                            max_depth=opts.get("maxDepth", 40), target_leaf=opts.get("targetLeafSize", 10),
                            indirect=opts.get("indirect", False))
    return bvh, g1, o


def _assert_same(bvh, g1, o):
    assert bvh._roots == o.roots()
    oi = o.index()
    if oi is None:
        assert g1.index is None
    else:
        assert g1.index.dtype == oi.dtype and np.array_equal(g1.index, oi)
    ind = o.indirect()
    if ind is None:
        assert bvh._indirectBuffer is None
    else:
        assert bvh._indirectBuffer.dtype == ind.dtype and np.array_equal(bvh._indirectBuffer, ind)


@pytest.mark.parametrize("strategy", [0, 1, 2])
@pytest.mark.parametrize("indirect", [False, True])
def test_knot_matrix(pkg, orc, strategy, indirect):
    geo = pkg.torus_knot(10, 3, 200, 40, noise_sigma=0.02, noise_seed=1)
    _assert_same(*_both(pkg, orc, geo, strategy=strategy, indirect=indirect))


@pytest.mark.parametrize("strategy", [0, 1, 2])
@pytest.mark.parametrize("leaf", [1, 3, 10, 25])
def test_leaf_sizes(pkg, orc, strategy, leaf):
    geo = pkg.icosahedron(2.0, 6)
    _assert_same(*_both(pkg, orc, geo, strategy=strategy, targetLeafSize=leaf))


@pytest.mark.parametrize("strategy", [0, 2])
def test_max_depth_truncation(pkg, orc, strategy):
    geo = pkg.torus(1, 0.4, 30, 60)
    bvh, g1, o = _both(pkg, orc, geo, strategy=strategy, maxDepth=3, targetLeafSize=1)
    _assert_same(bvh, g1, o)
    assert o.stats()["max_depth"] <= 3


@pytest.mark.parametrize("indirect", [False, True])
def test_groups_and_gaps(pkg, orc, indirect):
    geo = pkg.box()
    geo.groups = []
    geo.add_group(0, 6, 0)
    geo.add_group(12, 24, 1)                    # the -x face (index 6..11) is in no group
    bvh, g1, o = _both(pkg, orc, geo, strategy=2, indirect=indirect)
    _assert_same(bvh, g1, o)
    assert len(bvh._roots) == (1 if indirect else 2)


def test_overlapping_groups_and_infinite_count(pkg, orc):
    geo = pkg.torus(1, 0.4, 16, 32)
    n = geo.index.size
    geo.add_group(0, n // 2, 0)
    geo.add_group(n // 4, math.inf, 1)
    for strategy in (0, 1, 2):
        _assert_same(*_both(pkg, orc, geo, strategy=strategy))


def test_draw_range_and_range_option(pkg, orc):
    geo = pkg.torus(1, 0.4, 16, 32)
    geo.draw_range = (30, 300)
    _assert_same(*_both(pkg, orc, geo, strategy=2))
    geo2 = pkg.torus(1, 0.4, 16, 32)
    _assert_same(*_both(pkg, orc, geo2, strategy=2, range=(60, 900)))


@pytest.mark.parametrize("n_verts,dtype", [(65535, np.uint16), (65536, np.uint32)])
def test_created_index_width(pkg, orc, n_verts, dtype):
    rng = np.random.default_rng(3)
    pos = rng.uniform(-1, 1, size=(n_verts - n_verts % 3, 3)).astype(np.float32)
    pos = np.concatenate([pos, np.zeros((n_verts - pos.shape[0], 3), np.float32)])
    geo = pkg.Geometry(pos, None)
    bvh, g1, o = _both(pkg, orc, geo, strategy=0)
    assert g1.index.dtype == dtype
    _assert_same(bvh, g1, o)


def test_non_indexed_indirect(pkg, orc):
    rng = np.random.default_rng(4)
    pos = rng.uniform(-1, 1, size=(900, 3)).astype(np.float32)
    geo = pkg.Geometry(pos, None)
    bvh, g1, o = _both(pkg, orc, geo, strategy=2, indirect=True)
    assert g1.index is None
    _assert_same(bvh, g1, o)


def test_degenerate_inputs(pkg, orc):
    # all triangles identical: every split fails and the root stays a leaf
    pos = np.tile(np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), (40, 1))
    geo = pkg.Geometry(pos, None)
    for strategy in (0, 1, 2):
        bvh, g1, o = _both(pkg, orc, geo, strategy=strategy)
        _assert_same(bvh, g1, o)
        assert len(bvh._roots[0]) == 32
