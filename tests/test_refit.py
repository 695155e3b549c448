"""The oracle's restatement of MeshBVH#refit, pinned by the reference's own refit tests
(test/MeshBVH.test.js:291-367) and by properties of its change rule.  No GPU needed."""
import numpy as np

from refit_util import validate_bounds


def _sphere_bvh(pkg, orc, segs, leaf):
    geo = pkg.sphere(1, segs, segs)
    o = orc.OracleBVH.build(geo.position, geo.index, target_leaf=leaf)
    idx = np.empty(geo.index.size, dtype=np.uint32)
    orc.lib().orc_copy_index(o.h, idx.ctypes.data)
    return geo, o, idx


def test_refit_resizes_bounds_to_moved_vertex(pkg, orc):
    """MeshBVH.test.js:293-306: move one vertex, bounds stop containing it, refit fixes them."""
    geo, o, idx = _sphere_bvh(pkg, orc, 10, 10)
    assert validate_bounds(o.roots(), geo.position, idx)
    pos = geo.position.copy()
    pos[0, 0] = 10
    assert not validate_bounds(o.roots(), pos, idx)
    o.refit(pos)
    assert validate_bounds(o.roots(), pos, idx)


def test_refit_after_scaling_scales_the_root_box(pkg, orc):
    """MeshBVH.test.js:308-337: targetLeafSize 1, geometry scaled by 2, root box doubles."""
    geo, o, idx = _sphere_bvh(pkg, orc, 16, 1)
    before = np.frombuffer(o.roots()[0], dtype=np.float32)[:6].astype(np.float64)
    pos = geo.position * np.float32(2)
    o.refit(pos)
    after = np.frombuffer(o.roots()[0], dtype=np.float32)[:6].astype(np.float64)
    # the build pads boxes by 2^-24 relative, the refit box is exact: equal to 2x within float32
    assert np.allclose(after, 2 * before, rtol=0, atol=1e-5)
    assert validate_bounds(o.roots(), pos, idx)


def test_refit_change_rule(pkg, orc):
    """A second refit with unchanged vertices leaves every byte alone; moving one vertex rewrites
    only the boxes on the paths from its leaves to the root."""
    geo, o, idx = _sphere_bvh(pkg, orc, 24, 4)
    o.refit(geo.position)
    first = o.roots()[0]
    o.refit(geo.position)
    assert o.roots()[0] == first
    pos = geo.position.copy()
    pos[37] += np.float32(0.25)
    o.refit(pos)
    nodes_a = np.frombuffer(first, dtype=np.float32).reshape(-1, 8)[:, :6]
    nodes_b = np.frombuffer(o.roots()[0], dtype=np.float32).reshape(-1, 8)[:, :6]
    changed = np.nonzero((nodes_a != nodes_b).any(1))[0]
    assert 0 < changed.size < nodes_a.shape[0] // 4
    assert changed[0] == 0                      # the root is on every changed path
    assert validate_bounds(o.roots(), pos, idx)
