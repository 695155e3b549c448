"""The C ABI without a GPU: the library loads, exports every entry point include/bvhcuda.h declares,
and rejects malformed serialized BVHs on the host (status codes, never a trap).  The
corruptions mirror what a bad `MeshBVH.deserialize` input can hold: truncated buffers,
right-child offsets outside the buffer, leaf ranges past the triangle count, and trees deeper
than the traversal stack."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

HEADER = Path(__file__).resolve().parents[1] / "include" / "bvhcuda.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bvhc_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol(pkg):
    lib = pkg.lib()
    names = declared_functions()
    assert len(names) >= 14
    for name in names:
        assert hasattr(lib, name), name


def test_status_strings(pkg):
    lib = pkg.lib()
    for code in range(8):
        assert lib.bvhc_status_string(code)
    assert lib.bvhc_status_string(0) == b"ok"


def _create(pkg, roots, geo, version=1):
    lib = pkg.lib()
    bufs = [np.frombuffer(bytes(r), dtype=np.uint8) for r in roots]
    ptrs = (C.c_void_p * len(bufs))(*[b.ctypes.data for b in bufs])
    sizes = (C.c_uint64 * len(bufs))(*[b.size for b in bufs])
    out = C.c_void_p()
    pos = geo.position
    idx = geo.index
    st = lib.bvhc_mesh_create(0, version, ptrs, sizes, len(bufs), idx.ctypes.data, idx.dtype.itemsize, idx.size,
                              None, 0, 0, pos.ctypes.data, pos.shape[0], 3, C.byref(out))
    return st


@pytest.fixture(scope="module")
def knot(pkg):
    geo = pkg.torus_knot(10, 3, 32, 8)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    return geo, bvh._roots[0]


def test_rejects_truncated_buffer(pkg, knot):
    geo, root = knot
    assert _create(pkg, [root[:-4]], geo) == 2       # BVHC_ERR_INVALID_BVH


def test_rejects_right_child_out_of_range(pkg, knot):
    geo, root = knot
    bad = bytearray(root)
    bad[24:28] = np.uint32(len(root) // 32 + 5).tobytes()   # node 0 is internal
    assert _create(pkg, [bytes(bad)], geo) == 2


def test_rejects_leaf_range_past_triangles(pkg, knot):
    geo, root = knot
    u16 = np.frombuffer(root, dtype=np.uint16).reshape(-1, 16)
    leaf = int(np.nonzero(u16[:, 15] == 0xFFFF)[0][0])
    bad = bytearray(root)
    bad[leaf * 32 + 24: leaf * 32 + 28] = np.uint32(geo.triangle_count).tobytes()
    assert _create(pkg, [bytes(bad)], geo) == 2


def test_rejects_bad_split_axis(pkg, knot):
    geo, root = knot
    bad = bytearray(root)
    bad[28:32] = np.uint32(7).tobytes()
    assert _create(pkg, [bytes(bad)], geo) == 2


def test_rejects_too_deep_tree(pkg):
    # a chain of 80 internal nodes, each with a leaf as its right child
    geo = pkg.torus(1, 0.4, 8, 8)
    nodes = []
    depth = 80
    for d in range(depth):
        nodes.append(("internal", d))
    buf = bytearray()
    # pre-order: internal(0), internal(1) ... internal(79), leaf, then the right leaves in reverse order
    total = 2 * depth + 1
    words = np.zeros((total, 8), dtype=np.uint32)
    f = words.view(np.float32)
    f[:, :3] = -10
    f[:, 3:6] = 10
    for d in range(depth):
        node = d
        right = total - 1 - d           # right leaves placed from the end
        words[node, 6] = right - node
        words[node, 7] = 0
    for k in range(depth, total):
        words[k, 6] = 0
        words[k, 7] = 1 | (0xFFFF << 16)
    buf = words.tobytes()
    assert _create(pkg, [buf], geo) == 6            # BVHC_ERR_UNSUPPORTED


def test_invalid_arguments(pkg, knot):
    lib = pkg.lib()
    out = C.c_void_p()
    assert lib.bvhc_mesh_create(0, 1, None, None, 0, None, 0, 0, None, 0, 0, None, 0, 3, C.byref(out)) == 1
    assert lib.bvhc_raycast_first(None, None, 1, 0, 0.0, 1.0, None, 0, None) == 1
    assert lib.bvhc_build(None, 0, 3, None, 0, 0, None, 0, 0, -1, 2, 40, 10, 0, C.byref(out)) == 1


def test_autotune_candidates_and_argument_checks(pkg):
    """bvhc_autotune_candidates lists the autotuner's stage-1 variants without a GPU; the autotuner
    itself rejects bad arguments before touching the device."""
    from three_mesh_bvh_b200 import _native as N
    from three_mesh_bvh_b200 import autotune

    lib = pkg.lib()
    base = autotune.candidates()
    assert len(base) == 95 and len({tuple(c) for c in base}) == 95
    fields = autotune.FIELDS
    assert fields[:6] == ["persistent", "order", "refill", "occupancy", "compact", "sort"]
    assert fields[9:] == ["tile", "block", "stack", "tile_rows"]
    forms = {c[0] for c in base}
    assert forms == {0, 1, 2}
    assert any(c[7] == 1 for c in base)                                    # four-child records
    assert sum(1 for c in base if c[0] == 1 and c[7] == 1) == 8           # persistent over them
    assert {(c[4], c[5]) for c in base if c[0] == 1} == {(0, 0), (1, 0), (1, 1), (1, 2), (1, 3)}
    tiled = autotune.candidates((4096, 1920))
    # per pitch: child pairs (2 child orders x 3 register budgets), then four-child records (3 budgets)
    assert tiled[:95] == base and len(tiled) == 95 + 18
    assert {c[9] for c in tiled[95:]} == {4096, 1920} and all(c[0] == 2 and c[4] == 0 for c in tiled[95:])
    assert [c[7] for c in tiled[95:104]] == [0] * 6 + [1] * 3
    with pytest.raises(ValueError):
        autotune.candidates((-8,))
    assert lib.bvhc_autotune_candidates(None, 1, None, 0) == -1
    best = (N.BvhcTraversalConfig * 1)()
    counts = (C.c_uint64 * 1)(16)
    rays = (C.c_void_p * 1)(None)
    assert lib.bvhc_mesh_autotune(None, 1, rays, counts, 0, 0.0, 1.0, None, 0, None, 0, 3, None, best, None, None,
                                  None) == 1                                  # BVHC_ERR_INVALID_ARGUMENT

