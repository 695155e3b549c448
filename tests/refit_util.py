"""Bounds validation of serialized MeshBVH roots (the reference's validateBounds,
src/debug/Debug.js:207-260): every leaf box contains its triangles' vertices, every node box
lies inside its parent's."""
import numpy as np


def validate_bounds(roots, position, index, indirect=None):
    pos = np.asarray(position, dtype=np.float32).reshape(-1, 3)
    tri = np.asarray(index, dtype=np.int64).reshape(-1, 3)
    for buf in roots:
        f = np.frombuffer(buf, dtype=np.float32).reshape(-1, 8)
        u32 = np.frombuffer(buf, dtype=np.uint32).reshape(-1, 8)
        u16 = np.frombuffer(buf, dtype=np.uint16).reshape(-1, 16)
        stack = [(0, None)]
        while stack:
            node, parent = stack.pop()
            box = f[node, :6]
            if parent is not None:
                pb = f[parent, :6]
                if (box[:3] < pb[:3]).any() or (box[3:] > pb[3:]).any():
                    return False
            if u16[node, 15] == 0xFFFF:
                off, cnt = int(u32[node, 6]), int(u16[node, 14])
                if cnt:
                    t = np.arange(off, off + cnt)
                    if indirect is not None:
                        t = np.asarray(indirect)[t]
                    v = pos[tri[t].reshape(-1)]
                    if (v < box[:3]).any() or (v > box[3:]).any():
                        return False
            else:
                stack.append((node + 1, node))
                stack.append((node + int(u32[node, 6]), node))
    return True
