"""Instanced scenes for the BatchedMesh instance tests: random world matrices over a set of
geometries, world rays, and the mapping of a baked world mesh's faces back to instances."""
import numpy as np


def instance_matrices(rng, n, n_geoms, spread=150.0, scaled=True):
    geometry = rng.integers(0, n_geoms, n).astype(np.uint32)
    mats = np.zeros((n, 16))
    for j in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        x, y, z, w = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        if scaled:
            s = rng.uniform(0.5, 2.0) if j % 3 else 1.0
            sc = np.full(3, s) if j % 5 else rng.uniform(0.5, 2.0, 3)   # every fifth non-uniform
            rot = rot * sc[None, :]
        m = np.eye(4)
        m[:3, :3] = rot
        m[:3, 3] = rng.uniform(-spread, spread, 3)
        mats[j] = m.T.reshape(-1)   # column-major elements
    return geometry, mats


def world_rays(rng, n, radius=400.0, half=180.0):
    u = rng.normal(size=(n, 3))
    o = u / np.linalg.norm(u, axis=1, keepdims=True) * radius
    t = rng.uniform(-half, half, (n, 3))
    d = t - o
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return np.concatenate([o, d], 1).astype(np.float32)


def bake(geoms_tris, geometry, matrices, visible=None):
    """World triangles of every visible instance (float32) and, per baked face, (instance, local face)."""
    tris, owner, local = [], [], []
    for j, g in enumerate(geometry):
        if visible is not None and not visible[j]:
            continue
        t = geoms_tris[int(g)]
        m = matrices[j].reshape(4, 4).T
        w = t @ m[:3, :3].T + m[:3, 3]
        tris.append(w.astype(np.float32))
        owner.append(np.full(t.shape[0], j))
        local.append(np.arange(t.shape[0]))
    return np.concatenate(tris), np.concatenate(owner), np.concatenate(local)
