"""Oriented-box helpers for the intersectsBox tests: column-major 4x4 matrices composed from a
position, an XYZ Euler rotation and a scale (the standard quaternion-to-rotation formulas), and a
numpy restatement of the reference's separating-axis test used as a brute force over every
triangle."""
import numpy as np


def quaternion_xyz(ex, ey, ez):
    c1, c2, c3 = np.cos(ex / 2), np.cos(ey / 2), np.cos(ez / 2)
    s1, s2, s3 = np.sin(ex / 2), np.sin(ey / 2), np.sin(ez / 2)
    return np.array([s1 * c2 * c3 + c1 * s2 * s3, c1 * s2 * c3 - s1 * c2 * s3,
                     c1 * c2 * s3 + s1 * s2 * c3, c1 * c2 * c3 - s1 * s2 * s3])


def compose(position, quat, scale=(1.0, 1.0, 1.0)):
    """Column-major elements of T * R(quat) * S."""
    x, y, z, w = quat
    sx, sy, sz = scale
    m = np.zeros(16)
    m[0] = (1 - 2 * (y * y + z * z)) * sx
    m[1] = 2 * (x * y + w * z) * sx
    m[2] = 2 * (x * z - w * y) * sx
    m[4] = 2 * (x * y - w * z) * sy
    m[5] = (1 - 2 * (x * x + z * z)) * sy
    m[6] = 2 * (y * z + w * x) * sy
    m[8] = 2 * (x * z + w * y) * sz
    m[9] = 2 * (y * z - w * x) * sz
    m[10] = (1 - 2 * (x * x + y * y)) * sz
    m[12:15] = position
    m[15] = 1
    return m


def record(mn, mx, m):
    r = np.zeros(24, np.float32)
    r[0:3], r[4:7], r[8:24] = mn, mx, m
    return r


def random_boxes(rng, n, center, spread, shear=False):
    out = np.zeros((n, 24), np.float32)
    for i in range(n):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        m = compose(center + rng.uniform(-spread, spread, 3), q, rng.uniform(0.3, 3.0, 3))
        if shear:
            a = np.eye(4)
            a[0, 1], a[1, 2] = rng.uniform(-0.5, 0.5, 2)
            m = (m.reshape(4, 4).T @ a).T.reshape(-1)
        half = rng.uniform(0.2, 2.5, 3)
        out[i] = record(-half, half, m)
    return out


def _interval(axis, pts):
    v = np.einsum("...k,...jk->...j", axis, pts)
    return v.min(-1), v.max(-1)


def brute_force(tri, box):
    """Per triangle (T x 3 x 3, float64): the reference's OrientedBox.intersectsTriangle, returning
    (meets, smallest |gap| over the axes) with gap > 0 on separated axes."""
    e = box[8:24].astype(np.float64).reshape(4, 4).T  # row-major view of the column-major matrix
    mn, mx = box[0:3].astype(np.float64), box[4:7].astype(np.float64)
    corners = np.array([[mx[0] if i & 1 else mn[0], mx[1] if i & 2 else mn[1], mx[2] if i & 4 else mn[2]]
                        for i in range(8)])
    h = np.c_[corners, np.ones(8)] @ e.T
    p = h[:, :3] / h[:, 3:4]
    ax = np.stack([p[0] - p[1], p[0] - p[2], p[0] - p[4]])
    a, b, c = tri[:, 0], tri[:, 1], tri[:, 2]
    n = np.cross(c - b, a - b)
    l2 = (n * n).sum(1, keepdims=True)
    n = np.where(l2 > 0, n / np.sqrt(np.where(l2 > 0, l2, 1)), 0)
    ta = [n, a - b, b - c, c - a]
    T = tri.shape[0]
    sep = np.zeros(T, bool)
    gap = np.full(T, np.inf)

    def test(amn, amx, bmn, bmx):
        nonlocal sep, gap
        g = np.maximum(amn - bmx, bmn - amx)
        sep |= g > 0
        gap = np.minimum(gap, np.abs(g))

    P = np.broadcast_to(p, (T, 8, 3))
    for i in range(3):
        smn, smx = _interval(ax[i], p)
        tmn, tmx = _interval(np.broadcast_to(ax[i], (T, 3)), tri)
        test(smn, smx, tmn, tmx)
    for i in range(3):
        test(*_interval(ta[i], tri), *_interval(ta[i], P))
    for i in range(3):
        for j in range(4):
            axis = np.cross(np.broadcast_to(ax[i], (T, 3)), ta[j])
            test(*_interval(axis, tri), *_interval(axis, P))
    return ~sep, gap
