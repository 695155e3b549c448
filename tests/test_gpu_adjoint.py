"""Adjoint kernels against float64 references: the oracle's forward-mode dual-number Jacobian of
the ray/triangle formula (exact derivatives) and central finite differences (h = 1e-3) of the
replayed recorded triangles.  Gradients must agree within 1e-3 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-3
H = 1e-3


def _records(pkg, t):
    return t.cpu().numpy().view(np.uint8).reshape(-1).view(pkg.HIT_DTYPE)


@pytest.fixture(scope="module")
def knot(pkg, cuda):
    geo = pkg.torus_knot(10, 3, 300, 60, noise_sigma=0.02, noise_seed=1)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    return geo, bvh


def _expected(orc, geo, rays, rec, g_dist, g_bary):
    """Per-ray expected (grad_vertices accumulated, grad_origins, grad_directions) in float64."""
    gv = np.zeros((geo.position.shape[0], 3))
    go = np.zeros((rays.shape[0], 3))
    gd = np.zeros((rays.shape[0], 3))
    for i in range(rays.shape[0]):
        f = int(rec["face_index"][i])
        if f == 0xFFFFFFFF:
            continue
        ids = geo.index[3 * f:3 * f + 3].astype(np.int64)
        a, b, c = geo.position[ids].astype(np.float64)
        _, jac = orc.ray_triangle_jacobian(rays[i, :3], rays[i, 3:], a, b, c)
        up = np.zeros(5)
        up[0] = g_dist[i]
        up[2:5] = g_bary[i]
        g = up @ jac
        for k in range(3):
            gv[ids[k]] += g[3 * k:3 * k + 3]
        go[i] = g[9:12]
        gd[i] = g[12:15]
    return gv, go, gd


def _close(got, exp, rel=REL):
    scale = np.abs(exp).max()
    err = np.abs(got - exp)
    return err.max() <= rel * max(scale, 1e-12), err.max() / max(scale, 1e-12)


def test_raycast_backward_matches_float64_jacobian(pkg, orc, knot, cuda):
    import torch

    geo, bvh = knot
    rays = np.concatenate([pkg.rays_camera(96, 96), pkg.rays_sphere_to_box(4096, seed=31)])
    d_rays = torch.from_numpy(rays).to(cuda)
    hits = bvh.raycast_first_batch(d_rays)
    rng = np.random.default_rng(5)
    g_dist = rng.normal(size=rays.shape[0]).astype(np.float32)
    g_bary = rng.normal(size=(rays.shape[0], 3)).astype(np.float32)
    gv, go, gd = bvh.raycast_first_backward(d_rays, hits, torch.from_numpy(g_dist).to(cuda),
                                            torch.from_numpy(g_bary).to(cuda))
    bvh.synchronize()
    rec = _records(pkg, hits)
    ev, eo, ed = _expected(orc, geo, rays, rec, g_dist, g_bary)
    hit = rec["face_index"] != 0xFFFFFFFF
    assert hit.sum() > 2000
    for got, exp in ((go.cpu().numpy(), eo), (gd.cpu().numpy(), ed)):
        per_ray = np.abs(got - exp).max(1) / np.maximum(np.abs(exp).max(1), 1e-6)
        assert np.quantile(per_ray[hit], 1.0) <= REL, np.sort(per_ray[hit])[-5:]
    ok, worst = _close(gv.cpu().numpy(), ev)
    assert ok, worst


def _cos_incidence(geo, rays, faces, hit):
    """|cos| of the angle between each hitting ray and its triangle's normal (0 for misses)."""
    tri = geo.position[geo.index.astype(np.int64).reshape(-1, 3)[np.where(hit, faces, 0)]].astype(np.float64)
    n = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    d = rays[:, 3:].astype(np.float64)
    c = np.abs((n * d).sum(1)) / (np.linalg.norm(n, axis=1) * np.linalg.norm(d, axis=1))
    return np.where(hit, c, 0.0)


def test_raycast_backward_finite_differences(pkg, orc, knot, cuda):
    """Central differences (h = 1e-3) of the recorded triangles' distances, replayed in float64,
    against the GPU gradient of L = sum g_i distance_i with random weights g_i, on 4096 sampled
    vertices and on ray origins and directions.  (A loss with small residuals, such as
    sum (t - t*)^2 with t* within 0.01 of t, makes the gradient itself small while the difference
    quotient's truncation error keeps the size of the curvature, so a linear functional is the
    well-conditioned check of the same derivatives.)  Rays meeting their triangle at grazing
    incidence (|cos| < 0.3, silhouettes) are left out: t bends too sharply there for h = 1e-3;
    their exact derivatives are checked against the float64 Jacobian above."""
    import torch

    geo, bvh = knot
    rays = pkg.rays_camera(128, 128)
    d_rays = torch.from_numpy(rays).to(cuda)
    hits = bvh.raycast_first_batch(d_rays)
    rec = _records(pkg, hits)
    hit = rec["face_index"] != 0xFFFFFFFF
    hit &= _cos_incidence(geo, rays, rec["face_index"].astype(np.int64), hit) >= 0.3
    rng = np.random.default_rng(3)
    g = np.where(hit, rng.normal(size=rays.shape[0]), 0.0).astype(np.float32)
    g64 = g.astype(np.float64)  # float32 * float stays float32 under NumPy 2: keep the quotients in float64
    gv, go, gd = bvh.raycast_first_backward(d_rays, hits, torch.from_numpy(g).to(cuda))
    bvh.synchronize()
    gv, go, gd = gv.cpu().numpy(), go.cpu().numpy(), gd.cpu().numpy()
    faces = rec["face_index"].astype(np.int64)
    tri_of = geo.index.astype(np.int64).reshape(-1, 3)
    pos0 = geo.position.astype(np.float64)

    def dist(i, o, d, pos):
        vals, _ = orc.ray_triangle_jacobian(o, d, *pos[tri_of[faces[i]]])
        return vals[0]

    rays_of = {}
    for i in np.nonzero(hit)[0]:
        for v in tri_of[faces[i]]:
            rays_of.setdefault(int(v), []).append(i)
    used = np.array(sorted(rays_of))
    sample = rng.choice(used, size=min(4096, used.size), replace=False)
    fd = np.zeros((sample.size, 3))
    mag = np.zeros((sample.size, 3))   # sum over the vertex's rays of |g_i d dist_i / dv|
    for s_, v in enumerate(sample):
        for k in range(3):
            p_hi, p_lo = pos0.copy(), pos0.copy()
            p_hi[v, k] += H
            p_lo[v, k] -= H
            for i in rays_of[int(v)]:
                o, d = rays[i, :3], rays[i, 3:]
                term = g64[i] * (dist(i, o, d, p_hi) - dist(i, o, d, p_lo)) / (2 * H)
                fd[s_, k] += term
                mag[s_, k] += abs(term)
    # A vertex gradient is a sum over rays with random-sign weights; where the sum cancels, the
    # difference quotient's own truncation error (relative to each term) dominates the relative
    # error of the sum, so the error is measured against the size of the terms.
    scale = np.maximum(np.maximum(np.abs(fd).max(1), mag.max(1)), 1e-3)
    err = np.abs(gv[sample] - fd).max(1) / scale
    assert err.max() <= REL, np.sort(err)[-5:]
    for i in rng.choice(np.nonzero(hit)[0], size=256, replace=False):
        o0, d0 = rays[i, :3].astype(np.float64), rays[i, 3:].astype(np.float64)
        for got, which in ((go[i], 0), (gd[i], 1)):
            fdv = np.zeros(3)
            for k in range(3):
                vals = []
                for sgn in (1.0, -1.0):
                    o, d = o0.copy(), d0.copy()
                    (o if which == 0 else d)[k] += sgn * H
                    vals.append(g64[i] * dist(i, o, d, pos0))
                fdv[k] = (vals[0] - vals[1]) / (2 * H)
            assert np.abs(got - fdv).max() <= REL * max(np.abs(fdv).max(), 1e-3), (i, which, got, fdv)


def test_warp_aggregated_vertex_gradients_on_a_coarse_mesh(pkg, orc, cuda):
    """Many rays per triangle: lanes of a warp share faces, so the aggregated atomics are used."""
    import torch

    geo = pkg.torus(10, 3, 6, 8)
    bvh = pkg.MeshBVH(geo)
    rays = pkg.rays_camera(64, 64)
    d_rays = torch.from_numpy(rays).to(cuda)
    hits = bvh.raycast_first_batch(d_rays)
    g = np.random.default_rng(8).normal(size=rays.shape[0]).astype(np.float32)
    gv, _, _ = bvh.raycast_first_backward(d_rays, hits, torch.from_numpy(g).to(cuda))
    bvh.synchronize()
    rec = _records(pkg, hits)
    ev, _, _ = _expected(orc, geo, rays, rec, g, np.zeros((rays.shape[0], 3), np.float32))
    ok, worst = _close(gv.cpu().numpy(), ev)
    assert ok, worst


def test_closest_point_backward_finite_differences(pkg, orc, knot, cuda):
    """Central differences (h = 1e-3) of point-to-recorded-triangle distances, in float64, against
    the GPU gradient of L = sum g_i distance_i with random weights, on 4096 sampled queries and
    4096 sampled vertices.  The distance to a triangle is only once differentiable where the
    closest feature changes (face, edge, vertex regions), so a sample is compared only where the
    difference quotient has converged (h and h / 2 agree within 1e-4 relative); queries within 0.1
    of the surface are left out (curvature ~ 1 / distance)."""
    import torch

    geo, bvh = knot
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 24)
    d_pts = torch.from_numpy(pts).to(cuda)
    res = bvh.closest_point_batch(d_pts, 0.0, 5.0)
    rec = res.cpu().numpy().view(np.uint8).reshape(-1).view(pkg.CLOSEST_DTYPE)
    ok = (rec["face_index"] != 0xFFFFFFFF) & (rec["distance"] > 0.1)
    rng = np.random.default_rng(4)
    g = np.where(ok, rng.normal(size=pts.shape[0]), 0.0).astype(np.float32)
    g64 = g.astype(np.float64)  # float32 * float stays float32 under NumPy 2: keep the quotients in float64
    gv, gp = bvh.closest_point_backward(d_pts, res, torch.from_numpy(g).to(cuda))
    bvh.synchronize()
    gv, gp = gv.cpu().numpy(), gp.cpu().numpy()
    tri_of = geo.index.astype(np.int64).reshape(-1, 3)
    pos0 = geo.position.astype(np.float64)
    faces = rec["face_index"].astype(np.int64)

    def central(f, h):
        return (f(h) - f(-h)) / (2 * h)

    # each gradient is a 3-vector: compared as a vector, relative to its largest component
    compared = 0
    for i in rng.choice(np.nonzero(ok)[0], size=min(4096, int(ok.sum())), replace=False):
        a, b, c = pos0[tri_of[faces[i]]]
        p0 = pts[i].astype(np.float64)
        fd1, fd2 = np.zeros(3), np.zeros(3)
        for k in range(3):
            def f(h, k=k):
                p = p0.copy()
                p[k] += h
                return g64[i] * orc.point_triangle_distance(p, a, b, c)
            fd1[k], fd2[k] = central(f, H), central(f, H / 2)
        scale = max(np.abs(fd1).max(), 1e-3)
        if np.abs(fd1 - fd2).max() > 1e-4 * scale:
            continue
        compared += 1
        assert np.abs(gp[i] - fd1).max() <= REL * scale, (i, gp[i], fd1)
    assert compared > 2048
    q_of = {}
    for i in np.nonzero(ok)[0]:
        for v in tri_of[faces[i]]:
            q_of.setdefault(int(v), []).append(i)
    sample = rng.choice(np.array(sorted(q_of)), size=min(4096, len(q_of)), replace=False)
    compared = 0
    for v in sample:
        fd1, fd2, mag = np.zeros(3), np.zeros(3), np.zeros(3)
        for k in range(3):
            for i in q_of[int(v)]:
                def f(h, v=v, k=k, i=i):
                    p = pos0.copy()
                    p[v, k] += h
                    return g64[i] * orc.point_triangle_distance(pts[i], *p[tri_of[faces[i]]])
                t1 = central(f, H)
                fd1[k] += t1
                fd2[k] += central(f, H / 2)
                mag[k] += abs(t1)
        # measured against the size of the summed terms, as for the ray gradients
        scale = max(np.abs(fd1).max(), mag.max(), 1e-3)
        if np.abs(fd1 - fd2).max() > 1e-4 * scale:
            continue
        compared += 1
        assert np.abs(gv[v] - fd1).max() <= REL * scale, (v, gv[v], fd1)
    assert compared > 2048
