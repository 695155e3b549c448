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
    """L = sum (t - t*)^2 over rays, t* from a perturbed copy; FD over sampled vertices and rays.
    Central differences with h = 1e-3 are only trusted where t is smooth on that scale: rays that
    meet their triangle at grazing incidence (|cos| < 0.3, silhouettes) carry curvature large
    enough to swamp the difference quotient, so they are left out of L here (their exact
    derivatives are checked against the float64 Jacobian above)."""
    import torch

    geo, bvh = knot
    rays = pkg.rays_camera(128, 128)
    d_rays = torch.from_numpy(rays).to(cuda)
    hits = bvh.raycast_first_batch(d_rays)
    rec = _records(pkg, hits)
    hit = rec["face_index"] != 0xFFFFFFFF
    hit &= _cos_incidence(geo, rays, rec["face_index"].astype(np.int64), hit) >= 0.3
    rng = np.random.default_rng(3)
    t_star = rec["distance"].astype(np.float64) + rng.normal(0, 0.01, size=rays.shape[0])
    g = np.where(hit, 2 * (rec["distance"] - t_star), 0.0).astype(np.float32)
    gv, go, gd = bvh.raycast_first_backward(d_rays, hits, torch.from_numpy(g).to(cuda))
    bvh.synchronize()
    gv = gv.cpu().numpy()
    go = go.cpu().numpy()
    faces = rec["face_index"].astype(np.int64)
    tri_of = geo.index.astype(np.int64).reshape(-1, 3)

    def loss_for(ray_ids, pos):
        total = 0.0
        for i in ray_ids:
            a, b, c = pos[tri_of[faces[i]]]
            vals, _ = orc.ray_triangle_jacobian(rays[i, :3], rays[i, 3:], a, b, c)
            total += (vals[0] - t_star[i]) ** 2
        return total

    # vertices: only rays whose recorded triangle uses the vertex depend on it
    used = np.unique(tri_of[faces[hit]])
    sample = rng.choice(used, size=min(256, used.size), replace=False)
    rays_of = {}
    for i in np.nonzero(hit)[0]:
        for v in tri_of[faces[i]]:
            rays_of.setdefault(int(v), []).append(i)
    pos0 = geo.position.astype(np.float64)
    fd = np.zeros((sample.size, 3))
    for s, v in enumerate(sample):
        for k in range(3):
            p = pos0.copy()
            p[v, k] += H
            lp = loss_for(rays_of[int(v)], p)
            p[v, k] -= 2 * H
            lm = loss_for(rays_of[int(v)], p)
            fd[s, k] = (lp - lm) / (2 * H)
    err = np.abs(gv[sample] - fd).max(1) / np.maximum(np.abs(fd).max(1), 1e-3)
    assert err.max() <= REL, np.sort(err)[-5:]
    # ray origins
    for i in rng.choice(np.nonzero(hit)[0], size=64, replace=False):
        a, b, c = pos0[tri_of[faces[i]]]
        fdo = np.zeros(3)
        for k in range(3):
            o = rays[i, :3].astype(np.float64).copy()
            o[k] += H
            vp, _ = orc.ray_triangle_jacobian(o, rays[i, 3:], a, b, c)
            o[k] -= 2 * H
            vm, _ = orc.ray_triangle_jacobian(o, rays[i, 3:], a, b, c)
            fdo[k] = ((vp[0] - t_star[i]) ** 2 - (vm[0] - t_star[i]) ** 2) / (2 * H)
        assert np.abs(go[i] - fdo).max() <= REL * max(np.abs(fdo).max(), 1e-3)


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
    import torch

    geo, bvh = knot
    pts = pkg.grid_points(geo.position.min(0), geo.position.max(0), 16)
    d_pts = torch.from_numpy(pts).to(cuda)
    res = bvh.closest_point_batch(d_pts, 0.0, 5.0)
    rec = res.cpu().numpy().view(np.uint8).reshape(-1).view(pkg.CLOSEST_DTYPE)
    # L = sum of distances over queries at least 0.1 from the surface: closer queries bend the
    # distance field (curvature ~ 1 / distance) too sharply for h = 1e-3 central differences
    ok = (rec["face_index"] != 0xFFFFFFFF) & (rec["distance"] > 0.1)
    g = np.where(ok, 1.0, 0.0).astype(np.float32)
    gv, gp = bvh.closest_point_backward(d_pts, res, torch.from_numpy(g).to(cuda))
    bvh.synchronize()
    gv, gp = gv.cpu().numpy(), gp.cpu().numpy()
    tri_of = geo.index.astype(np.int64).reshape(-1, 3)
    pos0 = geo.position.astype(np.float64)
    faces = rec["face_index"].astype(np.int64)
    rng = np.random.default_rng(4)
    for i in rng.choice(np.nonzero(ok)[0], size=128, replace=False):
        a, b, c = pos0[tri_of[faces[i]]]
        fd = np.zeros(3)
        for k in range(3):
            p = pts[i].astype(np.float64).copy()
            p[k] += H
            dp = orc.point_triangle_distance(p, a, b, c)
            p[k] -= 2 * H
            dm = orc.point_triangle_distance(p, a, b, c)
            fd[k] = (dp - dm) / (2 * H)
        assert np.abs(gp[i] - fd).max() <= REL * max(np.abs(fd).max(), 1e-3), (i, gp[i], fd)
    # vertices
    q_of = {}
    for i in np.nonzero(ok)[0]:
        for v in tri_of[faces[i]]:
            q_of.setdefault(int(v), []).append(i)
    sample = rng.choice(np.array(sorted(q_of)), size=min(128, len(q_of)), replace=False)
    for v in sample:
        fd = np.zeros(3)
        for k in range(3):
            tot = []
            for sgn in (1, -1):
                p = pos0.copy()
                p[v, k] += sgn * H
                tot.append(sum(orc.point_triangle_distance(pts[i], *p[tri_of[faces[i]]]) for i in q_of[int(v)]))
            fd[k] = (tot[0] - tot[1]) / (2 * H)
        assert np.abs(gv[v] - fd).max() <= REL * max(np.abs(fd).max(), 1e-2), (v, gv[v], fd)
