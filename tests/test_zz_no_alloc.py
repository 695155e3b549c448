"""bvhc_raycast_first_noalloc: the raycastFirst entry point for callers that must not allocate
device memory (a fixed budget owned by another framework, a latency-critical thread, a host that
allocates only at start-up).  It is called here through the C ABI and compared with
bvhc_raycast_first, the existing entry point, on two calls in a row (its scratch array is shared
and keeps the previous call's contents, so the second call checks that nothing stale leaks in),
with host and with device buffers.  This file is collected last on purpose, and it also passes on
its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from parity import check_first

pytestmark = pytest.mark.gpu

MAX_HOST_RAYS = 65536
BVHC_ERR_SCRATCH_LIMIT = 8


@pytest.fixture(scope="module")
def mesh(pkg, cuda):
    geo = pkg.torus_knot(10, 3, 400, 100)
    bvh = pkg.MeshBVH(geo, {"strategy": pkg.SAH})
    bvh.set_traversal(1, 1, 16, 0)
    yield bvh
    bvh.dispose()


def _existing(pkg, bvh, rays):
    out = np.empty(rays.shape[0], dtype=pkg.HIT_DTYPE)
    st = pkg.lib().bvhc_raycast_first(bvh._device_mesh(), rays.ctypes.data, rays.shape[0], 0, 0.0, float("inf"),
                                      out.ctypes.data, 0, None)
    assert st == 0
    return out


def _assert_same(got, ref):
    exp = np.zeros(ref.shape[0], dtype=[("face_index", "<i8"), ("distance", "<f8"), ("point", "<f8", 3),
                                         ("barycoord", "<f8", 3)])
    hit = ref["face_index"] != 0xFFFFFFFF
    exp["face_index"] = np.where(hit, ref["face_index"].astype(np.int64), -1)
    exp["distance"] = ref["distance"]
    exp["point"] = ref["point"]
    exp["barycoord"] = ref["barycoord"]
    rep = check_first(got, exp)
    bad = {k: rep[k] for k in ("hitmiss", "face", "distance", "point", "barycoord") if rep[k]}
    assert not bad, rep


def test_host_buffers_two_calls(pkg, mesh):
    lib = pkg.lib()
    for seed in (21, 22):
        rays = pkg.rays_sphere_to_box(MAX_HOST_RAYS, seed=seed)
        out = np.empty(rays.shape[0], dtype=pkg.HIT_DTYPE)
        st = lib.bvhc_raycast_first_noalloc(mesh._device_mesh(), rays.ctypes.data, rays.shape[0], 0, 0.0,
                                            float("inf"), out.ctypes.data, 0, None)
        assert st == 0, lib.bvhc_status_string(st)
        _assert_same(out, _existing(pkg, mesh, rays))


def test_device_buffers_two_calls(pkg, mesh, cuda):
    import torch

    lib = pkg.lib()
    for seed in (23, 24):
        rays = pkg.rays_sphere_to_box(300_000, seed=seed)
        d_rays = torch.from_numpy(rays).to(cuda)
        d_out = torch.empty((rays.shape[0], 8), dtype=torch.float32, device=cuda)
        s = torch.cuda.current_stream().cuda_stream
        st = lib.bvhc_raycast_first_noalloc(mesh._device_mesh(), d_rays.data_ptr(), rays.shape[0], 0, 0.0,
                                            float("inf"), d_out.data_ptr(), 1, s)
        assert st == 0
        assert lib.bvhc_mesh_synchronize(mesh._device_mesh(), s) == 0
        got = d_out.cpu().numpy().view(np.uint8).reshape(-1).view(pkg.HIT_DTYPE)
        _assert_same(got, _existing(pkg, mesh, rays))


def test_rejects_host_batches_over_the_scratch_size(pkg, mesh):
    lib = pkg.lib()
    rays = pkg.rays_sphere_to_box(MAX_HOST_RAYS + 1, seed=25)
    out = np.empty(rays.shape[0], dtype=pkg.HIT_DTYPE)
    st = lib.bvhc_raycast_first_noalloc(mesh._device_mesh(), rays.ctypes.data, rays.shape[0], 0, 0.0, float("inf"),
                                        out.ctypes.data, 0, None)
    assert st == BVHC_ERR_SCRATCH_LIMIT
    assert b"65536" in lib.bvhc_status_string(st)
