// Adjoint (backward) kernels: gradients of raycastFirst's reported distance and barycentrics, and
// of closestPointToPoint's distance, with respect to vertex positions, ray origins / directions and
// query points.  No reference counterpart: the forward values are the reference's, the backward
// differentiates the same formulas.  Each kernel replays only the recorded triangle of a query (one
// thread per ray / point), so its cost is independent of the BVH.
//
// Ray / triangle (the Eberly determinant form the forward evaluates): with q = o - a, e1 = b - a,
// e2 = c - a and det(x, y, z) = x . (y x z),
//   N = det(d, e1, e2), U = det(d, q, e2), V = det(d, e1, q), T = det(q, e1, e2),
//   t = -T / N,  wb = U / N,  wc = V / N,  wa = 1 - wb - wc,  distance = t |d|.
// Reverse mode: gT = -g_t / N, gU = g_wb / N, gV = g_wc / N, gN = -(g_t t + g_wb wb + g_wc wc) / N, and
// each determinant's partials are cross products of the other two arguments, e.g.
// d det(x,y,z)/dx = y x z.  For g_wb = g_wc = 0 this reduces to dt/dv_k = w_k n / N,
// dt/do = -n / N and dt/dd = -t n / N with n = e1 x e2.
// Evaluated as written, the q-terms are products of |o - a| (the ray length scale) with 1 / N (the
// inverse triangle area scale) that cancel down to the triangle scale, losing about
// log2(|o - a| / |e|) bits in float32.  The kernel therefore substitutes q = q' - t d with
// q' = h - a = wb e1 + wc e2 (the hit point, from the recorded barycentrics): the d x d terms vanish,
// gN - t gT = -(g_wb wb + g_wc wc) / N drops the t-proportional parts, and dL/dd picks up t dL/do.
// Every remaining term is of the triangle's own scale.
//
// Closest point: for the distance dist = |p - c| to the closest point c = sum_k beta_k v_k of the
// recorded triangle, the envelope theorem gives d dist / dp = (p - c) / dist and
// d dist / dv_k = -beta_k (p - c) / dist (beta: barycentrics of c; zero gradient at dist = 0).
// c and beta are recomputed in float-float from the recorded triangle (Ericson's region method),
// so p - c carries no rounding of the reported float32 point and beta is exactly 0 for the
// vertices outside c's edge or vertex region.
//
// Vertex gradients are accumulated with atomicAdd; lanes of a warp that recorded the same face are
// first summed with warp shuffles so that the face's three vertices receive one atomic per
// component from the whole group.
#include <cuda_runtime.h>

#include <cstdint>

#include "bvhcuda.h"
#include "kernels.cuh"
#include "robust.cuh"

namespace bvhc {
namespace dev {

constexpr int kAdjBlock = 256;

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 mul3(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

__device__ __forceinline__ float3 load_vertex(const float* pos, uint32_t v) {
  return f3(__ldg(pos + 3 * v), __ldg(pos + 3 * v + 1), __ldg(pos + 3 * v + 2));
}

__device__ __forceinline__ float warp_sum(float x, unsigned mask) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(mask, x, o);
  return x;
}

// Adds g[k] (three float3) into vertices vid[k]; lanes with the same `face` are summed first.
__device__ __forceinline__ void scatter_vertex_grads(float* grad, uint32_t face, bool valid, const uint32_t vid[3],
                                                     const float3 g[3]) {
  const unsigned full = 0xFFFFFFFFu;
  unsigned key = valid ? face : 0xFFFFFFFFu;
  unsigned same = __match_any_sync(full, key);
  bool shared = __ballot_sync(full, valid && __popc(same) > 1) != 0u;
  if (!shared) {
    if (valid) {
      for (int k = 0; k < 3; ++k) {
        atomicAdd(grad + 3 * vid[k], g[k].x);
        atomicAdd(grad + 3 * vid[k] + 1, g[k].y);
        atomicAdd(grad + 3 * vid[k] + 2, g[k].z);
      }
    }
    return;
  }
  // one group (a distinct face) per round: every lane takes part in the shuffles
  unsigned remaining = __ballot_sync(full, valid);
  const unsigned lane = threadIdx.x & 31u;
  while (remaining) {
    unsigned leader = __ffs(remaining) - 1;
    unsigned leader_key = __shfl_sync(full, key, leader);
    bool mine = valid && key == leader_key;
    unsigned group = __ballot_sync(full, mine);
    float s[9];
    for (int k = 0; k < 3; ++k) {
      s[3 * k] = warp_sum(mine ? g[k].x : 0.0f, full);
      s[3 * k + 1] = warp_sum(mine ? g[k].y : 0.0f, full);
      s[3 * k + 2] = warp_sum(mine ? g[k].z : 0.0f, full);
    }
    if (lane == leader) {
      for (int k = 0; k < 3; ++k) {
        atomicAdd(grad + 3 * vid[k], s[3 * k]);
        atomicAdd(grad + 3 * vid[k] + 1, s[3 * k + 1]);
        atomicAdd(grad + 3 * vid[k] + 2, s[3 * k + 2]);
      }
    }
    remaining &= ~group;
  }
}

__global__ void __launch_bounds__(kAdjBlock) raycast_first_backward_kernel(
    const uint32_t* __restrict__ index, const float* __restrict__ pos, const float* __restrict__ rays,
    const bvhc_hit* __restrict__ hits, uint64_t n, const float* __restrict__ g_dist, const float* __restrict__ g_bary,
    float* __restrict__ g_vert, float* __restrict__ g_orig, float* __restrict__ g_dir) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool in = i < n;
  uint32_t face = in ? hits[i].face_index : BVHC_NO_HIT;
  bool valid = in && face != BVHC_NO_HIT;
  uint32_t vid[3] = {0, 0, 0};
  float3 gv[3] = {f3(0, 0, 0), f3(0, 0, 0), f3(0, 0, 0)};
  float3 go = f3(0, 0, 0), gd = f3(0, 0, 0);
  if (valid) {
    for (int k = 0; k < 3; ++k) vid[k] = __ldg(index + 3 * (uint64_t)face + k);
    float3 a = load_vertex(pos, vid[0]), b = load_vertex(pos, vid[1]), c = load_vertex(pos, vid[2]);
    const float* r = rays + 6 * i;
    float3 o = f3(r[0], r[1], r[2]), d = f3(r[3], r[4], r[5]);
    float3 e1 = sub3(b, a), e2 = sub3(c, a);
    float3 nrm = cross3(e1, e2);
    float N = dot3(d, nrm);
    float dl = sqrtf(dot3(d, d));
    // t and the barycentrics of the hit, as recorded by the forward pass (float-float, rounded once)
    float t = dl > 0.0f ? hits[i].distance / dl : 0.0f;
    float wb = hits[i].barycoord[1], wc = hits[i].barycoord[2];
    // q' = h - a, the hit point relative to a: the ray re-anchored at its hit point (o = h - t d)
    float3 qp;
    if (hits[i].barycoord[0] == 0.0f && wb == 0.0f && wc == 0.0f) {
      // the forward reported (0, 0, 0) for a triangle of vanishing area: fall back to q = o - a
      float3 q = sub3(o, a);
      wb = dot3(d, cross3(q, e2)) / N;
      wc = dot3(d, cross3(e1, q)) / N;
      qp = add3(q, mul3(d, t));
    } else {
      qp = add3(mul3(e1, wb), mul3(e2, wc));
    }
    float gdist = g_dist ? g_dist[i] : 0.0f;
    float gt = gdist * dl;
    float gwa = 0.0f, gwb = 0.0f, gwc = 0.0f;
    if (g_bary) {
      gwa = g_bary[3 * i];
      gwb = g_bary[3 * i + 1] - gwa;
      gwc = g_bary[3 * i + 2] - gwa;
    }
    float iN = 1.0f / N;
    float gT = -gt * iN, gU = gwb * iN, gV = gwc * iN;
    // gN - t gT: the t-proportional parts of gN and of the q-terms cancel analytically
    float gNp = -(gwb * wb + gwc * wc) * iN;
    float3 gq = add3(add3(mul3(cross3(e2, d), gU), mul3(cross3(d, e1), gV)), mul3(nrm, gT));
    float3 ge1 = add3(add3(mul3(cross3(qp, d), gV), mul3(cross3(e2, d), gNp)), mul3(cross3(e2, qp), gT));
    float3 ge2 = add3(add3(mul3(cross3(d, qp), gU), mul3(cross3(d, e1), gNp)), mul3(cross3(qp, e1), gT));
    gd = add3(add3(add3(mul3(cross3(qp, e2), gU), mul3(cross3(e1, qp), gV)), mul3(nrm, gNp)), mul3(gq, t));
    if (dl > 0.0f) gd = add3(gd, mul3(d, gdist * t / dl));
    go = gq;
    gv[0] = mul3(add3(add3(gq, ge1), ge2), -1.0f);
    gv[1] = ge1;
    gv[2] = ge2;
  }
  if (in) {
    if (g_orig) {
      g_orig[3 * i] = go.x;
      g_orig[3 * i + 1] = go.y;
      g_orig[3 * i + 2] = go.z;
    }
    if (g_dir) {
      g_dir[3 * i] = gd.x;
      g_dir[3 * i + 1] = gd.y;
      g_dir[3 * i + 2] = gd.z;
    }
  }
  if (g_vert) scatter_vertex_grads(g_vert, face, valid, vid, gv);
}

__global__ void __launch_bounds__(kAdjBlock) closest_point_backward_kernel(
    const uint32_t* __restrict__ index, const float* __restrict__ pos, const float* __restrict__ pts,
    const bvhc_closest* __restrict__ res, uint64_t n, const float* __restrict__ g_dist, float* __restrict__ g_vert,
    float* __restrict__ g_pts) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  bool in = i < n;
  uint32_t face = in ? res[i].face_index : BVHC_NO_HIT;
  bool valid = in && face != BVHC_NO_HIT && res[i].distance > 0.0f;
  uint32_t vid[3] = {0, 0, 0};
  float3 gv[3] = {f3(0, 0, 0), f3(0, 0, 0), f3(0, 0, 0)};
  float3 gp = f3(0, 0, 0);
  if (valid) {
    for (int k = 0; k < 3; ++k) vid[k] = __ldg(index + 3 * (uint64_t)face + k);
    float3 a = load_vertex(pos, vid[0]), b = load_vertex(pos, vid[1]), c = load_vertex(pos, vid[2]);
    float3 p = f3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    // The closest point again, in float-float: p - c without the rounding of the reported point
    // (whose error divided by the distance would enter u directly), and the barycentrics of its
    // Voronoi region (exactly zero for the vertices an edge or vertex region leaves out).
    CPFF cf = closest_ff(p, a, b, c);
    float dist = ff_to_f(ff_sqrt(cf.d2));
    float g = g_dist[i];
    if (dist > 0.0f) {
      float id = 1.0f / dist;
      float3 u = f3(ff_to_f(cf.r.x) * id, ff_to_f(cf.r.y) * id, ff_to_f(cf.r.z) * id);
      gp = mul3(u, g);
      float wa = 1.0f - cf.wb - cf.wc;
      gv[0] = mul3(u, -g * wa);
      gv[1] = mul3(u, -g * cf.wb);
      gv[2] = mul3(u, -g * cf.wc);
    }
  }
  if (in && g_pts) {
    g_pts[3 * i] = gp.x;
    g_pts[3 * i + 1] = gp.y;
    g_pts[3 * i + 2] = gp.z;
  }
  if (g_vert) scatter_vertex_grads(g_vert, face, valid, vid, gv);
}

}  // namespace dev

cudaError_t launch_raycast_first_backward(const uint32_t* index, const float* pos, const float* rays,
                                          const bvhc_hit* hits, uint64_t n, const float* g_dist, const float* g_bary,
                                          float* g_vert, float* g_orig, float* g_dir, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  unsigned int grid = (unsigned int)((n + dev::kAdjBlock - 1) / dev::kAdjBlock);
  dev::raycast_first_backward_kernel<<<grid, dev::kAdjBlock, 0, stream>>>(index, pos, rays, hits, n, g_dist, g_bary,
                                                                          g_vert, g_orig, g_dir);
  return cudaGetLastError();
}

cudaError_t launch_closest_point_backward(const uint32_t* index, const float* pos, const float* pts,
                                          const bvhc_closest* res, uint64_t n, const float* g_dist, float* g_vert,
                                          float* g_pts, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  unsigned int grid = (unsigned int)((n + dev::kAdjBlock - 1) / dev::kAdjBlock);
  dev::closest_point_backward_kernel<<<grid, dev::kAdjBlock, 0, stream>>>(index, pos, pts, res, n, g_dist, g_vert,
                                                                          g_pts);
  return cudaGetLastError();
}

}  // namespace bvhc
