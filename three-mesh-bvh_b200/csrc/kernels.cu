// Traversal kernels: raycastFirst, raycast (all hits) and closestPointToPoint.
//
// One ray or query per thread.  Each visit of an internal node reads one 64-byte child-pair
// record (both child boxes and links) with four 16-byte read-only loads; each leaf is a
// contiguous run of 48-byte triangle records.  The traversal stack lives in thread-local
// memory (L1-resident), bounded by kMaxStack; the mesh upload rejects deeper trees, and an
// overflow would set the device error word instead of faulting.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cstdint>

#include "kernels.cuh"
#include "raykey.cuh"
#include "robust.cuh"
#include "softf64.cuh"

namespace bvhc {
namespace dev {

constexpr int kBlock = 128;
constexpr float kInf = __builtin_huge_valf();
constexpr float kSlabMargin = 9.5367431640625e-07f;  // 2^-20, relative slack on slab distances
constexpr float kTiny = 1e-30f;                      // stand-in for a zero direction component

__device__ __forceinline__ float4 ld4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }

struct RayF {
  float3 o, d, inv;
  float d_l1;
};

__device__ __forceinline__ RayF make_ray(const float* __restrict__ rays, uint64_t i) {
  const float2* p = reinterpret_cast<const float2*>(rays + 6 * i);
  // rays are read once: streaming loads keep them from evicting the BVH from L2
  float2 r0 = __ldcs(p), r1 = __ldcs(p + 1), r2 = __ldcs(p + 2);
  RayF r;
  r.o = make_float3(r0.x, r0.y, r1.x);
  r.d = make_float3(r1.y, r2.x, r2.y);
  // A zero component is replaced by +-1e-30 so that (bound - origin) * inv is never 0 * inf:
  // the slab then becomes (-huge, +huge) or empty, which is what the reference's NaN guards in
  // intersectsNodeBounds (intersectUtils.js:52-54,70-72) amount to.
  float dx = fabsf(r.d.x) < kTiny ? copysignf(kTiny, r.d.x) : r.d.x;
  float dy = fabsf(r.d.y) < kTiny ? copysignf(kTiny, r.d.y) : r.d.y;
  float dz = fabsf(r.d.z) < kTiny ? copysignf(kTiny, r.d.z) : r.d.z;
  r.inv = make_float3(__frcp_rn(dx), __frcp_rn(dy), __frcp_rn(dz));
  r.d_l1 = fabsf(r.d.x) + fabsf(r.d.y) + fabsf(r.d.z);
  return r;
}

// Conservative slab test (intersectUtils.js:2-78).  Accepts whenever the reference's float64
// test could accept: the entry/exit distances carry at most ~3 roundings, and are widened by
// 2^-20 relative before the comparisons.  `entry` returns the widened entry distance.
__device__ __forceinline__ bool box_hit(float x0, float y0, float z0, float x1, float y1, float z1, const RayF& r,
                                        float near_d, float far_d, float& entry) {
  float tx0 = (x0 - r.o.x) * r.inv.x, tx1 = (x1 - r.o.x) * r.inv.x;
  float ty0 = (y0 - r.o.y) * r.inv.y, ty1 = (y1 - r.o.y) * r.inv.y;
  float tz0 = (z0 - r.o.z) * r.inv.z, tz1 = (z1 - r.o.z) * r.inv.z;
  float en = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
  float ex = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
  en *= en > 0.0f ? 1.0f - kSlabMargin : 1.0f + kSlabMargin;
  ex *= ex > 0.0f ? 1.0f + kSlabMargin : 1.0f - kSlabMargin;
  entry = en;
  return en <= ex && en <= far_d && ex >= near_d;
}

struct Tri {
  float3 a, b, c;
  uint32_t face, flags, material;
};

__device__ __forceinline__ Tri load_tri(const TriRecord* __restrict__ tris, uint32_t k) {
  const TriRecord* t = tris + k;
  float4 p0 = ld4(&t->v[0]), p1 = ld4(&t->v[4]), p2 = ld4(&t->v[8]);
  Tri r;
  r.a = make_float3(p0.x, p0.y, p0.z);
  r.b = make_float3(p0.w, p1.x, p1.y);
  r.c = make_float3(p1.z, p1.w, p2.x);
  r.face = __float_as_uint(p2.y);
  r.flags = __float_as_uint(p2.z);
  r.material = __float_as_uint(p2.w);
  return r;
}

// The side a triangle is tested with: the call's side, or with an array of materials the side of
// the triangle's group material (ThreeRayIntersectUtilities.js:170-205; a material index past the
// array reads as `undefined` and tests like FrontSide).  -1: the triangle is in no group and is
// not tested.
__device__ __forceinline__ int tri_side(const Tri& t, int side, const SideTable& tab) {
  if (!tab.per_material) return side;
  if (t.material == kNoMaterial) return -1;
  return t.material < (uint32_t)tab.n ? (int)tab.side[t.material] : kSideFront;
}

struct Pair {
  float l[6], r[6];
  uint32_t ll, lr, axis;
};

__device__ __forceinline__ Pair load_pair(const PairNode* __restrict__ nodes, uint32_t k) {
  const PairNode* n = nodes + k;
  float4 q0 = ld4(&n->f[0]), q1 = ld4(&n->f[4]), q2 = ld4(&n->f[8]), q3 = ld4(&n->link[0]);
  Pair p;
  p.l[0] = q0.x; p.l[1] = q0.y; p.l[2] = q0.z; p.l[3] = q0.w; p.l[4] = q1.x; p.l[5] = q1.y;
  p.r[0] = q1.z; p.r[1] = q1.w; p.r[2] = q2.x; p.r[3] = q2.y; p.r[4] = q2.z; p.r[5] = q2.w;
  p.ll = __float_as_uint(q3.x);
  p.lr = __float_as_uint(q3.y);
  p.axis = __float_as_uint(q3.z);
  return p;
}

// |d| in float-float.
__device__ __forceinline__ ff dir_length(float3 d) {
  ff s = ff_add(ff_add(two_prod(d.x, d.x), two_prod(d.y, d.y)), two_prod(d.z, d.z));
  return ff_sqrt(s);
}

// Full intersection record for a triangle known to be hit, in float-float, rounded once.
// barycoord follows Triangle.getBarycoord: (0, 0, 0) when the triangle's Gram determinant
// |e1 x e2|^2 vanishes at float64 resolution (the reference's `denom === 0` case).
__device__ void make_hit(const Tri& t, const RayF& r, ff tt, ff dist, bvhc_hit& h) {
  TriFF e = tri_eval_ff(t.a, t.b, t.c, r.o, r.d);
  ff3 px = {ff_add(ff_from(r.o.x), ff_mul_f(tt, r.d.x)), ff_add(ff_from(r.o.y), ff_mul_f(tt, r.d.y)),
            ff_add(ff_from(r.o.z), ff_mul_f(tt, r.d.z))};
  h.face_index = t.face;
  h.distance = ff_to_f(dist);
  h.point[0] = ff_to_f(px.x);
  h.point[1] = ff_to_f(px.y);
  h.point[2] = ff_to_f(px.z);
  ff3 e1 = ff3_diff(t.b, t.a), e2 = ff3_diff(t.c, t.a);
  ff3 n = ff3_cross(e1, e2);
  ff g = ff3_dot(n, n);
  ff l12 = ff_mul(ff3_dot(e1, e1), ff3_dot(e2, e2));
  if (g.hi <= 8.8817841970012523e-16f * l12.hi) {  // 2^-50
    h.barycoord[0] = h.barycoord[1] = h.barycoord[2] = 0.0f;
  } else {
    h.barycoord[0] = ff_to_f(ff_div(e.W, e.N));
    h.barycoord[1] = ff_to_f(ff_div(e.U, e.N));
    h.barycoord[2] = ff_to_f(ff_div(e.V, e.N));
  }
}

__device__ __forceinline__ void store_hit(bvhc_hit* p, const bvhc_hit& h) {
  float4* q = reinterpret_cast<float4*>(p);
  __stcs(q, make_float4(__uint_as_float(h.face_index), h.distance, h.point[0], h.point[1]));
  __stcs(q + 1, make_float4(h.point[2], h.barycoord[0], h.barycoord[1], h.barycoord[2]));
}

__device__ __forceinline__ void store_miss(bvhc_hit* p) {
  float4* q = reinterpret_cast<float4*>(p);
  __stcs(q, make_float4(__uint_as_float(BVHC_NO_HIT), kInf, 0.0f, 0.0f));
  __stcs(q + 1, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
}

// ---------------------------------------------------------------------------------------------
// raycastFirst leaf step shared by both kernel forms.  Candidate hits are ordered with float32 t
// values and their error bounds; float-float only settles candidates the bounds cannot separate
// (the reference keeps the strictly closer one; exact ties keep the candidate found first).
// ---------------------------------------------------------------------------------------------
constexpr float kTwoU = 1.1920928955078125e-07f;  // 2u

// near <= dist <= far for dist = t |d|, decided with the float32 bounds, else in float-float.
__device__ __forceinline__ bool in_range(float t, float t_err, const Tri& tr, const RayF& r, float dlen, float near_d,
                                         float far_d) {
  float dist = t * dlen;
  float derr = t_err * dlen + fabsf(dist) * kTwoU + 1e-30f;
  if (dist - derr >= near_d && dist + derr <= far_d) return true;
  if (dist + derr < near_d || dist - derr > far_d) return false;
  ff dl = ff_mul(tri_t_ff(tri_eval_ff(tr.a, tr.b, tr.c, r.o, r.d)), dir_length(r.d));
  return !ff_lt(dl, ff_from(near_d)) && !ff_lt(ff_from(far_d), dl);
}

struct Best {
  float t, err;
  uint32_t rec;
};

__device__ __forceinline__ void leaf_first(const MeshDev& m, uint32_t k, const RayF& r, float dlen, int side,
                                           const SideTable& sides, float near_d, float far_d, Best& best) {
  for (;;) {
    Tri t = load_tri(m.tris, k);
    int ts = tri_side(t, side, sides);
    float th, te;
    if (ts >= 0 && tri_hit_t(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts, th, te) &&
        in_range(th, te, t, r, dlen, near_d, far_d)) {
      bool take;
      if (best.rec == 0xFFFFFFFFu || th + te < best.t - best.err) {
        take = true;
      } else if (th - te > best.t + best.err) {
        take = false;
      } else {
        Tri bt = load_tri(m.tris, best.rec);
        ff tn = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, r.o, r.d));
        ff tb = tri_t_ff(tri_eval_ff(bt.a, bt.b, bt.c, r.o, r.d));
        take = ff_lt(tn, tb);
        if (take) {
          th = tn.hi;
          te = fabsf(tn.hi) * kTinyRel + 1e-30f;
        }
      }
      if (take) {
        best.t = th;
        best.err = te;
        best.rec = k;
      }
    }
    if (t.flags & kTriLast) break;
    ++k;
  }
}

// The reported record of the best hit: t, distance, point and barycentrics in float-float.
__device__ __forceinline__ void finish_first(const MeshDev& m, uint32_t rec, const RayF& r, bvhc_hit* o) {
  if (rec == 0xFFFFFFFFu) {
    store_miss(o);
    return;
  }
  Tri t = load_tri(m.tris, rec);
  ff tt = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, r.o, r.d));
  bvhc_hit h;
  make_hit(t, r, tt, ff_mul(tt, dir_length(r.d)), h);
  store_hit(o, h);
}

// ---------------------------------------------------------------------------------------------
// raycastFirst (raycastFirst.template.js:19-103, roots loop MeshBVH.js:558-577), one ray per
// thread.  ORDER 0 visits the near child by the sign of the ray direction on the split axis, as
// the reference does; ORDER 1 by the smaller entry distance.  A child whose (widened) entry
// distance is beyond the best hit so far is skipped, which can only drop triangles that are
// farther than that hit.
// ---------------------------------------------------------------------------------------------
template <int ORDER>
__device__ __forceinline__ bool left_first(const Pair& p, const RayF& r, float e0, float e1) {
  if (ORDER == 0) {
    float dir_axis = p.axis == 0 ? r.d.x : (p.axis == 1 ? r.d.y : r.d.z);
    return dir_axis >= 0.0f;
  }
  return e0 <= e1;
}

template <int ORDER>
__global__ void __launch_bounds__(kBlock) raycast_first_kernel(MeshDev m, const float* __restrict__ rays, uint64_t n,
                                                               int side, const SideTable sides, float near_d,
                                                               float far_d, bvhc_hit* __restrict__ out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  RayF r = make_ray(rays, i);
  float dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  uint32_t stack_link[kMaxStack];
  float stack_t[kMaxStack];
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      if (link & kLeafBit) {
        if (link != kEmptyLeaf) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
      } else {
        Pair p = load_pair(m.nodes, link);
        float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
        float e0, e1;
        bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
        bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
        bool lf = left_first<ORDER>(p, r, e0, e1);
        uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
        bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
        if (h1st) {
          if (h2nd) {
            if (sp >= kMaxStack) {
              atomicOr(m.err, kErrStackOverflow);
              store_miss(out + i);
              return;
            }
            stack_link[sp] = c2;
            stack_t[sp] = lf ? e1 : e0;
            ++sp;
          }
          link = c1;
          continue;
        }
        if (h2nd) {
          link = c2;
          continue;
        }
      }
      // pop, skipping entries that start beyond the best hit found since they were pushed
      bool found = false;
      float lim = (best.t + best.err) * (1.0f + kSlabMargin);
      while (sp > 0) {
        --sp;
        if (stack_t[sp] <= lim) {
          link = stack_link[sp];
          found = true;
          break;
        }
      }
      if (!found) break;
    }
  }
  finish_first(m, best.rec, r, out + i);
}

// ---------------------------------------------------------------------------------------------
// raycastFirst, warp-cooperative form for coherent rays (camera rays in pixel order).  The 32
// rays of a warp walk the tree together with one shared stack: every child pair is fetched once
// for the warp (a broadcast load), each lane tests it against its own ray, and the warp enters a
// child if any lane's ray enters it (nearest first by majority vote).  A leaf is tested by all
// lanes at once, so the triangle tests run at full SIMD width.  Each lane keeps its own entry
// distance for every stacked child; a stacked child is skipped when no lane still needs it.
// Visiting a node a lane's ray does not enter costs that lane nothing but idle time, and testing
// a triangle it would not have reached cannot change its closest hit.
// ---------------------------------------------------------------------------------------------
constexpr int kWarps = kBlock / 32;

template <int ORDER, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) raycast_first_packet_kernel(MeshDev m, const float* __restrict__ rays,
                                                                      uint64_t n, int side, const SideTable sides,
                                                                      float near_d, float far_d,
                                                                      bvhc_hit* __restrict__ out,
                                                                      const uint32_t* __restrict__ queue,
                                                                      const unsigned int* __restrict__ qcount) {
  __shared__ uint32_t s_link[kWarps][kMaxStack];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  // with a queue (root-box pre-pass, optionally sorted) a warp takes 32 consecutive queue entries
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  RayF r;
  float dlen = 1.0f;
  if (valid) {
    r = make_ray(rays, i);
    dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  } else {
    r.o = make_float3(0.f, 0.f, 0.f);
    r.d = make_float3(1.f, 0.f, 0.f);
    r.inv = make_float3(1.f, 1e30f, 1e30f);
    r.d_l1 = 1.f;
  }
  const unsigned valid_mask = __ballot_sync(full, valid);
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  float lane_t[kMaxStack];
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && valid) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
        pop = true;
      } else {
        Pair p = load_pair(m.nodes, link);
        float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
        float e0, e1;
        bool h0 = valid && box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
        bool h1 = valid && box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
        unsigned b0 = __ballot_sync(full, h0), b1 = __ballot_sync(full, h1);
        if (b0 && b1) {
          bool lf = left_first<ORDER>(p, r, e0, e1);
          bool left_wins = 2 * __popc(__ballot_sync(full, valid && lf)) >= __popc(valid_mask);
          if (sp >= kMaxStack) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            best.rec = 0xFFFFFFFFu;
            root = m.n_roots;
            break;
          }
          if (lane == 0) s_link[w][sp] = left_wins ? p.lr : p.ll;
          lane_t[sp] = left_wins ? (h1 ? e1 : kInf) : (h0 ? e0 : kInf);
          ++sp;
          link = left_wins ? p.ll : p.lr;
          __syncwarp();
        } else if (b0) {
          link = p.ll;
        } else if (b1) {
          link = p.lr;
        } else {
          pop = true;
        }
      }
      if (pop) {
        bool found = false;
        while (sp > 0) {
          --sp;
          float lim = (best.t + best.err) * (1.0f + kSlabMargin);
          if (__ballot_sync(full, valid && lane_t[sp] <= lim)) {
            link = s_link[w][sp];
            found = true;
            break;
          }
        }
        if (!found) break;
      }
    }
  }
  if (valid) finish_first(m, best.rec, r, out + i);
}

// ---------------------------------------------------------------------------------------------
// raycastFirst, warp-cooperative over the four-child records (m.quads): the same shared traversal
// as above with half as many node visits.  At a record each lane tests the four child boxes (one
// 16-byte load per bound plane serves all four); the children any lane enters are ordered by the
// entry distances of the first lane that enters one (the warp's rays are coherent), the nearest is
// visited and the others are stacked farthest first, each with every lane's own entry distance.
// ---------------------------------------------------------------------------------------------
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) raycast_first_packet4_kernel(
    MeshDev m, const float* __restrict__ rays, uint64_t n, int side, const SideTable sides, float near_d,
    float far_d, bvhc_hit* __restrict__ out, const uint32_t* __restrict__ queue,
    const unsigned int* __restrict__ qcount) {
  __shared__ uint32_t s_link[kWarps][kMaxStack];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  RayF r;
  float dlen = 1.0f;
  if (valid) {
    r = make_ray(rays, i);
    dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  } else {
    r.o = make_float3(0.f, 0.f, 0.f);
    r.d = make_float3(1.f, 0.f, 0.f);
    r.inv = make_float3(1.f, 1e30f, 1e30f);
    r.d_l1 = 1.f;
  }
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  float lane_t[kMaxStack];
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.quad_roots[root];
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && valid) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
        pop = true;
      } else {
        const QuadNode* qn = m.quads + link;
        const float4 lx = ld4(qn->lo[0]), ly = ld4(qn->lo[1]), lz = ld4(qn->lo[2]);
        const float4 hx = ld4(qn->hi[0]), hy = ld4(qn->hi[1]), hz = ld4(qn->hi[2]);
        const float4 lk = ld4(qn->link);
        const uint32_t ck[4] = {__float_as_uint(lk.x), __float_as_uint(lk.y), __float_as_uint(lk.z),
                                __float_as_uint(lk.w)};
        const float blo[3][4] = {{lx.x, lx.y, lx.z, lx.w}, {ly.x, ly.y, ly.z, ly.w}, {lz.x, lz.y, lz.z, lz.w}};
        const float bhi[3][4] = {{hx.x, hx.y, hx.z, hx.w}, {hy.x, hy.y, hy.z, hy.w}, {hz.x, hz.y, hz.z, hz.w}};
        const float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
        float e[4];
        bool h[4];
        unsigned b[4];
        unsigned any = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          h[c] = valid && ck[c] != kEmptyLeaf &&
                 box_hit(blo[0][c], blo[1][c], blo[2][c], bhi[0][c], bhi[1][c], bhi[2][c], r, near_d, lim, e[c]);
          b[c] = __ballot_sync(full, h[c]);
          any |= b[c];
        }
        if (!any) {
          pop = true;
        } else {
          const int leader = __ffs(any) - 1;
          float key[4];
          int idx[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float kc = __shfl_sync(full, h[c] ? e[c] : kInf, leader);
            key[c] = b[c] ? kc : kInf;
            idx[c] = c;
          }
          // sort the four (key, child) pairs, nearest first (warp-uniform values)
          auto cas = [&](int a, int c) {
            if (key[c] < key[a]) {
              float tk = key[a]; key[a] = key[c]; key[c] = tk;
              int ti = idx[a]; idx[a] = idx[c]; idx[c] = ti;
            }
          };
          cas(0, 1); cas(2, 3); cas(0, 2); cas(1, 3); cas(1, 2);
          if (sp + 3 > kMaxStack) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            best.rec = 0xFFFFFFFFu;
            root = m.n_roots;
            break;
          }
          // children that some lane enters, farthest pushed first; the nearest is visited now
          uint32_t next = kEmptyLeaf;
          bool have_next = false;
#pragma unroll
          for (int j = 3; j >= 0; --j) {
            const int c = idx[j];
            if (!b[c]) continue;
            if (j == 0) {
              next = ck[c];
              have_next = true;
            } else {
              if (lane == 0) s_link[w][sp] = ck[c];
              lane_t[sp] = h[c] ? e[c] : kInf;
              ++sp;
            }
          }
          if (have_next) {
            link = next;
          } else {  // the first key belonged to a child no lane enters: every entered one was stacked
            pop = true;
          }
          __syncwarp();
        }
      }
      if (pop) {
        bool found = false;
        while (sp > 0) {
          --sp;
          float plim = (best.t + best.err) * (1.0f + kSlabMargin);
          if (__ballot_sync(full, valid && lane_t[sp] <= plim)) {
            link = s_link[w][sp];
            found = true;
            break;
          }
        }
        if (!found) break;
      }
    }
  }
  if (valid) finish_first(m, best.rec, r, out + i);
}

// ---------------------------------------------------------------------------------------------
// raycast, all hits (raycast.template.js:15-53): left child then right child, every hit kept
// in DFS order.  The first `cap` hits are stored; counts[i] is the uncapped total.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kBlock) raycast_all_kernel(MeshDev m, const float* __restrict__ rays, uint64_t n,
                                                             int side, const SideTable sides, float near_d,
                                                             float far_d, uint32_t cap, uint32_t* __restrict__ counts,
                                                             bvhc_hit* __restrict__ hits,
                                                             const uint32_t* __restrict__ queue = nullptr,
                                                             const unsigned int* __restrict__ qcount = nullptr) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // with a queue, thread i traces ray queue[i] (the rays the pre-pass found entering the tree)
  if (queue) {
    if (i >= (uint64_t)__ldg(qcount)) return;
    i = __ldg(queue + i);
  }
  if (i >= n) return;
  RayF r = make_ray(rays, i);
  ff dlen = dir_length(r.d);
  uint32_t cnt = 0;
  uint32_t stack_link[kMaxStack];
  bvhc_hit* out = hits + i * (uint64_t)cap;
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      if (link & kLeafBit) {
        if (link != kEmptyLeaf) {
          uint32_t k = link & ~kLeafBit;
          for (;;) {
            Tri t = load_tri(m.tris, k);
            int ts = tri_side(t, side, sides);
            if (ts >= 0 && tri_hit(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts)) {
              ff tt = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, r.o, r.d));
              ff dist = ff_mul(tt, dlen);
              if (!ff_lt(dist, ff_from(near_d)) && !ff_lt(ff_from(far_d), dist)) {
                if (cnt < cap) {
                  bvhc_hit h;
                  make_hit(t, r, tt, dist, h);
                  store_hit(out + cnt, h);
                }
                ++cnt;
              }
            }
            if (t.flags & kTriLast) break;
            ++k;
          }
        }
      } else {
        Pair p = load_pair(m.nodes, link);
        float e0, e1;
        bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e0);
        bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e1);
        if (h0) {
          if (h1) {
            if (sp >= kMaxStack) {
              atomicOr(m.err, kErrStackOverflow);
              counts[i] = cnt;
              return;
            }
            stack_link[sp++] = p.lr;
          }
          link = p.ll;
          continue;
        }
        if (h1) {
          link = p.lr;
          continue;
        }
      }
      if (sp == 0) break;
      link = stack_link[--sp];
    }
  }
  counts[i] = cnt;
}

// raycast (all hits), persistent: warps take the rays the pre-pass queued through one work
// counter, and once kAllRefill lanes of a warp have finished their rays those lanes take the next
// ones (one atomic per refill for the whole warp).  The rays that enter the tree have traversal
// lengths from ~10 to ~1000 node reads, so a warp that only took new rays when all 32 were done
// would spend most of its time waiting on its longest one.  Each lane walks its ray exactly as
// raycast_all_kernel does (left child before right, every hit in DFS order).
constexpr int kAllRefill = 8;
constexpr int kAllBlocksPerSm = 8;

// 8 resident blocks per SM (64 registers), so that the launch's 8 blocks per SM are all resident:
// 4.35 -> 3.80 ms on the 2^24 incoherent rays of the 2M-triangle knot (12 blocks: 4.02 ms).
__global__ void __launch_bounds__(kBlock, kAllBlocksPerSm) raycast_all_persistent_kernel(
    MeshDev m, const float* __restrict__ rays, int side, const SideTable sides, float near_d, float far_d, uint32_t cap,
    uint32_t* __restrict__ counts, bvhc_hit* __restrict__ hits, const uint32_t* __restrict__ queue,
    const unsigned int* __restrict__ qcount, unsigned long long* __restrict__ work) {
  const unsigned full = 0xFFFFFFFFu;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_live = (uint64_t)__ldg(qcount);
  bool has = false, exhausted = false;
  uint64_t i = 0;
  RayF r;
  ff dlen = ff_from(0.0f);
  uint32_t cnt = 0, link = 0;
  int sp = 0, root = 0;
  uint32_t stack_link[kMaxStack];
  for (;;) {
    const unsigned idle = __ballot_sync(full, !has);
    if (idle != 0u && !exhausted) {
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader) base = atomicAdd(work, (unsigned long long)__popc(idle));
      base = __shfl_sync(full, base, leader);
      if (!has) {
        const uint64_t slot = base + (uint64_t)__popc(idle & ((1u << lane) - 1u));
        if (slot < n_live) {
          i = __ldg(queue + slot);
          r = make_ray(rays, i);
          dlen = dir_length(r.d);
          cnt = 0;
          root = 0;
          sp = 0;
          link = m.roots[0];
          has = true;
        }
      }
      exhausted = base + (unsigned long long)__popc(idle) >= n_live;  // warp-uniform
    }
    if (!__any_sync(full, has)) break;
    for (;;) {
      if (has) {
        bool pop = false;
        if (link & kLeafBit) {
          if (link != kEmptyLeaf) {
            bvhc_hit* out = hits + i * (uint64_t)cap;
            for (uint32_t k = link & ~kLeafBit;; ++k) {
              const Tri t = load_tri(m.tris, k);
              const int ts = tri_side(t, side, sides);
              if (ts >= 0 && tri_hit(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts)) {
                const ff tt = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, r.o, r.d));
                const ff dist = ff_mul(tt, dlen);
                if (!ff_lt(dist, ff_from(near_d)) && !ff_lt(ff_from(far_d), dist)) {
                  if (cnt < cap) {
                    bvhc_hit h;
                    make_hit(t, r, tt, dist, h);
                    store_hit(out + cnt, h);
                  }
                  ++cnt;
                }
              }
              if (t.flags & kTriLast) break;
            }
          }
          pop = true;
        } else {
          const Pair p = load_pair(m.nodes, link);
          float e0, e1;
          const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e0);
          const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e1);
          if (h0) {
            if (h1) {
              if (sp >= kMaxStack) {
                atomicOr(m.err, kErrStackOverflow);
                sp = 0;
                root = m.n_roots;  // give up on this ray
                pop = true;
              } else {
                stack_link[sp++] = p.lr;
              }
            }
            if (!pop) link = p.ll;
          } else if (h1) {
            link = p.lr;
          } else {
            pop = true;
          }
        }
        if (pop) {
          if (sp > 0) {
            link = stack_link[--sp];
          } else if (++root < m.n_roots) {
            link = m.roots[root];
          } else {
            counts[i] = cnt;
            has = false;
          }
        }
      }
      const int n_idle = __popc(__ballot_sync(full, !has));
      if (exhausted ? n_idle == 32 : n_idle >= kAllRefill) break;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// raycast (all hits), warp-cooperative: the 32 rays of a warp walk the tree together, left child
// before right child as the reference does, entering a child when any lane's ray enters its box
// (one shared stack of links; there is no early out, so no per-lane distances).  A lane that tests
// the triangles of a leaf its own traversal would not have reached finds no hit there (a ray that
// hits a triangle enters every box on its path), so each lane reports exactly its own hits, in its
// own DFS order.  With a queue (rays sorted by a Morton key), a warp takes 32 consecutive entries.
// ---------------------------------------------------------------------------------------------
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) raycast_all_packet_kernel(
    MeshDev m, const float* __restrict__ rays, uint64_t n, int side, const SideTable sides, float near_d,
    float far_d, uint32_t cap, uint32_t* __restrict__ counts, bvhc_hit* __restrict__ hits,
    const uint32_t* __restrict__ queue, const unsigned int* __restrict__ qcount) {
  __shared__ uint32_t s_link[kWarps][kMaxStack];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  RayF r;
  if (valid) {
    r = make_ray(rays, i);
  } else {
    r.o = make_float3(0.f, 0.f, 0.f);
    r.d = make_float3(1.f, 0.f, 0.f);
    r.inv = make_float3(1.f, 1e30f, 1e30f);
    r.d_l1 = 1.f;
  }
  const ff dlen = dir_length(r.d);
  uint32_t cnt = 0;
  bvhc_hit* out = hits + i * (uint64_t)cap;
  bool overflow = false;
  for (int root = 0; root < m.n_roots && !overflow; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && valid) {
          for (uint32_t k = link & ~kLeafBit;; ++k) {
            Tri t = load_tri(m.tris, k);
            int ts = tri_side(t, side, sides);
            if (ts >= 0 && tri_hit(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts)) {
              ff tt = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, r.o, r.d));
              ff dist = ff_mul(tt, dlen);
              if (!ff_lt(dist, ff_from(near_d)) && !ff_lt(ff_from(far_d), dist)) {
                if (cnt < cap) {
                  bvhc_hit h;
                  make_hit(t, r, tt, dist, h);
                  store_hit(out + cnt, h);
                }
                ++cnt;
              }
            }
            if (t.flags & kTriLast) break;
          }
        }
        pop = true;
      } else {
        Pair p = load_pair(m.nodes, link);
        float e0, e1;
        bool h0 = valid && box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e0);
        bool h1 = valid && box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e1);
        unsigned b0 = __ballot_sync(full, h0), b1 = __ballot_sync(full, h1);
        if (b0 && b1) {
          if (sp >= kMaxStack) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            overflow = true;
            break;
          }
          if (lane == 0) s_link[w][sp] = p.lr;
          ++sp;
          link = p.ll;
          __syncwarp();
        } else if (b0) {
          link = p.ll;
        } else if (b1) {
          link = p.lr;
        } else {
          pop = true;
        }
      }
      if (pop) {
        if (sp == 0) break;
        link = s_link[w][--sp];
      }
    }
  }
  if (valid) counts[i] = cnt;
}


// ---------------------------------------------------------------------------------------------
// closestPointToPoint (closestPointToPoint.js:6-78 through shapecast.js:41-214).
// At an internal node both child scores (squared distance from the point to the box) are
// computed; the lower-scoring child is visited first (left on ties), and a child is entered
// only if its score is below maxThreshold^2 (decided exactly) and not certainly above the best
// squared distance found so far.  No per-triangle maxThreshold test is made, as in the
// reference.  Candidate distances are compared in float32 with an error bound and re-compared
// in float-float when the bound does not separate them.
// ---------------------------------------------------------------------------------------------
constexpr float kU = 5.9604644775390625e-08f;  // 2^-24

__device__ __forceinline__ float box_score(const float* b, float3 p) {
  float dx = fmaxf(b[0], fminf(b[3], p.x)) - p.x;
  float dy = fmaxf(b[1], fminf(b[4], p.y)) - p.y;
  float dz = fmaxf(b[2], fminf(b[5], p.z)) - p.z;
  return dx * dx + dy * dy + dz * dz;
}

__device__ __noinline__ ff box_score_ff(const float* b, float3 p) {
  ff dx = two_diff(fmaxf(b[0], fminf(b[3], p.x)), p.x);
  ff dy = two_diff(fmaxf(b[1], fminf(b[4], p.y)), p.y);
  ff dz = two_diff(fmaxf(b[2], fminf(b[5], p.z)), p.z);
  return ff_add(ff_add(ff_mul(dx, dx), ff_mul(dy, dy)), ff_mul(dz, dz));
}

// score < maxThreshold^2, decided exactly (the box score carries at most 5 roundings, all terms
// positive, so 2^-20 relative slack separates every case the float32 value can settle).
__device__ __forceinline__ bool under_max(float s, const float* b, float3 p, ff max2) {
  if (s * (1.0f + kSlabMargin) < max2.hi * (1.0f - kSlabMargin)) return true;
  if (s * (1.0f - kSlabMargin) > max2.hi * (1.0f + kSlabMargin)) return false;
  return ff_lt(box_score_ff(b, p), max2);
}

// The best candidate of one query so far.
struct CPBest {
  float d2, err;     // float32 squared distance and its error bound
  uint32_t rec;      // triangle record (0xFFFFFFFF: none yet)
  float3 q;          // float32 closest point
  bool vertex;       // q is an input vertex, bit-exact
  bool ff_ok;        // ffv holds the float-float squared distance
  ff ffv;
};

__device__ __forceinline__ CPBest cp_none() {
  CPBest b;
  b.d2 = kInf;
  b.err = 0.0f;
  b.rec = 0xFFFFFFFFu;
  b.q = make_float3(0.f, 0.f, 0.f);
  b.vertex = false;
  b.ff_ok = false;
  b.ffv = {kInf, 0.0f};
  return b;
}

// Offers triangle record k to the query at p: a strictly smaller squared distance replaces the
// best (the reference's strict `<` on distSq), and an exact tie goes to the earlier record in
// leaf order (the reference keeps whichever its own traversal reached first; a fixed rule keeps
// the answer independent of how queries are grouped).  Returns the candidate's float32 squared
// distance and bound, and its float-float value when one was needed.
// With `cull`, a triangle whose bounding box is already farther than the best candidate is
// passed over without its closest point: its distance exceeds the best one, so it cannot win
// (callers that test minThreshold on every triangle pass false).
__device__ __forceinline__ void cp_offer(const MeshDev& m, float3 p, const Tri& t, uint32_t k, CPBest& b, float& d2,
                                         float& err, bool& have_ff, ff& cand_ff, bool cull = false) {
  if (cull && b.rec != 0xFFFFFFFFu) {
    // squared distance to the triangle's box: at most 4 roundings above the exact value's
    // relative 2^-22, so the 2^-20 shrink keeps it a lower bound
    const float dx = fmaxf(fmaxf(fminf(t.a.x, fminf(t.b.x, t.c.x)) - p.x, p.x - fmaxf(t.a.x, fmaxf(t.b.x, t.c.x))), 0.0f);
    const float dy = fmaxf(fmaxf(fminf(t.a.y, fminf(t.b.y, t.c.y)) - p.y, p.y - fmaxf(t.a.y, fmaxf(t.b.y, t.c.y))), 0.0f);
    const float dz = fmaxf(fmaxf(fminf(t.a.z, fminf(t.b.z, t.c.z)) - p.z, p.z - fmaxf(t.a.z, fmaxf(t.b.z, t.c.z))), 0.0f);
    const float lb = dx * dx + dy * dy + dz * dz;
    if (lb * (1.0f - 0x1p-20f) > b.d2 + b.err) {
      d2 = lb;
      err = 0.0f;
      have_ff = false;
      return;
    }
  }
  float3 q;
  float sc;
  d2 = closest_sq_f(p, t.a, t.b, t.c, q, sc);
  // |error| of each closest-point coordinate <= e (local-frame evaluation)
  float e = 32.0f * kU * sc;
  err = 3.5f * e * sqrtf(d2) + 3.0f * e * e;
  bool is_vertex = (q.x == t.a.x && q.y == t.a.y && q.z == t.a.z) ||
                   (q.x == t.b.x && q.y == t.b.y && q.z == t.b.z) ||
                   (q.x == t.c.x && q.y == t.c.y && q.z == t.c.z);
  bool take;
  have_ff = false;
  if (b.rec == 0xFFFFFFFFu) {
    take = d2 < kInf;  // the first finite candidate (distSq < Infinity)
  } else if (d2 + err < b.d2 - b.err) {
    take = true;
  } else if (d2 - err > b.d2 + b.err) {
    take = false;
  } else if (is_vertex && b.vertex && q.x == b.q.x && q.y == b.q.y && q.z == b.q.z) {
    take = k < b.rec;  // the same vertex: an exact tie, the earlier record in leaf order wins
  } else {
    // Undecided in float32: the float-float squared distances decide, and an exact tie goes to
    // the earlier record in leaf order.  Candidates are thus ranked by a total order that does
    // not depend on the order they are offered in, and every box that could hold a candidate at
    // the best distance is entered (box tests keep a relative slack), so the answer is the same
    // for any traversal order: per query, warp-shared, sorted or chunked.
    if (!b.ff_ok) {
      Tri bt = load_tri(m.tris, b.rec);
      b.ffv = closest_ff(p, bt.a, bt.b, bt.c).d2;
      b.ff_ok = true;
    }
    cand_ff = closest_ff(p, t.a, t.b, t.c).d2;
    have_ff = true;
    take = ff_lt(cand_ff, b.ffv) || (!ff_lt(b.ffv, cand_ff) && k < b.rec);
  }
  if (take) {
    b.d2 = d2;
    b.err = err;
    b.rec = k;
    b.q = q;
    b.vertex = is_vertex;
    b.ff_ok = have_ff;
    b.ffv = cand_ff;
  }
}

// The reported record: distance and closest point in float-float, rounded once.
__device__ __forceinline__ void cp_store(const MeshDev& m, float3 p, const CPBest& b, bvhc_closest* o) {
  if (b.rec == 0xFFFFFFFFu) {
    o->face_index = BVHC_NO_HIT;
    o->distance = kInf;
    o->point[0] = o->point[1] = o->point[2] = 0.0f;
    return;
  }
  Tri t = load_tri(m.tris, b.rec);
  CPFF c = closest_ff(p, t.a, t.b, t.c);
  o->face_index = t.face;
  o->distance = ff_to_f(ff_sqrt(c.d2));
  o->point[0] = ff_to_f(c.q.x);
  o->point[1] = ff_to_f(c.q.y);
  o->point[2] = ff_to_f(c.q.z);
}

__global__ void __launch_bounds__(kBlock) closest_point_kernel(MeshDev m, const float* __restrict__ pts, uint64_t n,
                                                               float min_t, float max_t,
                                                               bvhc_closest* __restrict__ out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float3 p = make_float3(__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2));
  ff max2 = two_prod(max_t, max_t);
  ff min2 = two_prod(min_t, min_t);
  CPBest b = cp_none();
  bool stop = false;
  uint32_t stack_link[kMaxStack];
  float stack_s[kMaxStack];
  for (int root = 0; root < m.n_roots && !stop; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      if (link & kLeafBit) {
        if (link != kEmptyLeaf) {
          uint32_t k = link & ~kLeafBit;
          for (;;) {
            Tri t = load_tri(m.tris, k);
            float d2, err;
            bool have_ff;
            ff cand_ff;
            cp_offer(m, p, t, k, b, d2, err, have_ff, cand_ff, !(min2.hi > 0.0f));
            // early out below minThreshold (closestPointToPoint.js:55-57)
            if (min2.hi > 0.0f) {
              bool below;
              if (d2 + err < min2.hi * (1.0f - kSlabMargin)) below = true;
              else if (d2 - err > min2.hi * (1.0f + kSlabMargin)) below = false;
              else below = ff_lt(have_ff ? cand_ff : closest_ff(p, t.a, t.b, t.c).d2, min2);
              if (below) { stop = true; break; }
            }
            if (t.flags & kTriLast) break;
            ++k;
          }
          if (stop) break;
        }
      } else {
        Pair pr = load_pair(m.nodes, link);
        float s0 = box_score(pr.l, p), s1 = box_score(pr.r, p);
        bool swap = s1 < s0;
        const float* b1 = swap ? pr.r : pr.l;
        const float* b2 = swap ? pr.l : pr.r;
        float sc1 = swap ? s1 : s0, sc2 = swap ? s0 : s1;
        uint32_t c1 = swap ? pr.lr : pr.ll, c2 = swap ? pr.ll : pr.lr;
        float best_hi = b.d2 + b.err;
        if (under_max(sc2, b2, p, max2)) {
          if (sp >= kMaxStack) {
            atomicOr(m.err, kErrStackOverflow);
            stop = true;
            break;
          }
          stack_link[sp] = c2;
          stack_s[sp] = sc2;
          ++sp;
        }
        if (sc1 * (1.0f - kSlabMargin) <= best_hi && under_max(sc1, b1, p, max2)) {
          link = c1;
          continue;
        }
      }
      bool found = false;
      while (sp > 0) {
        --sp;
        if (stack_s[sp] * (1.0f - kSlabMargin) <= b.d2 + b.err) {
          link = stack_link[sp];
          found = true;
          break;
        }
      }
      if (!found) break;
    }
  }
  cp_store(m, p, b, out + i);
}

// ---------------------------------------------------------------------------------------------
// closestPointToPoint, warp-cooperative form for spatially coherent queries (grids, SDF samples)
// with minThreshold 0.  The 32 queries of a warp walk the tree together with one shared stack of
// links: a child is entered when any lane wants it (its score under maxThreshold^2, decided
// exactly, and not certainly above that lane's best), and each lane keeps, for the current node
// and for every stacked child, whether it wants it (its own score, or NaN for "no").  A lane only
// tests the triangles of leaves it wants, so every lane reaches exactly the leaves its own
// traversal would and its result is the minimum over the same candidates: which leaves a query
// reaches, and so the "null iff no leaf is reached" rule, does not depend on the visiting order,
// and leaves skipped because of the best distance cannot hold a strictly closer triangle.  (With
// minThreshold > 0 the reference stops at the first triangle below it in its own order, which a
// shared order would not reproduce; those calls use the per-query kernel.)
// ---------------------------------------------------------------------------------------------
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) closest_point_packet_kernel(
    MeshDev m, const float* __restrict__ pts, uint64_t n, float max_t, bvhc_closest* __restrict__ out,
    const uint32_t* __restrict__ queue, const unsigned int* __restrict__ qcount) {
  __shared__ uint32_t s_link[kBlock / 32][kMaxStack];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  float3 p = make_float3(0.f, 0.f, 0.f);
  if (valid) p = make_float3(__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2));
  const ff max2 = two_prod(max_t, max_t);
  const float kNo = __int_as_float(0x7FFFFFFF);  // NaN: "this lane does not want the entry"
  CPBest b = cp_none();
  float lane_s[kMaxStack];
  bool overflow = false;
  for (int root = 0; root < m.n_roots && !overflow; ++root) {
    uint32_t link = m.roots[root];
    bool act = valid;  // this lane wants the current node (a root leaf has no bounds test)
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && act) {
          uint32_t k = link & ~kLeafBit;
          for (;;) {
            Tri t = load_tri(m.tris, k);
            float d2, err;
            bool have_ff;
            ff cand_ff;
            cp_offer(m, p, t, k, b, d2, err, have_ff, cand_ff, true);
            if (t.flags & kTriLast) break;
            ++k;
          }
        }
        pop = true;
      } else {
        Pair pr = load_pair(m.nodes, link);
        float s0 = box_score(pr.l, p), s1 = box_score(pr.r, p);
        float best_hi = b.d2 + b.err;
        bool w0 = act && s0 * (1.0f - kSlabMargin) <= best_hi && under_max(s0, pr.l, p, max2);
        bool w1 = act && s1 * (1.0f - kSlabMargin) <= best_hi && under_max(s1, pr.r, p, max2);
        unsigned b0 = __ballot_sync(full, w0), b1 = __ballot_sync(full, w1);
        if (b0 && b1) {
          // nearer child first by majority of the lanes that want both (a lane wanting one prefers it)
          bool pref_right = (w0 && w1) ? s1 < s0 : w1;
          unsigned voters = __ballot_sync(full, w0 || w1);
          bool right_first = 2 * __popc(__ballot_sync(full, (w0 || w1) && pref_right)) > __popc(voters);
          if (sp >= kMaxStack) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            b = cp_none();
            overflow = true;
            break;
          }
          if (lane == 0) s_link[w][sp] = right_first ? pr.ll : pr.lr;
          lane_s[sp] = right_first ? (w0 ? s0 : kNo) : (w1 ? s1 : kNo);
          ++sp;
          link = right_first ? pr.lr : pr.ll;
          act = right_first ? w1 : w0;
          __syncwarp();
        } else if (b0) {
          link = pr.ll;
          act = w0;
        } else if (b1) {
          link = pr.lr;
          act = w1;
        } else {
          pop = true;
        }
      }
      if (pop) {
        bool found = false;
        while (sp > 0) {
          --sp;
          bool ok = lane_s[sp] * (1.0f - kSlabMargin) <= b.d2 + b.err;  // false for NaN
          if (__ballot_sync(full, ok)) {
            link = s_link[w][sp];
            act = ok;
            found = true;
            break;
          }
        }
        if (!found) break;
      }
    }
  }
  if (valid) cp_store(m, p, b, out + i);
}

// ---------------------------------------------------------------------------------------------
// intersectsSphere (MeshBVH.js:796-809 through shapecast.js:41-214), one sphere per thread.  A
// child is entered when its box may meet the sphere (box score against r^2 with 2^-20 relative
// slack, a superset of the reference's `<=`), and a triangle meets the sphere when its closest
// point lies within r (sphereIntersectTriangle, MathUtilities.js:167-201, is that predicate
// evaluated through the edges and the plane): decided on the float32 squared distance with its
// error bound, else in float-float.  The answer, whether any triangle meets the sphere, does not
// depend on the visiting order; the first triangle found ends the query.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ bool sphere_meets(float3 c, ff r2, const Tri& t) {
  float3 q;
  float sc;
  float d2 = closest_sq_f(c, t.a, t.b, t.c, q, sc);
  float e = 32.0f * kU * sc;
  float err = 3.5f * e * sqrtf(d2) + 3.0f * e * e;
  const float kR = 1.1920928955078125e-07f;  // 2^-23: r2.hi against the exact r^2
  if (d2 + err < r2.hi * (1.0f - kR)) return true;
  if (d2 - err > r2.hi * (1.0f + kR)) return false;
  return !ff_lt(r2, closest_ff(c, t.a, t.b, t.c).d2);
}

__global__ void __launch_bounds__(kBlock) intersects_sphere_kernel(MeshDev m, const float* __restrict__ spheres,
                                                                   uint64_t n, uint8_t* __restrict__ out,
                                                                   const uint32_t* __restrict__ queue) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t i = queue ? (uint64_t)__ldg(queue + t) : t;
  const float4 sph = ld4(spheres + 4 * i);
  const float3 c = make_float3(sph.x, sph.y, sph.z);
  const ff r2 = two_prod(sph.w, sph.w);
  const float lim = r2.hi * (1.0f + kSlabMargin);
  bool hit = false;
  uint32_t stack[kMaxStack];
  for (int root = 0; root < m.n_roots && !hit; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      if (link & kLeafBit) {
        if (link != kEmptyLeaf) {
          for (uint32_t k = link & ~kLeafBit;; ++k) {
            Tri t = load_tri(m.tris, k);
            if (sphere_meets(c, r2, t)) {
              hit = true;
              break;
            }
            if (t.flags & kTriLast) break;
          }
          if (hit) break;
        }
      } else {
        Pair pr = load_pair(m.nodes, link);
        bool w0 = box_score(pr.l, c) * (1.0f - kSlabMargin) <= lim;
        bool w1 = box_score(pr.r, c) * (1.0f - kSlabMargin) <= lim;
        if (w0 && w1) {
          if (sp >= kMaxStack) {
            atomicOr(m.err, kErrStackOverflow);
            break;
          }
          stack[sp++] = pr.lr;
          link = pr.ll;
          continue;
        }
        if (w0 || w1) {
          link = w0 ? pr.ll : pr.lr;
          continue;
        }
      }
      if (sp == 0) break;
      link = stack[--sp];
    }
  }
  out[i] = hit ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// Triangles within a sphere through shapecast's CONTAINED path (shapecast.js:41-214; a CONTAINED
// node's whole range goes to the triangle callback with contained = true, :111-117), with the
// callbacks of the reference's sculpt / selection use: a node box is skipped when the sphere
// misses it (Sphere.intersectsBox), CONTAINED when its 8 corners lie within r
// (Sphere.containsPoint), else its triangles are tested (ExtendedTriangle.intersectsSphere).  One
// sphere per thread, left child before right; the triangles come out in the reference's order.
// The box relations decide which triangles enter untested, so they follow the reference's
// binary64 comparisons exactly: float32 with an error bound, else the binary64 sequence.
// ---------------------------------------------------------------------------------------------
// |p - c|^2 <= r^2 as the reference evaluates it (Vector3.distanceToSquared, radius * radius).
__device__ __forceinline__ bool within_r(float3 p, float3 c, float r) {
  const float dx = p.x - c.x, dy = p.y - c.y, dz = p.z - c.z;
  const float d2 = dx * dx + dy * dy + dz * dz, r2 = r * r;
  if (d2 * (1.0f + 0x1p-20f) < r2 * (1.0f - 0x1p-22f)) return true;
  if (d2 * (1.0f - 0x1p-20f) > r2 * (1.0f + 0x1p-22f)) return false;
  const sf::f64 ex = sf::sub(sf::from_f32(p.x), sf::from_f32(c.x)), ey = sf::sub(sf::from_f32(p.y), sf::from_f32(c.y)),
                ez = sf::sub(sf::from_f32(p.z), sf::from_f32(c.z)), R = sf::from_f32(r);
  return sf::le(sf::add(sf::add(sf::mul(ex, ex), sf::mul(ey, ey)), sf::mul(ez, ez)), sf::mul(R, R));
}

// 0 the sphere misses the box, 1 it meets it, 2 the box lies within the sphere.
__device__ int sphere_box_relation(const float* b, float3 c, float r) {
  const float3 q = make_float3(fmaxf(b[0], fminf(b[3], c.x)), fmaxf(b[1], fminf(b[4], c.y)), fmaxf(b[2], fminf(b[5], c.z)));
  if (!within_r(q, c, r)) return 0;
  for (int k = 0; k < 8; ++k)
    if (!within_r(make_float3((k & 1) ? b[3] : b[0], (k & 2) ? b[4] : b[1], (k & 4) ? b[5] : b[2]), c, r)) return 1;
  return 2;
}

// 8 resident blocks per SM (64 registers): 2.51 -> 2.16 ms for 2^18 brush spheres on the 2M-triangle
// knot (12 and 16 blocks: 2.43 / 2.38 ms; the any-hit sphere and box kernels lost time the same way).
__global__ void __launch_bounds__(kBlock, 8) sphere_triangles_kernel(MeshDev m, const float* __restrict__ spheres,
                                                                  uint64_t n, uint32_t cap,
                                                                  uint32_t* __restrict__ counts,
                                                                  uint32_t* __restrict__ faces,
                                                                  const uint32_t* __restrict__ queue) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t i = queue ? (uint64_t)__ldg(queue + t) : t;
  const float4 sph = ld4(spheres + 4 * i);
  const float3 c = make_float3(sph.x, sph.y, sph.z);
  const ff r2 = two_prod(sph.w, sph.w);
  uint32_t* out = faces + i * (uint64_t)cap;
  uint32_t cnt = 0;
  uint32_t stack_link[kMaxStack];
  uint8_t stack_rel[kMaxStack];
  uint32_t sub[kMaxStack];
  bool overflow = false;
  for (int root = 0; root < m.n_roots && !overflow; ++root) {
    int sp = 0;
    stack_link[sp] = m.roots[root];
    stack_rel[sp++] = 1;  // the root has no bounds test
    while (sp > 0 && !overflow) {
      --sp;
      const uint32_t link = stack_link[sp];
      const int rel = stack_rel[sp];
      if (rel == 2) {  // CONTAINED: every triangle of the subtree, in order, untested
        int ssp = 0;
        sub[ssp++] = link;
        while (ssp > 0) {
          const uint32_t l = sub[--ssp];
          if (l & kLeafBit) {
            if (l == kEmptyLeaf) continue;
            for (uint32_t k = l & ~kLeafBit;; ++k) {
              const Tri t = load_tri(m.tris, k);
              if (cnt < cap) out[cnt] = t.face;
              ++cnt;
              if (t.flags & kTriLast) break;
            }
          } else {
            if (ssp + 2 > kMaxStack) {
              overflow = true;
              break;
            }
            const Pair p = load_pair(m.nodes, l);
            sub[ssp++] = p.lr;
            sub[ssp++] = p.ll;
          }
        }
      } else if (link & kLeafBit) {
        if (link == kEmptyLeaf) continue;
        for (uint32_t k = link & ~kLeafBit;; ++k) {
          const Tri t = load_tri(m.tris, k);
          if (sphere_meets(c, r2, t)) {
            if (cnt < cap) out[cnt] = t.face;
            ++cnt;
          }
          if (t.flags & kTriLast) break;
        }
      } else {
        const Pair p = load_pair(m.nodes, link);
        const int rl = sphere_box_relation(p.l, c, sph.w), rr = sphere_box_relation(p.r, c, sph.w);
        if (sp + 2 > kMaxStack) {
          overflow = true;
          break;
        }
        if (rr) {
          stack_link[sp] = p.lr;
          stack_rel[sp++] = (uint8_t)rr;
        }
        if (rl) {
          stack_link[sp] = p.ll;
          stack_rel[sp++] = (uint8_t)rl;
        }
      }
    }
  }
  if (overflow) atomicOr(m.err, kErrStackOverflow);
  for (uint32_t q = cnt; q < cap; ++q) out[q] = 0xFFFFFFFFu;
  counts[i] = cnt;
}

// ---------------------------------------------------------------------------------------------
// intersectsBox (MeshBVH.js:780-792): an OrientedBox (src/math/OrientedBox.js:78-260) tested
// against node boxes (OrientedBox.intersectsBox: the three aligned extents, then the box's three
// edge directions) and triangles (OrientedBox.intersectsTriangle: the box's axes, the triangle's
// normal and two edges (ExtendedTriangle.js:57-86), then the twelve cross products), every test a
// SeparatingAxisBounds.isSeparated of two projection intervals.
//
// Each interval comparison is taken in float-float, whose values differ from the reference's
// binary64 ones by less than 2^-37 M^k (M bounds every coordinate and transform term involved,
// k the degree of the projection); it stands when the gap exceeds 2^-36 M^k (2^-34 M^3 for the
// cross axes; a margin grown by the unit normal's direction error for axes built on it).  A test
// with any comparison inside its margin, and every test of a non-affine box matrix, is evaluated
// again with the reference's exact binary64 operation sequence (softf64.cuh).  A query is 24
// floats: min xyz, pad, max xyz, pad, the column-major box-to-mesh matrix (three.js
// Matrix4.elements).
// ---------------------------------------------------------------------------------------------
namespace obb {

using sf::f64;

struct ObbF {
  ff3 p[8];               // corners, OrientedBox.update
  ff3 ax[3];              // satAxes: p[0] - p[1 << i]
  ff smin[3], smax[3];    // satBounds
  ff amin[3], amax[3];    // alignedSatBounds
  float mag;              // >= every |corner coordinate| and transform term
  bool exact;             // non-affine matrix: binary64 throughout
};

__device__ __forceinline__ ff ff_min(ff a, ff b) { return ff_lt(b, a) ? b : a; }
__device__ __forceinline__ ff ff_max(ff a, ff b) { return ff_lt(a, b) ? b : a; }
__device__ __forceinline__ ff ff3_get(const ff3& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }
__device__ __forceinline__ float absmax3(float3 v) { return fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z))); }

__device__ __noinline__ void make_ff(const float* q, ObbF& o) {
  const float* e = q + 8;
  o.exact = !(e[3] == 0.0f && e[7] == 0.0f && e[11] == 0.0f && e[15] == 1.0f);
  float mag = 0.0f;
  for (int i = 0; i < 8; ++i) {
    const float x = (i & 1) ? q[4] : q[0], y = (i & 2) ? q[5] : q[1], z = (i & 4) ? q[6] : q[2];
    ff c[3];
    for (int k = 0; k < 3; ++k) {
      c[k] = ff_add(ff_add(ff_add(two_prod(e[k], x), two_prod(e[4 + k], y)), two_prod(e[8 + k], z)), ff_from(e[12 + k]));
      mag = fmaxf(mag, fabsf(e[k] * x) + fabsf(e[4 + k] * y) + fabsf(e[8 + k] * z) + fabsf(e[12 + k]));
    }
    o.p[i] = {c[0], c[1], c[2]};
  }
  o.mag = mag * (1.0f + 0x1p-20f);
  for (int i = 0; i < 3; ++i) {
    o.ax[i] = ff3_sub(o.p[0], o.p[1 << i]);
    o.smin[i] = o.smax[i] = ff3_dot(o.ax[i], o.p[0]);
    for (int k = 1; k < 8; ++k) {
      const ff v = ff3_dot(o.ax[i], o.p[k]);
      o.smin[i] = ff_min(o.smin[i], v);
      o.smax[i] = ff_max(o.smax[i], v);
    }
  }
  for (int d = 0; d < 3; ++d) {
    o.amin[d] = o.amax[d] = ff3_get(o.p[0], d);
    for (int k = 1; k < 8; ++k) {
      o.amin[d] = ff_min(o.amin[d], ff3_get(o.p[k], d));
      o.amax[d] = ff_max(o.amax[d], ff3_get(o.p[k], d));
    }
  }
}

// --- float32 tier ------------------------------------------------------------------------------
// The same separating-axis tests in float32, built straight from the query (u = 2^-24):
//   corners    fma chains, within 3.01 u M of the exact ones (M >= every |corner coordinate|,
//              the sum of its terms' magnitudes),
//   axes       p[0] - p[1 << i] = -(max_i - min_i) * column i of the matrix, within 2.01 u of
//              each exact component,
//   bounds     dot products / extremes of those.
// Every margin below is about twice a bound on |float gap - exact gap| (the derivation is given
// per test), plus an absolute term for the reference's own binary64 rounding of its corners
// (~2^-51 M per coordinate, which a thin box's axes inherit).  A gap beyond the margin has the
// sign the reference's binary64 gap has; undecided tests go on to the float-float tier.
struct ObbS {
  float3 p[8], ax[3];
  float smin[3], smax[3], amin[3], amax[3];
  float n1[3];  // L1 norms of the axes
  float mag;    // >= every corner's sum of term magnitudes; 0 when the box is too large (undecided)
  bool exact;   // non-affine matrix: every test goes to binary64
};

__device__ __forceinline__ float dotf(float3 a, float3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
__device__ __forceinline__ float l1f(float3 a) { return fabsf(a.x) + fabsf(a.y) + fabsf(a.z); }
__device__ __forceinline__ float3 crossf(float3 a, float3 b) {
  return make_float3(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}
__device__ __forceinline__ float3 subf(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }

__device__ __forceinline__ int sep_f(float amn, float amx, float bmn, float bmx, float margin) {
  const float d1 = amn - bmx, d2 = bmn - amx;
  if (d1 > margin || d2 > margin) return 1;
  if (d1 < -margin && d2 < -margin) return 0;
  return -1;
}

__device__ __forceinline__ void interval_f(float3 axis, const float3* pts, int n, float& mn, float& mx) {
  mn = mx = dotf(axis, pts[0]);
  for (int k = 1; k < n; ++k) {
    const float v = dotf(axis, pts[k]);
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
}

__device__ __forceinline__ void make_s(const float* q, ObbS& s) {
  const float* e = q + 8;
  s.exact = !(e[3] == 0.0f && e[7] == 0.0f && e[11] == 0.0f && e[15] == 1.0f);
  float mag = 0.0f;
  for (int i = 0; i < 8; ++i) {
    const float x = (i & 1) ? q[4] : q[0], y = (i & 2) ? q[5] : q[1], z = (i & 4) ? q[6] : q[2];
    float c[3];
    for (int k = 0; k < 3; ++k) {
      c[k] = fmaf(e[k], x, fmaf(e[4 + k], y, fmaf(e[8 + k], z, e[12 + k])));
      mag = fmaxf(mag, fabsf(e[k] * x) + fabsf(e[4 + k] * y) + fabsf(e[8 + k] * z) + fabsf(e[12 + k]));
    }
    s.p[i] = make_float3(c[0], c[1], c[2]);
  }
  mag *= 1.0f + 0x1p-20f;
  for (int i = 0; i < 3; ++i) {
    const float w = q[4 + i] - q[i];
    s.ax[i] = make_float3(-e[4 * i] * w, -e[4 * i + 1] * w, -e[4 * i + 2] * w);
    s.n1[i] = l1f(s.ax[i]);
    interval_f(s.ax[i], s.p, 8, s.smin[i], s.smax[i]);
  }
  for (int d = 0; d < 3; ++d) {
    float mn = d == 0 ? s.p[0].x : (d == 1 ? s.p[0].y : s.p[0].z), mx = mn;
    for (int k = 1; k < 8; ++k) {
      const float v = d == 0 ? s.p[k].x : (d == 1 ? s.p[k].y : s.p[k].z);
      mn = fminf(mn, v);
      mx = fmaxf(mx, v);
    }
    s.amin[d] = mn;
    s.amax[d] = mx;
  }
  s.mag = mag < 1e30f ? mag : 0.0f;
}

// OrientedBox.intersectsBox on a node box: 1 meets, 0 separated, -1 undecided.
__device__ __forceinline__ int box_f(const ObbS& o, const float* b) {
  float m = o.mag;
  for (int k = 0; k < 6; ++k) m = fmaxf(m, fabsf(b[k]));
  if (!(o.mag > 0.0f) || !(m < 1e30f)) return -1;
  // aligned bounds: |error| <= 3.01 u M + 2 u m
  const float md = 0x1p-20f * m + 0x1p-120f;
  bool undecided = false;
  for (int d = 0; d < 3; ++d) {
    const int r = sep_f(o.amin[d], o.amax[d], b[d], b[d + 3], md);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  // the node box's interval on a box axis is sum_d min / max(a_d lo_d, a_d hi_d) (the extremes
  // over its 8 corners); |error| <= |a|_1 (6.02 u B + 9.02 u M)
  const float mr = 0x1p-36f * m * m + 0x1p-120f;
  for (int i = 0; i < 3; ++i) {
    const float3 a = o.ax[i];
    const float x0 = a.x * b[0], x1 = a.x * b[3], y0 = a.y * b[1], y1 = a.y * b[4], z0 = a.z * b[2], z1 = a.z * b[5];
    const float mn = fminf(x0, x1) + fminf(y0, y1) + fminf(z0, z1);
    const float mx = fmaxf(x0, x1) + fmaxf(y0, y1) + fmaxf(z0, z1);
    const int r = sep_f(o.smin[i], o.smax[i], mn, mx, 0x1p-19f * o.n1[i] * m + mr);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  return undecided ? -1 : 1;
}

// OrientedBox.intersectsTriangle: 1 meets, 0 separated, -1 undecided.
__device__ __forceinline__ int tri_f(const ObbS& o, float3 a, float3 b, float3 c) {
  const float m = fmaxf(o.mag, fmaxf(absmax3(a), fmaxf(absmax3(b), absmax3(c))));
  if (!(o.mag > 0.0f) || !(m < 1e30f)) return -1;
  const float mr = 0x1p-36f * m * m + 0x1p-120f;
  const float3 tp[3] = {a, b, c};
  bool undecided = false;
  // the box's axes against the triangle: |error| <= |a|_1 (6.01 u T + 9.02 u M)
  for (int i = 0; i < 3; ++i) {
    float mn, mx;
    interval_f(o.ax[i], tp, 3, mn, mx);
    const int r = sep_f(o.smin[i], o.smax[i], mn, mx, 0x1p-19f * o.n1[i] * m + mr);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  // unit normal of cross(c - b, a - b) (Triangle.getNormal): with S the sums of the cross
  // product's term magnitudes, its direction is within 8.2 u |S|_1 / |raw| + 4.5 u;
  // rho is twice that
  const float3 e1 = subf(c, b), e2 = subf(a, b);
  const float3 raw = crossf(e1, e2);
  const float s1 = fabsf(e1.y * e2.z) + fabsf(e1.z * e2.y) + fabsf(e1.z * e2.x) + fabsf(e1.x * e2.z) +
                   fabsf(e1.x * e2.y) + fabsf(e1.y * e2.x);
  const float l2 = dotf(raw, raw);
  const float inv = l2 > 0.0f ? rsqrtf(l2) : 0.0f;
  const float rho = 0x1p-20f * s1 * inv + 0x1p-20f;
  const bool normal_ok = l2 > 0x1p-100f && rho < 0x1p-10f;
  const float3 ta[4] = {make_float3(raw.x * inv, raw.y * inv, raw.z * inv), subf(a, b), subf(b, c), subf(c, a)};
  const float t1[4] = {1.7321f, l1f(ta[1]), l1f(ta[2]), l1f(ta[3])};
  // the normal: |error| <= m (3.46 rho_dir + 39.8 u); an edge: |error| <= 13.01 u |e|_1 m
  for (int i = 0; i < 3; ++i) {
    if (i == 0 && !normal_ok) {
      undecided = true;
      continue;
    }
    float tmn, tmx, bmn, bmx;
    interval_f(ta[i], tp, 3, tmn, tmx);
    interval_f(ta[i], o.p, 8, bmn, bmx);
    const float margin = (i == 0 ? m * (8.0f * rho + 0x1p-19f) : 0x1p-19f * t1[i] * m) + mr;
    const int r = sep_f(tmn, tmx, bmn, bmx, margin);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  // box axis x triangle axis: |error| <= 21 u |a|_1 |e|_1 m for an edge,
  // m |a|_1 (3.46 rho_dir + 48.5 u) for the normal
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 4; ++j) {
      if (j == 0 && !normal_ok) {
        undecided = true;
        continue;
      }
      const float3 axis = crossf(o.ax[i], ta[j]);
      float tmn, tmx, bmn, bmx;
      interval_f(axis, tp, 3, tmn, tmx);
      interval_f(axis, o.p, 8, bmn, bmx);
      const float margin =
          (j == 0 ? m * o.n1[i] * (8.0f * rho + 0x1p-18f) : 0x1p-18f * o.n1[i] * t1[j] * m) + mr * t1[j];
      const int r = sep_f(tmn, tmx, bmn, bmx, margin);
      if (r == 1) return 0;
      undecided |= r < 0;
    }
  }
  return undecided ? -1 : 1;
}

// 1: the intervals are separated, 0: they overlap, -1: within the margin.
__device__ __forceinline__ int sep(ff amn, ff amx, ff bmn, ff bmx, float margin) {
  const float d1 = ff_to_f(ff_sub(amn, bmx)), d2 = ff_to_f(ff_sub(bmn, amx));
  if (d1 > margin || d2 > margin) return 1;
  if (d1 < -margin && d2 < -margin) return 0;
  return -1;
}

__device__ __forceinline__ void interval(const ff3& axis, const ff3* pts, int n, ff& mn, ff& mx) {
  mn = mx = ff3_dot(axis, pts[0]);
  for (int k = 1; k < n; ++k) {
    const ff v = ff3_dot(axis, pts[k]);
    mn = ff_min(mn, v);
    mx = ff_max(mx, v);
  }
}

// OrientedBox.intersectsBox on a node box: 1 meets, 0 separated, -1 undecided.
__device__ __noinline__ int box_ff(const ObbF& o, const float* b) {
  float m = o.mag;
  for (int k = 0; k < 6; ++k) m = fmaxf(m, fabsf(b[k]));
  const float m1 = 0x1p-36f * m, m2 = 0x1p-36f * m * m;
  bool undecided = false;
  for (int d = 0; d < 3; ++d) {
    const int r = sep(o.amin[d], o.amax[d], ff_from(b[d]), ff_from(b[d + 3]), m1);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  ff3 corners[8];
  for (int k = 0; k < 8; ++k)
    corners[k] = {ff_from((k & 1) ? b[0] : b[3]), ff_from((k & 2) ? b[1] : b[4]), ff_from((k & 4) ? b[2] : b[5])};
  for (int i = 0; i < 3; ++i) {
    ff mn, mx;
    interval(o.ax[i], corners, 8, mn, mx);
    const int r = sep(o.smin[i], o.smax[i], mn, mx, m2);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  return undecided ? -1 : 1;
}

// OrientedBox.intersectsTriangle: 1 meets, 0 separated, -1 undecided.
__device__ __noinline__ int tri_ff(const ObbF& o, float3 a, float3 b, float3 c) {
  const float m = fmaxf(o.mag, fmaxf(absmax3(a), fmaxf(absmax3(b), absmax3(c))));
  const float m2 = 0x1p-36f * m * m, m3 = 0x1p-34f * m * m * m;
  const ff3 tp[3] = {{ff_from(a.x), ff_from(a.y), ff_from(a.z)}, {ff_from(b.x), ff_from(b.y), ff_from(b.z)},
                     {ff_from(c.x), ff_from(c.y), ff_from(c.z)}};
  // the triangle's axes: unit normal (Triangle.getNormal), a - b, b - c, c - a (exact in float-float)
  ff3 ta[4];
  ta[1] = ff3_diff(a, b);
  ta[2] = ff3_diff(b, c);
  ta[3] = ff3_diff(c, a);
  const ff3 raw = ff3_cross(ff3_diff(c, b), ff3_diff(a, b));
  const ff l2 = ff3_dot(raw, raw);
  // both cross products (the reference's binary64 one and this float-float one) are within
  // 2^-43 M^2 of the exact one per component, so the unit normals differ in direction by at most
  // rel = 2^-40 M^2 / |n|; a normal shorter than 2^-20 M^2 (or zero) goes to binary64
  if (!(l2.hi > 0x1p-40f * m * m * m * m)) return -1;
  const ff inv = ff_div(ff_from(1.0f), ff_sqrt(l2));
  ta[0] = ff3_scale(raw, inv);
  const float rel = 0x1p-40f * m * m * rsqrtf(l2.hi);
  const float mn_normal = (0x1p-36f + 8.0f * rel) * 4.0f * m;
  const float mn_cross_n = (0x1p-34f + 8.0f * rel) * 16.0f * m * m;
  bool undecided = false;
  for (int i = 0; i < 3; ++i) {
    ff mn, mx;
    interval(o.ax[i], tp, 3, mn, mx);
    const int r = sep(o.smin[i], o.smax[i], mn, mx, m2);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  for (int i = 0; i < 3; ++i) {
    ff tmn, tmx, bmn, bmx;
    interval(ta[i], tp, 3, tmn, tmx);
    interval(ta[i], o.p, 8, bmn, bmx);
    const int r = sep(tmn, tmx, bmn, bmx, i == 0 ? mn_normal : m2);
    if (r == 1) return 0;
    undecided |= r < 0;
  }
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 4; ++j) {
      const ff3 axis = ff3_cross(o.ax[i], ta[j]);
      ff tmn, tmx, bmn, bmx;
      interval(axis, tp, 3, tmn, tmx);
      interval(axis, o.p, 8, bmn, bmx);
      const int r = sep(tmn, tmx, bmn, bmx, j == 0 ? mn_cross_n : m3);
      if (r == 1) return 0;
      undecided |= r < 0;
    }
  }
  return undecided ? -1 : 1;
}

// --- the reference's exact binary64 sequence --------------------------------------------------

struct V { f64 x, y, z; };
__device__ __forceinline__ V vsub(V a, V b) { return {sf::sub(a.x, b.x), sf::sub(a.y, b.y), sf::sub(a.z, b.z)}; }
__device__ __forceinline__ f64 vdot(V a, V b) {
  return sf::add(sf::add(sf::mul(a.x, b.x), sf::mul(a.y, b.y)), sf::mul(a.z, b.z));
}
__device__ __forceinline__ V vcross(V a, V b) {
  return {sf::sub(sf::mul(a.y, b.z), sf::mul(a.z, b.y)), sf::sub(sf::mul(a.z, b.x), sf::mul(a.x, b.z)),
          sf::sub(sf::mul(a.x, b.y), sf::mul(a.y, b.x))};
}
__device__ __forceinline__ V vf(float3 p) { return {sf::from_f32(p.x), sf::from_f32(p.y), sf::from_f32(p.z)}; }
__device__ __forceinline__ f64 vget(const V& v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }
__device__ __forceinline__ bool separated(f64 amn, f64 amx, f64 bmn, f64 bmx) {  // isSeparated
  return sf::lt(bmx, amn) || sf::lt(amx, bmn);
}
__device__ __forceinline__ void interval_d(V axis, const V* pts, int n, f64& mn, f64& mx) {  // setFromPoints
  mn = sf::kInf;
  mx = sf::neg(sf::kInf);
  for (int k = 0; k < n; ++k) {
    const f64 v = vdot(axis, pts[k]);
    if (sf::lt(v, mn)) mn = v;
    if (sf::lt(mx, v)) mx = v;
  }
}

struct ObbD {
  V p[8], ax[3];
  f64 smin[3], smax[3], amin[3], amax[3];
};

__device__ __noinline__ void make_d(const float* q, ObbD& o) {
  f64 e[16];
  for (int k = 0; k < 16; ++k) e[k] = sf::from_f32(q[8 + k]);
  for (int i = 0; i < 8; ++i) {
    const f64 x = sf::from_f32((i & 1) ? q[4] : q[0]), y = sf::from_f32((i & 2) ? q[5] : q[1]),
              z = sf::from_f32((i & 4) ? q[6] : q[2]);
    const f64 w = sf::div(sf::kOne, sf::add(sf::add(sf::add(sf::mul(e[3], x), sf::mul(e[7], y)), sf::mul(e[11], z)), e[15]));
    f64 c[3];
    for (int k = 0; k < 3; ++k)
      c[k] = sf::mul(sf::add(sf::add(sf::add(sf::mul(e[k], x), sf::mul(e[4 + k], y)), sf::mul(e[8 + k], z)), e[12 + k]), w);
    o.p[i] = {c[0], c[1], c[2]};
  }
  for (int i = 0; i < 3; ++i) {
    o.ax[i] = vsub(o.p[0], o.p[1 << i]);
    interval_d(o.ax[i], o.p, 8, o.smin[i], o.smax[i]);
  }
  for (int d = 0; d < 3; ++d) {
    o.amin[d] = sf::kInf;
    o.amax[d] = sf::neg(sf::kInf);
    for (int k = 0; k < 8; ++k) {
      const f64 v = vget(o.p[k], d);
      if (sf::lt(v, o.amin[d])) o.amin[d] = v;
      if (sf::lt(o.amax[d], v)) o.amax[d] = v;
    }
  }
}

__device__ __forceinline__ f64 js_min(f64 a, f64 b) { return (sf::is_nan(a) || sf::is_nan(b)) ? sf::kNaN : (sf::lt(b, a) ? b : a); }
__device__ __forceinline__ f64 js_max(f64 a, f64 b) { return (sf::is_nan(a) || sf::is_nan(b)) ? sf::kNaN : (sf::lt(a, b) ? b : a); }

__device__ __noinline__ bool box_d(const ObbD& o, const float* b) {
  for (int d = 0; d < 3; ++d)
    if (separated(o.amin[d], o.amax[d], sf::from_f32(b[d]), sf::from_f32(b[d + 3]))) return false;
  const f64 zero = 0, one = sf::kOne;
  for (int i = 0; i < 3; ++i) {  // setFromBox: p = min * t + max * (1 - t), Math.min / Math.max
    f64 mn = sf::kInf, mx = sf::neg(sf::kInf);
    for (int x = 0; x <= 1; ++x)
      for (int y = 0; y <= 1; ++y)
        for (int z = 0; z <= 1; ++z) {
          const f64 tx = x ? one : zero, ty = y ? one : zero, tz = z ? one : zero;
          const V p{sf::add(sf::mul(sf::from_f32(b[0]), tx), sf::mul(sf::from_f32(b[3]), sf::sub(one, tx))),
                    sf::add(sf::mul(sf::from_f32(b[1]), ty), sf::mul(sf::from_f32(b[4]), sf::sub(one, ty))),
                    sf::add(sf::mul(sf::from_f32(b[2]), tz), sf::mul(sf::from_f32(b[5]), sf::sub(one, tz)))};
          const f64 v = vdot(o.ax[i], p);
          mn = js_min(v, mn);
          mx = js_max(v, mx);
        }
    if (separated(o.smin[i], o.smax[i], mn, mx)) return false;
  }
  return true;
}

__device__ __noinline__ bool tri_d(const ObbD& o, float3 fa, float3 fb, float3 fc) {
  const V a = vf(fa), b = vf(fb), c = vf(fc);
  const V tp[3] = {a, b, c};
  V n = vcross(vsub(c, b), vsub(a, b));  // Triangle.getNormal
  const f64 l2 = vdot(n, n);
  if (sf::lt(0, l2)) {
    const f64 s = sf::div(sf::kOne, sf::sqrt(l2));
    n = {sf::mul(n.x, s), sf::mul(n.y, s), sf::mul(n.z, s)};
  } else {
    n = {0, 0, 0};
  }
  const V ta[4] = {n, vsub(a, b), vsub(b, c), vsub(c, a)};
  f64 mn, mx, mn2, mx2;
  for (int i = 0; i < 3; ++i) {
    interval_d(o.ax[i], tp, 3, mn, mx);
    if (separated(o.smin[i], o.smax[i], mn, mx)) return false;
  }
  for (int i = 0; i < 3; ++i) {
    interval_d(ta[i], tp, 3, mn, mx);
    interval_d(ta[i], o.p, 8, mn2, mx2);
    if (separated(mn, mx, mn2, mx2)) return false;
  }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) {
      const V axis = vcross(o.ax[i], ta[j]);
      interval_d(axis, tp, 3, mn, mx);
      interval_d(axis, o.p, 8, mn2, mx2);
      if (separated(mn, mx, mn2, mx2)) return false;
    }
  return true;
}

}  // namespace obb

// One oriented box's predicates with the three tiers: float32, float-float (built on first
// need), the reference's binary64 sequence (built on first need; always for non-affine boxes).
struct BoxAny {
  float q[24];
  obb::ObbS s;
  obb::ObbF f;
  obb::ObbD d;
  bool have_f, have_d;
  __device__ void init(const float* __restrict__ boxes, uint64_t i) {
    for (int k = 0; k < 6; ++k) {
      const float4 v = ld4(boxes + 24 * i + 4 * k);
      q[4 * k] = v.x;
      q[4 * k + 1] = v.y;
      q[4 * k + 2] = v.z;
      q[4 * k + 3] = v.w;
    }
    obb::make_s(q, s);
    have_f = have_d = false;
  }
  __device__ void need_f() {
    if (!have_f) {
      obb::make_ff(q, f);
      have_f = true;
    }
  }
  __device__ void need_d() {
    if (!have_d) {
      obb::make_d(q, d);
      have_d = true;
    }
  }
  __device__ bool box(const float* b) {
    int r = s.exact ? -1 : obb::box_f(s, b);
    if (r < 0 && !s.exact) {
      need_f();
      r = obb::box_ff(f, b);
    }
    if (r < 0) {
      need_d();
      r = obb::box_d(d, b) ? 1 : 0;
    }
    return r == 1;
  }
  __device__ bool tri(const Tri& t) {
    int r = s.exact ? -1 : obb::tri_f(s, t.a, t.b, t.c);
    if (r < 0 && !s.exact) {
      need_f();
      r = obb::tri_ff(f, t.a, t.b, t.c);
    }
    if (r < 0) {
      need_d();
      r = obb::tri_d(d, t.a, t.b, t.c) ? 1 : 0;
    }
    return r == 1;
  }
};

// One box per thread in the "while-while" form: every lane walks child pairs until it holds a
// non-empty leaf (or its traversal ends), then the lanes holding leaves test their triangles
// together, so the costly triangle tests of a few lanes are not paid at every node step.
__global__ void __launch_bounds__(kBlock) intersects_box_kernel(MeshDev m, const float* __restrict__ boxes,
                                                                uint64_t n, uint8_t* __restrict__ out,
                                                                const uint32_t* __restrict__ queue) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t i = queue ? (uint64_t)__ldg(queue + t) : t;
  BoxAny q;
  q.init(boxes, i);
  bool hit = false;
  uint32_t stack[kMaxStack];
  for (int root = 0; root < m.n_roots && !hit; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    bool live = true;  // this root's traversal has work left
    while (live) {
      // node phase: down to a non-empty leaf, or to the end of the traversal
      while (!(link & kLeafBit) || link == kEmptyLeaf) {
        if (link & kLeafBit) {  // empty leaf: next entry
          if (sp == 0) {
            live = false;
            break;
          }
          link = stack[--sp];
          continue;
        }
        const Pair pr = load_pair(m.nodes, link);
        const bool w0 = q.box(pr.l), w1 = q.box(pr.r);
        if (w0 && w1) {
          if (sp >= kMaxStack) {
            atomicOr(m.err, kErrStackOverflow);
            live = false;
            break;
          }
          stack[sp++] = pr.lr;
          link = pr.ll;
        } else if (w0 || w1) {
          link = w0 ? pr.ll : pr.lr;
        } else if (sp > 0) {
          link = stack[--sp];
        } else {
          live = false;
          break;
        }
      }
      if (!live) break;
      // leaf phase
      for (uint32_t k = link & ~kLeafBit;; ++k) {
        const Tri t = load_tri(m.tris, k);
        if (q.tri(t)) {
          hit = true;
          break;
        }
        if (t.flags & kTriLast) break;
      }
      if (hit || sp == 0) break;
      link = stack[--sp];
    }
  }
  out[i] = hit ? 1 : 0;
}

// ---------------------------------------------------------------------------------------------
// Instanced raycastFirst: acceleratedBatchedMeshRaycast (ExtensionUtilities.js:87-161) with
// firstHitOnly, each instance through MeshBVH.raycastObject3D (MeshBVH.js:447-494) and
// convertRaycastIntersect (GeometryRayIntersectUtilities.js:3-17), then the closest world hit
// (the raycaster's stable sort by distance: equal distances keep the lower instance index).
//
// Two levels: a tree over the instances' world boxes, and for every instance box the ray enters,
// the instance's geometry tree in its local frame.  The local ray is the reference's: origin
// through the inverse matrix, direction through its 3 x 3 part and normalised
// (Ray.applyMatrix4 / Vector3.transformDirection), computed in float-float from the binary64
// inverse and rounded once; near and far are divided by |direction * world scale|.  The local
// hit point goes back through the world matrix and the world distance is |point - origin|.
// Instance boxes and local traversals are pruned by the closest world hit so far.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ RayF ray_from(float3 o, float3 d) {
  RayF r;
  r.o = o;
  r.d = d;
  const float dx = fabsf(d.x) < kTiny ? copysignf(kTiny, d.x) : d.x;
  const float dy = fabsf(d.y) < kTiny ? copysignf(kTiny, d.y) : d.y;
  const float dz = fabsf(d.z) < kTiny ? copysignf(kTiny, d.z) : d.z;
  r.inv = make_float3(__frcp_rn(dx), __frcp_rn(dy), __frcp_rn(dz));
  r.d_l1 = fabsf(d.x) + fabsf(d.y) + fabsf(d.z);
  return r;
}

__device__ __forceinline__ ff row_apply(const float* hi, const float* lo, int row, ff x, ff y, ff z, bool affine_t) {
  const int k = row * 4;
  ff s = ff_add(ff_add(ff_mul({hi[k], lo[k]}, x), ff_mul({hi[k + 1], lo[k + 1]}, y)), ff_mul({hi[k + 2], lo[k + 2]}, z));
  return affine_t ? ff_add(s, ff{hi[k + 3], lo[k + 3]}) : s;
}

// The per-thread raycastFirst walk of one geometry's roots, nearest child first, in "while-while"
// form (each lane descends internal nodes until it holds a leaf, then the lanes holding one test
// their triangles together).  Returns false on a stack overflow.
__device__ bool blas_first(const MeshDev& m, uint32_t r0, uint32_t r1, const RayF& r, float dlen, int side,
                           const SideTable& sides, float near_d, float far_d, Best& best) {
  uint32_t stack_link[kMaxStack];
  float stack_t[kMaxStack];
  for (uint32_t root = r0; root < r1; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    bool go = true;
    while (go) {
      while (go && !(link & kLeafBit)) {
        const Pair p = load_pair(m.nodes, link);
        const float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
        float e0, e1;
        const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
        const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
        const bool lf = e0 <= e1;
        const uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
        const bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
        if (h1st) {
          if (h2nd) {
            if (sp >= kMaxStack) return false;
            stack_link[sp] = c2;
            stack_t[sp] = lf ? e1 : e0;
            ++sp;
          }
          link = c1;
          continue;
        }
        if (h2nd) {
          link = c2;
          continue;
        }
        go = false;
        const float plim = (best.t + best.err) * (1.0f + kSlabMargin);
        while (sp > 0) {
          --sp;
          if (stack_t[sp] <= plim) {
            link = stack_link[sp];
            go = true;
            break;
          }
        }
      }
      if (!go) break;
      if (link != kEmptyLeaf) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
      go = false;
      const float plim = (best.t + best.err) * (1.0f + kSlabMargin);
      while (sp > 0) {
        --sp;
        if (stack_t[sp] <= plim) {
          link = stack_link[sp];
          go = true;
          break;
        }
      }
    }
  }
  return true;
}

// The local ray of instance I (Ray.applyMatrix4 with the inverse world matrix, direction
// normalised), near / far in local units, and |v| (the unnormalised local direction's length:
// world distance = local t |d| / |v|).  False for a zero local direction.
struct LocalRay {
  RayF r;
  float len, near_d, far_d, vlen;
};
__device__ __noinline__ bool local_ray(const InstanceDev& I, const RayF& w, float near_d, float far_d, LocalRay& L) {
  const ff ox = ff_from(w.o.x), oy = ff_from(w.o.y), oz = ff_from(w.o.z);
  const ff dx = ff_from(w.d.x), dy = ff_from(w.d.y), dz = ff_from(w.d.z);
  const ff lox = row_apply(I.inv_hi, I.inv_lo, 0, ox, oy, oz, true);
  const ff loy = row_apply(I.inv_hi, I.inv_lo, 1, ox, oy, oz, true);
  const ff loz = row_apply(I.inv_hi, I.inv_lo, 2, ox, oy, oz, true);
  const ff vx = row_apply(I.inv_hi, I.inv_lo, 0, dx, dy, dz, false);
  const ff vy = row_apply(I.inv_hi, I.inv_lo, 1, dx, dy, dz, false);
  const ff vz = row_apply(I.inv_hi, I.inv_lo, 2, dx, dy, dz, false);
  const ff vlen = ff_sqrt(ff_add(ff_add(ff_mul(vx, vx), ff_mul(vy, vy)), ff_mul(vz, vz)));
  if (!(vlen.hi > 0.0f)) return false;
  const float3 ld = make_float3(ff_to_f(ff_div(vx, vlen)), ff_to_f(ff_div(vy, vlen)), ff_to_f(ff_div(vz, vlen)));
  L.r = ray_from(make_float3(ff_to_f(lox), ff_to_f(loy), ff_to_f(loz)), ld);
  const float sx = ld.x * I.scale[0], sy = ld.y * I.scale[1], sz = ld.z * I.scale[2];
  const float sf_ = sqrtf(sx * sx + sy * sy + sz * sz);
  L.near_d = near_d / sf_;
  L.far_d = far_d / sf_;
  L.len = sqrtf(ld.x * ld.x + ld.y * ld.y + ld.z * ld.z);
  L.vlen = vlen.hi;
  return true;
}

// The reported record of instance I's hit on triangle record `rec`, in world space: an affine map
// keeps barycentric coordinates and carries the local hit point to the world one, so the
// triangle is carried to world space (float-float) and met with the exact world ray; this avoids
// the rounding of the local ray to float32, which the reference (local ray in float64) does not
// have.  Returns the world distance.
__device__ __noinline__ ff world_record(const MeshDev& m, const InstanceDev& I, uint32_t rec, const RayF& w,
                                        const RayF& lr, bvhc_hit& h) {
  const Tri t = load_tri(m.tris, rec);
  const ff tt = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, lr.o, lr.d));
  make_hit(t, lr, tt, ff_mul(tt, dir_length(lr.d)), h);
  const ff ox = ff_from(w.o.x), oy = ff_from(w.o.y), oz = ff_from(w.o.z);
  const ff dx = ff_from(w.d.x), dy = ff_from(w.d.y), dz = ff_from(w.d.z);
  ff3 P[3];
  const float3 V3s[3] = {t.a, t.b, t.c};
  for (int k = 0; k < 3; ++k) {
    const ff vx = ff_from(V3s[k].x), vy = ff_from(V3s[k].y), vz = ff_from(V3s[k].z);
    P[k] = {row_apply(I.m_hi, I.m_lo, 0, vx, vy, vz, true), row_apply(I.m_hi, I.m_lo, 1, vx, vy, vz, true),
            row_apply(I.m_hi, I.m_lo, 2, vx, vy, vz, true)};
  }
  const ff3 O{ox, oy, oz}, D{dx, dy, dz};
  const ff3 e1 = ff3_sub(P[1], P[0]), e2 = ff3_sub(P[2], P[0]), qv = ff3_sub(O, P[0]);
  const ff3 nn = ff3_cross(e1, e2);
  const ff N = ff3_dot(D, nn);
  ff wx, wy, wz;
  if (N.hi != 0.0f) {
    const ff U = ff3_dot(D, ff3_cross(qv, e2)), Vv = ff3_dot(D, ff3_cross(e1, qv));
    const ff W = ff_sub(ff_sub(N, U), Vv);
    const ff tw = ff_div(ff_neg(ff3_dot(qv, nn)), N);
    wx = ff_add(ox, ff_mul(tw, dx));
    wy = ff_add(oy, ff_mul(tw, dy));
    wz = ff_add(oz, ff_mul(tw, dz));
    if (h.barycoord[0] != 0.0f || h.barycoord[1] != 0.0f || h.barycoord[2] != 0.0f) {
      h.barycoord[0] = ff_to_f(ff_div(W, N));
      h.barycoord[1] = ff_to_f(ff_div(U, N));
      h.barycoord[2] = ff_to_f(ff_div(Vv, N));
    }
  } else {  // the world ray lies in the triangle's plane at float-float resolution
    const ff px = ff_add(ff_from(lr.o.x), ff_mul_f(tt, lr.d.x));
    const ff py = ff_add(ff_from(lr.o.y), ff_mul_f(tt, lr.d.y));
    const ff pz = ff_add(ff_from(lr.o.z), ff_mul_f(tt, lr.d.z));
    wx = row_apply(I.m_hi, I.m_lo, 0, px, py, pz, true);
    wy = row_apply(I.m_hi, I.m_lo, 1, px, py, pz, true);
    wz = row_apply(I.m_hi, I.m_lo, 2, px, py, pz, true);
  }
  const ff ex = ff_sub(wx, ox), ey = ff_sub(wy, oy), ez = ff_sub(wz, oz);
  const ff dist = ff_sqrt(ff_add(ff_add(ff_mul(ex, ex), ff_mul(ey, ey)), ff_mul(ez, ez)));
  h.distance = ff_to_f(dist);
  h.point[0] = ff_to_f(wx);
  h.point[1] = ff_to_f(wy);
  h.point[2] = ff_to_f(wz);
  return dist;
}

// One ray per thread: the instance tree nearest box first, pruned by the closest world hit so
// far; each entered instance box is walked in the instance's frame right away.  With a queue,
// thread i takes ray queue[i] (rays ordered by a Morton key, so that a warp's rays share paths)
// and writes that ray's row.
// Instance-tree stack: the tree is a median split (bvhc_scene_set_instances), so its depth is at most
// log2 of the instance count, below 32 for any instance count the ABI takes; half the geometry
// trees' kMaxStack keeps the per-thread frame (and its spill traffic at high occupancy) smaller.
constexpr int kTlasStack = 32;

// 14 resident blocks per SM (36 registers, some spilled): the kernel stalls on fetching its own
// large body and on its scattered loads, and more resident warps hide both; the instanced bench
// measured 35.6 / 28.4 / 22.7 / 20.4 / 20.4 ms at 5 / 8 / 12 / 14 / 16 blocks.
__global__ void __launch_bounds__(kBlock, 14) scene_raycast_first_kernel(MeshDev m, SceneDev sc,
                                                                        const float* __restrict__ rays, uint64_t n,
                                                                        const uint32_t* __restrict__ queue, int side,
                                                                        float near_d, float far_d,
                                                                        bvhc_hit* __restrict__ out,
                                                                        uint32_t* __restrict__ inst_out) {
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint64_t i = queue ? queue[t] : t;
  const RayF w = make_ray(rays, i);
  const float wlen = sqrtf(w.d.x * w.d.x + w.d.y * w.d.y + w.d.z * w.d.z);
  const SideTable no_sides{};
  bvhc_hit best_hit;
  ff best_dist = ff_from(kInf);
  uint32_t best_inst = 0xFFFFFFFFu;
  uint32_t stack_link[kTlasStack];
  float stack_t[kTlasStack];
  int sp = 0;
  uint32_t link = sc.root;
  bool go = link != kEmptyLeaf;
  // "while-while": every lane descends the instance tree until it holds an instance (or has none
  // left), then the lanes holding one walk their instances together, so the heavy local traversal
  // is not serialised across lanes that reach their instances at different steps
  while (go) {
    while (go && !(link & kLeafBit)) {
      const Pair p = load_pair(sc.nodes, link);
      const float lim = best_dist.hi == kInf ? kInf : best_dist.hi / wlen * (1.0f + 0x1p-16f);
      float e0, e1;
      const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], w, 0.0f, lim, e0);
      const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], w, 0.0f, lim, e1);
      const bool lf = e0 <= e1;
      const uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
      const bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
      if (h1st) {
        if (h2nd) {
          if (sp >= kTlasStack) {
            atomicOr(m.err, kErrStackOverflow);
            go = false;
            break;
          }
          stack_link[sp] = c2;
          stack_t[sp] = lf ? e1 : e0;
          ++sp;
        }
        link = c1;
        continue;
      }
      if (h2nd) {
        link = c2;
        continue;
      }
      go = false;
      while (sp > 0) {
        --sp;
        if (stack_t[sp] <= lim) {
          link = stack_link[sp];
          go = true;
          break;
        }
      }
    }
    if (!go) break;
    {
      const uint32_t j = link & ~kLeafBit;
      const InstanceDev& I = sc.inst[j];
      LocalRay L;
      if (local_ray(I, w, near_d, far_d, L)) {
        const float tlim = best_dist.hi == kInf ? kInf : best_dist.hi * L.vlen / wlen * (1.0f + 0x1p-16f);
        Best b{kInf, 0.0f, 0xFFFFFFFFu};
        const uint32_t g = I.geometry;
        if (!blas_first(m, sc.mesh_root_off[g], sc.mesh_root_off[g + 1], L.r, L.len, side, no_sides, L.near_d,
                        fminf(L.far_d, tlim), b)) {
          atomicOr(m.err, kErrStackOverflow);
          break;
        }
        if (b.rec != 0xFFFFFFFFu) {
          bvhc_hit h;
          const ff dist = world_record(m, I, b.rec, w, L.r, h);
          if (ff_lt(dist, best_dist) || (!ff_lt(best_dist, dist) && j < best_inst)) {
            best_dist = dist;
            best_inst = j;
            best_hit = h;
          }
        }
      }
    }
    go = false;
    const float lim = best_dist.hi == kInf ? kInf : best_dist.hi / wlen * (1.0f + 0x1p-16f);
    while (sp > 0) {
      --sp;
      if (stack_t[sp] <= lim) {
        link = stack_link[sp];
        go = true;
        break;
      }
    }
  }
  if (best_inst == 0xFFFFFFFFu) {
    store_miss(out + i);
  } else {
    store_hit(out + i, best_hit);
  }
  inst_out[i] = best_inst;
}

// Instanced raycast (all hits): the BatchedMesh raycast without firstHitOnly.  Every entered
// instance box (no pruning: the count covers every hit) is walked in the instance's frame with the
// reference's all-hits DFS (left child before right), each hit converted to world space and
// inserted into the ray's row kept sorted by (world distance, instance): the raycaster's stable
// sort of the per-instance hit lists concatenated in instance order.  Stores the first `cap`,
// counts[i] the total.
// 14 resident blocks per SM, as the first-hit kernel: 121.5 / 89.0 / 68.3 ms at 5 / 8 / 14 blocks
// for 2^22 world rays over 4096 instances (cap 16).
__global__ void __launch_bounds__(kBlock, 14) scene_raycast_all_kernel(MeshDev m, SceneDev sc,
                                                                      const float* __restrict__ rays, uint64_t n,
                                                                      int side, float near_d, float far_d, uint32_t cap,
                                                                      uint32_t* __restrict__ counts,
                                                                      bvhc_hit* __restrict__ hits,
                                                                      uint32_t* __restrict__ inst_out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RayF w = make_ray(rays, i);
  const SideTable no_sides{};
  bvhc_hit* row = hits + i * (uint64_t)cap;
  uint32_t* irow = inst_out + i * (uint64_t)cap;
  uint32_t cnt = 0, stored = 0;
  uint32_t tstack[kTlasStack];
  uint32_t bstack[kMaxStack];
  int tsp = 0;
  uint32_t link = sc.root;
  bool go = link != kEmptyLeaf;
  while (go) {
    while (go && !(link & kLeafBit)) {
      const Pair p = load_pair(sc.nodes, link);
      float e0, e1;
      const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], w, 0.0f, kInf, e0);
      const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], w, 0.0f, kInf, e1);
      if (h0 && h1) {
        if (tsp >= kTlasStack) {
          atomicOr(m.err, kErrStackOverflow);
          go = false;
          break;
        }
        tstack[tsp++] = p.lr;
        link = p.ll;
      } else if (h0 || h1) {
        link = h0 ? p.ll : p.lr;
      } else if (tsp > 0) {
        link = tstack[--tsp];
      } else {
        go = false;
      }
    }
    if (!go) break;
    const uint32_t j = link & ~kLeafBit;
    const InstanceDev& I = sc.inst[j];
    LocalRay L;
    if (local_ray(I, w, near_d, far_d, L)) {
      const ff dlen = dir_length(L.r.d);
      const uint32_t g = I.geometry;
      for (uint32_t root = sc.mesh_root_off[g]; root < sc.mesh_root_off[g + 1]; ++root) {
        uint32_t bl = m.roots[root];
        int bsp = 0;
        for (;;) {
          if (bl & kLeafBit) {
            if (bl != kEmptyLeaf) {
              for (uint32_t k = bl & ~kLeafBit;; ++k) {
                const Tri t = load_tri(m.tris, k);
                const int ts = tri_side(t, side, no_sides);
                if (ts >= 0 && tri_hit(t.a, t.b, t.c, L.r.o, L.r.d, L.r.d_l1, ts)) {
                  const ff tt = tri_t_ff(tri_eval_ff(t.a, t.b, t.c, L.r.o, L.r.d));
                  const ff dist = ff_mul(tt, dlen);
                  if (!ff_lt(dist, ff_from(L.near_d)) && !ff_lt(ff_from(L.far_d), dist)) {
                    ++cnt;
                    bvhc_hit h;
                    world_record(m, I, k, w, L.r, h);
                    // stable sorted insert by (distance, instance)
                    uint32_t pos = stored;
                    while (pos > 0) {
                      const float pd = row[pos - 1].distance;
                      if (pd < h.distance || (pd == h.distance && irow[pos - 1] <= j)) break;
                      --pos;
                    }
                    if (pos < cap) {
                      const uint32_t last = stored < cap ? stored : cap - 1;
                      for (uint32_t q = last; q > pos; --q) {
                        row[q] = row[q - 1];
                        irow[q] = irow[q - 1];
                      }
                      row[pos] = h;
                      irow[pos] = j;
                      if (stored < cap) ++stored;
                    }
                  }
                }
                if (t.flags & kTriLast) break;
              }
            }
          } else {
            const Pair p = load_pair(m.nodes, bl);
            float e0, e1;
            const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], L.r, L.near_d, L.far_d, e0);
            const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], L.r, L.near_d, L.far_d, e1);
            if (h0) {
              if (h1) {
                if (bsp >= kMaxStack) {
                  atomicOr(m.err, kErrStackOverflow);
                  break;
                }
                bstack[bsp++] = p.lr;
              }
              bl = p.ll;
              continue;
            }
            if (h1) {
              bl = p.lr;
              continue;
            }
          }
          if (bsp == 0) break;
          bl = bstack[--bsp];
        }
      }
    }
    if (tsp == 0) break;
    link = tstack[--tsp];
  }
  for (uint32_t q = stored; q < cap; ++q) {
    store_miss(row + q);
    irow[q] = 0xFFFFFFFFu;
  }
  counts[i] = cnt;
}

// Keys of world rays, ids in input order: kinds 1..3 a Morton key over the instances' box
// (ray_key); kind 4 the first instance the ray's nearest-first descent of the instance tree
// reaches (0xFFFFFF: none), so that a warp's rays walk the same geometry tree.
__global__ void __launch_bounds__(kBlock) scene_key_kernel(const float* __restrict__ rays, uint64_t n, int kind,
                                                           SceneBox box, SceneDev sc, uint32_t* __restrict__ ids,
                                                           uint32_t* __restrict__ keys, unsigned int* qcount) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *qcount = (unsigned int)n;
  if (i >= n) return;
  const RayF r = make_ray(rays, i);
  ids[i] = (uint32_t)i;
  if (kind != 4) {
    keys[i] = ray_key(kind, r.o, r.d, box);
    return;
  }
  uint32_t key = 0xFFFFFFu;
  uint32_t stack_link[kMaxStack];
  int sp = 0;
  uint32_t link = sc.root;
  bool go = link != kEmptyLeaf;
  while (go) {
    if (link & kLeafBit) {
      key = (link & ~kLeafBit) & 0xFFFFFFu;
      break;
    }
    const Pair p = load_pair(sc.nodes, link);
    float e0, e1;
    const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, 0.0f, kInf, e0);
    const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, 0.0f, kInf, e1);
    const bool lf = e0 <= e1;
    const uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
    const bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
    if (h1st) {
      if (h2nd && sp < kMaxStack) stack_link[sp++] = c2;
      link = c1;
    } else if (h2nd) {
      link = c2;
    } else if (sp > 0) {
      link = stack_link[--sp];
    } else {
      go = false;
    }
  }
  keys[i] = key;
}

// Morton key of each query point over the scene box (8 bits per axis), ids in input order, and the
// queue length; the queue is then sorted by key so that a warp takes 32 nearby points.
__global__ void __launch_bounds__(kBlock) point_key_kernel(const float* __restrict__ pts, uint64_t n, SceneBox box,
                                                          uint32_t* __restrict__ ids, uint32_t* __restrict__ keys,
                                                          unsigned int* __restrict__ qcount) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *qcount = (unsigned int)n;
  if (i >= n) return;
  float sx = box.hi[0] > box.lo[0] ? 1.0f / (box.hi[0] - box.lo[0]) : 0.0f;
  float sy = box.hi[1] > box.lo[1] ? 1.0f / (box.hi[1] - box.lo[1]) : 0.0f;
  float sz = box.hi[2] > box.lo[2] ? 1.0f / (box.hi[2] - box.lo[2]) : 0.0f;
  ids[i] = (uint32_t)i;
  keys[i] = morton3(quantise(__ldg(pts + 3 * i), box.lo[0], sx, 256.0f),
                    quantise(__ldg(pts + 3 * i + 1), box.lo[1], sy, 256.0f),
                    quantise(__ldg(pts + 3 * i + 2), box.lo[2], sz, 256.0f));
}

// Morton key of each shape's centre over the mesh box (8 bits per axis), ids in input order, and
// the queue length: kind 0 spheres (cx, cy, cz, r), kind 1 oriented boxes (the box-to-mesh matrix
// applied to the centre of the local box).  The shapecast kernels then take the queries in key
// order, so the 32 lanes of a warp hold nearby shapes whose traversals mostly coincide.
__global__ void __launch_bounds__(kBlock) shape_key_kernel(const float* __restrict__ q, uint64_t n, int kind,
                                                          SceneBox box, uint32_t* __restrict__ ids,
                                                          uint32_t* __restrict__ keys,
                                                          unsigned int* __restrict__ qcount) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *qcount = (unsigned int)n;
  if (i >= n) return;
  float p[3];
  if (kind == 0) {
    const float4 v = ld4(q + 4 * i);
    p[0] = v.x;
    p[1] = v.y;
    p[2] = v.z;
  } else {
    const float* b = q + 24 * i;
    const float* e = b + 8;
    const float x = 0.5f * (__ldg(b) + __ldg(b + 4)), y = 0.5f * (__ldg(b + 1) + __ldg(b + 5)),
                z = 0.5f * (__ldg(b + 2) + __ldg(b + 6));
    for (int k = 0; k < 3; ++k)
      p[k] = fmaf(__ldg(e + k), x, fmaf(__ldg(e + 4 + k), y, fmaf(__ldg(e + 8 + k), z, __ldg(e + 12 + k))));
  }
  uint32_t c[3];
  for (int a = 0; a < 3; ++a) {
    const float inv = box.hi[a] > box.lo[a] ? 1.0f / (box.hi[a] - box.lo[a]) : 0.0f;
    c[a] = quantise(p[a], box.lo[a], inv, 256.0f);
  }
  ids[i] = (uint32_t)i;
  keys[i] = morton3(c[0], c[1], c[2]);
}

// ---------------------------------------------------------------------------------------------
// raycastFirst, persistent form.  A fixed grid of warps pulls rays from a global work counter in
// chunks of 32..kChunk rays per warp (one atomicAdd per chunk); a lane whose ray is finished sits idle
// until `refill` lanes of its warp are idle, and then those lanes take the next rays of the warp's
// chunk together, so warps stay full while rays of very different cost (early misses, deep
// traversals) are mixed.  Each outer iteration runs the "while-while" phases: every lane walks
// child pairs until it reaches a leaf or finishes, then the lanes holding a leaf test it together.
// A finished hit is written as a pending (record, t) pair; finalize_first_kernel then computes the
// reported records one ray per thread, so the float-float work runs with full warps.
// ---------------------------------------------------------------------------------------------
constexpr unsigned kChunk = 256;

// Mesh of ray `rid` in a batch: the last mesh whose first ray is <= rid (ray_off is CSR).
__device__ __forceinline__ int mesh_of_ray(const BatchDev& bd, uint64_t rid) {
  int lo = 0, hi = bd.n_meshes - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(bd.ray_off + mid) <= rid) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// BATCHED: every ray belongs to one of many meshes packed into one node/triangle pool (the
// meshes of a BatchedMesh, ExtensionUtilities.js:87-161); a lane looks up its ray's mesh when it
// takes the ray and traverses that mesh's roots.  Otherwise the mesh's roots are m.roots[0..n).
// MINB: minimum resident blocks per SM requested from the register allocator (1 = no limit).
template <int ORDER, bool BATCHED, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) raycast_first_persistent_kernel(
    MeshDev m, const BatchDev bd, const float* __restrict__ rays, uint64_t n, int side, const SideTable sides,
    float near_d, float far_d, bvhc_hit* __restrict__ out, unsigned long long* __restrict__ work, int refill,
    const uint32_t* __restrict__ queue, const unsigned int* __restrict__ qcount) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  // with a queue (written by classify_kernel) the work items are its entries, else all rays
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  // rays per warp fetch: about eight fetches per warp over the launch, between 32 and kChunk, so
  // that small batches still spread over every resident warp
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  uint64_t chunk = n_work / (warps * 8);
  chunk = chunk < 32 ? 32 : (chunk > kChunk ? kChunk : (chunk & ~31ull));
  bool active = false;
  uint64_t rid = 0;
  RayF r;
  float dlen = 0.0f;
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  uint32_t link = 0;
  int sp = 0, root = 0, root_end = m.n_roots;
  uint32_t stack_link[kMaxStack];
  float stack_t[kMaxStack];
  uint64_t pool = 0, pool_end = 0;  // warp-uniform: this warp's untaken rays [pool, pool_end)
  bool drained = false;             // warp-uniform: the work counter is exhausted

  // Next link after a leaf or a dead end: pop the nearest stacked child whose entry distance does
  // not lie beyond the best hit, else move to the next root, else finish the ray.
  auto pop_next = [&]() {
    float lim = (best.t + best.err) * (1.0f + kSlabMargin);
    while (sp > 0) {
      --sp;
      if (stack_t[sp] <= lim) {
        link = stack_link[sp];
        return;
      }
    }
    if (++root < root_end) {
      link = m.roots[root];
      return;
    }
    if (best.rec == 0xFFFFFFFFu) {
      store_miss(out + rid);
    } else {
      // pending: the record index in face_index, finalize_first_kernel completes it
      __stcs(reinterpret_cast<float4*>(out + rid), make_float4(__uint_as_float(best.rec), best.t, 0.0f, 0.0f));
    }
    active = false;
  };

  for (;;) {
    unsigned idle = __ballot_sync(0xFFFFFFFFu, !active);
    if (idle == 0xFFFFFFFFu || (idle != 0u && __popc(idle) >= refill)) {
      unsigned need = __popc(idle);
      uint64_t avail = pool_end - pool;
      uint64_t nb = 0, ne = 0;
      if (need > avail && !drained) {
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(work, (unsigned long long)chunk);
        b = __shfl_sync(0xFFFFFFFFu, b, 0);
        if (b >= n_work) {
          drained = true;
        } else {
          nb = b;
          ne = b + chunk < n_work ? b + chunk : n_work;
        }
      }
      if (!active) {
        uint64_t rank = __popc(idle & lt_mask);
        bool got = true;
        if (rank < avail) rid = pool + rank;
        else if (rank - avail < ne - nb) rid = nb + (rank - avail);
        else got = false;
        if (got && queue) rid = __ldg(queue + rid);
        if (got) {
          active = true;
          r = make_ray(rays, rid);
          dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
          best = Best{kInf, 0.0f, 0xFFFFFFFFu};
          if (BATCHED) {
            int mesh = mesh_of_ray(bd, rid);
            root = (int)__ldg(bd.mesh_root_off + mesh);
            root_end = (int)__ldg(bd.mesh_root_off + mesh + 1);
          } else {
            root = 0;
            root_end = m.n_roots;
          }
          sp = 0;
          link = m.roots[root];
        }
      }
      if (need <= avail) {
        pool += need;
      } else {
        uint64_t used = need - avail;
        pool = nb + used < ne ? nb + used : ne;
        pool_end = ne;
      }
      if (idle == 0xFFFFFFFFu && __ballot_sync(0xFFFFFFFFu, active) == 0u) break;
    }
    if (!active) continue;
    // phase 1: child pairs, until this lane holds a leaf or has finished its ray
    while (active && !(link & kLeafBit)) {
      Pair p = load_pair(m.nodes, link);
      float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
      float e0, e1;
      bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
      bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
      bool lf = left_first<ORDER>(p, r, e0, e1);
      uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
      bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
      if (h1st && h2nd) {
        if (sp >= kMaxStack) {
          atomicOr(m.err, kErrStackOverflow);
          best.rec = 0xFFFFFFFFu;
          sp = 0;
          root = root_end;
          pop_next();
        } else {
          stack_link[sp] = c2;
          stack_t[sp] = lf ? e1 : e0;
          ++sp;
          link = c1;
        }
      } else if (h1st) {
        link = c1;
      } else if (h2nd) {
        link = c2;
      } else {
        pop_next();
      }
    }
    // phase 2: the leaf
    if (active) {
      if (link != kEmptyLeaf) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
      pop_next();
    }
  }
}

// Completes the pending hits of raycast_first_persistent_kernel, one ray per thread (grid-stride).
// With a queue only its entries can be pending; the other rays were finished by classify_kernel.
__global__ void __launch_bounds__(kBlock) finalize_first_kernel(MeshDev m, const float* __restrict__ rays, uint64_t n,
                                                                bvhc_hit* __restrict__ out,
                                                                const uint32_t* __restrict__ queue,
                                                                const unsigned int* __restrict__ qcount) {
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_work; k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = queue ? (uint64_t)__ldg(queue + k) : k;
    uint32_t rec = __float_as_uint(__ldcs(reinterpret_cast<const float*>(out + i)));
    if (rec == BVHC_NO_HIT) continue;
    RayF r = make_ray(rays, i);
    finish_first(m, rec, r, out + i);
  }
}

// Pre-pass for the persistent and warp-cooperative traversals: a ray whose box tests against every
// root's two children (with the root's own leaf case always live) all fail cannot hit anything; it
// is finished here with a coalesced miss record.  The other rays are appended to `queue` in ray
// order (one atomic per block reserves the block's run; positions within it come from ballots), so
// the traversal kernel's warps only carry rays that enter the tree.  With `keys`, each queued ray's
// ordering key (raykey.cuh, kind `kind`) is written beside its id.  With `miss_counts` (all-hits
// raycast) a ray that misses gets a hit count of 0 instead of a miss record.
constexpr int kClsThreads = 256;
constexpr int kClsItems = 8;
constexpr int kClsTile = kClsThreads * kClsItems;  // rays per block
constexpr int kClsWarps = kClsThreads / 32;

template <bool BATCHED>
__global__ void __launch_bounds__(kClsThreads) classify_kernel(
    MeshDev m, const BatchDev bd, const float* __restrict__ rays, uint64_t n, float near_d, float far_d,
    bvhc_hit* __restrict__ out, uint32_t* __restrict__ queue, unsigned int* __restrict__ qcount,
    uint32_t* __restrict__ keys, int kind, SceneBox box, uint32_t* __restrict__ miss_counts = nullptr) {
  __shared__ unsigned s_cnt[kClsItems * kClsWarps];  // live rays per (item round, warp), then prefixes
  __shared__ unsigned s_base;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kClsTile;
  unsigned ballot[kClsItems];
  uint32_t key[kClsItems];
#pragma unroll
  for (int j = 0; j < kClsItems; ++j) {
    uint64_t i = base + (uint64_t)j * kClsThreads + threadIdx.x;
    bool live = false;
    key[j] = 0;
    if (i < n) {
      RayF r = make_ray(rays, i);
      int root = 0, root_end = m.n_roots;
      if (BATCHED) {
        int mesh = mesh_of_ray(bd, i);
        root = (int)__ldg(bd.mesh_root_off + mesh);
        root_end = (int)__ldg(bd.mesh_root_off + mesh + 1);
      }
      for (; root < root_end && !live; ++root) {
        uint32_t link = __ldg(m.roots + root);
        if (link & kLeafBit) {
          live = link != kEmptyLeaf;
          continue;
        }
        Pair p = load_pair(m.nodes, link);
        float e;
        live = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e) ||
               box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e);
      }
      if (!live) {
        if (miss_counts) miss_counts[i] = 0;  // all hits: the uncapped count of a ray that misses
        else store_miss(out + i);
      }
      else if (keys) key[j] = ray_key(kind, r.o, r.d, box);
    }
    ballot[j] = __ballot_sync(0xFFFFFFFFu, live);
    if (lane == 0) s_cnt[j * kClsWarps + w] = (unsigned)__popc(ballot[j]);
  }
  __syncthreads();
  if (w == 0) {
    // exclusive scan of the 64 counts in (round, warp) order, which is ray order
    static_assert(kClsItems * kClsWarps == 64, "two counts per lane");
    unsigned a = s_cnt[2 * lane], b = s_cnt[2 * lane + 1];
    unsigned incl = a + b;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= (unsigned)o) incl += y;
    }
    unsigned excl = incl - a - b;
    s_cnt[2 * lane] = excl;
    s_cnt[2 * lane + 1] = excl + a;
    unsigned total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (lane == 0) s_base = total ? atomicAdd(qcount, total) : 0u;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kClsItems; ++j) {
    if (ballot[j] & (1u << lane)) {
      unsigned pos = s_base + s_cnt[j * kClsWarps + w] + (unsigned)__popc(ballot[j] & lt);
      queue[pos] = (uint32_t)(base + (uint64_t)j * kClsThreads + threadIdx.x);
      if (keys) keys[pos] = key[j];
    }
  }
}

}  // namespace dev

static unsigned int grid_for(uint64_t n) { return (unsigned int)((n + dev::kBlock - 1) / dev::kBlock); }

// Resident blocks per SM x SM count for a persistent kernel on the current device, cached per
// (device, kernel variant).
template <class K>
static unsigned int persistent_grid(K kernel, int variant) {
  constexpr int kDevs = 64, kVariants = 12;
  static unsigned int cache[kDevs][kVariants] = {};
  int dev_id = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev_id);
  if (dev_id >= 0 && dev_id < kDevs && cache[dev_id][variant]) return cache[dev_id][variant];
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, dev::kBlock, 0);
  unsigned int g = (unsigned int)(std::max(1, sms) * std::max(1, per_sm));
  if (dev_id >= 0 && dev_id < kDevs) cache[dev_id][variant] = g;
  return g;
}

struct PersistentArgs {
  MeshDev m;
  BatchDev bd;
  const float* rays;
  uint64_t n;
  int side;
  SideTable sides;
  float near_d, far_d;
  bvhc_hit* out;
  unsigned long long* work;
  int refill;
  const uint32_t* queue;
  const unsigned int* qcount;
};

template <int ORDER, bool BATCHED, int MINB>
static void launch_persistent(const PersistentArgs& a, cudaStream_t stream) {
  auto kernel = dev::raycast_first_persistent_kernel<ORDER, BATCHED, MINB>;
  int variant = ORDER * 6 + (BATCHED ? 3 : 0) + (MINB == 1 ? 0 : (MINB == 6 ? 1 : 2));
  unsigned int g = persistent_grid(kernel, variant);
  g = (unsigned int)std::min<uint64_t>(g, (a.n + dev::kBlock - 1) / dev::kBlock);
  kernel<<<g, dev::kBlock, 0, stream>>>(a.m, a.bd, a.rays, a.n, a.side, a.sides, a.near_d, a.far_d, a.out, a.work,
                                        a.refill, a.queue, a.qcount);
}

template <int ORDER, bool BATCHED>
static void launch_persistent_occ(const PersistentArgs& a, int occupancy, cudaStream_t stream) {
  if (occupancy == 0) launch_persistent<ORDER, BATCHED, 1>(a, stream);
  else if (occupancy == 1) launch_persistent<ORDER, BATCHED, 6>(a, stream);
  else launch_persistent<ORDER, BATCHED, 8>(a, stream);
}

// Root-box pre-pass into `queue`, then (single mesh, sort requested) the ray-ordering sort.
static cudaError_t prepare_queue(const MeshDev& m, const BatchDev* batch, const float* rays, uint64_t n, float near_d,
                                 float far_d, bvhc_hit* out, uint32_t* queue, unsigned int* qcount,
                                 const RaySort* sort, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(qcount, 0, sizeof(unsigned int), stream);
  if (e != cudaSuccess) return e;
  BatchDev bd = batch ? *batch : BatchDev{nullptr, nullptr, 0};
  const bool sorted = sort && !batch && sort->kind > 0;
  // a sorted queue is first written (with keys) where the sort's passes start, so they end in `queue`
  uint32_t* ids = queue;
  uint32_t* keys = nullptr;
  if (sorted) ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
  dev::SceneBox box{};
  if (sorted) {
    for (int a = 0; a < 3; ++a) {
      box.lo[a] = sort->lo[a];
      box.hi[a] = sort->hi[a];
    }
  }
  const int kind = sorted ? sort->kind : 0;
  const unsigned int g = (unsigned int)((n + dev::kClsTile - 1) / dev::kClsTile);
  if (batch)
    dev::classify_kernel<true><<<g, dev::kClsThreads, 0, stream>>>(m, bd, rays, n, near_d, far_d, out, ids, qcount,
                                                                   keys, kind, box);
  else
    dev::classify_kernel<false><<<g, dev::kClsThreads, 0, stream>>>(m, bd, rays, n, near_d, far_d, out, ids, qcount,
                                                                    keys, kind, box);
  e = cudaGetLastError();
  if (e != cudaSuccess || !sorted) return e;
  return launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream);
}

cudaError_t launch_raycast_first_persistent(const MeshDev& m, const BatchDev* batch, const float* rays, uint64_t n,
                                            int side, const SideTable& sides, float near_d, float far_d,
                                            bvhc_hit* out, unsigned long long* work, const TraversalConfig& cfg,
                                            cudaStream_t stream, uint32_t* queue, unsigned int* qcount,
                                            const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  const bool compact = queue != nullptr && qcount != nullptr && n < (1ull << 32);
  BatchDev bd = batch ? *batch : BatchDev{nullptr, nullptr, 0};
  if (compact) {
    e = prepare_queue(m, batch, rays, n, near_d, far_d, out, queue, qcount, sort, stream);
    if (e != cudaSuccess) return e;
  }
  PersistentArgs a{m, bd, rays, n, side, sides, near_d, far_d, out, work, cfg.refill,
                   compact ? queue : nullptr, compact ? qcount : nullptr};
  if (batch) {
    if (cfg.order == 0) launch_persistent_occ<0, true>(a, cfg.occupancy, stream);
    else launch_persistent_occ<1, true>(a, cfg.occupancy, stream);
  } else {
    if (cfg.order == 0) launch_persistent_occ<0, false>(a, cfg.occupancy, stream);
    else launch_persistent_occ<1, false>(a, cfg.occupancy, stream);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  unsigned int fg = (unsigned int)std::min<uint64_t>(grid_for(n), 8192);
  dev::finalize_first_kernel<<<fg, dev::kBlock, 0, stream>>>(m, rays, n, out, a.queue, a.qcount);
  return cudaGetLastError();
}

cudaError_t launch_raycast_first_packet(const MeshDev& m, const float* rays, uint64_t n, int side,
                                        const SideTable& sides, float near_d, float far_d, bvhc_hit* out, int order,
                                        int occupancy, int wide, cudaStream_t stream, uint32_t* queue,
                                        unsigned int* qcount, const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  const bool compact = queue != nullptr && qcount != nullptr && n < (1ull << 32);
  if (compact) {
    cudaError_t e = prepare_queue(m, nullptr, rays, n, near_d, far_d, out, queue, qcount, sort, stream);
    if (e != cudaSuccess) return e;
  } else {
    queue = nullptr;
    qcount = nullptr;
  }
  if (wide && m.quads && m.quad_roots) {
    auto k4 = occupancy == 0   ? dev::raycast_first_packet4_kernel<1>
              : occupancy == 1 ? dev::raycast_first_packet4_kernel<6>
                               : dev::raycast_first_packet4_kernel<8>;
    k4<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out, queue, qcount);
    return cudaGetLastError();
  }
  auto kernel = order == 0 ? (occupancy == 0 ? dev::raycast_first_packet_kernel<0, 1>
                                              : occupancy == 1 ? dev::raycast_first_packet_kernel<0, 6>
                                                               : dev::raycast_first_packet_kernel<0, 8>)
                            : (occupancy == 0 ? dev::raycast_first_packet_kernel<1, 1>
                                              : occupancy == 1 ? dev::raycast_first_packet_kernel<1, 6>
                                                               : dev::raycast_first_packet_kernel<1, 8>);
  kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out, queue, qcount);
  return cudaGetLastError();
}

cudaError_t launch_raycast_first(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                                 float near_d, float far_d, bvhc_hit* out, int order, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if (order == 0)
    dev::raycast_first_kernel<0><<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out);
  else
    dev::raycast_first_kernel<1><<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out);
  return cudaGetLastError();
}

cudaError_t launch_raycast_all(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                               float near_d, float far_d, uint32_t cap, uint32_t* counts, bvhc_hit* hits,
                               cudaStream_t stream, int variant, int occupancy, uint32_t* queue, unsigned int* qcount,
                               const RaySort* sort, unsigned long long* work) {
  if (n == 0) return cudaSuccess;
  if (variant == 0 || (variant == 2 && (!queue || !qcount || !sort || n >= (1ull << 32))) ||
      ((variant == 5 || variant == 9) && (!queue || !qcount || n >= (1ull << 32)))) {
    dev::raycast_all_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, cap,
                                                                      counts, hits);
    return cudaGetLastError();
  }
  cudaError_t e;
  if (variant == 9 && !work) variant = 5;
  if (variant == 5 || variant == 9) {
    // the root-box pre-pass gives the rays that miss a count of 0 and queues the others (in ray
    // order, or sorted by the key sort->kind) for one ray per thread: a warp then holds 32 rays
    // that enter the tree (neighbouring ones with a key); variant 9 walks the queue with
    // persistent warps that refill idle lanes
    if ((e = cudaMemsetAsync(qcount, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
    const unsigned int g = (unsigned int)((n + dev::kClsTile - 1) / dev::kClsTile);
    const bool keyed = sort && sort->kind > 0;
    uint32_t *ids = queue, *keys = nullptr;
    dev::SceneBox box{};
    if (keyed) {
      ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
      for (int a = 0; a < 3; ++a) {
        box.lo[a] = sort->lo[a];
        box.hi[a] = sort->hi[a];
      }
    }
    dev::classify_kernel<false><<<g, dev::kClsThreads, 0, stream>>>(m, BatchDev{nullptr, nullptr, 0}, rays, n, near_d,
                                                                    far_d, nullptr, ids, qcount, keys,
                                                                    keyed ? sort->kind : 0, box, counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (keyed && (e = launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
    if (variant == 9) {
      if ((e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), stream)) != cudaSuccess) return e;
      int dev_id = 0, sms = 148;
      cudaGetDevice(&dev_id);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
      dev::raycast_all_persistent_kernel<<<sms * dev::kAllBlocksPerSm, dev::kBlock, 0, stream>>>(m, rays, side, sides, near_d, far_d, cap,
                                                                              counts, hits, queue, qcount, work);
      return cudaGetLastError();
    }
    dev::raycast_all_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, cap,
                                                                      counts, hits, queue, qcount);
    return cudaGetLastError();
  }
  if (variant == 2) {
    // the root-box pre-pass gives the rays that miss a count of 0 and queues the others with their
    // keys, which are then sorted
    uint32_t *ids, *keys;
    ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
    dev::SceneBox box{};
    for (int a = 0; a < 3; ++a) {
      box.lo[a] = sort->lo[a];
      box.hi[a] = sort->hi[a];
    }
    if ((e = cudaMemsetAsync(qcount, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
    const unsigned int g = (unsigned int)((n + dev::kClsTile - 1) / dev::kClsTile);
    dev::classify_kernel<false><<<g, dev::kClsThreads, 0, stream>>>(m, BatchDev{nullptr, nullptr, 0}, rays, n, near_d,
                                                                    far_d, nullptr, ids, qcount, keys, sort->kind, box,
                                                                    counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
  } else {
    queue = nullptr;
    qcount = nullptr;
  }
  auto kernel = occupancy == 0   ? dev::raycast_all_packet_kernel<1>
                : occupancy == 1 ? dev::raycast_all_packet_kernel<6>
                                 : dev::raycast_all_packet_kernel<8>;
  kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, cap, counts, hits, queue,
                                                  qcount);
  return cudaGetLastError();
}

cudaError_t launch_closest_point(const MeshDev& m, const float* pts, uint64_t n, float min_t, float max_t,
                                 bvhc_closest* out, cudaStream_t stream, int variant, int occupancy, uint32_t* queue,
                                 unsigned int* qcount, const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  // the warp-cooperative form needs minThreshold 0 (see closest_point_packet_kernel)
  if (variant == 0 || !(min_t <= 0.0f) || (variant == 2 && (!queue || !qcount || !sort || n >= (1ull << 32)))) {
    dev::closest_point_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, pts, n, min_t, max_t, out);
    return cudaGetLastError();
  }
  cudaError_t e;
  if (variant == 2) {
    uint32_t *ids, *keys;
    ray_sort_input(2, sort->scratch, queue, &ids, &keys);
    dev::SceneBox box{};
    for (int a = 0; a < 3; ++a) {
      box.lo[a] = sort->lo[a];
      box.hi[a] = sort->hi[a];
    }
    dev::point_key_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(pts, n, box, ids, keys, qcount);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_ray_sort(2, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
  } else {
    queue = nullptr;
    qcount = nullptr;
  }
  auto kernel = occupancy == 0   ? dev::closest_point_packet_kernel<1>
                : occupancy == 1 ? dev::closest_point_packet_kernel<6>
                                 : dev::closest_point_packet_kernel<8>;
  kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, pts, n, max_t, out, queue, qcount);
  return cudaGetLastError();
}

namespace dev {

// Intersection attribute fields (ThreeRayIntersectUtilities.js:59-117): a vertex attribute at the
// hit point, Triangle.getInterpolation with the recorded barycentrics; with rays given (normals),
// the result is negated when it points along the ray.  Misses give zeros.
// ---------------------------------------------------------------------------------------------
// getTriangleHitPointInfo (src/utils/TriangleUtilities.js:65-147) for a batch of (point,
// triangle) pairs, in the integer-emulated binary64 of softf64.cuh so that the degenerate cases
// fall exactly as the reference's float64 arithmetic has them:
//   barycoord  the dot-product solve with v0 = c - a, v1 = b - a, v2 = p - a:
//              denom = (v0.v0)(v1.v1) - (v0.v1)^2, u = ((v1.v1)(v0.v2) - (v0.v1)(v1.v2)) / denom,
//              v = ((v0.v0)(v1.v2) - (v0.v1)(v0.v2)) / denom, barycoord = (1 - u - v, v, u);
//              (0, 0, 0) when denom is exactly 0 (Triangle.getBarycoord),
//   uv         the uvs weighted by that barycoord, (0, 0) for a degenerate triangle
//              (Triangle.getInterpolation),
//   normal     (c - b) x (a - b) scaled by 1 / |.|, (0, 0, 0) when its squared length is 0
//              (Triangle.getNormal),
//   face       the index's three vertex ids and the material of the first group that holds the
//              triangle's first index (0 when none does).
// ---------------------------------------------------------------------------------------------
namespace hpi {
using sf::f64;
struct V {
  f64 x, y, z;
};
__device__ __forceinline__ V load(const float* p) {
  return {sf::from_f32(__ldg(p)), sf::from_f32(__ldg(p + 1)), sf::from_f32(__ldg(p + 2))};
}
__device__ __forceinline__ V sub(V a, V b) { return {sf::sub(a.x, b.x), sf::sub(a.y, b.y), sf::sub(a.z, b.z)}; }
__device__ __forceinline__ f64 dot(V a, V b) {
  return sf::add(sf::add(sf::mul(a.x, b.x), sf::mul(a.y, b.y)), sf::mul(a.z, b.z));
}
__device__ __forceinline__ V cross(V a, V b) {
  return {sf::sub(sf::mul(a.y, b.z), sf::mul(a.z, b.y)), sf::sub(sf::mul(a.z, b.x), sf::mul(a.x, b.z)),
          sf::sub(sf::mul(a.x, b.y), sf::mul(a.y, b.x))};
}
}  // namespace hpi

__global__ void __launch_bounds__(kBlock) triangle_hit_point_info_kernel(
    const float* __restrict__ points, const uint32_t* __restrict__ faces, uint64_t n,
    const uint32_t* __restrict__ tri_vid, uint64_t n_tri, const float* __restrict__ pos, int pos_stride,
    const float* __restrict__ uv, int uv_stride, const GroupTable groups, bvhc_hit_point_info* __restrict__ out,
    unsigned int* err) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bvhc_hit_point_info r;
  r.a = r.b = r.c = BVHC_NO_HIT;
  r.material_index = 0;
  for (int k = 0; k < 3; ++k) r.normal[k] = r.barycoord[k] = 0.0f;
  r.uv[0] = r.uv[1] = 0.0f;
  const uint32_t f = __ldg(faces + i);
  if (f >= n_tri) {
    atomicOr(err, kErrBadFace);
    out[i] = r;
    return;
  }
  const uint32_t va = __ldg(tri_vid + 3 * (uint64_t)f), vb = __ldg(tri_vid + 3 * (uint64_t)f + 1),
                 vc = __ldg(tri_vid + 3 * (uint64_t)f + 2);
  r.a = va;
  r.b = vb;
  r.c = vc;
  const int64_t first = 3 * (int64_t)f;
  for (int g = 0; g < groups.n; ++g) {
    if (first >= groups.start[g] && (groups.count[g] < 0 || first < groups.start[g] + groups.count[g])) {
      r.material_index = (uint32_t)groups.material[g];
      break;
    }
  }
  const hpi::V A = hpi::load(pos + (uint64_t)va * pos_stride), B = hpi::load(pos + (uint64_t)vb * pos_stride),
               C = hpi::load(pos + (uint64_t)vc * pos_stride), P = hpi::load(points + 3 * i);
  // barycoord
  const hpi::V v0 = hpi::sub(C, A), v1 = hpi::sub(B, A), v2 = hpi::sub(P, A);
  const sf::f64 d00 = hpi::dot(v0, v0), d01 = hpi::dot(v0, v1), d02 = hpi::dot(v0, v2), d11 = hpi::dot(v1, v1),
                d12 = hpi::dot(v1, v2);
  const sf::f64 denom = sf::sub(sf::mul(d00, d11), sf::mul(d01, d01));
  const bool degenerate = sf::is_zero(denom);
  sf::f64 w[3] = {0, 0, 0};
  if (!degenerate) {
    const sf::f64 inv = sf::div(sf::kOne, denom);
    const sf::f64 u = sf::mul(sf::sub(sf::mul(d11, d02), sf::mul(d01, d12)), inv);
    const sf::f64 v = sf::mul(sf::sub(sf::mul(d00, d12), sf::mul(d01, d02)), inv);
    w[0] = sf::sub(sf::sub(sf::kOne, u), v);
    w[1] = v;
    w[2] = u;
    for (int k = 0; k < 3; ++k) r.barycoord[k] = sf::to_f32(w[k]);
  }
  // uv
  if (uv && !degenerate) {
    const float* ua = uv + (uint64_t)va * uv_stride;
    const float* ub = uv + (uint64_t)vb * uv_stride;
    const float* uc = uv + (uint64_t)vc * uv_stride;
    for (int k = 0; k < 2; ++k) {
      sf::f64 acc = sf::mul(sf::from_f32(__ldg(ua + k)), w[0]);
      acc = sf::add(acc, sf::mul(sf::from_f32(__ldg(ub + k)), w[1]));
      acc = sf::add(acc, sf::mul(sf::from_f32(__ldg(uc + k)), w[2]));
      r.uv[k] = sf::to_f32(acc);
    }
  }
  // normal
  const hpi::V nr = hpi::cross(hpi::sub(C, B), hpi::sub(A, B));
  const sf::f64 l2 = hpi::dot(nr, nr);
  if (sf::lt(0, l2)) {
    const sf::f64 s = sf::div(sf::kOne, sf::sqrt(l2));
    r.normal[0] = sf::to_f32(sf::mul(nr.x, s));
    r.normal[1] = sf::to_f32(sf::mul(nr.y, s));
    r.normal[2] = sf::to_f32(sf::mul(nr.z, s));
  }
  out[i] = r;
}

__global__ void __launch_bounds__(kBlock) hit_interpolate_kernel(const bvhc_hit* __restrict__ hits, uint64_t n,
                                                                 const uint32_t* __restrict__ tri_vid,
                                                                 const float* __restrict__ attr, int item_size,
                                                                 int stride, const float* __restrict__ rays,
                                                                 float* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bvhc_hit h = hits[i];
  float v[4] = {0.f, 0.f, 0.f, 0.f};
  if (h.face_index != BVHC_NO_HIT) {
    for (int k = 0; k < 3; ++k) {
      const float* a = attr + (uint64_t)__ldg(tri_vid + 3 * (uint64_t)h.face_index + k) * stride;
      for (int c = 0; c < item_size; ++c) v[c] += h.barycoord[k] * __ldg(a + c);
    }
    if (rays && item_size == 3) {
      const float* r = rays + 6 * i;
      if (v[0] * r[3] + v[1] * r[4] + v[2] * r[5] > 0.0f) {
        v[0] = -v[0];
        v[1] = -v[1];
        v[2] = -v[2];
      }
    }
  }
  for (int c = 0; c < item_size; ++c) out[i * item_size + c] = v[c];
}

}  // namespace dev

cudaError_t launch_hit_interpolate(const bvhc_hit* hits, uint64_t n, const uint32_t* tri_vid, const float* attr,
                                   int item_size, int stride, const float* rays, float* out, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  dev::hit_interpolate_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(hits, n, tri_vid, attr, item_size, stride,
                                                                       rays, out);
  return cudaGetLastError();
}

// Sorts the n shapes' ids by the Morton key of their centres into `queue`.
static cudaError_t sort_shapes(const float* shapes, uint64_t n, int kind, uint32_t* queue, unsigned int* qcount,
                               const RaySort& sort, cudaStream_t stream) {
  uint32_t *ids, *keys;
  ray_sort_input(2, sort.scratch, queue, &ids, &keys);
  dev::SceneBox box{};
  for (int a = 0; a < 3; ++a) {
    box.lo[a] = sort.lo[a];
    box.hi[a] = sort.hi[a];
  }
  dev::shape_key_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(shapes, n, kind, box, ids, keys, qcount);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_ray_sort(2, n, qcount, sort.scratch, queue, stream);
}

cudaError_t launch_intersects_sphere(const MeshDev& m, const float* spheres, uint64_t n, uint8_t* out,
                                     cudaStream_t stream, uint32_t* queue, unsigned int* qcount, const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  const bool sorted = queue && qcount && sort;
  if (sorted) {
    cudaError_t e = sort_shapes(spheres, n, 0, queue, qcount, *sort, stream);
    if (e != cudaSuccess) return e;
  }
  dev::intersects_sphere_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, spheres, n, out, sorted ? queue : nullptr);
  return cudaGetLastError();
}

cudaError_t launch_scene_raycast_first(const MeshDev& blas, const SceneDev& scene, const float* rays, uint64_t n,
                                       int side, float near_d, float far_d, bvhc_hit* hits, uint32_t* instance,
                                       cudaStream_t stream, const RaySort* sort, uint32_t* queue,
                                       unsigned int* qcount) {
  if (n == 0) return cudaSuccess;
  const bool sorted = sort && sort->kind > 0 && queue && qcount && n < (1ull << 32);
  if (sorted) {
    uint32_t *ids, *keys;
    ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
    dev::SceneBox box;
    for (int a = 0; a < 3; ++a) {
      box.lo[a] = sort->lo[a];
      box.hi[a] = sort->hi[a];
    }
    dev::scene_key_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(rays, n, sort->kind, box, scene, ids, keys,
                                                                     qcount);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if ((e = launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
  }
  dev::scene_raycast_first_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(
      blas, scene, rays, n, sorted ? queue : nullptr, side, near_d, far_d, hits, instance);
  return cudaGetLastError();
}

cudaError_t launch_scene_raycast_all(const MeshDev& blas, const SceneDev& scene, const float* rays, uint64_t n,
                                     int side, float near_d, float far_d, uint32_t cap, uint32_t* counts,
                                     bvhc_hit* hits, uint32_t* instance, cudaStream_t stream) {
  if (n == 0 || cap == 0) return cudaSuccess;
  dev::scene_raycast_all_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(blas, scene, rays, n, side, near_d, far_d,
                                                                        cap, counts, hits, instance);
  return cudaGetLastError();
}

cudaError_t launch_sphere_triangles(const MeshDev& m, const float* spheres, uint64_t n, uint32_t cap,
                                    uint32_t* counts, uint32_t* faces, cudaStream_t stream, uint32_t* queue,
                                    unsigned int* qcount, const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  const bool sorted = queue && qcount && sort;
  if (sorted) {
    cudaError_t e = sort_shapes(spheres, n, 0, queue, qcount, *sort, stream);
    if (e != cudaSuccess) return e;
  }
  dev::sphere_triangles_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, spheres, n, cap, counts, faces,
                                                                       sorted ? queue : nullptr);
  return cudaGetLastError();
}

cudaError_t launch_triangle_hit_point_info(const float* points, const uint32_t* faces, uint64_t n,
                                           const uint32_t* tri_vid, uint64_t n_tri, const float* pos, int pos_stride,
                                           const float* uv, int uv_stride, const GroupTable& groups,
                                           bvhc_hit_point_info* out, unsigned int* err, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  dev::triangle_hit_point_info_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(
      points, faces, n, tri_vid, n_tri, pos, pos_stride, uv, uv_stride, groups, out, err);
  return cudaGetLastError();
}

cudaError_t launch_intersects_box(const MeshDev& m, const float* boxes, uint64_t n, uint8_t* out,
                                  cudaStream_t stream, uint32_t* queue, unsigned int* qcount, const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  const bool sorted = queue && qcount && sort;
  if (sorted) {
    cudaError_t e = sort_shapes(boxes, n, 1, queue, qcount, *sort, stream);
    if (e != cudaSuccess) return e;
  }
  dev::intersects_box_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, boxes, n, out, sorted ? queue : nullptr);
  return cudaGetLastError();
}

}  // namespace bvhc
