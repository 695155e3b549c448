// Device helpers shared by the traversal kernels (kernels_*.cu): rays, child-pair and triangle
// records, the conservative slab test, the raycastFirst leaf step and reported record, and the
// child order.  Each kernel is defined in exactly one translation unit; these helpers are inline
// device code and compile into each unit that uses them.
//
// One ray or query per thread (or per warp lane of a shared traversal).  Each visit of an internal
// node reads one 64-byte child-pair record (both child boxes and links) with four 16-byte
// read-only loads; each leaf is a contiguous run of 48-byte triangle records.  Traversal stacks are
// bounded (the mesh upload rejects deeper trees), and an overflow sets the device error word
// instead of faulting.
#pragma once

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
constexpr int kWarps = kBlock / 32;
constexpr float kInf = __builtin_huge_valf();
constexpr float kSlabMargin = 9.5367431640625e-07f;  // 2^-20, relative slack on slab distances
constexpr float kTiny = 1e-30f;                      // stand-in for a zero direction component

__device__ __forceinline__ float4 ld4(const void* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
// 32 bytes in one load instruction (the 256-bit global load of sm_100) through the read-only path;
// p must be 32-byte aligned.
__device__ __forceinline__ void ld8(const void* p, float4& a, float4& b) {
  asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

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
  uint32_t ll, lr, axis, flags;
};

__device__ __forceinline__ Pair load_pair(const PairNode* __restrict__ nodes, uint32_t k) {
  const PairNode* n = nodes + k;
  // two 256-bit loads per record (every pair array is its own allocation of 64-byte records)
  float4 q0, q1, q2, q3;
  ld8(&n->f[0], q0, q1);
  ld8(&n->f[8], q2, q3);
  Pair p;
  p.l[0] = q0.x; p.l[1] = q0.y; p.l[2] = q0.z; p.l[3] = q0.w; p.l[4] = q1.x; p.l[5] = q1.y;
  p.r[0] = q1.z; p.r[1] = q1.w; p.r[2] = q2.x; p.r[3] = q2.y; p.r[4] = q2.z; p.r[5] = q2.w;
  p.ll = __float_as_uint(q3.x);
  p.lr = __float_as_uint(q3.y);
  p.axis = __float_as_uint(q3.z);
  p.flags = __float_as_uint(q3.w);
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
// e = tri_eval_ff of the triangle and ray, tt = its t, dist = the hit's distance.
static __device__ void make_hit(const Tri& t, const RayF& r, const TriFF& e, ff tt, ff dist, bvhc_hit& h) {
  ff3 px = {ff_add(ff_from(r.o.x), ff_mul_f(tt, r.d.x)), ff_add(ff_from(r.o.y), ff_mul_f(tt, r.d.y)),
            ff_add(ff_from(r.o.z), ff_mul_f(tt, r.d.z))};
  h.face_index = t.face;
  h.distance = ff_to_f(dist);
  h.point[0] = ff_to_f(px.x);
  h.point[1] = ff_to_f(px.y);
  h.point[2] = ff_to_f(px.z);
  if (tri_degenerate(t.a, t.b, t.c)) {
    h.barycoord[0] = h.barycoord[1] = h.barycoord[2] = 0.0f;
  } else {
    // W / N, U / N, V / N through one float-float reciprocal (relative error ~2^-44, rounded once
    // to float32)
    const ff rn = ff_div(ff{1.0f, 0.0f}, e.N);
    h.barycoord[0] = ff_to_f(ff_mul(e.W, rn));
    h.barycoord[1] = ff_to_f(ff_mul(e.U, rn));
    h.barycoord[2] = ff_to_f(ff_mul(e.V, rn));
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

// A pending record: the triangle record index in face_index, `t` in distance.  All 32 bytes are
// written, so that the record's DRAM sector is written whole (a half-sector store makes L2 fetch
// the other half first).
__device__ __forceinline__ void store_pending_record(bvhc_hit* o, uint32_t rec, float t) {
  float4* p = reinterpret_cast<float4*>(o);
  __stcs(p, make_float4(__uint_as_float(rec), t, 0.0f, 0.0f));
  __stcs(p + 1, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
}

// A traversal's result left for finalize_first_kernel: a miss record, or pending.
__device__ __forceinline__ void store_first_pending(bvhc_hit* o, const Best& b) {
  if (b.rec == 0xFFFFFFFFu) store_miss(o);
  else store_pending_record(o, b.rec, b.t);
}

// The reported record of the best hit: t, distance, point and barycentrics in float-float.
__device__ __forceinline__ void finish_first(const MeshDev& m, uint32_t rec, const RayF& r, bvhc_hit* o) {
  if (rec == 0xFFFFFFFFu) {
    store_miss(o);
    return;
  }
  Tri t = load_tri(m.tris, rec);
  const TriFF e = tri_eval_ff(t.a, t.b, t.c, r.o, r.d);
  const ff tt = tri_t_ff(e);
  bvhc_hit h;
  make_hit(t, r, e, tt, ff_mul(tt, dir_length(r.d)), h);
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


// Tiled ray order: the ray index space read as rows of `pitch` rays, cut into bands of R = 2^rl
// rows; work item i of a band is the ray at row (i mod 32) / C, column C (i / 32) + i mod C of that
// band with C = 32 / R (pitch a multiple of C), so each warp takes an R x C tile.  For rays
// generated per pixel in row-major order with pitch = the image width, that is an R x C pixel
// block.  Items past the last whole band keep their own index.  A bijection of [0, n): for i below
// the last whole band the row is below R and the column below pitch, so the ray stays in i's band.
__device__ __forceinline__ uint64_t tiled_index(uint64_t i, uint64_t pitch, int rl, uint64_t n) {
  const int cl = 5 - rl;
  const uint64_t band = pitch << rl;
  if (i >= n - n % band) return i;
  const uint64_t b = i / band, r = i - b * band;
  return b * band + ((r & 31u) >> cl) * pitch + ((r >> 5) << cl) + (r & ((1u << cl) - 1u));
}

// Pre-pass tiles (classify_kernel, kernels_first.cu).
constexpr int kClsThreads = 256;
constexpr int kClsItems = 8;
constexpr int kClsTile = kClsThreads * kClsItems;  // rays per block
constexpr int kClsWarps = kClsThreads / 32;

}  // namespace dev

static inline unsigned int grid_for(uint64_t n) { return (unsigned int)((n + dev::kBlock - 1) / dev::kBlock); }

// Traversal stack entries a launch may use: 32 when asked for and the tree is shallow enough that
// no traversal pushes more than 31 entries (one per internal level of a root-to-leaf path), else 64.
static inline int stack_entries(const MeshDev& m, int requested) {
  return requested == 32 && m.depth <= 30 ? 32 : 64;
}

// Root-box pre-pass into `queue`, then (single mesh, sort requested) the ray-ordering sort
// (kernels_first.cu).
cudaError_t prepare_queue(const MeshDev& m, const BatchDev* batch, const float* rays, uint64_t n, float near_d,
                          float far_d, bvhc_hit* out, uint32_t* queue, unsigned int* qcount, const RaySort* sort,
                          cudaStream_t stream);

// The root-box pre-pass over a single mesh's rays for the all-hits raycast (kernels_first.cu): rays
// that miss get a hit count of 0 in `miss_counts`, the others are queued in `ids`.
cudaError_t launch_classify_counts(const MeshDev& m, const float* rays, uint64_t n, float near_d, float far_d,
                                   uint32_t* ids, unsigned int* qcount, uint32_t* keys, int kind,
                                   const dev::SceneBox& box, uint32_t* miss_counts, cudaStream_t stream);

}  // namespace bvhc
