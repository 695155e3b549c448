// Instanced (BatchedMesh with world matrices) raycastFirst and raycast (all hits), and the world
// rays' ordering keys; and their launches.
#include <algorithm>

#include "traverse.cuh"

namespace bvhc {
namespace dev {

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

// Traversal stack of the geometry-tree walk, in thread-local memory.  (A form that kept the top 8
// entries in shared memory measured 22.5 ms against 20.3 ms on the instanced bench: the shared
// memory it takes is L1 capacity the node reads need.)
template <int STACK>
struct LocalStack {
  uint32_t link[STACK];
  float t[STACK];
  int sp;
  __device__ __forceinline__ void reset() { sp = 0; }
  __device__ __forceinline__ bool push(uint32_t l, float e) {
    if (sp >= STACK) return false;
    link[sp] = l;
    t[sp] = e;
    ++sp;
    return true;
  }
  __device__ __forceinline__ bool pop(uint32_t& l, float& e) {
    if (sp == 0) return false;
    --sp;
    l = link[sp];
    e = t[sp];
    return true;
  }
};

// The per-thread raycastFirst walk of one geometry's roots, nearest child first, in "while-while"
// form (each lane descends internal nodes until it holds a leaf, then the lanes holding one test
// their triangles together).  Returns false on a stack overflow.
template <class Stack>
__device__ bool blas_first(const MeshDev& m, uint32_t r0, uint32_t r1, const RayF& r, float dlen, int side,
                           const SideTable& sides, float near_d, float far_d, Best& best, Stack& st) {
  for (uint32_t root = r0; root < r1; ++root) {
    uint32_t link = m.roots[root];
    st.reset();
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
          if (h2nd && !st.push(c2, lf ? e1 : e0)) return false;
          link = c1;
          continue;
        }
        if (h2nd) {
          link = c2;
          continue;
        }
        go = false;
        const float plim = (best.t + best.err) * (1.0f + kSlabMargin);
        uint32_t l;
        float e;
        while (st.pop(l, e)) {
          if (e <= plim) {
            link = l;
            go = true;
            break;
          }
        }
      }
      if (!go) break;
      if (link != kEmptyLeaf) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
      go = false;
      const float plim = (best.t + best.err) * (1.0f + kSlabMargin);
      uint32_t l;
      float e;
      while (st.pop(l, e)) {
        if (e <= plim) {
          link = l;
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
  const TriFF e = tri_eval_ff(t.a, t.b, t.c, lr.o, lr.d);
  const ff tt = tri_t_ff(e);
  make_hit(t, lr, e, tt, ff_mul(tt, dir_length(lr.d)), h);
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
// ceil(log2) of the instance count: TSTACK = 16 serves up to 2^16 instances, 32 any count the ABI
// takes.  BSTACK (the geometry trees' walk) is 32 when every geometry tree is at most 30 deep, else
// 64.  Smaller stacks keep the per-thread frame (and its spill traffic at high occupancy) smaller.
constexpr int kTlasStack = 32;

// MINB resident blocks per SM (14: 32 registers, some spilled): the kernel stalls on fetching its
// own large body and on its scattered loads, and more resident warps hide both, while fewer
// registers spill more to local memory; the instanced bench tunes 14 / 10 / 8 (it measured 35.6 /
// 28.4 / 22.7 / 20.4 / 20.4 ms at 5 / 8 / 12 / 14 / 16 blocks with 64-entry stacks).
template <int TSTACK, int BSTACK, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) scene_raycast_first_kernel(MeshDev m, SceneDev sc,
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
  // the best world record so far lives in the ray's output row (rewritten when a closer instance
  // hit is found, a few times per ray at most), not in the thread's frame
  ff best_dist = ff_from(kInf);
  uint32_t best_inst = 0xFFFFFFFFu;
  uint32_t stack_link[TSTACK];
  float stack_t[TSTACK];
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
          if (sp >= TSTACK) {
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
        LocalStack<BSTACK> st;
        if (!blas_first(m, sc.mesh_root_off[g], sc.mesh_root_off[g + 1], L.r, L.len, side, no_sides, L.near_d,
                        fminf(L.far_d, tlim), b, st)) {
          atomicOr(m.err, kErrStackOverflow);
          break;
        }
        if (b.rec != 0xFFFFFFFFu) {
          bvhc_hit h;
          const ff dist = world_record(m, I, b.rec, w, L.r, h);
          if (ff_lt(dist, best_dist) || (!ff_lt(best_dist, dist) && j < best_inst)) {
            best_dist = dist;
            best_inst = j;
            store_hit(out + i, h);
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
  if (best_inst == 0xFFFFFFFFu) store_miss(out + i);
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

}  // namespace dev

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
  // the small stacks when both trees allow them, else the large ones; resident blocks per SM by
  // the scene's variant (0: 14, 1: 10, 2: 8)
  const bool small = scene.n_instances <= (1 << 16) && stack_entries(blas, 32) == 32;
  const int occ = scene.occupancy;
  auto kernel = small ? (occ == 1   ? dev::scene_raycast_first_kernel<16, 32, 10>
                         : occ == 2 ? dev::scene_raycast_first_kernel<16, 32, 8>
                                    : dev::scene_raycast_first_kernel<16, 32, 14>)
                      : (occ == 1   ? dev::scene_raycast_first_kernel<32, 64, 10>
                         : occ == 2 ? dev::scene_raycast_first_kernel<32, 64, 8>
                                    : dev::scene_raycast_first_kernel<32, 64, 14>);
  kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(blas, scene, rays, n, sorted ? queue : nullptr, side, near_d, far_d,
                                                  hits, instance);
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

}  // namespace bvhc
