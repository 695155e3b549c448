// closestPointToPoint, the shapecast queries (intersectsSphere, triangles within spheres,
// intersectsBox), getTriangleHitPointInfo and Intersection attribute interpolation; and their
// launches.
#include <algorithm>

#include "traverse.cuh"

namespace bvhc {
namespace dev {

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

// Squared distance from p to the box's centre: the visiting order's tie-break when both child
// boxes hold p (both scores 0), which the scores alone cannot order.
__device__ __forceinline__ float centre_d2(const float* b, float3 p) {
  const float dx = 0.5f * (b[0] + b[3]) - p.x, dy = 0.5f * (b[1] + b[4]) - p.y, dz = 0.5f * (b[2] + b[5]) - p.z;
  return dx * dx + dy * dy + dz * dz;
}

// Whether the right child should be visited first: the smaller score, equal scores by the nearer
// centre (the warp-cooperative forms; the per-query kernel keeps the reference's order).  The
// centre distances are computed only on equal scores (written as a branch: as one expression they
// were evaluated on every node, 4% of the grid's time).
__device__ __forceinline__ bool right_nearer(const Pair& pr, float s0, float s1, float3 p) {
  if (s1 != s0) return s1 < s0;
  return centre_d2(pr.r, p) < centre_d2(pr.l, p);
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
  uint32_t face;     // its faceIndex
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
  b.face = 0xFFFFFFFFu;
  b.q = make_float3(0.f, 0.f, 0.f);
  b.vertex = false;
  b.ff_ok = false;
  b.ffv = {kInf, 0.0f};
  return b;
}

// Offers triangle record k to the query at p: a strictly smaller squared distance replaces the
// best (the reference's strict `<` on distSq), and an exact tie goes to the smaller faceIndex
// (the reference keeps whichever its own traversal reached first; a fixed rule on the triangle
// itself keeps the answer independent of how queries are grouped and of how the triangles of a
// leaf are laid out).  Every record holds a distinct faceIndex.  Returns the candidate's float32
// squared distance and bound, and its float-float value when one was needed.
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
    take = t.face < b.face;  // the same vertex: an exact tie, the smaller faceIndex wins
  } else {
    // Undecided in float32: the float-float squared distances decide, and an exact tie goes to
    // the smaller faceIndex.  Candidates are thus ranked by a total order that does
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
    take = ff_lt(cand_ff, b.ffv) || (!ff_lt(b.ffv, cand_ff) && t.face < b.face);
  }
  if (take) {
    b.d2 = d2;
    b.err = err;
    b.rec = k;
    b.face = t.face;
    b.q = q;
    b.vertex = is_vertex;
    b.ff_ok = have_ff;
    b.ffv = cand_ff;
  }
}

// The reported record of triangle record `rec` (0xFFFFFFFF: none): distance and closest point in
// float-float, rounded once.
__device__ __forceinline__ void cp_store(const MeshDev& m, float3 p, uint32_t rec, bvhc_closest* o) {
  if (rec == 0xFFFFFFFFu) {
    o->face_index = BVHC_NO_HIT;
    o->distance = kInf;
    o->point[0] = o->point[1] = o->point[2] = 0.0f;
    return;
  }
  Tri t = load_tri(m.tris, rec);
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
  out[i].face_index = b.rec;  // pending, as in the warp-cooperative kernel
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
//
// GROUP = 32 walks the tree with the whole warp; 16 and 8 split the warp into groups of that many
// lanes (consecutive queries), each with its own shared stack: a group's node set is the union over
// fewer, closer queries, and groups at different nodes on the same code path still issue together.
template <int MINB, int GROUP>
__global__ void __launch_bounds__(kBlock, MINB) closest_point_packet_kernel(
    MeshDev m, const float* __restrict__ pts, uint64_t n, float max_t, bvhc_closest* __restrict__ out,
    const uint32_t* __restrict__ queue, const unsigned int* __restrict__ qcount, uint64_t pitch, int rows_log2) {
  static_assert(GROUP == 32 || GROUP == 16 || GROUP == 8, "group of 8, 16 or 32 lanes");
  __shared__ uint32_t s_link[kBlock / GROUP][kMaxStack];
  const int w = threadIdx.x / GROUP;                      // group within the block
  const unsigned lane = threadIdx.x & (GROUP - 1u);       // lane within the group
  const unsigned full = GROUP == 32 ? 0xFFFFFFFFu : ((1u << GROUP) - 1u) << ((threadIdx.x & 31u) & ~(GROUP - 1u));
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  else if (valid && pitch) i = tiled_index(i, pitch, rows_log2, n);  // tiles of grid points
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
        unsigned b0 = __ballot_sync(full, w0) & full, b1 = __ballot_sync(full, w1) & full;
        if (b0 && b1) {
          // nearer child first by majority of the lanes that want both (a lane wanting one prefers it)
          bool pref_right = (w0 && w1) ? right_nearer(pr, s0, s1, p) : w1;
          unsigned voters = __ballot_sync(full, w0 || w1) & full;
          bool right_first = 2 * __popc(__ballot_sync(full, (w0 || w1) && pref_right) & full) > __popc(voters);
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
          __syncwarp(full);
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
          if (__ballot_sync(full, ok) & full) {
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
  // pending: the record index in face_index; closest_point_finalize_kernel completes the record,
  // which keeps the float-float code out of this kernel
  if (valid) out[i].face_index = b.rec;
}

// Completes the records closest_point_kernel / closest_point_packet_kernel left pending, one query
// per thread in input order.
__global__ void __launch_bounds__(kBlock) closest_point_finalize_kernel(MeshDev m, const float* __restrict__ pts,
                                                                        uint64_t n, bvhc_closest* __restrict__ out) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float3 p = make_float3(__ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2));
  cp_store(m, p, out[i].face_index, out + i);
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

// Float bits mapped to unsigned integers that order as the floats do (negatives reversed below the
// positives), so that atomicMin / atomicMax on them give the float minimum / maximum.
__device__ __forceinline__ unsigned ordered_bits(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float from_ordered_bits(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

constexpr int kBoxThreads = 256;

// Bounding box of the query points (finite coordinates only) into qbox[0..2] (minimum) and
// qbox[3..5] (maximum) as ordered bits; qbox starts as 0xFFFFFFFF (minimum) and 0 (maximum).
__global__ void __launch_bounds__(kBoxThreads) points_box_kernel(const float* __restrict__ pts, uint64_t n,
                                                                 unsigned* __restrict__ qbox) {
  unsigned lo[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, hi[3] = {0u, 0u, 0u};
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    for (int a = 0; a < 3; ++a) {
      const float v = __ldg(pts + 3 * i + a);
      if (!isfinite(v)) continue;
      const unsigned u = ordered_bits(v);
      lo[a] = min(lo[a], u);
      hi[a] = max(hi[a], u);
    }
  }
  for (int a = 0; a < 3; ++a) {
    const unsigned l = __reduce_min_sync(0xFFFFFFFFu, lo[a]), h = __reduce_max_sync(0xFFFFFFFFu, hi[a]);
    if ((threadIdx.x & 31u) == 0) {
      atomicMin(qbox + a, l);
      atomicMax(qbox + 3 + a, h);
    }
  }
}

// Morton key of each query point over the query points' own box (8 bits per axis), ids in input
// order, and the queue length; the queue is then sorted by key so that a warp takes 32 nearby
// points.  (Over the mesh's box instead, the queries outside it -- a quarter of a grid padded by
// 10% -- would share clamped keys along every face and keep their input order.)
__global__ void __launch_bounds__(kBlock) point_key_kernel(const float* __restrict__ pts, uint64_t n,
                                                          const unsigned* __restrict__ qbox,
                                                          uint32_t* __restrict__ ids, uint32_t* __restrict__ keys,
                                                          unsigned int* __restrict__ qcount) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *qcount = (unsigned int)n;
  if (i >= n) return;
  SceneBox box;
  for (int a = 0; a < 3; ++a) {
    const unsigned l = __ldg(qbox + a), h = __ldg(qbox + 3 + a);
    box.lo[a] = l <= h ? from_ordered_bits(l) : 0.0f;
    box.hi[a] = l <= h ? from_ordered_bits(h) : 0.0f;
  }
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

}  // namespace dev

cudaError_t launch_closest_point(const MeshDev& m, const float* pts, uint64_t n, float min_t, float max_t,
                                 bvhc_closest* out, cudaStream_t stream, int variant, int occupancy, uint32_t* queue,
                                 unsigned int* qcount, const RaySort* sort, uint32_t tile, int tile_rows) {
  if (n == 0) return cudaSuccess;
  // the warp-cooperative forms need minThreshold 0 (see closest_point_packet_kernel): 1 / 2 with
  // whole warps, 3 / 4 with 16-lane groups, 5 / 6 with 8-lane groups; the even ones run over
  // Morton-sorted queries
  const bool sorted = variant > 0 && variant % 2 == 0;
  cudaError_t e;
  if (variant == 0 || !(min_t <= 0.0f) || (sorted && (!queue || !qcount || !sort || n >= (1ull << 32)))) {
    dev::closest_point_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, pts, n, min_t, max_t, out);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    dev::closest_point_finalize_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, pts, n, out);
    return cudaGetLastError();
  }
  if (sorted) {
    uint32_t *ids, *keys;
    ray_sort_input(2, sort->scratch, queue, &ids, &keys);
    // the query points' box, in the last row of the sort's digit totals (a three-pass sort leaves
    // it unused), then the keys over it
    unsigned* qbox = sort->scratch.totals + 3 * 256;
    if ((e = cudaMemsetAsync(qbox, 0xFF, 3 * sizeof(unsigned), stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(qbox + 3, 0, 3 * sizeof(unsigned), stream)) != cudaSuccess) return e;
    const unsigned int gb = (unsigned int)std::min<uint64_t>((n + dev::kBoxThreads - 1) / dev::kBoxThreads, 2048);
    dev::points_box_kernel<<<gb, dev::kBoxThreads, 0, stream>>>(pts, n, qbox);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    dev::point_key_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(pts, n, qbox, ids, keys, qcount);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = launch_ray_sort(2, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
  } else {
    queue = nullptr;
    qcount = nullptr;
  }
  using K = void (*)(MeshDev, const float*, uint64_t, float, bvhc_closest*, const uint32_t*, const unsigned int*,
                     uint64_t, int);
  static const K kernels[3][3] = {
      {dev::closest_point_packet_kernel<1, 32>, dev::closest_point_packet_kernel<6, 32>,
       dev::closest_point_packet_kernel<8, 32>},
      {dev::closest_point_packet_kernel<1, 16>, dev::closest_point_packet_kernel<6, 16>,
       dev::closest_point_packet_kernel<8, 16>},
      {dev::closest_point_packet_kernel<1, 8>, dev::closest_point_packet_kernel<6, 8>,
       dev::closest_point_packet_kernel<8, 8>}};
  const K kernel = kernels[std::min((variant - 1) / 2, 2)][occupancy < 0 ? 0 : occupancy > 2 ? 2 : occupancy];
  // input order (odd variants) may be read in tiles: rows of `tile` points (a grid's row), 2-D blocks
  const int rl = tile_rows_log2(tile_rows);
  const uint64_t pitch = (!queue && tile >= 8 && tile % (32u >> rl) == 0) ? (uint64_t)tile : 0;
  kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, pts, n, max_t, out, queue, qcount, pitch, rl);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  dev::closest_point_finalize_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, pts, n, out);
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
