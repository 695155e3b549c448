// Float32 leaf arithmetic with error-bounded filters and a float-float fallback.
//
// The reference evaluates three.js's ray/triangle and closest-point math in float64 on float32
// vertices.  The GPU has no FP64 budget here, so every decision that selects a result (the sign
// of the determinant and of the three barycentric numerators and of t, a box score against
// maxThreshold**2, the ordering of two candidate distances) is first taken in float32 together
// with an a-priori error bound.  Only when the float32 value lies inside its bound is the
// quantity recomputed in double-float ("float-float") arithmetic, which carries about 48
// significant bits.  The reported numbers (t, distance, point, barycentrics) are always
// computed in float-float and rounded once to float32.
//
// Float-float building blocks, written from the published algorithms:
//   two_sum  - Knuth, TAOCP vol. 2, 4.2.2 (error-free addition, 6 flops);
//   two_prod - error-free product via one fused multiply-add (Ogita, Rump, Oishi 2005);
//   ff_add / ff_mul / ff_div / ff_sqrt - the double-word algorithms analysed by
//     Joldes, Muller, Popescu, "Tight and rigorous error bounds for basic building blocks of
//     double-word arithmetic", ACM TOMS 44(2), 2017 (AccurateDWPlusDW, DWTimesDW, DWDivDW,
//     and a Newton step for the square root).
// The __f*_rn intrinsics keep nvcc from contracting or reordering these sequences.
#pragma once

#include <cstdint>

namespace bvhc {
namespace dev {

struct ff {
  float hi, lo;
};

__device__ __forceinline__ ff ff_from(float a) { return {a, 0.0f}; }

__device__ __forceinline__ ff two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return {s, e};
}

__device__ __forceinline__ ff fast_two_sum(float a, float b) {  // requires |a| >= |b| or a == 0
  float s = __fadd_rn(a, b);
  float e = __fsub_rn(b, __fsub_rn(s, a));
  return {s, e};
}

__device__ __forceinline__ ff two_diff(float a, float b) { return two_sum(a, -b); }

__device__ __forceinline__ ff two_prod(float a, float b) {
  float p = __fmul_rn(a, b);
  float e = __fmaf_rn(a, b, -p);
  return {p, e};
}

__device__ __forceinline__ ff ff_add(ff a, ff b) {
  ff s = two_sum(a.hi, b.hi);
  ff t = two_sum(a.lo, b.lo);
  float c = __fadd_rn(s.lo, t.hi);
  ff v = fast_two_sum(s.hi, c);
  float w = __fadd_rn(t.lo, v.lo);
  return fast_two_sum(v.hi, w);
}

__device__ __forceinline__ ff ff_neg(ff a) { return {-a.hi, -a.lo}; }
__device__ __forceinline__ ff ff_sub(ff a, ff b) { return ff_add(a, ff_neg(b)); }

__device__ __forceinline__ ff ff_mul(ff a, ff b) {
  ff p = two_prod(a.hi, b.hi);
  float t = __fmul_rn(a.lo, b.lo);
  t = __fmaf_rn(a.hi, b.lo, t);
  t = __fmaf_rn(a.lo, b.hi, t);
  float c = __fadd_rn(p.lo, t);
  return fast_two_sum(p.hi, c);
}

__device__ __forceinline__ ff ff_mul_f(ff a, float b) {
  ff p = two_prod(a.hi, b);
  float c = __fmaf_rn(a.lo, b, p.lo);
  return fast_two_sum(p.hi, c);
}

__device__ __forceinline__ ff ff_div(ff a, ff b) {
  float q1 = __fdiv_rn(a.hi, b.hi);
  ff r = ff_sub(a, ff_mul_f(b, q1));
  float q2 = __fdiv_rn(r.hi, b.hi);
  r = ff_sub(r, ff_mul_f(b, q2));
  float q3 = __fdiv_rn(r.hi, b.hi);
  ff q = fast_two_sum(q1, q2);
  return ff_add(q, ff_from(q3));
}

__device__ __forceinline__ ff ff_sqrt(ff a) {
  if (a.hi <= 0.0f) return {0.0f, 0.0f};
  float s = __fsqrt_rn(a.hi);
  ff r = ff_sub(a, two_prod(s, s));
  float c = __fdiv_rn(r.hi, __fmul_rn(2.0f, s));
  return fast_two_sum(s, c);
}

__device__ __forceinline__ int ff_sign(ff a) { return a.hi > 0.0f ? 1 : (a.hi < 0.0f ? -1 : 0); }
__device__ __forceinline__ bool ff_lt(ff a, ff b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
__device__ __forceinline__ float ff_to_f(ff a) { return __fadd_rn(a.hi, a.lo); }

struct ff3 {
  ff x, y, z;
};

__device__ __forceinline__ ff3 ff3_diff(float3 a, float3 b) { return {two_diff(a.x, b.x), two_diff(a.y, b.y), two_diff(a.z, b.z)}; }
__device__ __forceinline__ ff3 ff3_sub(ff3 a, ff3 b) { return {ff_sub(a.x, b.x), ff_sub(a.y, b.y), ff_sub(a.z, b.z)}; }
__device__ __forceinline__ ff3 ff3_add(ff3 a, ff3 b) { return {ff_add(a.x, b.x), ff_add(a.y, b.y), ff_add(a.z, b.z)}; }
__device__ __forceinline__ ff3 ff3_scale(ff3 a, ff s) { return {ff_mul(a.x, s), ff_mul(a.y, s), ff_mul(a.z, s)}; }
__device__ __forceinline__ ff3 ff3_cross(ff3 a, ff3 b) {
  return {ff_sub(ff_mul(a.y, b.z), ff_mul(a.z, b.y)), ff_sub(ff_mul(a.z, b.x), ff_mul(a.x, b.z)),
          ff_sub(ff_mul(a.x, b.y), ff_mul(a.y, b.x))};
}
__device__ __forceinline__ ff ff3_dot(ff3 a, ff3 b) { return ff_add(ff_add(ff_mul(a.x, b.x), ff_mul(a.y, b.y)), ff_mul(a.z, b.z)); }
__device__ __forceinline__ ff ff3_dot_f(float3 a, ff3 b) {
  return ff_add(ff_add(ff_mul_f(b.x, a.x), ff_mul_f(b.y, a.y)), ff_mul_f(b.z, a.z));
}

// ---------------------------------------------------------------------------------------------
// Ray / triangle (three.js Ray.intersectTriangle, the Eberly sign-of-determinant form).
// With e1 = b - a, e2 = c - a, q = o - a and n = e1 x e2:
//   N = d . n,  U = d . (q x e2),  V = d . (e1 x q),  W = N - U - V,  T = q . n.
// The reference hits iff N != 0, N's sign passes the side test (FrontSide needs N < 0, BackSide
// N > 0), s*U >= 0, s*V >= 0, s*W >= 0 and -s*T >= 0 with s = sign(N); then t = -T / N.
// (BackSide reverses the winding, which flips the sign of N and leaves the point-in-triangle
// and t >= 0 conditions unchanged, so all three sides reduce to this one set of signs.)
// ---------------------------------------------------------------------------------------------

enum { kSideFront = 0, kSideBack = 1, kSideDouble = 2 };

struct TriFF {
  ff N, U, V, W, T;
};

// The float-float determinants of a ray / triangle pair.  One out-of-line body serves every
// float-float triangle evaluation, which keeps kernels that call it from several places fetching
// one copy of the code.
static __device__ __noinline__ TriFF tri_eval_ff(float3 a, float3 b, float3 c, float3 o, float3 d) {
  ff3 e1 = ff3_diff(b, a), e2 = ff3_diff(c, a), q = ff3_diff(o, a);
  ff3 n = ff3_cross(e1, e2);
  TriFF r;
  r.N = ff3_dot_f(d, n);
  r.U = ff3_dot_f(d, ff3_cross(q, e2));
  r.V = ff3_dot_f(d, ff3_cross(e1, q));
  r.W = ff_sub(ff_sub(r.N, r.U), r.V);
  r.T = ff3_dot(q, n);
  return r;
}

// A triangle whose barycentrics the hit record leaves at zero: |n|^2 <= 2^-50 |e1|^2 |e2|^2 in
// float-float (n = e1 x e2).
static __device__ __noinline__ bool tri_degenerate_ff(float3 a, float3 b, float3 c) {
  const ff3 e1 = ff3_diff(b, a), e2 = ff3_diff(c, a);
  const ff3 n = ff3_cross(e1, e2);
  const ff g = ff3_dot(n, n);
  const ff l12 = ff_mul(ff3_dot(e1, e1), ff3_dot(e2, e2));
  return g.hi <= 8.8817841970012523e-16f * l12.hi;  // 2^-50
}

// The same decision, settled in float32 when it is clear.  The float32 normal differs from the
// exact one by at most about 9u |e1| |e2| (u = 2^-24: the edge differences, products and sums), so a
// float32 normal of at least 2^-16 |e1| |e2| (squared: 2^-32, with |e1|^2 |e2|^2 kept inside the
// normal float range) puts the exact |n|^2 above 2^-33 |e1|^2 |e2|^2, far from 2^-50: not
// degenerate.  Anything else takes the float-float test.
__device__ __forceinline__ bool tri_degenerate(float3 a, float3 b, float3 c) {
  const float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
  const float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
  const float nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
  const float gf = nx * nx + ny * ny + nz * nz;
  const float lf = (e1x * e1x + e1y * e1y + e1z * e1z) * (e2x * e2x + e2y * e2y + e2z * e2z);
  if (lf >= 0x1p-60f && lf <= 0x1p100f && gf >= 0x1p-32f * lf) return false;
  return tri_degenerate_ff(a, b, c);
}

__device__ __forceinline__ bool tri_decide_ff(const TriFF& r, int side) {
  int sn = ff_sign(r.N);
  if (sn == 0) return false;
  if (sn > 0 ? side == kSideFront : side == kSideBack) return false;
  return sn * ff_sign(r.U) >= 0 && sn * ff_sign(r.V) >= 0 && sn * ff_sign(r.W) >= 0 && -sn * ff_sign(r.T) >= 0;
}

static __device__ __noinline__ bool tri_hit_slow(float3 a, float3 b, float3 c, float3 o, float3 d, int side) {
  return tri_decide_ff(tri_eval_ff(a, b, c, o, d), side);
}

__device__ __forceinline__ float max3abs(float x, float y, float z) { return fmaxf(fabsf(x), fmaxf(fabsf(y), fabsf(z))); }

// Float32 filter.  For a determinant x . (y x z) evaluated in float32 from inputs that each carry
// one rounding (the vertex differences), the forward error is at most 8u * sum|x_i||y_j||z_k|
// (u = 2^-24), which is at most 16u * |x|_1 * |y|_inf * |z|_inf.  The bound used, 2^-19 * ...,
// doubles that to absorb the second-order terms and the rounding of the bound itself.
// `d_l1` is |d|_1 of the ray direction.  Returns true on a hit.
__device__ __forceinline__ bool tri_hit(float3 a, float3 b, float3 c, float3 o, float3 d, float d_l1, int side) {
  const float kB = 1.9073486328125e-06f;  // 2^-19
  float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
  float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
  float nx = e1y * e2z - e1z * e2y;
  float ny = e1z * e2x - e1x * e2z;
  float nz = e1x * e2y - e1y * e2x;
  float N = d.x * nx + d.y * ny + d.z * nz;
  float m1 = max3abs(e1x, e1y, e1z), m2 = max3abs(e2x, e2y, e2z);
  float bN = kB * d_l1 * m1 * m2;
  if (!(fabsf(N) > bN)) return tri_hit_slow(a, b, c, o, d, side);
  if (N > 0.0f ? side == kSideFront : side == kSideBack) return false;
  float qx = o.x - a.x, qy = o.y - a.y, qz = o.z - a.z;
  float mq = max3abs(qx, qy, qz);
  float s = N > 0.0f ? 1.0f : -1.0f;
  // U = d . (q x e2)
  float ux = qy * e2z - qz * e2y, uy = qz * e2x - qx * e2z, uz = qx * e2y - qy * e2x;
  float U = s * (d.x * ux + d.y * uy + d.z * uz);
  float bU = kB * d_l1 * mq * m2;
  if (U < -bU) return false;
  // V = d . (e1 x q)
  float vx = e1y * qz - e1z * qy, vy = e1z * qx - e1x * qz, vz = e1x * qy - e1y * qx;
  float V = s * (d.x * vx + d.y * vy + d.z * vz);
  float bV = kB * d_l1 * m1 * mq;
  if (V < -bV) return false;
  float W = fabsf(N) - U - V;
  float bW = bN + bU + bV + 2.384185791015625e-07f * (fabsf(N) + fabsf(U) + fabsf(V));  // + 4u(|N|+|U|+|V|)
  if (W < -bW) return false;
  // -s T = -s q . n
  float T = -s * (qx * nx + qy * ny + qz * nz);
  float bT = kB * (fabsf(qx) + fabsf(qy) + fabsf(qz)) * m1 * m2;
  if (T < -bT) return false;
  if (U > bU && V > bV && W > bW && T > bT) return true;
  return tri_hit_slow(a, b, c, o, d, side);
}

// t = -T / N in float-float, for a triangle already known to be hit.
__device__ __forceinline__ ff tri_t_ff(const TriFF& r) { return ff_div(ff_neg(r.T), r.N); }

constexpr float kTinyRel = 9.094947017729282e-13f;  // 2^-40: relative error of a float-float t

static __device__ __noinline__ bool tri_hit_slow_t(float3 a, float3 b, float3 c, float3 o, float3 d, int side, float& t,
                                            float& t_err) {
  TriFF r = tri_eval_ff(a, b, c, o, d);
  if (!tri_decide_ff(r, side)) return false;
  ff tt = tri_t_ff(r);
  t = tt.hi;
  t_err = fabsf(tt.hi) * kTinyRel + 1e-30f;
  return true;
}

// tri_hit, and on a hit the ray parameter t = -T / N with an absolute error bound `t_err`: from
// the float32 values (relative error <= bT/|T| + bN/|N| + 4u) when the filter settled every sign,
// otherwise from the float-float evaluation.
__device__ __forceinline__ bool tri_hit_t(float3 a, float3 b, float3 c, float3 o, float3 d, float d_l1, int side,
                                          float& t, float& t_err) {
  const float kB = 1.9073486328125e-06f;  // 2^-19
  float e1x = b.x - a.x, e1y = b.y - a.y, e1z = b.z - a.z;
  float e2x = c.x - a.x, e2y = c.y - a.y, e2z = c.z - a.z;
  float nx = e1y * e2z - e1z * e2y;
  float ny = e1z * e2x - e1x * e2z;
  float nz = e1x * e2y - e1y * e2x;
  float N = d.x * nx + d.y * ny + d.z * nz;
  float m1 = max3abs(e1x, e1y, e1z), m2 = max3abs(e2x, e2y, e2z);
  float bN = kB * d_l1 * m1 * m2;
  if (!(fabsf(N) > bN)) return tri_hit_slow_t(a, b, c, o, d, side, t, t_err);
  if (N > 0.0f ? side == kSideFront : side == kSideBack) return false;
  float qx = o.x - a.x, qy = o.y - a.y, qz = o.z - a.z;
  float mq = max3abs(qx, qy, qz);
  float s = N > 0.0f ? 1.0f : -1.0f;
  float ux = qy * e2z - qz * e2y, uy = qz * e2x - qx * e2z, uz = qx * e2y - qy * e2x;
  float U = s * (d.x * ux + d.y * uy + d.z * uz);
  float bU = kB * d_l1 * mq * m2;
  if (U < -bU) return false;
  float vx = e1y * qz - e1z * qy, vy = e1z * qx - e1x * qz, vz = e1x * qy - e1y * qx;
  float V = s * (d.x * vx + d.y * vy + d.z * vz);
  float bV = kB * d_l1 * m1 * mq;
  if (V < -bV) return false;
  float aN = fabsf(N);
  float W = aN - U - V;
  float bW = bN + bU + bV + 2.384185791015625e-07f * (aN + fabsf(U) + fabsf(V));
  if (W < -bW) return false;
  float T = -s * (qx * nx + qy * ny + qz * nz);
  float bT = kB * (fabsf(qx) + fabsf(qy) + fabsf(qz)) * m1 * m2;
  if (T < -bT) return false;
  if (U > bU && V > bV && W > bW && T > bT) {
    t = T / aN;
    t_err = t * (bT / T + bN / aN + 2.384185791015625e-07f);
    return true;
  }
  return tri_hit_slow_t(a, b, c, o, d, side, t, t_err);
}

// ---------------------------------------------------------------------------------------------
// Closest point on a triangle (Ericson, Real-Time Collision Detection, 5.1.5), evaluated in the
// local frame of vertex a so that rounding scales with the triangle and the query distance
// rather than with the absolute coordinates.
// ---------------------------------------------------------------------------------------------

// Float32 version: returns |p - q|^2 and the closest point q (world frame).
__device__ __forceinline__ float closest_sq_f(float3 p, float3 a, float3 b, float3 c, float3& q, float& scale) {
  float abx = b.x - a.x, aby = b.y - a.y, abz = b.z - a.z;
  float acx = c.x - a.x, acy = c.y - a.y, acz = c.z - a.z;
  float apx = p.x - a.x, apy = p.y - a.y, apz = p.z - a.z;
  scale = max3abs(abx, aby, abz) + max3abs(acx, acy, acz) + max3abs(apx, apy, apz);
  float lx, ly, lz;  // closest point relative to a
  float d1 = abx * apx + aby * apy + abz * apz;
  float d2 = acx * apx + acy * apy + acz * apz;
  float bpx = apx - abx, bpy = apy - aby, bpz = apz - abz;
  float d3 = abx * bpx + aby * bpy + abz * bpz;
  float d4 = acx * bpx + acy * bpy + acz * bpz;
  float cpx = apx - acx, cpy = apy - acy, cpz = apz - acz;
  float d5 = abx * cpx + aby * cpy + abz * cpz;
  float d6 = acx * cpx + acy * cpy + acz * cpz;
  float vc = d1 * d4 - d3 * d2;
  float vb = d5 * d2 - d1 * d6;
  float va = d3 * d6 - d5 * d4;
  if (d1 <= 0.0f && d2 <= 0.0f) {
    lx = 0.0f; ly = 0.0f; lz = 0.0f;
    q = a;
  } else if (d3 >= 0.0f && d4 <= d3) {
    lx = abx; ly = aby; lz = abz;
    q = b;
  } else if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    float v = d1 / (d1 - d3);
    lx = abx * v; ly = aby * v; lz = abz * v;
    q = make_float3(a.x + lx, a.y + ly, a.z + lz);
  } else if (d6 >= 0.0f && d5 <= d6) {
    lx = acx; ly = acy; lz = acz;
    q = c;
  } else if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    float w = d2 / (d2 - d6);
    lx = acx * w; ly = acy * w; lz = acz * w;
    q = make_float3(a.x + lx, a.y + ly, a.z + lz);
  } else if (va <= 0.0f && (d4 - d3) >= 0.0f && (d5 - d6) >= 0.0f) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    lx = abx + (acx - abx) * w; ly = aby + (acy - aby) * w; lz = abz + (acz - abz) * w;
    q = make_float3(a.x + lx, a.y + ly, a.z + lz);
  } else {
    float den = 1.0f / (va + vb + vc);
    float v = vb * den, w = vc * den;
    lx = abx * v + acx * w; ly = aby * v + acy * w; lz = abz * v + acz * w;
    q = make_float3(a.x + lx, a.y + ly, a.z + lz);
  }
  float rx = apx - lx, ry = apy - ly, rz = apz - lz;
  return rx * rx + ry * ry + rz * rz;
}

struct CPFF {
  ff3 q;    // closest point (world frame)
  ff d2;    // squared distance
  ff3 r;    // p - q
  float wb, wc;  // barycentric weights of q on b and c (exactly 0 off the region's own vertices)
};

// Float-float version of the same algorithm (used for the final answer and for ties).
static __device__ __noinline__ CPFF closest_ff(float3 p, float3 a, float3 b, float3 c) {
  ff3 ab = ff3_diff(b, a), ac = ff3_diff(c, a), ap = ff3_diff(p, a);
  ff3 l;
  float wb = 0.0f, wc = 0.0f;
  ff d1 = ff3_dot(ab, ap), d2 = ff3_dot(ac, ap);
  ff3 bp = ff3_sub(ap, ab), cp = ff3_sub(ap, ac);
  ff d3 = ff3_dot(ab, bp), d4 = ff3_dot(ac, bp);
  ff d5 = ff3_dot(ab, cp), d6 = ff3_dot(ac, cp);
  ff zero = ff_from(0.0f);
  if (ff_sign(d1) <= 0 && ff_sign(d2) <= 0) {
    l = {zero, zero, zero};
  } else if (ff_sign(d3) >= 0 && !ff_lt(d3, d4)) {
    l = ab;
    wb = 1.0f;
  } else {
    ff vc = ff_sub(ff_mul(d1, d4), ff_mul(d3, d2));
    if (ff_sign(vc) <= 0 && ff_sign(d1) >= 0 && ff_sign(d3) <= 0) {
      ff v = ff_div(d1, ff_sub(d1, d3));
      l = ff3_scale(ab, v);
      wb = v.hi;
    } else if (ff_sign(d6) >= 0 && !ff_lt(d6, d5)) {
      l = ac;
      wc = 1.0f;
    } else {
      ff vb = ff_sub(ff_mul(d5, d2), ff_mul(d1, d6));
      if (ff_sign(vb) <= 0 && ff_sign(d2) >= 0 && ff_sign(d6) <= 0) {
        ff w = ff_div(d2, ff_sub(d2, d6));
        l = ff3_scale(ac, w);
        wc = w.hi;
      } else {
        ff va = ff_sub(ff_mul(d3, d6), ff_mul(d5, d4));
        ff d43 = ff_sub(d4, d3), d56 = ff_sub(d5, d6);
        if (ff_sign(va) <= 0 && ff_sign(d43) >= 0 && ff_sign(d56) >= 0) {
          ff w = ff_div(d43, ff_add(d43, d56));
          l = ff3_add(ab, ff3_scale(ff3_sub(ac, ab), w));
          wb = 1.0f - w.hi;
          wc = w.hi;
        } else {
          ff den = ff_add(ff_add(va, vb), vc);
          ff v = ff_div(vb, den), w = ff_div(vc, den);
          l = ff3_add(ff3_scale(ab, v), ff3_scale(ac, w));
          wb = v.hi;
          wc = w.hi;
        }
      }
    }
  }
  ff3 r = ff3_sub(ap, l);
  CPFF out;
  out.d2 = ff3_dot(r, r);
  out.r = r;
  out.q = {ff_add(ff_from(a.x), l.x), ff_add(ff_from(a.y), l.y), ff_add(ff_from(a.z), l.z)};
  out.wb = wb;
  out.wc = wc;
  return out;
}

}  // namespace dev
}  // namespace bvhc
