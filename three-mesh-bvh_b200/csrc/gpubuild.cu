// Device SAH / CENTER build whose serialized output is byte-identical to the reference's.
//
// This is `new MeshBVH(geometry, {strategy, maxDepth, maxLeafSize, indirect, range})` followed by
// `MeshBVH.serialize()` (src/core/GeometryBVH.js:93-163, src/core/build/buildTree.js:10-152,
// splitUtils.js:21-294, sortUtils.js:4-62, buildUtils.js:35-92, computeBoundsUtils.js:4-68,
// MeshBVH.js:337-436), run on the GPU.  The reference's node buffers and its in-place reorder of
// the index (or indirect) buffer come out bit for bit, because every quantity that decides the
// tree is computed with the reference's own rounding:
//
//   * primitive boxes: the reference's double expressions evaluated in software binary64
//     (softf64.cuh) and rounded to float32 as its Float32Array stores do; fl32(center -/+ half)
//     equals the correctly rounded float32 difference / sum, which the device computes directly;
//   * node and bin boxes are min / max of those float32 values (exact, order-free), except that
//     a stored node bound keeps the FIRST primitive (in buffer order) holding the extreme value,
//     as the reference's `<` scans do, so -0 / +0 come out as they do there;
//   * bin indices `~~((c - left) / width)`: a float32 estimate accepted only when it is further
//     than 2^-16 from an integer (its error is below 2^-17.5), else the binary64 quotient;
//   * split costs (`TRAVERSAL_COST + PRIMITIVE_INTERSECT_COST * (pl * nl + pr * nr)`): a float32
//     estimate with relative error below 2^-20 ranks the candidates; when the best two, or the
//     best and the no-split cost, are within 2^-16 of each other, the contenders are re-evaluated
//     in binary64 and the reference's strict `<` scan order (axis, then bin) decides;
//   * split positions (`left + width + i * width`) and the partition test `center < pos` in
//     binary64;
//   * the partition is the reference's Hoare partition: its k-th swap exchanges the k-th
//     primitive of the left part that belongs right with the k-th primitive (counted from the
//     end) of the right part that belongs left, so ranks from prefix counts reproduce it.
//
// The reference's recursion is depth-first, but a node's outcome depends only on its own range,
// so the device processes nodes in any order and lays them out in pre-order at the end:
//   1. nodes with more than kSmall primitives, level by level, with grid-wide kernels over
//      2048-primitive chunks (shared-memory bins flushed with atomics, chunk-scanned swap ranks);
//   2. each remaining subtree by one warp, depth first, its records written in local pre-order;
//   3. one pass that places every large node and copies every subtree to its pre-order slot.
// The device executes no FP64 instruction.  AVERAGE (a sequential double sum) stays on the CPU
// builder.  Coordinates are assumed finite.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvhc_internal.h"
#include "softf64.cuh"

#ifdef BVHC_BUILD_TRACE
#include <chrono>
#include <cstdio>
#endif

namespace bvhc {
namespace {

using sf::f64;

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kBins = 32;                          // splitUtils.js:4 BIN_COUNT
constexpr int kBinWords = 7;                       // count, lo xyz, hi xyz (order-preserving codes)
constexpr int kNodeBinWords = 3 * kBins * kBinWords;
constexpr int kThreads = 256;
constexpr int kPer = 8;
constexpr int kChunk = kThreads * kPer;            // primitives per block in the large-node kernels
constexpr uint32_t kSmall = 1024;                  // subtrees of at most this many primitives: one warp
constexpr int kSubWarps = 4;
constexpr f64 kOneD = 0x3FF0000000000000ull;       // TRAVERSAL_COST (Constants.js:57)
constexpr f64 kPrimCostD = 0x3FF4000000000000ull;  // PRIMITIVE_INTERSECT_COST 1.25 (Constants.js:56)
constexpr f64 kTwoD = 0x4000000000000000ull;
constexpr f64 kHalfD = 0x3FE0000000000000ull;      // x / 2 and x * 0.5 round identically
constexpr f64 kInvBinsD = 0x3FA0000000000000ull;   // x / 32 and x * 2^-5 round identically
constexpr f64 kPadD = 0x3E70000000000000ull;       // FLOAT32_EPSILON 2^-24 (Constants.js:71)
constexpr float kBinEps = 0x1p-16f;
constexpr float kCostTol = 0x1p-16f;
constexpr uint32_t kEncPosInf = 0xFF800000u, kEncNegInf = 0x007FFFFFu;

#define GB_TRY(x)                                                                                  \
  do {                                                                                             \
    cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) throw DeviceBuildError(std::string("device build: ") + cudaGetErrorString(e_)); \
  } while (0)

// ---------------------------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t fenc(float f) {  // order-preserving code of a float
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fdec(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}
// Keys selecting the first primitive (lowest index) holding the extreme value, +0 == -0.
__device__ __forceinline__ unsigned long long key_min(float v, uint32_t e) {
  return ((unsigned long long)fenc(v == 0.0f ? 0.0f : v) << 32) | e;
}
__device__ __forceinline__ unsigned long long key_max(float v, uint32_t e) {
  return ((unsigned long long)fenc(v == 0.0f ? 0.0f : v) << 32) | (0xFFFFFFFFu - e);
}
__device__ __forceinline__ float fmin_lt(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float fmax_gt(float a, float b) { return b > a ? b : a; }

__device__ __forceinline__ bool goes_left(float c, f64 pos) { return sf::lt(sf::from_f32(c), pos); }

// computeSurfaceArea (ArrayBoxUtilities.js:101-108) in binary64.
__device__ __noinline__ f64 area_d(const float* lo, const float* hi) {
  const f64 d0 = sf::sub(sf::from_f32(hi[0]), sf::from_f32(lo[0]));
  const f64 d1 = sf::sub(sf::from_f32(hi[1]), sf::from_f32(lo[1]));
  const f64 d2 = sf::sub(sf::from_f32(hi[2]), sf::from_f32(lo[2]));
  return sf::mul(kTwoD, sf::add(sf::add(sf::mul(d0, d1), sf::mul(d1, d2)), sf::mul(d2, d0)));
}

// The split cost of splitUtils.js:162-166 / :268-272 in binary64.
__device__ __noinline__ f64 cost_d(const float* llo, const float* lhi, uint32_t lc, const float* rlo, const float* rhi, uint32_t rc,
                      f64 root_area) {
  f64 lp = 0, rp = 0;
  if (lc != 0) lp = sf::div(area_d(llo, lhi), root_area);
  if (rc != 0) rp = sf::div(area_d(rlo, rhi), root_area);
  return sf::add(kOneD, sf::mul(kPrimCostD, sf::add(sf::mul(lp, sf::from_u64(lc)), sf::mul(rp, sf::from_u64(rc)))));
}

// float32 estimate of area_d.  `ok` stays true only while every extent is 0 or in [2^-60, 2^60],
// where no step under- or overflows and the relative error is below 5 * 2^-24.
__device__ __forceinline__ bool extent_ok(float d) { return d == 0.0f || (d >= 0x1p-60f && d <= 0x1p60f); }
__device__ float area_f(const float* lo, const float* hi, bool& ok) {
  const float d0 = __fsub_rn(hi[0], lo[0]), d1 = __fsub_rn(hi[1], lo[1]), d2 = __fsub_rn(hi[2], lo[2]);
  ok = ok && extent_ok(d0) && extent_ok(d1) && extent_ok(d2);
  return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(d0, d1), __fmul_rn(d1, d2)), __fmul_rn(d2, d0)));
}

// Bin index `~~((c - left) / width)` clamped to 31 (splitUtils.js:199-204).
struct AxisBin {
  float l, r, lenf;
  bool fast;
};
__device__ AxisBin axis_bin(float l, float r) {
  AxisBin ab;
  ab.l = l;
  ab.r = r;
  ab.lenf = __fsub_rn(r, l);
  ab.fast = ab.lenf >= 0x1p-90f && ab.lenf <= 0x1p120f;
  return ab;
}
__device__ __noinline__ int bin_exact(float c, float l, float r) {  // the binary64 quotient
  const f64 left = sf::from_f32(l);
  const f64 width = sf::mul(sf::sub(sf::from_f32(r), left), kInvBinsD);
  const int b = sf::to_i32_trunc(sf::div(sf::sub(sf::from_f32(c), left), width));
  return b >= kBins ? kBins - 1 : (b < 0 ? 0 : b);
}
__device__ __forceinline__ int bin_of(float c, const AxisBin& ab) {
  if (ab.lenf == 0.0f) return 0;  // zero width: (c - left) / 0 is NaN, `~~NaN` is 0
  if (ab.fast) {
    if (c == ab.l) return 0;
    // three float32 roundings: |q - q64| < 32 * 3.01 * 2^-24 < 2^-17.5
    const float q = __fmul_rn(__fdiv_rn(__fsub_rn(c, ab.l), ab.lenf), 32.0f);
    if (q >= 31.0f + kBinEps) return kBins - 1;
    const float t = truncf(q);
    if ((t == 0.0f || q - t > kBinEps) && (t + 1.0f) - q > kBinEps) return (int)t;
  }
  return bin_exact(c, ab.l, ab.r);
}

struct Split {
  int axis;
  f64 pos;
};

__device__ __noinline__ Split binned_split_at(const float* cbox, int a, int i) {  // splitUtils.js:183
  const f64 L = sf::from_f32(cbox[a]);
  const f64 W = sf::mul(sf::sub(sf::from_f32(cbox[a + 3]), L), kInvBinsD);
  return {a, sf::add(sf::add(L, W), sf::mul(sf::from_u64((uint64_t)i), W))};
}

// Warp-wide binned SAH (splitUtils.js:176-281).  bins: [3][32][7] (any address space); lane i
// evaluates the split after bin i.  Warp-uniform; every lane returns the same split.
__device__ Split warp_sah_binned(const uint32_t* bins, uint32_t cnt, const float* box, const float* cbox) {
  const int lane = threadIdx.x & 31;
  uint32_t lc[3];
  float llo[3][3], lhi[3][3], rlo[3][3], rhi[3][3];
  bool valid[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const uint32_t* b = bins + (a * kBins + lane) * kBinWords;
    const uint32_t nb = b[0];
    float plo[3], phi[3], slo[3], shi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      plo[d] = slo[d] = fdec(b[1 + d]);
      phi[d] = shi[d] = fdec(b[4 + d]);
    }
    uint32_t c = nb;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t tc = __shfl_up_sync(kFull, c, o);
      if (lane >= o) c += tc;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float tl = __shfl_up_sync(kFull, plo[d], o), th = __shfl_up_sync(kFull, phi[d], o);
        const float ul = __shfl_down_sync(kFull, slo[d], o), uh = __shfl_down_sync(kFull, shi[d], o);
        if (lane >= o) {
          plo[d] = fmin_lt(plo[d], tl);
          phi[d] = fmax_gt(phi[d], th);
        }
        if (lane + o < 32) {
          slo[d] = fmin_lt(slo[d], ul);
          shi[d] = fmax_gt(shi[d], uh);
        }
      }
    }
    lc[a] = c;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      llo[a][d] = plo[d];
      lhi[a][d] = phi[d];
      const float nl = __shfl_down_sync(kFull, slo[d], 1), nh = __shfl_down_sync(kFull, shi[d], 1);
      rlo[a][d] = lane < 31 ? nl : __int_as_float(0x7F800000);
      rhi[a][d] = lane < 31 ? nh : __int_as_float(0xFF800000);
    }
    // the split after an empty bin i > 0 repeats the split after bin i - 1 exactly (same counts,
    // same boxes), so it can never win the reference's strict `<` scan
    valid[a] = lane < kBins - 1 && (lane == 0 || nb != 0);
  }

  // float32 ranking
  bool ok = true;
  const float rootf = area_f(box, box + 3, ok);
  ok = ok && rootf >= 0x1p-100f;
  float cf[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    cf[a] = __int_as_float(0x7F800000);
    if (valid[a]) {
      const uint32_t rc = cnt - lc[a];
      float lp = 0.0f, rp = 0.0f;
      if (lc[a] != 0) lp = __fdiv_rn(area_f(llo[a], lhi[a], ok), rootf);
      if (rc != 0) rp = __fdiv_rn(area_f(rlo[a], rhi[a], ok), rootf);
      ok = ok && (lp == 0.0f || lp >= 0x1p-100f) && (rp == 0.0f || rp >= 0x1p-100f);
      cf[a] = __fadd_rn(1.0f, __fmul_rn(1.25f, __fadd_rn(__fmul_rn(lp, (float)lc[a]), __fmul_rn(rp, (float)rc))));
    }
  }
  ok = __all_sync(kFull, ok);
  bool want[3] = {valid[0], valid[1], valid[2]};
  if (ok) {
    const float best0f = __fmul_rn(1.25f, (float)cnt);
    const float mine = fminf(cf[0], fminf(cf[1], cf[2]));
    const float m = __uint_as_float(__reduce_min_sync(kFull, __float_as_uint(mine)));  // all costs >= 1
    if (m > __fmul_rn(best0f, 1.0f + kCostTol)) return {-1, 0};
    const float hi = __fmul_rn(m, 1.0f + kCostTol);
    int ncont = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      want[a] = valid[a] && cf[a] <= hi;
      ncont += __popc(__ballot_sync(kFull, want[a]));
    }
    if (m < __fmul_rn(best0f, 1.0f - kCostTol)) {
      // the first contender in the reference's scan order (axis, then bin)
      int wa = 0, wl = 0;
      bool found = false;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const unsigned bal = __ballot_sync(kFull, want[a]);
        if (bal && !found) {
          found = true;
          wa = a;
          wl = __ffs(bal) - 1;
        }
      }
      if (ncont == 1) return binned_split_at(cbox, wa, wl);
      // contenders with the same counts and boxes as the first one have exactly its binary64
      // cost (the same partition reached along another axis, typically), so it wins the scan
      const uint32_t tlc = __shfl_sync(kFull, wa == 0 ? lc[0] : (wa == 1 ? lc[1] : lc[2]), wl);
      bool same = true;
#pragma unroll
      for (int a = 0; a < 3; ++a) same = same && (!want[a] || lc[a] == tlc);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float t0 = __shfl_sync(kFull, wa == 0 ? llo[0][d] : (wa == 1 ? llo[1][d] : llo[2][d]), wl);
        const float t1 = __shfl_sync(kFull, wa == 0 ? lhi[0][d] : (wa == 1 ? lhi[1][d] : lhi[2][d]), wl);
        const float t2 = __shfl_sync(kFull, wa == 0 ? rlo[0][d] : (wa == 1 ? rlo[1][d] : rlo[2][d]), wl);
        const float t3 = __shfl_sync(kFull, wa == 0 ? rhi[0][d] : (wa == 1 ? rhi[1][d] : rhi[2][d]), wl);
#pragma unroll
        for (int a = 0; a < 3; ++a)
          same = same && (!want[a] || (llo[a][d] == t0 && lhi[a][d] == t1 && rlo[a][d] == t2 && rhi[a][d] == t3));
      }
      if (__all_sync(kFull, same)) return binned_split_at(cbox, wa, wl);
    }
  }
  // binary64 over the contenders (all valid candidates when the float32 bound did not apply)
  const f64 root_area = area_d(box, box + 3);
  int64_t key = INT64_MAX;
  int sec = 1 << 20;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (want[a]) {
      const f64 c = cost_d(llo[a], lhi[a], lc[a], rlo[a], rhi[a], cnt - lc[a], root_area);
      if (!sf::is_nan(c) && sf::order_key(c) < key) {
        key = sf::order_key(c);
        sec = a * 32 + lane;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const int64_t ok2 = __shfl_xor_sync(kFull, (long long)key, o);
    const int os = __shfl_xor_sync(kFull, sec, o);
    if (ok2 < key || (ok2 == key && os < sec)) {
      key = ok2;
      sec = os;
    }
  }
  const f64 best0 = sf::mul(kPrimCostD, sf::from_u64(cnt));
  if (key == INT64_MAX || !(key < sf::order_key(best0))) return {-1, 0};
  return binned_split_at(cbox, sec >> 5, sec & 31);
}

// Every primitive center a candidate (splitUtils.js:63-174), for count < BIN_COUNT / 4.  One thread.
__device__ __noinline__ Split sah_small(const float* C, const float* L, const float* H, int64_t n, uint32_t off, uint32_t cnt,
                           const float* box) {
  const f64 root_area = area_d(box, box + 3);
  f64 best = sf::mul(kPrimCostD, sf::from_u64(cnt));
  Split s{-1, 0};
  for (int a = 0; a < 3; ++a) {
    float cand[kBins / 4];
    int m = 0;
    for (uint32_t i = 0; i < cnt; ++i) {  // stable insertion sort by center
      const float x = C[a * n + off + i];
      int j = m;
      while (j > 0 && cand[j - 1] > x) {
        cand[j] = cand[j - 1];
        --j;
      }
      cand[j] = x;
      ++m;
    }
    int k = 0;
    for (int i = 0; i < m; ++i)  // drop repeats of the previous candidate
      if (k == 0 || cand[i] != cand[k - 1]) cand[k++] = cand[i];
    for (int ci = 0; ci < k; ++ci) {
      float llo[3], lhi[3], rlo[3], rhi[3];
      for (int d = 0; d < 3; ++d) {
        llo[d] = rlo[d] = __int_as_float(0x7F800000);
        lhi[d] = rhi[d] = __int_as_float(0xFF800000);
      }
      uint32_t lc = 0;
      for (uint32_t i = 0; i < cnt; ++i) {
        const uint32_t e = off + i;
        const bool right = C[a * n + e] >= cand[ci];
        for (int d = 0; d < 3; ++d) {
          const float lo = L[d * n + e], hi = H[d * n + e];
          if (right) {
            rlo[d] = fmin_lt(rlo[d], lo);
            rhi[d] = fmax_gt(rhi[d], hi);
          } else {
            llo[d] = fmin_lt(llo[d], lo);
            lhi[d] = fmax_gt(lhi[d], hi);
          }
        }
        lc += right ? 0 : 1;
      }
      const f64 cost = cost_d(llo, lhi, lc, rlo, rhi, cnt - lc, root_area);
      if (sf::lt(cost, best)) {
        s.axis = a;
        best = cost;
        s.pos = sf::from_f32(cand[ci]);
      }
    }
  }
  return s;
}

// CENTER (splitUtils.js:25-35): longest centroid extent (strict `>`), split at its middle.
__device__ __noinline__ Split center_split(const float* cbox) {
  Split s{-1, 0};
  f64 best = sf::neg(sf::kInf);
  for (int i = 0; i < 3; ++i) {
    const f64 dist = sf::sub(sf::from_f32(cbox[i + 3]), sf::from_f32(cbox[i]));
    if (sf::lt(best, dist)) {
      best = dist;
      s.axis = i;
    }
  }
  if (s.axis >= 0) s.pos = sf::mul(sf::add(sf::from_f32(cbox[s.axis]), sf::from_f32(cbox[s.axis + 3])), kHalfD);
  return s;
}

__device__ __forceinline__ void swap_prims(float* C, float* L, float* H, uint32_t* perm, int64_t n, uint32_t a,
                                           uint32_t b) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    float t = C[d * n + a]; C[d * n + a] = C[d * n + b]; C[d * n + b] = t;
    t = L[d * n + a]; L[d * n + a] = L[d * n + b]; L[d * n + b] = t;
    t = H[d * n + a]; H[d * n + a] = H[d * n + b]; H[d * n + b] = t;
  }
  const uint32_t t = perm[a];
  perm[a] = perm[b];
  perm[b] = t;
}

// ---------------------------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------------------------

// computePrimitiveBounds (MeshBVH.js:365-436): per primitive slot, the padded box as center and
// fl32(center -/+ half).
__global__ void k_prims(const float* __restrict__ pos, int stride, const uint32_t* __restrict__ index, int has_index,
                        const uint32_t* __restrict__ indirect, int64_t base, int64_t n, float* C, float* L, float* H,
                        uint32_t* perm) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t slot = base + e;
    const int64_t tri = indirect ? (int64_t)indirect[slot] : slot;
    uint32_t v[3];
    for (int k = 0; k < 3; ++k) v[k] = has_index ? index[tri * 3 + k] : (uint32_t)(tri * 3 + k);
    for (int d = 0; d < 3; ++d) {
      const float a = pos[(int64_t)v[0] * stride + d], b = pos[(int64_t)v[1] * stride + d],
                  c = pos[(int64_t)v[2] * stride + d];
      float mn = a, mx = a;
      if (b < mn) mn = b;
      if (c < mn) mn = c;
      if (b > mx) mx = b;
      if (c > mx) mx = c;
      const f64 MN = sf::from_f32(mn);
      const f64 half = sf::mul(sf::sub(sf::from_f32(mx), MN), kHalfD);
      const float center = sf::to_f32(sf::add(MN, half));
      const float padded = sf::to_f32(sf::add(half, sf::mul(sf::add(sf::abs(MN), half), kPadD)));
      C[d * n + e] = center;
      L[d * n + e] = __fsub_rn(center, padded);
      H[d * n + e] = __fadd_rn(center, padded);
    }
    perm[e] = (uint32_t)e;
  }
}

// A contiguous primitive range (a node) cut into kChunk blocks.
struct Seg {
  uint32_t node, slot, off, cnt, first_block, pad;
};

__device__ __forceinline__ int find_seg(const Seg* segs, int n_segs, uint32_t block) {
  int lo = 0, hi = n_segs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (segs[mid].first_block <= block) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void k_bins_init(uint32_t* bins, int64_t words) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x) {
    const int w = (int)(i % kBinWords);
    bins[i] = w == 0 ? 0u : (w < 4 ? kEncPosInf : kEncNegInf);
  }
}

// Bin counts and boxes of the large nodes' chunks, aggregated per block in shared memory.
__global__ void __launch_bounds__(kThreads) k_bins(const Seg* __restrict__ segs, int n_segs,
                                                   const float* __restrict__ nbox, const float* __restrict__ C,
                                                   const float* __restrict__ L, const float* __restrict__ H, int64_t n,
                                                   uint32_t* bins) {
  __shared__ uint32_t sb[kNodeBinWords];
  __shared__ AxisBin sab[3];
  const Seg sg = segs[find_seg(segs, n_segs, blockIdx.x)];
  const uint32_t start = sg.off + (blockIdx.x - sg.first_block) * kChunk, end = min(start + kChunk, sg.off + sg.cnt);
  for (int i = threadIdx.x; i < kNodeBinWords; i += kThreads) {
    const int w = i % kBinWords;
    sb[i] = w == 0 ? 0u : (w < 4 ? kEncPosInf : kEncNegInf);
  }
  if (threadIdx.x < 3) sab[threadIdx.x] = axis_bin(nbox[sg.node * 12 + 6 + threadIdx.x], nbox[sg.node * 12 + 9 + threadIdx.x]);
  __syncthreads();
  for (int j = 0; j < kPer; ++j) {
    const uint32_t e = start + j * kThreads + threadIdx.x;
    if (e >= end) continue;
    float lo[3], hi[3];
    for (int d = 0; d < 3; ++d) {
      lo[d] = L[d * n + e];
      hi[d] = H[d * n + e];
    }
    for (int a = 0; a < 3; ++a) {
      uint32_t* b = sb + (a * kBins + bin_of(C[a * n + e], sab[a])) * kBinWords;
      atomicAdd(b, 1u);
      for (int d = 0; d < 3; ++d) {
        atomicMin(b + 1 + d, fenc(lo[d]));
        atomicMax(b + 4 + d, fenc(hi[d]));
      }
    }
  }
  __syncthreads();
  uint32_t* gb = bins + (size_t)sg.slot * kNodeBinWords;
  for (int k = threadIdx.x; k < 3 * kBins; k += kThreads) {
    const uint32_t* b = sb + k * kBinWords;
    if (b[0] == 0) continue;
    atomicAdd(gb + k * kBinWords, b[0]);
    for (int d = 0; d < 3; ++d) {
      atomicMin(gb + k * kBinWords + 1 + d, b[1 + d]);
      atomicMax(gb + k * kBinWords + 4 + d, b[4 + d]);
    }
  }
}

// One warp per large node: choose the split (SAH from the bins, or CENTER).
__global__ void k_choose(const Seg* __restrict__ segs, int n_segs, const float* __restrict__ nbox,
                         const uint32_t* __restrict__ bins, int strategy, int* axis_out, f64* pos_out) {
  const int slot = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (slot >= n_segs) return;
  const Seg sg = segs[slot];
  float box[6], cbox[6];
  for (int k = 0; k < 6; ++k) {
    box[k] = nbox[sg.node * 12 + k];
    cbox[k] = nbox[sg.node * 12 + 6 + k];
  }
  const Split s = strategy == kSah ? warp_sah_binned(bins + (size_t)slot * kNodeBinWords, sg.cnt, box, cbox)
                                   : center_split(cbox);
  if ((threadIdx.x & 31) == 0) {
    axis_out[slot] = s.axis;
    pos_out[slot] = s.pos;
  }
}

// Primitives of each large node that go left (center < pos).
__global__ void __launch_bounds__(kThreads) k_count(const Seg* __restrict__ segs, int n_segs,
                                                    const float* __restrict__ C, int64_t n, const int* __restrict__ axis,
                                                    const f64* __restrict__ pos, unsigned int* n_left) {
  const Seg sg = segs[find_seg(segs, n_segs, blockIdx.x)];
  const int a = axis[sg.slot];
  if (a < 0) return;
  const f64 p = pos[sg.slot];
  const uint32_t start = sg.off + (blockIdx.x - sg.first_block) * kChunk, end = min(start + kChunk, sg.off + sg.cnt);
  unsigned int total = 0;
  for (int j = 0; j < kPer; ++j) {
    const uint32_t e = start + j * kThreads + threadIdx.x;
    total += __syncthreads_count(e < end && goes_left(C[a * n + e], p));
  }
  if (threadIdx.x == 0 && total) atomicAdd(n_left + sg.slot, total);
}

// Block-wide exclusive count of `p` in thread order; `total` gets the block's count.
__device__ __forceinline__ uint32_t block_rank(bool p, uint32_t* s_warp, uint32_t& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned bal = __ballot_sync(kFull, p);
  if (lane == 0) s_warp[warp] = __popc(bal);
  __syncthreads();
  uint32_t before = 0;
  total = 0;
  for (int w = 0; w < kThreads / 32; ++w) {
    const uint32_t c = s_warp[w];
    before += w < warp ? c : 0;
    total += c;
  }
  __syncthreads();
  return before + __popc(bal & ((1u << lane) - 1u));
}

// Misplaced primitives per chunk: [2 * block] in the left part going right, [2 * block + 1] in
// the right part going left.
__global__ void __launch_bounds__(kThreads) k_pair_counts(const Seg* __restrict__ segs, int n_segs,
                                                          const float* __restrict__ C, int64_t n,
                                                          const int* __restrict__ axis, const f64* __restrict__ pos,
                                                          const unsigned int* __restrict__ n_left,
                                                          const uint8_t* __restrict__ split, uint32_t* chunk_cnt) {
  const Seg sg = segs[find_seg(segs, n_segs, blockIdx.x)];
  if (!split[sg.slot]) return;
  const int a = axis[sg.slot];
  const f64 p = pos[sg.slot];
  const uint32_t mid = sg.off + n_left[sg.slot];
  const uint32_t start = sg.off + (blockIdx.x - sg.first_block) * kChunk, end = min(start + kChunk, sg.off + sg.cnt);
  uint32_t ml = 0, mr = 0;
  for (int j = 0; j < kPer; ++j) {
    const uint32_t e = start + j * kThreads + threadIdx.x;
    const bool in = e < end;
    const bool gl = in && goes_left(C[a * n + e], p);
    ml += __syncthreads_count(in && e < mid && !gl);
    mr += __syncthreads_count(in && e >= mid && gl);
  }
  if (threadIdx.x == 0) {
    chunk_cnt[2 * blockIdx.x] = ml;
    chunk_cnt[2 * blockIdx.x + 1] = mr;
  }
}

// One warp per split node: rank bases of its chunks (left part ascending, right part from the end).
__global__ void k_pair_scan(const Seg* __restrict__ segs, int n_segs, const uint8_t* __restrict__ split,
                            const uint32_t* __restrict__ chunk_cnt, uint32_t* chunk_base) {
  const int slot = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (slot >= n_segs || !split[slot]) return;
  const Seg sg = segs[slot];
  const uint32_t nch = (sg.cnt + kChunk - 1) / kChunk, fb = sg.first_block;
  for (int side = 0; side < 2; ++side) {
    uint32_t run = 0;
    for (uint32_t k = 0; k < nch; k += 32) {
      const bool in = k + lane < nch;
      const uint32_t i = side == 0 ? k + lane : nch - 1 - (k + lane);
      const uint32_t v = in ? chunk_cnt[2 * (fb + i) + side] : 0;
      uint32_t incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += t;
      }
      if (in) chunk_base[2 * (fb + i) + side] = run + incl - v;
      run += __shfl_sync(kFull, incl, 31);
    }
  }
}

// Right-part primitives that go left record their positions by rank from the end.
__global__ void __launch_bounds__(kThreads) k_pair_mark(const Seg* __restrict__ segs, int n_segs,
                                                        const float* __restrict__ C, int64_t n,
                                                        const int* __restrict__ axis, const f64* __restrict__ pos,
                                                        const unsigned int* __restrict__ n_left,
                                                        const uint8_t* __restrict__ split,
                                                        const uint32_t* __restrict__ chunk_cnt,
                                                        const uint32_t* __restrict__ chunk_base, uint32_t* partner) {
  __shared__ uint32_t s_warp[kThreads / 32];
  const Seg sg = segs[find_seg(segs, n_segs, blockIdx.x)];
  if (!split[sg.slot]) return;
  const int a = axis[sg.slot];
  const f64 p = pos[sg.slot];
  const uint32_t mid = sg.off + n_left[sg.slot];
  const uint32_t start = sg.off + (blockIdx.x - sg.first_block) * kChunk, end = min(start + kChunk, sg.off + sg.cnt);
  const uint32_t chunk_total = chunk_cnt[2 * blockIdx.x + 1], base = chunk_base[2 * blockIdx.x + 1];
  uint32_t run = 0;
  for (int j = 0; j < kPer; ++j) {
    const uint32_t e = start + j * kThreads + threadIdx.x;
    const bool mis = e < end && e >= mid && goes_left(C[a * n + e], p);
    uint32_t tot;
    const uint32_t r = run + block_rank(mis, s_warp, tot);
    if (mis) partner[sg.off + base + (chunk_total - 1 - r)] = e;
    run += tot;
  }
}

// Left-part primitives that go right swap with their partners (the reference's Hoare swaps).
__global__ void __launch_bounds__(kThreads) k_pair_swap(const Seg* __restrict__ segs, int n_segs, float* C, float* L,
                                                        float* H, uint32_t* perm, int64_t n,
                                                        const int* __restrict__ axis, const f64* __restrict__ pos,
                                                        const unsigned int* __restrict__ n_left,
                                                        const uint8_t* __restrict__ split,
                                                        const uint32_t* __restrict__ chunk_base,
                                                        const uint32_t* __restrict__ partner) {
  __shared__ uint32_t s_warp[kThreads / 32];
  const Seg sg = segs[find_seg(segs, n_segs, blockIdx.x)];
  if (!split[sg.slot]) return;
  const int a = axis[sg.slot];
  const f64 p = pos[sg.slot];
  const uint32_t mid = sg.off + n_left[sg.slot];
  const uint32_t start = sg.off + (blockIdx.x - sg.first_block) * kChunk, end = min(start + kChunk, sg.off + sg.cnt);
  const uint32_t base = chunk_base[2 * blockIdx.x];
  uint32_t run = 0;
  for (int j = 0; j < kPer; ++j) {
    const uint32_t e = start + j * kThreads + threadIdx.x;
    const bool mis = e < end && e < mid && !goes_left(C[a * n + e], p);
    uint32_t tot;
    const uint32_t r = run + block_rank(mis, s_warp, tot);
    if (mis) swap_prims(C, L, H, perm, n, e, partner[sg.off + base + r]);
    run += tot;
  }
}

struct BoundKeys {
  unsigned long long kmin[3], kmax[3];
  uint32_t cmin[3], cmax[3];
};

__global__ void k_bounds_init(const uint32_t* __restrict__ ids, int n_ids, BoundKeys* keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ids) return;
  BoundKeys k;
  for (int d = 0; d < 3; ++d) {
    k.kmin[d] = ~0ull;
    k.kmax[d] = 0ull;
    k.cmin[d] = kEncPosInf;
    k.cmax[d] = kEncNegInf;
  }
  keys[ids[i]] = k;
}

// getBounds (computeBoundsUtils.js:4-68) over each segment's range, reduced per block.
__global__ void __launch_bounds__(kThreads) k_bounds(const Seg* __restrict__ segs, int n_segs,
                                                     const float* __restrict__ C, const float* __restrict__ L,
                                                     const float* __restrict__ H, int64_t n, BoundKeys* keys) {
  __shared__ BoundKeys sk[kThreads / 32];
  const Seg sg = segs[find_seg(segs, n_segs, blockIdx.x)];
  const uint32_t start = sg.off + (blockIdx.x - sg.first_block) * kChunk, end = min(start + kChunk, sg.off + sg.cnt);
  unsigned long long kmin[3] = {~0ull, ~0ull, ~0ull}, kmax[3] = {0ull, 0ull, 0ull};
  uint32_t cmin[3] = {kEncPosInf, kEncPosInf, kEncPosInf}, cmax[3] = {kEncNegInf, kEncNegInf, kEncNegInf};
  for (int j = 0; j < kPer; ++j) {
    const uint32_t e = start + j * kThreads + threadIdx.x;
    if (e >= end) break;
    for (int d = 0; d < 3; ++d) {
      kmin[d] = min(kmin[d], key_min(L[d * n + e], e));
      kmax[d] = max(kmax[d], key_max(H[d * n + e], e));
      const uint32_t c = fenc(C[d * n + e]);
      cmin[d] = min(cmin[d], c);
      cmax[d] = max(cmax[d], c);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int d = 0; d < 3; ++d) {
      kmin[d] = min(kmin[d], (unsigned long long)__shfl_xor_sync(kFull, kmin[d], o));
      kmax[d] = max(kmax[d], (unsigned long long)__shfl_xor_sync(kFull, kmax[d], o));
      cmin[d] = min(cmin[d], __shfl_xor_sync(kFull, cmin[d], o));
      cmax[d] = max(cmax[d], __shfl_xor_sync(kFull, cmax[d], o));
    }
  }
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; ++d) {
      sk[warp].kmin[d] = kmin[d];
      sk[warp].kmax[d] = kmax[d];
      sk[warp].cmin[d] = cmin[d];
      sk[warp].cmax[d] = cmax[d];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; ++w)
      for (int d = 0; d < 3; ++d) {
        kmin[d] = min(kmin[d], sk[w].kmin[d]);
        kmax[d] = max(kmax[d], sk[w].kmax[d]);
        cmin[d] = min(cmin[d], sk[w].cmin[d]);
        cmax[d] = max(cmax[d], sk[w].cmax[d]);
      }
    BoundKeys& g = keys[sg.node];
    for (int d = 0; d < 3; ++d) {
      atomicMin(&g.kmin[d], kmin[d]);
      atomicMax(&g.kmax[d], kmax[d]);
      atomicMin(&g.cmin[d], cmin[d]);
      atomicMax(&g.cmax[d], cmax[d]);
    }
  }
}

// Node box (the first primitive's value for each extreme) and centroid box from the keys.
__global__ void k_bounds_finish(const uint32_t* __restrict__ ids, int n_ids, const BoundKeys* __restrict__ keys,
                                const float* __restrict__ L, const float* __restrict__ H, int64_t n, float* nbox) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_ids) return;
  const uint32_t id = ids[i];
  const BoundKeys& k = keys[id];
  if (k.kmin[0] == ~0ull) {  // empty range: getBounds leaves the +/-Infinity initial box
    for (int d = 0; d < 3; ++d) {
      nbox[id * 12 + d] = nbox[id * 12 + 6 + d] = __int_as_float(0x7F800000);
      nbox[id * 12 + 3 + d] = nbox[id * 12 + 9 + d] = __int_as_float(0xFF800000);
    }
    return;
  }
  for (int d = 0; d < 3; ++d) {
    nbox[id * 12 + d] = L[d * n + (uint32_t)k.kmin[d]];
    nbox[id * 12 + 3 + d] = H[d * n + (0xFFFFFFFFu - (uint32_t)k.kmax[d])];
    nbox[id * 12 + 6 + d] = fdec(k.cmin[d]);
    nbox[id * 12 + 9 + d] = fdec(k.cmax[d]);
  }
}

// One warp: box (first primitive for each extreme) and centroid box of [off, off + cnt).
__device__ __noinline__ void warp_bounds(const float* C, const float* L, const float* H, int64_t n, uint32_t off, uint32_t cnt,
                            float* box, float* cbox) {
  const int lane = threadIdx.x & 31;
  float bmin[3], bmax[3], cmin[3], cmax[3];
  uint32_t imin[3], imax[3];
  for (int d = 0; d < 3; ++d) {
    bmin[d] = cmin[d] = __int_as_float(0x7F800000);
    bmax[d] = cmax[d] = __int_as_float(0xFF800000);
    imin[d] = imax[d] = 0xFFFFFFFFu;
  }
  for (uint32_t e = off + lane; e < off + cnt; e += 32) {
    for (int d = 0; d < 3; ++d) {
      const float lo = L[d * n + e], hi = H[d * n + e], c = C[d * n + e];
      if (lo < bmin[d]) { bmin[d] = lo; imin[d] = e; }
      if (hi > bmax[d]) { bmax[d] = hi; imax[d] = e; }
      cmin[d] = fmin_lt(cmin[d], c);
      cmax[d] = fmax_gt(cmax[d], c);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int d = 0; d < 3; ++d) {
      const float vl = __shfl_xor_sync(kFull, bmin[d], o), vh = __shfl_xor_sync(kFull, bmax[d], o);
      const uint32_t il = __shfl_xor_sync(kFull, imin[d], o), ih = __shfl_xor_sync(kFull, imax[d], o);
      if (vl < bmin[d] || (vl == bmin[d] && il < imin[d])) { bmin[d] = vl; imin[d] = il; }
      if (vh > bmax[d] || (vh == bmax[d] && ih < imax[d])) { bmax[d] = vh; imax[d] = ih; }
      cmin[d] = fmin_lt(cmin[d], __shfl_xor_sync(kFull, cmin[d], o));
      cmax[d] = fmax_gt(cmax[d], __shfl_xor_sync(kFull, cmax[d], o));
    }
  }
  for (int d = 0; d < 3; ++d) {
    box[d] = bmin[d];
    box[d + 3] = bmax[d];
    cbox[d] = cmin[d];
    cbox[d + 3] = cmax[d];
  }
}

// A node of the small-node phase.  Nodes of one level occupy a contiguous id range (children are
// allocated in pairs by the level that splits their parent); the small roots are ids [0, n_roots).
struct SmallNode {
  float box[6], cbox[6];
  uint32_t off, cnt, depth;
  int32_t left;   // first child id (the right child is left + 1); -1 for a leaf
  int32_t axis;
  uint32_t size;  // nodes in the subtree
  uint32_t dest;  // pre-order slot in the output
  uint32_t pad;
};

// One warp per node of level [lv[level], lv[level + 1]): the reference's splitNode step (leaf
// test, split choice, Hoare partition, child bounds); children are appended for the next level.
__global__ void __launch_bounds__(kSubWarps * 32, 8) k_small_level(SmallNode* nodes, const uint32_t* __restrict__ lv,
                                                                   int level, unsigned int* counter, float* C, float* L,
                                                                   float* H, uint32_t* perm, int64_t n,
                                                                   uint32_t* partner, int strategy, int max_depth,
                                                                   int leaf) {
  __shared__ uint32_t s_bins[kSubWarps][kNodeBinWords];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t* bins = s_bins[wib];
  const uint32_t first = lv[level], last = lv[level + 1];
  const uint32_t n_warps = gridDim.x * kSubWarps;
  for (uint32_t id = first + blockIdx.x * kSubWarps + wib; id < last; id += n_warps) {
    SmallNode* nd = nodes + id;
    const uint32_t off = nd->off, cnt = nd->cnt, depth = nd->depth;
    float box[6], cbox[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      box[k] = nd->box[k];
      cbox[k] = nd->cbox[k];
    }
    bool leaf_node = cnt <= (uint32_t)leaf || (int)depth >= max_depth;
    Split s{-1, 0};
    uint32_t nl = 0;
    if (!leaf_node) {
      if (strategy == kSah && cnt < kBins / 4) {
        if (lane == 0) s = sah_small(C, L, H, n, off, cnt, box);
        s.axis = __shfl_sync(kFull, s.axis, 0);
        s.pos = (f64)__shfl_sync(kFull, (long long)s.pos, 0);
      } else if (strategy == kSah) {
        for (int i = lane; i < kNodeBinWords; i += 32) {
          const int w = i % kBinWords;
          bins[i] = w == 0 ? 0u : (w < 4 ? kEncPosInf : kEncNegInf);
        }
        AxisBin ab[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) ab[a] = axis_bin(cbox[a], cbox[a + 3]);
        __syncwarp();
        for (uint32_t e = off + lane; e < off + cnt; e += 32) {
          float lo[3], hi[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            lo[d] = L[d * n + e];
            hi[d] = H[d * n + e];
          }
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            uint32_t* b = bins + (a * kBins + bin_of(C[a * n + e], ab[a])) * kBinWords;
            atomicAdd(b, 1u);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              atomicMin(b + 1 + d, fenc(lo[d]));
              atomicMax(b + 4 + d, fenc(hi[d]));
            }
          }
        }
        __syncwarp();
        s = warp_sah_binned(bins, cnt, box, cbox);
        __syncwarp();
      } else {
        s = center_split(cbox);
      }
      if (s.axis >= 0) {
        for (uint32_t k = 0; k < cnt; k += 32) {
          const uint32_t e = off + k + lane;
          nl += __popc(__ballot_sync(kFull, k + lane < cnt && goes_left(C[s.axis * n + e], s.pos)));
        }
      }
      leaf_node = s.axis < 0 || nl == 0 || nl == cnt;
    }
    if (leaf_node) {
      if (lane == 0) nd->left = -1;
      continue;
    }
    // Hoare pairing: the k-th left-part primitive going right swaps with the k-th right-part
    // primitive (from the end) going left
    const uint32_t end = off + cnt, nr = cnt - nl;
    uint32_t rank = 0;
    for (uint32_t k = 0; k < nr; k += 32) {
      const uint32_t e = end - 1 - (k + lane);
      const bool mis = k + lane < nr && goes_left(C[s.axis * n + e], s.pos);
      const unsigned bal = __ballot_sync(kFull, mis);
      if (mis) partner[off + rank + __popc(bal & ((1u << lane) - 1u))] = e;
      rank += __popc(bal);
    }
    __syncwarp();
    rank = 0;
    for (uint32_t k = 0; k < nl; k += 32) {
      const uint32_t e = off + k + lane;
      const bool mis = k + lane < nl && !goes_left(C[s.axis * n + e], s.pos);
      const unsigned bal = __ballot_sync(kFull, mis);
      if (mis) swap_prims(C, L, H, perm, n, e, partner[off + rank + __popc(bal & ((1u << lane) - 1u))]);
      rank += __popc(bal);
    }
    __syncwarp();
    float lbox[6], lcbox[6], rbox[6], rcbox[6];
    warp_bounds(C, L, H, n, off, nl, lbox, lcbox);
    warp_bounds(C, L, H, n, off + nl, nr, rbox, rcbox);
    uint32_t child = 0;
    if (lane == 0) child = atomicAdd(counter, 2u);
    child = __shfl_sync(kFull, child, 0);
    if (lane < 2) {
      SmallNode c;
      for (int k = 0; k < 6; ++k) {
        c.box[k] = lane == 0 ? lbox[k] : rbox[k];
        c.cbox[k] = lane == 0 ? lcbox[k] : rcbox[k];
      }
      c.off = lane == 0 ? off : off + nl;
      c.cnt = lane == 0 ? nl : nr;
      c.depth = depth + 1;
      c.left = -1;
      c.axis = -1;
      c.size = 0;
      c.dest = 0;
      c.pad = 0;
      nodes[child + lane] = c;
    }
    if (lane == 0) {
      nd->left = (int32_t)child;
      nd->axis = s.axis;
    }
  }
}

// The small roots' boxes from the large-node table.
__global__ void k_small_boxes(const uint32_t* __restrict__ ids, int n_roots, const float* __restrict__ nbox,
                              SmallNode* nodes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_roots) return;
  for (int k = 0; k < 6; ++k) {
    nodes[i].box[k] = nbox[ids[i] * 12 + k];
    nodes[i].cbox[k] = nbox[ids[i] * 12 + 6 + k];
  }
}

// lv[level + 2] = the node count once level `level` has appended its children.
__global__ void k_level_close(uint32_t* lv, int level, const unsigned int* counter) { lv[level + 2] = *counter; }

// Subtree sizes, deepest level first.
__global__ void k_sizes(SmallNode* nodes, const uint32_t* __restrict__ lv, int level) {
  const uint32_t first = lv[level], last = lv[level + 1];
  for (uint32_t id = first + blockIdx.x * blockDim.x + threadIdx.x; id < last; id += gridDim.x * blockDim.x) {
    SmallNode* nd = nodes + id;
    nd->size = nd->left < 0 ? 1u : 1u + nodes[nd->left].size + nodes[nd->left + 1].size;
  }
}

__global__ void k_set_dest(SmallNode* nodes, const uint32_t* __restrict__ dest, int n_roots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_roots) nodes[i].dest = dest[i];
}

// Pre-order slots, top level first: the left child follows its parent, the right child follows
// the left subtree (buildUtils.js:35-92).
__global__ void k_dests(SmallNode* nodes, const uint32_t* __restrict__ lv, int level) {
  const uint32_t first = lv[level], last = lv[level + 1];
  for (uint32_t id = first + blockIdx.x * blockDim.x + threadIdx.x; id < last; id += gridDim.x * blockDim.x) {
    const SmallNode* nd = nodes + id;
    if (nd->left < 0) continue;
    nodes[nd->left].dest = nd->dest + 1;
    nodes[nd->left + 1].dest = nd->dest + 1 + nodes[nd->left].size;
  }
}

// The 32-byte records of every small-phase node (_populateBuffer, buildUtils.js:35-92).
__global__ void k_write_small(const SmallNode* __restrict__ nodes, const unsigned int* __restrict__ counter,
                              uint32_t base, uint32_t* out) {
  const uint32_t total = *counter;
  for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < total; id += gridDim.x * blockDim.x) {
    const SmallNode& nd = nodes[id];
    uint32_t* o = out + (size_t)nd.dest * 8;
#pragma unroll
    for (int k = 0; k < 6; ++k) o[k] = __float_as_uint(nd.box[k]);
    if (nd.left < 0) {
      o[6] = base + nd.off;
      o[7] = (nd.cnt & 0xFFFFu) | 0xFFFF0000u;
    } else {
      o[6] = 1u + nodes[nd.left].size;
      o[7] = (uint32_t)nd.axis;
    }
  }
}

struct PlaceRec {
  uint32_t node, dest, w6, w7;
};

__global__ void k_place(const PlaceRec* __restrict__ recs, int n_recs, const float* __restrict__ nbox, uint32_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_recs) return;
  const PlaceRec r = recs[i];
  uint32_t* o = out + (size_t)r.dest * 8;
  for (int k = 0; k < 6; ++k) o[k] = __float_as_uint(nbox[r.node * 12 + k]);
  o[6] = r.w6;
  o[7] = r.w7;
}

__global__ void k_reorder(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ in, uint32_t* out, int64_t n,
                          int width) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
    for (int k = 0; k < width; ++k) out[e * width + k] = in[(int64_t)perm[e] * width + k];
}

// ---------------------------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------------------------

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  void alloc(size_t count) {
    if (count <= n) return;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    GB_TRY(cudaMalloc(reinterpret_cast<void**>(&p), std::max<size_t>(count, 1) * sizeof(T)));
    n = count;
  }
};

enum { kNodeLeaf = 0, kNodeInner = 1, kNodeSub = 2 };

struct HostNode {
  uint32_t off, cnt;
  int depth, kind = kNodeLeaf, left = -1, right = -1, axis = -1, sub = -1, root = 0;
};

int grid_for(int64_t n, int threads) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 64)); }

#ifdef BVHC_BUILD_TRACE
#define GB_TRACE(what) trace(what)
#else
#define GB_TRACE(what) ((void)0)
#endif

class DeviceBuilder {
 public:
  DeviceBuilder(Serialized& s, cudaStream_t stream, int strategy, int max_depth, int leaf)
      : s_(s), st_(stream), strategy_(strategy), max_depth_(max_depth), leaf_(leaf) {}

  void run(const float* pos, uint64_t n_verts, int stride, const std::vector<Range>& ranges) {
    base_ = ranges.front().offset;
    n_ = ranges.back().offset + ranges.back().count - base_;
    if (n_ < 0 || n_ >= (int64_t)0xFFFFFFFF) throw std::runtime_error("device build: primitive count out of range");
    const bool ind = s_.indirect;
    const int width = ind ? 1 : 3;

    DevBuf<float> d_pos;
    d_pos.alloc((size_t)n_verts * stride);
    GB_TRY(cudaMemcpyAsync(d_pos.p, pos, (size_t)n_verts * stride * sizeof(float), cudaMemcpyHostToDevice, st_));
    DevBuf<uint32_t> d_index, d_indirect;
    if (s_.has_index) {
      d_index.alloc(s_.index.size());
      GB_TRY(cudaMemcpyAsync(d_index.p, s_.index.data(), s_.index.size() * 4, cudaMemcpyHostToDevice, st_));
    }
    if (ind) {
      d_indirect.alloc(s_.indirect_buf.size());
      GB_TRY(cudaMemcpyAsync(d_indirect.p, s_.indirect_buf.data(), s_.indirect_buf.size() * 4, cudaMemcpyHostToDevice, st_));
    }
    prims_.alloc((size_t)n_ * 9);
    perm_.alloc((size_t)n_);
    partner_.alloc((size_t)n_);
    GB_TRACE("upload+alloc");
    C_ = prims_.p;
    L_ = prims_.p + 3 * n_;
    H_ = prims_.p + 6 * n_;
    k_prims<<<grid_for(n_, 256), 256, 0, st_>>>(d_pos.p, stride, s_.has_index ? d_index.p : nullptr, s_.has_index ? 1 : 0,
                                                ind ? d_indirect.p : nullptr, base_, n_, C_, L_, H_, perm_.p);
    GB_TRY(cudaGetLastError());

    // large-node scratch, sized once: each level's large nodes are disjoint ranges of more than
    // kSmall primitives, and only depths below max_depth split
    const int64_t nf_max = (int64_t)ranges.size() + n_ / (kSmall + 1) + 1;
    const int64_t blocks_max = n_ / kChunk + nf_max + 1;
    const int64_t cap = (int64_t)ranges.size() + 2 * std::min<int64_t>(n_, std::max(1, max_depth_) * (n_ / (kSmall + 1) + 1));
    nbox_.alloc((size_t)cap * 12);
    keys_.alloc((size_t)cap);
    segs_.alloc((size_t)2 * nf_max);
    ids_.alloc((size_t)2 * nf_max);
    axis_.alloc((size_t)nf_max);
    posd_.alloc((size_t)nf_max);
    nl_.alloc((size_t)nf_max);
    split_.alloc((size_t)nf_max);
    cc_.alloc((size_t)2 * blocks_max);
    cb_.alloc((size_t)2 * blocks_max);
    if (strategy_ == kSah) bins_.alloc((size_t)nf_max * kNodeBinWords);

    std::vector<int> frontier;
    std::vector<uint32_t> fresh;
    for (size_t r = 0; r < ranges.size(); ++r) {
      HostNode h;
      h.off = (uint32_t)(ranges[r].offset - base_);
      h.cnt = (uint32_t)ranges[r].count;
      h.depth = 0;
      h.root = (int)r;
      nodes_.push_back(h);
      fresh.push_back((uint32_t)r);
    }
    compute_bounds(fresh);
    for (uint32_t id : fresh) classify((int)id, frontier);
    GB_TRACE("prims+scratch");
    while (!frontier.empty()) split_level(frontier);
    GB_TRACE("large nodes");
    small_phase();
    GB_TRACE("small nodes");
    assemble(ranges.size());
    GB_TRACE("assemble+d2h");

    // the reordered partition buffer (index triples or indirect entries of [base, base + n))
    DevBuf<uint32_t> d_out;
    d_out.alloc((size_t)n_ * width);
    const uint32_t* d_in = (ind ? d_indirect.p : d_index.p) + (size_t)base_ * width;
    k_reorder<<<grid_for(n_, 256), 256, 0, st_>>>(perm_.p, d_in, d_out.p, n_, width);
    GB_TRY(cudaGetLastError());
    std::vector<uint32_t>& dst = ind ? s_.indirect_buf : s_.index;
    GB_TRY(cudaMemcpyAsync(dst.data() + (size_t)base_ * width, d_out.p, (size_t)n_ * width * 4, cudaMemcpyDeviceToHost, st_));
    GB_TRY(cudaStreamSynchronize(st_));
    GB_TRACE("reorder+d2h");
  }

 private:
#ifdef BVHC_BUILD_TRACE
  std::chrono::steady_clock::time_point t_ = std::chrono::steady_clock::now();
  void trace(const char* what) {  // phase timing for development builds
    cudaStreamSynchronize(st_);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "device build %-14s %8.3f ms\n", what, std::chrono::duration<double, std::milli>(now - t_).count());
    t_ = now;
  }
#endif
  Serialized& s_;
  cudaStream_t st_;
  int strategy_, max_depth_, leaf_;
  int64_t base_ = 0, n_ = 0;
  DevBuf<float> prims_, nbox_;
  DevBuf<uint32_t> perm_, partner_, ids_, cc_, cb_, bins_;
  DevBuf<BoundKeys> keys_;
  DevBuf<Seg> segs_;
  DevBuf<int> axis_;
  DevBuf<f64> posd_;
  DevBuf<unsigned int> nl_;
  DevBuf<uint8_t> split_;
  float *C_ = nullptr, *L_ = nullptr, *H_ = nullptr;
  std::vector<HostNode> nodes_;
  std::vector<int> subs_;  // node ids of the small-phase roots

  // One segment per node, cut into kChunk blocks; returns the block count.
  uint32_t make_segs(const std::vector<int>& ids, std::vector<Seg>& segs) {
    segs.clear();
    uint32_t blocks = 0;
    for (size_t i = 0; i < ids.size(); ++i) {
      const HostNode& h = nodes_[ids[i]];
      segs.push_back({(uint32_t)ids[i], (uint32_t)i, h.off, h.cnt, blocks, 0});
      blocks += (h.cnt + kChunk - 1) / kChunk;
    }
    return blocks;
  }

  template <class T>
  void upload(T* d, const std::vector<T>& h, size_t cap) {
    if (h.size() > cap) throw std::runtime_error("device build: scratch overflow");
    if (!h.empty()) GB_TRY(cudaMemcpyAsync(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st_));
  }

  void compute_bounds(const std::vector<uint32_t>& ids) {
    std::vector<int> iv(ids.begin(), ids.end());
    std::vector<Seg> segs;
    const uint32_t blocks = make_segs(iv, segs);
    upload(segs_.p, segs, segs_.n);
    upload(ids_.p, ids, ids_.n);
    const int n = (int)ids.size();
    k_bounds_init<<<(n + 255) / 256, 256, 0, st_>>>(ids_.p, n, keys_.p);
    if (blocks > 0) k_bounds<<<blocks, kThreads, 0, st_>>>(segs_.p, (int)segs.size(), C_, L_, H_, n_, keys_.p);
    k_bounds_finish<<<(n + 255) / 256, 256, 0, st_>>>(ids_.p, n, keys_.p, L_, H_, n_, nbox_.p);
    GB_TRY(cudaGetLastError());
  }

  void classify(int id, std::vector<int>& frontier) {
    HostNode& h = nodes_[id];
    if (h.cnt <= (uint32_t)leaf_ || h.depth >= max_depth_) {
      h.kind = kNodeLeaf;
    } else if (h.cnt <= kSmall) {
      h.kind = kNodeSub;
      h.sub = (int)subs_.size();
      subs_.push_back(id);
    } else {
      frontier.push_back(id);
    }
  }

  void split_level(std::vector<int>& frontier) {
    std::vector<Seg> segs;
    const uint32_t blocks = make_segs(frontier, segs);
    const int nf = (int)frontier.size();
    if (nf > (int)axis_.n || 2 * (size_t)blocks > cc_.n) throw std::runtime_error("device build: scratch overflow");
    upload(segs_.p, segs, segs_.n);
    if (strategy_ == kSah) {
      k_bins_init<<<grid_for((int64_t)nf * kNodeBinWords, 256), 256, 0, st_>>>(bins_.p, (int64_t)nf * kNodeBinWords);
      k_bins<<<blocks, kThreads, 0, st_>>>(segs_.p, nf, nbox_.p, C_, L_, H_, n_, bins_.p);
    }
    k_choose<<<(nf + 3) / 4, 128, 0, st_>>>(segs_.p, nf, nbox_.p, bins_.p, strategy_, axis_.p, posd_.p);
    GB_TRY(cudaMemsetAsync(nl_.p, 0, nf * sizeof(unsigned int), st_));
    k_count<<<blocks, kThreads, 0, st_>>>(segs_.p, nf, C_, n_, axis_.p, posd_.p, nl_.p);
    GB_TRY(cudaGetLastError());
    std::vector<int> axis(nf);
    std::vector<unsigned int> nl(nf);
    GB_TRY(cudaMemcpyAsync(axis.data(), axis_.p, nf * sizeof(int), cudaMemcpyDeviceToHost, st_));
    GB_TRY(cudaMemcpyAsync(nl.data(), nl_.p, nf * sizeof(unsigned int), cudaMemcpyDeviceToHost, st_));
    GB_TRY(cudaStreamSynchronize(st_));

    std::vector<uint8_t> split(nf, 0);
    std::vector<uint32_t> children;
    for (int i = 0; i < nf; ++i) {
      HostNode& h = nodes_[frontier[i]];
      if (axis[i] < 0 || nl[i] == 0 || nl[i] == h.cnt) {  // buildTree.js:60-72: no useful split
        h.kind = kNodeLeaf;
        continue;
      }
      split[i] = 1;
      h.kind = kNodeInner;
      h.axis = axis[i];
      HostNode l, r;
      l.off = h.off;
      l.cnt = nl[i];
      r.off = h.off + nl[i];
      r.cnt = h.cnt - nl[i];
      l.depth = r.depth = h.depth + 1;
      l.root = r.root = h.root;
      h.left = (int)nodes_.size();
      h.right = h.left + 1;
      nodes_.push_back(l);
      nodes_.push_back(r);
      children.push_back((uint32_t)h.left);
      children.push_back((uint32_t)h.right);
    }
    std::vector<int> next;
    if (!children.empty()) {
      if (nodes_.size() > keys_.n) throw std::runtime_error("device build: node table overflow");
      upload(split_.p, split, split_.n);
      k_pair_counts<<<blocks, kThreads, 0, st_>>>(segs_.p, nf, C_, n_, axis_.p, posd_.p, nl_.p, split_.p, cc_.p);
      k_pair_scan<<<(nf + 3) / 4, 128, 0, st_>>>(segs_.p, nf, split_.p, cc_.p, cb_.p);
      k_pair_mark<<<blocks, kThreads, 0, st_>>>(segs_.p, nf, C_, n_, axis_.p, posd_.p, nl_.p, split_.p, cc_.p, cb_.p,
                                                partner_.p);
      k_pair_swap<<<blocks, kThreads, 0, st_>>>(segs_.p, nf, C_, L_, H_, perm_.p, n_, axis_.p, posd_.p, nl_.p,
                                                split_.p, cb_.p, partner_.p);
      GB_TRY(cudaGetLastError());
      compute_bounds(children);
      for (uint32_t id : children) classify((int)id, next);
    }
    frontier.swap(next);
  }

  DevBuf<SmallNode> small_;
  DevBuf<uint32_t> lv_;
  DevBuf<unsigned int> counter_;
  int levels_ = 0;
  std::vector<uint32_t> sub_sizes_;

  // Every small root's subtree, level by level on the device.
  void small_phase() {
    const int ns = (int)subs_.size();
    sub_sizes_.assign(ns, 0);
    if (ns == 0) return;
    uint64_t cells = ns;
    int min_depth = max_depth_;
    std::vector<SmallNode> roots(ns);
    std::vector<uint32_t> root_ids(ns);
    for (int k = 0; k < ns; ++k) {
      const HostNode& h = nodes_[subs_[k]];
      SmallNode& r = roots[k];
      std::memset(&r, 0, sizeof r);
      r.off = h.off;
      r.cnt = h.cnt;
      r.depth = (uint32_t)h.depth;
      r.left = -1;
      r.axis = -1;
      root_ids[k] = (uint32_t)subs_[k];
      cells += 2 * (uint64_t)h.cnt;
      min_depth = std::min(min_depth, h.depth);
    }
    if (cells >= 0xFFFFFFFFull) throw std::runtime_error("device build: too many nodes");
    small_.alloc((size_t)cells);
    GB_TRY(cudaMemcpyAsync(small_.p, roots.data(), ns * sizeof(SmallNode), cudaMemcpyHostToDevice, st_));
    DevBuf<uint32_t> d_root_ids;
    d_root_ids.alloc(ns);
    GB_TRY(cudaMemcpyAsync(d_root_ids.p, root_ids.data(), ns * 4, cudaMemcpyHostToDevice, st_));
    k_small_boxes<<<(ns + 255) / 256, 256, 0, st_>>>(d_root_ids.p, ns, nbox_.p, small_.p);
    const int max_levels = std::max(1, max_depth_ - min_depth + 1);
    lv_.alloc((size_t)max_levels + 2);
    counter_.alloc(1);
    const uint32_t init[2] = {0u, (uint32_t)ns};
    GB_TRY(cudaMemcpyAsync(lv_.p, init, sizeof init, cudaMemcpyHostToDevice, st_));
    GB_TRY(cudaMemcpyAsync(counter_.p, &init[1], sizeof(unsigned int), cudaMemcpyHostToDevice, st_));
    const int grid = 148 * 8;
    levels_ = 0;
    for (int level = 0; level < max_levels; ++level) {
      k_small_level<<<grid, kSubWarps * 32, 0, st_>>>(small_.p, lv_.p, level, counter_.p, C_, L_, H_, perm_.p, n_,
                                                      partner_.p, strategy_, max_depth_, leaf_);
      k_level_close<<<1, 1, 0, st_>>>(lv_.p, level, counter_.p);
      GB_TRY(cudaGetLastError());
      levels_ = level + 1;
      if (level % 8 == 7) {  // stop once a level appends no children
        uint32_t b[2];
        GB_TRY(cudaMemcpyAsync(b, lv_.p + level + 1, sizeof b, cudaMemcpyDeviceToHost, st_));
        GB_TRY(cudaStreamSynchronize(st_));
        if (b[0] == b[1]) break;
      }
    }
    for (int level = levels_ - 1; level >= 0; --level) k_sizes<<<grid, 256, 0, st_>>>(small_.p, lv_.p, level);
    GB_TRY(cudaGetLastError());
    GB_TRY(cudaMemcpy2DAsync(sub_sizes_.data(), sizeof(uint32_t), &small_.p[0].size, sizeof(SmallNode),
                             sizeof(uint32_t), ns, cudaMemcpyDeviceToHost, st_));
    GB_TRY(cudaStreamSynchronize(st_));
  }

  // Pre-order placement (buildUtils.js:35-92): the large nodes on the host (children always have
  // larger ids than their parent), the small-phase subtrees on the device.
  void assemble(size_t n_roots) {
    const size_t nn = nodes_.size();
    std::vector<uint64_t> size(nn), pre(nn);
    for (size_t i = nn; i-- > 0;) {
      const HostNode& h = nodes_[i];
      size[i] = h.kind == kNodeInner ? 1 + size[h.left] + size[h.right] : (h.kind == kNodeSub ? sub_sizes_[h.sub] : 1);
    }
    std::vector<uint64_t> root_first(n_roots + 1, 0);
    for (size_t r = 0; r < n_roots; ++r) root_first[r + 1] = root_first[r] + size[r];
    const uint64_t total = root_first[n_roots];
    if (total >= 0xFFFFFFFFull) throw std::runtime_error("device build: too many nodes");
    std::vector<PlaceRec> recs;
    std::vector<uint32_t> sub_dest(subs_.size());
    for (size_t i = 0; i < nn; ++i) {
      const HostNode& h = nodes_[i];
      if (i < n_roots) pre[i] = 0;
      const uint32_t dest = (uint32_t)(root_first[h.root] + pre[i]);
      if (h.kind == kNodeInner) {
        pre[h.left] = pre[i] + 1;
        pre[h.right] = pre[i] + 1 + size[h.left];
        recs.push_back({(uint32_t)i, dest, (uint32_t)(1 + size[h.left]), (uint32_t)h.axis});
      } else if (h.kind == kNodeSub) {
        sub_dest[h.sub] = dest;
      } else {
        recs.push_back({(uint32_t)i, dest, (uint32_t)(base_ + h.off), (h.cnt & 0xFFFFu) | 0xFFFF0000u});
      }
    }
    DevBuf<uint32_t> d_out;
    d_out.alloc((size_t)total * 8);
    DevBuf<PlaceRec> d_recs;
    if (!recs.empty()) {
      d_recs.alloc(recs.size());
      upload(d_recs.p, recs, d_recs.n);
      k_place<<<((int)recs.size() + 255) / 256, 256, 0, st_>>>(d_recs.p, (int)recs.size(), nbox_.p, d_out.p);
    }
    DevBuf<uint32_t> d_dest;
    if (!subs_.empty()) {
      const int ns = (int)subs_.size();
      d_dest.alloc(ns);
      upload(d_dest.p, sub_dest, d_dest.n);
      k_set_dest<<<(ns + 255) / 256, 256, 0, st_>>>(small_.p, d_dest.p, ns);
      for (int level = 0; level < levels_; ++level) k_dests<<<148 * 8, 256, 0, st_>>>(small_.p, lv_.p, level);
      k_write_small<<<148 * 8, 256, 0, st_>>>(small_.p, counter_.p, (uint32_t)base_, d_out.p);
    }
    GB_TRY(cudaGetLastError());
    s_.roots.assign(n_roots, {});
    for (size_t r = 0; r < n_roots; ++r) {
      s_.roots[r].resize((size_t)size[r] * 32);
      GB_TRY(cudaMemcpyAsync(s_.roots[r].data(), d_out.p + (size_t)root_first[r] * 8, s_.roots[r].size(),
                             cudaMemcpyDeviceToHost, st_));
    }
    GB_TRY(cudaStreamSynchronize(st_));
  }
};

}  // namespace

void build_serialized_device(Serialized& s, const float* pos, uint64_t n_verts, int stride, const int64_t* groups,
                             int n_groups, int64_t range_start, int64_t range_count, int strategy, int max_depth,
                             int leaf, bool indirect, int device, void* stream) {
  std::vector<Range> ranges = prepare_build(s, n_verts, groups, n_groups, range_start, range_count, indirect);
  GB_TRY(cudaSetDevice(device));
  DeviceBuilder b(s, static_cast<cudaStream_t>(stream), strategy, max_depth, leaf);
  b.run(pos, n_verts, stride, ranges);
}

}  // namespace bvhc
