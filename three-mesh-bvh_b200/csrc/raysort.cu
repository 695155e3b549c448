// Ray ordering for coherence: after the root-box pre-pass has queued the rays that can hit the
// mesh, each queued ray gets a 30-bit Morton key and the queue is sorted by it, so that the rays a
// warp takes together start near each other and point the same way.  The traversal kernels then
// walk the queue in sorted order; results are still written to each ray's own slot, so ordering
// changes speed only, never results.
//
// Keys (kind):
//   1  direction: the normalised direction, quantised to 10 bits per axis over the bounds of the
//      queued rays' directions (measured by a reduction pass), interleaved (3-D Morton).
//   2  scene entry point: where the ray enters the mesh's bounding box (its origin if it starts
//      inside), 10 bits per axis over that box, interleaved.
//   3  entry point (6 bits per axis, interleaved) followed by the direction (4 bits per axis over
//      [-1, 1], interleaved).
//
// The sort is a stable least-significant-digit radix sort of (key, ray id) pairs, 8-bit digits,
// four passes for 30-bit keys.  Each pass: an upsweep counts each tile's digits (4096 items per
// block), a scan turns the digit x tile counts into output offsets (digit-major), and a scatter
// ranks each item within its tile (warp match + per-warp counts in shared memory, in item order,
// so equal digits keep their order) and writes it to its offset.  The item count is the queue
// length, read on the device, so nothing waits on the host.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace bvhc {
namespace dev {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 items per block
constexpr int kSortWarps = kSortThreads / 32;

__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every third bit of 30
  x &= 0x3FFu;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// v in [lo, lo + 1 / inv_ext] -> 0 .. levels - 1 (clamped; NaN -> 0)
__device__ __forceinline__ uint32_t quantise(float v, float lo, float inv_ext, float levels) {
  float s = fminf(fmaxf((v - lo) * inv_ext, 0.0f), 1.0f);
  return (uint32_t)fminf(s * levels, levels - 1.0f);
}

// Monotone map of floats to unsigned integers (for atomicMin / atomicMax bounds).
__device__ __forceinline__ uint32_t float_order(float f) {
  uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float order_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__device__ __forceinline__ float3 load_dir_normalised(const float* rays, uint32_t i) {
  const float* r = rays + 6 * (uint64_t)i;
  float3 d = make_float3(__ldg(r + 3), __ldg(r + 4), __ldg(r + 5));
  float l = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  float il = l > 0.0f ? 1.0f / l : 0.0f;
  return make_float3(d.x * il, d.y * il, d.z * il);
}

// bounds[0..2] = min, bounds[3..5] = max of the queued rays' normalised directions (ordered ints;
// the caller sets the min slots to 0xFFFFFFFF and the max slots to 0 first).
__global__ void __launch_bounds__(kSortThreads) dir_bounds_kernel(const float* __restrict__ rays,
                                                                  const uint32_t* __restrict__ queue,
                                                                  const unsigned int* __restrict__ qcount,
                                                                  uint32_t* __restrict__ bounds) {
  const uint32_t n = __ldg(qcount);
  float lo[3] = {__builtin_huge_valf(), __builtin_huge_valf(), __builtin_huge_valf()};
  float hi[3] = {-__builtin_huge_valf(), -__builtin_huge_valf(), -__builtin_huge_valf()};
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    float3 d = load_dir_normalised(rays, __ldg(queue + k));
    lo[0] = fminf(lo[0], d.x); lo[1] = fminf(lo[1], d.y); lo[2] = fminf(lo[2], d.z);
    hi[0] = fmaxf(hi[0], d.x); hi[1] = fmaxf(hi[1], d.y); hi[2] = fmaxf(hi[2], d.z);
  }
  for (int a = 0; a < 3; ++a) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[a] = fminf(lo[a], __shfl_xor_sync(0xFFFFFFFFu, lo[a], o));
      hi[a] = fmaxf(hi[a], __shfl_xor_sync(0xFFFFFFFFu, hi[a], o));
    }
  }
  if ((threadIdx.x & 31u) == 0 && lo[0] <= hi[0]) {
    for (int a = 0; a < 3; ++a) {
      atomicMin(bounds + a, float_order(lo[a]));
      atomicMax(bounds + 3 + a, float_order(hi[a]));
    }
  }
}

__global__ void __launch_bounds__(kSortThreads) ray_key_kernel(const float* __restrict__ rays,
                                                               const uint32_t* __restrict__ queue,
                                                               const unsigned int* __restrict__ qcount, int kind,
                                                               float3 scene_lo, float3 scene_hi,
                                                               const uint32_t* __restrict__ dir_bounds,
                                                               uint32_t* __restrict__ keys) {
  const uint32_t n = __ldg(qcount);
  float3 dlo = make_float3(-1.0f, -1.0f, -1.0f), dinv = make_float3(0.5f, 0.5f, 0.5f);
  if (kind == 1) {
    float l0 = order_float(__ldg(dir_bounds)), l1 = order_float(__ldg(dir_bounds + 1));
    float l2 = order_float(__ldg(dir_bounds + 2));
    float h0 = order_float(__ldg(dir_bounds + 3)), h1 = order_float(__ldg(dir_bounds + 4));
    float h2 = order_float(__ldg(dir_bounds + 5));
    dlo = make_float3(l0, l1, l2);
    dinv = make_float3(h0 > l0 ? 1.0f / (h0 - l0) : 0.0f, h1 > l1 ? 1.0f / (h1 - l1) : 0.0f,
                       h2 > l2 ? 1.0f / (h2 - l2) : 0.0f);
  }
  float3 sinv = make_float3(scene_hi.x > scene_lo.x ? 1.0f / (scene_hi.x - scene_lo.x) : 0.0f,
                            scene_hi.y > scene_lo.y ? 1.0f / (scene_hi.y - scene_lo.y) : 0.0f,
                            scene_hi.z > scene_lo.z ? 1.0f / (scene_hi.z - scene_lo.z) : 0.0f);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    uint32_t i = __ldg(queue + k);
    const float* r = rays + 6 * (uint64_t)i;
    float3 o = make_float3(__ldg(r), __ldg(r + 1), __ldg(r + 2));
    float3 d = load_dir_normalised(rays, i);
    uint32_t key;
    if (kind == 1) {
      key = morton3(quantise(d.x, dlo.x, dinv.x, 1024.0f), quantise(d.y, dlo.y, dinv.y, 1024.0f),
                    quantise(d.z, dlo.z, dinv.z, 1024.0f));
    } else {
      // entry into the scene box: max over axes of the near slab distance, not before the origin
      float ix = d.x != 0.0f ? 1.0f / d.x : 1e30f, iy = d.y != 0.0f ? 1.0f / d.y : 1e30f;
      float iz = d.z != 0.0f ? 1.0f / d.z : 1e30f;
      float tx = fminf((scene_lo.x - o.x) * ix, (scene_hi.x - o.x) * ix);
      float ty = fminf((scene_lo.y - o.y) * iy, (scene_hi.y - o.y) * iy);
      float tz = fminf((scene_lo.z - o.z) * iz, (scene_hi.z - o.z) * iz);
      float t = fmaxf(fmaxf(fmaxf(tx, ty), tz), 0.0f);
      float3 p = make_float3(o.x + d.x * t, o.y + d.y * t, o.z + d.z * t);
      if (kind == 2) {
        key = morton3(quantise(p.x, scene_lo.x, sinv.x, 1024.0f), quantise(p.y, scene_lo.y, sinv.y, 1024.0f),
                      quantise(p.z, scene_lo.z, sinv.z, 1024.0f));
      } else {
        uint32_t kp = morton3(quantise(p.x, scene_lo.x, sinv.x, 64.0f), quantise(p.y, scene_lo.y, sinv.y, 64.0f),
                              quantise(p.z, scene_lo.z, sinv.z, 64.0f));
        uint32_t kd = morton3(quantise(d.x, -1.0f, 0.5f, 16.0f), quantise(d.y, -1.0f, 0.5f, 16.0f),
                              quantise(d.z, -1.0f, 0.5f, 16.0f));
        key = (kp << 12) | kd;
      }
    }
    keys[k] = key;
  }
}

// Upsweep: hist[digit * nblocks + block] = count of `digit` in the block's tile; totals[digit] += it.
__global__ void __launch_bounds__(kSortThreads) radix_upsweep_kernel(const uint32_t* __restrict__ keys,
                                                                     const unsigned int* __restrict__ count, int shift,
                                                                     uint32_t nblocks, uint32_t* __restrict__ hist,
                                                                     uint32_t* __restrict__ totals) {
  __shared__ uint32_t h[256];
  const unsigned lane = threadIdx.x & 31u;
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t n = __ldg(count);
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  if (base < n) {
    for (int j = 0; j < kSortItems; ++j) {
      uint64_t idx = base + (uint64_t)j * kSortThreads + threadIdx.x;
      bool valid = idx < n;
      uint32_t dgt = valid ? (__ldg(keys + idx) >> shift) & 255u : 256u + lane;
      unsigned peers = __match_any_sync(0xFFFFFFFFu, dgt);
      if (valid && (peers & ((1u << lane) - 1u)) == 0u) atomicAdd(&h[dgt], (uint32_t)__popc(peers));
    }
  }
  __syncthreads();
  uint32_t c = h[threadIdx.x];
  hist[(uint64_t)threadIdx.x * nblocks + blockIdx.x] = c;
  if (c) atomicAdd(totals + threadIdx.x, c);
}

// Scan: block `digit` turns its row of tile counts into output offsets:
// offset(digit, b) = sum of totals of smaller digits + sum of the row's counts before b.
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) radix_scan_kernel(uint32_t* __restrict__ hist,
                                                                  const uint32_t* __restrict__ totals,
                                                                  uint32_t nblocks) {
  __shared__ uint32_t s_warp[kScanThreads / 32];
  __shared__ uint32_t s_base;
  const uint32_t digit = blockIdx.x;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  if (w == 0) {
    uint32_t s = 0;
    for (uint32_t k = lane; k < digit; k += 32) s += __ldg(totals + k);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    if (lane == 0) s_base = s;
  }
  uint32_t* row = hist + (uint64_t)digit * nblocks;
  const uint32_t per = (nblocks + kScanThreads - 1) / kScanThreads;
  const uint32_t start = threadIdx.x * per;
  const uint32_t end = start + per < nblocks ? start + per : nblocks;
  uint32_t local = 0;
  for (uint32_t b = start; b < end; ++b) local += row[b];
  // block exclusive scan of the per-thread sums
  uint32_t incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  if (lane == 31) s_warp[w] = incl;
  __syncthreads();
  if (w == 0) {
    uint32_t v = s_warp[lane];
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
      if (lane >= (unsigned)o) v += y;
    }
    s_warp[lane] = v;  // inclusive prefix of warp sums
  }
  __syncthreads();
  uint32_t run = s_base + (w > 0 ? s_warp[w - 1] : 0u) + incl - local;
  for (uint32_t b = start; b < end; ++b) {
    uint32_t c = row[b];
    row[b] = run;
    run += c;
  }
}

// Scatter: stable rank of each item within its tile, written to its digit's offset.
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, const unsigned int* __restrict__ count, int shift, uint32_t nblocks,
    const uint32_t* __restrict__ offsets) {
  __shared__ uint32_t run[256];
  __shared__ uint32_t wcnt[kSortWarps][256];
  const uint32_t n = __ldg(count);
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  if (base >= n) return;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  run[threadIdx.x] = __ldg(offsets + (uint64_t)threadIdx.x * nblocks + blockIdx.x);
  for (int j = 0; j < kSortItems; ++j) {
    for (int k = threadIdx.x; k < kSortWarps * 256; k += kSortThreads) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    uint64_t idx = base + (uint64_t)j * kSortThreads + threadIdx.x;
    bool valid = idx < n;
    uint32_t key = valid ? kin[idx] : 0u, val = valid ? vin[idx] : 0u;
    uint32_t dgt = valid ? (key >> shift) & 255u : 256u + lane;
    unsigned peers = __match_any_sync(0xFFFFFFFFu, dgt);
    uint32_t rank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[w][dgt] = (uint32_t)__popc(peers);
    __syncthreads();
    {  // per digit: exclusive prefix over the warps, continuing the tile's running offset
      uint32_t s = run[threadIdx.x];
      for (int ww = 0; ww < kSortWarps; ++ww) {
        uint32_t c = wcnt[ww][threadIdx.x];
        wcnt[ww][threadIdx.x] = s;
        s += c;
      }
      run[threadIdx.x] = s;
    }
    __syncthreads();
    if (valid) {
      uint32_t pos = wcnt[w][dgt] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
  }
}

}  // namespace dev

uint64_t ray_sort_tiles(uint64_t n) { return (n + dev::kSortTile - 1) / dev::kSortTile; }

cudaError_t launch_ray_sort(const float* rays, uint64_t n, int kind, const float scene_lo[3], const float scene_hi[3],
                            uint32_t* queue, const unsigned int* qcount, const RaySortScratch& s,
                            cudaStream_t stream) {
  if (n == 0 || kind < 1 || kind > 3) return cudaSuccess;
  const uint32_t nblocks = (uint32_t)ray_sort_tiles(n);
  // grid-stride passes over the queue: enough blocks to fill the GPU, no more than the items need
  const unsigned int gs = (unsigned int)(nblocks * (uint64_t)dev::kSortItems < 4096 ? nblocks * dev::kSortItems : 4096);
  cudaError_t e;
  if (kind == 1) {
    e = cudaMemsetAsync(s.dir_bounds, 0xFF, 3 * sizeof(uint32_t), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.dir_bounds + 3, 0, 3 * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    dev::dir_bounds_kernel<<<gs, dev::kSortThreads, 0, stream>>>(rays, queue, qcount, s.dir_bounds);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  dev::ray_key_kernel<<<gs, dev::kSortThreads, 0, stream>>>(
      rays, queue, qcount, kind, make_float3(scene_lo[0], scene_lo[1], scene_lo[2]),
      make_float3(scene_hi[0], scene_hi[1], scene_hi[2]), s.dir_bounds, s.keys[0]);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  e = cudaMemsetAsync(s.totals, 0, 4 * 256 * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  uint32_t* kbuf[2] = {s.keys[0], s.keys[1]};
  uint32_t* vbuf[2] = {queue, s.vals};
  for (int pass = 0; pass < 4; ++pass) {
    const int src = pass & 1, dst = src ^ 1;
    uint32_t* totals = s.totals + 256 * pass;
    dev::radix_upsweep_kernel<<<nblocks, dev::kSortThreads, 0, stream>>>(kbuf[src], qcount, 8 * pass, nblocks,
                                                                         s.hist, totals);
    dev::radix_scan_kernel<<<256, dev::kScanThreads, 0, stream>>>(s.hist, totals, nblocks);
    dev::radix_scatter_kernel<<<nblocks, dev::kSortThreads, 0, stream>>>(kbuf[src], vbuf[src], kbuf[dst], vbuf[dst],
                                                                          qcount, 8 * pass, nblocks, s.hist);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;  // four passes: the sorted ids are back in `queue`
}

}  // namespace bvhc
