// Ray ordering for coherence: the root-box pre-pass (classify_kernel) queues the rays that can hit
// the mesh together with a Morton key (raykey.cuh), and this file sorts the queue by that
// key, so that the rays a warp takes together start near each other and point the same way.  The
// traversal kernels then walk the queue in sorted order; results are still written to each ray's
// own slot, so ordering changes speed only, never results.
//
// The sort is a stable least-significant-digit radix sort of (key, ray id) pairs: one pass per
// 8-bit digit of the key kind's width.  Each pass:
//   upsweep  counts each tile's digits (4096 items per block) into a digit x tile matrix;
//   scan     turns the matrix into output offsets (digit-major: all of digit 0, then digit 1, ...);
//   scatter  ranks each item within its tile (warp match + per-warp counts in shared memory, in
//            item order, so equal digits keep their order), stages the tile in shared memory
//            grouped by digit, and writes each digit's run to its offset with consecutive threads
//            on consecutive addresses.
// The item count is the queue length, read on the device, so nothing waits on the host.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "raykey.cuh"

namespace bvhc {
namespace dev {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 items per block
constexpr int kSortWarps = kSortThreads / 32;

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
#pragma unroll 4
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
    s_warp[lane] = v;  // inclusive prefix of the warp sums
  }
  __syncthreads();
  uint32_t run = s_base + (w > 0 ? s_warp[w - 1] : 0u) + incl - local;
  for (uint32_t b = start; b < end; ++b) {
    uint32_t c = row[b];
    row[b] = run;
    run += c;
  }
}

// Scatter: stable rank within the tile, staging grouped by digit, coalesced runs to the offsets.
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(
    const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* __restrict__ kout,
    uint32_t* __restrict__ vout, const unsigned int* __restrict__ count, int shift, uint32_t nblocks,
    const uint32_t* __restrict__ offsets) {
  __shared__ uint32_t s_key[kSortTile];
  __shared__ uint32_t s_val[kSortTile];
  __shared__ uint32_t wcnt[kSortWarps][256];
  __shared__ uint32_t run[256];     // tile count of each digit, then its first slot in the tile
  __shared__ uint32_t goff[256];    // global offset of the digit's run minus its first tile slot
  __shared__ uint32_t s_wsum[kSortWarps];
  const uint32_t n = __ldg(count);
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  if (base >= n) return;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  run[threadIdx.x] = 0;
  uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    for (int k = threadIdx.x; k < kSortWarps * 256; k += kSortThreads) (&wcnt[0][0])[k] = 0;
    __syncthreads();
    uint64_t idx = base + (uint64_t)j * kSortThreads + threadIdx.x;
    bool valid = idx < n;
    key[j] = valid ? kin[idx] : 0u;
    val[j] = valid ? vin[idx] : 0u;
    uint32_t dgt = valid ? (key[j] >> shift) & 255u : 256u + lane;
    unsigned peers = __match_any_sync(0xFFFFFFFFu, dgt);
    uint32_t r = (uint32_t)__popc(peers & lt);
    if (valid && r == 0) wcnt[w][dgt] = (uint32_t)__popc(peers);
    __syncthreads();
    {  // per digit: exclusive prefix over the warps, continuing the tile's running count
      uint32_t s = run[threadIdx.x];
      for (int ww = 0; ww < kSortWarps; ++ww) {
        uint32_t c = wcnt[ww][threadIdx.x];
        wcnt[ww][threadIdx.x] = s;
        s += c;
      }
      run[threadIdx.x] = s;
    }
    __syncthreads();
    rank[j] = valid ? wcnt[w][dgt] + r : 0u;
    __syncthreads();  // every rank read before the next round clears the counts
  }
  // first tile slot of each digit: exclusive scan of the tile's digit counts
  uint32_t c = run[threadIdx.x];
  uint32_t incl = c;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= (unsigned)o) incl += y;
  }
  if (lane == 31) s_wsum[w] = incl;
  __syncthreads();
  uint32_t before = 0;
  for (unsigned ww = 0; ww < w; ++ww) before += s_wsum[ww];
  uint32_t first = before + incl - c;
  run[threadIdx.x] = first;
  goff[threadIdx.x] = __ldg(offsets + (uint64_t)threadIdx.x * nblocks + blockIdx.x) - first;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    uint64_t idx = base + (uint64_t)j * kSortThreads + threadIdx.x;
    if (idx < n) {
      uint32_t slot = run[(key[j] >> shift) & 255u] + rank[j];
      s_key[slot] = key[j];
      s_val[slot] = val[j];
    }
  }
  __syncthreads();
  const uint32_t cnt = n - base < (uint64_t)kSortTile ? (uint32_t)(n - base) : (uint32_t)kSortTile;
#pragma unroll
  for (int j = 0; j < kSortItems; ++j) {
    uint32_t slot = (uint32_t)j * kSortThreads + threadIdx.x;
    if (slot < cnt) {
      uint32_t k = s_key[slot];
      uint32_t pos = goff[(k >> shift) & 255u] + slot;
      kout[pos] = k;
      vout[pos] = s_val[slot];
    }
  }
}

}  // namespace dev

uint64_t ray_sort_tiles(uint64_t n) { return (n + dev::kSortTile - 1) / dev::kSortTile; }

void ray_sort_input(int kind, const RaySortScratch& s, uint32_t* queue, uint32_t** ids, uint32_t** keys) {
  const bool odd = ray_sort_passes(kind) & 1;
  *ids = odd ? s.vals : queue;
  *keys = odd ? s.keys[1] : s.keys[0];
}

cudaError_t launch_ray_sort(int kind, uint64_t n, const unsigned int* qcount, const RaySortScratch& s,
                            uint32_t* queue, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  const uint32_t nblocks = (uint32_t)ray_sort_tiles(n);
  const int passes = ray_sort_passes(kind);
  cudaError_t e = cudaMemsetAsync(s.totals, 0, passes * 256 * sizeof(uint32_t), stream);
  if (e != cudaSuccess) return e;
  // the pre-pass wrote the pairs where ray_sort_input put them, so the last pass ends in
  // (keys, queue)
  uint32_t *ids0, *keys0;
  ray_sort_input(kind, s, queue, &ids0, &keys0);
  uint32_t* kbuf[2] = {keys0, keys0 == s.keys[0] ? s.keys[1] : s.keys[0]};
  uint32_t* vbuf[2] = {ids0, ids0 == queue ? s.vals : queue};
  for (int pass = 0; pass < passes; ++pass) {
    const int src = pass & 1, dst = src ^ 1;
    uint32_t* totals = s.totals + 256 * pass;
    dev::radix_upsweep_kernel<<<nblocks, dev::kSortThreads, 0, stream>>>(kbuf[src], qcount, 8 * pass, nblocks,
                                                                         s.hist, totals);
    dev::radix_scan_kernel<<<256, dev::kScanThreads, 0, stream>>>(s.hist, totals, nblocks);
    dev::radix_scatter_kernel<<<nblocks, dev::kSortThreads, 0, stream>>>(kbuf[src], vbuf[src], kbuf[dst], vbuf[dst],
                                                                          qcount, 8 * pass, nblocks, s.hist);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace bvhc
