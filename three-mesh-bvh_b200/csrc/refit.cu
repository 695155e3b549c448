// Refit on the device (MeshBVH#refit, src/core/cast/refit.template.js:4-196, MeshBVH.js:504-508).
//
// After the vertex positions change, the triangle records take the new vertices and every box is
// rebuilt bottom-up.  One thread per leaf gathers its triangles' vertices (through the geometry
// index), writes them into the records and computes the leaf box as the min / max of the vertex
// coordinates (the reference's `<` / `>` updates from +-Infinity).  It then walks up: at each
// child-pair record it marks whether its side changed and counts its arrival; the first of the two
// children to arrive stops, the second (which now sees both children's final boxes) writes the
// pair's own box into the slot that holds it and continues upward.  No thread ever waits, so the
// walk ends after at most the tree depth.
//
// Change rule (force = false, the reference's): a leaf box is written and reported changed only
// when some bound differs from the stored one (`!==`); a pair's own box is recomputed as the union
// of its two child boxes only when a child changed, and is reported changed exactly then.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace bvhc {
namespace dev {

constexpr int kRefitBlock = 128;

__device__ __forceinline__ float* slot_box(PairNode* pairs, float* root_box, uint32_t slot) {
  if (slot & kRootSlot) return root_box + 6 * (slot & ~kRootSlot);
  return pairs[slot >> 1].f + 6 * (slot & 1u);
}

__global__ void __launch_bounds__(kRefitBlock) refit_kernel(RefitPlan plan, PairNode* __restrict__ pairs,
                                                            TriRecord* __restrict__ tris,
                                                            const uint32_t* __restrict__ tri_vid,
                                                            const float* __restrict__ pos, int stride, bool force) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= plan.n_leaves) return;
  const RefitLeaf leaf = plan.leaves[i];
  float lo[3] = {__builtin_huge_valf(), __builtin_huge_valf(), __builtin_huge_valf()};
  float hi[3] = {-__builtin_huge_valf(), -__builtin_huge_valf(), -__builtin_huge_valf()};
  for (uint32_t k = leaf.first; k < leaf.first + leaf.count; ++k) {
    TriRecord& r = tris[k];
    const uint64_t face = r.face;
    for (int v = 0; v < 3; ++v) {
      const float* p = pos + (uint64_t)__ldg(tri_vid + 3 * face + v) * stride;
      for (int a = 0; a < 3; ++a) {
        float x = __ldg(p + a);
        r.v[3 * v + a] = x;
        if (x < lo[a]) lo[a] = x;
        if (x > hi[a]) hi[a] = x;
      }
    }
  }
  float* box = slot_box(pairs, plan.root_box, leaf.slot);
  bool changed = force;
  for (int a = 0; a < 3; ++a) changed |= box[a] != lo[a] || box[3 + a] != hi[a];
  if (changed) {
    for (int a = 0; a < 3; ++a) {
      box[a] = lo[a];
      box[3 + a] = hi[a];
    }
  }
  uint32_t slot = leaf.slot;
  while (!(slot & kRootSlot)) {
    const uint32_t p = slot >> 1;
    if (changed) atomicOr(plan.flags + p, 1u << (slot & 1u));
    __threadfence();  // this side's box and flag before the arrival
    if (atomicAdd(plan.arrive + p, 1u) == 0u) return;  // the sibling finishes this pair
    __threadfence();
    changed = force || atomicOr(plan.flags + p, 0u) != 0u;
    slot = plan.parent[p];
    if (changed) {
      // both child boxes, read past L1 (the sibling may have written from another SM)
      const float* f = pairs[p].f;
      float* out = slot_box(pairs, plan.root_box, slot);
      for (int a = 0; a < 3; ++a) {
        float l0 = __ldcg(f + a), r0 = __ldcg(f + 6 + a);
        float l1 = __ldcg(f + 3 + a), r1 = __ldcg(f + 9 + a);
        out[a] = l0 < r0 ? l0 : r0;
        out[3 + a] = l1 > r1 ? l1 : r1;
      }
    }
  }
}

// Four-child records: each child box is copied from the child-pair slot it was collapsed from.
__global__ void __launch_bounds__(kRefitBlock) quad_boxes_kernel(QuadNode* __restrict__ quads, uint64_t n_quads,
                                                                 const uint32_t* __restrict__ src,
                                                                 const PairNode* __restrict__ pairs) {
  const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= 4 * n_quads) return;
  const uint32_t slot = __ldg(src + k);
  if (slot == kEmptyLeaf) return;
  const float* b = pairs[slot >> 1].f + 6 * (slot & 1u);
  QuadNode& q = quads[k >> 2];
  const int c = (int)(k & 3u);
  for (int a = 0; a < 3; ++a) {
    q.lo[a][c] = b[a];
    q.hi[a][c] = b[3 + a];
  }
}

}  // namespace dev

cudaError_t launch_quad_boxes(QuadNode* quads, uint64_t n_quads, const uint32_t* src, const PairNode* pairs,
                              cudaStream_t stream) {
  if (n_quads == 0) return cudaSuccess;
  const unsigned int grid = (unsigned int)((4 * n_quads + dev::kRefitBlock - 1) / dev::kRefitBlock);
  dev::quad_boxes_kernel<<<grid, dev::kRefitBlock, 0, stream>>>(quads, n_quads, src, pairs);
  return cudaGetLastError();
}

cudaError_t launch_refit(const RefitPlan& plan, PairNode* pairs, TriRecord* tris, const uint32_t* tri_vid,
                         const float* pos, int stride, bool force, cudaStream_t stream) {
  if (plan.n_leaves == 0) return cudaSuccess;
  cudaError_t e = cudaSuccess;
  if (plan.n_pairs) {
    e = cudaMemsetAsync(plan.arrive, 0, plan.n_pairs * sizeof(uint32_t), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(plan.flags, 0, plan.n_pairs * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
  }
  const unsigned int grid = (plan.n_leaves + dev::kRefitBlock - 1) / dev::kRefitBlock;
  dev::refit_kernel<<<grid, dev::kRefitBlock, 0, stream>>>(plan, pairs, tris, tri_vid, pos, stride, force);
  return cudaGetLastError();
}

}  // namespace bvhc
