// Kernel launch interface shared by the C-ABI translation unit and the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bvhcuda.h"
#include "layout.h"

namespace bvhc {

// Device error word bits (set with atomicOr; read and cleared by bvhc_mesh_synchronize).
enum : unsigned int {
  kErrStackOverflow = 1u,  // a traversal needed more than kMaxStack entries
};

struct MeshDev {
  const PairNode* nodes;
  const TriRecord* tris;
  const uint32_t* roots;  // one link per root
  int n_roots;
  unsigned int* err;
};

cudaError_t launch_raycast_first(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                                 float near_d, float far_d, bvhc_hit* out, cudaStream_t stream);
cudaError_t launch_raycast_all(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                               float near_d, float far_d, uint32_t cap, uint32_t* counts, bvhc_hit* hits,
                               cudaStream_t stream);
cudaError_t launch_closest_point(const MeshDev& m, const float* pts, uint64_t n, float min_t, float max_t,
                                 bvhc_closest* out, cudaStream_t stream);

}  // namespace bvhc
