// Internal declarations shared by the host-side translation units of libbvhcuda.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <vector>

#include "bvhcuda.h"

struct bvhc_serialized {
  // MeshBVH.serialize() result (src/core/MeshBVH.js:112-145): version 1 roots, index, indirect.
  std::vector<std::vector<uint8_t>> roots;
  bool has_index = false;
  int index_elem_bytes = 0;
  std::vector<uint32_t> index;       // widened to u32; narrowed to index_elem_bytes on export
  bool indirect = false;
  int indirect_elem_bytes = 0;
  std::vector<uint32_t> indirect_buf;
  // export copies at the serialized element width
  std::vector<uint8_t> index_bytes, indirect_bytes;
};

namespace bvhc {

using Serialized = bvhc_serialized;

enum { kCenter = 0, kAverage = 1, kSah = 2 };

struct Range {
  int64_t offset, count;
};

std::vector<Range> root_ranges(int64_t vertex_count, int64_t draw_start, int64_t draw_count, const int64_t* groups,
                               int n_groups);

// generateIndirectBuffer / ensureIndex (GeometryBVH.js:9-37, geometryUtils.js:15-47) on `s`, and
// the root primitive ranges to build over.
std::vector<Range> prepare_build(Serialized& s, uint64_t n_verts, const int64_t* groups, int n_groups,
                                 int64_t range_start, int64_t range_count, bool indirect);

void build_serialized(Serialized& s, const float* pos, uint64_t n_verts, int stride, const int64_t* groups,
                      int n_groups, int64_t range_start, int64_t range_count, int strategy, int max_depth,
                      int leaf, bool indirect);

// A CUDA runtime failure inside the device build.
struct DeviceBuildError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// The same build on a GPU (gpubuild.cu), byte-identical output; SAH and CENTER only.
void build_serialized_device(Serialized& s, const float* pos, uint64_t n_verts, int stride, const int64_t* groups,
                             int n_groups, int64_t range_start, int64_t range_count, int strategy, int max_depth,
                             int leaf, bool indirect, int device, void* stream);

}  // namespace bvhc
