// raycastFirst autotuner inside the library (no reference counterpart: the reference has one
// recursive traversal).  It times the traversal variants with CUDA events on the caller's stream,
// so a host without any GPU framework (the N-API addon) tunes a mesh with one call.
//
// Stage 1 times every candidate of the list below on each ray set, for each device leaf layout
// asked for; the layout with the smallest sum of the sets' best times is kept.  Stage 2 refines
// each set's best warp-cooperative or persistent candidate on that layout: threads per block (64,
// 128, 256; warp-cooperative form), the tile height of a tiled order (2, 4, 8 rows), the refill
// threshold (8, 24; persistent form), and the 32-entry traversal stack (when the tree is shallow
// enough).  Every variant returns the same hits (up to exact ties), so tuning changes speed only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "bvhcuda.h"

namespace {

bvhc_traversal_config make(int persistent, int order, int refill, int occupancy, int compact, int sort, int wide,
                           int tile) {
  bvhc_traversal_config c{};
  c.persistent = persistent;
  c.order = order;
  c.refill = refill;
  c.occupancy = occupancy;
  c.compact = compact;
  c.sort = sort;
  c.wide = wide;
  c.tile = tile;
  return c;
}

// Stage-1 candidates: one ray per thread (both child orders); warp-cooperative over child pairs
// (child order x register budget x queue) and over four-child records; persistent warps (child
// order x refill threshold x register budget x queue) and over four-child records (refill
// threshold x register budget x compaction); warp-cooperative in tiled ray order over
// child pairs (child order x register budget) and over four-child records (register budget), for
// each row pitch given.  Queue: none, compaction, compaction + ordering key 1, 2, 3.
std::vector<bvhc_traversal_config> stage1(const int32_t* tiles, int n_tiles) {
  static const int kQueue[5][2] = {{0, 0}, {1, 0}, {1, 1}, {1, 2}, {1, 3}};
  std::vector<bvhc_traversal_config> c;
  c.push_back(make(0, 0, 16, 0, 0, 0, 0, 0));
  c.push_back(make(0, 1, 16, 0, 0, 0, 0, 0));
  for (int order = 0; order < 2; ++order)
    for (int occ = 0; occ < 3; ++occ)
      for (const auto& q : kQueue) c.push_back(make(2, order, 16, occ, q[0], q[1], 0, 0));
  for (int occ = 0; occ < 3; ++occ)
    for (const auto& q : kQueue) c.push_back(make(2, 1, 16, occ, q[0], q[1], 1, 0));
  for (int order = 0; order < 2; ++order)
    for (int refill : {16, 32})
      for (int occ = 1; occ < 3; ++occ)
        for (const auto& q : kQueue) c.push_back(make(1, order, refill, occ, q[0], q[1], 0, 0));
  // persistent over four-child records (nearest child first), without a queue or with compaction
  for (int refill : {16, 32})
    for (int occ = 1; occ < 3; ++occ)
      for (int compact = 0; compact < 2; ++compact) c.push_back(make(1, 1, refill, occ, compact, 0, 1, 0));
  for (int k = 0; k < n_tiles; ++k) {
    for (int order = 0; order < 2; ++order)
      for (int occ = 0; occ < 3; ++occ) c.push_back(make(2, order, 16, occ, 0, 0, 0, tiles[k]));
    for (int occ = 0; occ < 3; ++occ) c.push_back(make(2, 1, 16, occ, 0, 0, 1, tiles[k]));  // four-child records
  }
  return c;
}

// A tiled-order row pitch bvhc_mesh_set_traversal accepts: a multiple of 8 in [8, 2^24].
bool valid_pitch(int32_t p) { return p >= 8 && p % 8 == 0 && p <= (1 << 24); }

struct Timer {
  cudaEvent_t a = nullptr, b = nullptr;
  ~Timer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

bvhc_status cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return BVHC_OK;
  return e == cudaErrorMemoryAllocation ? BVHC_ERR_OUT_OF_MEMORY : BVHC_ERR_CUDA;
}

// Mean time of `reps` calls after one warm-up call (which also grows the variant's scratch).
bvhc_status time_variant(bvhc_mesh* mesh, const bvhc_traversal_config& cfg, const float* rays, uint64_t n, int side,
                         float near_d, float far_d, bvhc_hit* out, int reps, cudaStream_t s, Timer& t, float* ms) {
  bvhc_status st = bvhc_mesh_set_traversal(mesh, &cfg);
  if (st != BVHC_OK) return st;
  st = bvhc_raycast_first(mesh, rays, n, side, near_d, far_d, out, BVHC_MEM_DEVICE, s);
  if (st != BVHC_OK) return st;
  cudaError_t e = cudaEventRecord(t.a, s);
  for (int r = 0; r < reps && e == cudaSuccess && st == BVHC_OK; ++r)
    st = bvhc_raycast_first(mesh, rays, n, side, near_d, far_d, out, BVHC_MEM_DEVICE, s);
  if (st != BVHC_OK) return st;
  if (e == cudaSuccess) e = cudaEventRecord(t.b, s);
  if (e == cudaSuccess) e = cudaEventSynchronize(t.b);
  float total = 0.0f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&total, t.a, t.b);
  if (e != cudaSuccess) return cuda_status(e);
  st = bvhc_mesh_synchronize(mesh, s);
  *ms = total / (float)reps;
  return st;
}

}  // namespace

extern "C" bvhc_status bvhc_mesh_autotune(bvhc_mesh* mesh, int n_sets, const float* const* rays,
                                          const uint64_t* counts, int side, float near_dist, float far_dist,
                                          const int32_t* leaf_sizes, int n_leaf_sizes, const int32_t* tile_pitches,
                                          int n_tile_pitches, int reps, void* stream, bvhc_traversal_config* best,
                                          float* best_ms, int32_t* leaf_size_out, float* leaf_total_ms) {
  if (!mesh || n_sets < 1 || !rays || !counts || !best || n_leaf_sizes < 0 || n_tile_pitches < 0 ||
      (n_leaf_sizes > 0 && !leaf_sizes) || (n_tile_pitches > 0 && !tile_pitches) || reps < 1 ||
      side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE)
    return BVHC_ERR_INVALID_ARGUMENT;
  uint64_t n_max = 0;
  for (int k = 0; k < n_sets; ++k) {
    if (!rays[k] || counts[k] == 0) return BVHC_ERR_INVALID_ARGUMENT;
    n_max = std::max(n_max, counts[k]);
  }
  for (int k = 0; k < n_tile_pitches; ++k)
    if (!valid_pitch(tile_pitches[k])) return BVHC_ERR_INVALID_ARGUMENT;
  const int current_leaf = bvhc_mesh_get_leaf_size(mesh);
  std::vector<int32_t> leaves(leaf_sizes, leaf_sizes + n_leaf_sizes);
  if (leaves.empty()) leaves.push_back(current_leaf);
  const std::vector<bvhc_traversal_config> cands = stage1(tile_pitches, n_tile_pitches);
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  bvhc_hit* out = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&out), n_max * sizeof(bvhc_hit));
  if (e != cudaSuccess) return cuda_status(e);
  Timer t;
  e = cudaEventCreate(&t.a);
  if (e == cudaSuccess) e = cudaEventCreate(&t.b);
  bvhc_status st = cuda_status(e);

  std::vector<bvhc_traversal_config> set_best(n_sets), chosen(n_sets);
  std::vector<float> set_ms(n_sets), chosen_ms(n_sets);
  float best_total = 0.0f;
  int best_leaf = -1;
  for (size_t li = 0; li < leaves.size() && st == BVHC_OK; ++li) {
    st = bvhc_mesh_set_leaf_size(mesh, leaves[li]);
    float total = 0.0f;
    for (int k = 0; k < n_sets && st == BVHC_OK; ++k) {
      set_ms[k] = -1.0f;
      for (const auto& c : cands) {
        float ms = 0.0f;
        st = time_variant(mesh, c, rays[k], counts[k], side, near_dist, far_dist, out, reps, s, t, &ms);
        if (st != BVHC_OK) break;
        if (set_ms[k] < 0.0f || ms < set_ms[k]) {
          set_ms[k] = ms;
          set_best[k] = c;
        }
      }
      total += set_ms[k];
    }
    if (st != BVHC_OK) break;
    if (leaf_total_ms) leaf_total_ms[li] = total;
    if (best_leaf < 0 || total < best_total) {
      best_total = total;
      best_leaf = leaves[li];
      chosen = set_best;
      chosen_ms = set_ms;
    }
  }
  if (st == BVHC_OK) st = bvhc_mesh_set_leaf_size(mesh, best_leaf);
  // stage 2: block size and stack depth around each set's best
  for (int k = 0; k < n_sets && st == BVHC_OK; ++k) {
    const bvhc_traversal_config base = chosen[k];
    if (base.persistent == 0 || (base.persistent == 2 && base.wide && !base.tile)) continue;
    std::vector<bvhc_traversal_config> more{base};
    if (base.persistent == 1)
      for (int refill : {8, 24})  // the refill thresholds between and below stage 1's 16 and 32
        if (refill != base.refill) {
          bvhc_traversal_config c = base;
          c.refill = refill;
          more.push_back(c);
        }
    if (base.persistent == 2) {
      for (int block : {64, 256}) {
        if (base.wide) break;  // the four-child kernel has one block size
        bvhc_traversal_config c = base;
        c.block = block;
        more.push_back(c);
      }
      // a tiled order's other tile heights (2 x 16, 8 x 4) where the row pitch allows them
      for (int rows : {2, 8})
        if (base.tile && base.tile % (32 / rows) == 0) {
          bvhc_traversal_config c = base;
          c.tile_rows = rows;
          more.push_back(c);
        }
    }
    float ref_ms = 0.0f;
    for (size_t j = 0; j < more.size() && st == BVHC_OK; ++j) {
      float ms = 0.0f;
      st = time_variant(mesh, more[j], rays[k], counts[k], side, near_dist, far_dist, out, reps, s, t, &ms);
      if (st != BVHC_OK) break;
      if (j == 0 || ms < ref_ms) {
        ref_ms = ms;
        chosen[k] = more[j];
      }
    }
    if (st != BVHC_OK) break;
    if (!chosen[k].wide) {  // the four-child kernels have one stack size
      bvhc_traversal_config shallow = chosen[k];
      shallow.stack = 32;
      float ms = 0.0f;
      st = time_variant(mesh, shallow, rays[k], counts[k], side, near_dist, far_dist, out, reps, s, t, &ms);
      if (st == BVHC_OK && ms < ref_ms) {
        ref_ms = ms;
        chosen[k] = shallow;
      }
    }
    chosen_ms[k] = ref_ms;
  }
  cudaError_t fe = cudaFree(out);
  if (st == BVHC_OK && fe != cudaSuccess) st = cuda_status(fe);
  if (st != BVHC_OK) return st;
  for (int k = 0; k < n_sets; ++k) {
    best[k] = chosen[k];
    if (best_ms) best_ms[k] = chosen_ms[k];
  }
  if (leaf_size_out) *leaf_size_out = best_leaf;
  return bvhc_mesh_set_traversal(mesh, &chosen[0]);
}

extern "C" int bvhc_autotune_candidates(const int32_t* tile_pitches, int n_tile_pitches, bvhc_traversal_config* out,
                                        int cap) {
  if (n_tile_pitches < 0 || (n_tile_pitches > 0 && !tile_pitches) || cap < 0 || (cap > 0 && !out)) return -1;
  for (int k = 0; k < n_tile_pitches; ++k)
    if (!valid_pitch(tile_pitches[k])) return -1;
  const std::vector<bvhc_traversal_config> c = stage1(tile_pitches, n_tile_pitches);
  for (int i = 0; i < (int)c.size() && i < cap; ++i) out[i] = c[i];
  return (int)c.size();
}
