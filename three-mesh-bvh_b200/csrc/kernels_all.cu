// raycast (all hits) kernels: one ray per thread, persistent warps over the pre-pass queue, and
// the warp-cooperative form; and their launch.
#include <algorithm>

#include "traverse.cuh"

namespace bvhc {
namespace dev {

// ---------------------------------------------------------------------------------------------
// raycast, all hits (raycast.template.js:15-53): left child then right child, every hit kept
// in DFS order.  The first `cap` hits are stored; counts[i] is the uncapped total.  The traversal
// kernels decide each hit and its near / far range exactly (float32 with error bounds, float-float
// where those do not settle it, as raycastFirst does) and leave the stored hit pending: its
// triangle record in face_index.  raycast_all_finalize_kernel then computes the reported records
// (t, distance, point, barycentrics in float-float) one ray per thread, which keeps that code out
// of the traversal loops (the camera set: 11.2 -> 6.9 ms of traversal).
// ---------------------------------------------------------------------------------------------

// One ray per thread: all n rays, or with a queue the queued ones (the rays that enter the tree, so
// that a warp's lanes mostly have hits to complete).
__global__ void __launch_bounds__(kBlock) raycast_all_finalize_kernel(MeshDev m, const float* __restrict__ rays,
                                                                      uint64_t n, uint32_t cap,
                                                                      const uint32_t* __restrict__ counts,
                                                                      bvhc_hit* __restrict__ hits,
                                                                      const uint32_t* __restrict__ queue,
                                                                      const unsigned int* __restrict__ qcount) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (queue) {
    if (i >= (uint64_t)__ldg(qcount)) return;
    i = __ldg(queue + i);
  }
  if (i >= n) return;
  const uint32_t c = min(__ldg(counts + i), cap);
  if (c == 0) return;
  const RayF r = make_ray(rays, i);
  const ff dlen = dir_length(r.d);
  bvhc_hit* out = hits + i * (uint64_t)cap;
  for (uint32_t k = 0; k < c; ++k) {
    const Tri t = load_tri(m.tris, out[k].face_index);
    const TriFF e = tri_eval_ff(t.a, t.b, t.c, r.o, r.d);
    const ff tt = tri_t_ff(e);
    bvhc_hit h;
    make_hit(t, r, e, tt, ff_mul(tt, dlen), h);
    store_hit(out + k, h);
  }
}

__global__ void __launch_bounds__(kBlock) raycast_all_kernel(MeshDev m, const float* __restrict__ rays, uint64_t n,
                                                             int side, const SideTable sides, float near_d,
                                                             float far_d, uint32_t cap, uint32_t* __restrict__ counts,
                                                             bvhc_hit* __restrict__ hits,
                                                             const uint32_t* __restrict__ queue = nullptr,
                                                             const unsigned int* __restrict__ qcount = nullptr) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // with a queue, thread i traces ray queue[i] (the rays the pre-pass found entering the tree)
  if (queue) {
    if (i >= (uint64_t)__ldg(qcount)) return;
    i = __ldg(queue + i);
  }
  if (i >= n) return;
  RayF r = make_ray(rays, i);
  const float dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  uint32_t cnt = 0;
  uint32_t stack_link[kMaxStack];
  bvhc_hit* out = hits + i * (uint64_t)cap;
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      if (link & kLeafBit) {
        if (link != kEmptyLeaf) {
          uint32_t k = link & ~kLeafBit;
          for (;;) {
            Tri t = load_tri(m.tris, k);
            int ts = tri_side(t, side, sides);
            float th, te;
            if (ts >= 0 && tri_hit_t(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts, th, te) &&
                in_range(th, te, t, r, dlen, near_d, far_d)) {
              if (cnt < cap) store_pending_record(out + cnt, k, 0.0f);
              ++cnt;
            }
            if (t.flags & kTriLast) break;
            ++k;
          }
        }
      } else {
        Pair p = load_pair(m.nodes, link);
        float e0, e1;
        bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e0);
        bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e1);
        if (h0) {
          if (h1) {
            if (sp >= kMaxStack) {
              atomicOr(m.err, kErrStackOverflow);
              counts[i] = cnt;
              return;
            }
            stack_link[sp++] = p.lr;
          }
          link = p.ll;
          continue;
        }
        if (h1) {
          link = p.lr;
          continue;
        }
      }
      if (sp == 0) break;
      link = stack_link[--sp];
    }
  }
  counts[i] = cnt;
}

// raycast (all hits), persistent: warps take the rays the pre-pass queued through one work
// counter, and once kAllRefill lanes of a warp have finished their rays those lanes take the next
// ones (one atomic per refill for the whole warp).  The rays that enter the tree have traversal
// lengths from ~10 to ~1000 node reads, so a warp that only took new rays when all 32 were done
// would spend most of its time waiting on its longest one.  Each lane walks its ray exactly as
// raycast_all_kernel does (left child before right, every hit in DFS order).
constexpr int kAllRefill = 8;
constexpr int kAllBlocksPerSm = 8;

// 8 resident blocks per SM (64 registers), so that the launch's 8 blocks per SM are all resident:
// 4.35 -> 3.80 ms on the 2^24 incoherent rays of the 2M-triangle knot (12 blocks: 4.02 ms).
__global__ void __launch_bounds__(kBlock, kAllBlocksPerSm) raycast_all_persistent_kernel(
    MeshDev m, const float* __restrict__ rays, int side, const SideTable sides, float near_d, float far_d, uint32_t cap,
    uint32_t* __restrict__ counts, bvhc_hit* __restrict__ hits, const uint32_t* __restrict__ queue,
    const unsigned int* __restrict__ qcount, unsigned long long* __restrict__ work) {
  const unsigned full = 0xFFFFFFFFu;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_live = (uint64_t)__ldg(qcount);
  bool has = false, exhausted = false;
  uint64_t i = 0;
  RayF r;
  float dlen = 0.0f;
  uint32_t cnt = 0, link = 0;
  int sp = 0, root = 0;
  uint32_t stack_link[kMaxStack];
  for (;;) {
    const unsigned idle = __ballot_sync(full, !has);
    if (idle != 0u && !exhausted) {
      const int leader = __ffs(idle) - 1;
      unsigned long long base = 0;
      if ((int)lane == leader) base = atomicAdd(work, (unsigned long long)__popc(idle));
      base = __shfl_sync(full, base, leader);
      if (!has) {
        const uint64_t slot = base + (uint64_t)__popc(idle & ((1u << lane) - 1u));
        if (slot < n_live) {
          i = __ldg(queue + slot);
          r = make_ray(rays, i);
          dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
          cnt = 0;
          root = 0;
          sp = 0;
          link = m.roots[0];
          has = true;
        }
      }
      exhausted = base + (unsigned long long)__popc(idle) >= n_live;  // warp-uniform
    }
    if (!__any_sync(full, has)) break;
    for (;;) {
      if (has) {
        bool pop = false;
        if (link & kLeafBit) {
          if (link != kEmptyLeaf) {
            bvhc_hit* out = hits + i * (uint64_t)cap;
            for (uint32_t k = link & ~kLeafBit;; ++k) {
              const Tri t = load_tri(m.tris, k);
              const int ts = tri_side(t, side, sides);
              float th, te;
              if (ts >= 0 && tri_hit_t(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts, th, te) &&
                  in_range(th, te, t, r, dlen, near_d, far_d)) {
                if (cnt < cap) store_pending_record(out + cnt, k, 0.0f);
                ++cnt;
              }
              if (t.flags & kTriLast) break;
            }
          }
          pop = true;
        } else {
          const Pair p = load_pair(m.nodes, link);
          float e0, e1;
          const bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e0);
          const bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e1);
          if (h0) {
            if (h1) {
              if (sp >= kMaxStack) {
                atomicOr(m.err, kErrStackOverflow);
                sp = 0;
                root = m.n_roots;  // give up on this ray
                pop = true;
              } else {
                stack_link[sp++] = p.lr;
              }
            }
            if (!pop) link = p.ll;
          } else if (h1) {
            link = p.lr;
          } else {
            pop = true;
          }
        }
        if (pop) {
          if (sp > 0) {
            link = stack_link[--sp];
          } else if (++root < m.n_roots) {
            link = m.roots[root];
          } else {
            counts[i] = cnt;
            has = false;
          }
        }
      }
      const int n_idle = __popc(__ballot_sync(full, !has));
      if (exhausted ? n_idle == 32 : n_idle >= kAllRefill) break;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// raycast (all hits), warp-cooperative: the 32 rays of a warp walk the tree together, left child
// before right child as the reference does, entering a child when any lane's ray enters its box
// (one shared stack of links; there is no early out, so no per-lane distances).  A lane that tests
// the triangles of a leaf its own traversal would not have reached finds no hit there (a ray that
// hits a triangle enters every box on its path), so each lane reports exactly its own hits, in its
// own DFS order.  With a queue (rays sorted by a Morton key), a warp takes 32 consecutive entries.
// ---------------------------------------------------------------------------------------------
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) raycast_all_packet_kernel(
    MeshDev m, const float* __restrict__ rays, uint64_t n, int side, const SideTable sides, float near_d,
    float far_d, uint32_t cap, uint32_t* __restrict__ counts, bvhc_hit* __restrict__ hits,
    const uint32_t* __restrict__ queue, const unsigned int* __restrict__ qcount, uint64_t pitch, int rows_log2) {
  __shared__ uint32_t s_link[kWarps][kMaxStack];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  else if (valid && pitch) i = tiled_index(i, pitch, rows_log2, n);  // tiles of per-pixel rays
  RayF r;
  if (valid) {
    r = make_ray(rays, i);
  } else {
    r.o = make_float3(0.f, 0.f, 0.f);
    r.d = make_float3(1.f, 0.f, 0.f);
    r.inv = make_float3(1.f, 1e30f, 1e30f);
    r.d_l1 = 1.f;
  }
  const float dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  uint32_t cnt = 0;
  bvhc_hit* out = hits + i * (uint64_t)cap;
  bool overflow = false;
  for (int root = 0; root < m.n_roots && !overflow; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && valid) {
          for (uint32_t k = link & ~kLeafBit;; ++k) {
            Tri t = load_tri(m.tris, k);
            int ts = tri_side(t, side, sides);
            float th, te;
            if (ts >= 0 && tri_hit_t(t.a, t.b, t.c, r.o, r.d, r.d_l1, ts, th, te) &&
                in_range(th, te, t, r, dlen, near_d, far_d)) {
              if (cnt < cap) store_pending_record(out + cnt, k, 0.0f);
              ++cnt;
            }
            if (t.flags & kTriLast) break;
          }
        }
        pop = true;
      } else {
        Pair p = load_pair(m.nodes, link);
        float e0, e1;
        bool h0 = valid && box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e0);
        bool h1 = valid && box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e1);
        unsigned b0 = __ballot_sync(full, h0), b1 = __ballot_sync(full, h1);
        if (b0 && b1) {
          if (sp >= kMaxStack) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            overflow = true;
            break;
          }
          if (lane == 0) s_link[w][sp] = p.lr;
          ++sp;
          link = p.ll;
          __syncwarp();
        } else if (b0) {
          link = p.ll;
        } else if (b1) {
          link = p.lr;
        } else {
          pop = true;
        }
      }
      if (pop) {
        if (sp == 0) break;
        link = s_link[w][--sp];
      }
    }
  }
  if (valid) counts[i] = cnt;
}


}  // namespace dev

// The traversal of launch_raycast_all; *used_queue says whether it ran over the pre-pass queue
// (which then holds every ray that can have a hit).
static cudaError_t traverse_all(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                                float near_d, float far_d, uint32_t cap, uint32_t* counts, bvhc_hit* hits,
                                cudaStream_t stream, int variant, int occupancy, uint32_t* queue, unsigned int* qcount,
                                const RaySort* sort, unsigned long long* work, uint32_t tile, int tile_rows,
                                bool* used_queue) {
  *used_queue = false;
  if (variant == 0 || (variant == 2 && (!queue || !qcount || !sort || n >= (1ull << 32))) ||
      ((variant == 5 || variant == 9) && (!queue || !qcount || n >= (1ull << 32)))) {
    dev::raycast_all_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, cap,
                                                                      counts, hits);
    return cudaGetLastError();
  }
  cudaError_t e;
  if (variant == 9 && !work) variant = 5;
  if (variant == 5 || variant == 9) {
    // the root-box pre-pass gives the rays that miss a count of 0 and queues the others (in ray
    // order, or sorted by the key sort->kind) for one ray per thread: a warp then holds 32 rays
    // that enter the tree (neighbouring ones with a key); variant 9 walks the queue with
    // persistent warps that refill idle lanes
    if ((e = cudaMemsetAsync(qcount, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
    const bool keyed = sort && sort->kind > 0;
    uint32_t *ids = queue, *keys = nullptr;
    dev::SceneBox box{};
    if (keyed) {
      ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
      for (int a = 0; a < 3; ++a) {
        box.lo[a] = sort->lo[a];
        box.hi[a] = sort->hi[a];
      }
    }
    if ((e = launch_classify_counts(m, rays, n, near_d, far_d, ids, qcount, keys, keyed ? sort->kind : 0, box, counts,
                                    stream)) != cudaSuccess)
      return e;
    if (keyed && (e = launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
    *used_queue = true;
    if (variant == 9) {
      if ((e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), stream)) != cudaSuccess) return e;
      int dev_id = 0, sms = 148;
      cudaGetDevice(&dev_id);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
      dev::raycast_all_persistent_kernel<<<sms * dev::kAllBlocksPerSm, dev::kBlock, 0, stream>>>(m, rays, side, sides, near_d, far_d, cap,
                                                                              counts, hits, queue, qcount, work);
      return cudaGetLastError();
    }
    dev::raycast_all_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, cap,
                                                                      counts, hits, queue, qcount);
    return cudaGetLastError();
  }
  if (variant == 2) {
    // the root-box pre-pass gives the rays that miss a count of 0 and queues the others with their
    // keys, which are then sorted
    uint32_t *ids, *keys;
    ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
    dev::SceneBox box{};
    for (int a = 0; a < 3; ++a) {
      box.lo[a] = sort->lo[a];
      box.hi[a] = sort->hi[a];
    }
    if ((e = cudaMemsetAsync(qcount, 0, sizeof(unsigned int), stream)) != cudaSuccess) return e;
    if ((e = launch_classify_counts(m, rays, n, near_d, far_d, ids, qcount, keys, sort->kind, box, counts, stream)) !=
        cudaSuccess)
      return e;
    if ((e = launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream)) != cudaSuccess) return e;
    *used_queue = true;
  } else {
    queue = nullptr;
    qcount = nullptr;
  }
  auto kernel = occupancy == 0   ? dev::raycast_all_packet_kernel<1>
                : occupancy == 1 ? dev::raycast_all_packet_kernel<6>
                                 : dev::raycast_all_packet_kernel<8>;
  const int rl = tile_rows_log2(tile_rows);
  const uint64_t pitch = (!queue && tile >= 8 && tile % (32u >> rl) == 0) ? (uint64_t)tile : 0;
  kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, cap, counts, hits, queue,
                                                  qcount, pitch, rl);
  return cudaGetLastError();
}

cudaError_t launch_raycast_all(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                               float near_d, float far_d, uint32_t cap, uint32_t* counts, bvhc_hit* hits,
                               cudaStream_t stream, int variant, int occupancy, uint32_t* queue, unsigned int* qcount,
                               const RaySort* sort, unsigned long long* work, uint32_t tile, int tile_rows) {
  if (n == 0) return cudaSuccess;
  bool used_queue = false;
  cudaError_t e = traverse_all(m, rays, n, side, sides, near_d, far_d, cap, counts, hits, stream, variant, occupancy,
                               queue, qcount, sort, work, tile, tile_rows, &used_queue);
  if (e != cudaSuccess || cap == 0) return e;
  dev::raycast_all_finalize_kernel<<<grid_for(n), dev::kBlock, 0, stream>>>(
      m, rays, n, cap, counts, hits, used_queue ? queue : nullptr, used_queue ? qcount : nullptr);
  return cudaGetLastError();
}

}  // namespace bvhc
