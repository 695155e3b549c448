// raycastFirst kernels: one ray per thread, the persistent form with lane refill and its finalize
// pass, and the root-box pre-pass (with the ray-ordering keys) that the persistent,
// warp-cooperative and all-hits forms share; and their launches.  The warp-cooperative forms are
// in kernels_packet.cu.
#include <algorithm>

#include "traverse.cuh"

namespace bvhc {
namespace dev {

// raycastFirst, one ray per thread (the child order is left_first, traverse.cuh).
template <int ORDER>
__global__ void __launch_bounds__(kBlock) raycast_first_kernel(MeshDev m, const float* __restrict__ rays, uint64_t n,
                                                               int side, const SideTable sides, float near_d,
                                                               float far_d, bvhc_hit* __restrict__ out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  RayF r = make_ray(rays, i);
  float dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  uint32_t stack_link[kMaxStack];
  float stack_t[kMaxStack];
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      if (link & kLeafBit) {
        if (link != kEmptyLeaf) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
      } else {
        Pair p = load_pair(m.nodes, link);
        float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
        float e0, e1;
        bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
        bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
        bool lf = left_first<ORDER>(p, r, e0, e1);
        uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
        bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
        if (h1st) {
          if (h2nd) {
            if (sp >= kMaxStack) {
              atomicOr(m.err, kErrStackOverflow);
              store_miss(out + i);
              return;
            }
            stack_link[sp] = c2;
            stack_t[sp] = lf ? e1 : e0;
            ++sp;
          }
          link = c1;
          continue;
        }
        if (h2nd) {
          link = c2;
          continue;
        }
      }
      // pop, skipping entries that start beyond the best hit found since they were pushed
      bool found = false;
      float lim = (best.t + best.err) * (1.0f + kSlabMargin);
      while (sp > 0) {
        --sp;
        if (stack_t[sp] <= lim) {
          link = stack_link[sp];
          found = true;
          break;
        }
      }
      if (!found) break;
    }
  }
  store_first_pending(out + i, best);  // finalize_first_kernel completes a hit
}

// ---------------------------------------------------------------------------------------------
// raycastFirst, persistent form.  A fixed grid of warps pulls rays from a global work counter in
// chunks of 32..kChunk rays per warp (one atomicAdd per chunk); a lane whose ray is finished sits idle
// until `refill` lanes of its warp are idle, and then those lanes take the next rays of the warp's
// chunk together, so warps stay full while rays of very different cost (early misses, deep
// traversals) are mixed.  Each outer iteration runs the "while-while" phases: every lane walks
// child pairs until it reaches a leaf or finishes, then the lanes holding a leaf test it together.
// A finished hit is written as a pending (record, t) pair; finalize_first_kernel then computes the
// reported records one ray per thread, so the float-float work runs with full warps.
// ---------------------------------------------------------------------------------------------
constexpr unsigned kChunk = 256;

// Mesh of ray `rid` in a batch: the last mesh whose first ray is <= rid (ray_off is CSR).
__device__ __forceinline__ int mesh_of_ray(const BatchDev& bd, uint64_t rid) {
  int lo = 0, hi = bd.n_meshes - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(bd.ray_off + mid) <= rid) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// BATCHED: every ray belongs to one of many meshes packed into one node/triangle pool (the
// meshes of a BatchedMesh, ExtensionUtilities.js:87-161); a lane looks up its ray's mesh when it
// takes the ray and traverses that mesh's roots.  Otherwise the mesh's roots are m.roots[0..n).
// MINB: minimum resident blocks per SM requested from the register allocator (1 = no limit).
// WIDE: walk the four-child records (m.quads, m.quad_roots; same leaves and triangle records):
// half the levels, so half as many dependent node loads per ray; at a record the children the ray
// enters are taken nearest first (ORDER does not apply) and the others stacked farthest first.
template <int ORDER, bool BATCHED, int MINB, int STACK, bool WIDE = false>
__global__ void __launch_bounds__(kBlock, MINB) raycast_first_persistent_kernel(
    MeshDev m, const BatchDev bd, const float* __restrict__ rays, uint64_t n, int side, const SideTable sides,
    float near_d, float far_d, bvhc_hit* __restrict__ out, unsigned long long* __restrict__ work, int refill,
    const uint32_t* __restrict__ queue, const unsigned int* __restrict__ qcount) {
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt_mask = (1u << lane) - 1u;
  // with a queue (written by classify_kernel) the work items are its entries, else all rays
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  // rays per warp fetch: about eight fetches per warp over the launch, between 32 and kChunk, so
  // that small batches still spread over every resident warp
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  uint64_t chunk = n_work / (warps * 8);
  chunk = chunk < 32 ? 32 : (chunk > kChunk ? kChunk : (chunk & ~31ull));
  bool active = false;
  uint64_t rid = 0;
  RayF r;
  float dlen = 0.0f;
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  uint32_t link = 0;
  int sp = 0, root = 0, root_end = m.n_roots;
  uint32_t stack_link[STACK];
  float stack_t[STACK];
  uint64_t pool = 0, pool_end = 0;  // warp-uniform: this warp's untaken rays [pool, pool_end)
  bool drained = false;             // warp-uniform: the work counter is exhausted

  // Next link after a leaf or a dead end: pop the nearest stacked child whose entry distance does
  // not lie beyond the best hit, else move to the next root, else finish the ray.
  auto pop_next = [&]() {
    float lim = (best.t + best.err) * (1.0f + kSlabMargin);
    while (sp > 0) {
      --sp;
      if (stack_t[sp] <= lim) {
        link = stack_link[sp];
        return;
      }
    }
    if (++root < root_end) {
      link = WIDE ? m.quad_roots[root] : m.roots[root];
      return;
    }
    store_first_pending(out + rid, best);  // finalize_first_kernel completes a hit
    active = false;
  };

  for (;;) {
    unsigned idle = __ballot_sync(0xFFFFFFFFu, !active);
    if (idle == 0xFFFFFFFFu || (idle != 0u && __popc(idle) >= refill)) {
      unsigned need = __popc(idle);
      uint64_t avail = pool_end - pool;
      uint64_t nb = 0, ne = 0;
      if (need > avail && !drained) {
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(work, (unsigned long long)chunk);
        b = __shfl_sync(0xFFFFFFFFu, b, 0);
        if (b >= n_work) {
          drained = true;
        } else {
          nb = b;
          ne = b + chunk < n_work ? b + chunk : n_work;
        }
      }
      if (!active) {
        uint64_t rank = __popc(idle & lt_mask);
        bool got = true;
        if (rank < avail) rid = pool + rank;
        else if (rank - avail < ne - nb) rid = nb + (rank - avail);
        else got = false;
        if (got && queue) rid = __ldg(queue + rid);
        if (got) {
          active = true;
          r = make_ray(rays, rid);
          dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
          best = Best{kInf, 0.0f, 0xFFFFFFFFu};
          if (BATCHED) {
            int mesh = mesh_of_ray(bd, rid);
            root = (int)__ldg(bd.mesh_root_off + mesh);
            root_end = (int)__ldg(bd.mesh_root_off + mesh + 1);
          } else {
            root = 0;
            root_end = m.n_roots;
          }
          sp = 0;
          link = WIDE ? m.quad_roots[root] : m.roots[root];
        }
      }
      if (need <= avail) {
        pool += need;
      } else {
        uint64_t used = need - avail;
        pool = nb + used < ne ? nb + used : ne;
        pool_end = ne;
      }
      if (idle == 0xFFFFFFFFu && __ballot_sync(0xFFFFFFFFu, active) == 0u) break;
    }
    if (!active) continue;
    // phase 1: child pairs (or four-child records), until this lane holds a leaf or has finished
    // its ray
    while (WIDE && active && !(link & kLeafBit)) {
      const QuadNode* qn = m.quads + link;
      float4 lx, ly, lz, hx, hy, hz;
      ld8(qn->lo[0], lx, ly);
      ld8(qn->lo[2], lz, hx);
      ld8(qn->hi[1], hy, hz);
      const float4 lk = ld4(qn->link);
      const uint32_t ck[4] = {__float_as_uint(lk.x), __float_as_uint(lk.y), __float_as_uint(lk.z),
                              __float_as_uint(lk.w)};
      const float blo[3][4] = {{lx.x, lx.y, lx.z, lx.w}, {ly.x, ly.y, ly.z, ly.w}, {lz.x, lz.y, lz.z, lz.w}};
      const float bhi[3][4] = {{hx.x, hx.y, hx.z, hx.w}, {hy.x, hy.y, hy.z, hy.w}, {hz.x, hz.y, hz.z, hz.w}};
      const float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
      float key[4];
      uint32_t cl[4];
      int nh = 0;
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        float e;
        const bool h = ck[c] != kEmptyLeaf &&
                       box_hit(blo[0][c], blo[1][c], blo[2][c], bhi[0][c], bhi[1][c], bhi[2][c], r, near_d, lim, e);
        key[c] = h ? e : kInf;
        cl[c] = ck[c];
        nh += h ? 1 : 0;
      }
      // the four (entry, child) pairs nearest first; children the ray misses sort last
      auto cas = [&](int a, int c) {
        if (key[c] < key[a]) {
          const float tk = key[a];
          key[a] = key[c];
          key[c] = tk;
          const uint32_t tl = cl[a];
          cl[a] = cl[c];
          cl[c] = tl;
        }
      };
      cas(0, 1);
      cas(2, 3);
      cas(0, 2);
      cas(1, 3);
      cas(1, 2);
      if (nh == 0) {
        pop_next();
      } else if (sp + nh - 1 > STACK) {
        atomicOr(m.err, kErrStackOverflow);
        best.rec = 0xFFFFFFFFu;
        sp = 0;
        root = root_end;
        pop_next();
      } else {
#pragma unroll
        for (int j = 3; j >= 1; --j)
          if (j < nh) {
            stack_link[sp] = cl[j];
            stack_t[sp] = key[j];
            ++sp;
          }
        link = cl[0];
      }
    }
    while (!WIDE && active && !(link & kLeafBit)) {
      Pair p = load_pair(m.nodes, link);
      float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
      float e0, e1;
      bool h0 = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
      bool h1 = box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
      bool lf = left_first<ORDER>(p, r, e0, e1);
      uint32_t c1 = lf ? p.ll : p.lr, c2 = lf ? p.lr : p.ll;
      bool h1st = lf ? h0 : h1, h2nd = lf ? h1 : h0;
      if (h1st && h2nd) {
        if (sp >= STACK) {
          atomicOr(m.err, kErrStackOverflow);
          best.rec = 0xFFFFFFFFu;
          sp = 0;
          root = root_end;
          pop_next();
        } else {
          stack_link[sp] = c2;
          stack_t[sp] = lf ? e1 : e0;
          ++sp;
          link = c1;
        }
      } else if (h1st) {
        link = c1;
      } else if (h2nd) {
        link = c2;
      } else {
        pop_next();
      }
    }
    // phase 2: the leaf
    if (active) {
      if (link != kEmptyLeaf) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
      pop_next();
    }
  }
}

// Completes the pending hits every raycastFirst traversal kernel leaves (per ray, persistent,
// warp-cooperative), one ray per thread (grid-stride).  With a queue only its entries can be
// pending; the other rays were finished by classify_kernel.
__global__ void __launch_bounds__(kBlock) finalize_first_kernel(MeshDev m, const float* __restrict__ rays, uint64_t n,
                                                                bvhc_hit* __restrict__ out,
                                                                const uint32_t* __restrict__ queue,
                                                                const unsigned int* __restrict__ qcount) {
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_work; k += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t i = queue ? (uint64_t)__ldg(queue + k) : k;
    uint32_t rec = __float_as_uint(__ldcs(reinterpret_cast<const float*>(out + i)));
    if (rec == BVHC_NO_HIT) continue;
    RayF r = make_ray(rays, i);
    finish_first(m, rec, r, out + i);
  }
}

// Pre-pass for the persistent and warp-cooperative traversals: a ray whose box tests against every
// root's two children (with the root's own leaf case always live) all fail cannot hit anything; it
// is finished here with a coalesced miss record.  The other rays are appended to `queue` in ray
// order (one atomic per block reserves the block's run; positions within it come from ballots), so
// the traversal kernel's warps only carry rays that enter the tree.  With `keys`, each queued ray's
// ordering key (raykey.cuh, kind `kind`) is written beside its id.  With `miss_counts` (all-hits
// raycast) a ray that misses gets a hit count of 0 instead of a miss record.

template <bool BATCHED>
__global__ void __launch_bounds__(kClsThreads) classify_kernel(
    MeshDev m, const BatchDev bd, const float* __restrict__ rays, uint64_t n, float near_d, float far_d,
    bvhc_hit* __restrict__ out, uint32_t* __restrict__ queue, unsigned int* __restrict__ qcount,
    uint32_t* __restrict__ keys, int kind, SceneBox box, uint32_t* __restrict__ miss_counts = nullptr) {
  __shared__ unsigned s_cnt[kClsItems * kClsWarps];  // live rays per (item round, warp), then prefixes
  __shared__ unsigned s_base;
  const unsigned lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kClsTile;
  unsigned ballot[kClsItems];
  uint32_t key[kClsItems];
#pragma unroll
  for (int j = 0; j < kClsItems; ++j) {
    uint64_t i = base + (uint64_t)j * kClsThreads + threadIdx.x;
    bool live = false;
    key[j] = 0;
    if (i < n) {
      RayF r = make_ray(rays, i);
      int root = 0, root_end = m.n_roots;
      if (BATCHED) {
        int mesh = mesh_of_ray(bd, i);
        root = (int)__ldg(bd.mesh_root_off + mesh);
        root_end = (int)__ldg(bd.mesh_root_off + mesh + 1);
      }
      for (; root < root_end && !live; ++root) {
        uint32_t link = __ldg(m.roots + root);
        if (link & kLeafBit) {
          live = link != kEmptyLeaf;
          continue;
        }
        Pair p = load_pair(m.nodes, link);
        float e;
        live = box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, far_d, e) ||
               box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, far_d, e);
      }
      if (!live) {
        if (miss_counts) miss_counts[i] = 0;  // all hits: the uncapped count of a ray that misses
        else store_miss(out + i);
      }
      else if (keys) key[j] = ray_key(kind, r.o, r.d, box);
    }
    ballot[j] = __ballot_sync(0xFFFFFFFFu, live);
    if (lane == 0) s_cnt[j * kClsWarps + w] = (unsigned)__popc(ballot[j]);
  }
  __syncthreads();
  if (w == 0) {
    // exclusive scan of the 64 counts in (round, warp) order, which is ray order
    static_assert(kClsItems * kClsWarps == 64, "two counts per lane");
    unsigned a = s_cnt[2 * lane], b = s_cnt[2 * lane + 1];
    unsigned incl = a + b;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= (unsigned)o) incl += y;
    }
    unsigned excl = incl - a - b;
    s_cnt[2 * lane] = excl;
    s_cnt[2 * lane + 1] = excl + a;
    unsigned total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (lane == 0) s_base = total ? atomicAdd(qcount, total) : 0u;
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < kClsItems; ++j) {
    if (ballot[j] & (1u << lane)) {
      unsigned pos = s_base + s_cnt[j * kClsWarps + w] + (unsigned)__popc(ballot[j] & lt);
      queue[pos] = (uint32_t)(base + (uint64_t)j * kClsThreads + threadIdx.x);
      if (keys) keys[pos] = key[j];
    }
  }
}

}  // namespace dev

// Resident blocks per SM x SM count for a persistent kernel on the current device, cached per
// (device, kernel variant).
template <class K>
static unsigned int persistent_grid(K kernel, int variant) {
  constexpr int kDevs = 64, kVariants = 30;
  static unsigned int cache[kDevs][kVariants] = {};
  int dev_id = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev_id);
  if (dev_id >= 0 && dev_id < kDevs && cache[dev_id][variant]) return cache[dev_id][variant];
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, dev::kBlock, 0);
  unsigned int g = (unsigned int)(std::max(1, sms) * std::max(1, per_sm));
  if (dev_id >= 0 && dev_id < kDevs) cache[dev_id][variant] = g;
  return g;
}

struct PersistentArgs {
  MeshDev m;
  BatchDev bd;
  const float* rays;
  uint64_t n;
  int side;
  SideTable sides;
  float near_d, far_d;
  bvhc_hit* out;
  unsigned long long* work;
  int refill;
  const uint32_t* queue;
  const unsigned int* qcount;
};

template <int ORDER, bool BATCHED, int MINB, int STACK, bool WIDE = false>
static void launch_persistent(const PersistentArgs& a, cudaStream_t stream) {
  auto kernel = dev::raycast_first_persistent_kernel<ORDER, BATCHED, MINB, STACK, WIDE>;
  const int occ_id = MINB == 1 ? 0 : (MINB == 6 ? 1 : 2);
  int variant = WIDE ? 24 + (BATCHED ? 3 : 0) + occ_id : (STACK == 32 ? 12 : 0) + ORDER * 6 + (BATCHED ? 3 : 0) + occ_id;
  unsigned int g = persistent_grid(kernel, variant);
  g = (unsigned int)std::min<uint64_t>(g, (a.n + dev::kBlock - 1) / dev::kBlock);
  kernel<<<g, dev::kBlock, 0, stream>>>(a.m, a.bd, a.rays, a.n, a.side, a.sides, a.near_d, a.far_d, a.out, a.work,
                                        a.refill, a.queue, a.qcount);
}

template <int ORDER, bool BATCHED, int STACK>
static void launch_persistent_occ(const PersistentArgs& a, int occupancy, cudaStream_t stream) {
  if (occupancy == 0) launch_persistent<ORDER, BATCHED, 1, STACK>(a, stream);
  else if (occupancy == 1) launch_persistent<ORDER, BATCHED, 6, STACK>(a, stream);
  else launch_persistent<ORDER, BATCHED, 8, STACK>(a, stream);
}

template <bool BATCHED>
static void launch_persistent_cfg(const PersistentArgs& a, const TraversalConfig& cfg, cudaStream_t stream) {
  if (cfg.wide && a.m.quads && a.m.quad_roots) {
    // four-child records: nearest child first, the 64-entry stack (a record stacks up to three);
    // a batch's meshes index their quad roots as their child-pair roots
    if (cfg.occupancy == 0) launch_persistent<1, BATCHED, 1, 64, true>(a, stream);
    else if (cfg.occupancy == 1) launch_persistent<1, BATCHED, 6, 64, true>(a, stream);
    else launch_persistent<1, BATCHED, 8, 64, true>(a, stream);
    return;
  }
  const bool s32 = stack_entries(a.m, cfg.stack) == 32;
  if (cfg.order == 0) {
    if (s32) launch_persistent_occ<0, BATCHED, 32>(a, cfg.occupancy, stream);
    else launch_persistent_occ<0, BATCHED, 64>(a, cfg.occupancy, stream);
  } else {
    if (s32) launch_persistent_occ<1, BATCHED, 32>(a, cfg.occupancy, stream);
    else launch_persistent_occ<1, BATCHED, 64>(a, cfg.occupancy, stream);
  }
}

// Root-box pre-pass into `queue`, then (single mesh, sort requested) the ray-ordering sort.
cudaError_t prepare_queue(const MeshDev& m, const BatchDev* batch, const float* rays, uint64_t n, float near_d,
                                 float far_d, bvhc_hit* out, uint32_t* queue, unsigned int* qcount,
                                 const RaySort* sort, cudaStream_t stream) {
  cudaError_t e = cudaMemsetAsync(qcount, 0, sizeof(unsigned int), stream);
  if (e != cudaSuccess) return e;
  BatchDev bd = batch ? *batch : BatchDev{nullptr, nullptr, 0};
  const bool sorted = sort && !batch && sort->kind > 0;
  // a sorted queue is first written (with keys) where the sort's passes start, so they end in `queue`
  uint32_t* ids = queue;
  uint32_t* keys = nullptr;
  if (sorted) ray_sort_input(sort->kind, sort->scratch, queue, &ids, &keys);
  dev::SceneBox box{};
  if (sorted) {
    for (int a = 0; a < 3; ++a) {
      box.lo[a] = sort->lo[a];
      box.hi[a] = sort->hi[a];
    }
  }
  const int kind = sorted ? sort->kind : 0;
  const unsigned int g = (unsigned int)((n + dev::kClsTile - 1) / dev::kClsTile);
  if (batch)
    dev::classify_kernel<true><<<g, dev::kClsThreads, 0, stream>>>(m, bd, rays, n, near_d, far_d, out, ids, qcount,
                                                                   keys, kind, box);
  else
    dev::classify_kernel<false><<<g, dev::kClsThreads, 0, stream>>>(m, bd, rays, n, near_d, far_d, out, ids, qcount,
                                                                    keys, kind, box);
  e = cudaGetLastError();
  if (e != cudaSuccess || !sorted) return e;
  return launch_ray_sort(sort->kind, n, qcount, sort->scratch, queue, stream);
}

cudaError_t launch_raycast_first_persistent(const MeshDev& m, const BatchDev* batch, const float* rays, uint64_t n,
                                            int side, const SideTable& sides, float near_d, float far_d,
                                            bvhc_hit* out, unsigned long long* work, const TraversalConfig& cfg,
                                            cudaStream_t stream, uint32_t* queue, unsigned int* qcount,
                                            const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(work, 0, sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return e;
  const bool compact = queue != nullptr && qcount != nullptr && n < (1ull << 32);
  BatchDev bd = batch ? *batch : BatchDev{nullptr, nullptr, 0};
  if (compact) {
    e = prepare_queue(m, batch, rays, n, near_d, far_d, out, queue, qcount, sort, stream);
    if (e != cudaSuccess) return e;
  }
  PersistentArgs a{m, bd, rays, n, side, sides, near_d, far_d, out, work, cfg.refill,
                   compact ? queue : nullptr, compact ? qcount : nullptr};
  if (batch) launch_persistent_cfg<true>(a, cfg, stream);
  else launch_persistent_cfg<false>(a, cfg, stream);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_finalize_first(m, rays, n, out, a.queue, a.qcount, stream);
}

cudaError_t launch_finalize_first(const MeshDev& m, const float* rays, uint64_t n, bvhc_hit* out,
                                  const uint32_t* queue, const unsigned int* qcount, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  unsigned int fg = (unsigned int)std::min<uint64_t>(grid_for(n), 8192);
  dev::finalize_first_kernel<<<fg, dev::kBlock, 0, stream>>>(m, rays, n, out, queue, qcount);
  return cudaGetLastError();
}

cudaError_t launch_raycast_first(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                                 float near_d, float far_d, bvhc_hit* out, int order, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  if (order == 0)
    dev::raycast_first_kernel<0><<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out);
  else
    dev::raycast_first_kernel<1><<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_finalize_first(m, rays, n, out, nullptr, nullptr, stream);
}

// The pre-pass over a single mesh's rays for the all-hits raycast: rays that miss get a hit count of
// 0 in `miss_counts`, the others are queued in `ids` (with their keys when kind > 0).
cudaError_t launch_classify_counts(const MeshDev& m, const float* rays, uint64_t n, float near_d, float far_d,
                                   uint32_t* ids, unsigned int* qcount, uint32_t* keys, int kind,
                                   const dev::SceneBox& box, uint32_t* miss_counts, cudaStream_t stream) {
  const unsigned int g = (unsigned int)((n + dev::kClsTile - 1) / dev::kClsTile);
  dev::classify_kernel<false><<<g, dev::kClsThreads, 0, stream>>>(m, BatchDev{nullptr, nullptr, 0}, rays, n, near_d,
                                                                  far_d, nullptr, ids, qcount, keys, kind, box,
                                                                  miss_counts);
  return cudaGetLastError();
}

}  // namespace bvhc
