// raycastFirst, warp-cooperative forms (over child pairs, in queue, input or tiled ray order, and
// over four-child records); and their launch.
#include <algorithm>

#include "traverse.cuh"

namespace bvhc {
namespace dev {

// ---------------------------------------------------------------------------------------------
// raycastFirst, warp-cooperative form for coherent rays (camera rays in pixel order).  The 32
// rays of a warp walk the tree together with one shared stack: every child pair is fetched once
// for the warp (a broadcast load), each lane tests it against its own ray, and the warp enters a
// child if any lane's ray enters it (nearest first by majority vote).  A leaf is tested by all
// lanes at once, so the triangle tests run at full SIMD width.  Each lane keeps its own entry
// distance for every stacked child; a stacked child is skipped when no lane still needs it.
// Visiting a node a lane's ray does not enter costs that lane nothing but idle time, and testing
// a triangle it would not have reached cannot change its closest hit.  The kernel leaves each hit
// pending (its triangle record); finalize_first_kernel computes the reported records, which keeps
// the float-float record code out of the traversal kernel.
// ---------------------------------------------------------------------------------------------

// BLOCK threads per block (64, 128 or 256), STACK shared-stack entries (32 or 64; the launch picks 32
// only for trees shallow enough that no traversal can need more).
template <int ORDER, int MINB, int BLOCK, int STACK>
__global__ void __launch_bounds__(BLOCK, MINB) raycast_first_packet_kernel(MeshDev m, const float* __restrict__ rays,
                                                                     uint64_t n, int side, const SideTable sides,
                                                                     float near_d, float far_d,
                                                                     bvhc_hit* __restrict__ out,
                                                                     const uint32_t* __restrict__ queue,
                                                                     const unsigned int* __restrict__ qcount,
                                                                     uint64_t pitch, int rows_log2) {
  __shared__ uint32_t s_link[BLOCK / 32][STACK];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  // with a queue (root-box pre-pass, optionally sorted) a warp takes 32 consecutive queue entries;
  // without one, 32 consecutive rays or (pitch > 0) a tile of them
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  else if (valid && pitch) i = tiled_index(i, pitch, rows_log2, n);
  RayF r;
  float dlen = 1.0f;
  if (valid) {
    r = make_ray(rays, i);
    dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  } else {
    r.o = make_float3(0.f, 0.f, 0.f);
    r.d = make_float3(1.f, 0.f, 0.f);
    r.inv = make_float3(1.f, 1e30f, 1e30f);
    r.d_l1 = 1.f;
  }
  const unsigned valid_mask = __ballot_sync(full, valid);
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  float lane_t[STACK];
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.roots[root];
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && valid) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
        pop = true;
      } else {
        Pair p = load_pair(m.nodes, link);
        float lim = fminf(far_d, (best.t + best.err) * (1.0f + kSlabMargin));
        float e0, e1;
        bool h0 = valid && box_hit(p.l[0], p.l[1], p.l[2], p.l[3], p.l[4], p.l[5], r, near_d, lim, e0);
        bool h1 = valid && box_hit(p.r[0], p.r[1], p.r[2], p.r[3], p.r[4], p.r[5], r, near_d, lim, e1);
        unsigned b0 = __ballot_sync(full, h0), b1 = __ballot_sync(full, h1);
        if (b0 && b1) {
          bool lf = left_first<ORDER>(p, r, e0, e1);
          bool left_wins = 2 * __popc(__ballot_sync(full, valid && lf)) >= __popc(valid_mask);
          if (sp >= STACK) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            best.rec = 0xFFFFFFFFu;
            root = m.n_roots;
            break;
          }
          if (lane == 0) s_link[w][sp] = left_wins ? p.lr : p.ll;
          lane_t[sp] = left_wins ? (h1 ? e1 : kInf) : (h0 ? e0 : kInf);
          ++sp;
          link = left_wins ? p.ll : p.lr;
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
        bool found = false;
        while (sp > 0) {
          --sp;
          float lim = (best.t + best.err) * (1.0f + kSlabMargin);
          if (__ballot_sync(full, valid && lane_t[sp] <= lim)) {
            link = s_link[w][sp];
            found = true;
            break;
          }
        }
        if (!found) break;
      }
    }
  }
  if (valid) store_first_pending(out + i, best);  // finalize_first_kernel completes a hit
}

// ---------------------------------------------------------------------------------------------
// raycastFirst, warp-cooperative over the four-child records (m.quads): the same shared traversal
// as above with half as many node visits.  At a record each lane tests the four child boxes (one
// 16-byte load per bound plane serves all four); the children any lane enters are ordered by the
// entry distances of the first lane that enters one (the warp's rays are coherent), the nearest is
// visited and the others are stacked farthest first, each with every lane's own entry distance.
// ---------------------------------------------------------------------------------------------
template <int MINB>
__global__ void __launch_bounds__(kBlock, MINB) raycast_first_packet4_kernel(
    MeshDev m, const float* __restrict__ rays, uint64_t n, int side, const SideTable sides, float near_d,
    float far_d, bvhc_hit* __restrict__ out, const uint32_t* __restrict__ queue,
    const unsigned int* __restrict__ qcount, uint64_t pitch, int rows_log2) {
  __shared__ uint32_t s_link[kWarps][kMaxStack];
  const unsigned full = 0xFFFFFFFFu;
  const int w = threadIdx.x >> 5;
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t n_work = queue ? (uint64_t)__ldg(qcount) : n;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if ((uint64_t)blockIdx.x * blockDim.x >= n_work) return;  // block-uniform
  const bool valid = i < n_work;
  if (valid && queue) i = __ldg(queue + i);
  else if (valid && pitch) i = tiled_index(i, pitch, rows_log2, n);
  RayF r;
  float dlen = 1.0f;
  if (valid) {
    r = make_ray(rays, i);
    dlen = sqrtf(r.d.x * r.d.x + r.d.y * r.d.y + r.d.z * r.d.z);
  } else {
    r.o = make_float3(0.f, 0.f, 0.f);
    r.d = make_float3(1.f, 0.f, 0.f);
    r.inv = make_float3(1.f, 1e30f, 1e30f);
    r.d_l1 = 1.f;
  }
  Best best{kInf, 0.0f, 0xFFFFFFFFu};
  float lane_t[kMaxStack];
  for (int root = 0; root < m.n_roots; ++root) {
    uint32_t link = m.quad_roots[root];
    int sp = 0;
    for (;;) {
      bool pop = false;
      if (link & kLeafBit) {
        if (link != kEmptyLeaf && valid) leaf_first(m, link & ~kLeafBit, r, dlen, side, sides, near_d, far_d, best);
        pop = true;
      } else {
        // 112 of the record's 128 bytes: three 256-bit loads and one 128-bit load (the quad array is
        // one allocation of 128-byte records)
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
        float e[4];
        bool h[4];
        unsigned b[4];
        unsigned any = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          h[c] = valid && ck[c] != kEmptyLeaf &&
                 box_hit(blo[0][c], blo[1][c], blo[2][c], bhi[0][c], bhi[1][c], bhi[2][c], r, near_d, lim, e[c]);
          b[c] = __ballot_sync(full, h[c]);
          any |= b[c];
        }
        if (!any) {
          pop = true;
        } else {
          const int leader = __ffs(any) - 1;
          float key[4];
          int idx[4];
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            float kc = __shfl_sync(full, h[c] ? e[c] : kInf, leader);
            key[c] = b[c] ? kc : kInf;
            idx[c] = c;
          }
          // sort the four (key, child) pairs, nearest first (warp-uniform values)
          auto cas = [&](int a, int c) {
            if (key[c] < key[a]) {
              float tk = key[a]; key[a] = key[c]; key[c] = tk;
              int ti = idx[a]; idx[a] = idx[c]; idx[c] = ti;
            }
          };
          cas(0, 1); cas(2, 3); cas(0, 2); cas(1, 3); cas(1, 2);
          if (sp + 3 > kMaxStack) {
            if (lane == 0) atomicOr(m.err, kErrStackOverflow);
            best.rec = 0xFFFFFFFFu;
            root = m.n_roots;
            break;
          }
          // children that some lane enters, farthest pushed first; the nearest is visited now
          uint32_t next = kEmptyLeaf;
          bool have_next = false;
#pragma unroll
          for (int j = 3; j >= 0; --j) {
            const int c = idx[j];
            if (!b[c]) continue;
            if (j == 0) {
              next = ck[c];
              have_next = true;
            } else {
              if (lane == 0) s_link[w][sp] = ck[c];
              lane_t[sp] = h[c] ? e[c] : kInf;
              ++sp;
            }
          }
          if (have_next) {
            link = next;
          } else {  // the first key belonged to a child no lane enters: every entered one was stacked
            pop = true;
          }
          __syncwarp();
        }
      }
      if (pop) {
        bool found = false;
        while (sp > 0) {
          --sp;
          float plim = (best.t + best.err) * (1.0f + kSlabMargin);
          if (__ballot_sync(full, valid && lane_t[sp] <= plim)) {
            link = s_link[w][sp];
            found = true;
            break;
          }
        }
        if (!found) break;
      }
    }
  }
  if (valid) store_first_pending(out + i, best);  // finalize_first_kernel completes a hit
}

}  // namespace dev

template <int BLOCK, int STACK>
static void launch_packet_kernel(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                                 float near_d, float far_d, bvhc_hit* out, int order, int occupancy,
                                 cudaStream_t stream, const uint32_t* queue, const unsigned int* qcount,
                                 uint64_t pitch, int rows_log2) {
  // occupancy 1 / 2 ask for 768 / 1024 resident threads per SM whatever the block size
  constexpr int k6 = 6 * 128 / BLOCK, k8 = 8 * 128 / BLOCK;
  auto kernel = order == 0 ? (occupancy == 0   ? dev::raycast_first_packet_kernel<0, 1, BLOCK, STACK>
                              : occupancy == 1 ? dev::raycast_first_packet_kernel<0, k6, BLOCK, STACK>
                                               : dev::raycast_first_packet_kernel<0, k8, BLOCK, STACK>)
                           : (occupancy == 0   ? dev::raycast_first_packet_kernel<1, 1, BLOCK, STACK>
                              : occupancy == 1 ? dev::raycast_first_packet_kernel<1, k6, BLOCK, STACK>
                                               : dev::raycast_first_packet_kernel<1, k8, BLOCK, STACK>);
  const unsigned int grid = (unsigned int)((n + BLOCK - 1) / BLOCK);
  kernel<<<grid, BLOCK, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out, queue, qcount, pitch, rows_log2);
}

cudaError_t launch_raycast_first_packet(const MeshDev& m, const float* rays, uint64_t n, int side,
                                        const SideTable& sides, float near_d, float far_d, bvhc_hit* out,
                                        const TraversalConfig& cfg, cudaStream_t stream, uint32_t* queue,
                                        unsigned int* qcount, const RaySort* sort) {
  if (n == 0) return cudaSuccess;
  const bool compact = queue != nullptr && qcount != nullptr && n < (1ull << 32);
  if (compact) {
    cudaError_t e = prepare_queue(m, nullptr, rays, n, near_d, far_d, out, queue, qcount, sort, stream);
    if (e != cudaSuccess) return e;
  } else {
    queue = nullptr;
    qcount = nullptr;
  }
  // the tiled order applies to the whole ray range (a queue is already in its own order)
  const int rl = tile_rows_log2(cfg.tile_rows);
  const uint64_t pitch = (!queue && cfg.tile >= 8 && cfg.tile % (32 >> rl) == 0) ? (uint64_t)cfg.tile : 0;
  if (cfg.wide && m.quads && m.quad_roots) {
    auto k4 = cfg.occupancy == 0   ? dev::raycast_first_packet4_kernel<1>
              : cfg.occupancy == 1 ? dev::raycast_first_packet4_kernel<6>
                                   : dev::raycast_first_packet4_kernel<8>;
    k4<<<grid_for(n), dev::kBlock, 0, stream>>>(m, rays, n, side, sides, near_d, far_d, out, queue, qcount, pitch,
                                                rl);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_finalize_first(m, rays, n, out, queue, qcount, stream);
  }
  const bool s32 = stack_entries(m, cfg.stack) == 32;
  const int block = cfg.block == 64 || cfg.block == 256 ? cfg.block : 128;
#define BVHC_PACKET(B, S) \
  launch_packet_kernel<B, S>(m, rays, n, side, sides, near_d, far_d, out, cfg.order, cfg.occupancy, stream, queue, \
                             qcount, pitch, rl)
  if (block == 64) {
    if (s32) BVHC_PACKET(64, 32);
    else BVHC_PACKET(64, 64);
  } else if (block == 256) {
    if (s32) BVHC_PACKET(256, 32);
    else BVHC_PACKET(256, 64);
  } else {
    if (s32) BVHC_PACKET(128, 32);
    else BVHC_PACKET(128, 64);
  }
#undef BVHC_PACKET
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_finalize_first(m, rays, n, out, queue, qcount, stream);
}

}  // namespace bvhc
