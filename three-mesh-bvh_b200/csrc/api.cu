// C ABI of libbvhcuda: build (CPU), upload (re-layout + validation) and GPU queries.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <thread>
#include <vector>

#include "bvhc_internal.h"
#include "kernels.cuh"
#include "layout.h"

using namespace bvhc;

// Rays per chunk of the pipelined host-memory raycastFirst path (24 MB in + 32 MB out per slot).
constexpr uint64_t kPipeChunk = 1ull << 20;

struct bvhc_mesh {
  int device = 0;
  PairNode* d_nodes = nullptr;
  TriRecord* d_tris = nullptr;
  uint32_t* d_roots = nullptr;
  unsigned int* d_err = nullptr;
  unsigned long long* d_work = nullptr;  // work counter of the persistent raycastFirst kernel
  unsigned long long* d_work_all = nullptr;  // work counter of the persistent raycast (all hits) kernel
  TraversalConfig cfg{1, 1, 16, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  float scene_lo[3] = {0.0f, 0.0f, 0.0f}, scene_hi[3] = {0.0f, 0.0f, 0.0f};  // box of every triangle
  uint64_t n_nodes = 0, n_tris = 0;
  int n_roots = 0;
  int max_depth = 0;
  std::vector<uint32_t> rec_face;   // faceIndex of every triangle record (material labelling)
  // staging buffers for BVHC_MEM_HOST calls (grow-only)
  void* d_in = nullptr;
  size_t in_cap = 0;
  void* d_out = nullptr;
  size_t out_cap = 0;
  void* d_out2 = nullptr;
  size_t out2_cap = 0;
  // pipelined host-memory raycastFirst: kPipes streams, staging slots and work counters (slot 0
  // uses d_work)
  static constexpr int kPipes = 3;
  cudaStream_t pipe[kPipes] = {};
  void* slot_in[kPipes] = {};
  void* slot_out[kPipes] = {};
  unsigned long long* d_work_pipe[kPipes] = {};
  // work queues (grow-only): [0] direct raycastFirst calls, [1], [2], [5] the three pipeline slots
  // (so that concurrently running chunks never share a queue), [3] closestPointToPoint, [4] raycast
  // (all hits), [6] the shapecasts' query order
  static constexpr int kSlots = 7;
  uint32_t* d_queue[kSlots] = {};
  size_t queue_cap[kSlots] = {};
  unsigned int* d_qcount[kSlots] = {};
  // ordering-sort scratch per queue slot (grow-only; sized for sort_cap[slot] queries)
  RaySortScratch sort_s[kSlots] = {};
  uint64_t sort_cap[kSlots] = {};
  // batched meshes (bvhc_batch_create): mesh k owns roots [mesh_root_off[k], mesh_root_off[k+1])
  int n_meshes = 0;
  std::vector<uint32_t> mesh_root_off;
  uint32_t* d_mesh_root_off = nullptr;
  uint64_t* d_ray_off = nullptr;   // per-call ray offsets (n_meshes + 1)
  // gradient support (bvhc_mesh_enable_gradients): triangle -> vertex ids and compact positions
  uint32_t* d_index32 = nullptr;
  float* d_pos = nullptr;
  uint64_t grad_tris = 0, grad_verts = 0;
  // the records as converted from the reference's tree (leaf layout 0), kept on the host so that
  // bvhc_mesh_set_leaf_size can re-lay the device records out; materials follow set_groups
  std::vector<PairNode> h_pairs;
  std::vector<TriRecord> h_tris;
  std::vector<uint32_t> h_roots;
  int h_max_depth = 0;
  // raycastFirst's own copy of the tree with split leaves (bvhc_mesh_set_leaf_size > 0).  Only
  // raycastFirst uses it: its result does not depend on the grouping of triangles into leaves,
  // while closestPointToPoint's maxThreshold / minThreshold rules and raycast's hit order follow
  // the reference's leaves, so those queries keep the records above (closest point on split
  // leaves, with maxThreshold tested at the reference leaf's level, measured slower on every
  // kernel form: per-triangle box culling already prunes inside a leaf).
  int leaf_size = 0;
  PairNode* d_nodes_f = nullptr;
  TriRecord* d_tris_f = nullptr;
  uint32_t* d_roots_f = nullptr;
  uint64_t n_nodes_f = 0, n_tris_f = 0;
  int max_depth_f = 0;
  std::vector<uint32_t> rec_face_f;
  // refit (bvhc_mesh_refit): the serialized root buffers (version 1 layout) with the position of
  // every pair's child boxes in them, the geometry index (empty: non-indexed), and per layout
  // ([0] reference records, [1] raycastFirst's split copy) the bottom-up plan
  std::vector<std::vector<uint8_t>> h_root_bytes;
  std::vector<uint64_t> slot_nodes;
  std::vector<uint32_t> h_index;
  uint64_t n_verts_geo = 0;
  RefitPlan refit[2];
  uint32_t* d_tri_vid = nullptr;
  void* d_refit_pos = nullptr;
  size_t refit_pos_cap = 0;

  // four-child records over raycastFirst's child-pair records (same triangle records), with the
  // child-pair slot each quad child's box comes from
  QuadNode* d_quads = nullptr;
  uint32_t* d_quad_roots = nullptr;
  uint32_t* d_quad_src = nullptr;
  uint64_t n_quads = 0;

  // the records raycastFirst traverses
  MeshDev view_first() const {
    MeshDev v = leaf_size ? MeshDev{d_nodes_f, d_tris_f, d_roots_f, n_roots, d_err} : view();
    v.quads = d_quads;
    v.quad_roots = d_quad_roots;
    v.depth = leaf_size ? max_depth_f : max_depth;
    return v;
  }

  MeshDev view() const {
    MeshDev v{d_nodes, d_tris, d_roots, n_roots, d_err};
    v.depth = max_depth;
    return v;
  }
};

namespace {

struct Status {
  bvhc_status code;
};

bvhc_status from_cuda(cudaError_t e) {
  if (e == cudaSuccess) return BVHC_OK;
  if (e == cudaErrorMemoryAllocation) return BVHC_ERR_OUT_OF_MEMORY;
  return BVHC_ERR_CUDA;
}

#define BVHC_CUDA_TRY(expr)                       \
  do {                                            \
    cudaError_t _e = (expr);                      \
    if (_e != cudaSuccess) return from_cuda(_e);  \
  } while (0)

bool aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

uint32_t read_index(const void* p, int elem, uint64_t i) {
  return elem == 2 ? (uint32_t) static_cast<const uint16_t*>(p)[i] : static_cast<const uint32_t*>(p)[i];
}

// Re-lays one serialized root (buildUtils.js:31-92 layout) into child-pair records and leaf-ordered
// triangle records.  Throws Status on invalid input.
struct Converter {
  const uint8_t* buf = nullptr;
  uint64_t n_nodes = 0;
  int version = 1;
  const void* index;
  int index_elem;
  uint64_t index_count;
  const void* indirect;
  int indirect_elem;
  uint64_t indirect_count;
  const float* pos;
  uint64_t n_verts;
  int stride;
  uint64_t n_prims;      // valid leaf range end
  uint64_t tri_count;    // triangles addressable through the index / positions
  std::vector<PairNode>& pairs;
  std::vector<TriRecord>& tris;
  uint64_t visits = 0;
  int max_depth = 0;
  // where each pair's child boxes live in the serialized buffers: (root << 40) | node, two per pair
  std::vector<uint64_t>* slot_nodes = nullptr;
  uint64_t root_id = 0;
  // a copy of this root's buffer in the current (version 1) format, for reading refit boxes back
  uint8_t* v1_copy = nullptr;

  Converter(std::vector<PairNode>& p, std::vector<TriRecord>& t) : pairs(p), tris(t) {}

  uint32_t u32(uint64_t node, int w) const {
    uint32_t v;
    std::memcpy(&v, buf + node * 32 + w * 4, 4);
    return v;
  }
  uint16_t u16(uint64_t node, int h) const {
    uint16_t v;
    std::memcpy(&v, buf + node * 32 + h * 2, 2);
    return v;
  }
  void box(uint64_t node, float* out) const { std::memcpy(out, buf + node * 32, 24); }
  bool is_leaf(uint64_t node) const { return u16(node, 15) == 0xFFFF; }

  uint64_t right_of(uint64_t node) const {
    uint64_t v = u32(node, 6);
    if (version == 0) {
      // version 0 stored the absolute uint32 offset of the right child (MeshBVH.js:206-230)
      if (v % 8 != 0) throw Status{BVHC_ERR_INVALID_BVH};
      return v / 8;
    }
    return node + v;
  }

  uint32_t emit_leaf(uint64_t node) {
    uint64_t off = u32(node, 6), cnt = u16(node, 14);
    if (off + cnt > n_prims) throw Status{BVHC_ERR_INVALID_BVH};
    if (cnt == 0) return kEmptyLeaf;
    if (tris.size() + cnt >= (uint64_t)kLeafBit) throw Status{BVHC_ERR_UNSUPPORTED};
    uint32_t first = (uint32_t)tris.size();
    for (uint64_t i = off; i < off + cnt; ++i) {
      uint64_t t = indirect ? read_index(indirect, indirect_elem, i) : i;
      if (t >= tri_count) throw Status{BVHC_ERR_INVALID_BVH};
      TriRecord r{};
      for (int k = 0; k < 3; ++k) {
        uint64_t v = index ? read_index(index, index_elem, 3 * t + k) : 3 * t + k;
        if (v >= n_verts) throw Status{BVHC_ERR_INVALID_BVH};
        const float* p = pos + v * (uint64_t)stride;
        r.v[3 * k + 0] = p[0];
        r.v[3 * k + 1] = p[1];
        r.v[3 * k + 2] = p[2];
      }
      r.face = (uint32_t)t;
      r.flags = (i + 1 == off + cnt) ? kTriLast : 0u;
      r.material = kNoMaterial;
      tris.push_back(r);
    }
    return kLeafBit | first;
  }

  uint32_t convert(uint64_t node, int depth) {
    if (++visits > 2 * n_nodes + 2) throw Status{BVHC_ERR_INVALID_BVH};  // shared subtrees
    if (depth >= kMaxStack - 1) throw Status{BVHC_ERR_UNSUPPORTED};
    max_depth = std::max(max_depth, depth);
    if (is_leaf(node)) return emit_leaf(node);
    uint64_t left = node + 1, right = right_of(node);
    uint32_t axis = u32(node, 7);
    if (left >= n_nodes || right >= n_nodes || right <= left || axis > 2) throw Status{BVHC_ERR_INVALID_BVH};
    if (pairs.size() >= (uint64_t)kLeafBit) throw Status{BVHC_ERR_UNSUPPORTED};
    uint32_t idx = (uint32_t)pairs.size();
    pairs.push_back(PairNode{});
    if (slot_nodes) {
      slot_nodes->push_back((root_id << 40) | left);
      slot_nodes->push_back((root_id << 40) | right);
    }
    if (v1_copy && version == 0) {  // the right child as a relative node offset (MeshBVH.js:206-230)
      uint32_t rel = (uint32_t)(right - node);
      std::memcpy(v1_copy + node * 32 + 24, &rel, 4);
    }
    uint32_t ll = convert(left, depth + 1);
    uint32_t lr = convert(right, depth + 1);
    PairNode& p = pairs[idx];
    box(left, &p.f[0]);
    box(right, &p.f[6]);
    p.link[0] = ll;
    p.link[1] = lr;
    p.axis = axis;
    p.flags = 0;
    return idx;
  }
};

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& src) {
  size_t bytes = std::max<size_t>(src.size() * sizeof(T), 16);
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), bytes);
  if (e != cudaSuccess) return e;
  if (!src.empty()) e = cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
  return e;
}

cudaError_t ensure(void** buf, size_t* cap, size_t bytes) {
  if (*cap >= bytes) return cudaSuccess;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc(buf, bytes);
  if (e == cudaSuccess) *cap = bytes;
  return e;
}

void free_sort_scratch(RaySortScratch& s) {
  cudaFree(s.keys[0]);
  cudaFree(s.keys[1]);
  cudaFree(s.vals);
  cudaFree(s.hist);
  cudaFree(s.totals);
  s = RaySortScratch{};
}

SideTable single_side() {
  SideTable t{};
  t.n = 0;
  t.per_material = 0;
  return t;
}

bool material_table(const int8_t* sides, int n, SideTable& t) {
  if (n < 0 || n > kMaxMaterials || (n > 0 && !sides)) return false;
  t = SideTable{};
  for (int i = 0; i < n; ++i) {
    if (sides[i] < BVHC_FRONT_SIDE || sides[i] > BVHC_DOUBLE_SIDE) return false;
    t.side[i] = sides[i];
  }
  t.n = n;
  t.per_material = 1;
  return true;
}

bvhc_status read_and_clear_error(bvhc_mesh* m, cudaStream_t s) {
  unsigned int h = 0;
  BVHC_CUDA_TRY(cudaMemcpyAsync(&h, m->d_err, sizeof h, cudaMemcpyDeviceToHost, s));
  BVHC_CUDA_TRY(cudaStreamSynchronize(s));
  if (h != 0) {
    BVHC_CUDA_TRY(cudaMemsetAsync(m->d_err, 0, sizeof h, s));
    BVHC_CUDA_TRY(cudaStreamSynchronize(s));
    return BVHC_ERR_DEVICE;
  }
  return BVHC_OK;
}

// fn(k, begin, end) over [0, n) in up to kHostThreads pieces of at least 1M elements, one host
// thread each (pieces whose thread cannot start run on the calling thread); returns the number
// of pieces.  Used for the passes over whole index buffers.
constexpr unsigned kHostThreads = 16;
template <class F>
static unsigned parallel_pieces(uint64_t n, F fn) {
  const uint64_t min_piece = 1ull << 20;
  const unsigned hw = std::max(1u, std::min(kHostThreads, std::thread::hardware_concurrency()));
  const unsigned t = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(hw, n / min_piece));
  const uint64_t piece = (n + t - 1) / t;
  std::vector<std::thread> pool;
  for (unsigned k = 1; k < t; ++k) {
    const uint64_t b = std::min(n, k * piece), e = std::min(n, b + piece);
    try {
      pool.emplace_back(fn, k, b, e);
    } catch (...) {
      fn(k, b, e);
    }
  }
  fn(0u, 0ull, std::min(n, piece));
  for (auto& th : pool) th.join();
  return t;
}

void export_width(const std::vector<uint32_t>& src, int elem, std::vector<uint8_t>& dst) {
  dst.resize(src.size() * (size_t)elem);
  parallel_pieces(src.size(), [&](unsigned, uint64_t b, uint64_t e) {
    if (elem == 4) {
      std::memcpy(dst.data() + 4 * b, src.data() + b, (e - b) * 4);
    } else {
      for (uint64_t i = b; i < e; ++i) {
        const uint16_t v = (uint16_t)src[i];
        std::memcpy(dst.data() + 2 * i, &v, 2);
      }
    }
  });
}

// Device leaf layout: every leaf of the reference's tree with more than `max_leaf` triangles becomes
// a subtree of child-pair records over its triangles (the reference's tree above it is kept as is).
// A range is split at the median of the triangle centroids along the longest axis of the centroid
// bounds (ties in input order), and each side gets the exact float32 bounds of its vertices.  Only
// the grouping of triangles into leaves changes; which triangle is nearest does not, so results are
// the same up to exact ties.
struct LeafSplitter {
  const std::vector<PairNode>& pairs;
  const std::vector<TriRecord>& tris;
  int max_leaf;
  std::vector<PairNode> out_pairs;
  std::vector<TriRecord> out_tris;
  int max_depth = 0;

  static void bounds(const TriRecord* t, size_t n, float* box) {
    for (int a = 0; a < 3; ++a) {
      box[a] = t[0].v[a];
      box[3 + a] = t[0].v[a];
    }
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) {
          box[a] = std::min(box[a], t[i].v[3 * k + a]);
          box[3 + a] = std::max(box[3 + a], t[i].v[3 * k + a]);
        }
  }

  uint32_t split(std::vector<TriRecord>& run, size_t lo, size_t hi, int depth) {
    if (depth >= kMaxStack - 1) throw Status{BVHC_ERR_UNSUPPORTED};
    max_depth = std::max(max_depth, depth);
    const size_t n = hi - lo;
    if ((int)n <= max_leaf) {
      uint32_t first = (uint32_t)out_tris.size();
      if (out_tris.size() + n >= (uint64_t)kLeafBit) throw Status{BVHC_ERR_UNSUPPORTED};
      for (size_t i = lo; i < hi; ++i) {
        TriRecord r = run[i];
        r.flags = (i + 1 == hi) ? kTriLast : 0u;
        out_tris.push_back(r);
      }
      return kLeafBit | first;
    }
    float c_lo[3], c_hi[3];
    auto centroid = [](const TriRecord& t, int a) { return t.v[a] + t.v[3 + a] + t.v[6 + a]; };
    for (int a = 0; a < 3; ++a) c_lo[a] = c_hi[a] = centroid(run[lo], a);
    for (size_t i = lo; i < hi; ++i)
      for (int a = 0; a < 3; ++a) {
        c_lo[a] = std::min(c_lo[a], centroid(run[i], a));
        c_hi[a] = std::max(c_hi[a], centroid(run[i], a));
      }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (c_hi[a] - c_lo[a] > c_hi[axis] - c_lo[axis]) axis = a;
    std::stable_sort(run.begin() + lo, run.begin() + hi, [&](const TriRecord& x, const TriRecord& y) {
      return centroid(x, axis) < centroid(y, axis);
    });
    const size_t mid = lo + n / 2;
    if (out_pairs.size() >= (uint64_t)kLeafBit) throw Status{BVHC_ERR_UNSUPPORTED};
    uint32_t idx = (uint32_t)out_pairs.size();
    out_pairs.push_back(PairNode{});
    uint32_t ll = split(run, lo, mid, depth + 1);
    uint32_t lr = split(run, mid, hi, depth + 1);
    PairNode& p = out_pairs[idx];
    bounds(run.data() + lo, mid - lo, &p.f[0]);
    bounds(run.data() + mid, hi - mid, &p.f[6]);
    p.link[0] = ll;
    p.link[1] = lr;
    p.axis = (uint32_t)axis;
    p.flags = 0;
    return idx;
  }

  uint32_t copy(uint32_t link, int depth) {
    if (link == kEmptyLeaf) return kEmptyLeaf;
    if (link & kLeafBit) {
      uint32_t k = link & ~kLeafBit;
      std::vector<TriRecord> run;
      for (;; ++k) {
        run.push_back(tris[k]);
        if (tris[k].flags & kTriLast) break;
      }
      return split(run, 0, run.size(), depth);
    }
    if (depth >= kMaxStack - 1) throw Status{BVHC_ERR_UNSUPPORTED};
    max_depth = std::max(max_depth, depth);
    uint32_t idx = (uint32_t)out_pairs.size();
    out_pairs.push_back(pairs[link]);
    uint32_t ll = copy(pairs[link].link[0], depth + 1);
    uint32_t lr = copy(pairs[link].link[1], depth + 1);
    out_pairs[idx].link[0] = ll;
    out_pairs[idx].link[1] = lr;
    return idx;
  }
};

// Four-child records from a child-pair tree: starting from a pair's two children, the internal
// child with the largest box surface area is replaced by its own two children until there are
// four children or only leaves.  `src` keeps, per quad child, the child-pair slot its box comes
// from (2 * pair + side; kEmptyLeaf for an unused child), so refits can copy boxes over.
struct QuadBuilder {
  const std::vector<PairNode>& pairs;
  std::vector<QuadNode> quads;
  std::vector<uint32_t> src;

  static float area(const float* b) {
    float dx = std::max(b[3] - b[0], 0.0f), dy = std::max(b[4] - b[1], 0.0f), dz = std::max(b[5] - b[2], 0.0f);
    return dx * dy + dy * dz + dz * dx;
  }

  uint32_t build(uint32_t pair) {
    struct Child {
      uint32_t link, slot;
      const float* box;
    };
    Child ch[4];
    int n = 2;
    ch[0] = {pairs[pair].link[0], 2 * pair, pairs[pair].f};
    ch[1] = {pairs[pair].link[1], 2 * pair + 1, pairs[pair].f + 6};
    while (n < 4) {
      int pick = -1;
      float best = -1.0f;
      for (int k = 0; k < n; ++k) {
        if (ch[k].link & kLeafBit) continue;
        float a = area(ch[k].box);
        if (a > best) {
          best = a;
          pick = k;
        }
      }
      if (pick < 0) break;
      const uint32_t p = ch[pick].link;
      ch[pick] = {pairs[p].link[0], 2 * p, pairs[p].f};
      ch[n++] = {pairs[p].link[1], 2 * p + 1, pairs[p].f + 6};
    }
    if (quads.size() >= (uint64_t)kLeafBit) throw Status{BVHC_ERR_UNSUPPORTED};
    const uint32_t idx = (uint32_t)quads.size();
    quads.push_back(QuadNode{});
    src.resize(4 * (size_t)(idx + 1), kEmptyLeaf);
    for (int k = 0; k < 4; ++k) {
      QuadNode& q = quads[idx];
      if (k < n) {
        for (int a = 0; a < 3; ++a) {
          q.lo[a][k] = ch[k].box[a];
          q.hi[a][k] = ch[k].box[3 + a];
        }
        q.link[k] = ch[k].link;
        src[4 * (size_t)idx + k] = ch[k].slot;
      } else {
        q.link[k] = kEmptyLeaf;
      }
    }
    for (int k = 0; k < n; ++k)
      if (!(ch[k].link & kLeafBit)) {
        uint32_t q = build(ch[k].link);
        quads[idx].link[k] = q;
      }
    return idx;
  }
};

}  // namespace

bool bvhc::mesh_launch_info(const bvhc_mesh* m, MeshDev* view, TraversalConfig* cfg, int* device) {
  if (!m) return false;
  *view = m->view_first();
  *cfg = m->cfg;
  *device = m->device;
  return true;
}

// Uploads converted records and allocates the per-mesh device state.  mesh_root_off is empty for a
// single mesh, or the n_meshes + 1 root offsets of a batch.
static bvhc_status finish_mesh(int device, const std::vector<PairNode>& pairs, const std::vector<TriRecord>& tris,
                               const std::vector<uint32_t>& root_links, int max_depth,
                               const std::vector<uint32_t>& mesh_root_off, bvhc_mesh** out) {
  auto* m = new bvhc_mesh();
  m->device = device;
  m->n_nodes = pairs.size();
  m->n_tris = tris.size();
  if (!tris.empty()) {
    for (int a = 0; a < 3; ++a) m->scene_lo[a] = m->scene_hi[a] = tris[0].v[a];
    for (const TriRecord& t : tris)
      for (int k = 0; k < 3; ++k)
        for (int a = 0; a < 3; ++a) {
          m->scene_lo[a] = std::min(m->scene_lo[a], t.v[3 * k + a]);
          m->scene_hi[a] = std::max(m->scene_hi[a], t.v[3 * k + a]);
        }
  }
  m->n_roots = (int)root_links.size();
  m->max_depth = max_depth;
  m->rec_face.resize(tris.size());
  for (size_t k = 0; k < tris.size(); ++k) m->rec_face[k] = tris[k].face;
  m->mesh_root_off = mesh_root_off;
  m->n_meshes = mesh_root_off.empty() ? 0 : (int)mesh_root_off.size() - 1;
  m->h_pairs = pairs;
  m->h_tris = tris;
  m->h_roots = root_links;
  m->h_max_depth = max_depth;
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = upload(&m->d_nodes, pairs);
  if (e == cudaSuccess) e = upload(&m->d_tris, tris);
  if (e == cudaSuccess) e = upload(&m->d_roots, root_links);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&m->d_err), sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&m->d_work), sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemset(m->d_err, 0, sizeof(unsigned int));
  if (e == cudaSuccess && m->n_meshes > 0) {
    e = upload(&m->d_mesh_root_off, mesh_root_off);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&m->d_ray_off), mesh_root_off.size() * 8);
  }
  if (e != cudaSuccess) {
    bvhc_mesh_destroy(m);
    return from_cuda(e);
  }
  *out = m;
  return BVHC_OK;
}

// Keeps what a refit needs on the host: the serialized roots (version 1 layout), where each pair's
// child boxes sit in them, and the geometry index as uint32.
static void keep_serialized(bvhc_mesh* m, std::vector<std::vector<uint8_t>> roots, std::vector<uint64_t> slot_nodes,
                            const void* index, int index_elem, uint64_t index_count, uint64_t n_verts) {
  m->h_root_bytes = std::move(roots);
  m->slot_nodes = std::move(slot_nodes);
  m->n_verts_geo = n_verts;
  if (index) {
    m->h_index.resize(index_count);
    for (uint64_t i = 0; i < index_count; ++i) m->h_index[i] = read_index(index, index_elem, i);
  }
}

// Four-child records over raycastFirst's child-pair layout (pairs + roots), replacing any before.
static cudaError_t install_quads(bvhc_mesh* m, const std::vector<PairNode>& pairs, const std::vector<uint32_t>& roots) {
  QuadBuilder qb{pairs};
  std::vector<uint32_t> qroots(roots.size());
  try {
    for (size_t r = 0; r < roots.size(); ++r) qroots[r] = (roots[r] & kLeafBit) ? roots[r] : qb.build(roots[r]);
  } catch (const Status&) {
    return cudaErrorInvalidValue;
  } catch (const std::bad_alloc&) {
    return cudaErrorMemoryAllocation;
  }
  QuadNode* q = nullptr;
  uint32_t *qr = nullptr, *qs = nullptr;
  cudaError_t e = upload(&q, qb.quads);
  if (e == cudaSuccess) e = upload(&qr, qroots);
  if (e == cudaSuccess) e = upload(&qs, qb.src);
  if (e != cudaSuccess) {
    cudaFree(q);
    cudaFree(qr);
    cudaFree(qs);
    return e;
  }
  cudaFree(m->d_quads);
  cudaFree(m->d_quad_roots);
  cudaFree(m->d_quad_src);
  m->d_quads = q;
  m->d_quad_roots = qr;
  m->d_quad_src = qs;
  m->n_quads = qb.quads.size();
  return cudaSuccess;
}

// 3 vertex ids per triangle on the device, from the geometry index (or 3t + k without one).
static cudaError_t ensure_tri_vid(bvhc_mesh* m) {
  if (m->d_tri_vid) return cudaSuccess;
  uint64_t n_tri = m->h_index.empty() ? m->n_verts_geo / 3 : m->h_index.size() / 3;
  std::vector<uint32_t> vid(3 * n_tri);
  for (uint64_t i = 0; i < vid.size(); ++i) vid[i] = m->h_index.empty() ? (uint32_t)i : m->h_index[i];
  return upload(&m->d_tri_vid, vid);
}

static void free_refit_plan(RefitPlan& p) {
  cudaFree(p.leaves);
  cudaFree(p.parent);
  cudaFree(p.arrive);
  cudaFree(p.flags);
  cudaFree(p.root_box);
  p = RefitPlan{};
}

// The bottom-up plan of one record layout: every leaf (a leaf child of a pair, or a root that is a
// leaf) with its triangle-record run and box slot, and every pair's parent slot.  root_boxes: 6
// floats per root (the roots' own boxes, which the child-pair records do not hold).
static cudaError_t build_refit_plan(const std::vector<PairNode>& pairs, const std::vector<TriRecord>& tris,
                                    const std::vector<uint32_t>& roots, const std::vector<float>& root_boxes,
                                    RefitPlan& plan) {
  std::vector<RefitLeaf> leaves;
  std::vector<uint32_t> parent(pairs.size(), kRootSlot);
  auto leaf_of = [&](uint32_t link, uint32_t slot) {
    RefitLeaf l{0, 0, slot};
    if (link != kEmptyLeaf) {
      l.first = link & ~kLeafBit;
      uint32_t k = l.first;
      while (!(tris[k].flags & kTriLast)) ++k;
      l.count = k - l.first + 1;
    }
    leaves.push_back(l);
  };
  for (size_t p = 0; p < pairs.size(); ++p)
    for (uint32_t s = 0; s < 2; ++s) {
      uint32_t link = pairs[p].link[s];
      uint32_t slot = (uint32_t)(2 * p + s);
      if (link & kLeafBit) leaf_of(link, slot);
      else parent[link] = slot;
    }
  for (size_t r = 0; r < roots.size(); ++r) {
    uint32_t slot = kRootSlot | (uint32_t)r;
    if (roots[r] & kLeafBit) leaf_of(roots[r], slot);
    else parent[roots[r]] = slot;
  }
  RefitPlan np;
  np.n_leaves = (uint32_t)leaves.size();
  np.n_pairs = (uint32_t)pairs.size();
  cudaError_t e = upload(&np.leaves, leaves);
  if (e == cudaSuccess) e = upload(&np.parent, parent);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&np.arrive), std::max<size_t>(pairs.size(), 1) * 4);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&np.flags), std::max<size_t>(pairs.size(), 1) * 4);
  if (e == cudaSuccess) e = upload(&np.root_box, root_boxes);
  if (e != cudaSuccess) {
    free_refit_plan(np);
    return e;
  }
  free_refit_plan(plan);
  plan = np;
  return cudaSuccess;
}

// The roots' own boxes, from the kept serialized buffers (node 0 of each root).
static std::vector<float> serialized_root_boxes(const bvhc_mesh* m) {
  std::vector<float> boxes(6 * m->h_root_bytes.size());
  for (size_t r = 0; r < m->h_root_bytes.size(); ++r) std::memcpy(&boxes[6 * r], m->h_root_bytes[r].data(), 24);
  return boxes;
}

extern "C" {

const char* bvhc_status_string(bvhc_status s) {
  switch (s) {
    case BVHC_OK: return "ok";
    case BVHC_ERR_INVALID_ARGUMENT: return "invalid argument";
    case BVHC_ERR_INVALID_BVH: return "invalid BVH buffer";
    case BVHC_ERR_CUDA: return "CUDA runtime error";
    case BVHC_ERR_OUT_OF_MEMORY: return "out of device memory";
    case BVHC_ERR_DEVICE: return "device-side error (traversal stack overflow)";
    case BVHC_ERR_UNSUPPORTED: return "unsupported input (tree deeper than the traversal stack, or too large)";
    case BVHC_ERR_BUILD: return "BVH build failed";
    case BVHC_ERR_SCRATCH_LIMIT:
      return "request exceeds the fixed scratch of bvhc_raycast_first_noalloc (at most 65536 host-memory rays)";
  }
  return "unknown status";
}

static bvhc_status build_impl(const float* positions, uint64_t n_verts, int stride_floats, const void* index,
                              int index_elem_bytes, uint64_t index_count, const int64_t* groups, int n_groups,
                              int64_t range_start, int64_t range_count, int strategy, int max_depth,
                              int target_leaf_size, int indirect, bool on_device, int device, void* stream,
                              bvhc_serialized** out) {
  if (!out || !positions || stride_floats < 3 || n_verts == 0) return BVHC_ERR_INVALID_ARGUMENT;
  if (index && index_elem_bytes != 2 && index_elem_bytes != 4) return BVHC_ERR_INVALID_ARGUMENT;
  if (strategy < BVHC_CENTER || strategy > BVHC_SAH || max_depth < 0 || target_leaf_size < 0) return BVHC_ERR_INVALID_ARGUMENT;
  if (n_groups > 0 && !groups) return BVHC_ERR_INVALID_ARGUMENT;
  if (on_device && strategy == BVHC_AVERAGE) return BVHC_ERR_UNSUPPORTED;
  *out = nullptr;
  try {
    auto* s = new bvhc_serialized();
    if (index) {
      s->has_index = true;
      s->index_elem_bytes = index_elem_bytes;
      s->index.resize(index_count);
      uint32_t tops[kHostThreads] = {};
      const unsigned pieces = parallel_pieces(index_count, [&](unsigned k, uint64_t b, uint64_t e) {
        uint32_t top = 0;
        if (index_elem_bytes == 4) {
          const uint32_t* p32 = static_cast<const uint32_t*>(index);
          for (uint64_t i = b; i < e; ++i) top = std::max(top, s->index[i] = p32[i]);
        } else {
          const uint16_t* p16 = static_cast<const uint16_t*>(index);
          for (uint64_t i = b; i < e; ++i) top = std::max(top, s->index[i] = p16[i]);
        }
        tops[k] = top;
      });
      uint32_t top = 0;
      for (unsigned k = 0; k < pieces; ++k) top = std::max(top, tops[k]);
      if (index_count && top >= n_verts) { delete s; return BVHC_ERR_INVALID_ARGUMENT; }
    }
    try {
      if (on_device)
        build_serialized_device(*s, positions, n_verts, stride_floats, groups, n_groups, range_start, range_count,
                                strategy, max_depth, target_leaf_size, indirect != 0, device, stream);
      else
        build_serialized(*s, positions, n_verts, stride_floats, groups, n_groups, range_start, range_count, strategy,
                         max_depth, target_leaf_size, indirect != 0);
    } catch (const std::bad_alloc&) {
      delete s;
      return BVHC_ERR_OUT_OF_MEMORY;
    } catch (const DeviceBuildError&) {
      delete s;
      return BVHC_ERR_CUDA;
    } catch (...) {
      delete s;
      return BVHC_ERR_BUILD;
    }
    if (s->has_index) export_width(s->index, s->index_elem_bytes, s->index_bytes);
    if (s->indirect) export_width(s->indirect_buf, s->indirect_elem_bytes, s->indirect_bytes);
    *out = s;
    return BVHC_OK;
  } catch (const std::bad_alloc&) {
    return BVHC_ERR_OUT_OF_MEMORY;
  }
}

bvhc_status bvhc_build(const float* positions, uint64_t n_verts, int stride_floats, const void* index,
                       int index_elem_bytes, uint64_t index_count, const int64_t* groups, int n_groups,
                       int64_t range_start, int64_t range_count, int strategy, int max_depth, int target_leaf_size,
                       int indirect, bvhc_serialized** out) {
  return build_impl(positions, n_verts, stride_floats, index, index_elem_bytes, index_count, groups, n_groups,
                    range_start, range_count, strategy, max_depth, target_leaf_size, indirect, false, 0, nullptr, out);
}

bvhc_status bvhc_build_device(const float* positions, uint64_t n_verts, int stride_floats, const void* index,
                              int index_elem_bytes, uint64_t index_count, const int64_t* groups, int n_groups,
                              int64_t range_start, int64_t range_count, int strategy, int max_depth,
                              int target_leaf_size, int indirect, int device, void* stream, bvhc_serialized** out) {
  return build_impl(positions, n_verts, stride_floats, index, index_elem_bytes, index_count, groups, n_groups,
                    range_start, range_count, strategy, max_depth, target_leaf_size, indirect, true, device, stream,
                    out);
}

int bvhc_serialized_root_count(const bvhc_serialized* s) { return s ? (int)s->roots.size() : 0; }

bvhc_status bvhc_serialized_root(const bvhc_serialized* s, int i, const void** data, uint64_t* bytes) {
  if (!s || !data || !bytes || i < 0 || i >= (int)s->roots.size()) return BVHC_ERR_INVALID_ARGUMENT;
  *data = s->roots[i].data();
  *bytes = s->roots[i].size();
  return BVHC_OK;
}

bvhc_status bvhc_serialized_index(const bvhc_serialized* s, const void** data, int* elem_bytes, uint64_t* count) {
  if (!s || !data || !elem_bytes || !count) return BVHC_ERR_INVALID_ARGUMENT;
  *data = s->has_index ? s->index_bytes.data() : nullptr;
  *elem_bytes = s->has_index ? s->index_elem_bytes : 0;
  *count = s->has_index ? s->index.size() : 0;
  return BVHC_OK;
}

bvhc_status bvhc_serialized_indirect(const bvhc_serialized* s, const void** data, int* elem_bytes, uint64_t* count) {
  if (!s || !data || !elem_bytes || !count) return BVHC_ERR_INVALID_ARGUMENT;
  *data = s->indirect ? s->indirect_bytes.data() : nullptr;
  *elem_bytes = s->indirect ? s->indirect_elem_bytes : 0;
  *count = s->indirect ? s->indirect_buf.size() : 0;
  return BVHC_OK;
}

void bvhc_serialized_free(bvhc_serialized* s) { delete s; }

bvhc_status bvhc_mesh_create(int device, int version, const void* const* roots, const uint64_t* root_bytes,
                             int n_roots, const void* index, int index_elem_bytes, uint64_t index_count,
                             const void* indirect, int indirect_elem_bytes, uint64_t indirect_count,
                             const float* positions, uint64_t n_verts, int stride_floats, bvhc_mesh** out) {
  if (!out || !roots || !root_bytes || n_roots <= 0 || !positions || stride_floats < 3 || n_verts == 0)
    return BVHC_ERR_INVALID_ARGUMENT;
  if (version != 0 && version != 1) return BVHC_ERR_INVALID_ARGUMENT;
  if (index && index_elem_bytes != 2 && index_elem_bytes != 4) return BVHC_ERR_INVALID_ARGUMENT;
  if (indirect && indirect_elem_bytes != 2 && indirect_elem_bytes != 4) return BVHC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::vector<PairNode> pairs;
  std::vector<TriRecord> tris;
  std::vector<uint32_t> root_links;
  std::vector<uint64_t> slot_nodes;
  std::vector<std::vector<uint8_t>> copies;
  int max_depth = 0;
  try {
    for (int r = 0; r < n_roots; ++r) {
      if (!roots[r] || root_bytes[r] == 0 || root_bytes[r] % 32 != 0) return BVHC_ERR_INVALID_BVH;
      Converter c(pairs, tris);
      const uint8_t* src = static_cast<const uint8_t*>(roots[r]);
      copies.emplace_back(src, src + root_bytes[r]);
      c.slot_nodes = &slot_nodes;
      c.root_id = (uint64_t)r;
      c.v1_copy = copies.back().data();
      c.buf = static_cast<const uint8_t*>(roots[r]);
      c.n_nodes = root_bytes[r] / 32;
      c.version = version;
      c.index = index;
      c.index_elem = index_elem_bytes;
      c.index_count = index_count;
      c.indirect = indirect;
      c.indirect_elem = indirect_elem_bytes;
      c.indirect_count = indirect_count;
      c.pos = positions;
      c.n_verts = n_verts;
      c.stride = stride_floats;
      c.tri_count = index ? index_count / 3 : n_verts / 3;
      c.n_prims = indirect ? indirect_count : c.tri_count;
      root_links.push_back(c.convert(0, 0));
      max_depth = std::max(max_depth, c.max_depth);
    }
  } catch (const Status& s) {
    return s.code;
  } catch (const std::bad_alloc&) {
    return BVHC_ERR_OUT_OF_MEMORY;
  }
  bvhc_status st = finish_mesh(device, pairs, tris, root_links, max_depth, {}, out);
  if (st == BVHC_OK) {
    keep_serialized(*out, std::move(copies), std::move(slot_nodes), index, index_elem_bytes, index_count, n_verts);
    cudaError_t e = install_quads(*out, (*out)->h_pairs, (*out)->h_roots);
    if (e != cudaSuccess) {
      bvhc_mesh_destroy(*out);
      *out = nullptr;
      return from_cuda(e);
    }
  }
  return st;
}

bvhc_status bvhc_batch_create(int device, int n_meshes, const int32_t* roots_per_mesh, const void* const* roots,
                              const uint64_t* root_bytes, const void* index, int index_elem_bytes,
                              uint64_t index_count, const float* positions, uint64_t n_verts, int stride_floats,
                              bvhc_mesh** out) {
  if (!out || n_meshes <= 0 || !roots_per_mesh || !roots || !root_bytes || !positions || stride_floats < 3 ||
      n_verts == 0)
    return BVHC_ERR_INVALID_ARGUMENT;
  if (index && index_elem_bytes != 2 && index_elem_bytes != 4) return BVHC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::vector<PairNode> pairs;
  std::vector<TriRecord> tris;
  std::vector<uint32_t> root_links;
  std::vector<uint32_t> mesh_root_off{0};
  std::vector<uint64_t> slot_nodes;
  std::vector<std::vector<uint8_t>> copies;
  int max_depth = 0;
  try {
    int r = 0;
    for (int k = 0; k < n_meshes; ++k) {
      if (roots_per_mesh[k] <= 0) return BVHC_ERR_INVALID_ARGUMENT;
      for (int j = 0; j < roots_per_mesh[k]; ++j, ++r) {
        if (!roots[r] || root_bytes[r] == 0 || root_bytes[r] % 32 != 0) return BVHC_ERR_INVALID_BVH;
        Converter c(pairs, tris);
        const uint8_t* src = static_cast<const uint8_t*>(roots[r]);
        copies.emplace_back(src, src + root_bytes[r]);
        c.slot_nodes = &slot_nodes;
        c.root_id = (uint64_t)r;
        c.v1_copy = copies.back().data();
        c.buf = static_cast<const uint8_t*>(roots[r]);
        c.n_nodes = root_bytes[r] / 32;
        c.version = 1;
        c.index = index;
        c.index_elem = index_elem_bytes;
        c.index_count = index_count;
        c.indirect = nullptr;
        c.indirect_elem = 0;
        c.indirect_count = 0;
        c.pos = positions;
        c.n_verts = n_verts;
        c.stride = stride_floats;
        c.tri_count = index ? index_count / 3 : n_verts / 3;
        c.n_prims = c.tri_count;
        root_links.push_back(c.convert(0, 0));
        max_depth = std::max(max_depth, c.max_depth);
      }
      mesh_root_off.push_back((uint32_t)root_links.size());
    }
  } catch (const Status& s) {
    return s.code;
  } catch (const std::bad_alloc&) {
    return BVHC_ERR_OUT_OF_MEMORY;
  }
  bvhc_status st = finish_mesh(device, pairs, tris, root_links, max_depth, mesh_root_off, out);
  if (st == BVHC_OK) {
    keep_serialized(*out, std::move(copies), std::move(slot_nodes), index, index_elem_bytes, index_count, n_verts);
    cudaError_t e = install_quads(*out, (*out)->h_pairs, (*out)->h_roots);
    if (e != cudaSuccess) {
      bvhc_mesh_destroy(*out);
      *out = nullptr;
      return from_cuda(e);
    }
  }
  return st;
}

void bvhc_mesh_destroy(bvhc_mesh* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  cudaFree(m->d_nodes);
  cudaFree(m->d_tris);
  cudaFree(m->d_roots);
  cudaFree(m->d_nodes_f);
  cudaFree(m->d_tris_f);
  cudaFree(m->d_roots_f);
  free_refit_plan(m->refit[0]);
  free_refit_plan(m->refit[1]);
  cudaFree(m->d_quads);
  cudaFree(m->d_quad_roots);
  cudaFree(m->d_quad_src);
  cudaFree(m->d_tri_vid);
  cudaFree(m->d_refit_pos);
  cudaFree(m->d_err);
  cudaFree(m->d_work);
  cudaFree(m->d_work_all);
  cudaFree(m->d_in);
  cudaFree(m->d_out);
  cudaFree(m->d_out2);
  for (int k = 0; k < bvhc_mesh::kPipes; ++k) {
    cudaFree(m->slot_in[k]);
    cudaFree(m->slot_out[k]);
    if (m->pipe[k]) cudaStreamDestroy(m->pipe[k]);
    if (k > 0) cudaFree(m->d_work_pipe[k]);
  }
  cudaFree(m->d_mesh_root_off);
  cudaFree(m->d_ray_off);
  cudaFree(m->d_index32);
  cudaFree(m->d_pos);
  for (int k = 0; k < bvhc_mesh::kSlots; ++k) {
    cudaFree(m->d_queue[k]);
    cudaFree(m->d_qcount[k]);
    free_sort_scratch(m->sort_s[k]);
  }
  delete m;
}

bvhc_status bvhc_mesh_get_info(const bvhc_mesh* m, bvhc_mesh_info* info) {
  if (!m || !info) return BVHC_ERR_INVALID_ARGUMENT;
  // the records raycastFirst traverses (the split-leaf copy when one is installed)
  const bool f = m->leaf_size > 0;
  info->node_records = f ? m->n_nodes_f : m->n_nodes;
  info->triangle_records = f ? m->n_tris_f : m->n_tris;
  info->device_bytes = m->n_nodes * sizeof(PairNode) + m->n_tris * sizeof(TriRecord) + m->n_roots * 4 + 4 +
                       (f ? m->n_nodes_f * sizeof(PairNode) + m->n_tris_f * sizeof(TriRecord) + m->n_roots * 4 : 0);
  info->max_depth = f ? m->max_depth_f : m->max_depth;
  info->root_count = m->n_roots;
  return BVHC_OK;
}

bvhc_status bvhc_mesh_synchronize(bvhc_mesh* m, void* stream) {
  if (!m) return BVHC_ERR_INVALID_ARGUMENT;
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  return read_and_clear_error(m, static_cast<cudaStream_t>(stream));
}

static cudaError_t ensure_sort_scratch(bvhc_mesh* m, int slot, uint64_t n) {
  if (m->sort_cap[slot] >= n) return cudaSuccess;
  RaySortScratch& s = m->sort_s[slot];
  free_sort_scratch(s);
  m->sort_cap[slot] = 0;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&s.keys[0]), n * 4);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s.keys[1]), n * 4);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s.vals), n * 4);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s.hist), 256 * ray_sort_tiles(n) * 4);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&s.totals), 4 * 256 * 4);
  if (e != cudaSuccess) {
    free_sort_scratch(s);
    return e;
  }
  m->sort_cap[slot] = n;
  return cudaSuccess;
}

// Compaction queue `slot` with room for n rays when the mesh's variant uses one (persistent or
// warp-cooperative form with compaction or ordering), else nulls; `sort` is filled when the variant
// orders the queue (single meshes only) and left untouched otherwise.
static cudaError_t queue_for(bvhc_mesh* m, int slot, uint64_t n, uint32_t** queue, unsigned int** qcount,
                             RaySort* sort = nullptr, bool* sorted = nullptr) {
  *queue = nullptr;
  *qcount = nullptr;
  if (sorted) *sorted = false;
  if (!m->cfg.persistent || !(m->cfg.compact || m->cfg.sort) || n >= (1ull << 32)) return cudaSuccess;
  cudaError_t e = ensure(reinterpret_cast<void**>(&m->d_queue[slot]), &m->queue_cap[slot], n * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  if (!m->d_qcount[slot]) {
    e = cudaMalloc(reinterpret_cast<void**>(&m->d_qcount[slot]), sizeof(unsigned int));
    if (e != cudaSuccess) return e;
  }
  *queue = m->d_queue[slot];
  *qcount = m->d_qcount[slot];
  if (sort && sorted && m->cfg.sort && m->n_meshes == 0) {
    e = ensure_sort_scratch(m, slot, n);
    if (e != cudaSuccess) return e;
    sort->kind = m->cfg.sort;
    for (int a = 0; a < 3; ++a) {
      sort->lo[a] = m->scene_lo[a];
      sort->hi[a] = m->scene_hi[a];
    }
    sort->scratch = m->sort_s[slot];
    *sorted = true;
  }
  return cudaSuccess;
}

static cudaError_t dispatch_first(bvhc_mesh* m, const float* rays, uint64_t n, int side, const SideTable& tab,
                                  float near_d, float far_d, bvhc_hit* out, unsigned long long* work, cudaStream_t s,
                                  int qslot = 0) {
  if (m->cfg.persistent) {
    uint32_t* q;
    unsigned int* qc;
    RaySort sort{};
    bool sorted = false;
    cudaError_t e = queue_for(m, qslot, n, &q, &qc, &sort, &sorted);
    if (e != cudaSuccess) return e;
    if (m->cfg.persistent == 2)
      return launch_raycast_first_packet(m->view_first(), rays, n, side, tab, near_d, far_d, out, m->cfg, s, q, qc,
                                         sorted ? &sort : nullptr);
    return launch_raycast_first_persistent(m->view_first(), nullptr, rays, n, side, tab, near_d, far_d, out, work,
                                           m->cfg, s, q, qc, sorted ? &sort : nullptr);
  }
  return launch_raycast_first(m->view_first(), rays, n, side, tab, near_d, far_d, out, m->cfg.order, s);
}

// raycastFirst over one mesh of a batch (view = that mesh's roots), with the batch's variant.
static cudaError_t dispatch_view(bvhc_mesh* m, const MeshDev& v, const float* rays, uint64_t n, int side,
                                 float near_d, float far_d, bvhc_hit* out, cudaStream_t s) {
  if (m->cfg.persistent == 2)
    return launch_raycast_first_packet(v, rays, n, side, single_side(), near_d, far_d, out, m->cfg, s);
  if (m->cfg.persistent) {
    uint32_t* q;
    unsigned int* qc;
    cudaError_t e = queue_for(m, 0, n, &q, &qc);
    if (e != cudaSuccess) return e;
    return launch_raycast_first_persistent(v, nullptr, rays, n, side, single_side(), near_d, far_d, out, m->d_work,
                                           m->cfg, s, q, qc);
  }
  return launch_raycast_first(v, rays, n, side, single_side(), near_d, far_d, out, m->cfg.order, s);
}

// Streams, staging slots and the second work counter of the pipelined host-memory path.
static cudaError_t ensure_pipeline(bvhc_mesh* m) {
  for (int k = 0; k < bvhc_mesh::kPipes; ++k) {
    if (!m->pipe[k]) {
      cudaError_t e = cudaStreamCreateWithFlags(&m->pipe[k], cudaStreamNonBlocking);
      if (e != cudaSuccess) return e;
    }
    size_t cap_in = 0, cap_out = 0;
    if (m->slot_in[k] == nullptr) {
      cudaError_t e = ensure(&m->slot_in[k], &cap_in, kPipeChunk * 24);
      if (e != cudaSuccess) return e;
    }
    if (m->slot_out[k] == nullptr) {
      cudaError_t e = ensure(&m->slot_out[k], &cap_out, kPipeChunk * sizeof(bvhc_hit));
      if (e != cudaSuccess) return e;
    }
    if (k == 0) {
      m->d_work_pipe[0] = m->d_work;
    } else if (!m->d_work_pipe[k]) {
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&m->d_work_pipe[k]), sizeof(unsigned long long));
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

static bool valid_config(const bvhc_traversal_config* cfg) {
  return cfg && cfg->persistent >= 0 && cfg->persistent <= 2 && (cfg->order == 0 || cfg->order == 1) &&
         cfg->refill >= 1 && cfg->refill <= 32 && cfg->occupancy >= 0 && cfg->occupancy <= 2 &&
         (cfg->compact == 0 || cfg->compact == 1) && cfg->sort >= 0 && cfg->sort <= 3 && cfg->closest >= 0 &&
         cfg->closest <= 6 && (cfg->wide == 0 || cfg->wide == 1) && cfg->all >= 0 && cfg->all <= 12 &&
         (cfg->tile == 0 || (cfg->tile >= 8 && cfg->tile <= (1 << 24) && cfg->tile % 8 == 0)) &&
         (cfg->tile_rows == 0 || cfg->tile_rows == 2 || cfg->tile_rows == 4 || cfg->tile_rows == 8) &&
         (cfg->tile == 0 || cfg->tile % (32 >> tile_rows_log2(cfg->tile_rows)) == 0) &&
         (cfg->block == 0 || cfg->block == 64 || cfg->block == 128 || cfg->block == 256) &&
         (cfg->stack == 0 || cfg->stack == 32 || cfg->stack == 64);
}

bvhc_status bvhc_mesh_set_traversal(bvhc_mesh* m, const bvhc_traversal_config* cfg) {
  if (!m || !valid_config(cfg)) return BVHC_ERR_INVALID_ARGUMENT;
  m->cfg = TraversalConfig{cfg->persistent, cfg->order, cfg->refill, cfg->occupancy, cfg->compact,
                           cfg->sort,       cfg->closest, cfg->wide, cfg->all,       cfg->tile,
                           cfg->block,      cfg->stack,   cfg->tile_rows};
  return BVHC_OK;
}

bvhc_status bvhc_mesh_set_leaf_size(bvhc_mesh* m, int max_leaf) {
  if (!m || max_leaf < 0 || max_leaf > 0xFFFF) return BVHC_ERR_INVALID_ARGUMENT;
  if (max_leaf == m->leaf_size) return BVHC_OK;
  std::vector<PairNode> pairs;
  std::vector<TriRecord> tris;
  std::vector<uint32_t> roots(m->h_roots.size());
  int depth = 0;
  if (max_leaf > 0) {
    LeafSplitter sp{m->h_pairs, m->h_tris, max_leaf};
    try {
      for (size_t r = 0; r < roots.size(); ++r) roots[r] = sp.copy(m->h_roots[r], 0);
    } catch (const Status& s) {
      return s.code;
    } catch (const std::bad_alloc&) {
      return BVHC_ERR_OUT_OF_MEMORY;
    }
    pairs.swap(sp.out_pairs);
    tris.swap(sp.out_tris);
    depth = sp.max_depth;
  }
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  BVHC_CUDA_TRY(cudaDeviceSynchronize());  // no launch may still read the old records
  PairNode* nodes = nullptr;
  TriRecord* recs = nullptr;
  uint32_t* rts = nullptr;
  if (max_leaf > 0) {
    cudaError_t e = upload(&nodes, pairs);
    if (e == cudaSuccess) e = upload(&recs, tris);
    if (e == cudaSuccess) e = upload(&rts, roots);
    if (e != cudaSuccess) {
      cudaFree(nodes);
      cudaFree(recs);
      cudaFree(rts);
      return from_cuda(e);
    }
  }
  cudaFree(m->d_nodes_f);
  cudaFree(m->d_tris_f);
  cudaFree(m->d_roots_f);
  m->d_nodes_f = nodes;
  m->d_tris_f = recs;
  m->d_roots_f = rts;
  m->n_nodes_f = pairs.size();
  m->n_tris_f = tris.size();
  m->max_depth_f = depth;
  m->rec_face_f.resize(tris.size());
  for (size_t k = 0; k < tris.size(); ++k) m->rec_face_f[k] = tris[k].face;
  m->leaf_size = max_leaf;
  free_refit_plan(m->refit[1]);
  if (max_leaf > 0 && !m->h_root_bytes.empty())  // so that a refit keeps this copy in step
    BVHC_CUDA_TRY(build_refit_plan(pairs, tris, roots, serialized_root_boxes(m), m->refit[1]));
  if (max_leaf > 0) BVHC_CUDA_TRY(install_quads(m, pairs, roots));
  else BVHC_CUDA_TRY(install_quads(m, m->h_pairs, m->h_roots));
  return BVHC_OK;
}

int bvhc_mesh_get_leaf_size(const bvhc_mesh* m) { return m ? m->leaf_size : -1; }

bvhc_status bvhc_mesh_refit(bvhc_mesh* m, const float* positions, uint64_t n_verts, int stride_floats, int mem,
                            void* stream) {
  if (!m || !positions || stride_floats < 3 || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE))
    return BVHC_ERR_INVALID_ARGUMENT;
  if (n_verts < m->n_verts_geo || m->h_root_bytes.empty()) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  BVHC_CUDA_TRY(ensure_tri_vid(m));
  if (!m->refit[0].leaves)
    BVHC_CUDA_TRY(build_refit_plan(m->h_pairs, m->h_tris, m->h_roots, serialized_root_boxes(m), m->refit[0]));
  const float* pos = positions;
  if (mem == BVHC_MEM_HOST) {
    const size_t bytes = n_verts * (size_t)stride_floats * sizeof(float);
    BVHC_CUDA_TRY(ensure(&m->d_refit_pos, &m->refit_pos_cap, bytes));
    BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_refit_pos, positions, bytes, cudaMemcpyHostToDevice, s));
    pos = static_cast<const float*>(m->d_refit_pos);
  } else if (!aligned(positions, 4)) {
    return BVHC_ERR_INVALID_ARGUMENT;
  }
  BVHC_CUDA_TRY(launch_refit(m->refit[0], m->d_nodes, m->d_tris, m->d_tri_vid, pos, stride_floats, false, s));
  if (m->leaf_size > 0 && m->refit[1].leaves)  // raycastFirst's copy: every box recomputed
    BVHC_CUDA_TRY(launch_refit(m->refit[1], m->d_nodes_f, m->d_tris_f, m->d_tri_vid, pos, stride_floats, true, s));
  if (m->d_quads)  // the four-child records take their boxes from raycastFirst's child pairs
    BVHC_CUDA_TRY(launch_quad_boxes(m->d_quads, m->n_quads, m->d_quad_src, m->leaf_size > 0 ? m->d_nodes_f : m->d_nodes,
                                    s));
  if (m->d_pos && m->grad_verts <= n_verts) {  // the adjoint's vertex copy follows the geometry
    BVHC_CUDA_TRY(cudaMemcpy2DAsync(m->d_pos, 3 * sizeof(float), pos, stride_floats * sizeof(float),
                                    3 * sizeof(float), m->grad_verts, cudaMemcpyDeviceToDevice, s));
  }
  if (mem == BVHC_MEM_HOST) return read_and_clear_error(m, s);
  return BVHC_OK;
}

int bvhc_mesh_root_count(const bvhc_mesh* m) { return m ? (int)m->h_root_bytes.size() : -1; }

uint64_t bvhc_mesh_root_bytes(const bvhc_mesh* m, int root) {
  if (!m || root < 0 || root >= (int)m->h_root_bytes.size()) return 0;
  return m->h_root_bytes[root].size();
}

bvhc_status bvhc_mesh_read_root(bvhc_mesh* m, int root, void* dst, uint64_t bytes) {
  if (!m || !dst || root < 0 || root >= (int)m->h_root_bytes.size() || bytes != m->h_root_bytes[root].size())
    return BVHC_ERR_INVALID_ARGUMENT;
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  std::vector<uint8_t> buf = m->h_root_bytes[root];
  if (m->refit[0].leaves) {  // boxes as the last refit left them
    std::vector<PairNode> pairs(m->n_nodes);
    std::vector<float> root_box(6 * m->h_root_bytes.size());
    BVHC_CUDA_TRY(cudaDeviceSynchronize());
    if (!pairs.empty())
      BVHC_CUDA_TRY(cudaMemcpy(pairs.data(), m->d_nodes, pairs.size() * sizeof(PairNode), cudaMemcpyDeviceToHost));
    BVHC_CUDA_TRY(cudaMemcpy(root_box.data(), m->refit[0].root_box, root_box.size() * sizeof(float),
                             cudaMemcpyDeviceToHost));
    std::memcpy(buf.data(), &root_box[6 * root], 24);
    for (size_t k = 0; k < m->slot_nodes.size(); ++k) {
      uint64_t key = m->slot_nodes[k];
      if ((int)(key >> 40) != root) continue;
      uint64_t node = key & ((1ull << 40) - 1);
      std::memcpy(buf.data() + node * 32, pairs[k >> 1].f + 6 * (k & 1), 24);
    }
  }
  std::memcpy(dst, buf.data(), bytes);
  return BVHC_OK;
}

bvhc_status bvhc_mesh_get_traversal(const bvhc_mesh* m, bvhc_traversal_config* cfg) {
  if (!m || !cfg) return BVHC_ERR_INVALID_ARGUMENT;
  cfg->persistent = m->cfg.persistent;
  cfg->order = m->cfg.order;
  cfg->refill = m->cfg.refill;
  cfg->occupancy = m->cfg.occupancy;
  cfg->compact = m->cfg.compact;
  cfg->sort = m->cfg.sort;
  cfg->closest = m->cfg.closest;
  cfg->wide = m->cfg.wide;
  cfg->all = m->cfg.all;
  cfg->tile = m->cfg.tile;
  cfg->block = m->cfg.block;
  cfg->stack = m->cfg.stack;
  cfg->tile_rows = m->cfg.tile_rows;
  return BVHC_OK;
}

static bvhc_status raycast_first_impl(bvhc_mesh* m, const float* rays, uint64_t n, int side, const SideTable& tab,
                                      float near_d, float far_d, bvhc_hit* out, int mem, void* stream) {
  if (!m || side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE))
    return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!rays || !out) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  if (mem == BVHC_MEM_DEVICE) {
    if (!aligned(rays, 8) || !aligned(out, 16)) return BVHC_ERR_INVALID_ARGUMENT;
    return from_cuda(dispatch_first(m, rays, n, side, tab, near_d, far_d, out, m->d_work, s));
  }
  if (n <= kPipeChunk) {
    BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, n * 24));
    BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, n * sizeof(bvhc_hit)));
    BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_in, rays, n * 24, cudaMemcpyHostToDevice, s));
    BVHC_CUDA_TRY(dispatch_first(m, static_cast<const float*>(m->d_in), n, side, tab, near_d, far_d,
                                 static_cast<bvhc_hit*>(m->d_out), m->d_work, s));
    BVHC_CUDA_TRY(cudaMemcpyAsync(out, m->d_out, n * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, s));
    return read_and_clear_error(m, s);
  }
  // Large host batches: chunks rotate over three streams, each with its own staging slot and work
  // counter, so the host->device copy of one chunk, the traversal of another and the device->host
  // copy of a third overlap (copies overlap only for page-locked host memory); with a third slot a
  // chunk's upload no longer waits for the download of the chunk two before it, and the
  // device->host link, the busiest, stays fed.
  BVHC_CUDA_TRY(ensure_pipeline(m));
  cudaEvent_t ready;
  BVHC_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  cudaEventRecord(ready, s);
  for (int k = 0; k < bvhc_mesh::kPipes; ++k) cudaStreamWaitEvent(m->pipe[k], ready, 0);
  cudaEventDestroy(ready);
  const int qslots[bvhc_mesh::kPipes] = {1, 2, 5};
  for (uint64_t j = 0, off = 0; off < n; ++j, off += kPipeChunk) {
    const int k = (int)(j % bvhc_mesh::kPipes);
    uint64_t cnt = std::min<uint64_t>(kPipeChunk, n - off);
    cudaStream_t st = m->pipe[k];
    BVHC_CUDA_TRY(cudaMemcpyAsync(m->slot_in[k], rays + 6 * off, cnt * 24, cudaMemcpyHostToDevice, st));
    BVHC_CUDA_TRY(dispatch_first(m, static_cast<const float*>(m->slot_in[k]), cnt, side, tab, near_d, far_d,
                                 static_cast<bvhc_hit*>(m->slot_out[k]), m->d_work_pipe[k], st, qslots[k]));
    BVHC_CUDA_TRY(cudaMemcpyAsync(out + off, m->slot_out[k], cnt * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, st));
  }
  for (int k = 0; k < bvhc_mesh::kPipes; ++k) BVHC_CUDA_TRY(cudaStreamSynchronize(m->pipe[k]));
  return read_and_clear_error(m, s);
}

static bvhc_status raycast_all_impl(bvhc_mesh* m, const float* rays, uint64_t n, int side, const SideTable& tab,
                                    float near_d, float far_d, uint32_t cap, uint32_t* counts, bvhc_hit* hits, int mem,
                                    void* stream) {
  if (!m || side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE))
    return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!rays || !counts || (cap > 0 && !hits)) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  if (mem == BVHC_MEM_DEVICE && (!aligned(rays, 8) || !aligned(counts, 4) || (cap > 0 && !aligned(hits, 16))))
    return BVHC_ERR_INVALID_ARGUMENT;
  // the warp-cooperative variants over sorted rays (all = 2..4: key kind all - 1) use queue slot 4
  // and its sort scratch; one ray per thread over the rays that enter the tree (all = 5 in ray
  // order, 6..8 sorted by key kind all - 5) too
  const int variant = m->cfg.all >= 9 ? 9 : (m->cfg.all >= 5 ? 5 : (m->cfg.all >= 2 ? 2 : m->cfg.all));
  const int key_of_variant = m->cfg.all >= 9 ? m->cfg.all - 9 : m->cfg.all - 5;
  uint32_t* q = nullptr;
  unsigned int* qc = nullptr;
  RaySort sort{};
  const int slot = 4;
  if ((variant == 5 || variant == 9) && n < (1ull << 32)) {
    BVHC_CUDA_TRY(ensure(reinterpret_cast<void**>(&m->d_queue[slot]), &m->queue_cap[slot], n * sizeof(uint32_t)));
    if (!m->d_qcount[slot])
      BVHC_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&m->d_qcount[slot]), sizeof(unsigned int)));
    if (variant == 9 && !m->d_work_all)
      BVHC_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&m->d_work_all), sizeof(unsigned long long)));
    q = m->d_queue[slot];
    qc = m->d_qcount[slot];
    if (key_of_variant > 0) {
      BVHC_CUDA_TRY(ensure_sort_scratch(m, slot, n));
      sort.kind = key_of_variant;
      for (int a = 0; a < 3; ++a) {
        sort.lo[a] = m->scene_lo[a];
        sort.hi[a] = m->scene_hi[a];
      }
      sort.scratch = m->sort_s[slot];
    }
  }
  if (variant == 2 && n < (1ull << 32)) {
    BVHC_CUDA_TRY(ensure(reinterpret_cast<void**>(&m->d_queue[slot]), &m->queue_cap[slot], n * sizeof(uint32_t)));
    if (!m->d_qcount[slot])
      BVHC_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&m->d_qcount[slot]), sizeof(unsigned int)));
    BVHC_CUDA_TRY(ensure_sort_scratch(m, slot, n));
    q = m->d_queue[slot];
    qc = m->d_qcount[slot];
    sort.kind = m->cfg.all - 1;
    for (int a = 0; a < 3; ++a) {
      sort.lo[a] = m->scene_lo[a];
      sort.hi[a] = m->scene_hi[a];
    }
    sort.scratch = m->sort_s[slot];
  }
  if (mem == BVHC_MEM_DEVICE)
    return from_cuda(launch_raycast_all(m->view(), rays, n, side, tab, near_d, far_d, cap, counts, hits, s, variant,
                                        m->cfg.occupancy, q, qc, sort.kind ? &sort : nullptr, m->d_work_all,
                                        (uint32_t)m->cfg.tile, m->cfg.tile_rows));
  BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, n * 24));
  BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, std::max<uint64_t>(n * cap * sizeof(bvhc_hit), 16)));
  BVHC_CUDA_TRY(ensure(&m->d_out2, &m->out2_cap, n * 4));
  BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_in, rays, n * 24, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(launch_raycast_all(m->view(), static_cast<const float*>(m->d_in), n, side, tab, near_d, far_d, cap,
                                   static_cast<uint32_t*>(m->d_out2), static_cast<bvhc_hit*>(m->d_out), s, variant,
                                   m->cfg.occupancy, q, qc, sort.kind ? &sort : nullptr, m->d_work_all,
                                   (uint32_t)m->cfg.tile, m->cfg.tile_rows));
  BVHC_CUDA_TRY(cudaMemcpyAsync(counts, m->d_out2, n * 4, cudaMemcpyDeviceToHost, s));
  if (cap > 0)
    BVHC_CUDA_TRY(cudaMemcpyAsync(hits, m->d_out, n * cap * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

bvhc_status bvhc_raycast_first(bvhc_mesh* m, const float* rays, uint64_t n, int side, float near_d, float far_d,
                               bvhc_hit* out, int mem, void* stream) {
  return raycast_first_impl(m, rays, n, side, single_side(), near_d, far_d, out, mem, stream);
}

bvhc_status bvhc_raycast(bvhc_mesh* m, const float* rays, uint64_t n, int side, float near_d, float far_d,
                         uint32_t cap, uint32_t* counts, bvhc_hit* hits, int mem, void* stream) {
  return raycast_all_impl(m, rays, n, side, single_side(), near_d, far_d, cap, counts, hits, mem, stream);
}

bvhc_status bvhc_raycast_first_materials(bvhc_mesh* m, const float* rays, uint64_t n, const int8_t* material_sides,
                                         int n_materials, float near_d, float far_d, bvhc_hit* out, int mem,
                                         void* stream) {
  SideTable tab;
  if (!material_table(material_sides, n_materials, tab)) return BVHC_ERR_INVALID_ARGUMENT;
  return raycast_first_impl(m, rays, n, BVHC_FRONT_SIDE, tab, near_d, far_d, out, mem, stream);
}

bvhc_status bvhc_raycast_materials(bvhc_mesh* m, const float* rays, uint64_t n, const int8_t* material_sides,
                                   int n_materials, float near_d, float far_d, uint32_t cap, uint32_t* counts,
                                   bvhc_hit* hits, int mem, void* stream) {
  SideTable tab;
  if (!material_table(material_sides, n_materials, tab)) return BVHC_ERR_INVALID_ARGUMENT;
  return raycast_all_impl(m, rays, n, BVHC_FRONT_SIDE, tab, near_d, far_d, cap, counts, hits, mem, stream);
}

bvhc_status bvhc_mesh_set_groups(bvhc_mesh* m, const int64_t* groups, int n_groups) {
  if (!m || n_groups < 0 || (n_groups > 0 && !groups)) return BVHC_ERR_INVALID_ARGUMENT;
  // material of a triangle: the group holding its first index entry (kNoMaterial: none)
  auto material_of = [&](uint32_t face, uint32_t* out) -> bvhc_status {
    int64_t first = 3 * (int64_t)face;
    uint32_t mat = kNoMaterial;
    for (int g = 0; g < n_groups; ++g) {
      int64_t start = groups[3 * g], count = groups[3 * g + 1], mi = groups[3 * g + 2];
      if (mi < 0 || mi >= (int64_t)kNoMaterial) return BVHC_ERR_INVALID_ARGUMENT;
      if (first >= start && (count < 0 || first < start + count)) {
        if (mat != kNoMaterial) return BVHC_ERR_UNSUPPORTED;  // triangle in two groups
        mat = (uint32_t)mi;
      }
    }
    *out = mat;
    return BVHC_OK;
  };
  std::vector<uint32_t> mat(m->rec_face.size(), kNoMaterial);
  for (size_t k = 0; k < m->rec_face.size(); ++k) {
    bvhc_status st = material_of(m->rec_face[k], &mat[k]);
    if (st != BVHC_OK) return st;
  }
  for (TriRecord& t : m->h_tris) {  // the host copy, for later leaf re-layouts
    bvhc_status st = material_of(t.face, &t.material);
    if (st != BVHC_OK) return st;
  }
  if (mat.empty()) return BVHC_OK;
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  BVHC_CUDA_TRY(cudaMemcpy2D(reinterpret_cast<char*>(m->d_tris) + offsetof(TriRecord, material), sizeof(TriRecord),
                             mat.data(), sizeof(uint32_t), sizeof(uint32_t), mat.size(), cudaMemcpyHostToDevice));
  if (m->leaf_size > 0 && !m->rec_face_f.empty()) {  // raycastFirst's split-leaf copy
    std::vector<uint32_t> mat_f(m->rec_face_f.size());
    for (size_t k = 0; k < mat_f.size(); ++k) {
      bvhc_status st = material_of(m->rec_face_f[k], &mat_f[k]);
      if (st != BVHC_OK) return st;
    }
    BVHC_CUDA_TRY(cudaMemcpy2D(reinterpret_cast<char*>(m->d_tris_f) + offsetof(TriRecord, material),
                               sizeof(TriRecord), mat_f.data(), sizeof(uint32_t), sizeof(uint32_t), mat_f.size(),
                               cudaMemcpyHostToDevice));
  }
  return BVHC_OK;
}

bvhc_status bvhc_hit_interpolate(bvhc_mesh* m, const bvhc_hit* hits, uint64_t n, const float* attribute,
                                 uint64_t n_verts, int item_size, int stride_floats, const float* rays, float* out,
                                 int mem, void* stream) {
  if (!m || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE) || item_size < 1 || item_size > 4 ||
      stride_floats < item_size || n_verts < m->n_verts_geo)
    return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!hits || !attribute || !out) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  BVHC_CUDA_TRY(ensure_tri_vid(m));
  if (mem == BVHC_MEM_DEVICE) {
    if (!aligned(hits, 4) || !aligned(attribute, 4) || !aligned(out, 4) || (rays && !aligned(rays, 4)))
      return BVHC_ERR_INVALID_ARGUMENT;
    return from_cuda(launch_hit_interpolate(hits, n, m->d_tri_vid, attribute, item_size, stride_floats, rays, out, s));
  }
  // host memory: hits, rays and the attribute go through one staging buffer, the result another
  const size_t hb = n * sizeof(bvhc_hit), rb = rays ? n * 24 : 0;
  const size_t ab = n_verts * (size_t)stride_floats * sizeof(float), ob = n * item_size * sizeof(float);
  BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, hb + rb + ab));
  BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, ob));
  char* base = static_cast<char*>(m->d_in);
  BVHC_CUDA_TRY(cudaMemcpyAsync(base, hits, hb, cudaMemcpyHostToDevice, s));
  if (rays) BVHC_CUDA_TRY(cudaMemcpyAsync(base + hb, rays, rb, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(cudaMemcpyAsync(base + hb + rb, attribute, ab, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(launch_hit_interpolate(reinterpret_cast<const bvhc_hit*>(base), n, m->d_tri_vid,
                                       reinterpret_cast<const float*>(base + hb + rb), item_size, stride_floats,
                                       rays ? reinterpret_cast<const float*>(base + hb) : nullptr,
                                       static_cast<float*>(m->d_out), s));
  BVHC_CUDA_TRY(cudaMemcpyAsync(out, m->d_out, ob, cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

bvhc_status bvhc_triangle_hit_point_info(bvhc_mesh* m, const float* points, const uint32_t* faces, uint64_t n,
                                         const float* positions, int pos_stride, const float* uv, int uv_stride,
                                         uint64_t n_verts, const int64_t* groups, int n_groups,
                                         bvhc_hit_point_info* out, int mem, void* stream) {
  if (!m || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE) || pos_stride < 3 || (uv && uv_stride < 2) ||
      n_verts < m->n_verts_geo || n_groups < 0 || (n_groups > 0 && !groups))
    return BVHC_ERR_INVALID_ARGUMENT;
  if (n_groups > kMaxMaterials) return BVHC_ERR_UNSUPPORTED;
  if (n == 0) return BVHC_OK;
  if (!points || !faces || !positions || !out) return BVHC_ERR_INVALID_ARGUMENT;
  GroupTable gt{};
  gt.n = n_groups;
  for (int g = 0; g < n_groups; ++g) {
    gt.start[g] = groups[3 * g];
    gt.count[g] = groups[3 * g + 1];
    gt.material[g] = (int32_t)groups[3 * g + 2];
  }
  const uint64_t n_tri = m->h_index.empty() ? m->n_verts_geo / 3 : m->h_index.size() / 3;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  BVHC_CUDA_TRY(ensure_tri_vid(m));
  if (mem == BVHC_MEM_DEVICE) {
    if (!aligned(points, 4) || !aligned(faces, 4) || !aligned(positions, 4) || (uv && !aligned(uv, 4)) ||
        !aligned(out, 4))
      return BVHC_ERR_INVALID_ARGUMENT;
    return from_cuda(launch_triangle_hit_point_info(points, faces, n, m->d_tri_vid, n_tri, positions, pos_stride, uv,
                                                    uv_stride, gt, out, m->d_err, s));
  }
  for (uint64_t i = 0; i < n; ++i)
    if (faces[i] >= n_tri) return BVHC_ERR_INVALID_ARGUMENT;
  // host memory: points, faces, positions and uv through one staging buffer (16-byte aligned parts)
  auto up16 = [](size_t b) { return (b + 15) & ~size_t(15); };
  const size_t pb = up16(n * 12), fb = up16(n * 4), vb = up16(n_verts * (size_t)pos_stride * 4),
               ub = uv ? n_verts * (size_t)uv_stride * 4 : 0, ob = n * sizeof(bvhc_hit_point_info);
  BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, pb + fb + vb + ub));
  BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, ob));
  char* base = static_cast<char*>(m->d_in);
  BVHC_CUDA_TRY(cudaMemcpyAsync(base, points, n * 12, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(cudaMemcpyAsync(base + pb, faces, n * 4, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(cudaMemcpyAsync(base + pb + fb, positions, n_verts * (size_t)pos_stride * 4, cudaMemcpyHostToDevice, s));
  if (uv) BVHC_CUDA_TRY(cudaMemcpyAsync(base + pb + fb + vb, uv, ub, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(launch_triangle_hit_point_info(
      reinterpret_cast<const float*>(base), reinterpret_cast<const uint32_t*>(base + pb), n, m->d_tri_vid, n_tri,
      reinterpret_cast<const float*>(base + pb + fb), pos_stride,
      uv ? reinterpret_cast<const float*>(base + pb + fb + vb) : nullptr, uv_stride, gt,
      static_cast<bvhc_hit_point_info*>(m->d_out), m->d_err, s));
  BVHC_CUDA_TRY(cudaMemcpyAsync(out, m->d_out, ob, cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

// Batches of at least kShapeSortMin shapecast queries are taken in the Morton order of their
// centres (queue slot 6 and its sort scratch); smaller ones in input order.
constexpr uint64_t kShapeSortMin = 4096;
static cudaError_t shape_order(bvhc_mesh* m, uint64_t n, uint32_t** q, unsigned int** qc, RaySort* sort) {
  *q = nullptr;
  *qc = nullptr;
  if (n < kShapeSortMin || n >= (1ull << 32)) return cudaSuccess;
  const int slot = 6;
  cudaError_t e = ensure(reinterpret_cast<void**>(&m->d_queue[slot]), &m->queue_cap[slot], n * sizeof(uint32_t));
  if (e == cudaSuccess && !m->d_qcount[slot])
    e = cudaMalloc(reinterpret_cast<void**>(&m->d_qcount[slot]), sizeof(unsigned int));
  if (e == cudaSuccess) e = ensure_sort_scratch(m, slot, n);
  if (e != cudaSuccess) return e;
  *q = m->d_queue[slot];
  *qc = m->d_qcount[slot];
  sort->kind = 2;
  for (int a = 0; a < 3; ++a) {
    sort->lo[a] = m->scene_lo[a];
    sort->hi[a] = m->scene_hi[a];
  }
  sort->scratch = m->sort_s[slot];
  return cudaSuccess;
}

bvhc_status bvhc_intersects_sphere(bvhc_mesh* m, const float* spheres, uint64_t n, uint8_t* out, int mem,
                                   void* stream) {
  if (!m || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE)) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!spheres || !out) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  if (mem == BVHC_MEM_DEVICE && !aligned(spheres, 16)) return BVHC_ERR_INVALID_ARGUMENT;
  uint32_t* q;
  unsigned int* qc;
  RaySort sort{};
  BVHC_CUDA_TRY(shape_order(m, n, &q, &qc, &sort));
  if (mem == BVHC_MEM_DEVICE) return from_cuda(launch_intersects_sphere(m->view(), spheres, n, out, s, q, qc, &sort));
  BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, n * 16));
  BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, n));
  BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_in, spheres, n * 16, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(launch_intersects_sphere(m->view(), static_cast<const float*>(m->d_in), n,
                                         static_cast<uint8_t*>(m->d_out), s, q, qc, &sort));
  BVHC_CUDA_TRY(cudaMemcpyAsync(out, m->d_out, n, cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

bvhc_status bvhc_intersects_box(bvhc_mesh* m, const float* boxes, uint64_t n, uint8_t* out, int mem, void* stream) {
  if (!m || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE)) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!boxes || !out) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  if (mem == BVHC_MEM_DEVICE && !aligned(boxes, 16)) return BVHC_ERR_INVALID_ARGUMENT;
  uint32_t* q;
  unsigned int* qc;
  RaySort sort{};
  BVHC_CUDA_TRY(shape_order(m, n, &q, &qc, &sort));
  if (mem == BVHC_MEM_DEVICE) return from_cuda(launch_intersects_box(m->view(), boxes, n, out, s, q, qc, &sort));
  BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, n * 96));
  BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, n));
  BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_in, boxes, n * 96, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(launch_intersects_box(m->view(), static_cast<const float*>(m->d_in), n,
                                      static_cast<uint8_t*>(m->d_out), s, q, qc, &sort));
  BVHC_CUDA_TRY(cudaMemcpyAsync(out, m->d_out, n, cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

bvhc_status bvhc_sphere_triangles(bvhc_mesh* m, const float* spheres, uint64_t n, uint32_t cap, uint32_t* counts,
                                  uint32_t* faces, int mem, void* stream) {
  if (!m || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE)) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!spheres || !counts || (cap > 0 && !faces)) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  const uint32_t c = cap > 0 ? cap : 1;
  if (mem == BVHC_MEM_DEVICE && (!aligned(spheres, 16) || !aligned(counts, 4) || (cap > 0 && !aligned(faces, 4))))
    return BVHC_ERR_INVALID_ARGUMENT;
  uint32_t* q;
  unsigned int* qc;
  RaySort sort{};
  BVHC_CUDA_TRY(shape_order(m, n, &q, &qc, &sort));
  if (mem == BVHC_MEM_DEVICE && cap > 0)
    return from_cuda(launch_sphere_triangles(m->view(), spheres, n, cap, counts, faces, s, q, qc, &sort));
  const bool host = mem == BVHC_MEM_HOST;
  if (host) BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, n * 16));
  BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, n * c * 4));
  if (host) BVHC_CUDA_TRY(ensure(&m->d_out2, &m->out2_cap, n * 4));
  if (host) BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_in, spheres, n * 16, cudaMemcpyHostToDevice, s));
  uint32_t* d_counts = host ? static_cast<uint32_t*>(m->d_out2) : counts;
  BVHC_CUDA_TRY(launch_sphere_triangles(m->view(), host ? static_cast<const float*>(m->d_in) : spheres, n, c, d_counts,
                                        static_cast<uint32_t*>(m->d_out), s, q, qc, &sort));
  if (!host) return BVHC_OK;  // counts only, on the device
  BVHC_CUDA_TRY(cudaMemcpyAsync(counts, d_counts, n * 4, cudaMemcpyDeviceToHost, s));
  if (cap > 0) BVHC_CUDA_TRY(cudaMemcpyAsync(faces, m->d_out, n * cap * 4, cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

// The warp-cooperative closest-point variants over Morton-sorted queries (closest = 2, 4 or 6,
// minThreshold 0): queue slot `slot` with its sort scratch sized for n queries; nulls for the
// other variants.
static cudaError_t closest_sort(bvhc_mesh* m, int slot, uint64_t n, float min_threshold, uint32_t** q,
                                unsigned int** qc, RaySort* sort) {
  *q = nullptr;
  *qc = nullptr;
  if (m->cfg.closest <= 0 || m->cfg.closest % 2 != 0 || n >= (1ull << 32) || !(min_threshold <= 0.0f))
    return cudaSuccess;
  cudaError_t e = ensure(reinterpret_cast<void**>(&m->d_queue[slot]), &m->queue_cap[slot], n * sizeof(uint32_t));
  if (e == cudaSuccess && !m->d_qcount[slot])
    e = cudaMalloc(reinterpret_cast<void**>(&m->d_qcount[slot]), sizeof(unsigned int));
  if (e == cudaSuccess) e = ensure_sort_scratch(m, slot, n);
  if (e != cudaSuccess) return e;
  *q = m->d_queue[slot];
  *qc = m->d_qcount[slot];
  sort->kind = 2;
  for (int a = 0; a < 3; ++a) {
    sort->lo[a] = m->scene_lo[a];
    sort->hi[a] = m->scene_hi[a];
  }
  sort->scratch = m->sort_s[slot];
  return cudaSuccess;
}

bvhc_status bvhc_closest_point_to_point(bvhc_mesh* m, const float* points, uint64_t n, float min_threshold,
                                        float max_threshold, bvhc_closest* out, int mem, void* stream) {
  if (!m || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE)) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!points || !out) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  if (mem == BVHC_MEM_DEVICE && (!aligned(points, 4) || !aligned(out, 4))) return BVHC_ERR_INVALID_ARGUMENT;
  const int variant = m->cfg.closest;
  const MeshDev v = m->view();
  uint32_t* q;
  unsigned int* qc;
  RaySort sort{};
  if (mem == BVHC_MEM_DEVICE || n <= kPipeChunk) {
    // one launch; the sorted variant uses queue slot 3
    BVHC_CUDA_TRY(closest_sort(m, 3, n, min_threshold, &q, &qc, &sort));
    if (mem == BVHC_MEM_DEVICE)
      return from_cuda(launch_closest_point(v, points, n, min_threshold, max_threshold, out, s, variant,
                                            m->cfg.occupancy, q, qc, q ? &sort : nullptr, (uint32_t)m->cfg.tile,
                                            m->cfg.tile_rows));
    BVHC_CUDA_TRY(ensure(&m->d_in, &m->in_cap, n * 12));
    BVHC_CUDA_TRY(ensure(&m->d_out, &m->out_cap, n * sizeof(bvhc_closest)));
    BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_in, points, n * 12, cudaMemcpyHostToDevice, s));
    BVHC_CUDA_TRY(launch_closest_point(v, static_cast<const float*>(m->d_in), n, min_threshold,
                                       max_threshold, static_cast<bvhc_closest*>(m->d_out), s, variant,
                                       m->cfg.occupancy, q, qc, q ? &sort : nullptr, (uint32_t)m->cfg.tile,
                                       m->cfg.tile_rows));
    BVHC_CUDA_TRY(cudaMemcpyAsync(out, m->d_out, n * sizeof(bvhc_closest), cudaMemcpyDeviceToHost, s));
    return read_and_clear_error(m, s);
  }
  // Large host batches: chunks of kPipeChunk points rotate over the raycastFirst pipeline's three
  // streams and staging slots (12 B in and 20 B out per point fit its 24 B / 32 B per ray), so the
  // copies of some chunks overlap the traversal of others; each stream sorts its own chunk in its
  // own queue slot.
  BVHC_CUDA_TRY(ensure_pipeline(m));
  const int qslots[bvhc_mesh::kPipes] = {1, 2, 5};
  uint32_t* qs[bvhc_mesh::kPipes];
  unsigned int* qcs[bvhc_mesh::kPipes];
  RaySort sorts[bvhc_mesh::kPipes] = {};
  for (int k = 0; k < bvhc_mesh::kPipes; ++k)
    BVHC_CUDA_TRY(closest_sort(m, qslots[k], kPipeChunk, min_threshold, &qs[k], &qcs[k], &sorts[k]));
  cudaEvent_t ready;
  BVHC_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  cudaEventRecord(ready, s);
  for (int k = 0; k < bvhc_mesh::kPipes; ++k) cudaStreamWaitEvent(m->pipe[k], ready, 0);
  cudaEventDestroy(ready);
  for (uint64_t j = 0, off = 0; off < n; ++j, off += kPipeChunk) {
    const int k = (int)(j % bvhc_mesh::kPipes);
    const uint64_t cnt = std::min<uint64_t>(kPipeChunk, n - off);
    cudaStream_t st = m->pipe[k];
    BVHC_CUDA_TRY(cudaMemcpyAsync(m->slot_in[k], points + 3 * off, cnt * 12, cudaMemcpyHostToDevice, st));
    BVHC_CUDA_TRY(launch_closest_point(v, static_cast<const float*>(m->slot_in[k]), cnt, min_threshold,
                                       max_threshold, static_cast<bvhc_closest*>(m->slot_out[k]), st, variant,
                                       m->cfg.occupancy, qs[k], qcs[k], qs[k] ? &sorts[k] : nullptr,
                                       (uint32_t)m->cfg.tile, m->cfg.tile_rows));
    BVHC_CUDA_TRY(
        cudaMemcpyAsync(out + off, m->slot_out[k], cnt * sizeof(bvhc_closest), cudaMemcpyDeviceToHost, st));
  }
  for (int k = 0; k < bvhc_mesh::kPipes; ++k) BVHC_CUDA_TRY(cudaStreamSynchronize(m->pipe[k]));
  return read_and_clear_error(m, s);
}

// ---------------------------------------------------------------------------------------------
// Batched meshes
// ---------------------------------------------------------------------------------------------
static bool valid_offsets(const bvhc_mesh* m, const uint64_t* ray_offsets) {
  if (!ray_offsets || ray_offsets[0] != 0) return false;
  for (int k = 0; k < m->n_meshes; ++k)
    if (ray_offsets[k + 1] < ray_offsets[k]) return false;
  return true;
}

bvhc_status bvhc_batch_raycast_first(bvhc_mesh* m, const float* rays, const uint64_t* ray_offsets, int side,
                                     float near_d, float far_d, bvhc_hit* out, void* stream) {
  if (!m || m->n_meshes <= 0 || side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE || !valid_offsets(m, ray_offsets))
    return BVHC_ERR_INVALID_ARGUMENT;
  uint64_t n = ray_offsets[m->n_meshes];
  if (n == 0) return BVHC_OK;
  if (!rays || !out || !aligned(rays, 8) || !aligned(out, 16)) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  BVHC_CUDA_TRY(cudaMemcpyAsync(m->d_ray_off, ray_offsets, (m->n_meshes + 1) * 8, cudaMemcpyHostToDevice, s));
  BatchDev bd{m->d_ray_off, m->d_mesh_root_off, m->n_meshes};
  uint32_t* q;
  unsigned int* qc;
  BVHC_CUDA_TRY(queue_for(m, 0, n, &q, &qc));
  return from_cuda(launch_raycast_first_persistent(m->view_first(), &bd, rays, n, side, single_side(), near_d, far_d,
                                                   out, m->d_work, m->cfg, s, q, qc));
}

bvhc_status bvhc_batch_raycast_first_per_mesh(bvhc_mesh* m, const float* rays, const uint64_t* ray_offsets, int side,
                                              float near_d, float far_d, bvhc_hit* out, void* stream) {
  if (!m || m->n_meshes <= 0 || side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE || !valid_offsets(m, ray_offsets))
    return BVHC_ERR_INVALID_ARGUMENT;
  if (ray_offsets[m->n_meshes] == 0) return BVHC_OK;
  if (!rays || !out || !aligned(rays, 8) || !aligned(out, 16)) return BVHC_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  for (int k = 0; k < m->n_meshes; ++k) {
    uint64_t off = ray_offsets[k], cnt = ray_offsets[k + 1] - off;
    if (cnt == 0) continue;
    MeshDev v = m->view_first();
    v.roots += m->mesh_root_off[k];  // this geometry's roots, in whichever layout the view uses
    if (v.quad_roots) v.quad_roots += m->mesh_root_off[k];
    v.n_roots = (int)(m->mesh_root_off[k + 1] - m->mesh_root_off[k]);
    BVHC_CUDA_TRY(dispatch_view(m, v, rays + 6 * off, cnt, side, near_d, far_d, out + off, s));
  }
  return BVHC_OK;
}

struct bvhc_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
};

bvhc_status bvhc_batch_graph_create(bvhc_mesh* m, const float* rays, const uint64_t* ray_offsets, int side,
                                    float near_d, float far_d, bvhc_hit* out, bvhc_graph** graph) {
  if (!m || !graph || m->n_meshes <= 0 || side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE ||
      !valid_offsets(m, ray_offsets))
    return BVHC_ERR_INVALID_ARGUMENT;
  uint64_t n = ray_offsets[m->n_meshes];
  if (n == 0 || !rays || !out || !aligned(rays, 8) || !aligned(out, 16)) return BVHC_ERR_INVALID_ARGUMENT;
  *graph = nullptr;
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  // the offsets are part of the captured work: copy them once, before capture
  BVHC_CUDA_TRY(cudaMemcpy(m->d_ray_off, ray_offsets, (m->n_meshes + 1) * 8, cudaMemcpyHostToDevice));
  cudaStream_t cs;
  BVHC_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  auto* g = new bvhc_graph();
  g->device = m->device;
  BatchDev bd{m->d_ray_off, m->d_mesh_root_off, m->n_meshes};
  uint32_t* q = nullptr;
  unsigned int* qc = nullptr;
  cudaError_t e = queue_for(m, 0, n, &q, &qc);  // allocated before capture: captured work cannot allocate
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t le = launch_raycast_first_persistent(m->view_first(), &bd, rays, n, side, single_side(), near_d, far_d,
                                                     out, m->d_work, m->cfg, cs, q, qc);
    e = cudaStreamEndCapture(cs, &g->graph);
    if (le != cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) {
    bvhc_graph_destroy(g);
    return from_cuda(e);
  }
  *graph = g;
  return BVHC_OK;
}

bvhc_status bvhc_graph_launch(bvhc_graph* g, void* stream) {
  if (!g || !g->exec) return BVHC_ERR_INVALID_ARGUMENT;
  BVHC_CUDA_TRY(cudaSetDevice(g->device));
  return from_cuda(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
}

void bvhc_graph_destroy(bvhc_graph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

int bvhc_batch_mesh_count(const bvhc_mesh* m) { return m ? m->n_meshes : 0; }

// ---------------------------------------------------------------------------------------------
// Instances (acceleratedBatchedMeshRaycast, ExtensionUtilities.js:87-161): world matrices of a
// batch's geometries and a tree over their world boxes.
// ---------------------------------------------------------------------------------------------
struct bvhc_scene {
  bvhc_mesh* batch = nullptr;
  int n_instances = 0;
  InstanceDev* d_inst = nullptr;
  size_t inst_cap = 0;
  PairNode* d_tlas = nullptr;
  size_t tlas_cap = 0;
  uint32_t root = kEmptyLeaf;
  void* d_in = nullptr;
  size_t in_cap = 0;
  void* d_out = nullptr;
  size_t out_cap = 0;
  void* d_ids = nullptr;
  size_t ids_cap = 0;
  // ray ordering (bvhc_scene_set_order): key kind, the instances' world box, sort scratch, queue
  int order = 0;
  int variant = 0;  // instanced raycastFirst kernel variant (bvhc_scene_set_variant)
  float box_lo[3] = {0, 0, 0}, box_hi[3] = {0, 0, 0};
  RaySortScratch sort_s = {};
  uint64_t sort_cap = 0;
  uint32_t* d_queue = nullptr;
  size_t queue_cap = 0;
  unsigned int* d_qcount = nullptr;
  void* d_cnt = nullptr;  // host-memory bvhc_scene_raycast: per-ray counts
  size_t cnt_cap = 0;
  void* inst_slot[bvhc_mesh::kPipes] = {};  // pipelined host-memory raycastFirst: instance ids per stream
};

namespace {

struct InstBox {
  float lo[3], hi[3];
  uint32_t id;
};

// Median split on the longest centroid extent down to one instance per leaf; the root record is
// written first.  Returns the link of the subtree over boxes [a, b).
uint32_t build_tlas(std::vector<InstBox>& boxes, size_t a, size_t b, std::vector<PairNode>& out) {
  if (b - a == 1) return kLeafBit | boxes[a].id;
  float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = a; i < b; ++i)
    for (int d = 0; d < 3; ++d) {
      const float c = 0.5f * boxes[i].lo[d] + 0.5f * boxes[i].hi[d];
      clo[d] = std::min(clo[d], c);
      chi[d] = std::max(chi[d], c);
    }
  int axis = 0;
  for (int d = 1; d < 3; ++d)
    if (chi[d] - clo[d] > chi[axis] - clo[axis]) axis = d;
  const size_t mid = a + (b - a) / 2;
  std::nth_element(boxes.begin() + a, boxes.begin() + mid, boxes.begin() + b, [axis](const InstBox& x, const InstBox& y) {
    return x.lo[axis] + x.hi[axis] < y.lo[axis] + y.hi[axis];
  });
  const size_t me = out.size();
  out.emplace_back();
  const uint32_t l = build_tlas(boxes, a, mid, out), r = build_tlas(boxes, mid, b, out);
  PairNode& n = out[me];
  for (int side = 0; side < 2; ++side) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = side ? mid : a; i < (side ? b : mid); ++i)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], boxes[i].lo[d]);
        hi[d] = std::max(hi[d], boxes[i].hi[d]);
      }
    for (int d = 0; d < 3; ++d) {
      n.f[6 * side + d] = lo[d];
      n.f[6 * side + 3 + d] = hi[d];
    }
  }
  n.link[0] = l;
  n.link[1] = r;
  n.axis = (uint32_t)axis;
  n.flags = 0;
  return (uint32_t)me;
}

void split_ff(double x, float& hi, float& lo) {
  hi = (float)x;
  lo = (float)(x - (double)hi);
}

float round_down(double x) {
  float f = (float)x;
  return (double)f > x ? std::nextafter(f, -INFINITY) : f;
}
float round_up(double x) {
  float f = (float)x;
  return (double)f < x ? std::nextafter(f, INFINITY) : f;
}

bvhc_status set_instances(bvhc_scene* sc, int n, const uint32_t* geometry, const double* matrices,
                          const uint8_t* visible) {
  bvhc_mesh* m = sc->batch;
  if (n < 0 || (n > 0 && (!geometry || !matrices))) return BVHC_ERR_INVALID_ARGUMENT;
  // each geometry's local box: the union of its roots' boxes
  const std::vector<float> root_boxes = serialized_root_boxes(m);
  std::vector<double> gbox((size_t)m->n_meshes * 6);
  for (int g = 0; g < m->n_meshes; ++g) {
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t r = m->mesh_root_off[g]; r < m->mesh_root_off[g + 1]; ++r)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], (double)root_boxes[6 * r + d]);
        hi[d] = std::max(hi[d], (double)root_boxes[6 * r + 3 + d]);
      }
    for (int d = 0; d < 3; ++d) {
      gbox[6 * g + d] = lo[d];
      gbox[6 * g + 3 + d] = hi[d];
    }
  }
  std::vector<InstanceDev> inst((size_t)n);
  std::vector<InstBox> boxes;
  for (int j = 0; j < n; ++j) {
    if (geometry[j] >= (uint32_t)m->n_meshes) return BVHC_ERR_INVALID_ARGUMENT;
    const double* e = matrices + 16 * (size_t)j;  // column-major: e[col * 4 + row]
    for (int k = 0; k < 16; ++k)
      if (!std::isfinite(e[k])) return BVHC_ERR_INVALID_ARGUMENT;
    if (e[3] != 0 || e[7] != 0 || e[11] != 0 || e[15] != 1) return BVHC_ERR_UNSUPPORTED;  // affine only
    InstanceDev& I = inst[j];
    I.geometry = geometry[j];
    // inverse of the affine matrix: inverse 3x3 (adjugate / determinant), translation -inv * t
    const double a00 = e[0], a01 = e[4], a02 = e[8], a10 = e[1], a11 = e[5], a12 = e[9], a20 = e[2], a21 = e[6],
                 a22 = e[10];
    const double c00 = a11 * a22 - a12 * a21, c01 = a02 * a21 - a01 * a22, c02 = a01 * a12 - a02 * a11;
    const double c10 = a12 * a20 - a10 * a22, c11 = a00 * a22 - a02 * a20, c12 = a02 * a10 - a00 * a12;
    const double c20 = a10 * a21 - a11 * a20, c21 = a01 * a20 - a00 * a21, c22 = a00 * a11 - a01 * a10;
    const double det = a00 * c00 + a01 * c10 + a02 * c20;
    const double rows[3][4] = {{a00, a01, a02, e[12]}, {a10, a11, a12, e[13]}, {a20, a21, a22, e[14]}};
    double inv[3][4] = {{c00, c01, c02, 0}, {c10, c11, c12, 0}, {c20, c21, c22, 0}};
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) inv[r][c] = det != 0 ? inv[r][c] / det : 0;
      inv[r][3] = -(inv[r][0] * e[12] + inv[r][1] * e[13] + inv[r][2] * e[14]);
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 4; ++c) {
        split_ff(rows[r][c], I.m_hi[4 * r + c], I.m_lo[4 * r + c]);
        split_ff(inv[r][c], I.inv_hi[4 * r + c], I.inv_lo[4 * r + c]);
      }
    for (int c = 0; c < 3; ++c)
      I.scale[c] = (float)std::sqrt(e[4 * c] * e[4 * c] + e[4 * c + 1] * e[4 * c + 1] + e[4 * c + 2] * e[4 * c + 2]);
    // a singular matrix maps every ray to a zero direction: the instance is never hit
    if ((visible && !visible[j]) || det == 0) continue;
    const double* gb = &gbox[6 * (size_t)geometry[j]];
    if (!(gb[0] <= gb[3])) continue;
    InstBox b;
    b.id = (uint32_t)j;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 8; ++k) {
      const double x = gb[(k & 1) ? 3 : 0], y = gb[(k & 2) ? 4 : 1], z = gb[(k & 4) ? 5 : 2];
      for (int r = 0; r < 3; ++r) {
        const double v = rows[r][0] * x + rows[r][1] * y + rows[r][2] * z + rows[r][3];
        lo[r] = std::min(lo[r], v);
        hi[r] = std::max(hi[r], v);
      }
    }
    for (int d = 0; d < 3; ++d) {  // widened so that rounding of the corners cannot cut a hit
      const double pad = 1e-6 * (hi[d] - lo[d]) + 1e-6 * std::max(std::fabs(lo[d]), std::fabs(hi[d]));
      b.lo[d] = round_down(lo[d] - pad);
      b.hi[d] = round_up(hi[d] + pad);
    }
    boxes.push_back(b);
  }
  for (int d = 0; d < 3; ++d) {
    sc->box_lo[d] = INFINITY;
    sc->box_hi[d] = -INFINITY;
    for (const InstBox& b : boxes) {
      sc->box_lo[d] = std::min(sc->box_lo[d], b.lo[d]);
      sc->box_hi[d] = std::max(sc->box_hi[d], b.hi[d]);
    }
  }
  std::vector<PairNode> nodes;
  uint32_t root = kEmptyLeaf;
  if (!boxes.empty()) root = build_tlas(boxes, 0, boxes.size(), nodes);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  if (n > 0) {
    BVHC_CUDA_TRY(ensure(reinterpret_cast<void**>(&sc->d_inst), &sc->inst_cap, inst.size() * sizeof(InstanceDev)));
    BVHC_CUDA_TRY(cudaMemcpy(sc->d_inst, inst.data(), inst.size() * sizeof(InstanceDev), cudaMemcpyHostToDevice));
  }
  if (!nodes.empty()) {
    BVHC_CUDA_TRY(ensure(reinterpret_cast<void**>(&sc->d_tlas), &sc->tlas_cap, nodes.size() * sizeof(PairNode)));
    BVHC_CUDA_TRY(cudaMemcpy(sc->d_tlas, nodes.data(), nodes.size() * sizeof(PairNode), cudaMemcpyHostToDevice));
  }
  sc->root = root;
  sc->n_instances = n;
  return BVHC_OK;
}

}  // namespace

bvhc_status bvhc_scene_create(bvhc_mesh* batch, int n_instances, const uint32_t* geometry, const double* matrices,
                              const uint8_t* visible, bvhc_scene** out) {
  if (!batch || !out || batch->n_meshes <= 0 || batch->h_root_bytes.empty()) return BVHC_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  auto* sc = new (std::nothrow) bvhc_scene();
  if (!sc) return BVHC_ERR_OUT_OF_MEMORY;
  sc->batch = batch;
  bvhc_status st = set_instances(sc, n_instances, geometry, matrices, visible);
  if (st != BVHC_OK) {
    bvhc_scene_destroy(sc);
    return st;
  }
  *out = sc;
  return BVHC_OK;
}

bvhc_status bvhc_scene_set_instances(bvhc_scene* scene, int n_instances, const uint32_t* geometry,
                                     const double* matrices, const uint8_t* visible) {
  if (!scene) return BVHC_ERR_INVALID_ARGUMENT;
  BVHC_CUDA_TRY(cudaSetDevice(scene->batch->device));
  BVHC_CUDA_TRY(cudaDeviceSynchronize());  // earlier queries may still read the instance arrays
  return set_instances(scene, n_instances, geometry, matrices, visible);
}

bvhc_status bvhc_scene_raycast_first(bvhc_scene* sc, const float* rays, uint64_t n, int side, float near_dist,
                                     float far_dist, bvhc_hit* hits, uint32_t* instance, int mem, void* stream) {
  if (!sc || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE)) return BVHC_ERR_INVALID_ARGUMENT;
  if (side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!rays || !hits || !instance) return BVHC_ERR_INVALID_ARGUMENT;
  bvhc_mesh* m = sc->batch;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  SceneDev sd{sc->d_tlas, sc->root, sc->d_inst, m->d_mesh_root_off};
  sd.n_instances = sc->n_instances;
  sd.occupancy = sc->variant;
  if (mem == BVHC_MEM_HOST && n > kPipeChunk) {
    // Large host batches: chunks of kPipeChunk rays rotate over the batch mesh's three pipeline
    // streams and staging slots (instance ids in a slot of the scene's own), so the copies of some
    // chunks overlap the traversal of others.  Each chunk keeps its input order (the ray sort of
    // bvhc_scene_set_order changes the traversal time by a few percent at most).
    BVHC_CUDA_TRY(ensure_pipeline(m));
    for (int k = 0; k < bvhc_mesh::kPipes; ++k)
      if (!sc->inst_slot[k]) BVHC_CUDA_TRY(cudaMalloc(&sc->inst_slot[k], kPipeChunk * 4));
    cudaEvent_t ready;
    BVHC_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    cudaEventRecord(ready, s);
    for (int k = 0; k < bvhc_mesh::kPipes; ++k) cudaStreamWaitEvent(m->pipe[k], ready, 0);
    cudaEventDestroy(ready);
    for (uint64_t j = 0, off = 0; off < n; ++j, off += kPipeChunk) {
      const int k = (int)(j % bvhc_mesh::kPipes);
      const uint64_t cnt = std::min<uint64_t>(kPipeChunk, n - off);
      cudaStream_t st = m->pipe[k];
      BVHC_CUDA_TRY(cudaMemcpyAsync(m->slot_in[k], rays + 6 * off, cnt * 24, cudaMemcpyHostToDevice, st));
      BVHC_CUDA_TRY(launch_scene_raycast_first(m->view_first(), sd, static_cast<const float*>(m->slot_in[k]), cnt, side,
                                               near_dist, far_dist, static_cast<bvhc_hit*>(m->slot_out[k]),
                                               static_cast<uint32_t*>(sc->inst_slot[k]), st));
      BVHC_CUDA_TRY(cudaMemcpyAsync(hits + off, m->slot_out[k], cnt * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, st));
      BVHC_CUDA_TRY(cudaMemcpyAsync(instance + off, sc->inst_slot[k], cnt * 4, cudaMemcpyDeviceToHost, st));
    }
    for (int k = 0; k < bvhc_mesh::kPipes; ++k) BVHC_CUDA_TRY(cudaStreamSynchronize(m->pipe[k]));
    return read_and_clear_error(m, s);
  }
  RaySort sort{};
  if (sc->order > 0 && n < (1ull << 32) && sc->root != kEmptyLeaf) {
    if (sc->sort_cap < n) {
      free_sort_scratch(sc->sort_s);
      sc->sort_cap = 0;
      RaySortScratch& t = sc->sort_s;
      cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&t.keys[0]), n * 4);
      if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&t.keys[1]), n * 4);
      if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&t.vals), n * 4);
      if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&t.hist), 256 * ray_sort_tiles(n) * 4);
      if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void**>(&t.totals), 4 * 256 * 4);
      if (e != cudaSuccess) {
        free_sort_scratch(t);
        return from_cuda(e);
      }
      sc->sort_cap = n;
    }
    BVHC_CUDA_TRY(ensure(reinterpret_cast<void**>(&sc->d_queue), &sc->queue_cap, n * 4));
    if (!sc->d_qcount) BVHC_CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(&sc->d_qcount), sizeof(unsigned int)));
    sort.kind = sc->order;
    for (int a = 0; a < 3; ++a) {
      sort.lo[a] = sc->box_lo[a];
      sort.hi[a] = sc->box_hi[a];
    }
    sort.scratch = sc->sort_s;
  }
  const RaySort* sp = sort.kind ? &sort : nullptr;
  if (mem == BVHC_MEM_DEVICE) {
    if (!aligned(rays, 8) || !aligned(hits, 16) || !aligned(instance, 4)) return BVHC_ERR_INVALID_ARGUMENT;
    return from_cuda(launch_scene_raycast_first(m->view_first(), sd, rays, n, side, near_dist, far_dist, hits, instance, s,
                                                sp, sc->d_queue, sc->d_qcount));
  }
  BVHC_CUDA_TRY(ensure(&sc->d_in, &sc->in_cap, n * 24));
  BVHC_CUDA_TRY(ensure(&sc->d_out, &sc->out_cap, n * sizeof(bvhc_hit)));
  BVHC_CUDA_TRY(ensure(&sc->d_ids, &sc->ids_cap, n * 4));
  BVHC_CUDA_TRY(cudaMemcpyAsync(sc->d_in, rays, n * 24, cudaMemcpyHostToDevice, s));
  BVHC_CUDA_TRY(launch_scene_raycast_first(m->view_first(), sd, static_cast<const float*>(sc->d_in), n, side, near_dist,
                                           far_dist, static_cast<bvhc_hit*>(sc->d_out),
                                           static_cast<uint32_t*>(sc->d_ids), s, sp, sc->d_queue, sc->d_qcount));
  BVHC_CUDA_TRY(cudaMemcpyAsync(hits, sc->d_out, n * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, s));
  BVHC_CUDA_TRY(cudaMemcpyAsync(instance, sc->d_ids, n * 4, cudaMemcpyDeviceToHost, s));
  return read_and_clear_error(m, s);
}

bvhc_status bvhc_scene_raycast(bvhc_scene* sc, const float* rays, uint64_t n, int side, float near_dist,
                               float far_dist, uint32_t cap, uint32_t* counts, bvhc_hit* hits, uint32_t* instance,
                               int mem, void* stream) {
  if (!sc || (mem != BVHC_MEM_HOST && mem != BVHC_MEM_DEVICE)) return BVHC_ERR_INVALID_ARGUMENT;
  if (side < BVHC_FRONT_SIDE || side > BVHC_DOUBLE_SIDE) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!rays || !counts || (cap > 0 && (!hits || !instance))) return BVHC_ERR_INVALID_ARGUMENT;
  bvhc_mesh* m = sc->batch;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  SceneDev sd{sc->d_tlas, sc->root, sc->d_inst, m->d_mesh_root_off};
  sd.n_instances = sc->n_instances;
  sd.occupancy = sc->variant;
  const uint32_t c = cap > 0 ? cap : 1;  // cap 0: counts only (one scratch slot per ray)
  if (mem == BVHC_MEM_DEVICE) {
    if (!aligned(rays, 8) || !aligned(counts, 4) || (cap > 0 && (!aligned(hits, 16) || !aligned(instance, 4))))
      return BVHC_ERR_INVALID_ARGUMENT;
    if (cap > 0)
      return from_cuda(launch_scene_raycast_all(m->view(), sd, rays, n, side, near_dist, far_dist, cap, counts, hits,
                                                instance, s));
  }
  const bool host = mem == BVHC_MEM_HOST;
  if (host) BVHC_CUDA_TRY(ensure(&sc->d_in, &sc->in_cap, n * 24));
  BVHC_CUDA_TRY(ensure(&sc->d_out, &sc->out_cap, n * c * sizeof(bvhc_hit)));
  BVHC_CUDA_TRY(ensure(&sc->d_ids, &sc->ids_cap, n * c * 4));
  if (host) BVHC_CUDA_TRY(ensure(&sc->d_cnt, &sc->cnt_cap, n * 4));
  if (host) BVHC_CUDA_TRY(cudaMemcpyAsync(sc->d_in, rays, n * 24, cudaMemcpyHostToDevice, s));
  const float* d_rays = host ? static_cast<const float*>(sc->d_in) : rays;
  uint32_t* d_counts = host ? static_cast<uint32_t*>(sc->d_cnt) : counts;
  BVHC_CUDA_TRY(launch_scene_raycast_all(m->view(), sd, d_rays, n, side, near_dist, far_dist, c, d_counts,
                                         static_cast<bvhc_hit*>(sc->d_out), static_cast<uint32_t*>(sc->d_ids), s));
  if (!host) return BVHC_OK;  // counts only, on the device
  BVHC_CUDA_TRY(cudaMemcpyAsync(counts, d_counts, n * 4, cudaMemcpyDeviceToHost, s));
  if (cap > 0) {
    BVHC_CUDA_TRY(cudaMemcpyAsync(hits, sc->d_out, n * cap * sizeof(bvhc_hit), cudaMemcpyDeviceToHost, s));
    BVHC_CUDA_TRY(cudaMemcpyAsync(instance, sc->d_ids, n * cap * 4, cudaMemcpyDeviceToHost, s));
  }
  return read_and_clear_error(m, s);
}

void bvhc_scene_destroy(bvhc_scene* sc) {
  if (!sc) return;
  if (sc->batch) cudaSetDevice(sc->batch->device);
  cudaFree(sc->d_inst);
  cudaFree(sc->d_tlas);
  cudaFree(sc->d_in);
  cudaFree(sc->d_out);
  cudaFree(sc->d_ids);
  cudaFree(sc->d_queue);
  cudaFree(sc->d_qcount);
  cudaFree(sc->d_cnt);
  for (void* p : sc->inst_slot) cudaFree(p);
  free_sort_scratch(sc->sort_s);
  delete sc;
}

bvhc_status bvhc_scene_set_variant(bvhc_scene* sc, int variant) {
  if (!sc || variant < 0 || variant > 2) return BVHC_ERR_INVALID_ARGUMENT;
  sc->variant = variant;
  return BVHC_OK;
}

bvhc_status bvhc_scene_set_order(bvhc_scene* scene, int kind) {
  if (!scene || kind < 0 || kind > 4) return BVHC_ERR_INVALID_ARGUMENT;
  scene->order = kind;
  return BVHC_OK;
}

// ---------------------------------------------------------------------------------------------
// Gradients
// ---------------------------------------------------------------------------------------------
bvhc_status bvhc_mesh_enable_gradients(bvhc_mesh* m, const void* index, int index_elem_bytes, uint64_t index_count,
                                       const float* positions, uint64_t n_verts, int stride_floats) {
  if (!m || !positions || n_verts == 0 || stride_floats < 3) return BVHC_ERR_INVALID_ARGUMENT;
  if (index && index_elem_bytes != 2 && index_elem_bytes != 4) return BVHC_ERR_INVALID_ARGUMENT;
  uint64_t n_tris = index ? index_count / 3 : n_verts / 3;
  std::vector<uint32_t> idx(n_tris * 3);
  for (uint64_t i = 0; i < n_tris * 3; ++i) {
    idx[i] = index ? read_index(index, index_elem_bytes, i) : (uint32_t)i;
    if (idx[i] >= n_verts) return BVHC_ERR_INVALID_ARGUMENT;
  }
  std::vector<float> pos(n_verts * 3);
  for (uint64_t v = 0; v < n_verts; ++v)
    for (int k = 0; k < 3; ++k) pos[3 * v + k] = positions[v * (uint64_t)stride_floats + k];
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  cudaFree(m->d_index32);
  cudaFree(m->d_pos);
  m->d_index32 = nullptr;
  m->d_pos = nullptr;
  BVHC_CUDA_TRY(upload(&m->d_index32, idx));
  BVHC_CUDA_TRY(upload(&m->d_pos, pos));
  m->grad_tris = n_tris;
  m->grad_verts = n_verts;
  return BVHC_OK;
}

bvhc_status bvhc_raycast_first_backward(bvhc_mesh* m, const float* rays, const bvhc_hit* hits, uint64_t n,
                                        const float* grad_distance, const float* grad_barycoord, float* grad_vertices,
                                        float* grad_origins, float* grad_directions, void* stream) {
  if (!m || !m->d_index32) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!rays || !hits || (!grad_distance && !grad_barycoord)) return BVHC_ERR_INVALID_ARGUMENT;
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  return from_cuda(launch_raycast_first_backward(m->d_index32, m->d_pos, rays, hits, n, grad_distance, grad_barycoord,
                                                 grad_vertices, grad_origins, grad_directions,
                                                 static_cast<cudaStream_t>(stream)));
}

bvhc_status bvhc_closest_point_backward(bvhc_mesh* m, const float* points, const bvhc_closest* results, uint64_t n,
                                        const float* grad_distance, float* grad_vertices, float* grad_points,
                                        void* stream) {
  if (!m || !m->d_index32) return BVHC_ERR_INVALID_ARGUMENT;
  if (n == 0) return BVHC_OK;
  if (!points || !results || !grad_distance) return BVHC_ERR_INVALID_ARGUMENT;
  BVHC_CUDA_TRY(cudaSetDevice(m->device));
  return from_cuda(launch_closest_point_backward(m->d_index32, m->d_pos, points, results, n, grad_distance,
                                                 grad_vertices, grad_points, static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
