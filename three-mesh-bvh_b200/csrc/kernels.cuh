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
  kErrBadFace = 2u,        // a faceIndex argument past the geometry's triangles
};

struct MeshDev {
  const PairNode* nodes;
  const TriRecord* tris;
  const uint32_t* roots;  // one link per root
  int n_roots;
  unsigned int* err;
  const QuadNode* quads = nullptr;     // four-child copy of `nodes` (same triangle records), if any
  const uint32_t* quad_roots = nullptr;
  int depth = kMaxStack - 2;           // deepest node level of these records (bounds the stack use)
};

cudaError_t launch_raycast_first(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                                 float near_d, float far_d, bvhc_hit* out, int order, cudaStream_t stream);
// Traversal variant chosen per call (autotuned): persistent vs one-ray-per-thread grid, child
// order, and the number of idle lanes that triggers a warp refill.
// log2 of a tiled order's rows per tile (tile_rows 2, 4 or 8; 0 means 4).
inline int tile_rows_log2(int rows) { return rows == 2 ? 1 : rows == 8 ? 3 : 2; }

struct TraversalConfig {
  int persistent;  // 1: persistent warps with lane refill; 0: one ray per thread; 2: warp-cooperative
  int order;       // 0: split-axis direction sign (reference order); 1: nearest entry first
  int refill;      // idle lanes (1..32) that trigger a refill in the persistent form
  int occupancy;   // persistent form register budget: 0 compiler's choice, 1 six blocks/SM, 2 eight
  int compact;     // 1 runs the root-box pre-pass and traverses only queued rays (persistent and
                   // warp-cooperative forms)
  int sort;        // 0: queue in ray order; 1..3: queue sorted by a Morton key (raysort.cu), implies
                   // the pre-pass
  int closest;     // closestPointToPoint: 0 one query per thread, 1 warp-cooperative, 2 warp-cooperative
                   // over Morton-sorted queries (1 and 2 only with minThreshold 0)
  int wide;        // warp-cooperative raycastFirst: 1 walks the four-child records
  int all;         // raycast (all hits): 0 one ray per thread, 1 warp-cooperative, 2..4 warp-cooperative
                   // over the rays that enter the tree, sorted by key kind all - 1, 5..8 one ray per
                   // thread over the rays that enter the tree (6..8 sorted by key kind all - 5), 9..12
                   // the same with persistent warps and lane refill (10..12 sorted by key all - 9)
  int tile;        // warp-cooperative raycastFirst without a queue: 0 consecutive rays per warp; a
                   // multiple of 8 takes R x 32/R tiles of the rays read as rows of `tile` rays
  int block;       // warp-cooperative raycastFirst threads per block: 64, 256, else 128
  int stack;       // raycastFirst traversal stack entries (warp-cooperative and persistent forms): 32
                   // when the tree allows it, else 64
  int tile_rows;   // R of the tiled order: 2, 4 or 8 (0: 4)
};

// Scratch of the ray-ordering sort for up to n queued rays (raysort.cu).
struct RaySortScratch {
  uint32_t* keys[2];  // n entries each
  uint32_t* vals;     // n entries: the queue's ping-pong partner
  uint32_t* hist;     // 256 * ray_sort_tiles(n) entries
  uint32_t* totals;   // 4 * 256 entries (one row per pass; the closest-point sort, three passes,
                      // keeps its query box in the last row)
};

// A sort request: key kind (1..3, raykey.cuh) and the scene box used by the entry-point keys.
struct RaySort {
  int kind;
  float lo[3], hi[3];
  RaySortScratch scratch;
};

uint64_t ray_sort_tiles(uint64_t n);
// Where the pre-pass writes the (key, id) pairs for a sort of key `kind`, so that the sort's last
// pass ends in `queue`.
void ray_sort_input(int kind, const RaySortScratch& s, uint32_t* queue, uint32_t** ids, uint32_t** keys);
// Sorts the *qcount (key, id) pairs at ray_sort_input's buffers by key, stably, into `queue` (ids);
// n bounds *qcount.
cudaError_t launch_ray_sort(int kind, uint64_t n, const unsigned int* qcount, const RaySortScratch& s,
                            uint32_t* queue, cudaStream_t stream);

// Many meshes in one node/triangle pool: rays [ray_off[k], ray_off[k+1]) belong to mesh k, whose
// roots are MeshDev::roots[mesh_root_off[k] .. mesh_root_off[k+1]).
struct BatchDev {
  const uint64_t* ray_off;        // n_meshes + 1 entries
  const uint32_t* mesh_root_off;  // n_meshes + 1 entries
  int n_meshes;
};

// `batch` null: one mesh (all of m.roots).  The work counter `work` is reset on `stream` first.
// With `queue` (n entries) and `qcount` given, a pre-pass finishes the rays that miss every root's
// child boxes and queues the others for the traversal (n must be below 2^32; otherwise no pre-pass).
cudaError_t launch_raycast_first_persistent(const MeshDev& m, const BatchDev* batch, const float* rays, uint64_t n,
                                            int side, const SideTable& sides, float near_d, float far_d,
                                            bvhc_hit* out, unsigned long long* work, const TraversalConfig& cfg,
                                            cudaStream_t stream, uint32_t* queue = nullptr,
                                            unsigned int* qcount = nullptr, const RaySort* sort = nullptr);
// Completes the pending records a traversal left in `out` (record index in face_index), for the
// queued rays (queue / qcount) or all n.
cudaError_t launch_finalize_first(const MeshDev& m, const float* rays, uint64_t n, bvhc_hit* out,
                                  const uint32_t* queue, const unsigned int* qcount, cudaStream_t stream);
// Warp-cooperative raycastFirst: the 32 rays of a warp share one traversal (coherent rays).  With a
// queue, the same pre-pass (and sort) as the persistent form runs first.
// wide = 1 with m.quads set runs over the four-child records.
cudaError_t launch_raycast_first_packet(const MeshDev& m, const float* rays, uint64_t n, int side,
                                        const SideTable& sides, float near_d, float far_d, bvhc_hit* out,
                                        const TraversalConfig& cfg, cudaStream_t stream, uint32_t* queue = nullptr,
                                        unsigned int* qcount = nullptr, const RaySort* sort = nullptr);
// closestPointToPoint.  variant 0: one query per thread; 1: warp-cooperative in input order; 2:
// warp-cooperative over the queries sorted by a Morton key of the point (queue, qcount and sort
// scratch for n queries required).  Variants 1 and 2 apply only with min_t <= 0 (else variant 0).
// Variant 1 reads the queries in tiled order when `tile` is a row length (see tiled_index).
cudaError_t launch_closest_point(const MeshDev& m, const float* pts, uint64_t n, float min_t, float max_t,
                                 bvhc_closest* out, cudaStream_t stream, int variant = 0, int occupancy = 0,
                                 uint32_t* queue = nullptr, unsigned int* qcount = nullptr,
                                 const RaySort* sort = nullptr, uint32_t tile = 0, int tile_rows = 0);

// raycast (all hits).  variant 0: one ray per thread; 1: warp-cooperative in input order; 2:
// warp-cooperative over the rays sorted by the key sort->kind (queue, qcount and sort scratch for
// n rays required, else variant 0 runs); 5: one ray per thread over the rays the root-box pre-pass
// queues (queue and qcount for n rays required; sorted by sort->kind when given); 9: the same
// queue walked by persistent warps with lane refill (also a zeroed-per-call work counter).  `tile`
// (variant 1): the warp-cooperative walk takes tile_rows x 32/tile_rows tiles of rays read as rows
// of `tile` rays.
cudaError_t launch_raycast_all(const MeshDev& m, const float* rays, uint64_t n, int side, const SideTable& sides,
                               float near_d, float far_d, uint32_t cap, uint32_t* counts, bvhc_hit* hits,
                               cudaStream_t stream, int variant = 0, int occupancy = 0, uint32_t* queue = nullptr,
                               unsigned int* qcount = nullptr, const RaySort* sort = nullptr,
                               unsigned long long* work = nullptr, uint32_t tile = 0, int tile_rows = 0);

// intersectsSphere: spheres n x 4 (centre, radius), 16-byte aligned; out[i] = 1 if the mesh meets
// sphere i.
// Shapecasts (intersectsSphere, triangles within spheres, intersectsBox): with queue, qcount and
// sort scratch for n queries, the queries are first sorted by the Morton key of their centres over
// sort->lo..hi and taken in that order (results stay in input order); otherwise in input order.
cudaError_t launch_intersects_sphere(const MeshDev& m, const float* spheres, uint64_t n, uint8_t* out,
                                     cudaStream_t stream, uint32_t* queue = nullptr, unsigned int* qcount = nullptr,
                                     const RaySort* sort = nullptr);

// Instances of a batch's geometries (bvhc_scene_*).  Matrices are the affine rows 0..2 of the
// instance's world matrix, row-major 3 x 4 (x' = r0 x + r1 y + r2 z + r3), as float-float pairs
// of the binary64 values, and the same for its inverse.
struct InstanceDev {
  float m_hi[12], m_lo[12];
  float inv_hi[12], inv_lo[12];
  float scale[3];     // column lengths of the world matrix (Vector3.setFromMatrixScale)
  uint32_t geometry;  // batch geometry: roots [mesh_root_off[g], mesh_root_off[g + 1])
};
// The instance tree (TLAS): child-pair records over instance world boxes; a leaf link is
// kLeafBit | instance.  root == kEmptyLeaf: no visible instance.
struct SceneDev {
  const PairNode* nodes;
  uint32_t root;
  const InstanceDev* inst;
  const uint32_t* mesh_root_off;
  int n_instances = 1 << 30;   // bounds the instance tree's depth (a median split)
  int occupancy = 0;           // raycastFirst kernel variant (bvhc_scene_set_variant)
};
// World-space raycastFirst over the instances: hits[i] in world space (distance, point; local
// barycoord and faceIndex), instance[i] the hit instance (0xFFFFFFFF: none).  With `sort` (kind
// 1..3, its box the instances' world box, scratch and a queue / qcount for n rays) the rays are
// traversed in the order of their Morton keys; kind 4 orders them by the first instance reached.
cudaError_t launch_scene_raycast_first(const MeshDev& blas, const SceneDev& scene, const float* rays, uint64_t n,
                                       int side, float near_d, float far_d, bvhc_hit* hits, uint32_t* instance,
                                       cudaStream_t stream, const RaySort* sort = nullptr, uint32_t* queue = nullptr,
                                       unsigned int* qcount = nullptr);

// Instanced raycast (all hits): per ray the total count and the first `cap` world-space hits by
// (distance, instance); instance n x cap (0xFFFFFFFF past the count).
cudaError_t launch_scene_raycast_all(const MeshDev& blas, const SceneDev& scene, const float* rays, uint64_t n,
                                     int side, float near_d, float far_d, uint32_t cap, uint32_t* counts,
                                     bvhc_hit* hits, uint32_t* instance, cudaStream_t stream);

// Triangles within each sphere (n x 4, 16-byte aligned) through shapecast's CONTAINED path:
// counts[i] the total, faces[i * cap ..] the first cap faceIndex values in traversal order.
cudaError_t launch_sphere_triangles(const MeshDev& m, const float* spheres, uint64_t n, uint32_t cap, uint32_t* counts,
                                    uint32_t* faces, cudaStream_t stream, uint32_t* queue = nullptr,
                                    unsigned int* qcount = nullptr, const RaySort* sort = nullptr);

// getTriangleHitPointInfo's material lookup: the first of n groups whose [start, start + count)
// (index units, count < 0 = Infinity) holds the triangle's first index gives its materialIndex.
struct GroupTable {
  int64_t start[kMaxMaterials], count[kMaxMaterials];
  int32_t material[kMaxMaterials];
  int32_t n;
};
// getTriangleHitPointInfo for n (point, faceIndex) pairs over the geometry index tri_vid (n_tri
// triangles), positions and optional uv (stride in floats); out-of-range faces set kErrBadFace.
cudaError_t launch_triangle_hit_point_info(const float* points, const uint32_t* faces, uint64_t n,
                                           const uint32_t* tri_vid, uint64_t n_tri, const float* pos, int pos_stride,
                                           const float* uv, int uv_stride, const GroupTable& groups,
                                           bvhc_hit_point_info* out, unsigned int* err, cudaStream_t stream);

// intersectsBox: boxes n x 24 (min xyz, pad, max xyz, pad, column-major box-to-mesh matrix),
// 16-byte aligned; out[i] = 1 if the oriented box meets the mesh.
cudaError_t launch_intersects_box(const MeshDev& m, const float* boxes, uint64_t n, uint8_t* out,
                                  cudaStream_t stream, uint32_t* queue = nullptr, unsigned int* qcount = nullptr,
                                  const RaySort* sort = nullptr);

// Vertex attribute at each hit (barycentric interpolation over the hit triangle's vertices, via
// tri_vid: 3 vertex ids per triangle); rays (nullable, item_size 3) flip results that point along
// the ray.  out: n x item_size.
cudaError_t launch_hit_interpolate(const bvhc_hit* hits, uint64_t n, const uint32_t* tri_vid, const float* attr,
                                   int item_size, int stride, const float* rays, float* out, cudaStream_t stream);

// Refit (refit.cu).  A box "slot" is where a node's box lives on the device: 2 * pair + side for a
// child box in a child-pair record, or kRootSlot | root for a root's own box (kept in root_box).
constexpr uint32_t kRootSlot = 0x80000000u;

struct RefitLeaf {
  uint32_t first, count, slot;  // triangle records [first, first + count); count 0 for an empty leaf
};

struct RefitPlan {
  RefitLeaf* leaves = nullptr;  // one per leaf, including empty leaves and root leaves
  uint32_t n_leaves = 0;
  uint32_t* parent = nullptr;   // per pair record: the slot holding the pair's own box
  uint32_t* arrive = nullptr;   // per pair record: children finished (zeroed before each refit)
  uint32_t* flags = nullptr;    // per pair record: bit s = child s's box changed
  uint32_t n_pairs = 0;
  float* root_box = nullptr;    // 6 floats per root
};

// New vertex positions into the triangle records, leaf boxes from them, and pair boxes bottom-up
// (one thread per leaf; the second child to finish a pair carries on upward).  force = false
// follows the reference's rule (MeshBVH#refit, refit.template.js:4-196): a leaf box is rewritten
// and reported changed only when it differs, a parent's box is recomputed only when a child
// changed; force = true recomputes every box.  tri_vid: 3 vertex ids per triangle (faceIndex).
cudaError_t launch_refit(const RefitPlan& plan, PairNode* pairs, TriRecord* tris, const uint32_t* tri_vid,
                         const float* pos, int stride, bool force, cudaStream_t stream);
// Copies every four-child record's child boxes from the child-pair slots they were collapsed from
// (src: 4 per record, kEmptyLeaf for an unused child).
cudaError_t launch_quad_boxes(QuadNode* quads, uint64_t n_quads, const uint32_t* src, const PairNode* pairs,
                              cudaStream_t stream);

// What another translation unit needs to launch on a mesh: its device view, traversal variant and
// device ordinal (defined in api.cu).  Returns false for a null mesh.
bool mesh_launch_info(const bvhc_mesh* mesh, MeshDev* view, TraversalConfig* cfg, int* device);

// Adjoint kernels (adjoint.cu).  index: 3 uint32 per triangle; pos: 3 float per vertex.
cudaError_t launch_raycast_first_backward(const uint32_t* index, const float* pos, const float* rays,
                                          const bvhc_hit* hits, uint64_t n, const float* g_dist, const float* g_bary,
                                          float* g_vert, float* g_orig, float* g_dir, cudaStream_t stream);
cudaError_t launch_closest_point_backward(const uint32_t* index, const float* pos, const float* pts,
                                          const bvhc_closest* res, uint64_t n, const float* g_dist, float* g_vert,
                                          float* g_pts, cudaStream_t stream);

}  // namespace bvhc
