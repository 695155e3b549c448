/*
 * libbvhcuda — a B200 (sm_100a) query engine for three-mesh-bvh's data-parallel hot path.
 *
 * The engine consumes the packed node buffers that `MeshBVH.serialize()` emits (32-byte nodes,
 * version 1) together with the geometry's position attribute and index, and answers batches of
 * `raycastFirst`, `raycast` (all hits) and `closestPointToPoint` queries on the GPU.  Results are
 * in the BVH's local frame, as with the reference's `MeshBVH` methods.
 *
 * Reference interfaces (three-mesh-bvh 0.9.14, paths relative to the project root):
 *   src/core/MeshBVH.js, src/core/BVH.js, src/core/cast/*.js, src/index.d.ts,
 *   src/utils/ExtensionUtilities.js.
 *
 * Conventions
 *   - Every entry point returns a bvhc_status; BVHC_OK is 0.  Nothing traps or aborts.
 *   - Buffers are caller-owned.  `mem` says whether the query buffers are host memory
 *     (BVHC_MEM_HOST: the call copies in, runs and copies out before returning) or device memory
 *     on the mesh's device (BVHC_MEM_DEVICE: the call only enqueues work on `stream`; call
 *     bvhc_mesh_synchronize to wait and collect device-side errors).
 *   - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 *   - One bvhc_mesh may be queried from one host thread at a time.
 *   - All GPU arithmetic is float32 (no FP64 instruction on the device); decisions whose float32
 *     error bound does not settle them are re-evaluated in double-float (float-float) arithmetic,
 *     and where the reference's exact binary64 rounding decides (the device build's splits, close
 *     calls of the oriented-box tests) in binary64 emulated with integer operations.
 */
#ifndef BVHCUDA_H
#define BVHCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bvhc_status {
  BVHC_OK = 0,
  BVHC_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad size, bad enum */
  BVHC_ERR_INVALID_BVH = 2,      /* node buffer fails validation (offsets, counts, depth) */
  BVHC_ERR_CUDA = 3,             /* a CUDA runtime call failed */
  BVHC_ERR_OUT_OF_MEMORY = 4,
  BVHC_ERR_DEVICE = 5,           /* a kernel set the device error word (e.g. stack overflow) */
  BVHC_ERR_UNSUPPORTED = 6,      /* valid input outside what this build supports */
  BVHC_ERR_BUILD = 7,            /* the CPU builder rejected the input */
  BVHC_ERR_SCRATCH_LIMIT = 8     /* request larger than bvhc_raycast_first_noalloc's fixed scratch */
} bvhc_status;

/* three.js side constants (FrontSide, BackSide, DoubleSide). */
enum { BVHC_FRONT_SIDE = 0, BVHC_BACK_SIDE = 1, BVHC_DOUBLE_SIDE = 2 };
/* Split strategies (src/core/Constants.js:9,18,28). */
enum { BVHC_CENTER = 0, BVHC_AVERAGE = 1, BVHC_SAH = 2 };
/* Memory kind of query buffers. */
enum { BVHC_MEM_HOST = 0, BVHC_MEM_DEVICE = 1 };

#define BVHC_NO_HIT 0xFFFFFFFFu

/* One ray/triangle intersection in the BVH's local frame (32 bytes).  face_index is the
 * reference's `faceIndex` (the triangle index after the build's in-place index reorder, or the
 * indirect-buffer entry); BVHC_NO_HIT when there is no hit.  barycoord is (wA, wB, wC) as
 * three.js `Triangle.getBarycoord` returns it.  Replaces the `Intersection` objects built by
 * src/utils/ThreeRayIntersectUtilities.js:49-145 (face/normal/uv are derived on the host from
 * face_index). */
typedef struct bvhc_hit {
  uint32_t face_index;
  float distance;
  float point[3];
  float barycoord[3];
} bvhc_hit;

/* closestPointToPoint result (20 bytes); face_index == BVHC_NO_HIT for the reference's `null`.
 * Replaces the HitPointInfo of src/core/cast/closestPointToPoint.js:67-76. */
typedef struct bvhc_closest {
  uint32_t face_index;
  float distance;
  float point[3];
} bvhc_closest;

/* getTriangleHitPointInfo's result (src/utils/TriangleUtilities.js:65-147): face.a / b / c,
 * face.materialIndex, face.normal, barycoord, uv ((0, 0) without a uv attribute). */
typedef struct bvhc_hit_point_info {
  uint32_t a, b, c;
  uint32_t material_index;
  float normal[3];
  float barycoord[3];
  float uv[2];
} bvhc_hit_point_info;

typedef struct bvhc_mesh_info {
  uint64_t node_records;     /* 64-byte child-pair records on the device */
  uint64_t triangle_records; /* 48-byte leaf-ordered triangle records on the device */
  uint64_t device_bytes;     /* device memory held by the mesh */
  int32_t max_depth;         /* deepest leaf over all roots */
  int32_t root_count;
} bvhc_mesh_info;

typedef struct bvhc_serialized bvhc_serialized; /* a MeshBVH.serialize() result owned by the library */
typedef struct bvhc_mesh bvhc_mesh;             /* a device-resident BVH + triangle set */

/* Human-readable text for a status code. */
const char* bvhc_status_string(bvhc_status status);

/* ---------------------------------------------------------------------------------------------
 * Build: `new MeshBVH(geometry, options)` followed by `MeshBVH.serialize(bvh)`
 * (src/core/GeometryBVH.js:93-163, src/core/build/buildTree.js:123-152,
 * src/core/MeshBVH.js:112-145).  bvhc_build runs on the CPU, bvhc_build_device on a GPU; run once
 * per mesh (or after the geometry changes); not part of the query path.
 *   positions        n_verts vertices, `stride_floats` floats apart (xyz first)
 *   index            optional geometry index (elem 2 or 4 bytes); NULL for non-indexed geometry,
 *                    in which case a non-indirect build creates one (geometryUtils.js:15-47)
 *   groups           n_groups (start, count) pairs in index units; count < 0 means Infinity
 *   range_start/count  draw range in index units; count < 0 means Infinity
 *   strategy         BVHC_CENTER / BVHC_AVERAGE / BVHC_SAH
 * The serialized index is the geometry index reordered in place by the build, exactly as the
 * reference reorders `geometry.index`. */
bvhc_status bvhc_build(const float* positions, uint64_t n_verts, int stride_floats, const void* index,
                       int index_elem_bytes, uint64_t index_count, const int64_t* groups, int n_groups,
                       int64_t range_start, int64_t range_count, int strategy, int max_depth,
                       int target_leaf_size, int indirect, bvhc_serialized** out);
/* The same build on GPU `device`, enqueued on `stream` (a cudaStream_t; NULL = the default stream)
 * and waited for before returning.  Same arguments and the same serialized bytes (roots and the
 * reordered index / indirect buffer) as bvhc_build, for BVHC_SAH and BVHC_CENTER; BVHC_AVERAGE
 * (a sequential double sum per node) returns BVHC_ERR_UNSUPPORTED.  Split decisions are made
 * with the reference's binary64 rounding, computed in integer arithmetic on the device. */
bvhc_status bvhc_build_device(const float* positions, uint64_t n_verts, int stride_floats, const void* index,
                              int index_elem_bytes, uint64_t index_count, const int64_t* groups, int n_groups,
                              int64_t range_start, int64_t range_count, int strategy, int max_depth,
                              int target_leaf_size, int indirect, int device, void* stream, bvhc_serialized** out);
int bvhc_serialized_root_count(const bvhc_serialized* s);
bvhc_status bvhc_serialized_root(const bvhc_serialized* s, int i, const void** data, uint64_t* bytes);
/* elem_bytes is 0 when there is no index / no indirect buffer. */
bvhc_status bvhc_serialized_index(const bvhc_serialized* s, const void** data, int* elem_bytes, uint64_t* count);
bvhc_status bvhc_serialized_indirect(const bvhc_serialized* s, const void** data, int* elem_bytes,
                                     uint64_t* count);
void bvhc_serialized_free(bvhc_serialized* s);

/* ---------------------------------------------------------------------------------------------
 * Upload: `MeshBVH.deserialize(data, geometry)` (src/core/MeshBVH.js:160-232) onto `device`.
 * Validates every root buffer (node alignment, child links, leaf ranges, depth) and re-lays the
 * tree as 64-byte child-pair records and the leaf triangles as 48-byte records in leaf order.
 * `version` 0 buffers (absolute right-child offsets) are converted as the reference does
 * (MeshBVH.js:206-230). */
bvhc_status bvhc_mesh_create(int device, int version, const void* const* roots, const uint64_t* root_bytes,
                             int n_roots, const void* index, int index_elem_bytes, uint64_t index_count,
                             const void* indirect, int indirect_elem_bytes, uint64_t indirect_count,
                             const float* positions, uint64_t n_verts, int stride_floats, bvhc_mesh** out);
void bvhc_mesh_destroy(bvhc_mesh* mesh);
bvhc_status bvhc_mesh_get_info(const bvhc_mesh* mesh, bvhc_mesh_info* info);
/* Traversal variant used by this mesh's raycastFirst calls (no reference counterpart: the
 * reference has one recursive traversal).  persistent = 1 runs a grid of resident warps that
 * refill idle lanes from a work counter once `refill` (1..32) lanes are idle; 0 runs one ray per
 * thread; 2 runs the 32 rays of a warp through one shared traversal (for coherent rays such as a
 * camera's).  Batched launches always use the persistent form.  order = 0 visits the near child
 * by the sign of the ray direction on the split axis (the reference's order), 1 by the smaller
 * entry distance.  occupancy selects the register budget of the persistent and warp-cooperative
 * kernels: 0 the compiler's choice, 1 at least six and 2 at least eight resident 128-thread
 * blocks per SM.  compact = 1
 * (persistent = 1 or 2) first finishes, in one coalesced pass, the rays that miss every root's
 * child boxes and traverses only the others.  sort (persistent = 1 or 2, single meshes; implies
 * the compaction pass) orders the remaining rays by a Morton key before the traversal: 1 the ray
 * direction (cube-map coordinates), 2 the point where the ray enters the mesh's bounding box, 3
 * that point (coarser) followed by the direction; 0 keeps the input order.  wide = 1 makes the
 * warp-cooperative and persistent forms (and batched launches) walk four-child records (collapsed
 * from raycastFirst's child pairs, same leaves; children taken nearest first, 64-entry stack).
 * closest selects closestPointToPoint's kernel: 0 one query per thread, 1 the 32 queries of a warp
 * through one shared traversal (for spatially coherent queries such as grids), 2 the same over the
 * queries sorted by a Morton key of the point, 3 and 4 as 1 and 2 with groups of 16 consecutive
 * queries (two shared traversals per warp), 5 and 6 with groups of 8; 1 to 6 apply with
 * minThreshold 0 (otherwise 0 runs), and use the occupancy setting too; 1, 3 and 5 also read the
 * queries in tiled order when `tile` is set (rows of `tile` points, e.g. a grid's row).
 * All forms return the same bytes.  all selects raycast's
 * (all hits) kernel: 0 one ray per thread, 1 the rays of a warp through one shared left-first
 * traversal (each ray's hits stay in the reference's DFS order), 2, 3 and 4 the same over the rays
 * that enter the tree (the others get a zero count), sorted by the key sort = all - 1 names above
 * (the direction, the entry point, the entry point and the direction), 5 one ray per thread over
 * the rays that enter the tree (the others get a zero count), 6, 7 and 8 the same sorted by key
 * sort = all - 5, 9 to 12 the same walked by persistent warps that refill idle lanes (10 to 12
 * sorted by key all - 9).  tile (warp-cooperative raycastFirst without compaction or ordering):
 * 0 gives each warp 32 consecutive rays; a multiple of 8 (at most 2^24) reads the rays as rows of
 * `tile` rays and gives each warp a tile of 4 rows x 8 rays, for rays generated per pixel of a
 * row-major image of that width (the ray-sort granularity without a sort); it applies to raycast's
 * warp-cooperative kernel (all = 1) too.  tile_rows (2, 4 or 8; 0 = 4) is the tile's height R, its
 * width 32 / R (tile must then be a multiple of 32 / R).  block: threads per
 * block of the warp-cooperative raycastFirst (64, 128 or 256; 0 = 128).  stack: traversal stack
 * entries of the warp-cooperative and persistent raycastFirst (32 or 64; 0 = 64); 32 applies to
 * trees of depth 30 or less and 64 runs otherwise.  Results are the same for every variant (up to
 * exact ties); the autotuner picks the fastest per mesh and workload. */
typedef struct bvhc_traversal_config {
  int32_t persistent;
  int32_t order;
  int32_t refill;
  int32_t occupancy;
  int32_t compact;
  int32_t sort;
  int32_t closest;
  int32_t wide;
  int32_t all;
  int32_t tile;
  int32_t block;
  int32_t stack;
  int32_t tile_rows;
} bvhc_traversal_config;
bvhc_status bvhc_mesh_set_traversal(bvhc_mesh* mesh, const bvhc_traversal_config* cfg);
bvhc_status bvhc_mesh_get_traversal(const bvhc_mesh* mesh, bvhc_traversal_config* cfg);

/* raycastFirst autotuner (no reference counterpart: the reference has one recursive traversal;
 * its only traversal knobs are the build's maxDepth / maxLeafSize, src/core/Constants.js:74-85,
 * and the shader stack depth, src/webgl/glsl/bvh_ray_functions.glsl.js:14-16).  Times the
 * traversal variants with CUDA events on `stream` over the caller's ray sets (device memory,
 * n_sets sets of counts[k] rays) and installs the fastest.  Stage 1: every candidate (one ray per
 * thread; warp-cooperative over child pairs or four-child records; persistent warps over either; with and
 * without the root-box compaction and each ordering key; register budgets; the tiled ray order for
 * each row pitch in tile_pitches, e.g. an image width) for every device leaf layout in leaf_sizes
 * (NULL / 0: the current one); the layout with the smallest sum of the sets' best times wins.
 * Stage 2: threads per block, the tiled order's tile height, the persistent form's refill
 * threshold and the 32-entry stack around each set's best.  Each variant is run
 * once untimed, then `reps` times.  Outputs: best[k] and best_ms[k] per set (best_ms nullable),
 * the chosen layout (nullable) and each layout's total (leaf_total_ms[n_leaf_sizes], nullable).
 * The mesh is left with the chosen layout and set 0's variant; callers switch variants per set
 * with bvhc_mesh_set_traversal.  Waits for the device; allocates a hit buffer for the largest set. */
bvhc_status bvhc_mesh_autotune(bvhc_mesh* mesh, int n_sets, const float* const* rays, const uint64_t* counts, int side,
                               float near_dist, float far_dist, const int32_t* leaf_sizes, int n_leaf_sizes,
                               const int32_t* tile_pitches, int n_tile_pitches, int reps, void* stream,
                               bvhc_traversal_config* best, float* best_ms, int32_t* leaf_size_out,
                               float* leaf_total_ms);
/* bvhc_mesh_autotune's stage-1 candidates for these row pitches, in the order it times them: the
 * first min(count, cap) are written to out; returns the count (-1 for invalid arguments). */
int bvhc_autotune_candidates(const int32_t* tile_pitches, int n_tile_pitches, bvhc_traversal_config* out, int cap);

/* Device leaf layout of raycastFirst (no reference counterpart; the reference's own leaves are
 * maxLeafSize-bounded, buildTree.js:64-89): max_leaf > 0 gives raycastFirst (single, material,
 * batched and no-alloc forms) its own copy of the tree in which every leaf of more than max_leaf
 * triangles is a subtree of exact-bounds child pairs (median split of the centroids along their
 * longest axis); 0 drops the copy.  The nearest hit does not depend on how triangles are grouped
 * into leaves, so results are the same up to exact ties.  raycast and closestPointToPoint keep the
 * reference's leaves (their hit order and maxThreshold / minThreshold rules follow them).  Waits for
 * the device; graphs captured before must be captured again.  bvhc_mesh_get_leaf_size returns the
 * current setting (-1 for a null mesh); bvhc_mesh_get_info describes raycastFirst's records. */
bvhc_status bvhc_mesh_set_leaf_size(bvhc_mesh* mesh, int max_leaf);
int bvhc_mesh_get_leaf_size(const bvhc_mesh* mesh);

/* MeshBVH#refit() (src/core/MeshBVH.js:504-508, src/core/cast/refit.template.js:4-196) on the
 * device, after the geometry's vertices moved: `positions` (n_verts >= the mesh's vertex count,
 * `stride_floats` apart; host or device memory per `mem`) replace the vertices of every triangle
 * record, and the boxes are rebuilt bottom-up with the reference's rule (a leaf box is rewritten
 * only when it differs from the stored one, a parent's only when a child changed), so the boxes
 * are bit-identical to the reference's refit of the same buffers.  raycastFirst's split-leaf copy,
 * if any, is refit too, and the gradient vertex copy (bvhc_mesh_enable_gradients) follows.  The
 * topology (index, triangle count) must not change.  Device-memory calls only enqueue on `stream`.
 * bvhc_mesh_read_root copies root `root`'s serialized buffer (version 1 layout) with the boxes as
 * the last refit left them (MeshBVH.serialize after refit); it waits for the device. */
bvhc_status bvhc_mesh_refit(bvhc_mesh* mesh, const float* positions, uint64_t n_verts, int stride_floats, int mem,
                            void* stream);
int bvhc_mesh_root_count(const bvhc_mesh* mesh);
uint64_t bvhc_mesh_root_bytes(const bvhc_mesh* mesh, int root);
bvhc_status bvhc_mesh_read_root(bvhc_mesh* mesh, int root, void* dst, uint64_t bytes);

/* Waits for the mesh's work on `stream` and reports (and clears) the device error word. */
bvhc_status bvhc_mesh_synchronize(bvhc_mesh* mesh, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Queries.  rays: n x 6 float32 (origin xyz, direction xyz); points: n x 3 float32.
 */

/* MeshBVH#raycastFirst(ray, side, near, far) for every ray (src/core/MeshBVH.js:558-577,
 * src/core/cast/raycastFirst.template.js:9-103).  out: n bvhc_hit. */
bvhc_status bvhc_raycast_first(bvhc_mesh* mesh, const float* rays, uint64_t n, int side, float near_dist,
                               float far_dist, bvhc_hit* out, int mem, void* stream);

/* MeshBVH#raycast(ray, side, near, far) for every ray (src/core/MeshBVH.js:532-545,
 * src/core/cast/raycast.template.js:7-53).  Stores at most `cap` hits per ray, in the
 * reference's DFS order, at hits[i * cap ..]; counts[i] receives the uncapped hit count. */
bvhc_status bvhc_raycast(bvhc_mesh* mesh, const float* rays, uint64_t n, int side, float near_dist, float far_dist,
                         uint32_t cap, uint32_t* counts, bvhc_hit* hits, int mem, void* stream);

/* Labels every triangle with the materialIndex of the geometry group that holds it, for the
 * material-array raycasts below.  groups: n_groups (start, count, materialIndex) triplets in index
 * units, count < 0 meaning Infinity (BufferGeometry.groups).  A triangle in no group is never hit
 * by a material-array raycast (the reference tests it against no material); a triangle in two or
 * more groups is rejected with BVHC_ERR_UNSUPPORTED. */
bvhc_status bvhc_mesh_set_groups(bvhc_mesh* mesh, const int64_t* groups, int n_groups);

/* raycastFirst / raycast with an array of materials as `materialOrSide`
 * (src/utils/ThreeRayIntersectUtilities.js:170-205): material_sides[m] (host memory, at most 64
 * entries) is the side of material m; each triangle is tested with its group material's side, and
 * with FrontSide when its material index is past the array. */
bvhc_status bvhc_raycast_first_materials(bvhc_mesh* mesh, const float* rays, uint64_t n, const int8_t* material_sides,
                                         int n_materials, float near_dist, float far_dist, bvhc_hit* out, int mem,
                                         void* stream);
bvhc_status bvhc_raycast_materials(bvhc_mesh* mesh, const float* rays, uint64_t n, const int8_t* material_sides,
                                   int n_materials, float near_dist, float far_dist, uint32_t cap, uint32_t* counts,
                                   bvhc_hit* hits, int mem, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Batched meshes: the bounds trees of a BatchedMesh (computeBatchedBoundsTree,
 * src/utils/ExtensionUtilities.js:216-268): one MeshBVH per geometry, all over one shared index
 * and position buffer (each built with `range` = its draw range, so leaf offsets are absolute
 * triangle indices).  bvhc_batch_create packs them into one device pool; the result is a
 * bvhc_mesh whose roots are grouped per geometry (roots_per_mesh[k] roots of geometry k, taken in
 * order from roots / root_bytes).  Replaces the per-instance serial raycast loop of
 * acceleratedBatchedMeshRaycast (ExtensionUtilities.js:87-161) for rays already in each
 * geometry's local frame.
 */
bvhc_status bvhc_batch_create(int device, int n_meshes, const int32_t* roots_per_mesh, const void* const* roots,
                              const uint64_t* root_bytes, const void* index, int index_elem_bytes,
                              uint64_t index_count, const float* positions, uint64_t n_verts, int stride_floats,
                              bvhc_mesh** out);
int bvhc_batch_mesh_count(const bvhc_mesh* batch);
/* raycastFirst for every geometry's rays in ONE persistent launch: rays (device memory) of
 * geometry k are rows [ray_offsets[k], ray_offsets[k+1]) (host array of n_meshes + 1 entries,
 * ray_offsets[0] = 0); results land in the same rows of out (device memory). */
bvhc_status bvhc_batch_raycast_first(bvhc_mesh* batch, const float* rays, const uint64_t* ray_offsets, int side,
                                     float near_dist, float far_dist, bvhc_hit* out, void* stream);
/* The same work as one launch per geometry, back to back on `stream` (the comparison baseline). */
bvhc_status bvhc_batch_raycast_first_per_mesh(bvhc_mesh* batch, const float* rays, const uint64_t* ray_offsets,
                                              int side, float near_dist, float far_dist, bvhc_hit* out,
                                              void* stream);
/* Captures bvhc_batch_raycast_first on fixed device buffers into a CUDA graph (work-counter reset,
 * persistent traversal, finalize); bvhc_graph_launch replays it on `stream`. */
typedef struct bvhc_graph bvhc_graph;
bvhc_status bvhc_batch_graph_create(bvhc_mesh* batch, const float* rays, const uint64_t* ray_offsets, int side,
                                    float near_dist, float far_dist, bvhc_hit* out, bvhc_graph** graph);
bvhc_status bvhc_graph_launch(bvhc_graph* graph, void* stream);
void bvhc_graph_destroy(bvhc_graph* graph);

/* Instances of a batch's geometries: the BatchedMesh raycast (acceleratedBatchedMeshRaycast,
 * src/utils/ExtensionUtilities.js:87-161) with Raycaster.firstHitOnly, on world-space rays.
 * Instance j shows geometry geometry[j] under the world matrix matrices[16 j .. 16 j + 15]
 * (float64, column-major as three.js Matrix4.elements: the BatchedMesh's matrixWorld times the
 * instance matrix; affine, else BVHC_ERR_UNSUPPORTED); visible (n bytes, NULL = all) is
 * getVisibleAt.  The scene keeps a pointer to `batch`, which must outlive it; a tree over the
 * instances' world boxes is built on the host.  bvhc_scene_set_instances replaces the instances
 * (after the queries already enqueued have finished). */
typedef struct bvhc_scene bvhc_scene;
bvhc_status bvhc_scene_create(bvhc_mesh* batch, int n_instances, const uint32_t* geometry, const double* matrices,
                              const uint8_t* visible, bvhc_scene** out);
bvhc_status bvhc_scene_set_instances(bvhc_scene* scene, int n_instances, const uint32_t* geometry,
                                     const double* matrices, const uint8_t* visible);
/* For each world ray (n x 6 float32): each visible instance's raycastFirst in its local frame
 * (MeshBVH.raycastObject3D, src/core/MeshBVH.js:447-494: the ray through the inverse matrix,
 * direction normalised, near / far divided by |direction * world scale|), the hit point mapped
 * back to world space with its distance from the ray origin (convertRaycastIntersect,
 * src/utils/GeometryRayIntersectUtilities.js:3-17), and the closest of them (equal distances
 * keep the lower instance).  hits: world distance and point, the geometry's faceIndex and local
 * barycoord; instance[i]: the hit's instance (the Intersection's batchId), BVHC_NO_HIT if none. */
bvhc_status bvhc_scene_raycast_first(bvhc_scene* scene, const float* rays, uint64_t n, int side, float near_dist,
                                     float far_dist, bvhc_hit* hits, uint32_t* instance, int mem, void* stream);
/* The same without firstHitOnly (the BatchedMesh raycast, then the raycaster's sort): every hit of
 * every visible instance, in world space, ordered by distance (equal distances: instance order,
 * then each instance's DFS order).  Stores the first `cap` hits per ray at hits[i * cap ..] and
 * their instances at instance[i * cap ..] (BVHC_NO_HIT past the count); counts[i] receives the
 * total.  cap 0 computes the counts only. */
bvhc_status bvhc_scene_raycast(bvhc_scene* scene, const float* rays, uint64_t n, int side, float near_dist,
                               float far_dist, uint32_t cap, uint32_t* counts, bvhc_hit* hits, uint32_t* instance,
                               int mem, void* stream);
void bvhc_scene_destroy(bvhc_scene* scene);
/* Kernel variant of bvhc_scene_raycast_first (no reference counterpart; results are the same for
 * every variant): resident blocks per SM 14 (0), 10 (1) or 8 (2) -- more blocks hide more latency
 * and leave fewer registers per thread.  The first-hit query walks raycastFirst's records
 * (bvhc_mesh_set_leaf_size applies); the all-hits query the reference's. */
bvhc_status bvhc_scene_set_variant(bvhc_scene* scene, int variant);
/* Ray order of bvhc_scene_raycast_first: 0 input order; 1, 2, 3 the rays sorted by a Morton key
 * (direction; entry point into the instances' world box; that point and the direction); 4 sorted
 * by the first instance the ray reaches in the instance tree, so that the rays of a warp walk the
 * same geometry tree.  Results are the same; results land in the rays' rows. */
bvhc_status bvhc_scene_set_order(bvhc_scene* scene, int kind);

/* raycastFirst that allocates nothing.  No counterpart in the reference: it exists for callers
 * that must not call cudaMalloc -- code inside someone else's fixed device-memory budget, a
 * latency-critical thread where an allocation could stall or fail, or a host that allocates only
 * at start-up.  Same arguments and results as bvhc_raycast_first (the persistent traversal with the
 * mesh's order / refill / occupancy).  Its scratch (work counter, and device staging of host
 * buffers) is a fixed 3.6 MB device array that each GPU loading the library holds until exit:
 *   - host-memory calls take at most 65,536 rays; more returns BVHC_ERR_SCRATCH_LIMIT;
 *   - device-memory calls are not size-limited;
 *   - all calls share the array: calls that overlap on the GPU (other streams or threads) race;
 *   - the first call on a device looks the array up on that device: make it before any stream
 *     capture.  A cudaDeviceReset ends the context the address belongs to (and every mesh made on
 *     the device before it); the next call on that device, with a mesh made after the reset, looks
 *     the array up again and is a set-up call in the same sense. */
bvhc_status bvhc_raycast_first_noalloc(bvhc_mesh* mesh, const float* rays, uint64_t n, int side, float near_dist,
                                       float far_dist, bvhc_hit* out, int mem, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Gradients (no reference counterpart: the forward values are the reference's raycastFirst and
 * closestPointToPoint results; the backward differentiates the same formulas).  All buffers are
 * device memory; work is enqueued on `stream`.
 */
/* Uploads the geometry's triangle -> vertex map and positions, which the backward passes use to
 * replay each query's recorded triangle and to address vertex gradients. */
bvhc_status bvhc_mesh_enable_gradients(bvhc_mesh* mesh, const void* index, int index_elem_bytes, uint64_t index_count,
                                       const float* positions, uint64_t n_verts, int stride_floats);
/* Backward of raycastFirst: rays (n x 6) and the forward's hits; grad_distance (n, nullable) and
 * grad_barycoord (n x 3, nullable) are dL/d(distance) and dL/d(barycoord).  grad_vertices
 * (n_verts x 3) is ACCUMULATED into (the caller zeroes it); grad_origins / grad_directions (n x 3)
 * are written; any output may be NULL.  Misses contribute nothing. */
bvhc_status bvhc_raycast_first_backward(bvhc_mesh* mesh, const float* rays, const bvhc_hit* hits, uint64_t n,
                                        const float* grad_distance, const float* grad_barycoord, float* grad_vertices,
                                        float* grad_origins, float* grad_directions, void* stream);
/* Backward of closestPointToPoint's distance: points (n x 3), the forward's results,
 * grad_distance (n).  grad_vertices accumulated, grad_points (n x 3) written; zero for null results
 * and for points on the surface (distance 0). */
bvhc_status bvhc_closest_point_backward(bvhc_mesh* mesh, const float* points, const bvhc_closest* results, uint64_t n,
                                        const float* grad_distance, float* grad_vertices, float* grad_points,
                                        void* stream);

/* Intersection attribute fields (src/utils/ThreeRayIntersectUtilities.js:59-117): for every hit,
 * a vertex attribute (`item_size` 1..4 floats per vertex, `stride_floats` apart, n_verts >= the
 * mesh's vertex count) interpolated at the hit point with the hit's barycoord
 * (Triangle.getInterpolation) — uv, uv1, normal or any other attribute.  With `rays` given (the
 * hits' rays, n x 6) a 3-component result pointing along its ray is negated, as the reference does
 * for `normal`.  out: n x item_size floats; misses give zeros. */
bvhc_status bvhc_hit_interpolate(bvhc_mesh* mesh, const bvhc_hit* hits, uint64_t n, const float* attribute,
                                 uint64_t n_verts, int item_size, int stride_floats, const float* rays, float* out,
                                 int mem, void* stream);

/* getTriangleHitPointInfo(point, geometry, triangleIndex) (src/utils/TriangleUtilities.js:65-147)
 * for n (point, faceIndex) pairs, e.g. closestPointToPoint's results: face a / b / c from the
 * mesh's (reordered) index, materialIndex of the first of n_groups (start, count, materialIndex)
 * triplets (index units, count < 0 = Infinity; host memory, at most 64) holding the triangle's first
 * index (0 when none does), the face normal (Triangle.getNormal), barycoord (Triangle.getBarycoord)
 * and uv (Triangle.getInterpolation; (0, 0) when `uv` is null), computed in integer-emulated
 * binary64 so degenerate triangles give the reference's zeros.  points n x 3, faces n, positions
 * and uv with n_verts >= the mesh's vertex count rows `pos_stride` / `uv_stride` floats apart.
 * A faceIndex past the geometry's triangles: BVHC_ERR_INVALID_ARGUMENT for host memory; in
 * device memory it gives a zero record with a, b, c = BVHC_NO_HIT and the device error word
 * reports it. */
bvhc_status bvhc_triangle_hit_point_info(bvhc_mesh* mesh, const float* points, const uint32_t* faces, uint64_t n,
                                         const float* positions, int pos_stride, const float* uv, int uv_stride,
                                         uint64_t n_verts, const int64_t* groups, int n_groups,
                                         bvhc_hit_point_info* out, int mem, void* stream);

/* MeshBVH#intersectsSphere(sphere) for every sphere (src/core/MeshBVH.js:796-809: shapecast with
 * the sphere/box and sphere/triangle tests, src/math/MathUtilities.js:167-201).  spheres: n x 4
 * float32 (centre xyz, radius; device buffers 16-byte aligned); out[i] = 1 when some triangle lies
 * within the radius of the centre, else 0. */
bvhc_status bvhc_intersects_sphere(bvhc_mesh* mesh, const float* spheres, uint64_t n, uint8_t* out, int mem,
                                   void* stream);

/* The triangles within each sphere, collected through shapecast's CONTAINED path (src/core/cast/
 * shapecast.js:41-214: a node box the sphere contains hands its whole triangle range on with
 * contained = true, :111-117) with the callbacks of the reference's sculpting / selection use:
 * a box the sphere misses is skipped (Sphere.intersectsBox), one whose 8 corners lie within the
 * radius is CONTAINED (Sphere.containsPoint), other boxes' triangles are tested one by one
 * (ExtendedTriangle.intersectsSphere).  spheres: n x 4 float32 (centre, radius; device buffers
 * 16-byte aligned); counts[i] the number collected; faces[i * cap ..] the first cap faceIndex
 * values in the reference's traversal order (left child before right, a range in buffer order),
 * BVHC_NO_HIT past the count.  cap 0 computes the counts only. */
bvhc_status bvhc_sphere_triangles(bvhc_mesh* mesh, const float* spheres, uint64_t n, uint32_t cap, uint32_t* counts,
                                  uint32_t* faces, int mem, void* stream);

/* MeshBVH#intersectsBox(box, boxToMesh) for every box (src/core/MeshBVH.js:780-792: shapecast
 * with OrientedBox.intersectsBox / intersectsTriangle, src/math/OrientedBox.js:78-260).  boxes:
 * n x 24 float32 (min xyz, pad, max xyz, pad, then the column-major box-to-mesh matrix as three.js
 * Matrix4.elements; device buffers 16-byte aligned); out[i] = 1 when some triangle meets the
 * oriented box, else 0.  Decisions follow the reference's binary64 arithmetic (float-float with
 * an exact binary64 recheck of close calls). */
bvhc_status bvhc_intersects_box(bvhc_mesh* mesh, const float* boxes, uint64_t n, uint8_t* out, int mem,
                                void* stream);

/* MeshBVH#closestPointToPoint(point, target, minThreshold, maxThreshold) for every point
 * (src/core/MeshBVH.js:874-884, src/core/cast/closestPointToPoint.js:6-78). */
bvhc_status bvhc_closest_point_to_point(bvhc_mesh* mesh, const float* points, uint64_t n, float min_threshold,
                                        float max_threshold, bvhc_closest* out, int mem, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BVHCUDA_H */
