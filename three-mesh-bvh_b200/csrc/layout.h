// Device-resident layout of a MeshBVH, shared by the host re-layout code and the kernels.
//
// The serialized reference node (src/core/build/buildUtils.js:31-92) is 32 bytes: its own box
// plus either (right-child offset, split axis) or (triangle offset, count, leaf flag).  A query
// visiting an internal node always reads BOTH children's boxes (intersectsNodeBounds on c1 and
// c2, or both shapecast scores), so the device layout stores, per internal node, one 64-byte
// "child pair" record holding the two child boxes and the two child links.  One visit is then
// one 64-byte, 64-byte-aligned read (two 32-byte sectors), instead of two scattered 32-byte
// reads.  The root's own box is never tested by the reference and is not stored.
//
// Leaf triangles are copied into 48-byte records in DFS leaf order, vertices inline, so that a
// leaf is one contiguous run of 16-byte-aligned loads and needs no index indirection.
#pragma once

#include <cstdint>

namespace bvhc {

// Child link: internal child -> child-pair record index; leaf child -> kLeafBit | first
// triangle record; an empty leaf -> kEmptyLeaf.
constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kEmptyLeaf = 0xFFFFFFFFu;
constexpr int kMaxStack = 64;  // deepest supported tree (the reference's default maxDepth is 40)

struct alignas(64) PairNode {
  // f[0..5]  left child  box (min xyz, max xyz)
  // f[6..11] right child box
  float f[12];
  uint32_t link[2];   // left, right child links
  uint32_t axis;      // split axis of this node (0, 1, 2)
  uint32_t flags;     // 0 (reserved)
};
static_assert(sizeof(PairNode) == 64, "PairNode must be 64 bytes");

// Four-child record for raycastFirst's warp-cooperative traversal, collapsed from the child-pair
// tree (each internal child replaced by its own two children, largest surface area first, until
// four children or only leaves remain).  Planes are stored per axis for the four children, so one
// 16-byte load gives one bound of all four boxes.  Unused children have link kEmptyLeaf.
struct alignas(64) QuadNode {
  float lo[3][4];     // lo[axis][child]
  float hi[3][4];     // hi[axis][child]
  uint32_t link[4];   // internal child -> quad record index; leaf -> kLeafBit | first triangle record
  uint32_t pad[4];
};
static_assert(sizeof(QuadNode) == 128, "QuadNode must be 128 bytes");

struct alignas(16) TriRecord {
  // v[0..8] = a.xyz, b.xyz, c.xyz ; face = reference faceIndex ; flags bit 0 = last in leaf ;
  // material = materialIndex of the geometry group holding the triangle (kNoMaterial: none)
  float v[9];
  uint32_t face;
  uint32_t flags;
  uint32_t material;
};
static_assert(sizeof(TriRecord) == 48, "TriRecord must be 48 bytes");

constexpr uint32_t kTriLast = 1u;
constexpr uint32_t kNoMaterial = 0xFFFFFFFFu;
constexpr int kMaxMaterials = 64;

// Per-call side selection: a single side for every triangle, or one side per material.
struct SideTable {
  int8_t side[kMaxMaterials];
  int32_t n;        // number of materials
  int32_t per_material;
};

}  // namespace bvhc
