// Morton keys that order rays for coherent traversal (computed by the root-box pre-pass, sorted by
// raysort.cu, one 8-bit radix pass per started byte of key_bits(kind)).
//   1  direction as a cube-map coordinate: the face of the dominant axis (3 bits) followed by the
//      two minor components divided by the major one, 13 bits each over [-1, 1], interleaved
//      (2-D Morton; 29 bits).  For a pinhole camera this is image space: the order is a Morton
//      walk over cells of about a pixel (a 45-degree view spans ~3400 of the 8192 levels).
//   2  scene entry point: where the ray enters the mesh's bounding box (its origin if it starts
//      inside), 8 bits per axis over that box, interleaved (3-D Morton; 24 bits).
//   3  entry point (5 bits per axis, interleaved) followed by the normalised direction (3 bits per
//      axis over [-1, 1], interleaved; 24 bits).
#pragma once

#include <cstdint>

namespace bvhc {

// Radix passes (8-bit digits) that sort keys of `kind`.
inline int ray_sort_passes(int kind) { return kind == 1 ? 4 : 3; }

namespace dev {

__device__ __forceinline__ uint32_t spread3(uint32_t x) {  // 10 bits -> every third bit of 30
  x &= 0x3FFu;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__device__ __forceinline__ uint32_t spread2(uint32_t x) {  // 16 bits -> every second bit of 32
  x &= 0xFFFFu;
  x = (x | (x << 8)) & 0x00FF00FFu;
  x = (x | (x << 4)) & 0x0F0F0F0Fu;
  x = (x | (x << 2)) & 0x33333333u;
  x = (x | (x << 1)) & 0x55555555u;
  return x;
}

__device__ __forceinline__ uint32_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  return spread3(x) | (spread3(y) << 1) | (spread3(z) << 2);
}

// v in [lo, lo + 1 / inv_ext] -> 0 .. levels - 1 (clamped; NaN -> 0)
__device__ __forceinline__ uint32_t quantise(float v, float lo, float inv_ext, float levels) {
  float s = fminf(fmaxf((v - lo) * inv_ext, 0.0f), 1.0f);
  return (uint32_t)fminf(s * levels, levels - 1.0f);
}

struct SceneBox {
  float lo[3], hi[3];
};

// Key of a ray (origin o, direction d, any length) for key kind 1..3; 0 for other kinds.
__device__ __forceinline__ uint32_t ray_key(int kind, float3 o, float3 d, const SceneBox& box) {
  if (kind == 1) {
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    float u, v, m;
    uint32_t face;
    if (ax >= ay && ax >= az) {
      face = d.x < 0.0f ? 1u : 0u;
      u = d.y; v = d.z; m = ax;
    } else if (ay >= az) {
      face = d.y < 0.0f ? 3u : 2u;
      u = d.x; v = d.z; m = ay;
    } else {
      face = d.z < 0.0f ? 5u : 4u;
      u = d.x; v = d.y; m = az;
    }
    float im = m > 0.0f ? 1.0f / m : 0.0f;
    return (face << 26) | spread2(quantise(u * im, -1.0f, 0.5f, 8192.0f)) |
           (spread2(quantise(v * im, -1.0f, 0.5f, 8192.0f)) << 1);
  }
  if (kind != 2 && kind != 3) return 0u;
  // entry into the scene box: the largest near-slab distance, not before the origin
  float ix = d.x != 0.0f ? 1.0f / d.x : 1e30f, iy = d.y != 0.0f ? 1.0f / d.y : 1e30f;
  float iz = d.z != 0.0f ? 1.0f / d.z : 1e30f;
  float tx = fminf((box.lo[0] - o.x) * ix, (box.hi[0] - o.x) * ix);
  float ty = fminf((box.lo[1] - o.y) * iy, (box.hi[1] - o.y) * iy);
  float tz = fminf((box.lo[2] - o.z) * iz, (box.hi[2] - o.z) * iz);
  float t = fmaxf(fmaxf(fmaxf(tx, ty), tz), 0.0f);
  float px = o.x + d.x * t, py = o.y + d.y * t, pz = o.z + d.z * t;
  float sx = box.hi[0] > box.lo[0] ? 1.0f / (box.hi[0] - box.lo[0]) : 0.0f;
  float sy = box.hi[1] > box.lo[1] ? 1.0f / (box.hi[1] - box.lo[1]) : 0.0f;
  float sz = box.hi[2] > box.lo[2] ? 1.0f / (box.hi[2] - box.lo[2]) : 0.0f;
  if (kind == 2) {
    return morton3(quantise(px, box.lo[0], sx, 256.0f), quantise(py, box.lo[1], sy, 256.0f),
                   quantise(pz, box.lo[2], sz, 256.0f));
  }
  float l = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z);
  float il = l > 0.0f ? 1.0f / l : 0.0f;
  uint32_t kp = morton3(quantise(px, box.lo[0], sx, 32.0f), quantise(py, box.lo[1], sy, 32.0f),
                        quantise(pz, box.lo[2], sz, 32.0f));
  uint32_t kd = morton3(quantise(d.x * il, -1.0f, 0.5f, 8.0f), quantise(d.y * il, -1.0f, 0.5f, 8.0f),
                        quantise(d.z * il, -1.0f, 0.5f, 8.0f));
  return (kp << 9) | kd;
}

}  // namespace dev
}  // namespace bvhc
