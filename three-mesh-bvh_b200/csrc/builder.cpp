// CPU SAH / CENTER / AVERAGE builder that emits the reference's serialized MeshBVH layout.
//
// This is the build stage in front of the GPU query path: `new MeshBVH(geometry, options)` and
// `MeshBVH.serialize()` (src/core/GeometryBVH.js:93-163, src/core/build/buildTree.js:123-152,
// src/core/MeshBVH.js:112-145).  It reproduces the reference's tree and its in-place reorder of
// the geometry index bit for bit, because the reference's `faceIndex` values and the
// closest-point result beyond `maxThreshold` depend on that exact tree.
//
// Engineering differences from the reference's recursive JS (the numeric rules are identical):
//   * primitive boxes are kept as float32 (lo, hi, center) triples, precomputed once, because
//     every reference use of the padded (center, half) pair reduces to fl32(center -/+ half);
//   * SAH bins for the three axes are filled in one pass over the primitives, and the split
//     costs are then scanned in the reference's axis-major order with its strict `<`;
//   * nodes are written straight into the pre-order buffer with an explicit work stack, the
//     right-child offset being patched when the right child is emitted.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

#include "bvhc_internal.h"

namespace bvhc {
namespace {

constexpr int kBins = 32;                       // splitUtils.js:4 BIN_COUNT
constexpr double kPrimCost = 1.25;              // Constants.js:56 PRIMITIVE_INTERSECT_COST
constexpr double kTravCost = 1.0;               // Constants.js:57 TRAVERSAL_COST
const double kPad = std::ldexp(1.0, -24);       // Constants.js:71 FLOAT32_EPSILON
const float kFInf = std::numeric_limits<float>::infinity();

struct Prim {
  float c[3];   // padded-box center  (primitiveBounds[2d])
  float lo[3];  // fl32(center - half)
  float hi[3];  // fl32(center + half)
};

struct Box {
  float v[6];
  void empty() { v[0] = v[1] = v[2] = kFInf; v[3] = v[4] = v[5] = -kFInf; }
  void grow(const Prim& p) {
    for (int d = 0; d < 3; ++d) {
      if (p.lo[d] < v[d]) v[d] = p.lo[d];
      if (p.hi[d] > v[d + 3]) v[d + 3] = p.hi[d];
    }
  }
  void join(const Box& o) {
    for (int d = 0; d < 3; ++d) {
      v[d] = o.v[d] < v[d] ? o.v[d] : v[d];
      v[d + 3] = o.v[d + 3] > v[d + 3] ? o.v[d + 3] : v[d + 3];
    }
  }
  double area() const {
    double dx = (double)v[3] - v[0], dy = (double)v[4] - v[1], dz = (double)v[5] - v[2];
    return 2 * (dx * dy + dy * dz + dz * dx);
  }
};

int longest_axis(const float* b) {
  int axis = -1;
  double best = -std::numeric_limits<double>::infinity();
  for (int i = 0; i < 3; ++i) {
    double e = (double)b[i + 3] - (double)b[i];
    if (e > best) { best = e; axis = i; }
  }
  return axis;
}

class Builder {
 public:
  Builder(Serialized& s, const float* pos, int stride, int strategy, int max_depth, int leaf)
      : s_(s), pos_(pos), stride_(stride), strategy_(strategy), max_depth_(max_depth), leaf_(leaf) {}

  void run(const std::vector<Range>& roots) {
    int64_t first = roots.front().offset;
    int64_t last = roots.back().offset + roots.back().count;
    base_ = first;
    prims_.resize((size_t)(last - first));
    for (int64_t i = first; i < last; ++i) prims_[(size_t)(i - first)] = make_prim(i);
    s_.roots.clear();
    for (const Range& r : roots) s_.roots.push_back(build_root(r));
  }

 private:
  Serialized& s_;
  const float* pos_;
  int stride_, strategy_, max_depth_, leaf_;
  int64_t base_ = 0;
  std::vector<Prim> prims_;

  Prim& prim(int64_t i) { return prims_[(size_t)(i - base_)]; }

  uint32_t vertex_of(int64_t tri, int k) const {
    return s_.has_index ? s_.index[(size_t)tri * 3 + k] : (uint32_t)(tri * 3 + k);
  }

  // MeshBVH.computePrimitiveBounds (MeshBVH.js:365-436): double arithmetic, float32 stores.
  Prim make_prim(int64_t i) {
    int64_t tri = s_.indirect ? (int64_t)s_.indirect_buf[(size_t)i] : i;
    const float* va = pos_ + (size_t)vertex_of(tri, 0) * stride_;
    const float* vb = pos_ + (size_t)vertex_of(tri, 1) * stride_;
    const float* vc = pos_ + (size_t)vertex_of(tri, 2) * stride_;
    Prim p;
    for (int d = 0; d < 3; ++d) {
      double a = va[d], b = vb[d], c = vc[d];
      double mn = std::min(a, std::min(b, c)), mx = std::max(a, std::max(b, c));
      double half = (mx - mn) / 2;
      float center = (float)(mn + half);
      float padded = (float)(half + (std::fabs(mn) + half) * kPad);
      p.c[d] = center;
      p.lo[d] = (float)((double)center - (double)padded);
      p.hi[d] = (float)((double)center + (double)padded);
    }
    return p;
  }

  // getBounds (computeBoundsUtils.js:4-68)
  void range_bounds(int64_t off, int64_t cnt, float* box, float* cbox) {
    Box b, cb;
    b.empty();
    cb.empty();
    for (int64_t i = off; i < off + cnt; ++i) {
      const Prim& p = prim(i);
      b.grow(p);
      for (int d = 0; d < 3; ++d) {
        if (p.c[d] < cb.v[d]) cb.v[d] = p.c[d];
        if (p.c[d] > cb.v[d + 3]) cb.v[d + 3] = p.c[d];
      }
    }
    std::memcpy(box, b.v, sizeof b.v);
    std::memcpy(cbox, cb.v, sizeof cb.v);
  }

  // SAH with every primitive center as a candidate (splitUtils.js:63-174), one axis.
  void sah_small(int a, int64_t off, int64_t cnt, double root_area, double& best, int& axis, double& pos) {
    float cand[kBins / 4];
    int n = 0;
    for (int64_t i = off; i < off + cnt; ++i) cand[n++] = prim(i).c[a];
    std::sort(cand, cand + n);
    n = (int)(std::unique(cand, cand + n) - cand);
    for (int k = 0; k < n; ++k) {
      Box l, r;
      l.empty();
      r.empty();
      int64_t lc = 0;
      for (int64_t i = off; i < off + cnt; ++i) {
        const Prim& p = prim(i);
        if ((double)p.c[a] >= (double)cand[k]) r.grow(p);
        else { l.grow(p); ++lc; }
      }
      int64_t rc = cnt - lc;
      double lp = lc != 0 ? l.area() / root_area : 0.0;
      double rp = rc != 0 ? r.area() / root_area : 0.0;
      double cost = kTravCost + kPrimCost * (lp * (double)lc + rp * (double)rc);
      if (cost < best) { axis = a; best = cost; pos = cand[k]; }
    }
  }

  // getOptimalSplit (splitUtils.js:21-294)
  void choose_split(const float* box, const float* cbox, int64_t off, int64_t cnt, int& axis, double& pos) {
    axis = -1;
    pos = 0;
    if (strategy_ == kCenter) {
      axis = longest_axis(cbox);
      if (axis != -1) pos = ((double)cbox[axis] + (double)cbox[axis + 3]) / 2;
      return;
    }
    if (strategy_ == kAverage) {
      axis = longest_axis(box);
      if (axis != -1) {
        double sum = 0;
        for (int64_t i = off; i < off + cnt; ++i) sum += prim(i).c[axis];
        pos = sum / (double)cnt;
      }
      return;
    }
    if (strategy_ != kSah) return;
    Box node;
    std::memcpy(node.v, box, sizeof node.v);
    double root_area = node.area();
    double best = kPrimCost * (double)cnt;
    if (cnt < kBins / 4) {
      for (int a = 0; a < 3; ++a) sah_small(a, off, cnt, root_area, best, axis, pos);
      return;
    }
    // 32 uniform bins per axis over the centroid extent (splitUtils.js:176-281), filled in one pass.
    double left_edge[3], width[3];
    for (int a = 0; a < 3; ++a) {
      left_edge[a] = cbox[a];
      width[a] = ((double)cbox[a + 3] - (double)cbox[a]) / kBins;
    }
    Box bins[3][kBins];
    int64_t counts[3][kBins] = {};
    for (int a = 0; a < 3; ++a)
      for (int i = 0; i < kBins; ++i) bins[a][i].empty();
    for (int64_t i = off; i < off + cnt; ++i) {
      const Prim& p = prim(i);
      for (int a = 0; a < 3; ++a) {
        double q = ((double)p.c[a] - left_edge[a]) / width[a];
        // truncation toward zero; NaN (zero-width extent) lands in bin 0; overflow clamps to the last bin
        int bi = q != q ? 0 : (q >= (double)kBins ? kBins - 1 : (int)q);
        counts[a][bi]++;
        bins[a][bi].grow(p);
      }
    }
    for (int a = 0; a < 3; ++a) {
      Box suffix[kBins];
      suffix[kBins - 1] = bins[a][kBins - 1];
      for (int i = kBins - 2; i >= 0; --i) {
        suffix[i] = bins[a][i];
        suffix[i].join(suffix[i + 1]);
      }
      Box left;
      int64_t lc = 0;
      for (int i = 0; i < kBins - 1; ++i) {
        if (counts[a][i] != 0) {
          if (lc == 0) left = bins[a][i];
          else left.join(bins[a][i]);
        }
        lc += counts[a][i];
        int64_t rc = cnt - lc;
        double lp = lc != 0 ? left.area() / root_area : 0.0;
        double rp = rc != 0 ? suffix[i + 1].area() / root_area : 0.0;
        double cost = kTravCost + kPrimCost * (lp * (double)lc + rp * (double)rc);
        if (cost < best) {
          axis = a;
          best = cost;
          pos = left_edge[a] + width[a] + (double)i * width[a];
        }
      }
    }
  }

  // Hoare partition of the partition buffer and the primitive boxes (sortUtils.js:4-62).
  int64_t split_range(int64_t off, int64_t cnt, int axis, double pos) {
    uint32_t* buf = s_.indirect ? s_.indirect_buf.data() : s_.index.data();
    const int w = s_.indirect ? 1 : 3;
    int64_t l = off, r = off + cnt - 1;
    for (;;) {
      while (l <= r && (double)prim(l).c[axis] < pos) ++l;
      while (l <= r && (double)prim(r).c[axis] >= pos) --r;
      if (l >= r) return l;
      for (int k = 0; k < w; ++k) std::swap(buf[(size_t)l * w + k], buf[(size_t)r * w + k]);
      std::swap(prim(l), prim(r));
      ++l;
      --r;
    }
  }

  struct Task {
    int64_t off, cnt;
    int depth;
    int64_t parent;  // node that receives this node's right-child offset, or -1
    float box[6], cbox[6];
  };

  std::vector<uint8_t> build_root(const Range& root) {
    std::vector<uint32_t> words;  // the node buffer as 8 words per node
    std::vector<Task> stack;
    Task t0{root.offset, root.count, 0, -1, {}, {}};
    range_bounds(root.offset, root.count, t0.box, t0.cbox);
    stack.push_back(t0);
    while (!stack.empty()) {
      Task t = stack.back();
      stack.pop_back();
      int64_t idx = (int64_t)words.size() / 8;
      if (t.parent >= 0) {
        int64_t rel = idx - t.parent;
        if (rel > (int64_t)4294967296LL) throw std::runtime_error("relative child offset exceeds 32 bits");
        words[(size_t)t.parent * 8 + 6] = (uint32_t)rel;
      }
      words.resize(words.size() + 8, 0);
      uint32_t* w = &words[(size_t)idx * 8];
      std::memcpy(w, t.box, sizeof t.box);

      bool leaf = t.cnt <= leaf_ || t.depth >= max_depth_;
      int axis = -1;
      int64_t mid = -1;
      if (!leaf) {
        double pos;
        choose_split(t.box, t.cbox, t.off, t.cnt, axis, pos);
        if (axis != -1) mid = split_range(t.off, t.cnt, axis, pos);
        leaf = axis == -1 || mid == t.off || mid == t.off + t.cnt;
      }
      if (leaf) {
        w[6] = (uint32_t)t.off;
        w[7] = (uint32_t)(t.cnt & 0xFFFF) | 0xFFFF0000u;  // count (u16 at byte 28) + leaf flag (byte 30)
        continue;
      }
      w[7] = (uint32_t)axis;
      Task lt{t.off, mid - t.off, t.depth + 1, -1, {}, {}};
      Task rt{mid, t.off + t.cnt - mid, t.depth + 1, idx, {}, {}};
      range_bounds(lt.off, lt.cnt, lt.box, lt.cbox);
      range_bounds(rt.off, rt.cnt, rt.box, rt.cbox);
      stack.push_back(rt);
      stack.push_back(lt);
    }
    std::vector<uint8_t> out(words.size() * 4);
    std::memcpy(out.data(), words.data(), out.size());
    return out;
  }
};

}  // namespace

// getRootPrimitiveRanges (geometryUtils.js:60-159) with stride 3.
std::vector<Range> root_ranges(int64_t vertex_count, int64_t draw_start, int64_t draw_count,
                               const int64_t* groups, int n_groups) {
  const double inf = std::numeric_limits<double>::infinity();
  double prim_count = (double)vertex_count / 3;
  double start = (double)draw_start / 3;
  double end = ((double)draw_start + (draw_count < 0 ? inf : (double)draw_count)) / 3;
  double off = std::max(0.0, start);
  double cnt = std::min(prim_count, end) - off;
  Range draw{(int64_t)std::floor(off), (int64_t)std::floor(cnt)};
  if (n_groups <= 0) return {draw};
  struct Ev { double at; int delta; };
  std::vector<Ev> ev;
  double lo = (double)draw.offset, hi = (double)(draw.offset + draw.count);
  for (int g = 0; g < n_groups; ++g) {
    double gs = (double)groups[2 * g] / 3;
    double gc = groups[2 * g + 1] < 0 ? prim_count - gs : (double)groups[2 * g + 1] / 3;
    double ge = gs + gc;
    if (gs < hi && ge > lo) {
      ev.push_back({std::max(lo, gs), +1});
      ev.push_back({std::min(hi, ge), -1});
    }
  }
  std::stable_sort(ev.begin(), ev.end(), [](const Ev& a, const Ev& b) { return a.at < b.at; });
  std::vector<Range> out;
  int active = 0;
  double prev = -inf;
  for (const Ev& e : ev) {
    if (active != 0 && e.at != prev) out.push_back({(int64_t)prev, (int64_t)(e.at - prev)});
    active += e.delta;
    prev = e.at;
  }
  return out;
}

std::vector<Range> prepare_build(Serialized& s, uint64_t n_verts, const int64_t* groups, int n_groups,
                                 int64_t range_start, int64_t range_count, bool indirect) {
  std::vector<Range> ranges;
  if (indirect) {
    // generateIndirectBuffer (GeometryBVH.js:9-37)
    int64_t vc = s.has_index ? (int64_t)s.index.size() : (int64_t)n_verts;
    std::vector<Range> rr = root_ranges(vc, range_start, range_count, groups, n_groups);
    s.indirect = true;
    s.indirect_elem_bytes = (rr.back().offset + rr.back().count > 65536) ? 4 : 2;
    s.indirect_buf.clear();
    for (const Range& r : rr)
      for (int64_t i = 0; i < r.count; ++i) s.indirect_buf.push_back((uint32_t)(r.offset + i));
    ranges = {{0, (int64_t)s.indirect_buf.size()}};
  } else {
    if (!s.has_index) {
      // ensureIndex (geometryUtils.js:15-47)
      s.has_index = true;
      s.index_elem_bytes = n_verts > 65535 ? 4 : 2;
      s.index.resize((size_t)n_verts);
      for (uint64_t i = 0; i < n_verts; ++i) s.index[(size_t)i] = (uint32_t)i;
    }
    ranges = root_ranges((int64_t)s.index.size(), range_start, range_count, groups, n_groups);
  }
  if (ranges.empty()) throw std::runtime_error("geometry has no triangles in its draw range / groups");
  return ranges;
}

void build_serialized(Serialized& s, const float* pos, uint64_t n_verts, int stride, const int64_t* groups,
                      int n_groups, int64_t range_start, int64_t range_count, int strategy, int max_depth,
                      int leaf, bool indirect) {
  std::vector<Range> ranges = prepare_build(s, n_verts, groups, n_groups, range_start, range_count, indirect);
  Builder b(s, pos, stride, strategy, max_depth, leaf);
  b.run(ranges);
}

}  // namespace bvhc
