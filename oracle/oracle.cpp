// Oracle: a float64 CPU restatement of three-mesh-bvh 0.9.14's BVH build and query path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA engine is compared against.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load liboracle.so.
// The product (libbvhcuda) never links, loads or calls it.
//
// JavaScript numbers are IEEE-754 doubles and Float32Array stores round to nearest float32, so
// plain C++ doubles with `(float)` casts at the reference's Float32Array stores reproduce the
// reference arithmetic operation for operation.  The file must be compiled without FMA
// contraction or fast-math (-ffp-contract=off), which the Makefile beside it does.
//
// The reference's triangle arithmetic lives in three.js r185 (`Ray.intersectTriangle`,
// `Triangle.getBarycoord`, `Triangle.getNormal`, `Triangle.closestPointToPoint`), which is not
// vendored.  Those functions are restated here from the published methods they implement:
//   * ray/triangle: D. Eberly, Geometric Tools, "Intersection of a Ray and a Triangle"
//     (sign-of-determinant form, DdN / DdQxE2 / DdE1xQ / QdN, non-strict barycentric tests);
//   * barycentric coordinates: C. Ericson, Real-Time Collision Detection, section 3.4
//     (dot-product solve; a zero Gram determinant yields (0, 0, 0));
//   * closest point on triangle: C. Ericson, Real-Time Collision Detection, section 5.1.5.
//
// Parity pins for this oracle (the reference holds no numeric golden vectors for this path):
//   * Utils.geometryUtils.test.js:6-90   degenerate triangle known answer;
//   * ShapeCasts.test.js:700-754         sphere distance known answers;
//   * ShapeCasts.test.js:872-1027        hit counts and group/side first hit;
//   * RandomRaycasts.test.js:179-208     BVH traversal == brute force over every triangle.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <thread>
#include <vector>

namespace {

constexpr int CENTER = 0, AVERAGE = 1, SAH = 2;             // Constants.js:9,18,28
constexpr double PRIMITIVE_INTERSECT_COST = 1.25;           // Constants.js:56
constexpr double TRAVERSAL_COST = 1.0;                      // Constants.js:57
constexpr int BYTES_PER_NODE = 32;                          // Constants.js:61
constexpr int UINT32_PER_NODE = 8;                          // Constants.js:62
constexpr uint16_t IS_LEAFNODE_FLAG = 0xFFFF;               // Constants.js:63
const double FLOAT32_EPSILON = std::ldexp(1.0, -24);        // Constants.js:71
constexpr int BIN_COUNT = 32;                               // splitUtils.js:4
constexpr int FRONT_SIDE = 0, BACK_SIDE = 1, DOUBLE_SIDE = 2;  // three.js side constants
const double INF = std::numeric_limits<double>::infinity();

struct V3 { double x, y, z; };
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double dist_sq(V3 a, V3 b) {
  double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  return dx * dx + dy * dy + dz * dz;
}

struct Range { int64_t offset, count; };

// ---------------------------------------------------------------------------------------------
// Geometry + BVH state (GeometryBVH.js / MeshBVH.js)
// ---------------------------------------------------------------------------------------------
struct Bvh {
  std::vector<float> pos;            // copy of the position attribute
  int stride = 3;                    // floats per vertex in `pos`
  int64_t n_verts = 0;
  bool has_index = false;
  int index_elem_bytes = 0;          // 2 or 4 when an index exists
  std::vector<uint32_t> index;       // geometry index (reordered in place by a non-indirect build)
  bool indirect = false;
  int indirect_elem_bytes = 0;
  std::vector<uint32_t> indirect_buf;
  std::vector<std::vector<uint8_t>> roots;
  // material-array queries: geometry groups (start, count, materialIndex) in index units and one
  // side per material; empty `sides` means a single side for every triangle
  std::vector<int64_t> groups;
  std::vector<int> sides;

  int64_t vertex_count() const { return has_index ? (int64_t)index.size() : n_verts; }  // geometryUtils.js:3-7
  V3 vertex(int64_t v) const {
    const float* p = &pos[(size_t)v * stride];
    return {(double)p[0], (double)p[1], (double)p[2]};
  }
  // intersectTri: index resolution (ThreeRayIntersectUtilities.js:156-168)
  void tri_vertices(int64_t tri, int64_t abc[3]) const {
    for (int k = 0; k < 3; ++k) abc[k] = has_index ? (int64_t)index[(size_t)tri * 3 + k] : tri * 3 + k;
  }
  int64_t resolve(int64_t i) const { return indirect ? (int64_t)indirect_buf[(size_t)i] : i; }
};

// ---------------------------------------------------------------------------------------------
// Root ranges (geometryUtils.js:60-159)
// ---------------------------------------------------------------------------------------------
struct GroupIn { int64_t start; double count; };  // count may be +Infinity

std::vector<Range> get_root_primitive_ranges(int64_t vertex_count, int64_t draw_start, double draw_count,
                                             const std::vector<GroupIn>& groups, int stride) {
  // getFullPrimitiveRange (geometryUtils.js:62-75)
  double primitive_count = (double)vertex_count / stride;
  double start = (double)draw_start / stride;
  double end = ((double)draw_start + draw_count) / stride;
  double offset = std::max(0.0, start);
  double count = std::min(primitive_count, end) - offset;
  Range draw{(int64_t)std::floor(offset), (int64_t)std::floor(count)};
  if (groups.empty()) return {draw};

  struct Ev { double pos; bool is_start; };
  std::vector<Ev> events;
  double draw_start_p = (double)draw.offset, draw_end_p = (double)(draw.offset + draw.count);
  for (const auto& g : groups) {
    double goff = (double)g.start / stride;
    double gcount = std::isfinite(g.count / stride) ? g.count / stride : (primitive_count - goff);
    double gend = goff + gcount;
    if (goff < draw_end_p && gend > draw_start_p) {
      events.push_back({std::max(draw_start_p, goff), true});
      events.push_back({std::min(draw_end_p, gend), false});
    }
  }
  // geometryUtils.js:130-142 orders by position; the order among equal positions never changes the
  // emitted ranges because a range is only pushed when the position advances.
  std::stable_sort(events.begin(), events.end(), [](const Ev& a, const Ev& b) { return a.pos < b.pos; });
  std::vector<Range> ranges;
  int active = 0;
  double last = 0;
  bool have_last = false;
  for (const auto& e : events) {
    if (active != 0 && (!have_last || e.pos != last)) ranges.push_back({(int64_t)last, (int64_t)(e.pos - last)});
    active += e.is_start ? 1 : -1;
    last = e.pos;
    have_last = true;
  }
  return ranges;
}

// ---------------------------------------------------------------------------------------------
// Build (MeshBVH.js:337-436, buildTree.js, splitUtils.js, sortUtils.js, buildUtils.js,
// computeBoundsUtils.js, ArrayBoxUtilities.js)
// ---------------------------------------------------------------------------------------------
struct Node {
  float bounds[6];
  bool leaf = false;
  int64_t offset = 0, count = 0;
  int split_axis = 0;
  Node* left = nullptr;
  Node* right = nullptr;
  ~Node() { delete left; delete right; }
};

struct Builder {
  Bvh& bvh;
  int strategy, max_depth, target_leaf;
  std::vector<float> pb;   // primitiveBounds Float32Array: [cx, hx, cy, hy, cz, hz] per primitive
  int64_t pb_offset = 0;   // primitiveBounds.offset
  float centroid_cache[6];

  // splitUtils.js:5-17 module-level bin state
  struct Bin { int64_t count; float bounds[6], right_cache[6], left_cache[6]; double candidate; };
  Bin bins[BIN_COUNT];
  float left_bounds[6];

  Builder(Bvh& b, int s, int md, int tl) : bvh(b), strategy(s), max_depth(md), target_leaf(tl) {}

  float& P(int64_t prim, int k) { return pb[(size_t)(prim - pb_offset) * 6 + k]; }

  // MeshBVH.computePrimitiveBounds (MeshBVH.js:365-436)
  void compute_primitive_bounds(int64_t offset, int64_t count) {
    for (int64_t i = offset; i < offset + count; ++i) {
      int64_t tri = bvh.resolve(i);
      int64_t abc[3];
      bvh.tri_vertices(tri, abc);
      for (int el = 0; el < 3; ++el) {
        double a = bvh.pos[(size_t)abc[0] * bvh.stride + el];
        double b = bvh.pos[(size_t)abc[1] * bvh.stride + el];
        double c = bvh.pos[(size_t)abc[2] * bvh.stride + el];
        double mn = a; if (b < mn) mn = b; if (c < mn) mn = c;
        double mx = a; if (b > mx) mx = b; if (c > mx) mx = c;
        double half = (mx - mn) / 2;
        P(i, el * 2 + 0) = (float)(mn + half);
        P(i, el * 2 + 1) = (float)(half + (std::fabs(mn) + half) * FLOAT32_EPSILON);
      }
    }
  }

  // getBounds (computeBoundsUtils.js:4-68)
  void get_bounds(int64_t offset, int64_t count, float* target, float* centroid) {
    double mn[3] = {INF, INF, INF}, mx[3] = {-INF, -INF, -INF};
    double cmn[3] = {INF, INF, INF}, cmx[3] = {-INF, -INF, -INF};
    for (int64_t i = offset; i < offset + count; ++i) {
      for (int d = 0; d < 3; ++d) {
        double c = P(i, 2 * d), h = P(i, 2 * d + 1);
        double l = c - h, r = c + h;
        if (l < mn[d]) mn[d] = l;
        if (r > mx[d]) mx[d] = r;
        if (c < cmn[d]) cmn[d] = c;
        if (c > cmx[d]) cmx[d] = c;
      }
    }
    for (int d = 0; d < 3; ++d) {
      target[d] = (float)mn[d]; target[d + 3] = (float)mx[d];
      centroid[d] = (float)cmn[d]; centroid[d + 3] = (float)cmx[d];
    }
  }

  // ArrayBoxUtilities.js:22-41
  static int longest_edge(const float* b) {
    int idx = -1;
    double best = -INF;
    for (int i = 0; i < 3; ++i) {
      double dist = (double)b[i + 3] - (double)b[i];
      if (dist > best) { best = dist; idx = i; }
    }
    return idx;
  }
  // ArrayBoxUtilities.js:101-108
  static double surface_area(const float* b) {
    double d0 = (double)b[3] - b[0], d1 = (double)b[4] - b[1], d2 = (double)b[5] - b[2];
    return 2 * (d0 * d1 + d1 * d2 + d2 * d0);
  }
  // ArrayBoxUtilities.js:82-99 (expandByPrimitiveBounds)
  void expand(int64_t prim, float* b) {
    for (int d = 0; d < 3; ++d) {
      double c = P(prim, 2 * d), h = P(prim, 2 * d + 1);
      double tmin = c - h, tmax = c + h;
      if (tmin < b[d]) b[d] = (float)tmin;
      if (tmax > b[d + 3]) b[d + 3] = (float)tmax;
    }
  }
  static void make_empty(float* b) {
    for (int d = 0; d < 3; ++d) { b[d] = (float)INF; b[d + 3] = (float)-INF; }
  }
  static void union_bounds(const float* a, const float* b, float* t) {  // ArrayBoxUtilities.js:58-79
    for (int d = 0; d < 3; ++d) {
      t[d] = a[d] < b[d] ? a[d] : b[d];
      t[d + 3] = a[d + 3] > b[d + 3] ? a[d + 3] : b[d + 3];
    }
  }

  // getOptimalSplit (splitUtils.js:21-294)
  void optimal_split(const float* node_bounds, const float* centroid, int64_t offset, int64_t count,
                     int& axis, double& pos) {
    axis = -1;
    pos = 0;
    if (strategy == CENTER) {
      axis = longest_edge(centroid);
      if (axis != -1) pos = ((double)centroid[axis] + (double)centroid[axis + 3]) / 2;
    } else if (strategy == AVERAGE) {
      axis = longest_edge(node_bounds);
      if (axis != -1) {
        double avg = 0;
        for (int64_t i = offset; i < offset + count; ++i) avg += P(i, axis * 2);
        pos = avg / (double)count;
      }
    } else if (strategy == SAH) {
      double root_area = surface_area(node_bounds);
      double best_cost = PRIMITIVE_INTERSECT_COST * (double)count;
      for (int a = 0; a < 3; ++a) {
        double axis_left = centroid[a], axis_right = centroid[a + 3];
        double axis_length = axis_right - axis_left;
        double bin_width = axis_length / BIN_COUNT;
        if (count < BIN_COUNT / 4) {
          // splitUtils.js:63-174: every primitive center is a candidate
          std::vector<Bin*> tb;
          int64_t b = 0;
          for (int64_t i = offset; i < offset + count; ++i, ++b) {
            Bin* bin = &bins[b];
            bin->candidate = P(i, 2 * a);
            bin->count = 0;
            make_empty(bin->right_cache);
            make_empty(bin->left_cache);
            make_empty(bin->bounds);
            expand(i, bin->bounds);
            tb.push_back(bin);
          }
          std::stable_sort(tb.begin(), tb.end(), [](const Bin* x, const Bin* y) { return x->candidate < y->candidate; });
          int64_t split_count = count;
          for (int64_t bi = 0; bi < split_count; ++bi) {
            while (bi + 1 < split_count && tb[bi + 1]->candidate == tb[bi]->candidate) {
              tb.erase(tb.begin() + bi + 1);
              --split_count;
            }
          }
          for (int64_t i = offset; i < offset + count; ++i) {
            double center = P(i, 2 * a);
            for (int64_t bi = 0; bi < split_count; ++bi) {
              Bin* bin = tb[bi];
              if (center >= bin->candidate) {
                expand(i, bin->right_cache);
              } else {
                expand(i, bin->left_cache);
                bin->count++;
              }
            }
          }
          for (int64_t bi = 0; bi < split_count; ++bi) {
            Bin* bin = tb[bi];
            int64_t lc = bin->count, rc = count - bin->count;
            double lp = 0, rp = 0;
            if (lc != 0) lp = surface_area(bin->left_cache) / root_area;
            if (rc != 0) rp = surface_area(bin->right_cache) / root_area;
            double cost = TRAVERSAL_COST + PRIMITIVE_INTERSECT_COST * (lp * (double)lc + rp * (double)rc);
            if (cost < best_cost) { axis = a; best_cost = cost; pos = bin->candidate; }
          }
        } else {
          // splitUtils.js:176-281: 32 uniform bins over the centroid extent
          for (int i = 0; i < BIN_COUNT; ++i) {
            bins[i].count = 0;
            bins[i].candidate = axis_left + bin_width + (double)i * bin_width;
            make_empty(bins[i].bounds);
          }
          for (int64_t i = offset; i < offset + count; ++i) {
            double tri_center = P(i, 2 * a);
            double rel = tri_center - axis_left;
            double q = rel / bin_width;
            int bin_index = std::isnan(q) ? 0 : (int)std::trunc(q);  // `~~` of a value in [0, 32]
            if (bin_index >= BIN_COUNT) bin_index = BIN_COUNT - 1;
            bins[bin_index].count++;
            expand(i, bins[bin_index].bounds);
          }
          std::memcpy(bins[BIN_COUNT - 1].right_cache, bins[BIN_COUNT - 1].bounds, sizeof(float) * 6);
          for (int i = BIN_COUNT - 2; i >= 0; --i) union_bounds(bins[i].bounds, bins[i + 1].right_cache, bins[i].right_cache);
          int64_t left_count = 0;
          for (int i = 0; i < BIN_COUNT - 1; ++i) {
            int64_t bc = bins[i].count;
            if (bc != 0) {
              if (left_count == 0) std::memcpy(left_bounds, bins[i].bounds, sizeof(float) * 6);
              else union_bounds(bins[i].bounds, left_bounds, left_bounds);
            }
            left_count += bc;
            double lp = 0, rp = 0;
            if (left_count != 0) lp = surface_area(left_bounds) / root_area;
            int64_t right_count = count - left_count;
            if (right_count != 0) rp = surface_area(bins[i + 1].right_cache) / root_area;
            double cost = TRAVERSAL_COST + PRIMITIVE_INTERSECT_COST * (lp * (double)left_count + rp * (double)right_count);
            if (cost < best_cost) { axis = a; best_cost = cost; pos = bins[i].candidate; }
          }
        }
      }
    }
  }

  // partition (sortUtils.js:4-62): Hoare partition of the partition buffer and the bounds
  int64_t partition(int64_t offset, int64_t count, int axis, double pos) {
    int64_t left = offset, right = offset + count - 1;
    uint32_t* buf = bvh.indirect ? bvh.indirect_buf.data() : bvh.index.data();
    int stride = bvh.indirect ? 1 : 3;
    while (true) {
      while (left <= right && (double)P(left, axis * 2) < pos) ++left;
      while (left <= right && (double)P(right, axis * 2) >= pos) --right;
      if (left < right) {
        for (int i = 0; i < stride; ++i) std::swap(buf[left * stride + i], buf[right * stride + i]);
        for (int i = 0; i < 6; ++i) std::swap(P(left, i), P(right, i));
        ++left;
        --right;
      } else {
        return left;
      }
    }
  }

  // splitNode (buildTree.js:46-119)
  void split_node(Node* node, int64_t offset, int64_t count, int depth) {
    if (count <= target_leaf || depth >= max_depth) {
      node->leaf = true; node->offset = offset; node->count = count;
      return;
    }
    int axis;
    double pos;
    optimal_split(node->bounds, centroid_cache, offset, count, axis, pos);
    int64_t split_offset = axis == -1 ? -1 : partition(offset, count, axis, pos);
    if (axis == -1 || split_offset == offset || split_offset == offset + count) {
      node->leaf = true; node->offset = offset; node->count = count;
      return;
    }
    node->split_axis = axis;
    node->left = new Node();
    int64_t lcount = split_offset - offset;
    get_bounds(offset, lcount, node->left->bounds, centroid_cache);
    split_node(node->left, offset, lcount, depth + 1);
    node->right = new Node();
    int64_t rcount = count - lcount;
    get_bounds(split_offset, rcount, node->right->bounds, centroid_cache);
    split_node(node->right, split_offset, rcount, depth + 1);
  }

  static int64_t count_nodes(const Node* n) { return n->leaf ? 1 : 1 + count_nodes(n->left) + count_nodes(n->right); }

  // _populateBuffer (buildUtils.js:35-92)
  static int64_t populate(uint8_t* buf, int64_t byte_offset, const Node* n) {
    float* f32 = reinterpret_cast<float*>(buf + byte_offset);
    for (int i = 0; i < 6; ++i) f32[i] = n->bounds[i];
    uint32_t* u32 = reinterpret_cast<uint32_t*>(buf + byte_offset);
    uint16_t* u16 = reinterpret_cast<uint16_t*>(buf + byte_offset);
    if (n->leaf) {
      u32[6] = (uint32_t)n->offset;
      u16[14] = (uint16_t)n->count;
      u16[15] = IS_LEAFNODE_FLAG;
      return byte_offset + BYTES_PER_NODE;
    }
    int64_t right_byte = populate(buf, byte_offset + BYTES_PER_NODE, n->left);
    int64_t rel = right_byte / BYTES_PER_NODE - byte_offset / BYTES_PER_NODE;
    if (rel > (int64_t)4294967296LL) throw std::runtime_error("MeshBVH: Cannot store relative child node offset greater than 32 bits.");
    u32[6] = (uint32_t)rel;
    u32[7] = (uint32_t)n->split_axis;
    return populate(buf, right_byte, n->right);
  }

  // buildPackedTree (buildTree.js:123-152)
  void build(const std::vector<Range>& root_ranges) {
    Range first = root_ranges.front(), last = root_ranges.back();
    Range full{first.offset, last.offset + last.count - first.offset};
    pb.assign((size_t)full.count * 6, 0.0f);
    pb_offset = full.offset;
    compute_primitive_bounds(full.offset, full.count);
    bvh.roots.clear();
    for (const Range& r : root_ranges) {
      Node root;
      get_bounds(r.offset, r.count, root.bounds, centroid_cache);
      split_node(&root, r.offset, r.count, 0);
      int64_t n = count_nodes(&root);
      std::vector<uint8_t> buf((size_t)n * BYTES_PER_NODE, 0);
      populate(buf.data(), 0, &root);
      bvh.roots.push_back(std::move(buf));
    }
  }
};

// ---------------------------------------------------------------------------------------------
// Node buffer accessors (nodeBufferUtils.js:3-47)
// ---------------------------------------------------------------------------------------------
struct NodeView {
  const uint8_t* buf;
  bool is_leaf(int64_t n32) const { return reinterpret_cast<const uint16_t*>(buf)[n32 * 2 + 15] == IS_LEAFNODE_FLAG; }
  uint32_t offset(int64_t n32) const { return reinterpret_cast<const uint32_t*>(buf)[n32 + 6]; }
  uint16_t count(int64_t n32) const { return reinterpret_cast<const uint16_t*>(buf)[n32 * 2 + 14]; }
  int64_t left(int64_t n32) const { return n32 + UINT32_PER_NODE; }
  int64_t right(int64_t n32) const { return n32 + (int64_t)reinterpret_cast<const uint32_t*>(buf)[n32 + 6] * UINT32_PER_NODE; }
  uint32_t split_axis(int64_t n32) const { return reinterpret_cast<const uint32_t*>(buf)[n32 + 7]; }
  double f(int64_t i) const { return (double)reinterpret_cast<const float*>(buf)[i]; }
};

// ---------------------------------------------------------------------------------------------
// Leaf arithmetic (three.js r185 functions restated from their published methods)
// ---------------------------------------------------------------------------------------------
struct Ray { V3 o, d; };

// Eberly ray/triangle, as called by checkIntersection (ThreeRayIntersectUtilities.js:21-47)
bool ray_intersect_triangle(const Ray& ray, V3 a, V3 b, V3 c, bool backface_culling, V3& point) {
  V3 edge1 = sub(b, a), edge2 = sub(c, a);
  V3 normal = cross(edge1, edge2);
  double DdN = dot(ray.d, normal);
  double sign;
  if (DdN > 0) {
    if (backface_culling) return false;
    sign = 1;
  } else if (DdN < 0) {
    sign = -1;
    DdN = -DdN;
  } else {
    return false;
  }
  V3 diff = sub(ray.o, a);
  double DdQxE2 = sign * dot(ray.d, cross(diff, edge2));
  if (DdQxE2 < 0) return false;
  double DdE1xQ = sign * dot(ray.d, cross(edge1, diff));
  if (DdE1xQ < 0) return false;
  if (DdQxE2 + DdE1xQ > DdN) return false;
  double QdN = -sign * dot(diff, normal);
  if (QdN < 0) return false;
  double t = QdN / DdN;
  point = add(ray.o, scale(ray.d, t));
  return true;
}

// Ericson RTCD 3.4 barycentric coordinates, returned as (weight a, weight b, weight c)
V3 barycoord(V3 p, V3 a, V3 b, V3 c) {
  V3 v0 = sub(b, a), v1 = sub(c, a), v2 = sub(p, a);
  double d00 = dot(v0, v0), d01 = dot(v0, v1), d11 = dot(v1, v1);
  double d20 = dot(v2, v0), d21 = dot(v2, v1);
  double denom = d00 * d11 - d01 * d01;
  if (denom == 0) return {0, 0, 0};
  double wb = (d11 * d20 - d01 * d21) / denom;
  double wc = (d00 * d21 - d01 * d20) / denom;
  return {1 - wb - wc, wb, wc};
}

// Face normal: (c - b) x (a - b), normalised; zero for a zero-area triangle
V3 face_normal(V3 a, V3 b, V3 c) {
  V3 n = cross(sub(c, b), sub(a, b));
  double l2 = dot(n, n);
  if (l2 > 0) return scale(n, 1 / std::sqrt(l2));
  return {0, 0, 0};
}

// Ericson RTCD 5.1.5 closest point on triangle
V3 closest_point_on_triangle(V3 p, V3 a, V3 b, V3 c) {
  V3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) return a;
  V3 bp = sub(p, b);
  double d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) return b;
  double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) {
    double v = d1 / (d1 - d3);
    return add(a, scale(ab, v));
  }
  V3 cp = sub(p, c);
  double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) return c;
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    double w = d2 / (d2 - d6);
    return add(a, scale(ac, w));
  }
  double va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
    double w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    return add(b, scale(sub(c, b), w));
  }
  double denom = 1 / (va + vb + vc);
  double v = vb * denom, w = vc * denom;
  return add(add(a, scale(ab, v)), scale(ac, w));
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// C ABI (ctypes)
// ---------------------------------------------------------------------------------------------
extern "C" {

struct orc_hit {
  int64_t face_index;     // -1 = miss
  double distance;
  double point[3];
  double barycoord[3];
  double normal[3];
  int64_t face[3];        // face.a, face.b, face.c
  int64_t material_index; // face.materialIndex
};

struct orc_cp {
  int64_t face_index;     // -1 = null result
  double distance;
  double point[3];
};

struct orc_bvh;

}  // extern "C"

struct orc_bvh { Bvh b; };

namespace {

// checkBufferGeometryIntersection + intersectTri (ThreeRayIntersectUtilities.js:49-230)
bool intersect_tri(const Bvh& g, int side, const Ray& ray, int64_t tri, double near, double far, orc_hit* out) {
  int64_t abc[3];
  g.tri_vertices(tri, abc);
  V3 a = g.vertex(abc[0]), b = g.vertex(abc[1]), c = g.vertex(abc[2]);
  V3 point;
  bool hit = side == BACK_SIDE ? ray_intersect_triangle(ray, c, b, a, true, point)
                               : ray_intersect_triangle(ray, a, b, c, side != DOUBLE_SIDE, point);
  if (!hit) return false;
  double distance = std::sqrt(dist_sq(ray.o, point));
  if (distance < near || distance > far) return false;
  out->face_index = tri;
  out->distance = distance;
  out->point[0] = point.x; out->point[1] = point.y; out->point[2] = point.z;
  V3 bc = barycoord(point, a, b, c);
  out->barycoord[0] = bc.x; out->barycoord[1] = bc.y; out->barycoord[2] = bc.z;
  V3 n = face_normal(a, b, c);
  out->normal[0] = n.x; out->normal[1] = n.y; out->normal[2] = n.z;
  out->face[0] = abc[0]; out->face[1] = abc[1]; out->face[2] = abc[2];
  out->material_index = 0;
  return true;
}

// intersectTri with an array of materials (ThreeRayIntersectUtilities.js:170-205): one test per
// group that contains the triangle, with that group's material side (a missing material reads as
// `undefined`, which tests like FrontSide); all-hits mode keeps every group's hit, first-hit mode
// the first.  Without materials this is the single-side test.
template <class Sink>
bool intersect_tri_groups(const Bvh& g, int side, const Ray& ray, int64_t tri, double near, double far, Sink sink) {
  if (g.sides.empty()) {
    orc_hit h;
    if (!intersect_tri(g, side, ray, tri, near, far, &h)) return false;
    return sink(h);
  }
  int64_t first = tri * 3;
  for (size_t k = 0; k + 2 < g.groups.size(); k += 3) {
    int64_t start = g.groups[k], count = g.groups[k + 1], mat = g.groups[k + 2];
    if (first >= start && (count < 0 || first < start + count)) {
      int s = (mat >= 0 && mat < (int64_t)g.sides.size()) ? g.sides[(size_t)mat] : FRONT_SIDE;
      orc_hit h;
      if (intersect_tri(g, s, ray, tri, near, far, &h)) {
        h.material_index = mat;
        if (sink(h)) return true;
      }
    }
  }
  return false;
}

// intersectsNodeBounds (intersectUtils.js:2-78)
bool intersects_node_bounds(const NodeView& nv, int64_t n32, const Ray& ray, double near, double far) {
  double tmin, tmax, tymin, tymax, tzmin, tzmax;
  double invx = 1 / ray.d.x, invy = 1 / ray.d.y, invz = 1 / ray.d.z;
  double ox = ray.o.x, oy = ray.o.y, oz = ray.o.z;
  double minx = nv.f(n32), maxx = nv.f(n32 + 3);
  double miny = nv.f(n32 + 1), maxy = nv.f(n32 + 4);
  double minz = nv.f(n32 + 2), maxz = nv.f(n32 + 5);
  if (invx >= 0) { tmin = (minx - ox) * invx; tmax = (maxx - ox) * invx; }
  else { tmin = (maxx - ox) * invx; tmax = (minx - ox) * invx; }
  if (invy >= 0) { tymin = (miny - oy) * invy; tymax = (maxy - oy) * invy; }
  else { tymin = (maxy - oy) * invy; tymax = (miny - oy) * invy; }
  if ((tmin > tymax) || (tymin > tmax)) return false;
  if (tymin > tmin || std::isnan(tmin)) tmin = tymin;
  if (tymax < tmax || std::isnan(tmax)) tmax = tymax;
  if (invz >= 0) { tzmin = (minz - oz) * invz; tzmax = (maxz - oz) * invz; }
  else { tzmin = (maxz - oz) * invz; tzmax = (minz - oz) * invz; }
  if ((tmin > tzmax) || (tzmin > tmax)) return false;
  if (tzmin > tmin || tmin != tmin) tmin = tzmin;
  if (tzmax < tmax || tmax != tmax) tmax = tzmax;
  return tmin <= far && tmax >= near;
}

struct Counters { int64_t nodes = 0, tris = 0; };

// _raycastFirst (raycastFirst.template.js:19-103) with intersectClosestTri (iterationUtils.template.js:24-53)
bool raycast_first_rec(const Bvh& g, const NodeView& nv, int64_t n32, int side, const Ray& ray, double near,
                       double far, orc_hit* res, Counters& ctr) {
  if (nv.is_leaf(n32)) {
    int64_t offset = nv.offset(n32), count = nv.count(n32);
    double dist = INF;
    bool found = false;
    for (int64_t i = offset; i < offset + count; ++i) {
      orc_hit h;
      ctr.tris++;
      bool hit = intersect_tri_groups(g, side, ray, g.resolve(i), near, far, [&](const orc_hit& x) {
        h = x;
        return true;  // intersectTri returns the first group's hit
      });
      if (hit && h.distance < dist) {
        *res = h;
        dist = h.distance;
        found = true;
      }
    }
    return found;
  }
  int axis = (int)nv.split_axis(n32);
  double ray_dir = axis == 0 ? ray.d.x : axis == 1 ? ray.d.y : ray.d.z;
  bool left_to_right = ray_dir >= 0;
  int64_t c1, c2;
  if (left_to_right) { c1 = nv.left(n32); c2 = nv.right(n32); }
  else { c1 = nv.right(n32); c2 = nv.left(n32); }
  orc_hit r1, r2;
  ctr.nodes++;
  bool has1 = intersects_node_bounds(nv, c1, ray, near, far) && raycast_first_rec(g, nv, c1, side, ray, near, far, &r1, ctr);
  ctr.nodes++;  // c2's bounds are read either by the early-out test or by intersectsNodeBounds
  if (has1) {
    double point = r1.point[axis];
    bool outside = left_to_right ? point <= nv.f(c2 + axis) : point >= nv.f(c2 + axis + 3);
    if (outside) { *res = r1; return true; }
  }
  bool has2 = intersects_node_bounds(nv, c2, ray, near, far) && raycast_first_rec(g, nv, c2, side, ray, near, far, &r2, ctr);
  if (has1 && has2) { *res = r1.distance <= r2.distance ? r1 : r2; return true; }
  if (has1) { *res = r1; return true; }
  if (has2) { *res = r2; return true; }
  return false;
}

// MeshBVH.raycastFirst roots loop (MeshBVH.js:558-577)
void raycast_first(const Bvh& g, int side, const Ray& ray, double near, double far, orc_hit* out, Counters& ctr) {
  out->face_index = -1;
  bool have = false;
  for (const auto& root : g.roots) {
    NodeView nv{root.data()};
    orc_hit h;
    ctr.nodes++;  // the root record
    if (raycast_first_rec(g, nv, 0, side, ray, near, far, &h, ctr)) {
      if (!have || h.distance < out->distance) { *out = h; have = true; }
    }
  }
}

// _raycast (raycast.template.js:15-53) with intersectTris (iterationUtils.template.js:4-22)
void raycast_all_rec(const Bvh& g, const NodeView& nv, int64_t n32, int side, const Ray& ray, double near, double far,
                     std::vector<orc_hit>& hits, Counters& ctr) {
  if (nv.is_leaf(n32)) {
    int64_t offset = nv.offset(n32), count = nv.count(n32);
    for (int64_t i = offset; i < offset + count; ++i) {
      ctr.tris++;
      intersect_tri_groups(g, side, ray, g.resolve(i), near, far, [&](const orc_hit& x) {
        hits.push_back(x);
        return false;  // all-hits mode keeps every group's hit
      });
    }
    return;
  }
  int64_t l = nv.left(n32);
  ctr.nodes++;
  if (intersects_node_bounds(nv, l, ray, near, far)) raycast_all_rec(g, nv, l, side, ray, near, far, hits, ctr);
  int64_t r = nv.right(n32);
  ctr.nodes++;
  if (intersects_node_bounds(nv, r, ray, near, far)) raycast_all_rec(g, nv, r, side, ray, near, far, hits, ctr);
}

// closestPointToPoint (cast/closestPointToPoint.js:6-78) through shapecast (BVH.js:342-413,
// shapecast.js:41-214) and iterateOverTriangles (iterationUtils.template.js:55-93)
struct CPState {
  V3 p;
  double min_sq, max_sq;
  double closest_sq = INF;
  int64_t closest_tri = -1;
  V3 closest_point{0, 0, 0};
};

double box_score(const NodeView& nv, int64_t n32, V3 p) {
  // temp.copy(point).clamp(box.min, box.max); temp.distanceToSquared(point)
  double mn[3] = {nv.f(n32), nv.f(n32 + 1), nv.f(n32 + 2)};
  double mx[3] = {nv.f(n32 + 3), nv.f(n32 + 4), nv.f(n32 + 5)};
  double pv[3] = {p.x, p.y, p.z}, t[3];
  for (int k = 0; k < 3; ++k) t[k] = std::max(mn[k], std::min(mx[k], pv[k]));
  V3 tv{t[0], t[1], t[2]};
  return dist_sq(tv, p);
}

bool cp_range(const Bvh& g, int64_t offset, int64_t count, CPState& st, Counters& ctr) {
  for (int64_t i = offset; i < offset + count; ++i) {
    int64_t tri = g.resolve(i);
    int64_t abc[3];
    g.tri_vertices(tri, abc);
    ctr.tris++;
    V3 cp = closest_point_on_triangle(st.p, g.vertex(abc[0]), g.vertex(abc[1]), g.vertex(abc[2]));
    double d2 = dist_sq(st.p, cp);
    if (d2 < st.closest_sq) { st.closest_point = cp; st.closest_sq = d2; st.closest_tri = tri; }
    if (d2 < st.min_sq) return true;
  }
  return false;
}

bool cp_traverse(const Bvh& g, const NodeView& nv, int64_t n32, CPState& st, Counters& ctr) {
  if (nv.is_leaf(n32)) return cp_range(g, nv.offset(n32), nv.count(n32), st, ctr);
  int64_t c1 = nv.left(n32), c2 = nv.right(n32);
  ctr.nodes += 2;
  double s1 = box_score(nv, c1, st.p), s2 = box_score(nv, c2, st.p);
  if (s2 < s1) { std::swap(c1, c2); std::swap(s1, s2); }
  if (s1 < st.closest_sq && s1 < st.max_sq) {
    if (cp_traverse(g, nv, c1, st, ctr)) return true;
  }
  if (s2 < st.closest_sq && s2 < st.max_sq) {
    if (cp_traverse(g, nv, c2, st, ctr)) return true;
  }
  return false;
}

void closest_point(const Bvh& g, V3 p, double min_t, double max_t, orc_cp* out, Counters& ctr) {
  CPState st;
  st.p = p;
  st.min_sq = min_t * min_t;
  st.max_sq = max_t * max_t;
  for (const auto& root : g.roots) {
    NodeView nv{root.data()};
    ctr.nodes++;
    if (cp_traverse(g, nv, 0, st, ctr)) break;
  }
  if (st.closest_sq == INF) {
    out->face_index = -1;
    out->distance = INF;
    out->point[0] = out->point[1] = out->point[2] = 0;
    return;
  }
  out->face_index = st.closest_tri;
  out->distance = std::sqrt(st.closest_sq);
  out->point[0] = st.closest_point.x; out->point[1] = st.closest_point.y; out->point[2] = st.closest_point.z;
}

// ---------------------------------------------------------------------------------------------
// MeshBVH#intersectsSphere (MeshBVH.js:796-809): shapecast with intersectsBounds = the sphere meets
// the box (squared distance from the centre to the clamped centre <= r^2) and intersectsTriangle =
// sphereIntersectTriangle (src/math/MathUtilities.js:167-201): the sphere meets one of the three
// edges (closest point of the segment within r), or the triangle's plane is within r and the
// centre's projection on it lies in the triangle (barycentric test, Ericson RTCD 3.4; a triangle
// with a zero Gram determinant contains nothing).  The result does not depend on the visiting
// order: it is whether any reached triangle meets the sphere.
// ---------------------------------------------------------------------------------------------
// JavaScript Math.min / Math.max (NaN propagates)
inline double js_min(double a, double b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
inline double js_max(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }

double segment_distance(V3 p, V3 s, V3 e) {
  V3 d = sub(e, s);
  double t = dot(sub(p, s), d) / dot(d, d);
  t = js_max(0.0, js_min(1.0, t));
  return std::sqrt(dist_sq(add(s, scale(d, t)), p));
}

bool sphere_meets_triangle(V3 c, double r, V3 a, V3 b, V3 cc) {
  if (segment_distance(c, a, b) <= r) return true;
  if (segment_distance(c, a, cc) <= r) return true;
  if (segment_distance(c, b, cc) <= r) return true;
  V3 n = cross(sub(cc, b), sub(a, b));
  double len = std::sqrt(dot(n, n));
  if (len > 0) n = scale(n, 1.0 / len);
  double constant = -dot(a, n);
  double dp = dot(n, c) + constant;
  if (std::fabs(dp) <= r) {
    V3 pp = add(c, scale(n, -dp));
    V3 v0 = sub(cc, a), v1 = sub(b, a), v2 = sub(pp, a);
    double d00 = dot(v0, v0), d01 = dot(v0, v1), d02 = dot(v0, v2), d11 = dot(v1, v1), d12 = dot(v1, v2);
    double den = d00 * d11 - d01 * d01;
    if (den == 0) return false;
    double u = (d11 * d02 - d01 * d12) / den, v = (d00 * d12 - d01 * d02) / den;
    double wa = 1 - u - v, wb = v;
    if (wa >= 0 && wb >= 0 && wa + wb <= 1) return true;
  }
  return false;
}

bool sphere_traverse(const Bvh& g, const NodeView& nv, int64_t n32, V3 c, double r, Counters& ctr) {
  if (nv.is_leaf(n32)) {
    for (int64_t i = nv.offset(n32); i < nv.offset(n32) + nv.count(n32); ++i) {
      int64_t abc[3];
      g.tri_vertices(g.resolve(i), abc);
      ctr.tris++;
      if (sphere_meets_triangle(c, r, g.vertex(abc[0]), g.vertex(abc[1]), g.vertex(abc[2]))) return true;
    }
    return false;
  }
  const int64_t kids[2] = {nv.left(n32), nv.right(n32)};
  for (int64_t k : kids) {
    ctr.nodes++;
    if (box_score(nv, k, c) <= r * r && sphere_traverse(g, nv, k, c, r, ctr)) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------------------------
// intersectsBox (MeshBVH.js:780-792): OrientedBox (src/math/OrientedBox.js:78-260) against the
// node boxes and triangles, with SeparatingAxisBounds (src/math/SeparatingAxisBounds.js:1-81) and
// ExtendedTriangle's separating axes (src/math/ExtendedTriangle.js:57-86).
// ---------------------------------------------------------------------------------------------
struct SatB { double mn, mx; };
inline bool separated(SatB a, SatB b) { return a.mn > b.mx || b.mn > a.mx; }  // isSeparated

SatB sat_points(V3 axis, const V3* pts, int n) {  // setFromPoints
  SatB r{INF, -INF};
  for (int i = 0; i < n; ++i) {
    double v = dot(axis, pts[i]);
    r.mn = v < r.mn ? v : r.mn;
    r.mx = v > r.mx ? v : r.mx;
  }
  return r;
}

SatB sat_box(V3 axis, const double* bmin, const double* bmax) {  // setFromBox (Math.min / Math.max)
  SatB r{INF, -INF};
  for (int x = 0; x <= 1; ++x)
    for (int y = 0; y <= 1; ++y)
      for (int z = 0; z <= 1; ++z) {
        V3 p{bmin[0] * x + bmax[0] * (1 - x), bmin[1] * y + bmax[1] * (1 - y), bmin[2] * z + bmax[2] * (1 - z)};
        double v = dot(axis, p);
        r.mn = js_min(v, r.mn);
        r.mx = js_max(v, r.mx);
      }
  return r;
}

// The homogeneous transform of a point by a column-major 4x4 matrix, divided by w.
V3 apply_matrix4(V3 v, const double* e) {
  double w = 1 / (e[3] * v.x + e[7] * v.y + e[11] * v.z + e[15]);
  return {(e[0] * v.x + e[4] * v.y + e[8] * v.z + e[12]) * w, (e[1] * v.x + e[5] * v.y + e[9] * v.z + e[13]) * w,
          (e[2] * v.x + e[6] * v.y + e[10] * v.z + e[14]) * w};
}

struct Obb {
  V3 p[8];     // points
  V3 ax[3];    // satAxes
  SatB sb[3];  // satBounds
  SatB al[3];  // alignedSatBounds
};

Obb obb_make(const double* mn, const double* mx, const double* e) {  // OrientedBox.update
  Obb o;
  for (int x = 0; x <= 1; ++x)
    for (int y = 0; y <= 1; ++y)
      for (int z = 0; z <= 1; ++z) {
        V3 v{x ? mx[0] : mn[0], y ? mx[1] : mn[1], z ? mx[2] : mn[2]};
        o.p[x | (y << 1) | (z << 2)] = apply_matrix4(v, e);
      }
  for (int i = 0; i < 3; ++i) {
    o.ax[i] = sub(o.p[0], o.p[1 << i]);
    o.sb[i] = sat_points(o.ax[i], o.p, 8);
  }
  for (int d = 0; d < 3; ++d) {
    SatB r{INF, -INF};
    for (int k = 0; k < 8; ++k) {
      double v = d == 0 ? o.p[k].x : (d == 1 ? o.p[k].y : o.p[k].z);
      r.mn = v < r.mn ? v : r.mn;
      r.mx = v > r.mx ? v : r.mx;
    }
    o.al[d] = r;
  }
  return o;
}

bool obb_meets_box(const Obb& o, const double* bmin, const double* bmax) {  // OrientedBox.intersectsBox
  for (int d = 0; d < 3; ++d)
    if (separated(o.al[d], SatB{bmin[d], bmax[d]})) return false;
  for (int i = 0; i < 3; ++i)
    if (separated(o.sb[i], sat_box(o.ax[i], bmin, bmax))) return false;
  return true;
}

bool obb_meets_triangle(const Obb& o, V3 a, V3 b, V3 c) {  // OrientedBox.intersectsTriangle
  const V3 tp[3] = {a, b, c};
  const V3 ta[4] = {face_normal(a, b, c), sub(a, b), sub(b, c), sub(c, a)};
  for (int i = 0; i < 3; ++i)
    if (separated(o.sb[i], sat_points(o.ax[i], tp, 3))) return false;
  for (int i = 0; i < 3; ++i)
    if (separated(sat_points(ta[i], tp, 3), sat_points(ta[i], o.p, 8))) return false;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 4; ++j) {
      V3 ax = cross(o.ax[i], ta[j]);
      if (separated(sat_points(ax, tp, 3), sat_points(ax, o.p, 8))) return false;
    }
  return true;
}

bool box_traverse(const Bvh& g, const NodeView& nv, int64_t n32, const Obb& o, Counters& ctr) {
  if (nv.is_leaf(n32)) {
    for (int64_t i = nv.offset(n32); i < nv.offset(n32) + nv.count(n32); ++i) {
      int64_t abc[3];
      g.tri_vertices(g.resolve(i), abc);
      ctr.tris++;
      if (obb_meets_triangle(o, g.vertex(abc[0]), g.vertex(abc[1]), g.vertex(abc[2]))) return true;
    }
    return false;
  }
  const int64_t kids[2] = {nv.left(n32), nv.right(n32)};
  for (int64_t k : kids) {
    ctr.nodes++;
    const double bmin[3] = {nv.f(k), nv.f(k + 1), nv.f(k + 2)}, bmax[3] = {nv.f(k + 3), nv.f(k + 4), nv.f(k + 5)};
    if (obb_meets_box(o, bmin, bmax) && box_traverse(g, nv, k, o, ctr)) return true;
  }
  return false;
}

// ---------------------------------------------------------------------------------------------
// Triangles within a sphere through shapecast's CONTAINED path (shapecast.js:41-214, the range
// of a CONTAINED node passed on with contained = true, :111-117), with the callbacks of the
// reference's sculpt / selection use: a node box is NOT_INTERSECTED when the sphere misses it
// (Sphere.intersectsBox: the centre clamped to the box within r), CONTAINED when all 8 corners
// lie within r (Sphere.containsPoint), else INTERSECTED; a triangle is collected when contained
// or when it meets the sphere (ExtendedTriangle.intersectsSphere).
// ---------------------------------------------------------------------------------------------
int sphere_box_relation(const NodeView& nv, int64_t n32, V3 c, double r) {
  const double r2 = r * r;
  const double lo[3] = {nv.f(n32), nv.f(n32 + 1), nv.f(n32 + 2)}, hi[3] = {nv.f(n32 + 3), nv.f(n32 + 4), nv.f(n32 + 5)};
  const double cc[3] = {c.x, c.y, c.z};
  double q[3];
  for (int d = 0; d < 3; ++d) q[d] = std::max(lo[d], std::min(hi[d], cc[d]));  // Vector3.clamp
  if (!(dist_sq(V3{q[0], q[1], q[2]}, c) <= r2)) return 0;
  for (int k = 0; k < 8; ++k) {
    V3 p{(k & 1) ? hi[0] : lo[0], (k & 2) ? hi[1] : lo[1], (k & 4) ? hi[2] : lo[2]};
    if (!(dist_sq(p, c) <= r2)) return 1;
  }
  return 2;
}

void subtree_range(const NodeView& nv, int64_t n32, int64_t& first, int64_t& end, Counters& ctr) {
  // getLeftEndOffset / getRightEndOffset: the outermost leaves of the subtree
  int64_t l = n32;
  while (!nv.is_leaf(l)) l = nv.left(l), ctr.nodes++;
  first = nv.offset(l);
  int64_t r = n32;
  while (!nv.is_leaf(r)) r = nv.right(r), ctr.nodes++;
  end = nv.offset(r) + nv.count(r);
}

// ctr.nodes counts the child boxes tested plus the records walked to a contained subtree's end
// leaves; ctr.tris the triangles tested one by one.
void sphere_collect(const Bvh& g, const NodeView& nv, int64_t n32, V3 c, double r, bool contained,
                    std::vector<int64_t>& out, Counters& ctr) {
  if (contained || nv.is_leaf(n32)) {
    int64_t first, end;
    if (nv.is_leaf(n32)) {
      first = nv.offset(n32);
      end = first + nv.count(n32);
    } else {
      subtree_range(nv, n32, first, end, ctr);
    }
    for (int64_t i = first; i < end; ++i) {
      const int64_t tri = g.resolve(i);
      if (contained) {
        out.push_back(tri);
        continue;
      }
      int64_t abc[3];
      g.tri_vertices(tri, abc);
      ctr.tris++;
      if (sphere_meets_triangle(c, r, g.vertex(abc[0]), g.vertex(abc[1]), g.vertex(abc[2]))) out.push_back(tri);
    }
    return;
  }
  const int64_t kids[2] = {nv.left(n32), nv.right(n32)};
  for (int64_t k : kids) {
    ctr.nodes++;
    const int rel = sphere_box_relation(nv, k, c, r);
    if (rel == 2) sphere_collect(g, nv, k, c, r, true, out, ctr);
    else if (rel == 1) sphere_collect(g, nv, k, c, r, false, out, ctr);
  }
}

template <class F>
void parallel_for(int64_t n, int threads, F f) {
  if (threads <= 1 || n < 64) { f(0, n); return; }
  std::vector<std::thread> pool;
  int64_t chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    int64_t s = t * chunk, e = std::min(n, s + chunk);
    if (s >= e) break;
    pool.emplace_back([=] { f(s, e); });
  }
  for (auto& th : pool) th.join();
}

Ray load_ray(const float* r) { return {{r[0], r[1], r[2]}, {r[3], r[4], r[5]}}; }

}  // namespace

extern "C" {

// Build a MeshBVH (GeometryBVH constructor + init, GeometryBVH.js:93-163).  `index` may be null for a
// non-indexed geometry; `groups` holds (start, count) pairs in index units, count < 0 meaning
// Infinity; draw_count < 0 means Infinity.  Returns null on error.
orc_bvh* orc_build(const float* pos, int64_t n_verts, int stride, const uint32_t* index, int64_t index_count,
                   int index_elem_bytes, const int64_t* groups, int n_groups, int64_t draw_start,
                   int64_t draw_count, int strategy, int max_depth, int target_leaf, int indirect) {
  try {
    auto* h = new orc_bvh();
    Bvh& g = h->b;
    g.pos.assign(pos, pos + (size_t)n_verts * stride);
    g.stride = stride;
    g.n_verts = n_verts;
    if (index) {
      g.has_index = true;
      g.index.assign(index, index + index_count);
      g.index_elem_bytes = index_elem_bytes;
    }
    std::vector<GroupIn> gr;
    for (int i = 0; i < n_groups; ++i) gr.push_back({groups[2 * i], groups[2 * i + 1] < 0 ? INF : (double)groups[2 * i + 1]});
    double dcount = draw_count < 0 ? INF : (double)draw_count;
    std::vector<Range> ranges;
    if (indirect) {
      // generateIndirectBuffer (GeometryBVH.js:9-37)
      ranges = get_root_primitive_ranges(g.vertex_count(), draw_start, dcount, gr, 3);
      g.indirect = true;
      const Range& last = ranges.back();
      g.indirect_elem_bytes = (last.offset + last.count > 65536) ? 4 : 2;
      for (const Range& r : ranges)
        for (int64_t i = 0; i < r.count; ++i) g.indirect_buf.push_back((uint32_t)(r.offset + i));
      ranges = {{0, (int64_t)g.indirect_buf.size()}};
    } else {
      if (!g.has_index) {
        // ensureIndex (geometryUtils.js:15-47)
        g.has_index = true;
        g.index_elem_bytes = n_verts > 65535 ? 4 : 2;
        g.index.resize((size_t)n_verts);
        for (int64_t i = 0; i < n_verts; ++i) g.index[(size_t)i] = (uint32_t)i;
      }
      ranges = get_root_primitive_ranges(g.vertex_count(), draw_start, dcount, gr, 3);
    }
    Builder b(g, strategy, max_depth, target_leaf);
    b.build(ranges);
    return h;
  } catch (...) {
    return nullptr;
  }
}

// MeshBVH.deserialize (MeshBVH.js:160-232) for version-1 data: adopt the buffers as given.
orc_bvh* orc_from_serialized(const void* const* roots, const int64_t* root_bytes, int n_roots, const uint32_t* index,
                             int64_t index_count, const uint32_t* indirect_buf, int64_t n_indirect, const float* pos,
                             int64_t n_verts, int stride) {
  auto* h = new orc_bvh();
  Bvh& g = h->b;
  g.pos.assign(pos, pos + (size_t)n_verts * stride);
  g.stride = stride;
  g.n_verts = n_verts;
  if (index) { g.has_index = true; g.index.assign(index, index + index_count); g.index_elem_bytes = 4; }
  if (indirect_buf) { g.indirect = true; g.indirect_buf.assign(indirect_buf, indirect_buf + n_indirect); g.indirect_elem_bytes = 4; }
  for (int i = 0; i < n_roots; ++i) {
    const uint8_t* p = static_cast<const uint8_t*>(roots[i]);
    g.roots.emplace_back(p, p + root_bytes[i]);
  }
  return h;
}

void orc_free(orc_bvh* h) { delete h; }

// MeshBVH#refit() with no node set (src/core/cast/refit.template.js:4-196, MeshBVH.js:504-508): new
// vertex positions, then per root a post-order walk.  A leaf's box becomes the min / max of its
// triangles' vertex coordinates (float32 values, compared and stored in a Float32Array), and it
// reports a change only when some bound differs from the stored one (`!==`); an internal node is
// rewritten as the union of its children's stored boxes only when a child changed.
static bool refit_node(Bvh& g, uint8_t* buf, int64_t n32) {
  NodeView v{buf};
  float* f = reinterpret_cast<float*>(buf);
  if (v.is_leaf(n32)) {
    const int64_t off = v.offset(n32), cnt = v.count(n32);
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = off; i < off + cnt; ++i) {
      int64_t abc[3];
      g.tri_vertices(g.resolve(i), abc);
      for (int k = 0; k < 3; ++k) {
        const float* p = &g.pos[(size_t)abc[k] * g.stride];
        for (int a = 0; a < 3; ++a) {
          if (p[a] < lo[a]) lo[a] = p[a];
          if (p[a] > hi[a]) hi[a] = p[a];
        }
      }
    }
    bool changed = false;
    for (int a = 0; a < 3; ++a) changed |= f[n32 + a] != lo[a] || f[n32 + 3 + a] != hi[a];
    if (!changed) return false;
    for (int a = 0; a < 3; ++a) {
      f[n32 + a] = lo[a];
      f[n32 + 3 + a] = hi[a];
    }
    return true;
  }
  const int64_t l = v.left(n32), r = v.right(n32);
  const bool lc = refit_node(g, buf, l);
  const bool rc = refit_node(g, buf, r);
  if (lc || rc) {
    for (int a = 0; a < 3; ++a) {
      f[n32 + a] = f[l + a] < f[r + a] ? f[l + a] : f[r + a];
      f[n32 + 3 + a] = f[l + 3 + a] > f[r + 3 + a] ? f[l + 3 + a] : f[r + 3 + a];
    }
  }
  return lc || rc;
}

void orc_refit(orc_bvh* h, const float* pos, int64_t n_verts, int stride) {
  Bvh& g = h->b;
  g.pos.assign(pos, pos + (size_t)n_verts * stride);
  g.stride = stride;
  g.n_verts = n_verts;
  for (auto& root : g.roots) refit_node(g, root.data(), 0);
}

// Material-array mode for raycast queries: `groups` holds (start, count, materialIndex) triplets in
// index units (count < 0 = Infinity) and `sides` one side per material; n_sides = 0 turns it off.
void orc_set_materials(orc_bvh* h, const int64_t* groups, int n_groups, const int* sides, int n_sides) {
  h->b.groups.assign(groups, groups + 3 * n_groups);
  h->b.sides.assign(sides, sides + n_sides);
}
int orc_num_roots(const orc_bvh* h) { return (int)h->b.roots.size(); }
int64_t orc_root_bytes(const orc_bvh* h, int i) { return (int64_t)h->b.roots[i].size(); }
void orc_copy_root(const orc_bvh* h, int i, void* dst) { std::memcpy(dst, h->b.roots[i].data(), h->b.roots[i].size()); }
int orc_index_elem_bytes(const orc_bvh* h) { return h->b.has_index ? h->b.index_elem_bytes : 0; }
int64_t orc_index_count(const orc_bvh* h) { return (int64_t)h->b.index.size(); }
void orc_copy_index(const orc_bvh* h, uint32_t* dst) { std::memcpy(dst, h->b.index.data(), h->b.index.size() * 4); }
int orc_indirect_elem_bytes(const orc_bvh* h) { return h->b.indirect ? h->b.indirect_elem_bytes : 0; }
int64_t orc_indirect_count(const orc_bvh* h) { return (int64_t)h->b.indirect_buf.size(); }
void orc_copy_indirect(const orc_bvh* h, uint32_t* dst) { std::memcpy(dst, h->b.indirect_buf.data(), h->b.indirect_buf.size() * 4); }

// MeshBVH.raycastFirst over a batch of float32 rays (n x [ox oy oz dx dy dz]).  node_reads and
// tri_tests (nullable) receive, per ray, the node records and triangles the reference touches.
void orc_raycast_first(const orc_bvh* h, const float* rays, int64_t n, int side, double near, double far,
                       orc_hit* out, int64_t* node_reads, int64_t* tri_tests, int threads) {
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      Counters c;
      raycast_first(h->b, side, load_ray(rays + 6 * i), near, far, &out[i], c);
      if (node_reads) node_reads[i] = c.nodes;
      if (tri_tests) tri_tests[i] = c.tris;
    }
  });
}

// MeshBVH.raycast (all hits, DFS order) with at most `cap` hits stored per ray; counts[i] is the
// uncapped number of hits.
void orc_raycast_all(const orc_bvh* h, const float* rays, int64_t n, int side, double near, double far, int cap,
                     int32_t* counts, orc_hit* hits, int64_t* node_reads, int64_t* tri_tests, int threads) {
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    std::vector<orc_hit> tmp;
    for (int64_t i = s; i < e; ++i) {
      tmp.clear();
      Counters c;
      Ray ray = load_ray(rays + 6 * i);
      for (const auto& root : h->b.roots) {
        NodeView nv{root.data()};
        c.nodes++;
        raycast_all_rec(h->b, nv, 0, side, ray, near, far, tmp, c);
      }
      counts[i] = (int32_t)tmp.size();
      for (int k = 0; k < (int)tmp.size() && k < cap; ++k) hits[i * cap + k] = tmp[k];
      if (node_reads) node_reads[i] = c.nodes;
      if (tri_tests) tri_tests[i] = c.tris;
    }
  });
}

// MeshBVH.closestPointToPoint over a batch of float32 points (n x 3).
void orc_closest_point(const orc_bvh* h, const float* pts, int64_t n, double min_t, double max_t, orc_cp* out,
                       int64_t* node_reads, int64_t* tri_tests, int threads) {
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      Counters c;
      V3 p{pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]};
      closest_point(h->b, p, min_t, max_t, &out[i], c);
      if (node_reads) node_reads[i] = c.nodes;
      if (tri_tests) tri_tests[i] = c.tris;
    }
  });
}

// intersectsSphere for n spheres (cx, cy, cz, r as float32); out[i] = 1 if the mesh meets sphere i.
// The roots are tried in order (BVH.js:396-411); a root that is a leaf is tested without a box.
void orc_intersects_sphere(const orc_bvh* h, const float* spheres, int64_t n, uint8_t* out, int64_t* node_reads,
                           int64_t* tri_tests, int threads) {
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      Counters c;
      V3 p{spheres[4 * i], spheres[4 * i + 1], spheres[4 * i + 2]};
      double r = spheres[4 * i + 3];
      bool hit = false;
      for (const auto& root : h->b.roots) {
        NodeView nv{root.data()};
        c.nodes++;
        if (sphere_traverse(h->b, nv, 0, p, r, c)) {
          hit = true;
          break;
        }
      }
      out[i] = hit ? 1 : 0;
      if (node_reads) node_reads[i] = c.nodes;
      if (tri_tests) tri_tests[i] = c.tris;
    }
  });
}

// ---------------------------------------------------------------------------------------------
// Instanced raycastFirst: acceleratedBatchedMeshRaycast (ExtensionUtilities.js:87-161) with
// firstHitOnly.  Every visible instance in order: the world ray into the instance's frame
// (MeshBVH.raycastObject3D, MeshBVH.js:447-494: Ray.applyMatrix4 with the inverse matrix, the
// direction normalised; near / far divided by |direction * world scale|), raycastFirst there, the
// hit point back through the world matrix and the distance recomputed from the world origin
// (convertRaycastIntersect, GeometryRayIntersectUtilities.js:3-17); then the closest hit, equal
// distances keeping the lower instance (the raycaster's stable sort).
// ---------------------------------------------------------------------------------------------
// Inverse of a column-major 4x4 matrix by cofactors; all zeros when the determinant is 0.
void invert4(const double* m, double* r) {
  double inv[16];
  inv[0] = m[5] * m[10] * m[15] - m[5] * m[11] * m[14] - m[9] * m[6] * m[15] + m[9] * m[7] * m[14] +
           m[13] * m[6] * m[11] - m[13] * m[7] * m[10];
  inv[4] = -m[4] * m[10] * m[15] + m[4] * m[11] * m[14] + m[8] * m[6] * m[15] - m[8] * m[7] * m[14] -
           m[12] * m[6] * m[11] + m[12] * m[7] * m[10];
  inv[8] = m[4] * m[9] * m[15] - m[4] * m[11] * m[13] - m[8] * m[5] * m[15] + m[8] * m[7] * m[13] +
           m[12] * m[5] * m[11] - m[12] * m[7] * m[9];
  inv[12] = -m[4] * m[9] * m[14] + m[4] * m[10] * m[13] + m[8] * m[5] * m[14] - m[8] * m[6] * m[13] -
            m[12] * m[5] * m[10] + m[12] * m[6] * m[9];
  inv[1] = -m[1] * m[10] * m[15] + m[1] * m[11] * m[14] + m[9] * m[2] * m[15] - m[9] * m[3] * m[14] -
           m[13] * m[2] * m[11] + m[13] * m[3] * m[10];
  inv[5] = m[0] * m[10] * m[15] - m[0] * m[11] * m[14] - m[8] * m[2] * m[15] + m[8] * m[3] * m[14] +
           m[12] * m[2] * m[11] - m[12] * m[3] * m[10];
  inv[9] = -m[0] * m[9] * m[15] + m[0] * m[11] * m[13] + m[8] * m[1] * m[15] - m[8] * m[3] * m[13] -
           m[12] * m[1] * m[11] + m[12] * m[3] * m[9];
  inv[13] = m[0] * m[9] * m[14] - m[0] * m[10] * m[13] - m[8] * m[1] * m[14] + m[8] * m[2] * m[13] +
            m[12] * m[1] * m[10] - m[12] * m[2] * m[9];
  inv[2] = m[1] * m[6] * m[15] - m[1] * m[7] * m[14] - m[5] * m[2] * m[15] + m[5] * m[3] * m[14] +
           m[13] * m[2] * m[7] - m[13] * m[3] * m[6];
  inv[6] = -m[0] * m[6] * m[15] + m[0] * m[7] * m[14] + m[4] * m[2] * m[15] - m[4] * m[3] * m[14] -
           m[12] * m[2] * m[7] + m[12] * m[3] * m[6];
  inv[10] = m[0] * m[5] * m[15] - m[0] * m[7] * m[13] - m[4] * m[1] * m[15] + m[4] * m[3] * m[13] +
            m[12] * m[1] * m[7] - m[12] * m[3] * m[5];
  inv[14] = -m[0] * m[5] * m[14] + m[0] * m[6] * m[13] + m[4] * m[1] * m[14] - m[4] * m[2] * m[13] -
            m[12] * m[1] * m[6] + m[12] * m[2] * m[5];
  inv[3] = -m[1] * m[6] * m[11] + m[1] * m[7] * m[10] + m[5] * m[2] * m[11] - m[5] * m[3] * m[10] -
           m[9] * m[2] * m[7] + m[9] * m[3] * m[6];
  inv[7] = m[0] * m[6] * m[11] - m[0] * m[7] * m[10] - m[4] * m[2] * m[11] + m[4] * m[3] * m[10] +
           m[8] * m[2] * m[7] - m[8] * m[3] * m[6];
  inv[11] = -m[0] * m[5] * m[11] + m[0] * m[7] * m[9] + m[4] * m[1] * m[11] - m[4] * m[3] * m[9] -
            m[8] * m[1] * m[7] + m[8] * m[3] * m[5];
  inv[15] = m[0] * m[5] * m[10] - m[0] * m[6] * m[9] - m[4] * m[1] * m[10] + m[4] * m[2] * m[9] +
            m[8] * m[1] * m[6] - m[8] * m[2] * m[5];
  double det = m[0] * inv[0] + m[1] * inv[4] + m[2] * inv[8] + m[3] * inv[12];
  if (det == 0) {
    for (int k = 0; k < 16; ++k) r[k] = 0;
    return;
  }
  for (int k = 0; k < 16; ++k) r[k] = inv[k] / det;
}

V3 transform_direction(V3 v, const double* e) {  // Vector3.transformDirection: 3x3 part, then normalise
  V3 d{e[0] * v.x + e[4] * v.y + e[8] * v.z, e[1] * v.x + e[5] * v.y + e[9] * v.z, e[2] * v.x + e[6] * v.y + e[10] * v.z};
  double len = std::sqrt(dot(d, d));
  double s = 1 / (len != 0 ? len : 1);
  return {d.x * s, d.y * s, d.z * s};
}

void orc_scene_raycast_first(const orc_bvh* const* geoms, int n_instances, const uint32_t* geometry,
                             const double* matrices, const uint8_t* visible, const float* rays, int64_t n, int side,
                             double near, double far, orc_hit* out, int64_t* instance, int threads) {
  std::vector<double> inv((size_t)n_instances * 16);
  for (int j = 0; j < n_instances; ++j) invert4(matrices + 16 * j, &inv[(size_t)16 * j]);
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      const Ray w = load_ray(rays + 6 * i);
      orc_hit best;
      best.face_index = -1;
      best.distance = INF;
      int64_t best_j = -1;
      for (int j = 0; j < n_instances; ++j) {
        if (visible && !visible[j]) continue;
        const double* M = matrices + 16 * j;
        const double* Mi = &inv[(size_t)16 * j];
        Ray lr{apply_matrix4(w.o, Mi), transform_direction(w.d, Mi)};
        const V3 ws{std::sqrt(M[0] * M[0] + M[1] * M[1] + M[2] * M[2]), std::sqrt(M[4] * M[4] + M[5] * M[5] + M[6] * M[6]),
                    std::sqrt(M[8] * M[8] + M[9] * M[9] + M[10] * M[10])};
        const V3 sd{lr.d.x * ws.x, lr.d.y * ws.y, lr.d.z * ws.z};
        const double scale = std::sqrt(dot(sd, sd));
        orc_hit h;
        Counters c;
        raycast_first(geoms[geometry[j]]->b, side, lr, near / scale, far / scale, &h, c);
        if (h.face_index < 0) continue;
        const V3 pw = apply_matrix4(V3{h.point[0], h.point[1], h.point[2]}, M);
        const double dist = std::sqrt(dist_sq(pw, w.o));
        if (best_j < 0 || dist < best.distance) {
          best = h;
          best.distance = dist;
          best.point[0] = pw.x;
          best.point[1] = pw.y;
          best.point[2] = pw.z;
          best_j = j;
        }
      }
      out[i] = best;
      instance[i] = best_j;
    }
  });
}

// The same without firstHitOnly: every visible instance's MeshBVH.raycast hits (DFS order) in
// instance order, each converted to world space, then the raycaster's stable sort by distance.
// Stores the first `cap` per ray (instance[i * cap + k] their instances) and the total count.
void orc_scene_raycast_all(const orc_bvh* const* geoms, int n_instances, const uint32_t* geometry,
                           const double* matrices, const uint8_t* visible, const float* rays, int64_t n, int side,
                           double near, double far, int cap, int32_t* counts, orc_hit* hits, int64_t* instance,
                           int threads) {
  std::vector<double> inv((size_t)n_instances * 16);
  for (int j = 0; j < n_instances; ++j) invert4(matrices + 16 * j, &inv[(size_t)16 * j]);
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    std::vector<orc_hit> local;
    std::vector<std::pair<orc_hit, int64_t>> all;
    for (int64_t i = s; i < e; ++i) {
      const Ray w = load_ray(rays + 6 * i);
      all.clear();
      for (int j = 0; j < n_instances; ++j) {
        if (visible && !visible[j]) continue;
        const double* M = matrices + 16 * j;
        const double* Mi = &inv[(size_t)16 * j];
        Ray lr{apply_matrix4(w.o, Mi), transform_direction(w.d, Mi)};
        const V3 ws{std::sqrt(M[0] * M[0] + M[1] * M[1] + M[2] * M[2]), std::sqrt(M[4] * M[4] + M[5] * M[5] + M[6] * M[6]),
                    std::sqrt(M[8] * M[8] + M[9] * M[9] + M[10] * M[10])};
        const V3 sd{lr.d.x * ws.x, lr.d.y * ws.y, lr.d.z * ws.z};
        const double scale = std::sqrt(dot(sd, sd));
        const Bvh& g = geoms[geometry[j]]->b;
        local.clear();
        Counters c;
        for (const auto& root : g.roots) {
          NodeView nv{root.data()};
          raycast_all_rec(g, nv, 0, side, lr, near / scale, far / scale, local, c);
        }
        for (orc_hit h : local) {
          const V3 pw = apply_matrix4(V3{h.point[0], h.point[1], h.point[2]}, M);
          h.distance = std::sqrt(dist_sq(pw, w.o));
          h.point[0] = pw.x;
          h.point[1] = pw.y;
          h.point[2] = pw.z;
          all.emplace_back(h, (int64_t)j);
        }
      }
      std::stable_sort(all.begin(), all.end(), [](const std::pair<orc_hit, int64_t>& a,
                                                  const std::pair<orc_hit, int64_t>& b) {
        return a.first.distance < b.first.distance;
      });
      counts[i] = (int32_t)all.size();
      for (int k = 0; k < cap; ++k) {
        if (k < (int)all.size()) {
          hits[i * cap + k] = all[k].first;
          instance[i * cap + k] = all[k].second;
        } else {
          hits[i * cap + k].face_index = -1;
          instance[i * cap + k] = -1;
        }
      }
    }
  });
}

// spheres: n x 4 float32.  counts[i] = triangles collected; faces[i * cap ..] the first cap of them
// in traversal order (-1 past the count).
void orc_sphere_triangles(const orc_bvh* h, const float* spheres, int64_t n, int cap, int32_t* counts, int64_t* faces,
                          int64_t* node_reads, int64_t* tri_tests, int threads) {
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    std::vector<int64_t> out;
    for (int64_t i = s; i < e; ++i) {
      out.clear();
      Counters ctr;
      const V3 c{spheres[4 * i], spheres[4 * i + 1], spheres[4 * i + 2]};
      const double r = spheres[4 * i + 3];
      for (const auto& root : h->b.roots) {
        NodeView nv{root.data()};
        sphere_collect(h->b, nv, 0, c, r, false, out, ctr);
      }
      if (node_reads) node_reads[i] = ctr.nodes;
      if (tri_tests) tri_tests[i] = ctr.tris;
      counts[i] = (int32_t)out.size();
      for (int k = 0; k < cap; ++k) faces[i * cap + k] = k < (int)out.size() ? out[k] : -1;
    }
  });
}

// boxes: n x 24 float32 (min xyz, pad, max xyz, pad, the column-major box-to-mesh matrix).
void orc_intersects_box(const orc_bvh* h, const float* boxes, int64_t n, uint8_t* out, int64_t* node_reads,
                        int64_t* tri_tests, int threads) {
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      const float* q = boxes + 24 * i;
      const double mn[3] = {q[0], q[1], q[2]}, mx[3] = {q[4], q[5], q[6]};
      double m[16];
      for (int k = 0; k < 16; ++k) m[k] = q[8 + k];
      const Obb o = obb_make(mn, mx, m);
      Counters c;
      bool hit = false;
      for (const auto& root : h->b.roots) {
        NodeView nv{root.data()};
        c.nodes++;
        if (box_traverse(h->b, nv, 0, o, c)) {
          hit = true;
          break;
        }
      }
      out[i] = hit ? 1 : 0;
      if (node_reads) node_reads[i] = c.nodes;
      if (tri_tests) tri_tests[i] = c.tris;
    }
  });
}

// Brute force over every triangle the BVH covers (the roots' ranges, in order): all hits, the way
// three.js's un-accelerated Mesh.raycast visits them.
void orc_brute_raycast_all(const orc_bvh* h, const float* rays, int64_t n, int side, double near, double far, int cap,
                           int32_t* counts, orc_hit* hits, int threads) {
  std::vector<Range> ranges;
  for (const auto& root : h->b.roots) {
    // collect the leaf ranges of each root in buffer order
    NodeView nv{root.data()};
    int64_t nodes = (int64_t)root.size() / BYTES_PER_NODE;
    for (int64_t k = 0; k < nodes; ++k)
      if (nv.is_leaf(k * UINT32_PER_NODE)) ranges.push_back({nv.offset(k * UINT32_PER_NODE), nv.count(k * UINT32_PER_NODE)});
  }
  std::sort(ranges.begin(), ranges.end(), [](const Range& a, const Range& b) { return a.offset < b.offset; });
  parallel_for(n, threads, [&](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      Ray ray = load_ray(rays + 6 * i);
      int32_t cnt = 0;
      for (const Range& r : ranges)
        for (int64_t t = r.offset; t < r.offset + r.count; ++t) {
          intersect_tri_groups(h->b, side, ray, h->b.resolve(t), near, far, [&](const orc_hit& hh) {
            if (cnt < cap) hits[i * cap + cnt] = hh;
            ++cnt;
            return false;
          });
        }
      counts[i] = cnt;
    }
  });
}

// Single triangle test (three.js Ray.intersectTriangle semantics), for unit tests.
int orc_ray_triangle(const double* o, const double* d, const double* a, const double* b, const double* c, int side,
                     double near, double far, orc_hit* out) {
  Bvh g;
  g.stride = 3;
  g.n_verts = 3;
  g.pos = {(float)a[0], (float)a[1], (float)a[2], (float)b[0], (float)b[1], (float)b[2], (float)c[0], (float)c[1], (float)c[2]};
  Ray ray{{o[0], o[1], o[2]}, {d[0], d[1], d[2]}};
  out->face_index = -1;
  return intersect_tri(g, side, ray, 0, near, far, out) ? 1 : 0;
}

// Single closest-point-on-triangle evaluation (Ericson 5.1.5), for unit tests.
void orc_closest_point_triangle(const double* p, const double* a, const double* b, const double* c, double* out) {
  V3 r = closest_point_on_triangle({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
  out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

// Gradient reference for the engine's adjoint kernels: the ray/triangle quantities of the Eberly
// formula (N = d.(e1 x e2), U = d.(q x e2), V = d.(e1 x q), T = q.(e1 x e2), t = -T/N,
// wb = U/N, wc = V/N, wa = 1 - wb - wc, distance = t |d|) evaluated on forward-mode dual numbers
// carrying the 15 partials with respect to a, b, c, o, d.  Exact float64 derivatives, independent
// of the engine's hand-written reverse mode.
struct Dual {
  double v;
  double g[15];
};
static Dual dconst(double v) { Dual r{v, {}}; return r; }
static Dual dvar(double v, int i) { Dual r{v, {}}; r.g[i] = 1; return r; }
static Dual operator+(const Dual& a, const Dual& b) { Dual r{a.v + b.v, {}}; for (int i = 0; i < 15; ++i) r.g[i] = a.g[i] + b.g[i]; return r; }
static Dual operator-(const Dual& a, const Dual& b) { Dual r{a.v - b.v, {}}; for (int i = 0; i < 15; ++i) r.g[i] = a.g[i] - b.g[i]; return r; }
static Dual operator*(const Dual& a, const Dual& b) {
  Dual r{a.v * b.v, {}};
  for (int i = 0; i < 15; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r;
}
static Dual operator/(const Dual& a, const Dual& b) {
  Dual r{a.v / b.v, {}};
  for (int i = 0; i < 15; ++i) r.g[i] = (a.g[i] * b.v - a.v * b.g[i]) / (b.v * b.v);
  return r;
}
static Dual dsqrt(const Dual& a) {
  Dual r{std::sqrt(a.v), {}};
  for (int i = 0; i < 15; ++i) r.g[i] = a.g[i] / (2 * r.v);
  return r;
}
struct D3 { Dual x, y, z; };
static D3 dsub(const D3& a, const D3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static Dual ddot(const D3& a, const D3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static D3 dcross(const D3& a, const D3& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

// out[0..4] = distance, t, wa, wb, wc; grads[5][15] = their partials w.r.t. (a, b, c, o, d).
void orc_ray_triangle_jacobian(const double* o, const double* d, const double* a, const double* b, const double* c,
                               double* out5, double* grads) {
  D3 A{dvar(a[0], 0), dvar(a[1], 1), dvar(a[2], 2)}, B{dvar(b[0], 3), dvar(b[1], 4), dvar(b[2], 5)};
  D3 Cc{dvar(c[0], 6), dvar(c[1], 7), dvar(c[2], 8)}, O{dvar(o[0], 9), dvar(o[1], 10), dvar(o[2], 11)};
  D3 Dd{dvar(d[0], 12), dvar(d[1], 13), dvar(d[2], 14)};
  D3 e1 = dsub(B, A), e2 = dsub(Cc, A), q = dsub(O, A);
  D3 n = dcross(e1, e2);
  Dual N = ddot(Dd, n), U = ddot(Dd, dcross(q, e2)), V = ddot(Dd, dcross(e1, q)), T = ddot(q, n);
  Dual t = dconst(0) - T / N, wb = U / N, wc = V / N;
  Dual wa = dconst(1) - wb - wc;
  Dual dist = t * dsqrt(ddot(Dd, Dd));
  const Dual* vals[5] = {&dist, &t, &wa, &wb, &wc};
  for (int k = 0; k < 5; ++k) {
    out5[k] = vals[k]->v;
    for (int i = 0; i < 15; ++i) grads[15 * k + i] = vals[k]->g[i];
  }
}

// Distance from p to triangle (a, b, c) (closest point by Ericson 5.1.5), for finite differences.
double orc_point_triangle_distance(const double* p, const double* a, const double* b, const double* c) {
  V3 P{p[0], p[1], p[2]};
  V3 r = closest_point_on_triangle(P, {a[0], a[1], a[2]}, {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
  return std::sqrt(dist_sq(P, r));
}

// Statistics in the style of getBVHExtremes (debug/Debug.js:36-134): node count, leaf count,
// max depth, total leaf triangles.
void orc_stats(const orc_bvh* h, int64_t* out4) {
  int64_t nodes = 0, leaves = 0, maxd = 0, tris = 0;
  for (const auto& root : h->b.roots) {
    NodeView nv{root.data()};
    std::vector<std::pair<int64_t, int64_t>> st{{0, 0}};
    while (!st.empty()) {
      auto [n, d] = st.back();
      st.pop_back();
      ++nodes;
      maxd = std::max(maxd, d);
      if (nv.is_leaf(n)) { ++leaves; tris += nv.count(n); }
      else { st.push_back({nv.left(n), d + 1}); st.push_back({nv.right(n), d + 1}); }
    }
  }
  out4[0] = nodes; out4[1] = leaves; out4[2] = maxd; out4[3] = tris;
}

}  // extern "C"
