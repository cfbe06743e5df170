// Oracle (test infrastructure only): CPU restatement of GGEMS's meshed-solid
// host preparation, used to check the product's builder bit for bit and to
// feed meshed scenes to the oracle and to GGEMS's own mesh kernels.
//
//   binary STL reader + bounding spheres  src/io/GGEMSSTLReader.cc:71-253
//   world transform of the triangles      src/geometries/GGEMSMeshedSolid.cc:230-300 (UpdateTriangles)
//   octree box                            src/geometries/GGEMSMeshedSolid.cc:340-455
//                                         (ComputeOctreeCenter / ComputeHalfWidthCenter)
//   octree nodes + triangle insertion     src/geometries/GGEMSOctree.cc:40-316
//
// Output layout (include/ggems_b200.h, gg_solid): triangles[n][13] = p0, p1, p2,
// sphere center, radius; nodes[m][6] = center, half width; node_first[m+1] and
// node_triangles[] list each node's triangles in the order GGEMS's linked list
// visits them (the last inserted first).
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <vector>

#include "ggems_b200.h"

namespace {

struct P3 {
  float x, y, z;
};

float dot(P3 a, P3 b) {
  float d = a.x * b.x;
  d += a.y * b.y;
  d += a.z * b.z;
  return d;
}

struct Tri {
  P3 p[3];
  P3 c;
  float r;
};

// GGEMSMeshTriangle: Ritter-style bounding sphere of the three vertices.
Tri make_triangle(P3 a, P3 b, P3 c) {
  Tri t;
  t.p[0] = a;
  t.p[1] = b;
  t.p[2] = c;
  int minx = 0, maxx = 0, miny = 0, maxy = 0, minz = 0, maxz = 0;
  for (int i = 1; i < 3; ++i) {
    if (t.p[i].x < t.p[minx].x) minx = i;
    if (t.p[i].x > t.p[maxx].x) maxx = i;
    if (t.p[i].y < t.p[miny].y) miny = i;
    if (t.p[i].y > t.p[maxy].y) maxy = i;
    if (t.p[i].z < t.p[minz].z) minz = i;
    if (t.p[i].z > t.p[maxz].z) maxz = i;
  }
  P3 dx{t.p[maxx].x - t.p[minx].x, t.p[maxx].y - t.p[minx].y, t.p[maxx].z - t.p[minx].z};
  P3 dy{t.p[maxy].x - t.p[miny].x, t.p[maxy].y - t.p[miny].y, t.p[maxy].z - t.p[miny].z};
  P3 dz{t.p[maxz].x - t.p[minz].x, t.p[maxz].y - t.p[minz].y, t.p[maxz].z - t.p[minz].z};
  float d2x = dot(dx, dx), d2y = dot(dy, dy), d2z = dot(dz, dz);
  int lo = minx, hi = maxx;
  if (d2y > d2x && d2y > d2z) {
    lo = miny;
    hi = maxy;
  } else if (d2z > d2y && d2z > d2x) {
    lo = minz;
    hi = maxz;
  }
  P3 center{(t.p[lo].x + t.p[hi].x) * 0.5f, (t.p[lo].y + t.p[hi].y) * 0.5f, (t.p[lo].z + t.p[hi].z) * 0.5f};
  P3 d{t.p[hi].x - center.x, t.p[hi].y - center.y, t.p[hi].z - center.z};
  float radius = sqrtf(dot(d, d));
  for (int i = 0; i < 3; ++i) {
    P3 v{t.p[i].x - center.x, t.p[i].y - center.y, t.p[i].z - center.z};
    float dist2 = dot(v, v);
    if (dist2 > radius * radius) {
      float dist = sqrtf(dist2);
      float grown = (radius + dist) * 0.5f;
      float k = (grown - radius) / dist;
      radius = grown;
      center.x += v.x * k;
      center.y += v.y * k;
      center.z += v.z * k;
    }
  }
  t.c = center;
  t.r = radius;
  return t;
}

bool read_stl(const char* path, std::vector<Tri>& out) {
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  char header[80];
  uint32_t n = 0;
  in.read(header, 80);
  in.read(reinterpret_cast<char*>(&n), 4);
  if (!in) return false;
  out.clear();
  out.reserve(n);
  for (uint32_t i = 0; i < n; ++i) {
    float v[12];
    uint16_t attribute;
    in.read(reinterpret_cast<char*>(v), 48);
    in.read(reinterpret_cast<char*>(&attribute), 2);
    if (!in) return false;
    out.push_back(make_triangle(P3{v[3], v[4], v[5]}, P3{v[6], v[7], v[8]}, P3{v[9], v[10], v[11]}));
  }
  return true;
}

// Octree box: vertex bounds (initialised with FLT_MAX / FLT_MIN as GGEMS
// does), grown by 2.5 % per side and rounded outwards to whole millimetres.
void octree_box(const std::vector<Tri>& tris, float center[3], float half[3]) {
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
  for (const Tri& t : tris)
    for (int j = 0; j < 3; ++j) {
      const float c[3] = {t.p[j].x, t.p[j].y, t.p[j].z};
      for (int a = 0; a < 3; ++a) {
        if (c[a] < lo[a]) lo[a] = c[a];
        if (c[a] > hi[a]) hi[a] = c[a];
      }
    }
  for (int a = 0; a < 3; ++a) {
    float grow = (hi[a] - lo[a]) * 0.025f;
    lo[a] -= grow;
    hi[a] += grow;
    lo[a] = lo[a] < 0.0f ? std::floor(lo[a]) : std::ceil(lo[a]);
    hi[a] = hi[a] < 0.0f ? std::floor(hi[a]) : std::ceil(hi[a]);
    center[a] = (hi[a] + lo[a]) * 0.5f;
    half[a] = (hi[a] - lo[a]) * 0.5f;
  }
}

}  // namespace

extern "C" {

// Number of triangles in a binary STL file and of octree nodes at `depth`.
__attribute__((visibility("default"))) int gg_oracle_mesh_counts(const char* stl_path, int depth, int32_t* triangles,
                                                                 int32_t* nodes) {
  std::ifstream in(stl_path, std::ios::binary);
  if (!in || depth < 1 || depth > 10) return GG_ERROR_INVALID_ARGUMENT;
  char header[80];
  uint32_t n = 0;
  in.read(header, 80);
  in.read(reinterpret_cast<char*>(&n), 4);
  if (!in) return GG_ERROR_INVALID_ARGUMENT;
  *triangles = static_cast<int32_t>(n);
  *nodes = static_cast<int32_t>(std::pow(8.0f, static_cast<float>(depth)) - 1) / 7;
  return GG_OK;
}

// Build the meshed solid: STL triangles moved by `matrix` (the solid's
// GGfloat44 geometry transformation, row-major), octree of `depth` levels.
// Outputs are caller-allocated with the sizes gg_oracle_mesh_counts gives;
// border_min/border_max receive the octree box (the solid's OBB).
__attribute__((visibility("default"))) int gg_oracle_build_mesh(const char* stl_path, const float* matrix, int depth,
                                                                float* triangles, float* nodes, int32_t* node_first,
                                                                int32_t* node_triangles, float* border_min,
                                                                float* border_max) {
  std::vector<Tri> tris;
  if (!read_stl(stl_path, tris) || depth < 1 || depth > 10) return GG_ERROR_INVALID_ARGUMENT;
  // UpdateTriangles: rows of the rotation part, then the translation column.
  const P3 r0{matrix[0], matrix[1], matrix[2]}, r1{matrix[4], matrix[5], matrix[6]}, r2{matrix[8], matrix[9], matrix[10]};
  const P3 tr{matrix[3], matrix[7], matrix[11]};
  for (Tri& t : tris) {
    for (int j = 0; j < 3; ++j) {
      P3 q{dot(r0, t.p[j]), dot(r1, t.p[j]), dot(r2, t.p[j])};
      t.p[j] = P3{q.x + tr.x, q.y + tr.y, q.z + tr.z};
    }
    P3 q{dot(r0, t.c), dot(r1, t.c), dot(r2, t.c)};
    t.c = P3{q.x + tr.x, q.y + tr.y, q.z + tr.z};
  }
  float center[3], half[3];
  octree_box(tris, center, half);
  const int total = static_cast<int>(std::pow(8.0f, static_cast<float>(depth)) - 1) / 7;
  struct Node {
    float c[3], h[3];
    int first_child;
  };
  std::vector<Node> node(total);
  node[0] = Node{{center[0], center[1], center[2]}, {half[0], half[1], half[2]}, 1};
  int id = 1;
  for (int level = 2; level <= depth; ++level) {
    const int through = (static_cast<int>(std::pow(8, level)) - 1) / 7;
    const int in_level = through - (static_cast<int>(std::pow(8.0, level - 1)) - 1) / 7;
    for (int j = 0; j < in_level; ++j) {
      const int mother = (((id + 1) + 6) >> 3) - 1;
      float step[3];
      for (int a = 0; a < 3; ++a)
        step[a] = static_cast<float>(half[a] / std::pow(2.0f, static_cast<float>(level) - 1.0f));
      const int k = j % 8;
      const float off[3] = {(k & 1) ? step[0] : -step[0], (k & 2) ? step[1] : -step[1], (k & 4) ? step[2] : -step[2]};
      for (int a = 0; a < 3; ++a) {
        node[id].c[a] = node[mother].c[a] + off[a];
        node[id].h[a] = step[a];
      }
      node[id].first_child = 8 * (id + 1) - 7;
      ++id;
    }
  }
  // InsertTriangles: descend while the bounding sphere stays on one side of
  // every center plane; the triangle is prepended to the list of the node
  // where it straddles (or of the deepest node reached).
  std::vector<std::vector<int32_t>> lists(total);
  for (size_t t = 0; t < tris.size(); ++t) {
    const float tc[3] = {tris[t].c.x, tris[t].c.y, tris[t].c.z};
    int cur = 0;
    for (int level = 0; level < depth; ++level) {
      int index = 0, straddle = 0;
      for (int a = 0; a < 3; ++a) {
        float delta = tc[a] - node[cur].c[a];
        if (fabsf(delta) <= tris[t].r) {
          straddle = 1;
          break;
        }
        if (delta > 0.0f) index |= (1 << a);
      }
      if (!straddle && level != depth - 1) {
        cur = node[cur].first_child + index;
      } else {
        lists[cur].push_back(static_cast<int32_t>(t));
        break;
      }
    }
  }
  for (size_t t = 0; t < tris.size(); ++t) {
    float* o = triangles + t * GG_TRIANGLE_FLOATS;
    for (int j = 0; j < 3; ++j) {
      o[3 * j] = tris[t].p[j].x;
      o[3 * j + 1] = tris[t].p[j].y;
      o[3 * j + 2] = tris[t].p[j].z;
    }
    o[9] = tris[t].c.x;
    o[10] = tris[t].c.y;
    o[11] = tris[t].c.z;
    o[12] = tris[t].r;
  }
  int32_t k = 0;
  for (int n = 0; n < total; ++n) {
    for (int a = 0; a < 3; ++a) {
      nodes[6 * n + a] = node[n].c[a];
      nodes[6 * n + 3 + a] = node[n].h[a];
    }
    node_first[n] = k;
    for (auto it = lists[n].rbegin(); it != lists[n].rend(); ++it) node_triangles[k++] = *it;
  }
  node_first[total] = k;
  for (int a = 0; a < 3; ++a) {
    border_min[a] = center[a] - half[a];
    border_max[a] = center[a] + half[a];
  }
  return GG_OK;
}

}  // extern "C"
