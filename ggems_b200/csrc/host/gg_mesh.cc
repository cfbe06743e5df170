// Meshed solid preparation (see gg_mesh.hh).  Every float operation keeps the
// reference's order so that triangles, bounding spheres and the octree are
// bit-identical to GGEMS's.  Sources followed:
//   binary STL + bounding sphere   src/io/GGEMSSTLReader.cc:71-253
//   triangle transform             src/geometries/GGEMSMeshedSolid.cc:230-300
//   octree box                     src/geometries/GGEMSMeshedSolid.cc:340-455
//   octree nodes / insertion       src/geometries/GGEMSOctree.cc:40-316
#include "gg_mesh.hh"

#include <cfloat>
#include <cmath>
#include <fstream>

#include "ggems_b200.h"
#include "gg_host.hh"

namespace gg {

namespace {

struct Vec {
  float x, y, z;
};

inline float dot(Vec a, Vec b) {
  float r = a.x * b.x;
  r += a.y * b.y;
  r += a.z * b.z;
  return r;
}
inline Vec minus(Vec a, Vec b) { return Vec{a.x - b.x, a.y - b.y, a.z - b.z}; }

struct Facet {
  Vec v[3];
  Vec center;
  float radius;
};

// Bounding sphere: start from the vertex pair most separated along a
// principal axis, then grow to enclose each vertex in turn.
void bound(Facet& f) {
  int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (int i = 1; i < 3; ++i) {
    const float c[3] = {f.v[i].x, f.v[i].y, f.v[i].z};
    for (int a = 0; a < 3; ++a) {
      const float clo[3] = {f.v[lo[a]].x, f.v[lo[a]].y, f.v[lo[a]].z};
      const float chi[3] = {f.v[hi[a]].x, f.v[hi[a]].y, f.v[hi[a]].z};
      if (c[a] < clo[a]) lo[a] = i;
      if (c[a] > chi[a]) hi[a] = i;
    }
  }
  float span[3];
  for (int a = 0; a < 3; ++a) {
    Vec d = minus(f.v[hi[a]], f.v[lo[a]]);
    span[a] = dot(d, d);
  }
  int a = 0;
  if (span[1] > span[0] && span[1] > span[2]) a = 1;
  else if (span[2] > span[1] && span[2] > span[0]) a = 2;
  const Vec p = f.v[lo[a]], q = f.v[hi[a]];
  Vec c{(p.x + q.x) * 0.5f, (p.y + q.y) * 0.5f, (p.z + q.z) * 0.5f};
  Vec d = minus(q, c);
  float r = sqrtf(dot(d, d));
  for (int i = 0; i < 3; ++i) {
    Vec w = minus(f.v[i], c);
    float w2 = dot(w, w);
    if (w2 > r * r) {
      float len = sqrtf(w2);
      float grown = (r + len) * 0.5f;
      float k = (grown - r) / len;
      r = grown;
      c.x += w.x * k;
      c.y += w.y * k;
      c.z += w.z * k;
    }
  }
  f.center = c;
  f.radius = r;
}

std::vector<Facet> read_binary_stl(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error("GGEMSSTLReader", "Read", "Problem reading filename: " + path);
  char header[80];
  uint32_t n = 0;
  in.read(header, 80);
  in.read(reinterpret_cast<char*>(&n), 4);
  if (!in) throw Error("GGEMSSTLReader", "Read", "Truncated STL header: " + path);
  std::vector<Facet> facets(n);
  for (uint32_t i = 0; i < n; ++i) {
    float rec[12];
    uint16_t attribute;
    in.read(reinterpret_cast<char*>(rec), sizeof(rec));
    in.read(reinterpret_cast<char*>(&attribute), 2);
    if (!in) throw Error("GGEMSSTLReader", "Read", "Truncated STL file: " + path);
    for (int k = 0; k < 3; ++k) facets[i].v[k] = Vec{rec[3 + 3 * k], rec[4 + 3 * k], rec[5 + 3 * k]};
    bound(facets[i]);
  }
  return facets;
}

}  // namespace

MeshedSolid build_meshed_solid(const std::string& stl_path, const float matrix[16], int depth) {
  if (depth < 1 || depth > 8) throw Error("GGEMSOctree", "GGEMSOctree", "Max. depth too large in Octree!!!");
  std::vector<Facet> facets = read_binary_stl(stl_path);
  if (facets.empty()) throw Error("GGEMSMeshedSolid", "LoadVolumeImage", "no triangle in " + stl_path);

  // Rotation rows then translation column of the geometry transformation.
  const Vec row[3] = {{matrix[0], matrix[1], matrix[2]}, {matrix[4], matrix[5], matrix[6]}, {matrix[8], matrix[9], matrix[10]}};
  const Vec shift{matrix[3], matrix[7], matrix[11]};
  auto move = [&](Vec p) { return Vec{dot(row[0], p) + shift.x, dot(row[1], p) + shift.y, dot(row[2], p) + shift.z}; };
  for (Facet& f : facets) {
    for (Vec& v : f.v) v = move(v);
    f.center = move(f.center);
  }

  // Octree box: vertex bounds (high side starts at FLT_MIN, as in GGEMS),
  // grown 2.5 % per side, rounded outwards to whole units.
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
  for (const Facet& f : facets)
    for (const Vec& v : f.v) {
      const float c[3] = {v.x, v.y, v.z};
      for (int a = 0; a < 3; ++a) {
        if (c[a] < lo[a]) lo[a] = c[a];
        if (c[a] > hi[a]) hi[a] = c[a];
      }
    }
  float center[3], half[3];
  for (int a = 0; a < 3; ++a) {
    const float grow = (hi[a] - lo[a]) * 0.025f;
    float l = lo[a] - grow, h = hi[a] + grow;
    l = l < 0.0f ? std::floor(l) : std::ceil(l);
    h = h < 0.0f ? std::floor(h) : std::ceil(h);
    center[a] = (h + l) * 0.5f;
    half[a] = (h - l) * 0.5f;
  }

  // Nodes level by level; children of node m are 8m+1 .. 8m+8, child k is
  // offset by +/- half the parent's half width along x (bit 0), y (bit 1), z (bit 2).
  const int total = static_cast<int>(std::pow(8.0f, static_cast<float>(depth)) - 1) / 7;
  MeshedSolid out;
  out.nodes.assign(static_cast<size_t>(total) * 6, 0.0f);
  for (int a = 0; a < 3; ++a) {
    out.nodes[a] = center[a];
    out.nodes[3 + a] = half[a];
  }
  int id = 1;
  for (int level = 2; level <= depth; ++level) {
    const int count = (static_cast<int>(std::pow(8, level)) - 1) / 7 - (static_cast<int>(std::pow(8.0, level - 1)) - 1) / 7;
    float step[3];
    for (int a = 0; a < 3; ++a) step[a] = static_cast<float>(half[a] / std::pow(2.0f, static_cast<float>(level) - 1.0f));
    for (int j = 0; j < count; ++j, ++id) {
      const int parent = (id - 1) >> 3;
      const int k = j & 7;
      for (int a = 0; a < 3; ++a) {
        out.nodes[6 * id + a] = out.nodes[6 * parent + a] + (((k >> a) & 1) ? step[a] : -step[a]);
        out.nodes[6 * id + 3 + a] = step[a];
      }
    }
  }

  // Each triangle goes to the deepest node whose center planes its bounding
  // sphere does not touch; a node's list is visited last-inserted first.
  std::vector<std::vector<int32_t>> owned(total);
  for (size_t t = 0; t < facets.size(); ++t) {
    const float c[3] = {facets[t].center.x, facets[t].center.y, facets[t].center.z};
    int node = 0;
    for (int level = 0; level < depth; ++level) {
      int octant = 0;
      bool straddles = false;
      for (int a = 0; a < 3 && !straddles; ++a) {
        const float delta = c[a] - out.nodes[6 * node + a];
        if (fabsf(delta) <= facets[t].radius) straddles = true;
        else if (delta > 0.0f) octant |= 1 << a;
      }
      if (straddles || level == depth - 1) {
        owned[node].push_back(static_cast<int32_t>(t));
        break;
      }
      node = 8 * node + 1 + octant;
    }
  }

  out.number_of_triangles = static_cast<int32_t>(facets.size());
  out.triangles.resize(facets.size() * GG_TRIANGLE_FLOATS);
  for (size_t t = 0; t < facets.size(); ++t) {
    float* o = out.triangles.data() + t * GG_TRIANGLE_FLOATS;
    for (int k = 0; k < 3; ++k) {
      o[3 * k] = facets[t].v[k].x;
      o[3 * k + 1] = facets[t].v[k].y;
      o[3 * k + 2] = facets[t].v[k].z;
    }
    o[9] = facets[t].center.x;
    o[10] = facets[t].center.y;
    o[11] = facets[t].center.z;
    o[12] = facets[t].radius;
  }
  out.node_first.resize(total + 1);
  out.node_triangles.reserve(facets.size());
  for (int n = 0; n < total; ++n) {
    out.node_first[n] = static_cast<int32_t>(out.node_triangles.size());
    out.node_triangles.insert(out.node_triangles.end(), owned[n].rbegin(), owned[n].rend());
  }
  out.node_first[total] = static_cast<int32_t>(out.node_triangles.size());
  for (int a = 0; a < 3; ++a) {
    out.border_min[a] = center[a] - half[a];
    out.border_max[a] = center[a] + half[a];
  }
  return out;
}

}  // namespace gg
