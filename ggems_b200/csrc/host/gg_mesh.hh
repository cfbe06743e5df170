// Meshed solid preparation for the GGEMS-compatible host API: binary STL
// reading, world transform of the triangles, octree box and triangle
// insertion, as GGEMSMeshedPhantom::Initialize does it
// (src/navigators/GGEMSMeshedPhantom.cc:72-130).
#ifndef GG_MESH_HH
#define GG_MESH_HH

#include <cstdint>
#include <string>
#include <vector>

namespace gg {

struct MeshedSolid {
  int32_t number_of_triangles = 0;
  std::vector<float> triangles;         // [n][GG_TRIANGLE_FLOATS]: p0, p1, p2, sphere center, radius
  std::vector<float> nodes;             // [m][6]: center, half width
  std::vector<int32_t> node_first;      // [m + 1]
  std::vector<int32_t> node_triangles;  // per node, in linked-list visiting order
  float border_min[3] = {0, 0, 0};      // octree box = the solid's OBB (identity matrix)
  float border_max[3] = {0, 0, 0};
};

// `matrix`: the solid's GGfloat44 geometry transformation (row-major).
MeshedSolid build_meshed_solid(const std::string& stl_path, const float matrix[16], int octree_depth);

}  // namespace gg

#endif
