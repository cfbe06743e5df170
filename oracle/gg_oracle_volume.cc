// Oracle (test infrastructure only): CPU restatement of GGEMS's phantom-volume
// steps, used to check the product's gg_volume_* kernels bit for bit.
//
//   voxel index + centre, inside tests  src/kernels/DrawGGEMSBox.cl:71-97,
//                                       DrawGGEMSTube.cl:71-93, DrawGGEMSSphere.cl:71-88
//   range table -> labels               include/GGEMS/geometries/GGEMSVoxelizedSolid.hh:162-257
//                                       (ConvertImageToLabel: every line rewrites the
//                                       voxels its range holds, in file order; 255 = none)
//
// The draw restatement is pinned against the reference's own Draw kernels
// built through the OpenCL shim (oracle/_ref); the label conversion is host
// code inside a class template that needs GGEMS's OpenCL manager, so it is
// anchored on its source only.
#include <cstdint>
#include <cstring>

#include "ggems_b200.h"

namespace {

template <class T>
void draw(T* volume, const int32_t dim[3], const float es[3], const gg_shape& s) {
  const uint64_t n = static_cast<uint64_t>(dim[0]) * dim[1] * dim[2];
  const int dx = dim[0], dy = dim[1];
  for (uint64_t id = 0; id < n; ++id) {
    // index arithmetic of the reference, in its types (size_t, then int)
    const int iy = static_cast<int>((id % static_cast<uint64_t>(static_cast<int64_t>(dx * dx))) /
                                    static_cast<uint64_t>(static_cast<int64_t>(dx)));
    const int ix = static_cast<int>((id % static_cast<uint64_t>(static_cast<int64_t>(dx * dy))) -
                                    static_cast<uint64_t>(static_cast<int64_t>(iy * dx)));
    const int iz = static_cast<int>(id / static_cast<uint64_t>(static_cast<int64_t>(dx * dy)));
    const int idx[3] = {ix, iy, iz};
    float c[3];
    for (int a = 0; a < 3; ++a) {
      const float half = es[a] / 2.0f;
      const float f = (1.0f - static_cast<float>(dim[a])) + 2.0f * static_cast<float>(idx[a]);
      const float centre = half * f;
      c[a] = centre - s.position[a];
    }
    bool inside = false;
    if (s.type == GG_SHAPE_BOX) {
      const float hw = s.size[0] / 2.0f, hh = s.size[1] / 2.0f, hd = s.size[2] / 2.0f;
      inside = c[2] <= hd && c[2] >= -hd && c[1] <= hh && c[1] >= -hh && c[0] <= hw && c[0] >= -hw;
    } else if (s.type == GG_SHAPE_TUBE) {
      const float h2 = s.size[2] / 2.0f;
      const float xx = c[0] * c[0], yy = c[1] * c[1];
      const float rx2 = s.size[0] * s.size[0], ry2 = s.size[1] * s.size[1];
      const float e = xx / rx2 + yy / ry2;
      inside = c[2] <= h2 && c[2] >= -h2 && e <= 1.0f;
    } else if (s.type == GG_SHAPE_SPHERE) {
      const float xx = c[0] * c[0], yy = c[1] * c[1], zz = c[2] * c[2];
      const float d2 = (xx + yy) + zz;
      inside = d2 <= s.size[0] * s.size[0];
    }
    if (inside) volume[id] = static_cast<T>(s.label_value);
  }
}

template <class T>
int64_t labels(const T* image, uint64_t n, const float* first, const float* last, int ranges, uint8_t* out) {
  for (uint64_t i = 0; i < n; ++i) out[i] = 255;
  for (int r = 0; r < ranges; ++r) {
    for (uint64_t i = 0; i < n; ++i) {
      const float v = static_cast<float>(image[i]);
      if ((v == first[r] && v == last[r]) || (v >= first[r] && v < last[r])) out[i] = static_cast<uint8_t>(r);
    }
  }
  int64_t missing = 0;
  for (uint64_t i = 0; i < n; ++i) missing += out[i] == 255;
  return missing;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) int gg_oracle_draw(void* volume, int32_t met_type, const int32_t dim[3],
                                                          const float es[3], const gg_shape* shape) {
  switch (met_type) {
    case GG_MET_CHAR: draw(static_cast<int8_t*>(volume), dim, es, *shape); break;
    case GG_MET_UCHAR: draw(static_cast<uint8_t*>(volume), dim, es, *shape); break;
    case GG_MET_SHORT: draw(static_cast<int16_t*>(volume), dim, es, *shape); break;
    case GG_MET_USHORT: draw(static_cast<uint16_t*>(volume), dim, es, *shape); break;
    case GG_MET_INT: draw(static_cast<int32_t*>(volume), dim, es, *shape); break;
    case GG_MET_UINT: draw(static_cast<uint32_t*>(volume), dim, es, *shape); break;
    case GG_MET_FLOAT: draw(static_cast<float*>(volume), dim, es, *shape); break;
    default: return GG_ERROR_INVALID_ARGUMENT;
  }
  return GG_OK;
}

__attribute__((visibility("default"))) int gg_oracle_labels(const void* image, int32_t met_type, uint64_t n,
                                                            const float* first, const float* last, int32_t ranges,
                                                            uint8_t* out, int64_t* unconverted) {
  int64_t m = 0;
  switch (met_type) {
    case GG_MET_CHAR: m = labels(static_cast<const int8_t*>(image), n, first, last, ranges, out); break;
    case GG_MET_UCHAR: m = labels(static_cast<const uint8_t*>(image), n, first, last, ranges, out); break;
    case GG_MET_SHORT: m = labels(static_cast<const int16_t*>(image), n, first, last, ranges, out); break;
    case GG_MET_USHORT: m = labels(static_cast<const uint16_t*>(image), n, first, last, ranges, out); break;
    case GG_MET_INT: m = labels(static_cast<const int32_t*>(image), n, first, last, ranges, out); break;
    case GG_MET_UINT: m = labels(static_cast<const uint32_t*>(image), n, first, last, ranges, out); break;
    case GG_MET_FLOAT: m = labels(static_cast<const float*>(image), n, first, last, ranges, out); break;
    default: return GG_ERROR_INVALID_ARGUMENT;
  }
  if (unconverted) *unconverted = m;
  return GG_OK;
}

}  // extern "C"
