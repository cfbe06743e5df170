// Volume creator of the GGEMS-compatible API: GGEMSVolumeCreatorManager and
// the analytic shapes GGEMSBox / GGEMSTube / GGEMSSphere
// (src/geometries/GGEMSVolumeCreatorManager.cc, GGEMSVolume.cc, GGEMSBox.cc,
// GGEMSTube.cc, GGEMSSphere.cc), with their extern "C" functions.  The image
// lives on the first activated device (gg_volume_*, include/ggems_b200.h),
// shapes are drawn there, and write() brings it back for the MHD file and
// writes the label -> material range file.
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "gg_api.hh"
#include "ggems_b200.h"

using namespace gg;

#define GG_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

int met_type_of(const std::string& t) {
  if (t == "MET_CHAR") return GG_MET_CHAR;
  if (t == "MET_UCHAR") return GG_MET_UCHAR;
  if (t == "MET_SHORT") return GG_MET_SHORT;
  if (t == "MET_USHORT") return GG_MET_USHORT;
  if (t == "MET_INT") return GG_MET_INT;
  if (t == "MET_UINT") return GG_MET_UINT;
  if (t == "MET_FLOAT") return GG_MET_FLOAT;
  return -1;
}
size_t met_size(int t) { return t <= GG_MET_UCHAR ? 1 : (t <= GG_MET_USHORT ? 2 : 4); }

class VolumeCreatorManager {
 public:
  static VolumeCreatorManager& instance() {
    static VolumeCreatorManager m;
    return m;
  }
  float element_sizes[3] = {0.0f, 0.0f, 0.0f};
  uint64_t dimensions[3] = {0, 0, 0};
  std::string data_type = "MET_FLOAT";
  std::string output_image, output_range;
  std::map<float, std::string> label_to_material;
  gg_volume* volume = nullptr;

  void set_data_type(const std::string& t) {
    data_type = t;
    if (met_type_of(t) < 0)
      throw Error("GGEMSVolumeCreatorManager", "SetDataType",
                  "Your type in not compatible. The type has to be:\n    - MET_CHAR\n    - MET_UCHAR\n    - MET_SHORT\n"
                  "    - MET_USHORT\n    - MET_INT\n    - MET_UINT\n    - MET_FLOAT\n");
  }
  void add_label_and_material(float label, const std::string& material) {
    auto r = label_to_material.insert(std::make_pair(label, material));
    if (!r.second) {
      std::ostringstream oss;
      oss << "The label: " << r.first->first << " already exists...";
      throw Error("GGEMSVolumeCreatorManager", "AddLabelAndMaterial", oss.str());
    }
  }
  // GGEMSVolumeCreatorManager::CheckParameters (GGEMSVolumeCreatorManager.cc:200-223)
  void check() const {
    if (dimensions[0] == 0 && dimensions[1] == 0 && dimensions[2] == 0)
      throw Error("GGEMSVolumeCreatorManager", "CheckParameters", "Phantom dimensions have to be > 0!!!");
    if (element_sizes[0] == 0.0f && element_sizes[1] == 0.0f && element_sizes[2] == 0.0f)
      throw Error("GGEMSVolumeCreatorManager", "CheckParameters", "Phantom voxel sizes have to be > 0.0!!!");
    if (output_image.empty())
      throw Error("GGEMSVolumeCreatorManager", "CheckParameters",
                  "A output image filename has to be done to phantom manager!!!");
  }
  int32_t dim(int a) const { return static_cast<int32_t>(dimensions[a]); }
  // GGEMSVolumeCreatorManager::Initialize: a zero-filled image of data_type.
  void initialize() {
    check();
    release();
    for (int a = 0; a < 3; ++a)
      if (dimensions[a] > 0x7fffffffull) throw Error("GGEMSVolumeCreatorManager", "Initialize", "dimension too large");
    const int32_t d[3] = {dim(0), dim(1), dim(2)};
    const auto& devs = Simulation::instance().device_indices;
    const int device = devs.empty() ? 0 : devs[0];
    if (gg_volume_create(device, met_type_of(data_type), d, element_sizes, &volume) != GG_OK)
      throw Error("GGEMSVolumeCreatorManager", "Initialize", gg_last_error());
  }
  // GGEMSVolumeCreatorManager::Write (GGEMSVolumeCreatorManager.cc:249-294)
  void write() const {
    if (!volume) throw Error("GGEMSVolumeCreatorManager", "Write", "the volume is not initialized");
    const int t = met_type_of(data_type);
    const uint64_t n = dimensions[0] * dimensions[1] * dimensions[2];
    std::vector<char> host(n * met_size(t));
    if (gg_volume_download(volume, host.data(), host.size()) != GG_OK)
      throw Error("GGEMSVolumeCreatorManager", "Write", gg_last_error());
    const int32_t d[3] = {dim(0), dim(1), dim(2)};
    write_mhd(output_image, data_type, d, element_sizes, host.data(), met_size(t));
    std::ofstream range(output_range, std::ios::out);
    for (auto& kv : label_to_material) range << kv.first << " " << kv.first << " " << kv.second << std::endl;
  }
  void release() {
    if (volume) gg_volume_destroy(volume);
    volume = nullptr;
  }
  // GGEMSVolumeCreatorManager::Clean (GGEMSVolumeCreatorManager.cc:74-103)
  void clean() {
    release();
    for (int a = 0; a < 3; ++a) {
      element_sizes[a] = 0.0f;
      dimensions[a] = 0;
    }
    data_type = "MET_FLOAT";
    output_image.clear();
    output_range.clear();
    label_to_material.clear();
  }
};

// GGEMSVolume (src/geometries/GGEMSVolume.cc): label 1, centred.
class Volume {
 public:
  explicit Volume(int type) { shape.type = type; }
  virtual ~Volume() = default;
  gg_shape shape{};
  float label_value = 1.0f;
  float position[3] = {0.0f, 0.0f, 0.0f};
  void set_material(const std::string& m) { VolumeCreatorManager::instance().add_label_and_material(label_value, m); }
  void set_position(float x, float y, float z, const std::string& unit) {
    position[0] = distance_unit(x, unit);
    position[1] = distance_unit(y, unit);
    position[2] = distance_unit(z, unit);
  }
  virtual const char* name() const = 0;
  // GGEMSBox::Draw etc.: one launch over the manager's image.
  void draw() {
    gg_volume* v = VolumeCreatorManager::instance().volume;
    if (!v) throw Error(name(), "Draw", "the volume creator manager is not initialized");
    shape.label_value = label_value;
    std::memcpy(shape.position, position, sizeof(position));
    if (gg_volume_draw(v, &shape, 1) != GG_OK) throw Error(name(), "Draw", gg_last_error());
  }
};

class Box : public Volume {
 public:
  Box(float w, float h, float d, const std::string& unit) : Volume(GG_SHAPE_BOX) {
    shape.size[0] = distance_unit(w, unit);
    shape.size[1] = distance_unit(h, unit);
    shape.size[2] = distance_unit(d, unit);
  }
  const char* name() const override { return "GGEMSBox"; }
};
class Tube : public Volume {
 public:
  Tube(float rx, float ry, float h, const std::string& unit) : Volume(GG_SHAPE_TUBE) {
    shape.size[0] = distance_unit(rx, unit);
    shape.size[1] = distance_unit(ry, unit);
    shape.size[2] = distance_unit(h, unit);
  }
  const char* name() const override { return "GGEMSTube"; }
};
class Sphere : public Volume {
 public:
  Sphere(float r, const std::string& unit) : Volume(GG_SHAPE_SPHERE) { shape.size[0] = distance_unit(r, unit); }
  const char* name() const override { return "GGEMSSphere"; }
};

template <class F>
void guarded(F f) {
  try {
    f();
  } catch (const std::exception& e) {
    set_last_error(e.what());
    std::cerr << e.what() << std::endl;
  }
}
template <class R, class F>
R guarded_value(R fallback, F f) {
  try {
    return f();
  } catch (const std::exception& e) {
    set_last_error(e.what());
    std::cerr << e.what() << std::endl;
    return fallback;
  }
}
std::string S(const char* s) { return s ? std::string(s) : std::string(); }

}  // namespace

// ---- GGEMSVolumeCreatorManager.hh ----
GG_EXPORT VolumeCreatorManager* get_instance_volume_creator_manager(void) { return &VolumeCreatorManager::instance(); }
GG_EXPORT void set_volume_dimension_volume_creator_manager(VolumeCreatorManager* m, size_t w, size_t h, size_t d) {
  m->dimensions[0] = w;
  m->dimensions[1] = h;
  m->dimensions[2] = d;
}
GG_EXPORT void set_element_sizes_volume_creator_manager(VolumeCreatorManager* m, float w, float h, float d, const char* unit) {
  guarded([&] {
    m->element_sizes[0] = distance_unit(w, S(unit));
    m->element_sizes[1] = distance_unit(h, S(unit));
    m->element_sizes[2] = distance_unit(d, S(unit));
  });
}
GG_EXPORT void set_output_image_filename_volume_creator_manager(VolumeCreatorManager* m, const char* f) { m->output_image = S(f); }
GG_EXPORT void set_output_range_to_material_filename_volume_creator_manager(VolumeCreatorManager* m, const char* f) {
  m->output_range = S(f);
}
GG_EXPORT void initialize_volume_creator_manager(VolumeCreatorManager* m) { guarded([&] { m->initialize(); }); }
GG_EXPORT void write_volume_creator_manager(VolumeCreatorManager* m) { guarded([&] { m->write(); }); }
// GGEMSVolumeCreatorManager::SetMaterial: the background (label 0).
GG_EXPORT void set_material_volume_creator_manager(VolumeCreatorManager* m, const char* material) {
  m->label_to_material.insert(std::make_pair(0.0f, S(material)));
}
GG_EXPORT void set_data_type_volume_creator_manager(VolumeCreatorManager* m, const char* t) { guarded([&] { m->set_data_type(S(t)); }); }
GG_EXPORT void clean_volume_creator_manager(VolumeCreatorManager* m) { m->clean(); }

// ---- GGEMSBox.hh / GGEMSTube.hh / GGEMSSphere.hh ----
GG_EXPORT Box* create_box(float w, float h, float d, const char* unit) {
  return guarded_value<Box*>(nullptr, [&] { return new Box(w, h, d, S(unit)); });
}
GG_EXPORT Tube* create_tube(float rx, float ry, float h, const char* unit) {
  return guarded_value<Tube*>(nullptr, [&] { return new Tube(rx, ry, h, S(unit)); });
}
GG_EXPORT Sphere* create_sphere(float r, const char* unit) {
  return guarded_value<Sphere*>(nullptr, [&] { return new Sphere(r, S(unit)); });
}
GG_EXPORT void delete_box(Box* v) { delete v; }
GG_EXPORT void delete_tube(Tube* v) { delete v; }
GG_EXPORT void delete_sphere(Sphere* v) { delete v; }
GG_EXPORT void set_position_box(Box* v, float x, float y, float z, const char* unit) { guarded([&] { v->set_position(x, y, z, S(unit)); }); }
GG_EXPORT void set_position_tube(Tube* v, float x, float y, float z, const char* unit) { guarded([&] { v->set_position(x, y, z, S(unit)); }); }
GG_EXPORT void set_position_sphere(Sphere* v, float x, float y, float z, const char* unit) { guarded([&] { v->set_position(x, y, z, S(unit)); }); }
GG_EXPORT void set_material_box(Box* v, const char* m) { guarded([&] { v->set_material(S(m)); }); }
GG_EXPORT void set_material_tube(Tube* v, const char* m) { guarded([&] { v->set_material(S(m)); }); }
GG_EXPORT void set_material_sphere(Sphere* v, const char* m) { guarded([&] { v->set_material(S(m)); }); }
GG_EXPORT void set_label_value_box(Box* v, float l) { v->label_value = l; }
GG_EXPORT void set_label_value_tube(Tube* v, float l) { v->label_value = l; }
GG_EXPORT void set_label_value_sphere(Sphere* v, float l) { v->label_value = l; }
// Initialize compiles the shape's kernel for the manager's type in GGEMS; the
// kernels here are built ahead of time for every type, so there is nothing to do.
GG_EXPORT void initialize_box(Box*) {}
GG_EXPORT void initialize_tube(Tube*) {}
GG_EXPORT void initialize_sphere(Sphere*) {}
GG_EXPORT void draw_box(Box* v) { guarded([&] { v->draw(); }); }
GG_EXPORT void draw_tube(Tube* v) { guarded([&] { v->draw(); }); }
GG_EXPORT void draw_sphere(Sphere* v) { guarded([&] { v->draw(); }); }
