// GGEMS-compatible host classes backed by the B200 transport layer.
//
// Mirrors the reference's public C++ classes for the photon path
// (include/GGEMS/global/GGEMS.hh, sources/, navigators/, physics/) closely
// enough that the reference's extern "C" surface and Python ctypes module map
// onto them one to one.  Devices are driven through include/ggems_b200.h.
#ifndef GG_API_HH
#define GG_API_HH

#include <array>
#include <cfloat>
#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "ggems_b200.h"
#include "gg_mesh.hh"
#include "gg_physics.hh"

namespace gg {

// GGEMSGeometryTransformation (src/maths/GGEMSGeometryTransformation.cc:143-336).
struct Transformation {
  std::array<float, 16> matrix;
  std::array<float, 3> position{FLT_MIN, FLT_MIN, FLT_MIN};
  std::array<float, 3> rotation{FLT_MIN, FLT_MIN, FLT_MIN};
  Transformation();
  void set_axis(const float axis[3][3]);
  void set_translation(float x, float y, float z);
  void set_rotation(float rx, float ry, float rz);
};

// ---------------------------------------------------------------- sources --
class Source {
 public:
  explicit Source(const std::string& name);
  virtual ~Source() = default;
  std::string name;
  uint64_t number_of_particles = 0;
  int particle_type = 99;
  Transformation transformation;
  std::vector<std::pair<double, double>> energy_mappings;  // (energy MeV, intensity)
  int is_interp = 1;
  std::vector<float> energy_spectrum, energy_cdf;          // FillEnergy output (n+1)
  void set_position(float x, float y, float z, const std::string& unit);
  void set_rotation(float rx, float ry, float rz, const std::string& unit);
  void set_particle_type(const std::string& type);
  void set_monoenergy(float e, const std::string& unit);
  void set_polyenergy(const std::string& file);
  void set_energy_peak(float e, float intensity, const std::string& unit);
  virtual void initialize();
  virtual gg_source descriptor() const = 0;
  virtual std::string kind() const = 0;

 protected:
  void check() const;
  void fill_energy();
};

class XRaySource : public Source {
 public:
  explicit XRaySource(const std::string& name);
  float beam_aperture = FLT_MIN;
  float focal_spot_size[3] = {FLT_MIN, FLT_MIN, FLT_MIN};
  void set_beam_aperture(float a, const std::string& unit);
  void set_focal_spot_size(float w, float h, float d, const std::string& unit);
  void initialize() override;
  gg_source descriptor() const override;
  std::string kind() const override { return "GGEMSXRaySource"; }
};

class VoxelizedSource : public Source {
 public:
  explicit VoxelizedSource(const std::string& name);
  std::string phantom_source_file;
  int32_t number_of_voxels[3] = {0, 0, 0};
  float voxel_sizes[3] = {0, 0, 0};
  float border_min[3] = {0, 0, 0};
  std::vector<int32_t> activity_index;
  std::vector<float> activity_cdf;
  void initialize() override;
  gg_source descriptor() const override;
  std::string kind() const override { return "GGEMSVoxelizedSource"; }
};

// ------------------------------------------------------------- navigators --
class DosimetryCalculator;

struct SolidSpec {
  gg_solid solid{};
  std::vector<uint8_t> labels;
  std::shared_ptr<MeshedSolid> mesh;  // meshed solids only
};

class Navigator {
 public:
  explicit Navigator(const std::string& name);
  virtual ~Navigator() = default;
  std::string name;
  bool is_update_pos = false, is_update_rot = false;
  float position[3] = {0, 0, 0}, rotation[3] = {0, 0, 0};
  float threshold = 0.0f;
  std::vector<std::string> materials;     // GGEMSMaterials::AddMaterial order
  std::vector<int32_t> processes;         // GGEMSCrossSections::AddProcess order
  float photon_distance_cut = 1.e-3f;     // PHOTON_DISTANCE_CUT
  std::string output_basename;
  DosimetryCalculator* dose_calculator = nullptr;
  bool is_tle = false;
  NavigatorTables tables;
  std::vector<SolidSpec> solids;
  void set_position(float x, float y, float z, const std::string& unit);
  void set_rotation(float rx, float ry, float rz, const std::string& unit);
  void set_threshold(float t, const std::string& unit);
  void add_process(const std::string& process, const std::string& particle);
  void set_distance_cut(const std::string& particle, float value, const std::string& unit);
  virtual void initialize(int first_solid_id) = 0;
  void build_tables();
  virtual std::string kind() const = 0;
};

// Label volume of GGEMSVoxelizedSolid::ConvertImageToLabel
// (include/GGEMS/geometries/GGEMSVoxelizedSolid.hh:162-257): reads the MHD
// image and the range file; voxel value v gets label k of the k-th range line
// when v == first == last or first <= v < last.  Fills the material list in
// range-file order when `materials` is given.
std::vector<uint8_t> voxelized_labels(const std::string& phantom_file, const std::string& range_file,
                                      std::vector<std::string>* materials, MHDHeader* header);

class VoxelizedPhantom : public Navigator {
 public:
  explicit VoxelizedPhantom(const std::string& name);
  std::string phantom_file, range_file;
  void initialize(int first_solid_id) override;
  std::string kind() const override { return "GGEMSVoxelizedPhantom"; }
};

// GGEMSMeshedPhantom (src/navigators/GGEMSMeshedPhantom.cc): one meshed
// solid of one material, triangles moved to world coordinates, octree.
class MeshedPhantom : public Navigator {
 public:
  explicit MeshedPhantom(const std::string& name);
  std::string phantom_file;
  int octree_depth = 1;  // GGEMSMeshedPhantom::mesh_octree_depth_ default
  void initialize(int first_solid_id) override;
  std::string kind() const override { return "GGEMSMeshedPhantom"; }
};

class CTSystem : public Navigator {
 public:
  explicit CTSystem(const std::string& name);
  std::string type;
  uint64_t modules[2] = {0, 0};
  uint64_t elements[3] = {0, 0, 0};
  float element_size[3] = {0, 0, 0};
  float sid = 0.0f, sdd = 0.0f;
  float global_position[3] = {0, 0, 0};
  bool is_scatter = false;
  void initialize(int first_solid_id) override;
  std::string kind() const override { return "GGEMSCTSystem"; }
};

class DosimetryCalculator {
 public:
  std::string output = "dosi";
  Navigator* navigator = nullptr;
  bool photon_tracking = false, edep = false, hit = false, edep_squared = false, uncertainty = false;
  float scale_factor = 1.0f;
  bool water_reference = false;
  float minimum_density = 0.0f;
  float dosel_sizes[3] = {-1.0f, -1.0f, -1.0f};
  gg_dose_map map{};
  void attach(const std::string& navigator_name);
  void set_dosel_size(float x, float y, float z, const std::string& unit);
  void initialize(const SolidSpec& solid);
};

// GGEMSWorld (include/GGEMS/navigators/GGEMSWorld.hh:55-215): a grid centred
// on the origin recording the photons' flights between solids.  Creating one
// registers it with the simulation (GGEMSNavigatorManager::StoreWorld).
class World {
 public:
  World();
  std::string output = "world";
  uint64_t dimensions[3] = {0, 0, 0};
  float sizes[3] = {-1.0f, -1.0f, -1.0f};
  bool photon_tracking = false, energy_tracking = false, energy_squared_tracking = false, momentum = false;
  void set_element_size(float x, float y, float z, const std::string& unit);
  void check() const;
};

// ------------------------------------------------------------------ GGEMS --
struct Device {
  gg_context* context = nullptr;
  int index = 0;
  double balance = 1.0;
};

// GGEMSProfilerManager (src/tools/GGEMSProfilerManager.cc:83-104): device time
// per label (CUDA events of the launches), summed over runs.
class Profiler {
 public:
  static Profiler& instance();
  void add(const std::string& label, double ms);
  void print_summary(std::ostream& out) const;
  void reset();

 private:
  std::vector<std::pair<std::string, double>> labels_;
  mutable std::mutex mutex_;
};

class Simulation {
 public:
  static Simulation& instance();
  std::vector<std::unique_ptr<Source>> sources;
  std::vector<std::unique_ptr<Navigator>> navigators;
  std::vector<DosimetryCalculator*> dosimetry;
  std::unique_ptr<World> world;
  std::vector<int> device_indices;        // activated devices (empty: device 0)
  std::vector<double> device_balance;     // per activated device
  int cs_number_of_bins = 220;            // CROSS_SECTION_TABLE_NUMBER_BINS
  float cs_min_energy = 990.0f * 1.e-6f;  // CROSS_SECTION_TABLE_ENERGY_MIN
  float cs_max_energy = 250.0f * 1.0f;    // CROSS_SECTION_TABLE_ENERGY_MAX
  Navigator* navigator(const std::string& name) const;
  void clean();
};

class GGEMS {
 public:
  GGEMS();
  ~GGEMS();
  bool verbose[10] = {false};
  bool is_tracking = false;
  int tracking_id = 0;
  static constexpr int kTrackingCapacity = 4096;  // recorded points per run and device
  void initialize(uint32_t seed);
  // Host half of initialize(): sources, navigators, tables and the scene, no device.
  void prepare();
  void run();
  // scene as handed to the transport layer (valid after prepare / initialize)
  const gg_scene* scene() const { return prepared_ ? &scene_ : nullptr; }
  const std::vector<uint32_t>& random_states(size_t device) const { return states_[device]; }
  std::vector<Device> devices;
  float last_run_ms = 0.0f;
  int64_t last_run_launches = 0;
  uint64_t last_run_particles = 0;

 private:
  void build_scene();
  void save_results();
  bool initialized_ = false;
  bool prepared_ = false;
  uint32_t seed_ = 0;
  std::vector<gg_physics_tables> tables_;
  std::vector<gg_solid> solids_;
  std::vector<gg_dose_map> dose_maps_;
  std::vector<int32_t> histogram_sizes_;
  std::vector<float> rayleigh_fit_;
  std::vector<std::pair<Navigator*, int>> solid_owner_;  // navigator, solid index inside it
  gg_scene scene_{};
  std::vector<std::vector<uint32_t>> states_;
  std::vector<std::vector<int32_t>> histograms_;
  std::vector<std::vector<double>> edep_, edep2_;
  std::vector<std::vector<int32_t>> hit_, ptrack_;
  gg_world world_{};
  std::vector<int32_t> world_photon_;
  std::vector<double> world_energy_, world_energy2_, world_momentum_[3];
};

}  // namespace gg

#endif
