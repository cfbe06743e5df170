// ggems.hh - GGEMS's C++ classes for the photon path, over libggems.so.
//
// A GGEMS C++ program (GGEMS v1.3, include/GGEMS/**) uses these classes with the
// same names, methods, argument order, units and defaults: GGEMS,
// GGEMSOpenCLManager, GGEMSMaterialsDatabaseManager, GGEMSProcessesManager,
// GGEMSRangeCutsManager, GGEMSSourceManager, GGEMSXRaySource,
// GGEMSVoxelizedSource, GGEMSVoxelizedPhantom, GGEMSMeshedPhantom,
// GGEMSCTSystem, GGEMSDosimetryCalculator, GGEMSWorld, GGEMSVolumeCreatorManager,
// GGEMSBox, GGEMSTube and GGEMSSphere.  Each object is a handle to the
// library's own, which the simulation owns (in GGEMS sources and navigators
// register themselves with their managers); GGEMS and
// GGEMSDosimetryCalculator are deleted with their handle.  Where GGEMS throws,
// the methods throw std::runtime_error with GGEMS's message.  Header only; link
// with libggems.so.  Do not include with ggems_api.h (the C declarations of the
// same functions, with the GGEMS names as opaque C types).
#ifndef GGEMS_CPP_HH
#define GGEMS_CPP_HH

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>

namespace ggems_c {
extern "C" {
const char* ggems_last_error(void);
void ggems_clear_error(void);
void set_ggems_verbose(int);
void* create_ggems(void);
void delete_ggems(void*);
void initialize_ggems(void*, uint32_t);
void run_ggems(void*);
void set_opencl_verbose_ggems(void*, bool);
void set_material_database_verbose_ggems(void*, bool);
void set_source_ggems(void*, bool);
void set_navigator_ggems(void*, bool);
void set_memory_ram_ggems(void*, bool);
void set_process_ggems(void*, bool);
void set_range_cuts_ggems(void*, bool);
void set_random_ggems(void*, bool);
void set_profiling_ggems(void*, bool);
void set_tracking_ggems(void*, bool, int);
void* get_instance_ggems_opencl_manager(void);
void print_infos_opencl_manager(void*);
void set_device_index_ggems_opencl_manager(void*, uint64_t);
void set_device_to_activate_opencl_manager(void*, const char*, const char*);
void set_device_balancing_opencl_manager(void*, const char*);
void clean_opencl_manager(void*);
void* get_instance_materials_manager(void);
void set_materials_ggems_materials_manager(void*, const char*);
void print_available_chemical_elements_ggems_materials_manager(void*);
void print_available_materials_ggems_materials_manager(void*);
void* get_instance_processes_manager(void);
void add_process_processes_manager(void*, const char*, const char*, const char*);
void set_cross_section_table_number_of_bins_processes_manager(void*, uint64_t);
void set_cross_section_table_minimum_energy_processes_manager(void*, float, const char*);
void set_cross_section_table_maximum_energy_processes_manager(void*, float, const char*);
void print_infos_processes_manager(void*);
void print_available_processes_manager(void*);
void print_tables_processes_manager(void*, bool);
void* get_instance_range_cuts_manager(void);
void set_cut_range_cuts_manager(void*, const char*, const char*, float, const char*);
void* get_instance_ggems_source_manager(void);
void print_infos_source_manager(void*);
void* create_ggems_xray_source(const char*);
void set_position_ggems_xray_source(void*, float, float, float, const char*);
void set_number_of_particles_xray_source(void*, uint64_t);
void set_source_particle_type_ggems_xray_source(void*, const char*);
void set_beam_aperture_ggems_xray_source(void*, float, const char*);
void set_focal_spot_size_ggems_xray_source(void*, float, float, float, const char*);
void set_rotation_ggems_xray_source(void*, float, float, float, const char*);
void set_monoenergy_ggems_xray_source(void*, float, const char*);
void set_polyenergy_ggems_xray_source(void*, const char*);
void* create_ggems_voxelized_source(const char*);
void set_position_ggems_voxelized_source(void*, float, float, float, const char*);
void set_rotation_ggems_voxelized_source(void*, float, float, float, const char*);
void set_number_of_particles_voxelized_source(void*, uint64_t);
void set_source_particle_type_ggems_voxelized_source(void*, const char*);
void set_monoenergy_ggems_voxelized_source(void*, float, const char*);
void set_polyenergy_ggems_voxelized_source(void*, const char*);
void set_phantom_source_ggems_voxelized_source(void*, const char*);
void* create_ggems_voxelized_phantom(const char*);
void set_phantom_file_ggems_voxelized_phantom(void*, const char*, const char*);
void set_position_ggems_voxelized_phantom(void*, float, float, float, const char*);
void set_rotation_ggems_voxelized_phantom(void*, float, float, float, const char*);
void* create_ggems_meshed_phantom(const char*);
void set_phantom_file_ggems_meshed_phantom(void*, const char*);
void set_position_ggems_meshed_phantom(void*, float, float, float, const char*);
void set_rotation_ggems_meshed_phantom(void*, float, float, float, const char*);
void set_material_name_ggems_meshed_phantom(void*, const char*);
void set_mesh_octree_depth_ggems_meshed_phantom(void*, int);
void* create_ggems_ct_system(const char*);
void set_number_of_modules_ggems_ct_system(void*, uint64_t, uint64_t);
void set_ct_system_type_ggems_ct_system(void*, const char*);
void set_number_of_detection_elements_ggems_ct_system(void*, uint64_t, uint64_t, uint64_t);
void set_size_of_detection_elements_ggems_ct_system(void*, float, float, float, const char*);
void set_material_name_ggems_ct_system(void*, const char*);
void set_source_isocenter_distance_ggems_ct_system(void*, float, const char*);
void set_source_detector_distance_ggems_ct_system(void*, float, const char*);
void set_rotation_ggems_ct_system(void*, float, float, float, const char*);
void set_save_ggems_ct_system(void*, const char*);
void set_threshold_ggems_ct_system(void*, float, const char*);
void store_scatter_ggems_ct_system(void*, bool);
void set_global_system_position_ggems_ct_system(void*, float, float, float, const char*);
void* create_ggems_dosimetry_calculator(void);
void delete_dosimetry_calculator(void*);
void scale_factor_dosimetry_calculator(void*, float);
void water_reference_dosimetry_calculator(void*, bool);
void minimum_density_dosimetry_calculator(void*, float, const char*);
void set_dosel_size_dosimetry_calculator(void*, float, float, float, const char*);
void set_dose_output_dosimetry_calculator(void*, const char*);
void dose_photon_tracking_dosimetry_calculator(void*, bool);
void dose_edep_dosimetry_calculator(void*, bool);
void dose_hit_dosimetry_calculator(void*, bool);
void dose_edep_squared_dosimetry_calculator(void*, bool);
void dose_uncertainty_dosimetry_calculator(void*, bool);
void dose_tle_navigator(void*, bool);
void attach_to_navigator_dosimetry_calculator(void*, const char*);
void* create_ggems_world(void);
void set_dimension_ggems_world(void*, size_t, size_t, size_t);
void set_size_ggems_world(void*, float, float, float, const char*);
void photon_tracking_ggems_world(void*, bool);
void energy_tracking_ggems_world(void*, bool);
void energy_squared_tracking_ggems_world(void*, bool);
void set_output_ggems_world(void*, const char*);
void momentum_ggems_world(void*, bool);
void* get_instance_volume_creator_manager(void);
void set_volume_dimension_volume_creator_manager(void*, size_t, size_t, size_t);
void set_element_sizes_volume_creator_manager(void*, float, float, float, const char*);
void set_output_image_filename_volume_creator_manager(void*, const char*);
void set_output_range_to_material_filename_volume_creator_manager(void*, const char*);
void initialize_volume_creator_manager(void*);
void write_volume_creator_manager(void*);
void set_material_volume_creator_manager(void*, const char*);
void set_data_type_volume_creator_manager(void*, const char*);
void clean_volume_creator_manager(void*);
void* create_box(float, float, float, const char*);
void delete_box(void*);
void set_position_box(void*, float, float, float, const char*);
void set_material_box(void*, const char*);
void set_label_value_box(void*, float);
void initialize_box(void*);
void draw_box(void*);
void* create_tube(float, float, float, const char*);
void delete_tube(void*);
void set_position_tube(void*, float, float, float, const char*);
void set_material_tube(void*, const char*);
void set_label_value_tube(void*, float);
void initialize_tube(void*);
void draw_tube(void*);
void* create_sphere(float, const char*);
void delete_sphere(void*);
void set_position_sphere(void*, float, float, float, const char*);
void set_material_sphere(void*, const char*);
void set_label_value_sphere(void*, float);
void initialize_sphere(void*);
void draw_sphere(void*);
}

// Throws the message the last call recorded (GGEMS's exception text), if any.
inline void check() {
  const char* e = ggems_last_error();
  if (e && *e) {
    std::string m(e);
    ggems_clear_error();
    throw std::runtime_error(m);
  }
}
template <class F>
inline auto call(F f) -> decltype(f()) {
  ggems_clear_error();
  if constexpr (std::is_void<decltype(f())>::value) {
    f();
    check();
  } else {
    auto r = f();
    check();
    return r;
  }
}

// A handle to an object the library owns.
class Handle {
 public:
  Handle(const Handle&) = delete;
  Handle& operator=(const Handle&) = delete;

 protected:
  explicit Handle(void* h) : h_(h) {}
  void* h_;
};
}  // namespace ggems_c

// ---- GGEMSPrint.hh ----
inline void GGEMSVerbosity(int verbosity) { ggems_c::set_ggems_verbose(verbosity); }

// ---- GGEMS.hh ----
class GGEMS : ggems_c::Handle {
 public:
  GGEMS() : Handle(ggems_c::create_ggems()) {}
  ~GGEMS() { ggems_c::delete_ggems(h_); }
  void Initialize(uint32_t seed = 0) { ggems_c::call([&] { ggems_c::initialize_ggems(h_, seed); }); }
  void Run() { ggems_c::call([&] { ggems_c::run_ggems(h_); }); }
  void SetOpenCLVerbose(bool v) { ggems_c::set_opencl_verbose_ggems(h_, v); }
  void SetMaterialDatabaseVerbose(bool v) { ggems_c::set_material_database_verbose_ggems(h_, v); }
  void SetSourceVerbose(bool v) { ggems_c::set_source_ggems(h_, v); }
  void SetNavigatorVerbose(bool v) { ggems_c::set_navigator_ggems(h_, v); }
  void SetMemoryRAMVerbose(bool v) { ggems_c::set_memory_ram_ggems(h_, v); }
  void SetProcessVerbose(bool v) { ggems_c::set_process_ggems(h_, v); }
  void SetRangeCutsVerbose(bool v) { ggems_c::set_range_cuts_ggems(h_, v); }
  void SetRandomVerbose(bool v) { ggems_c::set_random_ggems(h_, v); }
  void SetProfilingVerbose(bool v) { ggems_c::set_profiling_ggems(h_, v); }
  void SetTrackingVerbose(bool v, int particle_id) { ggems_c::set_tracking_ggems(h_, v, particle_id); }
};

// ---- singletons ----
class GGEMSOpenCLManager : ggems_c::Handle {
 public:
  static GGEMSOpenCLManager& GetInstance() {
    static GGEMSOpenCLManager m;
    return m;
  }
  void PrintInfos() const { ggems_c::print_infos_opencl_manager(h_); }
  void DeviceToActivate(std::size_t device_id) {
    ggems_c::call([&] { ggems_c::set_device_index_ggems_opencl_manager(h_, device_id); });
  }
  void DeviceToActivate(std::string const& device_type, std::string const& device_vendor = "") {
    ggems_c::call([&] { ggems_c::set_device_to_activate_opencl_manager(h_, device_type.c_str(), device_vendor.c_str()); });
  }
  void DeviceBalancing(std::string const& balancing) {
    ggems_c::call([&] { ggems_c::set_device_balancing_opencl_manager(h_, balancing.c_str()); });
  }
  void Clean() { ggems_c::clean_opencl_manager(h_); }

 private:
  GGEMSOpenCLManager() : Handle(ggems_c::get_instance_ggems_opencl_manager()) {}
};

class GGEMSMaterialsDatabaseManager : ggems_c::Handle {
 public:
  static GGEMSMaterialsDatabaseManager& GetInstance() {
    static GGEMSMaterialsDatabaseManager m;
    return m;
  }
  void SetMaterialsDatabase(std::string const& filename) {
    ggems_c::call([&] { ggems_c::set_materials_ggems_materials_manager(h_, filename.c_str()); });
  }
  void PrintAvailableChemicalElements() const { ggems_c::print_available_chemical_elements_ggems_materials_manager(h_); }
  void PrintAvailableMaterials() const { ggems_c::print_available_materials_ggems_materials_manager(h_); }

 private:
  GGEMSMaterialsDatabaseManager() : Handle(ggems_c::get_instance_materials_manager()) {}
};

class GGEMSProcessesManager : ggems_c::Handle {
 public:
  static GGEMSProcessesManager& GetInstance() {
    static GGEMSProcessesManager m;
    return m;
  }
  void AddProcess(std::string const& process, std::string const& particle, std::string const& phantom) {
    ggems_c::call([&] { ggems_c::add_process_processes_manager(h_, process.c_str(), particle.c_str(), phantom.c_str()); });
  }
  void SetCrossSectionTableNumberOfBins(std::size_t bins) {
    ggems_c::call([&] { ggems_c::set_cross_section_table_number_of_bins_processes_manager(h_, bins); });
  }
  void SetCrossSectionTableMinimumEnergy(float energy, char const* unit = "keV") {
    ggems_c::call([&] { ggems_c::set_cross_section_table_minimum_energy_processes_manager(h_, energy, unit); });
  }
  void SetCrossSectionTableMaximumEnergy(float energy, char const* unit = "keV") {
    ggems_c::call([&] { ggems_c::set_cross_section_table_maximum_energy_processes_manager(h_, energy, unit); });
  }
  void PrintInfos() const { ggems_c::print_infos_processes_manager(h_); }
  void PrintAvailableProcesses() const { ggems_c::print_available_processes_manager(h_); }
  void PrintPhysicTables(bool print) { ggems_c::print_tables_processes_manager(h_, print); }

 private:
  GGEMSProcessesManager() : Handle(ggems_c::get_instance_processes_manager()) {}
};

class GGEMSRangeCutsManager : ggems_c::Handle {
 public:
  static GGEMSRangeCutsManager& GetInstance() {
    static GGEMSRangeCutsManager m;
    return m;
  }
  void SetLengthCut(std::string const& phantom, std::string const& particle, float value, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_cut_range_cuts_manager(h_, phantom.c_str(), particle.c_str(), value, unit.c_str()); });
  }

 private:
  GGEMSRangeCutsManager() : Handle(ggems_c::get_instance_range_cuts_manager()) {}
};

class GGEMSSourceManager : ggems_c::Handle {
 public:
  static GGEMSSourceManager& GetInstance() {
    static GGEMSSourceManager m;
    return m;
  }
  void PrintInfos() const { ggems_c::print_infos_source_manager(h_); }

 private:
  GGEMSSourceManager() : Handle(ggems_c::get_instance_ggems_source_manager()) {}
};

// ---- sources ----
class GGEMSXRaySource : ggems_c::Handle {
 public:
  explicit GGEMSXRaySource(std::string const& name)
      : Handle(ggems_c::call([&] { return ggems_c::create_ggems_xray_source(name.c_str()); })) {}
  void SetSourceParticleType(std::string const& type) {
    ggems_c::call([&] { ggems_c::set_source_particle_type_ggems_xray_source(h_, type.c_str()); });
  }
  void SetNumberOfParticles(std::size_t n) { ggems_c::call([&] { ggems_c::set_number_of_particles_xray_source(h_, n); }); }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_ggems_xray_source(h_, x, y, z, unit.c_str()); });
  }
  void SetRotation(float rx, float ry, float rz, std::string const& unit = "deg") {
    ggems_c::call([&] { ggems_c::set_rotation_ggems_xray_source(h_, rx, ry, rz, unit.c_str()); });
  }
  void SetBeamAperture(float aperture, std::string const& unit = "deg") {
    ggems_c::call([&] { ggems_c::set_beam_aperture_ggems_xray_source(h_, aperture, unit.c_str()); });
  }
  void SetFocalSpotSize(float w, float h, float d, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_focal_spot_size_ggems_xray_source(h_, w, h, d, unit.c_str()); });
  }
  void SetMonoenergy(float energy, std::string const& unit = "keV") {
    ggems_c::call([&] { ggems_c::set_monoenergy_ggems_xray_source(h_, energy, unit.c_str()); });
  }
  void SetPolyenergy(std::string const& file) {
    ggems_c::call([&] { ggems_c::set_polyenergy_ggems_xray_source(h_, file.c_str()); });
  }
};

class GGEMSVoxelizedSource : ggems_c::Handle {
 public:
  explicit GGEMSVoxelizedSource(std::string const& name)
      : Handle(ggems_c::call([&] { return ggems_c::create_ggems_voxelized_source(name.c_str()); })) {}
  void SetSourceParticleType(std::string const& type) {
    ggems_c::call([&] { ggems_c::set_source_particle_type_ggems_voxelized_source(h_, type.c_str()); });
  }
  void SetNumberOfParticles(std::size_t n) {
    ggems_c::call([&] { ggems_c::set_number_of_particles_voxelized_source(h_, n); });
  }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_ggems_voxelized_source(h_, x, y, z, unit.c_str()); });
  }
  void SetRotation(float rx, float ry, float rz, std::string const& unit = "deg") {
    ggems_c::call([&] { ggems_c::set_rotation_ggems_voxelized_source(h_, rx, ry, rz, unit.c_str()); });
  }
  void SetPhantomSourceFile(std::string const& file) {
    ggems_c::call([&] { ggems_c::set_phantom_source_ggems_voxelized_source(h_, file.c_str()); });
  }
  void SetMonoenergy(float energy, std::string const& unit = "keV") {
    ggems_c::call([&] { ggems_c::set_monoenergy_ggems_voxelized_source(h_, energy, unit.c_str()); });
  }
  void SetPolyenergy(std::string const& file) {
    ggems_c::call([&] { ggems_c::set_polyenergy_ggems_voxelized_source(h_, file.c_str()); });
  }
};

// ---- navigators ----
class GGEMSVoxelizedPhantom : ggems_c::Handle {
 public:
  explicit GGEMSVoxelizedPhantom(std::string const& name)
      : Handle(ggems_c::call([&] { return ggems_c::create_ggems_voxelized_phantom(name.c_str()); })) {}
  void SetPhantomFile(std::string const& phantom, std::string const& range) {
    ggems_c::call([&] { ggems_c::set_phantom_file_ggems_voxelized_phantom(h_, phantom.c_str(), range.c_str()); });
  }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_ggems_voxelized_phantom(h_, x, y, z, unit.c_str()); });
  }
  void SetRotation(float rx, float ry, float rz, std::string const& unit = "deg") {
    ggems_c::call([&] { ggems_c::set_rotation_ggems_voxelized_phantom(h_, rx, ry, rz, unit.c_str()); });
  }
};

class GGEMSMeshedPhantom : ggems_c::Handle {
 public:
  explicit GGEMSMeshedPhantom(std::string const& name)
      : Handle(ggems_c::call([&] { return ggems_c::create_ggems_meshed_phantom(name.c_str()); })) {}
  void SetPhantomFile(std::string const& stl) {
    ggems_c::call([&] { ggems_c::set_phantom_file_ggems_meshed_phantom(h_, stl.c_str()); });
  }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_ggems_meshed_phantom(h_, x, y, z, unit.c_str()); });
  }
  void SetRotation(float rx, float ry, float rz, std::string const& unit = "deg") {
    ggems_c::call([&] { ggems_c::set_rotation_ggems_meshed_phantom(h_, rx, ry, rz, unit.c_str()); });
  }
  void SetMaterialName(std::string const& material) {
    ggems_c::call([&] { ggems_c::set_material_name_ggems_meshed_phantom(h_, material.c_str()); });
  }
  void SetMeshOctreeDepth(int depth) { ggems_c::set_mesh_octree_depth_ggems_meshed_phantom(h_, depth); }
};

class GGEMSCTSystem : ggems_c::Handle {
 public:
  explicit GGEMSCTSystem(std::string const& name)
      : Handle(ggems_c::call([&] { return ggems_c::create_ggems_ct_system(name.c_str()); })) {}
  void SetCTSystemType(std::string const& type) {
    ggems_c::call([&] { ggems_c::set_ct_system_type_ggems_ct_system(h_, type.c_str()); });
  }
  void SetNumberOfModules(std::size_t x, std::size_t y) {
    ggems_c::call([&] { ggems_c::set_number_of_modules_ggems_ct_system(h_, x, y); });
  }
  void SetNumberOfDetectionElementsInsideModule(std::size_t x, std::size_t y, std::size_t z) {
    ggems_c::call([&] { ggems_c::set_number_of_detection_elements_ggems_ct_system(h_, x, y, z); });
  }
  void SetSizeOfDetectionElements(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_size_of_detection_elements_ggems_ct_system(h_, x, y, z, unit.c_str()); });
  }
  void SetMaterialName(std::string const& material) {
    ggems_c::call([&] { ggems_c::set_material_name_ggems_ct_system(h_, material.c_str()); });
  }
  void SetSourceIsocenterDistance(float d, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_source_isocenter_distance_ggems_ct_system(h_, d, unit.c_str()); });
  }
  void SetSourceDetectorDistance(float d, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_source_detector_distance_ggems_ct_system(h_, d, unit.c_str()); });
  }
  void SetRotation(float rx, float ry, float rz, std::string const& unit = "deg") {
    ggems_c::call([&] { ggems_c::set_rotation_ggems_ct_system(h_, rx, ry, rz, unit.c_str()); });
  }
  void SetGlobalSystemPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_global_system_position_ggems_ct_system(h_, x, y, z, unit.c_str()); });
  }
  void SetThreshold(float threshold, std::string const& unit = "keV") {
    ggems_c::call([&] { ggems_c::set_threshold_ggems_ct_system(h_, threshold, unit.c_str()); });
  }
  void StoreOutput(std::string const& basename) {
    ggems_c::call([&] { ggems_c::set_save_ggems_ct_system(h_, basename.c_str()); });
  }
  void StoreScatter(bool scatter) { ggems_c::call([&] { ggems_c::store_scatter_ggems_ct_system(h_, scatter); }); }
};

class GGEMSDosimetryCalculator : ggems_c::Handle {
 public:
  GGEMSDosimetryCalculator() : Handle(ggems_c::call([] { return ggems_c::create_ggems_dosimetry_calculator(); })) {}
  ~GGEMSDosimetryCalculator() { ggems_c::delete_dosimetry_calculator(h_); }
  void AttachToNavigator(std::string const& navigator) {
    ggems_c::call([&] { ggems_c::attach_to_navigator_dosimetry_calculator(h_, navigator.c_str()); });
  }
  void SetDoselSizes(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_dosel_size_dosimetry_calculator(h_, x, y, z, unit.c_str()); });
  }
  void SetOutputDosimetryBasename(std::string const& basename) {
    ggems_c::call([&] { ggems_c::set_dose_output_dosimetry_calculator(h_, basename.c_str()); });
  }
  void SetScaleFactor(float s) { ggems_c::scale_factor_dosimetry_calculator(h_, s); }
  void SetPhotonTracking(bool v) { ggems_c::dose_photon_tracking_dosimetry_calculator(h_, v); }
  void SetEdep(bool v) { ggems_c::dose_edep_dosimetry_calculator(h_, v); }
  void SetHitTracking(bool v) { ggems_c::dose_hit_dosimetry_calculator(h_, v); }
  void SetEdepSquared(bool v) { ggems_c::dose_edep_squared_dosimetry_calculator(h_, v); }
  void SetUncertainty(bool v) { ggems_c::dose_uncertainty_dosimetry_calculator(h_, v); }
  void SetWaterReference(bool v) { ggems_c::water_reference_dosimetry_calculator(h_, v); }
  void SetMinimumDensity(float density, std::string const& unit = "g/cm3") {
    ggems_c::call([&] { ggems_c::minimum_density_dosimetry_calculator(h_, density, unit.c_str()); });
  }
  void SetTLE(bool v) { ggems_c::call([&] { ggems_c::dose_tle_navigator(h_, v); }); }
};

class GGEMSWorld : ggems_c::Handle {
 public:
  GGEMSWorld() : Handle(ggems_c::call([] { return ggems_c::create_ggems_world(); })) {}
  void SetOutputWorldBasename(std::string const& basename) { ggems_c::set_output_ggems_world(h_, basename.c_str()); }
  void SetDimension(std::size_t x, std::size_t y, std::size_t z) { ggems_c::set_dimension_ggems_world(h_, x, y, z); }
  void SetElementSize(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_size_ggems_world(h_, x, y, z, unit.c_str()); });
  }
  void SetPhotonTracking(bool v) { ggems_c::photon_tracking_ggems_world(h_, v); }
  void SetEnergyTracking(bool v) { ggems_c::energy_tracking_ggems_world(h_, v); }
  void SetEnergySquaredTracking(bool v) { ggems_c::energy_squared_tracking_ggems_world(h_, v); }
  void SetMomentum(bool v) { ggems_c::momentum_ggems_world(h_, v); }
};

// ---- volume creator ----
class GGEMSVolumeCreatorManager : ggems_c::Handle {
 public:
  static GGEMSVolumeCreatorManager& GetInstance() {
    static GGEMSVolumeCreatorManager m;
    return m;
  }
  void SetVolumeDimensions(std::size_t w, std::size_t h, std::size_t d) {
    ggems_c::set_volume_dimension_volume_creator_manager(h_, w, h, d);
  }
  void SetElementSizes(float w, float h, float d, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_element_sizes_volume_creator_manager(h_, w, h, d, unit.c_str()); });
  }
  void SetOutputImageFilename(std::string const& f) {
    ggems_c::set_output_image_filename_volume_creator_manager(h_, f.c_str());
  }
  void SetRangeToMaterialDataFilename(std::string const& f) {
    ggems_c::set_output_range_to_material_filename_volume_creator_manager(h_, f.c_str());
  }
  void SetMaterial(std::string const& material) { ggems_c::set_material_volume_creator_manager(h_, material.c_str()); }
  void SetDataType(std::string const& type) {
    ggems_c::call([&] { ggems_c::set_data_type_volume_creator_manager(h_, type.c_str()); });
  }
  void Initialize() { ggems_c::call([&] { ggems_c::initialize_volume_creator_manager(h_); }); }
  void Write() { ggems_c::call([&] { ggems_c::write_volume_creator_manager(h_); }); }
  void Clean() { ggems_c::clean_volume_creator_manager(h_); }

 private:
  GGEMSVolumeCreatorManager() : Handle(ggems_c::get_instance_volume_creator_manager()) {}
};

class GGEMSBox : ggems_c::Handle {
 public:
  GGEMSBox(float width, float height, float depth, std::string const& unit = "mm")
      : Handle(ggems_c::call([&] { return ggems_c::create_box(width, height, depth, unit.c_str()); })) {}
  ~GGEMSBox() { ggems_c::delete_box(h_); }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_box(h_, x, y, z, unit.c_str()); });
  }
  void SetLabelValue(float v) { ggems_c::set_label_value_box(h_, v); }
  void SetMaterial(std::string const& m) { ggems_c::call([&] { ggems_c::set_material_box(h_, m.c_str()); }); }
  void Initialize() { ggems_c::initialize_box(h_); }
  void Draw() { ggems_c::call([&] { ggems_c::draw_box(h_); }); }
};

class GGEMSTube : ggems_c::Handle {
 public:
  GGEMSTube(float radius_x, float radius_y, float height, std::string const& unit = "mm")
      : Handle(ggems_c::call([&] { return ggems_c::create_tube(radius_x, radius_y, height, unit.c_str()); })) {}
  ~GGEMSTube() { ggems_c::delete_tube(h_); }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_tube(h_, x, y, z, unit.c_str()); });
  }
  void SetLabelValue(float v) { ggems_c::set_label_value_tube(h_, v); }
  void SetMaterial(std::string const& m) { ggems_c::call([&] { ggems_c::set_material_tube(h_, m.c_str()); }); }
  void Initialize() { ggems_c::initialize_tube(h_); }
  void Draw() { ggems_c::call([&] { ggems_c::draw_tube(h_); }); }
};

class GGEMSSphere : ggems_c::Handle {
 public:
  GGEMSSphere(float radius, std::string const& unit = "mm")
      : Handle(ggems_c::call([&] { return ggems_c::create_sphere(radius, unit.c_str()); })) {}
  ~GGEMSSphere() { ggems_c::delete_sphere(h_); }
  void SetPosition(float x, float y, float z, std::string const& unit = "mm") {
    ggems_c::call([&] { ggems_c::set_position_sphere(h_, x, y, z, unit.c_str()); });
  }
  void SetLabelValue(float v) { ggems_c::set_label_value_sphere(h_, v); }
  void SetMaterial(std::string const& m) { ggems_c::call([&] { ggems_c::set_material_sphere(h_, m.c_str()); }); }
  void Initialize() { ggems_c::initialize_sphere(h_); }
  void Draw() { ggems_c::call([&] { ggems_c::draw_sphere(h_); }); }
};

#endif
