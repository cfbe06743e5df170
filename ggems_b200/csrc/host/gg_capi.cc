// extern "C" surface of libggems.so, with the names and argument meaning of
// GGEMS v1.3's C ABI (the bottom of each include/GGEMS/**/*.hh header) for
// the photon path.  The reference lets its C++ exceptions escape through
// these functions (which aborts a ctypes caller); here every wrapper catches,
// prints the same "[GGEMS Class::Method] EXCEPTION!!! ..." text on stderr and
// records it, so ggems_last_error() returns it and the Python module raises.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <memory>
#include <sstream>

#include "gg_api.hh"

using namespace gg;

#define GG_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

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

struct Singleton {
  int dummy;
};
Singleton g_opencl_manager, g_source_manager, g_processes_manager, g_range_cuts_manager, g_materials_manager,
    g_profiler_manager, g_ram_manager;

}  // namespace

// ---- error reporting (no counterpart in the reference, which aborts) ----
GG_EXPORT const char* ggems_last_error(void) { return last_error(); }
GG_EXPORT void ggems_clear_error(void) { clear_last_error(); }

// ---- GGEMSPrint.hh ----
GG_EXPORT void set_ggems_verbose(int verbosity) { set_verbosity(verbosity); }

// ---- GGEMS.hh ----
GG_EXPORT GGEMS* create_ggems(void) { return new (std::nothrow) GGEMS(); }
GG_EXPORT void delete_ggems(GGEMS* g) { delete g; }
GG_EXPORT void initialize_ggems(GGEMS* g, uint32_t seed) { guarded([&] { g->initialize(seed); }); }
GG_EXPORT void run_ggems(GGEMS* g) { guarded([&] { g->run(); }); }
GG_EXPORT void set_opencl_verbose_ggems(GGEMS* g, bool v) { g->verbose[0] = v; }
GG_EXPORT void set_material_database_verbose_ggems(GGEMS* g, bool v) { g->verbose[1] = v; }
GG_EXPORT void set_source_ggems(GGEMS* g, bool v) { g->verbose[2] = v; }
GG_EXPORT void set_navigator_ggems(GGEMS* g, bool v) { g->verbose[3] = v; }
GG_EXPORT void set_memory_ram_ggems(GGEMS* g, bool v) { g->verbose[4] = v; }
GG_EXPORT void set_process_ggems(GGEMS* g, bool v) { g->verbose[5] = v; }
GG_EXPORT void set_range_cuts_ggems(GGEMS* g, bool v) { g->verbose[6] = v; }
GG_EXPORT void set_random_ggems(GGEMS* g, bool v) { g->verbose[7] = v; }
GG_EXPORT void set_profiling_ggems(GGEMS* g, bool v) { g->verbose[8] = v; }
GG_EXPORT void set_tracking_ggems(GGEMS* g, bool v, int id) {
  g->is_tracking = v;
  g->tracking_id = id;
}
// Scene / run statistics for tests and benchmarks (no counterpart in the reference).
GG_EXPORT const gg_scene* ggems_scene(GGEMS* g) { return g->scene(); }
GG_EXPORT int ggems_number_of_devices(GGEMS* g) { return static_cast<int>(g->devices.size()); }
GG_EXPORT gg_context* ggems_device_context(GGEMS* g, int d) {
  return (d >= 0 && d < static_cast<int>(g->devices.size())) ? g->devices[d].context : nullptr;
}
GG_EXPORT const uint32_t* ggems_initial_random_states(GGEMS* g, int d) { return g->random_states(d).data(); }
GG_EXPORT void ggems_last_run(GGEMS* g, float* ms, int64_t* launches, uint64_t* particles) {
  if (ms) *ms = g->last_run_ms;
  if (launches) *launches = g->last_run_launches;
  if (particles) *particles = g->last_run_particles;
}
// Host-only initialisation of the registered simulation (sources, navigators,
// tables) and its scene, without any device; used by CPU references.
GG_EXPORT const gg_scene* ggems_host_scene(void) {
  return guarded_value<const gg_scene*>(nullptr, [&] {
    static GGEMS* host = new GGEMS();
    host->prepare();
    return host->scene();
  });
}
GG_EXPORT int ggems_number_of_sources(void) { return static_cast<int>(Simulation::instance().sources.size()); }
GG_EXPORT int ggems_source_descriptor(int i, gg_source* out, uint64_t* number_of_particles) {
  auto& s = Simulation::instance().sources;
  if (i < 0 || i >= static_cast<int>(s.size()) || !out) return GG_ERROR_INVALID_ARGUMENT;
  *out = s[i]->descriptor();
  if (number_of_particles) *number_of_particles = s[i]->number_of_particles;
  return GG_OK;
}

// ---- GGEMSOpenCLManager.hh (device selection for the CUDA layer) ----
GG_EXPORT void* get_instance_ggems_opencl_manager(void) { return &g_opencl_manager; }
GG_EXPORT void print_infos_opencl_manager(void*) {
  int32_t n = 0;
  gg_device_count(&n);
  std::cout << "[GGEMS B200 device manager] CUDA devices: " << n << std::endl;
}
GG_EXPORT void set_device_index_ggems_opencl_manager(void*, uint64_t id) {
  auto& v = Simulation::instance().device_indices;
  if (std::find(v.begin(), v.end(), static_cast<int>(id)) == v.end()) v.push_back(static_cast<int>(id));
}
// device_type: "gpu", "all", or a ';'-separated list of indices ("0;1"); the
// vendor is accepted for compatibility (every device here is an NVIDIA GPU).
GG_EXPORT void set_device_to_activate_opencl_manager(void*, const char* type, const char* vendor) {
  guarded([&] {
    (void)vendor;
    std::string t = S(type);
    auto& v = Simulation::instance().device_indices;
    v.clear();
    int32_t n = 0;
    gg_device_count(&n);
    if (t == "gpu" || t == "all") {
      for (int i = 0; i < (t == "all" ? n : std::max(n, 1)); ++i) v.push_back(i);
      if (t == "gpu" && !v.empty()) v.resize(n > 0 ? n : 1);
    } else if (t == "cpu") {
      throw Error("GGEMSOpenCLManager", "DeviceToActivate", "the B200 build runs on GPUs only: no CPU device");
    } else {
      std::stringstream ss(t);
      std::string item;
      while (std::getline(ss, item, ';'))
        if (!item.empty()) v.push_back(std::stoi(item));
    }
  });
}
GG_EXPORT void set_device_balancing_opencl_manager(void*, const char* balancing) {
  guarded([&] {
    auto& b = Simulation::instance().device_balance;
    b.clear();
    std::stringstream ss(S(balancing));
    std::string item;
    double sum = 0.0;
    while (std::getline(ss, item, ';'))
      if (!item.empty()) {
        b.push_back(std::stod(item));
        sum += b.back();
      }
    if (sum > 1.0 + 1e-6 || sum < 1.0 - 1e-6)
      throw Error("GGEMSOpenCLManager", "SetDeviceBalancing", "Device balancing has to be 1 !!!");
  });
}
GG_EXPORT void clean_opencl_manager(void*) { Simulation::instance().clean(); }

// ---- GGEMSMaterialsDatabaseManager.hh ----
GG_EXPORT void* get_instance_materials_manager(void) { return &g_materials_manager; }
GG_EXPORT void set_materials_ggems_materials_manager(void*, const char* filename) {
  guarded([&] { MaterialsDatabase::instance().load(S(filename)); });
}
GG_EXPORT void print_available_chemical_elements_ggems_materials_manager(void*) {
  guarded([&] {
    for (auto& n : MaterialsDatabase::instance().element_names()) std::cout << n << std::endl;
  });
}
GG_EXPORT void print_available_materials_ggems_materials_manager(void*) {
  guarded([&] {
    for (auto& n : MaterialsDatabase::instance().material_names()) std::cout << n << std::endl;
  });
}

// ---- GGEMSProcessesManager.hh ----
GG_EXPORT void* get_instance_processes_manager(void) { return &g_processes_manager; }
GG_EXPORT void add_process_processes_manager(void*, const char* process, const char* particle, const char* phantom) {
  guarded([&] {
    auto& sim = Simulation::instance();
    if (S(phantom) == "all") {
      for (auto& n : sim.navigators) n->add_process(S(process), S(particle));
    } else {
      sim.navigator(S(phantom))->add_process(S(process), S(particle));
    }
  });
}
GG_EXPORT void set_cross_section_table_number_of_bins_processes_manager(void*, uint64_t bins) {
  auto& sim = Simulation::instance();
  sim.cs_number_of_bins = static_cast<int>(std::min<uint64_t>(bins, GG_MAX_CROSS_SECTION_BINS));
}
GG_EXPORT void set_cross_section_table_minimum_energy_processes_manager(void*, float e, const char* unit) {
  guarded([&] {
    float v = energy_unit(e, S(unit));
    if (v < 990.0f * 1.e-6f)
      throw Error("GGEMSProcessesManager", "SetCrossSectionTableMinimumEnergy", "The minimum of energy in the cross section table is 990 eV");
    Simulation::instance().cs_min_energy = v;
  });
}
GG_EXPORT void set_cross_section_table_maximum_energy_processes_manager(void*, float e, const char* unit) {
  guarded([&] {
    float v = energy_unit(e, S(unit));
    if (v > 250.0f) throw Error("GGEMSProcessesManager", "SetCrossSectionTableMaximumEnergy", "The maximum of energy in the cross section table is 250 MeV");
    Simulation::instance().cs_max_energy = v;
  });
}
GG_EXPORT void print_infos_processes_manager(void*) {
  for (auto& n : Simulation::instance().navigators) {
    std::cout << n->name << ":";
    for (int p : n->processes) std::cout << " " << (p == 0 ? "Compton" : p == 1 ? "Photoelectric" : "Rayleigh");
    std::cout << std::endl;
  }
}
GG_EXPORT void print_available_processes_manager(void*) {
  std::cout << "Available processes: Compton, Photoelectric, Rayleigh (gamma)" << std::endl;
}
GG_EXPORT void print_tables_processes_manager(void*, bool) {}

// ---- GGEMSRangeCutsManager.hh ----
GG_EXPORT void* get_instance_range_cuts_manager(void) { return &g_range_cuts_manager; }
GG_EXPORT void set_cut_range_cuts_manager(void*, const char* phantom, const char* particle, float value, const char* unit) {
  guarded([&] {
    auto& sim = Simulation::instance();
    if (S(phantom) == "all") {
      for (auto& n : sim.navigators) n->set_distance_cut(S(particle), value, S(unit));
    } else {
      sim.navigator(S(phantom))->set_distance_cut(S(particle), value, S(unit));
    }
  });
}

// ---- GGEMSSourceManager.hh ----
GG_EXPORT void* get_instance_ggems_source_manager(void) { return &g_source_manager; }
GG_EXPORT void initialize_source_manager(void*, uint32_t) {
  guarded([&] {
    for (auto& s : Simulation::instance().sources) s->initialize();
  });
}
GG_EXPORT void print_infos_source_manager(void*) {
  for (auto& s : Simulation::instance().sources)
    std::cout << s->kind() << " '" << s->name << "': " << s->number_of_particles << " particles" << std::endl;
}
GG_EXPORT void clean_source_manager(void*) {}

// ---- GGEMSXRaySource.hh ----
GG_EXPORT XRaySource* create_ggems_xray_source(const char* name) {
  return guarded_value<XRaySource*>(nullptr, [&] { return new XRaySource(S(name)); });
}
GG_EXPORT void set_position_ggems_xray_source(XRaySource* s, float x, float y, float z, const char* unit) {
  guarded([&] { s->set_position(x, y, z, S(unit)); });
}
GG_EXPORT void set_number_of_particles_xray_source(XRaySource* s, uint64_t n) { s->number_of_particles = n; }
GG_EXPORT void set_source_particle_type_ggems_xray_source(XRaySource* s, const char* t) {
  guarded([&] { s->set_particle_type(S(t)); });
}
GG_EXPORT void set_beam_aperture_ggems_xray_source(XRaySource* s, float a, const char* unit) {
  guarded([&] { s->set_beam_aperture(a, S(unit)); });
}
GG_EXPORT void set_focal_spot_size_ggems_xray_source(XRaySource* s, float w, float h, float d, const char* unit) {
  guarded([&] { s->set_focal_spot_size(w, h, d, S(unit)); });
}
GG_EXPORT void set_rotation_ggems_xray_source(XRaySource* s, float rx, float ry, float rz, const char* unit) {
  guarded([&] { s->set_rotation(rx, ry, rz, S(unit)); });
}
GG_EXPORT void set_monoenergy_ggems_xray_source(XRaySource* s, float e, const char* unit) {
  guarded([&] { s->set_monoenergy(e, S(unit)); });
}
GG_EXPORT void set_polyenergy_ggems_xray_source(XRaySource* s, const char* file) {
  guarded([&] { s->set_polyenergy(S(file)); });
}
GG_EXPORT void set_energy_peak_ggems_xray_source(XRaySource* s, float e, const char* unit, float intensity) {
  guarded([&] { s->set_energy_peak(e, intensity, S(unit)); });
}

// ---- GGEMSVoxelizedSource.hh ----
GG_EXPORT VoxelizedSource* create_ggems_voxelized_source(const char* name) {
  return guarded_value<VoxelizedSource*>(nullptr, [&] { return new VoxelizedSource(S(name)); });
}
GG_EXPORT void set_position_ggems_voxelized_source(VoxelizedSource* s, float x, float y, float z, const char* unit) {
  guarded([&] { s->set_position(x, y, z, S(unit)); });
}
GG_EXPORT void set_rotation_ggems_voxelized_source(VoxelizedSource* s, float rx, float ry, float rz, const char* unit) {
  guarded([&] { s->set_rotation(rx, ry, rz, S(unit)); });
}
GG_EXPORT void set_number_of_particles_voxelized_source(VoxelizedSource* s, uint64_t n) { s->number_of_particles = n; }
GG_EXPORT void set_source_particle_type_ggems_voxelized_source(VoxelizedSource* s, const char* t) {
  guarded([&] { s->set_particle_type(S(t)); });
}
GG_EXPORT void set_monoenergy_ggems_voxelized_source(VoxelizedSource* s, float e, const char* unit) {
  guarded([&] { s->set_monoenergy(e, S(unit)); });
}
GG_EXPORT void set_polyenergy_ggems_voxelized_source(VoxelizedSource* s, const char* file) {
  guarded([&] { s->set_polyenergy(S(file)); });
}
GG_EXPORT void set_phantom_source_ggems_voxelized_source(VoxelizedSource* s, const char* file) {
  s->phantom_source_file = S(file);
}
GG_EXPORT void set_energy_peak_ggems_voxelized_source(VoxelizedSource* s, float e, const char* unit, float intensity) {
  guarded([&] { s->set_energy_peak(e, intensity, S(unit)); });
}

// ---- GGEMSVoxelizedPhantom.hh ----
GG_EXPORT VoxelizedPhantom* create_ggems_voxelized_phantom(const char* name) {
  return guarded_value<VoxelizedPhantom*>(nullptr, [&] { return new VoxelizedPhantom(S(name)); });
}
GG_EXPORT void set_phantom_file_ggems_voxelized_phantom(VoxelizedPhantom* p, const char* phantom, const char* range) {
  p->phantom_file = S(phantom);
  p->range_file = S(range);
}
GG_EXPORT void set_position_ggems_voxelized_phantom(VoxelizedPhantom* p, float x, float y, float z, const char* unit) {
  guarded([&] { p->set_position(x, y, z, S(unit)); });
}
GG_EXPORT void set_rotation_ggems_voxelized_phantom(VoxelizedPhantom* p, float rx, float ry, float rz, const char* unit) {
  guarded([&] { p->set_rotation(rx, ry, rz, S(unit)); });
}
// Visualisation setters: accepted, no effect (no graphics stack in this build).
GG_EXPORT void set_visible_ggems_voxelized_phantom(VoxelizedPhantom*, bool) {}
GG_EXPORT void set_material_visible_ggems_voxelized_phantom(VoxelizedPhantom*, const char*, bool) {}
GG_EXPORT void set_material_color_ggems_voxelized_phantom(VoxelizedPhantom*, const char*, unsigned char, unsigned char, unsigned char) {}
GG_EXPORT void set_material_color_name_ggems_voxelized_phantom(VoxelizedPhantom*, const char*, const char*) {}

// ---- GGEMSMeshedPhantom.hh ----
GG_EXPORT MeshedPhantom* create_ggems_meshed_phantom(const char* name) {
  return guarded_value<MeshedPhantom*>(nullptr, [&] { return new MeshedPhantom(S(name)); });
}
GG_EXPORT void set_phantom_file_ggems_meshed_phantom(MeshedPhantom* p, const char* file) { p->phantom_file = S(file); }
GG_EXPORT void set_position_ggems_meshed_phantom(MeshedPhantom* p, float x, float y, float z, const char* unit) {
  guarded([&] { p->set_position(x, y, z, S(unit)); });
}
GG_EXPORT void set_rotation_ggems_meshed_phantom(MeshedPhantom* p, float rx, float ry, float rz, const char* unit) {
  guarded([&] { p->set_rotation(rx, ry, rz, S(unit)); });
}
// GGEMSNavigator::SetMaterialName: registers the phantom's (single) material.
GG_EXPORT void set_material_name_ggems_meshed_phantom(MeshedPhantom* p, const char* material) {
  guarded([&] { p->materials.push_back(S(material)); });
}
GG_EXPORT void set_mesh_octree_depth_ggems_meshed_phantom(MeshedPhantom* p, int depth) { p->octree_depth = depth; }
// Visualisation setters: accepted, no effect (no graphics stack in this build).
GG_EXPORT void set_visible_ggems_meshed_phantom(MeshedPhantom*, bool) {}
GG_EXPORT void set_material_color_ggems_meshed_phantom(MeshedPhantom*, const char*, unsigned char, unsigned char, unsigned char) {}
GG_EXPORT void set_material_color_name_ggems_meshed_phantom(MeshedPhantom*, const char*, const char*) {}

// GGEMSWorld (src/navigators/GGEMSWorld.cc:605-671)
GG_EXPORT World* create_ggems_world(void) {
  return guarded_value<World*>(nullptr, [&] { return new World(); });
}
GG_EXPORT void set_dimension_ggems_world(World* w, size_t x, size_t y, size_t z) {
  w->dimensions[0] = x;
  w->dimensions[1] = y;
  w->dimensions[2] = z;
}
GG_EXPORT void set_size_ggems_world(World* w, float x, float y, float z, const char* unit) {
  guarded([&] { w->set_element_size(x, y, z, S(unit)); });
}
GG_EXPORT void photon_tracking_ggems_world(World* w, bool on) { w->photon_tracking = on; }
GG_EXPORT void energy_tracking_ggems_world(World* w, bool on) { w->energy_tracking = on; }
GG_EXPORT void energy_squared_tracking_ggems_world(World* w, bool on) { w->energy_squared_tracking = on; }
GG_EXPORT void set_output_ggems_world(World* w, const char* basename) { w->output = S(basename); }
GG_EXPORT void momentum_ggems_world(World* w, bool on) { w->momentum = on; }

// Meshed solid of an STL file as the host API prepares it (test hook; no
// counterpart in the reference).  Output sizes: triangles n*GG_TRIANGLE_FLOATS,
// nodes m*6, node_first m+1, node_triangles n, with n / m from the first call
// (all output pointers NULL).
GG_EXPORT int ggems_build_mesh(const char* stl, const float* matrix, int depth, int32_t* n_triangles, int32_t* n_nodes,
                               float* triangles, float* nodes, int32_t* node_first, int32_t* node_triangles,
                               float* border_min, float* border_max) {
  return guarded_value<int>(GG_ERROR_INVALID_ARGUMENT, [&] {
    MeshedSolid m = build_meshed_solid(S(stl), matrix, depth);
    *n_triangles = m.number_of_triangles;
    *n_nodes = static_cast<int32_t>(m.node_first.size()) - 1;
    if (triangles) std::copy(m.triangles.begin(), m.triangles.end(), triangles);
    if (nodes) std::copy(m.nodes.begin(), m.nodes.end(), nodes);
    if (node_first) std::copy(m.node_first.begin(), m.node_first.end(), node_first);
    if (node_triangles) std::copy(m.node_triangles.begin(), m.node_triangles.end(), node_triangles);
    if (border_min) std::copy(m.border_min, m.border_min + 3, border_min);
    if (border_max) std::copy(m.border_max, m.border_max + 3, border_max);
    return static_cast<int>(GG_OK);
  });
}

// ---- GGEMSCTSystem.hh ----
GG_EXPORT CTSystem* create_ggems_ct_system(const char* name) {
  return guarded_value<CTSystem*>(nullptr, [&] { return new CTSystem(S(name)); });
}
GG_EXPORT void set_number_of_modules_ggems_ct_system(CTSystem* c, uint64_t mx, uint64_t my) {
  c->modules[0] = mx;
  c->modules[1] = my;
}
GG_EXPORT void set_ct_system_type_ggems_ct_system(CTSystem* c, const char* type) {
  guarded([&] {
    std::string t = S(type);
    std::transform(t.begin(), t.end(), t.begin(), ::tolower);
    if (t != "curved" && t != "flat") throw Error("GGEMSCTSystem", "SetCTSystemType", "Available CT system types: 'curved' or 'flat'");
    c->type = t;
  });
}
GG_EXPORT void set_number_of_detection_elements_ggems_ct_system(CTSystem* c, uint64_t x, uint64_t y, uint64_t z) {
  c->elements[0] = x;
  c->elements[1] = y;
  c->elements[2] = z;
}
GG_EXPORT void set_size_of_detection_elements_ggems_ct_system(CTSystem* c, float x, float y, float z, const char* unit) {
  guarded([&] {
    c->element_size[0] = distance_unit(x, S(unit));
    c->element_size[1] = distance_unit(y, S(unit));
    c->element_size[2] = distance_unit(z, S(unit));
  });
}
GG_EXPORT void set_material_name_ggems_ct_system(CTSystem* c, const char* material) { c->materials = {S(material)}; }
GG_EXPORT void set_source_isocenter_distance_ggems_ct_system(CTSystem* c, float d, const char* unit) {
  guarded([&] { c->sid = distance_unit(d, S(unit)); });
}
GG_EXPORT void set_source_detector_distance_ggems_ct_system(CTSystem* c, float d, const char* unit) {
  guarded([&] { c->sdd = distance_unit(d, S(unit)); });
}
GG_EXPORT void set_rotation_ggems_ct_system(CTSystem* c, float rx, float ry, float rz, const char* unit) {
  guarded([&] { c->set_rotation(rx, ry, rz, S(unit)); });
}
GG_EXPORT void set_save_ggems_ct_system(CTSystem* c, const char* basename) { c->output_basename = S(basename); }
GG_EXPORT void set_threshold_ggems_ct_system(CTSystem* c, float t, const char* unit) {
  guarded([&] { c->set_threshold(t, S(unit)); });
}
GG_EXPORT void store_scatter_ggems_ct_system(CTSystem* c, bool s) { c->is_scatter = s; }
GG_EXPORT void set_global_system_position_ggems_ct_system(CTSystem* c, float x, float y, float z, const char* unit) {
  guarded([&] {
    c->global_position[0] = distance_unit(x, S(unit));
    c->global_position[1] = distance_unit(y, S(unit));
    c->global_position[2] = distance_unit(z, S(unit));
  });
}
GG_EXPORT void set_visible_ggems_ct_system(CTSystem*, bool) {}
GG_EXPORT void set_material_color_ggems_ct_system(CTSystem*, const char*, unsigned char, unsigned char, unsigned char) {}
GG_EXPORT void set_material_color_name_ggems_ct_system(CTSystem*, const char*, const char*) {}

// ---- GGEMSDosimetryCalculator.hh ----
GG_EXPORT DosimetryCalculator* create_ggems_dosimetry_calculator(void) { return new (std::nothrow) DosimetryCalculator(); }
GG_EXPORT void delete_dosimetry_calculator(DosimetryCalculator* d) {
  for (auto& n : Simulation::instance().navigators)
    if (n->dose_calculator == d) n->dose_calculator = nullptr;
  delete d;
}
GG_EXPORT void scale_factor_dosimetry_calculator(DosimetryCalculator* d, float s) { d->scale_factor = s; }
GG_EXPORT void water_reference_dosimetry_calculator(DosimetryCalculator* d, bool b) { d->water_reference = b; }
GG_EXPORT void minimum_density_dosimetry_calculator(DosimetryCalculator* d, float v, const char* unit) {
  guarded([&] { d->minimum_density = density_unit(v, S(unit)); });
}
GG_EXPORT void set_dosel_size_dosimetry_calculator(DosimetryCalculator* d, float x, float y, float z, const char* unit) {
  guarded([&] { d->set_dosel_size(x, y, z, S(unit)); });
}
GG_EXPORT void set_dose_output_dosimetry_calculator(DosimetryCalculator* d, const char* f) { d->output = S(f); }
GG_EXPORT void dose_photon_tracking_dosimetry_calculator(DosimetryCalculator* d, bool b) { d->photon_tracking = b; }
GG_EXPORT void dose_edep_dosimetry_calculator(DosimetryCalculator* d, bool b) { d->edep = b; }
GG_EXPORT void dose_hit_dosimetry_calculator(DosimetryCalculator* d, bool b) { d->hit = b; }
GG_EXPORT void dose_edep_squared_dosimetry_calculator(DosimetryCalculator* d, bool b) { d->edep_squared = b; }
GG_EXPORT void dose_uncertainty_dosimetry_calculator(DosimetryCalculator* d, bool b) { d->uncertainty = b; }
GG_EXPORT void dose_tle_navigator(DosimetryCalculator* d, bool b) {
  guarded([&] {
    if (!d->navigator) throw Error("GGEMSDosimetryCalculator", "SetTLE", "attach the calculator to a navigator first");
    d->navigator->is_tle = b;
  });
}
GG_EXPORT void attach_to_navigator_dosimetry_calculator(DosimetryCalculator* d, const char* navigator) {
  guarded([&] { d->attach(S(navigator)); });
}

// ---- GGEMSMaterials.hh / GGEMSCrossSections.hh (standalone table queries) ----
namespace {
struct MaterialsHandle {
  std::vector<std::string> names;
  NavigatorTables tables;
  bool built = false;
  std::vector<int32_t> processes;
  float photon_cut = 1.e-3f;
};
struct CrossSectionsHandle {
  MaterialsHandle* materials;
  std::vector<int32_t> processes;
  NavigatorTables tables;
  bool built = false;
};
int material_index(const std::vector<std::string>& names, const std::string& n) {
  auto it = std::find(names.begin(), names.end(), n);
  if (it == names.end()) throw Error("GGEMSMaterials", "GetMaterialIndex", "Material '" + n + "' not found!!!");
  return static_cast<int>(it - names.begin());
}
}  // namespace

GG_EXPORT MaterialsHandle* create_ggems_materials(void) { return new (std::nothrow) MaterialsHandle(); }
GG_EXPORT void add_material_ggems_materials(MaterialsHandle* m, const char* name) { m->names.push_back(S(name)); }
GG_EXPORT void initialize_ggems_materials(MaterialsHandle* m) {
  guarded([&] {
    const Simulation& sim = Simulation::instance();
    m->tables = build_navigator_tables(m->names, sim.cs_number_of_bins, sim.cs_min_energy, sim.cs_max_energy, {}, m->photon_cut);
    m->built = true;
  });
}
GG_EXPORT void print_material_properties_ggems_materials(MaterialsHandle* m) {
  for (size_t i = 0; i < m->names.size(); ++i)
    std::cout << m->names[i] << (m->built ? " density " + std::to_string(m->tables.density[i] / (units::g / units::cm3)) + " g/cm3" : "")
              << std::endl;
}
GG_EXPORT float get_density_ggems_materials(MaterialsHandle* m, const char* name) {
  return guarded_value<float>(0.0f, [&] {
    return MaterialsDatabase::instance().material(S(name)).density / units::g * units::cm3;
  });
}
GG_EXPORT float get_energy_cut_ggems_materials(MaterialsHandle* m, const char* name, const char* particle, float distance,
                                               const char* unit) {
  return guarded_value<float>(0.0f, [&] {
    if (S(particle) != "gamma") throw Error("GGEMSMaterials", "GetEnergyCut", "only the photon cut is built in this build");
    const Simulation& sim = Simulation::instance();
    float cut = distance_unit(distance, S(unit));
    NavigatorTables t = build_navigator_tables({S(name)}, sim.cs_number_of_bins, sim.cs_min_energy, sim.cs_max_energy, {}, cut);
    (void)m;
    return t.photon_energy_cut[0] / units::keV;
  });
}
GG_EXPORT float get_atomic_number_density_ggems_materials(MaterialsHandle* m, const char* name) {
  return guarded_value<float>(0.0f, [&] {
    int i = material_index(m->names, S(name));
    if (!m->built) throw Error("GGEMSMaterials", "GetAtomicNumberDensity", "materials not initialized");
    return m->tables.atomic_number_density[m->tables.element_offset[i]] / (units::mol / units::cm3);
  });
}
GG_EXPORT void clean_ggems_materials(MaterialsHandle*) {}

GG_EXPORT CrossSectionsHandle* create_ggems_cross_sections(MaterialsHandle* m) {
  auto* c = new (std::nothrow) CrossSectionsHandle();
  if (c) c->materials = m;
  return c;
}
GG_EXPORT void add_process_ggems_cross_sections(CrossSectionsHandle* c, const char* process, const char* particle, bool) {
  guarded([&] {
    if (S(particle) != "gamma") throw Error("GGEMSCrossSections", "AddProcess", "incident particle has to be a 'gamma'");
    int id = S(process) == "Compton" ? 0 : S(process) == "Photoelectric" ? 1 : S(process) == "Rayleigh" ? 2 : -1;
    if (id < 0) throw Error("GGEMSCrossSections", "AddProcess", "Unknown process!!!");
    if (std::find(c->processes.begin(), c->processes.end(), id) == c->processes.end()) c->processes.push_back(id);
  });
}
GG_EXPORT void initialize_ggems_cross_sections(CrossSectionsHandle* c) {
  guarded([&] {
    const Simulation& sim = Simulation::instance();
    c->tables = build_navigator_tables(c->materials->names, sim.cs_number_of_bins, sim.cs_min_energy, sim.cs_max_energy,
                                       c->processes, c->materials->photon_cut);
    c->built = true;
  });
}
// GGEMSCrossSections::GetPhotonCrossSection (src/physics/GGEMSCrossSections.cc:270-330): cm2/g.
GG_EXPORT float get_cs_ggems_cross_sections(CrossSectionsHandle* c, const char* process, const char* material, float energy,
                                            const char* unit) {
  return guarded_value<float>(0.0f, [&] {
    if (!c->built) throw Error("GGEMSCrossSections", "GetPhotonCrossSection", "cross sections not initialized");
    const NavigatorTables& t = c->tables;
    float e = energy_unit(energy, S(unit));
    if (e < t.min_energy || e > t.max_energy)
      throw Error("GGEMSCrossSections", "GetPhotonCrossSection", "Problem energy: out of the cross-section table range");
    int pid = S(process) == "Compton" ? 0 : S(process) == "Photoelectric" ? 1 : S(process) == "Rayleigh" ? 2 : -1;
    if (pid < 0) throw Error("GGEMSCrossSections", "GetPhotonCrossSection", "Unknown process!!!");
    int mat = 0;
    for (size_t i = 0; i < t.materials.size(); ++i)
      if (t.materials[i] == S(material)) {
        mat = static_cast<int>(i);
        break;
      }
    float density = MaterialsDatabase::instance().material(S(material)).density;
    const int nb = t.number_of_bins;
    int low = 0, high = nb - 1;
    while (high - low > 1) {
      int mid = (high + low) / 2;
      if (t.energy_bins[mid] == e) {
        low = mid;
        break;
      }
      if (t.energy_bins[mid] < e) low = mid;
      else high = mid;
    }
    const size_t block = t.materials.size() * static_cast<size_t>(nb);
    float ea = t.energy_bins[low], eb = t.energy_bins[low + 1];
    float ca = t.cross_sections[pid * block + low + nb * mat], cb = t.cross_sections[pid * block + low + 1 + nb * mat];
    float cs;
    if (ea > eb) cs = cb;
    else if (ea >= e) cs = ca;
    else if (eb <= e) cs = cb;
    else cs = ca + (e - ea) * (cb - ca) / (eb - ea);
    return (cs / density) / (units::cm * units::cm / units::g);
  });
}
GG_EXPORT void clean_ggems_cross_sections(CrossSectionsHandle*) {}

// ---- GGEMSAttenuations.hh (mu / mu_en queries on the TLE tables) ----
namespace {
struct AttenuationsHandle {
  MaterialsHandle* materials;
  NavigatorTables tables;
  bool built = false;
};
// GGEMSAttenuations::GetAttenuation / GetEnergyAttenuation
// (src/physics/GGEMSAttenuations.cc:268-335): cm^-1, linear in the 220-bin table.
float attenuation_query(AttenuationsHandle* a, const std::vector<float>& table, const char* material, float energy,
                        const char* unit, const char* method) {
  if (!a->built) throw Error("GGEMSAttenuations", method, "attenuations not initialized");
  const std::vector<float>& eb = a->tables.attenuation_energy_bins;
  const float e = energy_unit(energy, S(unit));
  if (e < 0.001f || e > 1.0f) {  // ATTENUATION_ENERGY_MIN / _MAX
    std::ostringstream oss;
    oss << "Problem energy: " << e << " " << S(unit) << " is not in the range [" << 0.001f << ", " << 1.0f << "] MeV!!!";
    throw Error("GGEMSAttenuations", method, oss.str());
  }
  const int mat = material_index(a->materials->names, S(material));
  const int nb = GG_ATTENUATION_BINS;
  int low = 0, high = nb - 1;
  while (high - low > 1) {
    int mid = (high + low) / 2;
    if (eb[mid] == e) {
      low = mid;
      break;
    }
    if (eb[mid] < e) low = mid;
    else high = mid;
  }
  const float ea = eb[low], ebb = eb[low + 1];
  const float va = table[low + static_cast<size_t>(nb) * mat], vb = table[low + 1 + static_cast<size_t>(nb) * mat];
  if (ea > ebb) return vb;
  if (ea >= e) return va;
  if (ebb <= e) return vb;
  return va + (e - ea) * (vb - va) / (ebb - ea);
}
}  // namespace

GG_EXPORT AttenuationsHandle* create_ggems_attenuations(MaterialsHandle* m, CrossSectionsHandle*) {
  auto* a = new (std::nothrow) AttenuationsHandle();
  if (a) a->materials = m;
  return a;
}
GG_EXPORT void initialize_ggems_attenuations(AttenuationsHandle* a) {
  guarded([&] {
    const Simulation& sim = Simulation::instance();
    a->tables = build_navigator_tables(a->materials->names, sim.cs_number_of_bins, sim.cs_min_energy,
                                       sim.cs_max_energy, {}, a->materials->photon_cut);
    a->built = true;
  });
}
GG_EXPORT float get_mu_ggems_attenuations(AttenuationsHandle* a, const char* material, float energy, const char* unit) {
  return guarded_value<float>(0.0f, [&] { return attenuation_query(a, a->tables.mu, material, energy, unit, "GetAttenuation"); });
}
GG_EXPORT float get_mu_en_ggems_attenuations(AttenuationsHandle* a, const char* material, float energy,
                                             const char* unit) {
  return guarded_value<float>(0.0f, [&] {
    return attenuation_query(a, a->tables.mu_en, material, energy, unit, "GetEnergyAttenuation");
  });
}
GG_EXPORT void clean_ggems_attenuations(AttenuationsHandle*) {}

// ---- GGEMSProfilerManager.hh / GGEMSRAMManager.hh ----
GG_EXPORT void* get_instance_profiler_manager(void) { return &g_profiler_manager; }
GG_EXPORT void print_summary_profiler_manager(void*) { Profiler::instance().print_summary(std::cout); }
GG_EXPORT void* get_instance_ggems_ram_manager(void) { return &g_ram_manager; }
GG_EXPORT void print_infos_ram_manager(void*) {}

// ---- table export (no counterpart in the reference) ----
// Builds one navigator's physics tables for `material_names` (label order)
// from the loaded material database (loading `materials_file` first if the
// database is empty), with the given cross-section table binning, process
// order and photon range cut.  Output arrays are caller-allocated with the
// sizes of gg_physics_tables: energy_bins[nbins], cross_sections[3*nmat*nbins],
// rayleigh_per_atom[101*nbins], density / photon_cut / n_elements /
// element_offset[nmat], atomic_number / atomic_number_density[sum of elements].
GG_EXPORT int ggems_build_tables(const char* materials_file, const char* const* material_names, int n_materials,
                                 int number_of_bins, float min_energy, float max_energy, const int* process_ids,
                                 int n_processes, float photon_distance_cut, float* energy_bins, float* cross_sections,
                                 float* rayleigh, float* density, float* photon_cut, int32_t* n_elements,
                                 int32_t* element_offset, uint8_t* atomic_number, float* atomic_number_density,
                                 int32_t* total_elements) {
  return guarded_value<int>(GG_ERROR_INVALID_ARGUMENT, [&] {
    if (materials_file && !MaterialsDatabase::instance().ready()) MaterialsDatabase::instance().load(S(materials_file));
    std::vector<std::string> names(material_names, material_names + n_materials);
    std::vector<int32_t> procs(process_ids, process_ids + n_processes);
    NavigatorTables t = build_navigator_tables(names, number_of_bins, min_energy, max_energy, procs, photon_distance_cut);
    std::copy(t.energy_bins.begin(), t.energy_bins.end(), energy_bins);
    std::copy(t.cross_sections.begin(), t.cross_sections.end(), cross_sections);
    std::copy(t.rayleigh_per_atom.begin(), t.rayleigh_per_atom.end(), rayleigh);
    std::copy(t.density.begin(), t.density.end(), density);
    std::copy(t.photon_energy_cut.begin(), t.photon_energy_cut.end(), photon_cut);
    std::copy(t.number_of_elements.begin(), t.number_of_elements.end(), n_elements);
    std::copy(t.element_offset.begin(), t.element_offset.end(), element_offset);
    std::copy(t.atomic_number.begin(), t.atomic_number.end(), atomic_number);
    std::copy(t.atomic_number_density.begin(), t.atomic_number_density.end(), atomic_number_density);
    *total_elements = static_cast<int32_t>(t.atomic_number.size());
    return static_cast<int>(GG_OK);
  });
}

// Voxelized phantom labels as GGEMSVoxelizedSolid::ConvertImageToLabel builds
// them (no counterpart in the reference's C ABI).  dims receives the MHD
// DimSize; labels (nx*ny*nz, may be NULL to query dims) the material index.
GG_EXPORT int ggems_phantom_labels(const char* phantom_file, const char* range_file, int32_t* dims, float* spacing,
                                   uint8_t* labels) {
  return guarded_value<int>(GG_ERROR_INVALID_ARGUMENT, [&] {
    MHDHeader h;
    std::vector<uint8_t> out = voxelized_labels(S(phantom_file), S(range_file), nullptr, &h);
    for (int i = 0; i < 3; ++i) {
      dims[i] = h.dim[i];
      if (spacing) spacing[i] = h.spacing[i];
    }
    if (labels) std::copy(out.begin(), out.end(), labels);
    return static_cast<int>(GG_OK);
  });
}
