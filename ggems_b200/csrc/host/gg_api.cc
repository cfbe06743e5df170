// GGEMS-compatible host classes (see gg_api.hh).
#include "gg_api.hh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <thread>

namespace gg {

namespace {

// GGfloat44MultGGfloat44 (GGEMSMatrixOperations.hh:136-184): float products summed left to right.
std::array<float, 16> mat_mul(const std::array<float, 16>& a, const std::array<float, 16>& b) {
  std::array<float, 16> r{};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j)
      r[i * 4 + j] = a[i * 4 + 0] * b[0 * 4 + j] + a[i * 4 + 1] * b[1 * 4 + j] + a[i * 4 + 2] * b[2 * 4 + j] +
                     a[i * 4 + 3] * b[3 * 4 + j];
  return r;
}

void check_device(int rc, const char* what) {
  if (rc != GG_OK) throw Error("GGEMSOpenCLManager", what, std::string("device layer: ") + gg_last_error());
}

void log(int level, const std::string& cls, const std::string& method, const std::string& msg) {
  if (verbosity() >= level) std::cout << "[GGEMS " << cls << "::" << method << "] " << msg << std::endl;
}

}  // namespace

// ------------------------------------------------------- transformation --
Transformation::Transformation() {
  matrix = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
}
void Transformation::set_axis(const float a[3][3]) {
  matrix = {a[0][0], a[0][1], a[0][2], 0.0f, a[1][0], a[1][1], a[1][2], 0.0f,
            a[2][0], a[2][1], a[2][2], 0.0f, 0.0f,    0.0f,    0.0f,    1.0f};
}
void Transformation::set_translation(float x, float y, float z) {
  position = {x, y, z};
  std::array<float, 16> t = {1, 0, 0, x, 0, 1, 0, y, 0, 0, 1, z, 0, 0, 0, 1};
  matrix = mat_mul(t, matrix);
}
void Transformation::set_rotation(float rx, float ry, float rz) {
  rotation = {rx, ry, rz};
  float c = std::cos(rx), s = std::sin(rx);
  std::array<float, 16> Rx = {1, 0, 0, 0, 0, c, -s, 0, 0, s, c, 0, 0, 0, 0, 1};
  c = std::cos(ry);
  s = std::sin(ry);
  std::array<float, 16> Ry = {c, 0, s, 0, 0, 1, 0, 0, -s, 0, c, 0, 0, 0, 0, 1};
  c = std::cos(rz);
  s = std::sin(rz);
  std::array<float, 16> Rz = {c, -s, 0, 0, s, c, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  std::array<float, 16> R = mat_mul(Rz, mat_mul(Ry, Rx));
  matrix = mat_mul(R, matrix);
}

// --------------------------------------------------------------- sources --
Source::Source(const std::string& n) : name(n) { Simulation::instance().sources.emplace_back(this); }

void Source::set_position(float x, float y, float z, const std::string& unit) {
  transformation.set_translation(distance_unit(x, unit), distance_unit(y, unit), distance_unit(z, unit));
}
void Source::set_rotation(float rx, float ry, float rz, const std::string& unit) {
  transformation.set_rotation(angle_unit(rx, unit), angle_unit(ry, unit), angle_unit(rz, unit));
}
void Source::set_particle_type(const std::string& type) {
  if (type == "gamma") particle_type = 0;
  else if (type == "e-") particle_type = 1;
  else if (type == "e+") particle_type = 2;
  else throw Error("GGEMSSourceManager", "SetParticleType", "Unknown particle!!!");
}
void Source::set_monoenergy(float e, const std::string& unit) {
  energy_mappings.clear();
  energy_mappings.emplace_back(energy_unit(e, unit), 1.0);
  is_interp = 0;
}
void Source::set_polyenergy(const std::string& file) {
  energy_mappings.clear();
  std::ifstream in(file);
  if (!in) throw Error("GGEMSFileStream", "CheckInputStream", "Problem reading filename: " + file);
  std::string line;
  while (std::getline(in, line)) {
    if (is_blank(line)) continue;  // the reference would push an uninitialised bin here
    std::istringstream iss(line);
    double e = 0.0, w = 0.0;
    iss >> e >> w;
    energy_mappings.emplace_back(e, w);
  }
}
void Source::set_energy_peak(float e, float intensity, const std::string& unit) {
  energy_mappings.emplace_back(energy_unit(e, unit), intensity);
  is_interp = 0;
}
void Source::check() const {
  if (particle_type == 99) throw Error("GGEMSSource", "CheckParameters", "You have to set a particle type for the source");
  if (particle_type != 0) throw Error("GGEMSSource", "CheckParameters", "Only photon sources are transported by this build");
  if (name.empty()) throw Error("GGEMSSource", "CheckParameters", "You have to set a name for the source!!!");
  if (number_of_particles == 0) throw Error("GGEMSSource", "CheckParameters", "You have to set a number of particles > 0!!!");
  if (transformation.position[0] == FLT_MIN || transformation.position[1] == FLT_MIN || transformation.position[2] == FLT_MIN)
    throw Error("GGEMSSource", "CheckParameters", "You have to set a position for the source!!!");
  if (transformation.rotation[0] == FLT_MIN || transformation.rotation[1] == FLT_MIN || transformation.rotation[2] == FLT_MIN)
    throw Error("GGEMSSource", "CheckParameters", "You have to set a rotation for the source!!!");
  if (energy_mappings.empty()) throw Error("GGEMSSource", "FillEnergy", "no energy defined for the source");
}
// GGEMSSource::FillEnergy (src/sources/GGEMSSource.cc:265-316)
void Source::fill_energy() {
  const size_t n = energy_mappings.size();
  energy_spectrum.assign(n + 1, 0.0f);
  energy_cdf.assign(n + 1, 0.0f);
  double sum = 0.0;
  for (auto& e : energy_mappings) sum += e.second;
  std::vector<double> tmp(n + 1, 0.0);
  for (size_t i = 0; i < n; ++i) {
    tmp[i + 1] = energy_mappings[i].second;
    energy_spectrum[i] = static_cast<float>(energy_mappings[i].first);
  }
  energy_spectrum[n] = energy_spectrum[n - 1];
  energy_cdf[0] = static_cast<float>(tmp[0]);
  for (size_t i = 1; i <= n; ++i) {
    tmp[i] = tmp[i] + tmp[i - 1];
    energy_cdf[i] = static_cast<float>(tmp[i] / sum);
  }
  energy_cdf[n] = 1.0f;
}
void Source::initialize() {
  check();
  fill_energy();
}

XRaySource::XRaySource(const std::string& n) : Source(n) {
  const float axis[3][3] = {{0.0f, 0.0f, -1.0f}, {0.0f, 1.0f, 0.0f}, {1.0f, 0.0f, 0.0f}};  // GGEMSXRaySource.cc:50-56
  transformation.set_axis(axis);
}
void XRaySource::set_beam_aperture(float a, const std::string& unit) { beam_aperture = angle_unit(a, unit); }
void XRaySource::set_focal_spot_size(float w, float h, float d, const std::string& unit) {
  focal_spot_size[0] = distance_unit(w, unit);
  focal_spot_size[1] = distance_unit(h, unit);
  focal_spot_size[2] = distance_unit(d, unit);
}
void XRaySource::initialize() {
  Source::check();
  if (beam_aperture == FLT_MIN) throw Error("GGEMSXRaySource", "CheckParameters", "You have to set a beam aperture for the source!!!");
  if (beam_aperture < 0.0f) throw Error("GGEMSXRaySource", "CheckParameters", "The beam aperture must be >= 0!!!");
  for (float f : focal_spot_size) {
    if (f == FLT_MIN) throw Error("GGEMSXRaySource", "CheckParameters", "You have to set a focal spot size!!!");
    if (f < 0.0f) throw Error("GGEMSXRaySource", "CheckParameters", "The focal spot size is a posivite value!!!");
  }
  fill_energy();
}
gg_source XRaySource::descriptor() const {
  gg_source s{};
  s.type = GG_SOURCE_XRAY;
  s.particle_type = particle_type;
  std::memcpy(s.matrix, transformation.matrix.data(), sizeof(s.matrix));
  s.beam_aperture = beam_aperture;
  std::memcpy(s.focal_spot_size, focal_spot_size, sizeof(s.focal_spot_size));
  s.number_of_energy_bins = static_cast<int32_t>(energy_mappings.size());
  s.energy_spectrum = energy_spectrum.data();
  s.energy_cdf = energy_cdf.data();
  s.is_interp = is_interp;
  return s;
}

VoxelizedSource::VoxelizedSource(const std::string& n) : Source(n) {
  const float axis[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  transformation.set_axis(axis);
}
// GGEMSVoxelizedSource::FillVoxelActivity (src/sources/GGEMSVoxelizedSource.cc:287-380)
void VoxelizedSource::initialize() {
  Source::check();
  if (phantom_source_file.empty())
    throw Error("GGEMSVoxelizedSource", "CheckParameters", "You have to set a MHD phantom source file for voxelized source!!!");
  fill_energy();
  MHDHeader h = read_mhd(phantom_source_file);
  if (h.type != "MET_FLOAT") throw Error("GGEMSVoxelizedSource", "FillVoxelActivity", "For voxelized source, data type is MET_FLOAT only!!!");
  std::vector<float> act = read_mhd_values(h);
  for (int i = 0; i < 3; ++i) {
    number_of_voxels[i] = h.dim[i];
    voxel_sizes[i] = h.spacing[i];
    border_min[i] = -static_cast<float>(h.dim[i]) * h.spacing[i] * 0.5f;
  }
  int32_t n_active = 0;
  for (float a : act)
    if (a != 0.0f) ++n_active;
  if (n_active == 0) throw Error("GGEMSVoxelizedSource", "FillVoxelActivity", "no active voxel");
  activity_index.assign(n_active + 1, 0);
  activity_cdf.assign(n_active + 1, 0.0f);
  std::vector<float> tmp(n_active + 1, 0.0f);
  float sum = 0.0f;
  int32_t index = 1;
  for (size_t i = 0; i < act.size(); ++i) {
    if (act[i] != 0.0f) {
      activity_index[index] = static_cast<int32_t>(i);
      tmp[index] = act[i];
      sum += act[i];
      ++index;
    }
  }
  // Entry 0 is never written by the reference (left as device memory); it is 0 here.
  activity_index[n_active] = activity_index[n_active - 1];
  activity_cdf[0] = tmp[0];
  for (int32_t i = 1; i <= n_active; ++i) {
    tmp[i] = tmp[i] + tmp[i - 1];
    activity_cdf[i] = tmp[i] / sum;
  }
  activity_cdf[n_active] = 1.0f;
}
gg_source VoxelizedSource::descriptor() const {
  gg_source s{};
  s.type = GG_SOURCE_VOXELIZED;
  s.particle_type = particle_type;
  std::memcpy(s.matrix, transformation.matrix.data(), sizeof(s.matrix));
  s.number_of_energy_bins = static_cast<int32_t>(energy_mappings.size());
  s.energy_spectrum = energy_spectrum.data();
  s.energy_cdf = energy_cdf.data();
  s.is_interp = is_interp;
  std::memcpy(s.number_of_voxels, number_of_voxels, sizeof(s.number_of_voxels));
  std::memcpy(s.voxel_sizes, voxel_sizes, sizeof(s.voxel_sizes));
  std::memcpy(s.border_min, border_min, sizeof(s.border_min));
  s.number_of_activity_bins = static_cast<int64_t>(activity_index.size());
  s.activity_index = activity_index.data();
  s.activity_cdf = activity_cdf.data();
  return s;
}

// ------------------------------------------------------------ navigators --
Navigator::Navigator(const std::string& n) : name(n) { Simulation::instance().navigators.emplace_back(this); }

void Navigator::set_position(float x, float y, float z, const std::string& unit) {
  is_update_pos = true;
  position[0] = distance_unit(x, unit);
  position[1] = distance_unit(y, unit);
  position[2] = distance_unit(z, unit);
}
void Navigator::set_rotation(float rx, float ry, float rz, const std::string& unit) {
  is_update_rot = true;
  rotation[0] = angle_unit(rx, unit);
  rotation[1] = angle_unit(ry, unit);
  rotation[2] = angle_unit(rz, unit);
}
void Navigator::set_threshold(float t, const std::string& unit) { threshold = energy_unit(t, unit); }

// GGEMSCrossSections::AddProcess (src/physics/GGEMSCrossSections.cc:93-150)
void Navigator::add_process(const std::string& process, const std::string& particle) {
  int id = process == "Compton" ? 0 : process == "Photoelectric" ? 1 : process == "Rayleigh" ? 2 : -1;
  if (id < 0)
    throw Error("GGEMSCrossSections", "AddProcess",
                "Unknown process!!! The available processes in GGEMS are: 'Compton', 'Photoelectric', 'Rayleigh'");
  if (particle != "gamma") throw Error("GGEMSCrossSections", "AddProcess", "incident particle has to be a 'gamma'");
  if (std::find(processes.begin(), processes.end(), id) != processes.end()) return;  // already activated
  processes.push_back(id);
}
void Navigator::set_distance_cut(const std::string& particle, float value, const std::string& unit) {
  float cut = distance_unit(value, unit);
  if (particle == "gamma") {
    if (cut < 1.e-3f) throw Error("GGEMSRangeCuts", "SetPhotonDistanceCut", "Distance cut for photon is too small!!! Minimum value is 0.001 mm!!!");
    photon_distance_cut = cut;
  } else if (particle != "e-" && particle != "e+") {
    throw Error("GGEMSMaterials", "SetCut", "Particle name " + particle + " unknown!!! The particles are: gamma, e-, e+");
  }
}
void Navigator::build_tables() {
  const Simulation& sim = Simulation::instance();
  tables = build_navigator_tables(materials, sim.cs_number_of_bins, sim.cs_min_energy, sim.cs_max_energy, processes,
                                  photon_distance_cut);
}

VoxelizedPhantom::VoxelizedPhantom(const std::string& n) : Navigator(n) {}

std::vector<uint8_t> voxelized_labels(const std::string& phantom_file, const std::string& range_file,
                                      std::vector<std::string>* materials, MHDHeader* header) {
  MHDHeader h = read_mhd(phantom_file);
  std::vector<float> values = read_mhd_values(h);
  std::vector<uint8_t> labels(values.size(), 255);
  std::ifstream in(range_file);
  if (!in) throw Error("GGEMSFileStream", "CheckInputStream", "Problem reading filename: " + range_file);
  std::string line;
  int label = 0;
  if (materials) materials->clear();
  while (std::getline(in, line)) {
    if (is_blank(line)) continue;
    std::istringstream iss(line);
    float first = 0.0f, last = 0.0f;
    std::string material;
    iss >> first >> last >> material;
    if (label == 255) throw Error("GGEMSMaterials", "AddMaterial", "Limit of material reached. The limit is 255 materials!!!");
    if (materials) materials->push_back(material);
    for (size_t i = 0; i < values.size(); ++i) {
      float v = values[i];
      if ((v == first && v == last) || (v >= first && v < last)) labels[i] = static_cast<uint8_t>(label);
    }
    ++label;
  }
  for (uint8_t l : labels)
    if (l == 255) throw Error("GGEMSVoxelizedSolid", "ConvertImageToLabel", "Errors(s) in the range data file!!!");
  if (header) *header = h;
  return labels;
}

// GGEMSVoxelizedPhantom::Initialize + GGEMSVoxelizedSolid::LoadVolumeImage / ConvertImageToLabel
// (src/navigators/GGEMSVoxelizedPhantom.cc:88-160, include/GGEMS/geometries/GGEMSVoxelizedSolid.hh:162-257).
void VoxelizedPhantom::initialize(int first_solid_id) {
  (void)first_solid_id;
  if (phantom_file.empty()) throw Error("GGEMSVoxelizedPhantom", "CheckParameters", "You have to set a mhd file containing the voxelized phantom!!!");
  if (range_file.empty()) throw Error("GGEMSVoxelizedPhantom", "CheckParameters", "You have to set a file with the range to material data!!!");
  if (output_basename.empty() && false) throw Error("GGEMSNavigator", "CheckParameters", "Output basename not set!!!");
  MHDHeader h;
  SolidSpec spec;
  spec.labels = voxelized_labels(phantom_file, range_file, &materials, &h);
  gg_solid& s = spec.solid;
  s.type = GG_SOLID_VOXELIZED;
  Transformation tr;  // identity axis (GGEMSVoxelizedSolid.cc:56-62)
  if (is_update_rot) tr.set_rotation(rotation[0], rotation[1], rotation[2]);
  if (is_update_pos) tr.set_translation(position[0], position[1], position[2]);
  std::memcpy(s.obb.matrix, tr.matrix.data(), sizeof(s.obb.matrix));
  for (int i = 0; i < 3; ++i) {
    s.number_of_voxels[i] = h.dim[i];
    s.voxel_sizes[i] = h.spacing[i];
    s.obb.border_min[i] = -static_cast<float>(h.dim[i]) * h.spacing[i] * 0.5f;
    s.obb.border_max[i] = static_cast<float>(h.dim[i]) * h.spacing[i] * 0.5f;
  }
  s.threshold = threshold;
  s.histogram = -1;
  s.scatter_histogram = -1;
  s.dose_map = -1;
  solids.clear();
  solids.push_back(std::move(spec));
  build_tables();
  if (dose_calculator) dose_calculator->initialize(solids[0]);
}

MeshedPhantom::MeshedPhantom(const std::string& n) : Navigator(n) {}

// GGEMSMeshedPhantom::Initialize (src/navigators/GGEMSMeshedPhantom.cc:72-130):
// rotation then position, triangles moved by the full transformation, octree,
// OBB = octree box with an identity matrix.  TLE is ignored with a warning.
void MeshedPhantom::initialize(int first_solid_id) {
  (void)first_solid_id;
  if (phantom_file.empty()) throw Error("GGEMSMeshedPhantom", "CheckParameters", "You have to set a mesh file in STL format!!!");
  if (materials.empty()) throw Error("GGEMSMeshedPhantom", "Initialize", "You have to set a material for the meshed phantom!!!");
  if (is_tle) std::cerr << "[GGEMS GGEMSMeshedPhantom::Initialize] WARNING!!! TLE is not possible for meshed phantom" << std::endl;
  Transformation tr;  // identity axis (GGEMSMeshedSolid.cc:55-62)
  if (is_update_rot) tr.set_rotation(rotation[0], rotation[1], rotation[2]);
  if (is_update_pos) tr.set_translation(position[0], position[1], position[2]);
  SolidSpec spec;
  spec.mesh = std::make_shared<MeshedSolid>(build_meshed_solid(phantom_file, tr.matrix.data(), octree_depth));
  gg_solid& s = spec.solid;
  s.type = GG_SOLID_MESHED;
  for (int i = 0; i < 16; ++i) s.obb.matrix[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  for (int i = 0; i < 3; ++i) {
    s.obb.border_min[i] = spec.mesh->border_min[i];
    s.obb.border_max[i] = spec.mesh->border_max[i];
  }
  s.threshold = threshold;
  s.histogram = -1;
  s.scatter_histogram = -1;
  s.dose_map = -1;
  s.number_of_triangles = spec.mesh->number_of_triangles;
  s.number_of_nodes = static_cast<int32_t>(spec.mesh->node_first.size()) - 1;
  solids.clear();
  solids.push_back(std::move(spec));
  build_tables();
  if (dose_calculator) dose_calculator->initialize(solids[0]);
}

CTSystem::CTSystem(const std::string& n) : Navigator(n) {}

// GGEMSCTSystem::Initialize / InitializeFlatGeometry / InitializeCurvedGeometry
// (src/navigators/GGEMSCTSystem.cc:131-300).
void CTSystem::initialize(int first_solid_id) {
  (void)first_solid_id;
  if (type != "curved" && type != "flat") throw Error("GGEMSCTSystem", "CheckParameters", "Available CT system types: 'curved' or 'flat'");
  if (sdd == 0.0f) throw Error("GGEMSCTSystem", "CheckParameters", "For CT system, source detector distance (SDD) has to be > 0.0 mm!!!");
  if (sid > sdd) throw Error("GGEMSCTSystem", "CheckParameters", "Source isocenter distance must be inferior to source detector distance!!!");
  if (modules[0] == 0 || modules[1] == 0) throw Error("GGEMSSystem", "CheckParameters", "In system parameters, number of module in x and y axis (local axis) has to be > 0!!!");
  if (elements[0] == 0 || elements[1] == 0 || elements[2] == 0) throw Error("GGEMSSystem", "CheckParameters", "In system parameters, number of detection elements in x, y and z axis (local axis) has to be > 0!!!");
  if (element_size[0] == 0.0f || element_size[1] == 0.0f || element_size[2] == 0.0f) throw Error("GGEMSSystem", "CheckParameters", "In system parameters, size of detection elements (local axis) has to be > 0.0 mm!!!");
  if (materials.empty()) throw Error("GGEMSSystem", "CheckParameters", "In system parameters, a material has to be defined!!!");
  if (output_basename.empty()) throw Error("GGEMSNavigator", "CheckParameters", "Output basename not set!!!");
  materials.resize(1);
  const uint64_t n = modules[0] * modules[1];
  solids.assign(n, SolidSpec());
  const float axis[3][3] = {{0.0f, 0.0f, 1.0f}, {0.0f, 1.0f, 0.0f}, {-1.0f, 0.0f, 0.0f}};  // GGEMSSolidBox.cc:77-83
  std::vector<Transformation> tr(n);
  for (auto& t : tr) t.set_axis(axis);
  const float bx = static_cast<float>(elements[0]) * element_size[0];
  const float by = static_cast<float>(elements[1]) * element_size[1];
  const float bz = static_cast<float>(elements[2]) * element_size[2];
  if (type == "curved") {
    float c = (static_cast<float>(elements[1]) * element_size[1]) * 0.5f;
    float rho = std::sqrt(sdd * sdd + c * c);
    float alpha = 2.0f * std::asin(c / rho);
    float ox = -sid, oy = 0.0f, px = sdd - sid, py = 0.0f;
    for (uint64_t j = 0; j < modules[1]; ++j) {
      float step = alpha * (static_cast<float>(j) + 0.5f * (1.0f - static_cast<float>(modules[1])));
      float gx = (px - ox) * std::cos(step) - (py - oy) * std::sin(step) + ox;
      float gy = (px - ox) * std::sin(step) + (py - oy) * std::cos(step) + oy;
      for (uint64_t i = 0; i < modules[0]; ++i) {
        float gz = static_cast<float>(elements[0]) * element_size[0] * (static_cast<float>(i) + 0.5f * (1.0f - static_cast<float>(modules[0])));
        Transformation& t = tr[i + j * modules[0]];
        t.set_rotation(0.0f, 0.0f, step);
        t.set_translation(gx + global_position[0], gy + global_position[1], gz + global_position[2]);
      }
    }
  } else {
    float gx = sdd - sid;
    for (uint64_t j = 0; j < modules[1]; ++j) {
      float gy = static_cast<float>(elements[1]) * element_size[1] * (static_cast<float>(j) + 0.5f * (1.0f - static_cast<float>(modules[1])));
      for (uint64_t i = 0; i < modules[0]; ++i) {
        float gz = static_cast<float>(elements[0]) * element_size[0] * (static_cast<float>(i) + 0.5f * (1.0f - static_cast<float>(modules[0])));
        Transformation& t = tr[i + j * modules[0]];
        t.set_rotation(0.0f, 0.0f, 0.0f);
        t.set_translation(gx + global_position[0], gy + global_position[1], gz + global_position[2]);
      }
    }
  }
  if (is_update_rot)
    for (auto& t : tr) t.set_rotation(rotation[0], rotation[1], rotation[2]);
  for (uint64_t k = 0; k < n; ++k) {
    gg_solid& s = solids[k].solid;
    s.type = GG_SOLID_BOX;
    std::memcpy(s.obb.matrix, tr[k].matrix.data(), sizeof(s.obb.matrix));
    s.obb.border_min[0] = -bx * 0.5f;
    s.obb.border_min[1] = -by * 0.5f;
    s.obb.border_min[2] = -bz * 0.5f;
    s.obb.border_max[0] = bx * 0.5f;
    s.obb.border_max[1] = by * 0.5f;
    s.obb.border_max[2] = bz * 0.5f;
    s.virtual_element_number[0] = static_cast<int32_t>(elements[0]);
    s.virtual_element_number[1] = static_cast<int32_t>(elements[1]);
    s.virtual_element_number[2] = static_cast<int32_t>(elements[2]);
    s.box_size[0] = bx;
    s.box_size[1] = by;
    s.box_size[2] = bz;
    s.threshold = threshold;
    s.dose_map = -1;
  }
  build_tables();
}

// -------------------------------------------------------------- dosimetry --
void DosimetryCalculator::attach(const std::string& navigator_name) {
  navigator = Simulation::instance().navigator(navigator_name);
  navigator->dose_calculator = this;
}
void DosimetryCalculator::set_dosel_size(float x, float y, float z, const std::string& unit) {
  dosel_sizes[0] = distance_unit(x, unit);
  dosel_sizes[1] = distance_unit(y, unit);
  dosel_sizes[2] = distance_unit(z, unit);
}
// GGEMSDosimetryCalculator::Initialize (src/navigators/GGEMSDosimetryCalculator.cc:435-530)
void DosimetryCalculator::initialize(const SolidSpec& spec) {
  const gg_solid& s = spec.solid;
  if (s.type == GG_SOLID_MESHED && dosel_sizes[0] <= 0.0f && dosel_sizes[1] <= 0.0f && dosel_sizes[2] <= 0.0f)
    throw Error("GGEMSDosimetryCalculator", "Initialize",
                "a meshed phantom has no voxel size: set the dosel size with set_dosel_size");
  float vs[3] = {dosel_sizes[0], dosel_sizes[1], dosel_sizes[2]};
  if (dosel_sizes[0] < 0.0f && dosel_sizes[1] < 0.0f && dosel_sizes[2] < 0.0f)
    for (int i = 0; i < 3; ++i) vs[i] = s.voxel_sizes[i];
  if (photon_tracking)
    for (int i = 0; i < 3; ++i)
      if (vs[i] != s.voxel_sizes[i])
        throw Error("GGEMSDosimetryCalculator", "Initialize",
                    "Dosel size and voxel size in voxelized phantom have to be the same when photon tracking is activated!!!");
  map = gg_dose_map{};
  for (int i = 0; i < 3; ++i) {
    map.size_of_dosels[i] = vs[i];
    map.inv_size_of_dosels[i] = 1.0f / vs[i];
    map.border_min[i] = s.obb.border_min[i];
    map.border_max[i] = s.obb.border_max[i];
    float size = s.obb.border_max[i] - s.obb.border_min[i];
    map.number_of_dosels[i] = static_cast<int32_t>(static_cast<uint64_t>(size / vs[i]));
  }
  map.slice_number_of_dosels = map.number_of_dosels[0] * map.number_of_dosels[1];
  map.total_number_of_dosels = map.slice_number_of_dosels * map.number_of_dosels[2];
  map.record_edep_squared = (edep_squared || uncertainty) ? 1 : 0;
  map.record_hit = (hit || uncertainty) ? 1 : 0;
  map.record_photon_tracking = photon_tracking ? 1 : 0;
  // GGEMSVoxelizedPhantom::Initialize enables TLE on its voxelized solid
  // (src/navigators/GGEMSVoxelizedPhantom.cc:115-116); other navigators ignore it.
  map.tle = (navigator && navigator->is_tle && s.type == GG_SOLID_VOXELIZED) ? 1 : 0;
}

// ------------------------------------------------------------ simulation --
Simulation& Simulation::instance() {
  static Simulation s;
  return s;
}
Navigator* Simulation::navigator(const std::string& name) const {
  for (auto& n : navigators)
    if (n->name == name) return n.get();
  throw Error("GGEMSNavigatorManager", "GetNavigator", "Navigator '" + name + "' not found!!!");
}
void Simulation::clean() {
  sources.clear();
  navigators.clear();
  dosimetry.clear();
  world.reset();
}

World::World() { Simulation::instance().world.reset(this); }
void World::set_element_size(float x, float y, float z, const std::string& unit) {
  sizes[0] = distance_unit(x, unit);
  sizes[1] = distance_unit(y, unit);
  sizes[2] = distance_unit(z, unit);
}
// GGEMSWorld::CheckParameters (src/navigators/GGEMSWorld.cc:172-190)
void World::check() const {
  if (dimensions[0] == 0 || dimensions[1] == 0 || dimensions[2] == 0)
    throw Error("GGEMSWorld", "CheckParameters", "Dimensions of world have to be set");
  if (sizes[0] < 0.0f || sizes[1] < 0.0f || sizes[2] < 0.0f)
    throw Error("GGEMSWorld", "CheckParameters", "Size of elements in world");
}

GGEMS::GGEMS() {}
GGEMS::~GGEMS() {
  for (auto& d : devices)
    if (d.context) gg_context_destroy(d.context);
}

// GGEMS::Initialize (src/global/GGEMS.cc:199-297): sources (with the random
// streams) first, then navigators, then the scene goes to every device.
void GGEMS::prepare() {
  Simulation& sim = Simulation::instance();
  if (!MaterialsDatabase::instance().ready()) throw Error("GGEMS", "Initialize", "Materials are not loaded in GGEMS!!!");
  if (sim.sources.empty()) throw Error("GGEMSSourceManager", "Initialize", "No source defined!!!");
  for (auto& s : sim.sources) s->initialize();
  // Navigators (GGEMSNavigatorManager::Initialize), solids numbered in registration order.
  int next_id = 0;
  for (auto& n : sim.navigators) {
    n->initialize(next_id);
    next_id += static_cast<int>(n->solids.size());
  }
  build_scene();
  prepared_ = true;
}

void GGEMS::initialize(uint32_t seed) {
  Simulation& sim = Simulation::instance();
  if (!MaterialsDatabase::instance().ready()) throw Error("GGEMS", "Initialize", "Materials are not loaded in GGEMS!!!");
  if (sim.sources.empty()) throw Error("GGEMSSourceManager", "Initialize", "No source defined!!!");
  // Devices (GGEMSOpenCLManager device activation, balancing).
  for (auto& d : devices)
    if (d.context) gg_context_destroy(d.context);
  devices.clear();
  std::vector<int> idx = sim.device_indices.empty() ? std::vector<int>{0} : sim.device_indices;
  for (size_t i = 0; i < idx.size(); ++i) {
    Device d;
    d.index = idx[i];
    d.balance = i < sim.device_balance.size() ? sim.device_balance[i] : 1.0 / static_cast<double>(idx.size());
    check_device(gg_context_create(d.index, &d.context), "ActivateDevice");
    devices.push_back(d);
  }
  // Seeds: GGEMSPseudoRandomGenerator (src/randoms/GGEMSPseudoRandomGenerator.cc:123-167); device d takes
  // the d-th block of 4 * MAXIMUM_PARTICLES std::mt19937 outputs.
  if (seed == 0) {
    std::ifstream ur("/dev/urandom", std::ios::binary);
    ur.read(reinterpret_cast<char*>(&seed), sizeof(seed));
  }
  seed_ = seed;
  states_.assign(devices.size(), std::vector<uint32_t>(5 * static_cast<size_t>(GG_MAXIMUM_PARTICLES)));
  for (size_t d = 0; d < devices.size(); ++d) {
    check_device(gg_seed_random_states(states_[d].data(), GG_MAXIMUM_PARTICLES, seed,
                                       static_cast<int64_t>(d) * GG_MAXIMUM_PARTICLES),
                 "InitializeSeeds");
    check_device(gg_set_random_states(devices[d].context, states_[d].data(), GG_MAXIMUM_PARTICLES), "InitializeSeeds");
  }
  prepare();
  for (auto& d : devices) check_device(gg_upload_scene(d.context, &scene_), "UploadScene");
  // GGEMS_TRACKING (set_tracking_ggems): the kernels record the tracked particle id's states
  for (auto& d : devices)
    check_device(gg_set_tracking(d.context, is_tracking ? tracking_id : -1, kTrackingCapacity), "Tracking");
  initialized_ = true;
  log(1, "GGEMS", "Initialize", "GGEMS initialization succeeded");
}

void GGEMS::build_scene() {
  Simulation& sim = Simulation::instance();
  tables_.clear();
  solids_.clear();
  dose_maps_.clear();
  histogram_sizes_.clear();
  solid_owner_.clear();
  for (size_t ni = 0; ni < sim.navigators.size(); ++ni) {
    Navigator* n = sim.navigators[ni].get();
    NavigatorTables& t = n->tables;
    gg_physics_tables pt{};
    pt.number_of_bins = t.number_of_bins;
    pt.number_of_materials = static_cast<int32_t>(t.materials.size());
    pt.number_of_processes = static_cast<int32_t>(t.process_ids.size());
    for (size_t p = 0; p < t.process_ids.size() && p < 3; ++p) pt.process_id[p] = t.process_ids[p];
    pt.energy_bins = t.energy_bins.data();
    pt.cross_sections = t.cross_sections.data();
    bool rayleigh = std::find(t.process_ids.begin(), t.process_ids.end(), 2) != t.process_ids.end();
    pt.rayleigh_per_atom = rayleigh ? t.rayleigh_per_atom.data() : nullptr;
    pt.density = t.density.data();
    pt.photon_energy_cut = t.photon_energy_cut.data();
    pt.number_of_elements = t.number_of_elements.data();
    pt.element_offset = t.element_offset.data();
    pt.atomic_number = t.atomic_number.data();
    pt.atomic_number_density = t.atomic_number_density.data();
    pt.total_elements = static_cast<int32_t>(t.atomic_number.size());
    pt.attenuation_energy_bins = t.attenuation_energy_bins.empty() ? nullptr : t.attenuation_energy_bins.data();
    pt.mu_en = t.mu_en.empty() ? nullptr : t.mu_en.data();
    tables_.push_back(pt);
    for (size_t k = 0; k < n->solids.size(); ++k) {
      SolidSpec& spec = n->solids[k];
      gg_solid s = spec.solid;
      s.navigator = static_cast<int32_t>(ni);
      s.labels = spec.labels.empty() ? nullptr : spec.labels.data();
      if (spec.mesh) {
        s.triangles = spec.mesh->triangles.data();
        s.nodes = spec.mesh->nodes.data();
        s.node_first = spec.mesh->node_first.data();
        s.node_triangles = spec.mesh->node_triangles.empty() ? nullptr : spec.mesh->node_triangles.data();
      }
      if (auto* ct = dynamic_cast<CTSystem*>(n)) {
        s.histogram = static_cast<int32_t>(histogram_sizes_.size());
        histogram_sizes_.push_back(static_cast<int32_t>(ct->elements[0] * ct->elements[1]));
        s.scatter_histogram = -1;
        if (ct->is_scatter) {
          s.scatter_histogram = static_cast<int32_t>(histogram_sizes_.size());
          histogram_sizes_.push_back(static_cast<int32_t>(ct->elements[0] * ct->elements[1]));
        }
      }
      if (n->dose_calculator && k == 0) {
        s.dose_map = static_cast<int32_t>(dose_maps_.size());
        dose_maps_.push_back(n->dose_calculator->map);
      }
      solids_.push_back(s);
      solid_owner_.emplace_back(n, static_cast<int>(k));
    }
  }
  const PhysicsData& pd = physics_data();
  rayleigh_fit_.assign(9 * 101, 0.0f);
  for (int i = 0; i < 9; ++i) std::memcpy(&rayleigh_fit_[i * 101], pd.get<float>("rayleigh_pp" + std::to_string(i)), 101 * 4);
  scene_ = gg_scene{};
  scene_.number_of_tables = static_cast<int32_t>(tables_.size());
  scene_.tables = tables_.data();
  scene_.number_of_solids = static_cast<int32_t>(solids_.size());
  scene_.solids = solids_.data();
  scene_.number_of_dose_maps = static_cast<int32_t>(dose_maps_.size());
  scene_.dose_maps = dose_maps_.data();
  scene_.number_of_histograms = static_cast<int32_t>(histogram_sizes_.size());
  scene_.histogram_sizes = histogram_sizes_.data();
  scene_.rayleigh_fit = rayleigh_fit_.data();
  scene_.world = nullptr;
  if (World* w = sim.world.get()) {
    // GGEMSWorld::Initialize (src/navigators/GGEMSWorld.cc:264-298)
    w->check();
    world_ = gg_world{};
    for (int a = 0; a < 3; ++a) {
      if (w->dimensions[a] > 0x7fffffffull) throw Error("GGEMSWorld", "CheckParameters", "world dimension too large");
      world_.dimensions[a] = static_cast<int32_t>(w->dimensions[a]);
      world_.sizes[a] = w->sizes[a];
    }
    world_.photon_tracking = w->photon_tracking ? 1 : 0;
    world_.energy_tracking = w->energy_tracking ? 1 : 0;
    world_.energy_squared_tracking = w->energy_squared_tracking ? 1 : 0;
    world_.momentum = w->momentum ? 1 : 0;
    scene_.world = &world_;
  }
}

Profiler& Profiler::instance() {
  static Profiler p;
  return p;
}
void Profiler::add(const std::string& label, double ms) {
  std::lock_guard<std::mutex> lock(mutex_);
  for (auto& kv : labels_)
    if (kv.first == label) {
      kv.second += ms;
      return;
    }
  labels_.emplace_back(label, ms);
}
void Profiler::reset() {
  std::lock_guard<std::mutex> lock(mutex_);
  labels_.clear();
}
// GGEMSChrono::DisplayTime (src/tools/GGEMSChrono.cc:38-49) format
void Profiler::print_summary(std::ostream& out) const {
  std::lock_guard<std::mutex> lock(mutex_);
  for (const auto& kv : labels_) {
    const long long ms = static_cast<long long>(kv.second);
    char line[256];
    std::snprintf(line, sizeof(line), "Elapsed time (%s): %02lld hours %02lld mins %02lld secs %03lld ms",
                  kv.first.c_str(), ms / 3600000, (ms / 60000) % 60, (ms / 1000) % 60, ms % 1000);
    out << "[GGEMS GGEMSChrono::DisplayTime] " << line << std::endl;
  }
}

// The tracked particle's states in the spirit of the GGEMS_TRACKING printf
// blocks of the reference kernels (e.g. TrackThroughGGEMSVoxelizedSolid.cl:184-210).
void print_track(std::ostream& out, const std::vector<gg_track_point>& pts, int id, int device, int source) {
  static const char* kKind[] = {"primary", "enter solid", "step", "interaction", "leave solid", "dead"};
  auto process = [](int p) -> const char* {
    switch (p) {
      case GG_COMPTON_SCATTERING: return "Compton";
      case GG_PHOTOELECTRIC_EFFECT: return "photoelectric";
      case GG_RAYLEIGH_SCATTERING: return "Rayleigh";
      case GG_TRANSPORTATION: return "transportation";
      default: return "-";
    }
  };
  const char* tag = "[GGEMS Tracking] ";
  out << tag << "################################################################################\n";
  out << tag << "Particle id: " << id << ", device " << device << ", source " << source << ", " << pts.size()
      << " points\n";
  char line[320];
  for (const auto& t : pts) {
    std::snprintf(line, sizeof(line),
                  "history %d %-12s solid %2d %-14s position (x, y, z): %e %e %e mm, direction: %e %e %e, energy: %e keV\n",
                  t.history, (t.kind >= 0 && t.kind < 6) ? kKind[t.kind] : "?", t.solid, process(t.process),
                  t.position[0], t.position[1], t.position[2], t.direction[0], t.direction[1], t.direction[2],
                  t.E / units::keV);
    out << tag << line;
  }
  out.flush();
}

// GGEMS::Run / RunOnDevice (src/global/GGEMS.cc:303-414): one host thread per
// device; each runs every source's share of primaries; then results are saved.
void GGEMS::run() {
  if (!initialized_) throw Error("GGEMS", "Run", "GGEMS is not initialized!!!");
  Simulation& sim = Simulation::instance();
  std::vector<int> errors(devices.size(), GG_OK);
  std::vector<std::string> messages(devices.size());
  std::vector<float> ms(devices.size(), 0.0f);
  std::vector<int64_t> launches(devices.size(), 0);
  uint64_t total = 0;
  for (auto& s : sim.sources) total += s->number_of_particles;
  std::vector<std::vector<std::vector<gg_track_point>>> traces(devices.size());  // per device, per source
  auto worker = [&](size_t d) {
    for (auto& src : sim.sources) {
      // GGEMSSource::OrganizeParticlesInBatch (src/sources/GGEMSSource.cc:379-401)
      const size_t nd = devices.size();
      uint64_t n = 0;
      if (nd == 1) {
        n = src->number_of_particles;
      } else if (sim.device_balance.empty()) {
        n = src->number_of_particles / nd + (d < src->number_of_particles % nd ? 1 : 0);
      } else {
        uint64_t sum = 0;
        std::vector<uint64_t> per(nd);
        for (size_t i = 0; i < nd; ++i) {
          per[i] = static_cast<uint64_t>(static_cast<float>(src->number_of_particles) * static_cast<float>(devices[i].balance));
          sum += per[i];
        }
        if (sum != src->number_of_particles)
          per[0] += static_cast<uint64_t>(std::llabs(static_cast<long long>(src->number_of_particles - sum)));
        n = per[d];
      }
      gg_source desc = src->descriptor();
      int rc = gg_run_source(devices[d].context, &desc, n);
      if (rc == GG_OK) rc = gg_synchronize(devices[d].context);
      if (rc != GG_OK) {
        errors[d] = rc;
        messages[d] = gg_last_error();
        return;
      }
      float t = 0.0f;
      int64_t l = 0;
      gg_last_run_stats(devices[d].context, &t, &l);
      ms[d] += t;
      launches[d] += l;
      Profiler::instance().add("transport kernel, device index " + std::to_string(devices[d].index), t);
      if (is_tracking) {
        std::vector<gg_track_point> pts(kTrackingCapacity);
        int32_t count = 0;
        if (gg_read_tracking(devices[d].context, pts.data(), kTrackingCapacity, &count) == GG_OK) {
          pts.resize(std::min(count, kTrackingCapacity));
          traces[d].push_back(std::move(pts));
        }
      }
    }
  };
  std::vector<std::thread> threads;
  for (size_t d = 0; d < devices.size(); ++d) threads.emplace_back(worker, d);
  for (auto& t : threads) t.join();
  for (size_t d = 0; d < devices.size(); ++d)
    for (size_t s = 0; s < traces[d].size(); ++s) print_track(std::cout, traces[d][s], tracking_id, static_cast<int>(d), static_cast<int>(s));
  for (size_t d = 0; d < devices.size(); ++d)
    if (errors[d] != GG_OK) throw Error("GGEMS", "RunOnDevice", messages[d]);
  last_run_ms = *std::max_element(ms.begin(), ms.end());
  last_run_launches = 0;
  for (auto l : launches) last_run_launches += l;
  last_run_particles = total;
  save_results();
  // GGEMS::Run ends with the profiler summary when profiling is verbose (src/global/GGEMS.cc)
  if (verbose[8]) Profiler::instance().print_summary(std::cout);
}

// SaveResults of GGEMSSystem (src/navigators/GGEMSSystem.cc:165-260) and
// GGEMSDosimetryCalculator (src/navigators/GGEMSDosimetryCalculator.cc:536-800):
// tallies are read from every device and summed on the host.
void GGEMS::save_results() {
  Simulation& sim = Simulation::instance();
  const size_t nh = histogram_sizes_.size(), nd = dose_maps_.size();
  histograms_.assign(nh, {});
  for (size_t h = 0; h < nh; ++h) histograms_[h].assign(histogram_sizes_[h], 0);
  edep_.assign(nd, {});
  edep2_.assign(nd, {});
  hit_.assign(nd, {});
  ptrack_.assign(nd, {});
  for (size_t m = 0; m < nd; ++m) {
    size_t n = static_cast<size_t>(dose_maps_[m].total_number_of_dosels);
    edep_[m].assign(n, 0.0);
    edep2_[m].assign(n, 0.0);
    hit_[m].assign(n, 0);
    ptrack_[m].assign(n, 0);
  }
  const size_t nw = scene_.world ? static_cast<size_t>(world_.dimensions[0]) * world_.dimensions[1] * world_.dimensions[2] : 0;
  world_photon_.assign(nw, 0);
  world_energy_.assign(nw, 0.0);
  world_energy2_.assign(nw, 0.0);
  for (auto& v : world_momentum_) v.assign(nw, 0.0);
  for (auto& dev : devices) {
    std::vector<std::vector<int32_t>> h(nh);
    std::vector<int32_t*> hp(nh);
    for (size_t i = 0; i < nh; ++i) {
      h[i].assign(histogram_sizes_[i], 0);
      hp[i] = h[i].data();
    }
    std::vector<std::vector<double>> e(nd), e2(nd);
    std::vector<std::vector<int32_t>> hi(nd), pt(nd);
    std::vector<double*> ep(nd), e2p(nd);
    std::vector<int32_t*> hip(nd), ptp(nd);
    for (size_t m = 0; m < nd; ++m) {
      size_t n = static_cast<size_t>(dose_maps_[m].total_number_of_dosels);
      e[m].assign(n, 0.0);
      e2[m].assign(n, 0.0);
      hi[m].assign(n, 0);
      pt[m].assign(n, 0);
      ep[m] = e[m].data();
      e2p[m] = e2[m].data();
      hip[m] = hi[m].data();
      ptp[m] = pt[m].data();
    }
    gg_tally_buffers tb{hp.data(), ep.data(), e2p.data(), hip.data(), ptp.data()};
    std::vector<int32_t> wp(nw, 0);
    std::vector<double> we(nw, 0.0), we2(nw, 0.0), wm[3];
    if (nw) {
      for (auto& v : wm) v.assign(nw, 0.0);
      tb.world_photon_tracking = wp.data();
      tb.world_energy = we.data();
      tb.world_energy_squared = we2.data();
      tb.world_momentum_x = wm[0].data();
      tb.world_momentum_y = wm[1].data();
      tb.world_momentum_z = wm[2].data();
    }
    check_device(gg_read_tallies(dev.context, &tb), "ReadTallies");
    for (size_t k = 0; k < nw; ++k) {
      world_photon_[k] += wp[k];
      world_energy_[k] += we[k];
      world_energy2_[k] += we2[k];
      for (int a = 0; a < 3; ++a) world_momentum_[a][k] += wm[a][k];
    }
    for (size_t i = 0; i < nh; ++i)
      for (size_t k = 0; k < h[i].size(); ++k) histograms_[i][k] += h[i][k];
    for (size_t m = 0; m < nd; ++m)
      for (size_t k = 0; k < e[m].size(); ++k) {
        edep_[m][k] += e[m][k];
        edep2_[m][k] += e2[m][k];
        hit_[m][k] += hi[m][k];
        ptrack_[m][k] += pt[m][k];
      }
  }
  // CT systems: one image of all modules (GGEMSSystem::SaveResults layout).
  for (size_t s = 0; s < solids_.size(); ++s) {
    auto* ct = dynamic_cast<CTSystem*>(solid_owner_[s].first);
    if (!ct || solid_owner_[s].second != 0) continue;
    const uint64_t ex = ct->elements[0], ey = ct->elements[1];
    int32_t dim[3] = {static_cast<int32_t>(ct->modules[0] * ex), static_cast<int32_t>(ct->modules[1] * ey),
                      static_cast<int32_t>(ct->elements[2])};
    std::vector<int32_t> out(static_cast<size_t>(dim[0]) * dim[1] * dim[2], 0), sout(out.size(), 0);
    for (uint64_t jj = 0; jj < ct->modules[1]; ++jj)
      for (uint64_t ii = 0; ii < ct->modules[0]; ++ii) {
        const gg_solid& so = solids_[s + ii + jj * ct->modules[0]];
        for (uint64_t j = 0; j < ey; ++j)
          for (uint64_t i = 0; i < ex; ++i) {
            size_t o = (i + ii * ex) + (j + jj * ey) * dim[0];
            out[o] += histograms_[so.histogram][i + j * ex];
            if (so.scatter_histogram >= 0) sout[o] += histograms_[so.scatter_histogram][i + j * ex];
          }
      }
    write_mhd(ct->output_basename, "MET_INT", dim, ct->element_size, out.data(), 4);
    if (ct->is_scatter) {
      std::string b = ct->output_basename;
      size_t f = b.find(".mhd");
      b = (f == std::string::npos) ? b + "-scatter.mhd" : b.substr(0, f) + "-scatter.mhd";
      write_mhd(b, "MET_INT", dim, ct->element_size, sout.data(), 4);
    }
  }
  // Dosimetry outputs.
  for (size_t s = 0; s < solids_.size(); ++s) {
    Navigator* n = solid_owner_[s].first;
    if (!n->dose_calculator || solid_owner_[s].second != 0) continue;
    DosimetryCalculator* dc = n->dose_calculator;
    const int m = solids_[s].dose_map;
    const gg_dose_map& dm = dose_maps_[m];
    const size_t nn = static_cast<size_t>(dm.total_number_of_dosels);
    // Every device converts its own tallies (GGEMSDosimetryCalculator::ComputeDose);
    // the saved images are the sums over devices (SaveDose / SaveUncertainty,
    // src/navigators/GGEMSDosimetryCalculator.cc:726-800).
    std::vector<float> dose(nn, 0.0f), unc(nn, 0.0f), dose_d(nn), unc_d(nn);
    for (auto& dev : devices) {
      check_device(gg_compute_dose(dev.context, m, static_cast<int32_t>(s), dc->scale_factor, dc->water_reference ? 1 : 0,
                                   dc->minimum_density, dose_d.data(), dc->uncertainty ? unc_d.data() : nullptr),
                   "ComputeDose");
      for (size_t k = 0; k < nn; ++k) {
        dose[k] += dose_d[k];
        if (dc->uncertainty) unc[k] += unc_d[k];
      }
    }
    int32_t dim[3] = {dm.number_of_dosels[0], dm.number_of_dosels[1], dm.number_of_dosels[2]};
    write_mhd(dc->output + "_dose.mhd", "MET_FLOAT", dim, dm.size_of_dosels, dose.data(), 4);
    if (dc->uncertainty) write_mhd(dc->output + "_uncertainty.mhd", "MET_FLOAT", dim, dm.size_of_dosels, unc.data(), 4);
    if (dc->edep) write_mhd(dc->output + "_edep.mhd", "MET_DOUBLE", dim, dm.size_of_dosels, edep_[m].data(), 8);
    if (dc->edep_squared) write_mhd(dc->output + "_edep_squared.mhd", "MET_DOUBLE", dim, dm.size_of_dosels, edep2_[m].data(), 8);
    if (dc->hit) write_mhd(dc->output + "_hit.mhd", "MET_INT", dim, dm.size_of_dosels, hit_[m].data(), 4);
    if (dc->photon_tracking)
      write_mhd(dc->output + "_photon_tracking.mhd", "MET_INT", dim, dm.size_of_dosels, ptrack_[m].data(), 4);
  }
  // GGEMSWorld::SaveResults (src/navigators/GGEMSWorld.cc:405-602)
  if (World* w = scene_.world ? sim.world.get() : nullptr) {
    const int32_t* dim = world_.dimensions;
    const std::string& b = w->output;
    if (w->photon_tracking) write_mhd(b + "_world_photon_tracking.mhd", "MET_INT", dim, world_.sizes, world_photon_.data(), 4);
    if (w->energy_tracking) write_mhd(b + "_world_edep.mhd", "MET_DOUBLE", dim, world_.sizes, world_energy_.data(), 8);
    if (w->energy_squared_tracking)
      write_mhd(b + "_world_edep_squared.mhd", "MET_DOUBLE", dim, world_.sizes, world_energy2_.data(), 8);
    if (w->momentum) {
      const char* axis[3] = {"x", "y", "z"};
      for (int a = 0; a < 3; ++a)
        write_mhd(b + "_world_momentum_" + axis[a] + ".mhd", "MET_DOUBLE", dim, world_.sizes, world_momentum_[a].data(), 8);
    }
  }
}

}  // namespace gg
