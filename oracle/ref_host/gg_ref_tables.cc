// Test infrastructure only (host-table pin).  Builds the navigator tables with
// GGEMS's own host code -- GGEMSMaterialsDatabaseManager, GGEMSMaterials
// (BuildMaterialTables, GGEMSRangeCuts::ConvertCutsFromDistanceToEnergy),
// GGEMSCrossSections + GGEMSEMProcess with the Compton / photoelectric /
// Rayleigh per-atom formulas, and GGEMSAttenuations -- compiled unmodified from
// a reference checkout by oracle/build.py, and hands them out in the layout of
// the oracle's gg_oracle_build_tables / gg_oracle_build_attenuations, so the
// tests can compare the product's and the oracle's tables with the
// reference's bit for bit.
//
// The reference's GGEMSOpenCLManager owns OpenCL contexts, queues and device
// buffers; the table builders only allocate buffers, map them to fill them
// and unmap them.  This file defines those members over host memory (one
// "device", index 0); CL/cl.hpp beside it supplies the types.  The reference's
// GGEMSNavigatorManager is only reached from printing paths of the process
// manager, so only its constructor and destructor are defined.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "GGEMS/global/GGEMSOpenCLManager.hh"
#include "GGEMS/materials/GGEMSMaterials.hh"
#include "GGEMS/materials/GGEMSMaterialsDatabaseManager.hh"
#include "GGEMS/navigators/GGEMSNavigatorManager.hh"
#include "GGEMS/physics/GGEMSAttenuations.hh"
#include "GGEMS/physics/GGEMSCrossSections.hh"
#include "GGEMS/physics/GGEMSMuData.hh"
#include "GGEMS/physics/GGEMSParticleCrossSections.hh"
#include "GGEMS/physics/GGEMSProcessesManager.hh"
#include "GGEMS/tools/GGEMSPrint.hh"

// ---- GGEMSOpenCLManager over host memory ----

GGEMSOpenCLManager::GGEMSOpenCLManager(void) : work_group_size_(64) {
  device_name_.push_back("host memory (table pin)");
  device_global_mem_size_.push_back(1ULL << 40);
  device_max_mem_alloc_size_.push_back(1ULL << 40);
  devices_.push_back(nullptr);
  ComputingDevice d;
  d.index_ = 0;
  d.context_ = new cl::Context;
  d.queue_ = new cl::CommandQueue;
  computing_devices_.push_back(d);
}

GGEMSOpenCLManager::~GGEMSOpenCLManager(void) {
  for (auto& d : computing_devices_) d.Clean();
}

void GGEMSOpenCLManager::CheckOpenCLError(GGint const& error, std::string const& class_name,
                                          std::string const& method_name) const {
  if (error != CL_SUCCESS) throw std::runtime_error(class_name + "::" + method_name + ": error " + std::to_string(error));
}

void GGEMSOpenCLManager::HandleEvent(cl::Event&, char*) {}

cl::Buffer* GGEMSOpenCLManager::Allocate(void* host_ptr, GGsize const& size, GGsize const&, cl_mem_flags flags,
                                         std::string const&) {
  auto* b = new cl::Buffer(size);  // zero-filled
  if (host_ptr && (flags & (CL_MEM_COPY_HOST_PTR | CL_MEM_USE_HOST_PTR))) std::memcpy(b->data(), host_ptr, size);
  return b;
}

void GGEMSOpenCLManager::Deallocate(cl::Buffer* buffer, GGsize, GGsize const&, std::string const&) { delete buffer; }

// ---- GGEMSNavigatorManager: no navigators in the table pin ----

GGEMSNavigatorManager::GGEMSNavigatorManager(void) : navigators_(nullptr), number_of_navigators_(0), world_(nullptr) {}

GGEMSNavigatorManager::~GGEMSNavigatorManager(void) {}

// ---- the pin's entry points ----

namespace {

std::mutex g_mutex;
std::string g_error;

const char* process_name(int id) {
  switch (id) {
    case 0: return "Compton";
    case 1: return "Photoelectric";
    case 2: return "Rayleigh";
    default: return nullptr;
  }
}

void load_database(const char* materials_file) {
  GGEMSMaterialsDatabaseManager& db = GGEMSMaterialsDatabaseManager::GetInstance();
  if (!db.IsReady()) db.SetMaterialsDatabase(materials_file);
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* gg_ref_tables_error(void) { return g_error.c_str(); }

// The same arguments and outputs as gg_oracle_build_tables (energies in MeV,
// lengths in mm, GGEMS's internal units throughout); the physics data come
// from the reference's own headers instead of a data file.
__attribute__((visibility("default"))) int gg_ref_build_tables(
    const char* materials_file, const char* const* material_names, int n_materials, int number_of_bins,
    float min_energy, float max_energy, const int* process_ids, int n_processes, float photon_distance_cut,
    float* energy_bins, float* cross_sections, float* rayleigh, float* density, float* photon_cut,
    int32_t* n_elements, int32_t* element_offset, uint8_t* atomic_number, float* atomic_number_density,
    int32_t* total_elements) {
  std::lock_guard<std::mutex> lock(g_mutex);
  try {
    set_ggems_verbose(0);
    load_database(materials_file);
    GGEMSProcessesManager& pm = GGEMSProcessesManager::GetInstance();
    pm.SetCrossSectionTableNumberOfBins(static_cast<GGsize>(number_of_bins));
    pm.SetCrossSectionTableMinimumEnergy(min_energy, "MeV");
    pm.SetCrossSectionTableMaximumEnergy(max_energy, "MeV");

    GGEMSMaterials materials;
    for (int i = 0; i < n_materials; ++i) materials.AddMaterial(material_names[i]);
    materials.SetDistanceCut("gamma", photon_distance_cut, "mm");
    materials.Initialize();
    GGEMSCrossSections cs(&materials);
    for (int p = 0; p < n_processes; ++p) {
      const char* name = process_name(process_ids[p]);
      if (!name) throw std::runtime_error("unknown process id");
      cs.AddProcess(name, "gamma");
    }
    cs.Initialize();

    const auto* mt = static_cast<const GGEMSMaterialTables*>(materials.GetMaterialTables(0)->data());
    const auto* xs = static_cast<const GGEMSParticleCrossSections*>(cs.GetCrossSections(0)->data());
    for (int i = 0; i < n_materials; ++i) {
      n_elements[i] = static_cast<int32_t>(mt->number_of_chemical_elements_[i]);
      element_offset[i] = static_cast<int32_t>(mt->index_of_chemical_elements_[i]);
      density[i] = mt->density_of_material_[i];
      photon_cut[i] = mt->photon_energy_cut_[i];
    }
    const int total = static_cast<int>(mt->total_number_of_chemical_elements_);
    for (int k = 0; k < total; ++k) {
      atomic_number[k] = mt->atomic_number_Z_[k];
      atomic_number_density[k] = mt->atomic_number_density_[k];
    }
    *total_elements = total;
    for (int i = 0; i < number_of_bins; ++i) energy_bins[i] = xs->energy_bins_[i];
    const size_t block = static_cast<size_t>(n_materials) * number_of_bins;
    std::memset(cross_sections, 0, 3 * block * sizeof(float));
    std::memset(rayleigh, 0, static_cast<size_t>(101) * number_of_bins * sizeof(float));
    for (int p = 0; p < n_processes; ++p) {
      const int pid = process_ids[p];
      std::memcpy(cross_sections + pid * block, xs->photon_cross_sections_[pid], block * sizeof(float));
      if (pid == 2)
        std::memcpy(rayleigh, xs->photon_cross_sections_per_atom_[2],
                    static_cast<size_t>(101) * number_of_bins * sizeof(float));
    }
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return 1;
  }
}

// The same outputs as gg_oracle_build_attenuations: energy_bins[220] and
// mu / mu_en[n_materials * 220] from GGEMSAttenuations::Initialize.
__attribute__((visibility("default"))) int gg_ref_build_attenuations(const char* materials_file,
                                                                    const char* const* material_names,
                                                                    int n_materials, float* energy_bins, float* mu,
                                                                    float* mu_en) {
  std::lock_guard<std::mutex> lock(g_mutex);
  try {
    set_ggems_verbose(0);
    load_database(materials_file);
    GGEMSMaterials materials;
    for (int i = 0; i < n_materials; ++i) materials.AddMaterial(material_names[i]);
    materials.Initialize();
    GGEMSCrossSections cs(&materials);
    cs.AddProcess("Compton", "gamma");
    cs.Initialize();
    GGEMSAttenuations att(&materials, &cs);
    att.Initialize();
    const auto* t = static_cast<const GGEMSMuMuEnData*>(att.GetAttenuations(0)->data());
    for (int i = 0; i < ATTENUATION_TABLE_NUMBER_BINS; ++i) energy_bins[i] = t->energy_bins_[i];
    const size_t n = static_cast<size_t>(n_materials) * ATTENUATION_TABLE_NUMBER_BINS;
    std::memcpy(mu, t->mu_, n * sizeof(float));
    std::memcpy(mu_en, t->mu_en_, n * sizeof(float));
    return 0;
  } catch (std::exception const& e) {
    g_error = e.what();
    return 1;
  }
}

}  // extern "C"
