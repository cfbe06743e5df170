// Host-side physics tables for the GGEMS-compatible API: the chemical element
// list, the material database, per-navigator material tables, cross-section
// tables and photon energy cuts.
#ifndef GG_PHYSICS_HH
#define GG_PHYSICS_HH

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "gg_host.hh"

namespace gg {

struct ChemicalElement {
  uint8_t Z;
  float molar_mass;               // internal units (element_M * g/mol)
  float mean_excitation_energy;   // internal units
  int state;                      // 0 solid, 1 gas
};

struct SingleMaterial {
  float density;                  // internal units
  std::vector<std::string> element_names;
  std::vector<float> fractions;
};

// GGEMSMaterialsDatabaseManager (src/materials/GGEMSMaterialsDatabaseManager.cc).
class MaterialsDatabase {
 public:
  static MaterialsDatabase& instance();
  void load(const std::string& filename);   // SetMaterialsDatabase
  bool ready() const { return !materials_.empty(); }
  const SingleMaterial& material(const std::string& name) const;
  const ChemicalElement& element(const std::string& name) const;
  float atomic_number_density(const std::string& material, size_t index) const;
  std::vector<std::string> material_names() const;
  std::vector<std::string> element_names() const;
  void clear() { materials_.clear(); }

 private:
  MaterialsDatabase();
  std::map<std::string, SingleMaterial> materials_;
  std::map<std::string, ChemicalElement> elements_;
};

// One navigator's tables, laid out as the C ABI's gg_physics_tables.
struct NavigatorTables {
  std::vector<std::string> materials;
  int32_t number_of_bins = 0;
  float min_energy = 0.f, max_energy = 0.f;
  std::vector<int32_t> process_ids;            // AddProcess order
  std::vector<float> energy_bins;              // [nbins]
  std::vector<float> cross_sections;           // [3][nmat*nbins]
  std::vector<float> rayleigh_per_atom;        // [101*nbins]
  std::vector<float> density;                  // [nmat]
  std::vector<float> photon_energy_cut;        // [nmat]
  std::vector<int32_t> number_of_elements;     // [nmat]
  std::vector<int32_t> element_offset;         // [nmat]
  std::vector<uint8_t> atomic_number;          // [total]
  std::vector<float> atomic_number_density;    // [total]
  // GGEMSAttenuations tables (mu, mu_en in cm^-1), built for every navigator
  std::vector<float> attenuation_energy_bins;  // [GG_ATTENUATION_BINS]
  std::vector<float> mu;                       // [nmat*GG_ATTENUATION_BINS]
  std::vector<float> mu_en;                    // [nmat*GG_ATTENUATION_BINS]
};

// Builds material tables, photon energy cuts and cross sections for
// `materials` (label order), as GGEMSMaterials::BuildMaterialTables,
// GGEMSRangeCuts::ConvertCutsFromDistanceToEnergy and
// GGEMSCrossSections::Initialize do.
NavigatorTables build_navigator_tables(const std::vector<std::string>& materials, int number_of_bins, float min_energy,
                                       float max_energy, const std::vector<int32_t>& process_ids,
                                       float photon_distance_cut);

// Per-atom cross sections (mm^2), exposed for table queries.
float compton_cross_section_per_atom(float energy, uint8_t Z);
float photoelectric_cross_section_per_atom(float energy, uint8_t Z);
float rayleigh_cross_section_per_atom(float energy, uint8_t Z);

}  // namespace gg

#endif
