// Physics tables of the GGEMS-compatible host API (see gg_physics.hh).
//
// Every float operation keeps the reference's order and precision (this file
// is compiled without FMA contraction) so that the tables are bit-identical
// to GGEMS's.  Sources followed:
//   material database        src/materials/GGEMSMaterialsDatabaseManager.cc:97-140, src/io/GGEMSTextReader.cc:40-126
//   atomic number density    include/GGEMS/materials/GGEMSMaterialsDatabaseManager.hh:244-255
//   material tables          src/materials/GGEMSMaterials.cc:209-300
//   energy bins              src/physics/GGEMSCrossSections.cc:198-208
//   per-material sum         src/physics/GGEMSEMProcess.cc:129-143
//   Compton per atom         src/physics/GGEMSComptonScattering.cc:75-101
//   photoelectric per atom   src/physics/GGEMSPhotoElectricEffect.cc:76-98
//   Rayleigh per atom        src/physics/GGEMSRayleighScattering.cc:80-102
//   photon range cut         src/physics/GGEMSRangeCuts.cc:129-232, 325-384, 544-590
//   log energy table         src/physics/GGEMSLogEnergyTable.cc:40-161
//   attenuation (mu, mu_en)  src/physics/GGEMSAttenuations.cc:40-82, 142-230
#include "gg_physics.hh"

#include "ggems_b200.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <sstream>

namespace gg {

namespace {
constexpr float kAvogadro = 6.02214179e+23f;
// LinearInterpolation (GGEMSMathAlgorithms.hh:76-86)
float lerp_table(float xa, float ya, float xb, float yb, float x) {
  if (xa > xb) return yb;
  if (xa >= x) return ya;
  if (xb <= x) return yb;
  return ya + (x - xa) * (yb - ya) / (xb - xa);
}
constexpr float kElectronMassC2 = 0.510998910f;
constexpr float kAtomicMassUnit = 0.01036426891f;
}  // namespace

MaterialsDatabase& MaterialsDatabase::instance() {
  static MaterialsDatabase db;
  return db;
}

MaterialsDatabase::MaterialsDatabase() {
  const PhysicsData& pd = physics_data();
  const char* names = pd.get<char>("element_names");
  const uint8_t* z = pd.get<uint8_t>("element_z");
  const float* m = pd.get<float>("element_molar_mass");
  const float* I = pd.get<float>("element_mean_excitation");
  const int32_t* st = pd.get<int32_t>("element_state");
  const size_t n = pd.count("element_z", 1);
  for (size_t i = 0; i < n; ++i) {
    ChemicalElement e;
    e.Z = z[i];
    e.molar_mass = m[i] * (units::g / units::mol);
    e.mean_excitation_energy = I[i] * units::eV;
    e.state = st[i];
    elements_.emplace(std::string(names + 16 * i), e);
  }
}

void MaterialsDatabase::load(const std::string& filename) {
  if (!materials_.empty()) return;  // "Material database if already loaded!!!"
  std::ifstream in(filename);
  if (!in) throw Error("GGEMSFileStream", "CheckInputStream", "Problem reading filename: " + filename);
  std::string line;
  while (std::getline(in, line)) {
    skip_comment(in, line);
    if (is_blank(line)) continue;
    remove_space(line);
    SingleMaterial mat;
    std::string name = line.substr(line.find_first_not_of("\t "), line.find(":"));
    // GGEMSMaterialReader::ReadMaterialDensity
    size_t first = line.find_first_of("0123456789", line.find("d="));
    size_t last = line.find_first_not_of("0123456789.", first);
    float density = 0.0f;
    std::stringstream(line.substr(first, last != std::string::npos ? last - first : last)) >> density;
    size_t semi = line.find_first_of(";");
    std::string unit = line.substr(last, semi != std::string::npos ? semi - last : semi);
    if (unit == "g/cm3") density *= units::g / units::cm3;
    else if (unit == "mg/cm3") density *= units::mg / units::cm3;
    else throw Error("GGEMSMaterialReader", "ReadMaterialDensity", "Unknown density unit in material database file!!!");
    mat.density = density;
    // ReadMaterialNumberOfElements
    size_t nf = line.find_first_of("0123456789", line.find("n="));
    size_t nl = line.find_last_of(";");
    size_t count = 0;
    std::stringstream(line.substr(nf, nl != std::string::npos ? nl - nf : nl)) >> count;
    for (size_t i = 0; i < count; ++i) {
      if (!std::getline(in, line)) throw Error("GGEMSMaterialsDatabaseManager", "LoadMaterialsDatabase", "truncated material " + name);
      remove_space(line);
      size_t a = line.find("name=") + 5;
      size_t b = line.find_first_of(";");
      mat.element_names.push_back(line.substr(a, b != std::string::npos ? b - a : b));
      size_t ff = line.find_first_of("0123456789", line.find("f="));
      size_t fl = line.find_last_of(";");
      float frac = 0.0f;
      std::stringstream(line.substr(ff, fl != std::string::npos ? fl - ff : fl)) >> frac;
      mat.fractions.push_back(frac);
    }
    materials_.emplace(name, mat);
  }
}

const SingleMaterial& MaterialsDatabase::material(const std::string& name) const {
  auto it = materials_.find(name);
  if (it == materials_.end())
    throw Error("GGEMSMaterialsDatabaseManager", "GetMaterial", "Material '" + name + "' not found in the database!!!");
  return it->second;
}

const ChemicalElement& MaterialsDatabase::element(const std::string& name) const {
  auto it = elements_.find(name);
  if (it == elements_.end())
    throw Error("GGEMSMaterialsDatabaseManager", "GetChemicalElement",
                "Chemical element '" + name + "' not found in the database!!!");
  return it->second;
}

float MaterialsDatabase::atomic_number_density(const std::string& material_name, size_t index) const {
  const SingleMaterial& m = material(material_name);
  const ChemicalElement& e = element(m.element_names[index]);
  double v = static_cast<double>(kAvogadro) / static_cast<double>(e.molar_mass) * static_cast<double>(m.density) *
             static_cast<double>(m.fractions[index]);
  return static_cast<float>(v);
}

std::vector<std::string> MaterialsDatabase::material_names() const {
  std::vector<std::string> out;
  for (auto& kv : materials_) out.push_back(kv.first);
  return out;
}
std::vector<std::string> MaterialsDatabase::element_names() const {
  std::vector<std::string> out;
  for (auto& kv : elements_) out.push_back(kv.first);
  return out;
}

float compton_cross_section_per_atom(float energy, uint8_t Z) {
  float cs = 0.0f;
  if (Z < 1 || energy < 1e-4f) return cs;
  float p1 = Z * (2.7965e-23f + 1.9756e-27f * Z + -3.9178e-29f * Z * Z);
  float p2 = Z * (-1.8300e-23f + -1.0205e-24f * Z + 6.8241e-27f * Z * Z);
  float p3 = Z * (6.7527e-22f + -7.3913e-24f * Z + 6.0480e-27f * Z * Z);
  float p4 = Z * (-1.9798e-21f + 2.7079e-24f * Z + 3.0274e-26f * Z * Z);
  float T0 = (Z < 1.5f) ? 40.0e-3f : 15.0e-3f;
  float x = fmaxf(energy, T0) / kElectronMassC2;
  cs = p1 * logf(1.0f + 2.0f * x) / x + (p2 + p3 * x + p4 * x * x) / (1.0f + 20.0f * x + 230.0f * x * x + 440.0f * x * x * x);
  if (energy < T0) {
    x = (T0 + 1.0e-3f) / kElectronMassC2;
    float upper =
        p1 * logf(1.0f + 2.0f * x) / x + (p2 + p3 * x + p4 * x * x) / (1.0f + 20.0f * x + 230.0f * x * x + 440.0f * x * x * x);
    float slope = (-T0 * (upper - cs)) / (cs * 1.0e-3f);
    float curv = (Z > 1.5f) ? 0.375f - 0.0556f * logf(Z) : 0.15f;
    float le = logf(energy / T0);
    cs *= expf(-le * (slope + curv * le));
  }
  return cs;
}

float photoelectric_cross_section_per_atom(float energy, uint8_t Z) {
  const PhysicsData& pd = physics_data();
  const float* ion = pd.get<float>("sandia_ionization_potentials");
  const int16_t* cumul = pd.get<int16_t>("sandia_cumulative_intervals");
  const int16_t* nint = pd.get<int16_t>("sandia_number_of_intervals");
  const float* ratio = pd.get<float>("sandia_z_to_a_ratio");
  const float* table = pd.get<float>("sandia_table");
  float e_min = std::fmax(ion[Z], 10.0f) * units::eV;
  if (energy < e_min) return 0.0f;
  int pos = cumul[Z - 1] + nint[Z];
  while (energy < static_cast<float>(table[pos * 5]) * units::keV) --pos;
  float aover_avo = kAtomicMassUnit * static_cast<float>(Z) / ratio[Z];
  double inv = 1.0 / static_cast<double>(energy);
  double inv2 = inv * inv;
  const double a = static_cast<double>(aover_avo);
  return static_cast<float>(inv * static_cast<double>(table[pos * 5 + 1]) * a * 0.160217648e-22 +
                            inv2 * static_cast<double>(table[pos * 5 + 2]) * a * 0.160217648e-25 +
                            inv * inv2 * static_cast<double>(table[pos * 5 + 3]) * a * 0.160217648e-28 +
                            inv2 * inv2 * static_cast<double>(table[pos * 5 + 4]) * a * 0.160217648e-31);
}

namespace {
// LogLogInterpolation (include/GGEMS/maths/GGEMSMathAlgorithms.hh:89-103), host flavour.
float log_log(float x, float x0, float y0, float x1, float y1) {
  if (x < x0) return y0;
  if (x > x1) return y1;
  x0 = 1.0f / x0;
  return std::pow(10.0f, std::log10(y0) + std::log10(y1 / y0) * (std::log10(x * x0) / std::log10(x1 * x0)));
}
}  // namespace

float rayleigh_cross_section_per_atom(float energy, uint8_t Z) {
  const PhysicsData& pd = physics_data();
  const int32_t* cumul = pd.get<int32_t>("rayleigh_cs_cumulative");
  const int32_t* nint = pd.get<int32_t>("rayleigh_cs_intervals");
  const float* cs = pd.get<float>("rayleigh_cross_section");
  if (energy < 250e-6f || energy > 100e3f) return 0.0f;
  const int start = cumul[Z];
  const int stop = start + 2 * (nint[Z] - 1);
  int pos = start;
  while (pos < stop && !(cs[pos] >= energy)) pos += 2;
  if (energy < 1e3f) return static_cast<float>(1.0e-22f * log_log(energy, cs[pos - 2], cs[pos - 1], cs[pos], cs[pos + 1]));
  return 1.0e-22f * cs[pos - 1];
}

namespace {

// GGEMSRangeCuts::ComputePhotonCrossSection (GGEMSRangeCuts.cc:325-384).
float range_cut_photon_cross_section(uint8_t atomic_number, float energy) {
  const float t1keV = 1.0f * units::keV, t200keV = 200.f * units::keV, t100MeV = 100.f * units::MeV;
  float gZ = -1.0f, s200keV = 0, s1keV = 0, tmin = 0, tlow = 0, smin = 0, slow = 0, cmin = 0, clow = 0, chigh = 0;
  if (std::abs(atomic_number - gZ) > 0.1f) {
    gZ = atomic_number;
    const float zsq = gZ * gZ;
    const float zlog = logf(gZ);
    const float zlogsq = zlog * zlog;
    s200keV = (0.2651f - 0.1501f * zlog + 0.02283f * zlogsq) * zsq;
    tmin = (0.552f + 218.5f / gZ + 557.17f / zsq) * units::MeV;
    smin = (0.01239f + 0.005585f * zlog - 0.000923f * zlogsq) * expf(1.5f * zlog);
    cmin = logf(s200keV / smin) / (logf(tmin / t200keV) * logf(tmin / t200keV));
    tlow = 0.2f * expf(-7.355f / sqrtf(gZ)) * units::MeV;
    slow = s200keV * expf(0.042f * gZ * logf(t200keV / tlow) * logf(t200keV / tlow));
    s1keV = 300.0f * zsq;
    clow = logf(s1keV / slow) / logf(tlow / t1keV);
    chigh = (7.55e-5f - 0.0542e-5f * gZ) * zsq * gZ / logf(t100MeV / tmin);
  }
  float xs;
  if (energy < tlow) xs = energy < t1keV ? slow * expf(clow * logf(tlow / t1keV)) : slow * expf(clow * logf(tlow / energy));
  else if (energy < t200keV) xs = s200keV * expf(0.042f * gZ * logf(t200keV / energy) * logf(t200keV / energy));
  else if (energy < tmin) xs = smin * expf(cmin * logf(tmin / energy) * logf(tmin / energy));
  else xs = smin + chigh * logf(energy / tmin);
  return xs * units::barn;
}

// GGEMSLogEnergyTable (src/physics/GGEMSLogEnergyTable.cc).
class LogEnergyTable {
 public:
  LogEnergyTable(float low, float high, size_t bins) : nodes_(bins + 1), data_(bins + 1, 0.0f), edges_(bins + 1) {
    width_ = logf(high / low) / static_cast<float>(bins);
    base_ = logf(low) / width_;
    edges_[0] = low;
    for (size_t i = 1; i + 1 < nodes_; ++i) edges_[i] = expf((base_ + static_cast<float>(i)) * width_);
    edges_[nodes_ - 1] = high;
  }
  float edge(size_t i) const { return edges_[i]; }
  float data(size_t i) const { return data_[i]; }
  void set(size_t i, float v) { data_[i] = v; }
  float value(float e) const {
    if (e <= edges_.front()) return data_[0];
    if (e >= edges_.back()) return data_[nodes_ - 1];
    size_t i = find_bin(e);
    float xa = edges_[i], ya = data_[i], xb = edges_[i + 1], yb = data_[i + 1];
    if (xa > xb) return yb;
    if (xa >= e) return ya;
    if (xb <= e) return yb;
    return ya + (e - xa) * (yb - ya) / (xb - xa);
  }

 private:
  size_t find_bin(float e) const {
    if (e < edges_[1]) return 0;
    if (e >= edges_[nodes_ - 2]) return nodes_ - 2;
    if (e < edges_[0] || e > edges_[1]) {  // index 0 rejected: FindBinLocation
      size_t bin = static_cast<size_t>(logf(e) / width_ - base_);
      if (bin + 2 > nodes_) bin = nodes_ - 2;
      else if (bin > 0 && e < edges_[bin]) --bin;
      else if (bin + 2 < nodes_ && e > edges_[bin + 1]) ++bin;
      return bin;
    }
    return 0;
  }
  size_t nodes_;
  float width_ = 0, base_ = 0;
  std::vector<float> data_, edges_;
};

// Photon branch of GGEMSRangeCuts::ConvertToEnergy.
float photon_energy_cut(const uint8_t* Z, const float* density, int n, float cut, float min_energy) {
  const float max_energy = 10.0f * units::GeV;
  const size_t bins = 300;
  std::vector<LogEnergyTable> loss;
  for (int i = 0; i < n; ++i) {
    LogEnergyTable t(min_energy, max_energy, bins);
    for (size_t j = 0; j < bins; ++j) t.set(j, range_cut_photon_cross_section(Z[i], t.edge(j)));
    loss.push_back(t);
  }
  LogEnergyTable range(min_energy, max_energy, bins);
  for (size_t i = 0; i < bins; ++i) {
    float sigma = 0.0f;
    for (int j = 0; j < n; ++j) sigma += density[j] * loss[j].data(i);
    range.set(i, 5.0f / sigma);
  }
  // ConvertLengthToEnergyCut
  const float epsilon = 0.01f;
  float rmax = -1.e10f * units::mm, t1 = min_energy, r1 = range.data(0), t2 = max_energy, kinetic;
  if (cut < r1) {
    kinetic = t1;
  } else {
    for (size_t i = 0; i < bins; ++i) {
      float t = range.edge(i), r = range.data(i);
      if (r > rmax) rmax = r;
      if (r < cut) {
        t1 = t;
        r1 = r;
      } else if (r > cut) {
        t2 = t;
        break;
      }
    }
    if (cut >= rmax) {
      kinetic = max_energy;
    } else {
      float t3 = sqrtf(t1 * t2);
      float r3 = range.value(t3);
      while (fabsf(1.0f - r3 / cut) > epsilon) {
        if (cut <= r3) t2 = t3;
        else t1 = t3;
        t3 = sqrtf(t1 * t2);
        r3 = range.value(t3);
      }
      kinetic = t3;
    }
  }
  if (kinetic < min_energy) kinetic = min_energy;
  else if (kinetic > max_energy) kinetic = max_energy;
  return kinetic;
}

// mu and mu_en (cm^-1) of every material on GG_ATTENUATION_BINS log-spaced
// energies from 1 keV to 1 MeV, mixed from GGEMS's per-element tables by mass
// fraction the way GGEMSAttenuations::Initialize does it.  Two details of that
// code are kept because the TLE dose depends on them: the energy row of
// element Z is searched over the whole concatenated element table up to the
// end of Z's rows (so the search usually lands in an earlier element's rows),
// and landing on Z's first row adds that row without the mass fraction.
void build_attenuations(NavigatorTables& t, const MaterialsDatabase& db) {
  const PhysicsData& pd = physics_data();
  const int32_t* rows_of = pd.get<int32_t>("mu_nb_energy_bins");
  const int32_t* first_row = pd.get<int32_t>("mu_index_energy");
  // GGEMSMuDataConstants has rows for Z = 1..92 only (kMuNbElements); GGEMS
  // reads past the end of its tables for heavier elements (undefined values).
  // Here such elements add nothing to mu and mu_en, which only the TLE dose
  // mode reads.
  const int max_z = static_cast<int>(pd.count("mu_index_energy", 4)) - 1;
  const float* raw = pd.get<float>("mu_data");
  const size_t n_rows = pd.count("mu_data", 4) / 3;
  std::vector<float> e(n_rows), mu(n_rows), mu_en(n_rows);
  for (size_t r = 0; r < n_rows; ++r) {
    e[r] = raw[3 * r];
    mu[r] = raw[3 * r + 1];
    mu_en[r] = raw[3 * r + 2];
  }
  constexpr int kBins = GG_ATTENUATION_BINS;
  const float lo = 0.001f, hi = 1.0f;
  const float slope = logf(hi / lo);
  t.attenuation_energy_bins.resize(kBins);
  for (int i = 0; i < kBins; ++i)
    t.attenuation_energy_bins[i] =
        lo * expf(slope * (static_cast<float>(i) / (static_cast<float>(kBins) - 1.0f))) * units::MeV;
  const size_t nm = t.materials.size();
  t.mu.assign(nm * kBins, 0.0f);
  t.mu_en.assign(nm * kBins, 0.0f);
  const float g_cm3 = units::g / units::cm3;
  for (size_t m = 0; m < nm; ++m) {
    const SingleMaterial& mat = db.material(t.materials[m]);
    for (int i = 0; i < kBins; ++i) {
      const float energy = t.attenuation_energy_bins[i];
      float a = 0.0f, b = 0.0f;
      for (size_t k = 0; k < mat.element_names.size(); ++k) {
        const int Z = db.element(mat.element_names[k]).Z;
        if (Z > max_z) continue;
        const float w = mat.fractions[k];
        // bisection over rows [0, first_row[Z] + rows_of[Z]) (GGEMSMathAlgorithms.hh BinarySearch)
        int left = 0, right = first_row[Z] + rows_of[Z] - 1, row = -1;
        while (right - left > 1 && row < 0) {
          const int mid = (left + right) / 2;
          if (e[mid] == energy) row = mid;
          else if (e[mid] < energy) left = mid;
          else right = mid;
        }
        if (row < 0) row = left;
        if (row == first_row[Z]) {
          a += mu[row];
          b += mu_en[row];
        } else if (row == 0) {
          // GGEMS interpolates from the row before the table here (row -1, an
          // out-of-range read); the energy is at or above row 0's (the bins
          // start at the table's first energy), where LinearInterpolation
          // returns row 0's value whatever the row before holds.
          a += w * mu[0];
          b += w * mu_en[0];
        } else {
          a += w * lerp_table(e[row - 1], mu[row - 1], e[row], mu[row], energy);
          b += w * lerp_table(e[row - 1], mu_en[row - 1], e[row], mu_en[row], energy);
        }
      }
      t.mu[m * kBins + i] = a * mat.density / g_cm3;
      t.mu_en[m * kBins + i] = b * mat.density / g_cm3;
    }
  }
}

}  // namespace

NavigatorTables build_navigator_tables(const std::vector<std::string>& materials, int number_of_bins, float min_energy,
                                       float max_energy, const std::vector<int32_t>& process_ids,
                                       float photon_distance_cut) {
  const MaterialsDatabase& db = MaterialsDatabase::instance();
  if (materials.empty()) throw Error("GGEMSMaterials", "BuildMaterialTables", "no material registered");
  if (materials.size() > 255) throw Error("GGEMSMaterials", "AddMaterial", "Limit of material reached. The limit is 255 materials!!!");
  NavigatorTables t;
  t.materials = materials;
  t.number_of_bins = number_of_bins;
  t.min_energy = min_energy;
  t.max_energy = max_energy;
  t.process_ids = process_ids;
  const int nm = static_cast<int>(materials.size());
  int offset = 0;
  for (int i = 0; i < nm; ++i) {
    const SingleMaterial& m = db.material(materials[i]);
    t.number_of_elements.push_back(static_cast<int32_t>(m.element_names.size()));
    t.element_offset.push_back(offset);
    t.density.push_back(m.density);
    for (size_t j = 0; j < m.element_names.size(); ++j) {
      t.atomic_number.push_back(db.element(m.element_names[j]).Z);
      t.atomic_number_density.push_back(db.atomic_number_density(materials[i], j));
    }
    t.photon_energy_cut.push_back(photon_energy_cut(t.atomic_number.data() + offset,
                                                    t.atomic_number_density.data() + offset,
                                                    static_cast<int>(m.element_names.size()), photon_distance_cut,
                                                    min_energy));
    offset += static_cast<int>(m.element_names.size());
  }
  const float slope = logf(max_energy / min_energy);
  for (int i = 0; i < number_of_bins; ++i)
    t.energy_bins.push_back(min_energy * expf(slope * (static_cast<float>(i) / (static_cast<float>(number_of_bins) - 1.0f))) *
                            units::MeV);
  const size_t block = static_cast<size_t>(nm) * number_of_bins;
  t.cross_sections.assign(3 * block, 0.0f);
  t.rayleigh_per_atom.assign(static_cast<size_t>(101) * number_of_bins, 0.0f);
  for (int32_t pid : process_ids) {
    for (int j = 0; j < nm; ++j) {
      for (int i = 0; i < number_of_bins; ++i) {
        const float energy = t.energy_bins[i];
        float sum = 0.0f;
        for (int k = 0; k < t.number_of_elements[j]; ++k) {
          const uint8_t Z = t.atomic_number[t.element_offset[j] + k];
          float per_atom = pid == 0 ? compton_cross_section_per_atom(energy, Z)
                           : pid == 1 ? photoelectric_cross_section_per_atom(energy, Z)
                                      : rayleigh_cross_section_per_atom(energy, Z);
          if (pid == 2) t.rayleigh_per_atom[i + static_cast<size_t>(Z) * number_of_bins] = per_atom;
          sum += t.atomic_number_density[t.element_offset[j] + k] * per_atom;
        }
        t.cross_sections[pid * block + i + static_cast<size_t>(j) * number_of_bins] = sum;
      }
    }
  }
  build_attenuations(t, db);
  return t;
}

}  // namespace gg
