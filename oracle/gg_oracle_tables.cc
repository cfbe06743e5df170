// CPU oracle for GGEMS's host-side table building -- TEST INFRASTRUCTURE ONLY.
//
// Restates, in plain C++, how GGEMS v1.3 turns a material database and a
// process list into the tables photon transport reads:
//   * material database text parsing (src/materials/GGEMSMaterialsDatabaseManager.cc:97-140,
//     src/io/GGEMSTextReader.cc:40-208);
//   * material tables (src/materials/GGEMSMaterials.cc:209-300,
//     include/GGEMS/materials/GGEMSMaterialsDatabaseManager.hh:244-255);
//   * energy bins and per-material cross sections (src/physics/GGEMSCrossSections.cc:170-219,
//     src/physics/GGEMSEMProcess.cc:65-143) with the per-atom Compton
//     (src/physics/GGEMSComptonScattering.cc:75-101), photoelectric
//     (src/physics/GGEMSPhotoElectricEffect.cc:76-98) and Rayleigh
//     (src/physics/GGEMSRayleighScattering.cc:80-102) formulas;
//   * the photon range cut converted to an energy cut (src/physics/GGEMSRangeCuts.cc:129-626,
//     src/physics/GGEMSLogEnergyTable.cc:40-161).
// Physics data (Sandia, Rayleigh, elements) come from ggems_b200/data/physics_data.bin.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "ggems_b200.h"

namespace {

// Units (include/GGEMS/tools/GGEMSSystemOfUnits.hh) and constants (GGEMSConstants.hh).
constexpr float kEV = 1.e-6f;
constexpr float kKeV = 1.e-3f;
constexpr float kMeV = 1.f;
constexpr float kGeV = 1.e+3f;
constexpr float kGram = 6.241509704e+21f;
constexpr float kMg = 6.241509704e+18f;
constexpr float kCm3 = 1.e3f;
constexpr float kMol = 1.0f;
constexpr float kBarn = 1.e-22f;
constexpr float kAvogadro = 6.02214179e+23f;
constexpr float kElectronMassC2 = 0.510998910f;
constexpr float kAtomicMassUnit = 0.01036426891f;

struct PhysicsData {
  std::map<std::string, std::vector<char>> arrays;
  template <class T>
  const T* get(const char* name) const {
    auto it = arrays.find(name);
    return it == arrays.end() ? nullptr : reinterpret_cast<const T*>(it->second.data());
  }
  size_t count(const char* name, size_t es) const {
    auto it = arrays.find(name);
    return it == arrays.end() ? 0 : it->second.size() / es;
  }
};

bool load_physics(const char* path, PhysicsData& pd) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  char magic[8];
  f.read(magic, 8);
  if (std::memcmp(magic, "GGPHYS01", 8) != 0) return false;
  uint32_t count = 0;
  f.read(reinterpret_cast<char*>(&count), 4);
  for (uint32_t i = 0; i < count; ++i) {
    char name[32];
    uint32_t code, n;
    f.read(name, 32);
    f.read(reinterpret_cast<char*>(&code), 4);
    f.read(reinterpret_cast<char*>(&n), 4);
    size_t es = code == 2 ? 2 : code == 3 ? 1 : 4;
    std::vector<char> buf(es * n);
    f.read(buf.data(), static_cast<std::streamsize>(buf.size()));
    pd.arrays[std::string(name)] = std::move(buf);
  }
  return static_cast<bool>(f);
}

struct Element {
  uint8_t Z;
  float M;  // internal units
};
struct Material {
  float density;
  std::vector<std::string> elements;
  std::vector<float> fractions;
};

void remove_space(std::string& l) {
  for (char c : std::string("\t \n\r\f\v")) l.erase(std::remove(l.begin(), l.end(), c), l.end());
}
bool blank(const std::string& l) { return l.find_first_not_of("\t\n ") == std::string::npos; }

bool parse_database(const char* path, std::map<std::string, Material>& out) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line;
  while (std::getline(in, line)) {
    while (true) {  // GGEMSTextReader::SkipComment
      size_t pos = line.find_first_not_of("\t ");
      if (pos == std::string::npos) break;
      if (line[pos] == '#') {
        if (!std::getline(in, line)) break;
      } else {
        break;
      }
    }
    if (blank(line)) continue;
    remove_space(line);
    Material m;
    std::string name = line.substr(line.find_first_not_of("\t "), line.find(":"));
    size_t first = line.find_first_of("0123456789", line.find("d="));
    size_t last = line.find_first_not_of("0123456789.", first);
    float density = 0.0f;
    std::stringstream(line.substr(first, last - first)) >> density;
    std::string unit = line.substr(last, line.find_first_of(";") - last);
    if (unit == "g/cm3") density *= kGram / kCm3;
    else if (unit == "mg/cm3") density *= kMg / kCm3;
    else return false;
    m.density = density;
    size_t nf = line.find_first_of("0123456789", line.find("n="));
    size_t nl = line.find_last_of(";");
    size_t n = 0;
    std::stringstream(line.substr(nf, nl - nf)) >> n;
    for (size_t i = 0; i < n; ++i) {
      std::getline(in, line);
      remove_space(line);
      size_t a = line.find("name=") + 5;
      m.elements.push_back(line.substr(a, line.find_first_of(";") - a));
      size_t ff = line.find_first_of("0123456789", line.find("f="));
      float frac = 0.0f;
      std::stringstream(line.substr(ff, line.find_last_of(";") - ff)) >> frac;
      m.fractions.push_back(frac);
    }
    out.emplace(name, m);
  }
  return true;
}

float compton_per_atom(float energy, uint8_t Z) {
  float cs = 0.0f;
  if (Z < 1 || energy < 1e-4f) return cs;
  float p1Z = Z * (2.7965e-23f + 1.9756e-27f * Z + -3.9178e-29f * Z * Z);
  float p2Z = Z * (-1.8300e-23f + -1.0205e-24f * Z + 6.8241e-27f * Z * Z);
  float p3Z = Z * (6.7527e-22f + -7.3913e-24f * Z + 6.0480e-27f * Z * Z);
  float p4Z = Z * (-1.9798e-21f + 2.7079e-24f * Z + 3.0274e-26f * Z * Z);
  float T0 = (Z < 1.5f) ? 40.0e-3f : 15.0e-3f;
  float d1 = fmaxf(energy, T0) / kElectronMassC2;
  cs = p1Z * logf(1.0f + 2.0f * d1) / d1 +
       (p2Z + p3Z * d1 + p4Z * d1 * d1) / (1.0f + 20.0f * d1 + 230.0f * d1 * d1 + 440.0f * d1 * d1 * d1);
  if (energy < T0) {
    d1 = (T0 + 1.0e-3f) / kElectronMassC2;
    float d2 = p1Z * logf(1.0f + 2.0f * d1) / d1 +
               (p2Z + p3Z * d1 + p4Z * d1 * d1) / (1.0f + 20.0f * d1 + 230.0f * d1 * d1 + 440.0f * d1 * d1 * d1);
    float d3 = (-T0 * (d2 - cs)) / (cs * 1.0e-3f);
    float d4 = (Z > 1.5f) ? 0.375f - 0.0556f * logf(Z) : 0.15f;
    float d5 = logf(energy / T0);
    cs *= expf(-d5 * (d3 + d4 * d5));
  }
  return cs;
}

float photoelectric_per_atom(const PhysicsData& pd, float energy, uint8_t Z) {
  const float* ion = pd.get<float>("sandia_ionization_potentials");
  const int16_t* cum = pd.get<int16_t>("sandia_cumulative_intervals");
  const int16_t* nint = pd.get<int16_t>("sandia_number_of_intervals");
  const float* zta = pd.get<float>("sandia_z_to_a_ratio");
  const float* st = pd.get<float>("sandia_table");
  float e_min = std::fmax(ion[Z], 10.0f) * kEV;
  if (energy < e_min) return 0.0f;
  int start = cum[Z - 1];
  int stop = start + nint[Z];
  int pos = stop;
  while (energy < static_cast<float>(st[pos * 5 + 0]) * kKeV) --pos;
  float aover_avo = kAtomicMassUnit * static_cast<float>(Z) / zta[Z];
  double ei = 1.0 / static_cast<double>(energy);
  double ei2 = ei * ei;
  return static_cast<float>(ei * static_cast<double>(st[pos * 5 + 1]) * static_cast<double>(aover_avo) * 0.160217648e-22 +
                            ei2 * static_cast<double>(st[pos * 5 + 2]) * static_cast<double>(aover_avo) * 0.160217648e-25 +
                            ei * ei2 * static_cast<double>(st[pos * 5 + 3]) * static_cast<double>(aover_avo) * 0.160217648e-28 +
                            ei2 * ei2 * static_cast<double>(st[pos * 5 + 4]) * static_cast<double>(aover_avo) * 0.160217648e-31);
}

float loglog(float x, float x0, float y0, float x1, float y1) {  // GGEMSMathAlgorithms.hh:89-103 (host)
  if (x < x0) return y0;
  if (x > x1) return y1;
  x0 = 1.0f / x0;
  return std::pow(10.0f, std::log10(y0) + std::log10(y1 / y0) * (std::log10(x * x0) / std::log10(x1 * x0)));
}

float rayleigh_per_atom(const PhysicsData& pd, float energy, uint8_t Z) {
  const int32_t* cum = pd.get<int32_t>("rayleigh_cs_cumulative");
  const int32_t* nint = pd.get<int32_t>("rayleigh_cs_intervals");
  const float* cs = pd.get<float>("rayleigh_cross_section");
  if (energy < 250e-6f || energy > 100e3f) return 0.0f;
  int start = cum[Z];
  int stop = start + 2 * (nint[Z] - 1);
  int pos = start;
  for (; pos < stop; pos += 2) {
    if (cs[pos] >= static_cast<float>(energy)) break;
  }
  if (energy < 1e3f) return static_cast<float>(1.0e-22f * loglog(energy, cs[pos - 2], cs[pos - 1], cs[pos], cs[pos + 1]));
  return 1.0e-22f * cs[pos - 1];
}

// GGEMSRangeCuts::ComputePhotonCrossSection (GGEMSRangeCuts.cc:325-384)
float range_photon_cross_section(uint8_t atomic_number, float energy) {
  float t1keV = 1.0f * kKeV, t200keV = 200.f * kKeV, t100MeV = 100.f * kMeV;
  float gZ = -1.0f, s200keV = 0, s1keV = 0, tmin = 0, tlow = 0, smin = 0, slow = 0, cmin = 0, clow = 0, chigh = 0;
  if (std::abs(atomic_number - gZ) > 0.1f) {
    gZ = atomic_number;
    float const Zsq = gZ * gZ;
    float const Zlog = logf(gZ);
    float const Zlogsq = Zlog * Zlog;
    s200keV = (0.2651f - 0.1501f * Zlog + 0.02283f * Zlogsq) * Zsq;
    tmin = (0.552f + 218.5f / gZ + 557.17f / Zsq) * kMeV;
    smin = (0.01239f + 0.005585f * Zlog - 0.000923f * Zlogsq) * expf(1.5f * Zlog);
    cmin = logf(s200keV / smin) / (logf(tmin / t200keV) * logf(tmin / t200keV));
    tlow = 0.2f * expf(-7.355f / sqrtf(gZ)) * kMeV;
    slow = s200keV * expf(0.042f * gZ * logf(t200keV / tlow) * logf(t200keV / tlow));
    s1keV = 300.0f * Zsq;
    clow = logf(s1keV / slow) / logf(tlow / t1keV);
    chigh = (7.55e-5f - 0.0542e-5f * gZ) * Zsq * gZ / logf(t100MeV / tmin);
  }
  float xs = 0.0f;
  if (energy < tlow) {
    if (energy < t1keV) xs = slow * expf(clow * logf(tlow / t1keV));
    else xs = slow * expf(clow * logf(tlow / energy));
  } else if (energy < t200keV) {
    xs = s200keV * expf(0.042f * gZ * logf(t200keV / energy) * logf(t200keV / energy));
  } else if (energy < tmin) {
    xs = smin * expf(cmin * logf(tmin / energy) * logf(tmin / energy));
  } else {
    xs = smin + chigh * logf(energy / tmin);
  }
  return xs * kBarn;
}

// GGEMSLogEnergyTable (src/physics/GGEMSLogEnergyTable.cc:40-161)
struct LogTable {
  float bin_width, base_bin, edge_min, edge_max;
  size_t nodes;
  std::vector<float> data, bins;
  LogTable(float low, float high, size_t n) {
    bin_width = logf(high / low) / static_cast<float>(n);
    base_bin = logf(low) / bin_width;
    nodes = n + 1;
    data.assign(nodes, 0.0f);
    bins.resize(nodes);
    bins[0] = low;
    for (size_t i = 1; i < nodes - 1; ++i) bins[i] = expf((base_bin + static_cast<float>(i)) * bin_width);
    bins[nodes - 1] = high;
    edge_min = bins.front();
    edge_max = bins.back();
  }
  size_t find_bin_location(float e) const {
    size_t bin = static_cast<size_t>(logf(e) / bin_width - base_bin);
    if (bin + 2 > nodes) bin = nodes - 2;
    else if (bin > 0 && e < bins[bin]) --bin;
    else if (bin + 2 < nodes && e > bins[bin + 1]) ++bin;
    return bin;
  }
  size_t find_bin(float e, size_t index) const {
    size_t id = index;
    if (e < bins[1]) id = 0;
    else if (e >= bins[nodes - 2]) id = nodes - 2;
    else if (index >= nodes || e < bins[index] || e > bins[index + 1]) id = find_bin_location(e);
    return id;
  }
  float value(float e) const {
    if (e <= edge_min) return data[0];
    if (e >= edge_max) return data[nodes - 1];
    size_t li = find_bin(e, 0);
    float xa = bins[li], ya = data[li], xb = bins[li + 1], yb = data[li + 1];
    if (xa > xb) return yb;
    if (xa >= e) return ya;
    if (xb <= e) return yb;
    return ya + (e - xa) * (yb - ya) / (xb - xa);
  }
};

// Photon branch of GGEMSRangeCuts::ConvertToEnergy (GGEMSRangeCuts.cc:129-208, 214-232, 544-590).
float photon_energy_cut(const std::vector<uint8_t>& Z, const std::vector<float>& density, float cut, float min_energy) {
  const float max_energy = 10.0f * kGeV;
  const size_t nbins = 300;
  std::vector<LogTable> elems;
  for (size_t i = 0; i < Z.size(); ++i) {
    LogTable t(min_energy, max_energy, nbins);
    for (size_t j = 0; j < nbins; ++j) t.data[j] = range_photon_cross_section(Z[i], t.bins[j]);
    elems.push_back(t);
  }
  LogTable range(min_energy, max_energy, nbins);
  for (size_t i = 0; i < nbins; ++i) {
    float sigma = 0.0f;
    for (size_t j = 0; j < Z.size(); ++j) sigma += density[j] * elems[j].data[i];
    range.data[i] = 5.0f / sigma;
  }
  // ConvertLengthToEnergyCut (GGEMSRangeCuts.cc:544-590)
  float epsilon = 0.01f, rmax = -1.e10f, t1 = min_energy, r1 = range.data[0], t2 = max_energy;
  float kinetic;
  if (cut < r1) {
    kinetic = t1;
  } else {
    for (size_t i = 0; i < nbins; ++i) {
      float t = range.bins[i], r = range.data[i];
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

// LinearInterpolation (GGEMSMathAlgorithms.hh:76-86).
float lerp(float xa, float ya, float xb, float yb, float x) {
  if (xa > xb) return yb;
  if (xa >= x) return ya;
  if (xb <= x) return yb;
  return ya + (x - xa) * (yb - ya) / (xb - xa);
}

}  // namespace

extern "C" {

// Build one navigator's tables for `material_names` (in label order).
// Outputs are caller-allocated: energy_bins[nbins], cross_sections[3*nmat*nbins],
// rayleigh_per_atom[101*nbins], density/photon_cut/n_elements/element_offset[nmat],
// atomic_number/atomic_number_density[sum of elements].
__attribute__((visibility("default"))) int gg_oracle_build_tables(
    const char* materials_file, const char* physics_file, const char* const* material_names, int n_materials,
    int number_of_bins, float min_energy, float max_energy, const int* process_ids, int n_processes,
    float photon_distance_cut, float* energy_bins, float* cross_sections, float* rayleigh, float* density,
    float* photon_cut, int32_t* n_elements, int32_t* element_offset, uint8_t* atomic_number,
    float* atomic_number_density, int32_t* total_elements) {
  PhysicsData pd;
  if (!load_physics(physics_file, pd)) return GG_ERROR_INVALID_ARGUMENT;
  std::map<std::string, Material> db;
  if (!parse_database(materials_file, db)) return GG_ERROR_INVALID_ARGUMENT;
  std::map<std::string, Element> elements;
  const char* names = pd.get<char>("element_names");
  const uint8_t* ez = pd.get<uint8_t>("element_z");
  const float* em = pd.get<float>("element_molar_mass");
  size_t ne = pd.count("element_z", 1);
  for (size_t i = 0; i < ne; ++i) elements[std::string(names + 16 * i)] = Element{ez[i], em[i] * (kGram / kMol)};

  int offset = 0;
  for (int i = 0; i < n_materials; ++i) {
    auto it = db.find(material_names[i]);
    if (it == db.end()) return GG_ERROR_INVALID_ARGUMENT;
    const Material& m = it->second;
    n_elements[i] = static_cast<int32_t>(m.elements.size());
    element_offset[i] = offset;
    density[i] = m.density;
    std::vector<uint8_t> zs;
    std::vector<float> dens;
    for (size_t j = 0; j < m.elements.size(); ++j) {
      const Element& e = elements.at(m.elements[j]);
      atomic_number[offset + j] = e.Z;
      double v = static_cast<double>(kAvogadro) / static_cast<double>(e.M) * static_cast<double>(m.density) *
                 static_cast<double>(m.fractions[j]);
      atomic_number_density[offset + j] = static_cast<float>(v);
      zs.push_back(e.Z);
      dens.push_back(static_cast<float>(v));
    }
    photon_cut[i] = photon_energy_cut(zs, dens, photon_distance_cut, min_energy);
    offset += n_elements[i];
  }
  *total_elements = offset;

  float slope = logf(max_energy / min_energy);
  for (int i = 0; i < number_of_bins; ++i)
    energy_bins[i] = min_energy * expf(slope * (static_cast<float>(i) / (static_cast<float>(number_of_bins) - 1.0f))) * kMeV;

  const size_t block = static_cast<size_t>(n_materials) * number_of_bins;
  std::fill(cross_sections, cross_sections + 3 * block, 0.0f);
  std::fill(rayleigh, rayleigh + static_cast<size_t>(101) * number_of_bins, 0.0f);
  for (int p = 0; p < n_processes; ++p) {
    int pid = process_ids[p];
    for (int j = 0; j < n_materials; ++j) {
      for (int i = 0; i < number_of_bins; ++i) {
        float energy = energy_bins[i];
        float sum = 0.0f;
        for (int k = 0; k < n_elements[j]; ++k) {
          uint8_t Z = atomic_number[element_offset[j] + k];
          float per_atom = pid == GG_COMPTON_SCATTERING ? compton_per_atom(energy, Z)
                           : pid == GG_PHOTOELECTRIC_EFFECT ? photoelectric_per_atom(pd, energy, Z)
                                                            : rayleigh_per_atom(pd, energy, Z);
          if (pid == GG_RAYLEIGH_SCATTERING) rayleigh[i + Z * number_of_bins] = per_atom;
          sum += atomic_number_density[element_offset[j] + k] * per_atom;
        }
        cross_sections[pid * block + i + static_cast<size_t>(j) * number_of_bins] = sum;
      }
    }
  }
  return GG_OK;
}

// GGEMSAttenuations::GGEMSAttenuations + Initialize (src/physics/GGEMSAttenuations.cc:40-82,
// 142-230): mu and mu_en per material on 220 log-spaced bins (1 keV - 1 MeV),
// mixing the per-element tables of GGEMSMuDataConstants by mass fraction.
// Reproduced as written, including two details: the energy index is searched
// from the start of the concatenated element table up to the end of element
// Z's rows, and a hit on an element's first row adds that row unweighted by
// the mass fraction.  Outputs: energy_bins[220], mu/mu_en[n_materials*220]
// (cm^-1, [bin + 220*material]).
__attribute__((visibility("default"))) int gg_oracle_build_attenuations(
    const char* materials_file, const char* physics_file, const char* const* material_names, int n_materials,
    float* energy_bins, float* mu, float* mu_en) {
  PhysicsData pd;
  if (!load_physics(physics_file, pd)) return GG_ERROR_INVALID_ARGUMENT;
  std::map<std::string, Material> db;
  if (!parse_database(materials_file, db)) return GG_ERROR_INVALID_ARGUMENT;
  const char* names = pd.get<char>("element_names");
  const uint8_t* ez = pd.get<uint8_t>("element_z");
  size_t ne = pd.count("element_z", 1);
  std::map<std::string, uint8_t> z_of;
  for (size_t i = 0; i < ne; ++i) z_of[std::string(names + 16 * i)] = ez[i];
  const int32_t* nb_bins = pd.get<int32_t>("mu_nb_energy_bins");
  const int32_t* index_energy = pd.get<int32_t>("mu_index_energy");
  const float* data = pd.get<float>("mu_data");
  const int n_elem_tables = 92;  // kMuNbElements
  std::vector<float> energies, mu_t, mu_en_t;
  size_t index_data = 0;
  for (int i = 0; i <= n_elem_tables; ++i) {
    for (int j = 0; j < nb_bins[i]; ++j) {
      energies.push_back(data[index_data++]);
      mu_t.push_back(data[index_data++]);
      mu_en_t.push_back(data[index_data++]);
    }
  }
  constexpr int kBins = GG_ATTENUATION_BINS;
  const float emin = 0.001f, emax = 1.0f;
  float slope = logf(emax / emin);
  for (int i = 0; i < kBins; ++i)
    energy_bins[i] = emin * expf(slope * (static_cast<float>(i) / (static_cast<float>(kBins) - 1.0f))) * kMeV;
  for (int m = 0; m < n_materials; ++m) {
    auto it = db.find(material_names[m]);
    if (it == db.end()) return GG_ERROR_INVALID_ARGUMENT;
    const Material& mat = it->second;
    for (int i = 0; i < kBins; ++i) {
      const float energy = energy_bins[i];
      float mu_over_rho = 0.0f, mu_en_over_rho = 0.0f;
      for (size_t k = 0; k < mat.elements.size(); ++k) {
        const int Z = z_of.at(mat.elements[k]);
        if (Z > n_elem_tables) continue;  // no mu data beyond Z = 92 (GGEMS reads past its table)
        const float frac = mat.fractions[k];
        const int first = index_energy[Z];
        int low = 0, high = first + nb_bins[Z] - 1;  // BinarySearch (GGEMSMathAlgorithms.hh:46-63)
        int e_index = 0;
        bool found = false;
        while (high - low > 1) {
          int mid = (high + low) / 2;
          if (energies[mid] == energy) {
            e_index = mid;
            found = true;
            break;
          }
          if (energies[mid] < energy) low = mid;
          else high = mid;
        }
        if (!found) e_index = low;
        if (e_index == first) {
          mu_over_rho += mu_t[e_index];
          mu_en_over_rho += mu_en_t[e_index];
        } else if (e_index == 0) {
          // the reference reads the row before its table here; LinearInterpolation
          // then returns row 0's value (x >= its energy)
          mu_over_rho += frac * mu_t[0];
          mu_en_over_rho += frac * mu_en_t[0];
        } else {
          mu_over_rho += frac * lerp(energies[e_index - 1], mu_t[e_index - 1], energies[e_index], mu_t[e_index], energy);
          mu_en_over_rho +=
              frac * lerp(energies[e_index - 1], mu_en_t[e_index - 1], energies[e_index], mu_en_t[e_index], energy);
        }
      }
      mu[m * kBins + i] = mu_over_rho * mat.density / (kGram / kCm3);
      mu_en[m * kBins + i] = mu_en_over_rho * mat.density / (kGram / kCm3);
    }
  }
  return GG_OK;
}

}  // extern "C"
