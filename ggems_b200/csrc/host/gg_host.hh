// Host-side support for the GGEMS-compatible C++ API: units, errors, physics
// data, text readers and MHD images.
#ifndef GG_HOST_HH
#define GG_HOST_HH

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace gg {

// ---- units (include/GGEMS/tools/GGEMSSystemOfUnits.hh), float arithmetic ----
namespace units {
constexpr float nm = 1.e-6f, um = 1.e-3f, mm = 1.0f, cm = 10.f, m = 1.e3f, km = 1.e6f, pc = 3.0856775807e+19f;
constexpr float cm3 = 1.e3f, m3 = 1.e9f;
constexpr float rad = 1.0f, mrad = 1.e-3f, deg = 3.141592653589793238463f / 180.0f, sr = 1.0f;
constexpr float eV = 1.e-6f, keV = 1.e-3f, MeV = 1.f, GeV = 1.e+3f, TeV = 1.e+6f, PeV = 1.e+9f;
constexpr float kg = 6.241509704e+24f, g = 6.241509704e+21f, mg = 6.241509704e+18f, mol = 1.0f;
constexpr float Gy = 1.0e-12f;
constexpr float barn = 1.e-22f;
}  // namespace units

float distance_unit(float v, const std::string& unit);
float energy_unit(float v, const std::string& unit);
float angle_unit(float v, const std::string& unit);
float density_unit(float v, const std::string& unit);

// Errors are reported the way GGEMSMisc::ThrowException formats them
// (class, method, message); the C ABI catches them and records the text.
struct Error : std::runtime_error {
  Error(const std::string& cls, const std::string& method, const std::string& msg);
};
void set_last_error(const std::string& msg);
const char* last_error();
void clear_last_error();
int verbosity();
void set_verbosity(int v);

// ---- physics data (ggems_b200/data/physics_data.bin) ----
struct PhysicsData {
  std::map<std::string, std::vector<char>> arrays;
  template <class T>
  const T* get(const std::string& name) const {
    auto it = arrays.find(name);
    if (it == arrays.end()) throw Error("PhysicsData", "get", "missing array " + name);
    return reinterpret_cast<const T*>(it->second.data());
  }
  size_t count(const std::string& name, size_t es) const;
};
const PhysicsData& physics_data();
std::string data_directory();

// ---- text readers (src/io/GGEMSTextReader.cc) ----
void skip_comment(std::istream& in, std::string& line, char comment = '#');
bool is_blank(const std::string& line);
void remove_space(std::string& line);

// ---- MHD image (src/io/GGEMSMHDImage.cc) ----
struct MHDHeader {
  int32_t dim[3] = {0, 0, 0};
  float spacing[3] = {0.f, 0.f, 0.f};
  std::string type;
  std::string raw_file;   // as written in the header
  std::string directory;  // directory of the header, with trailing separator
};
MHDHeader read_mhd(const std::string& header);
// Reads the raw voxels as float values (the conversion ConvertImageToLabel applies).
std::vector<float> read_mhd_values(const MHDHeader& h);
void write_mhd(const std::string& header, const std::string& type, const int32_t dim[3], const float spacing[3],
               const void* data, size_t element_size);

}  // namespace gg

#endif
