// Host utilities for the GGEMS-compatible API (see gg_host.hh).
#include "gg_host.hh"

#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <mutex>
#include <sstream>

namespace gg {

namespace {
thread_local std::string t_last_error;
int g_verbosity = 0;
}  // namespace

Error::Error(const std::string& cls, const std::string& method, const std::string& msg)
    : std::runtime_error("[GGEMS " + cls + "::" + method + "] EXCEPTION!!! " + msg) {}

void set_last_error(const std::string& msg) { t_last_error = msg; }
const char* last_error() { return t_last_error.c_str(); }
void clear_last_error() { t_last_error.clear(); }
int verbosity() { return g_verbosity; }
void set_verbosity(int v) { g_verbosity = v; }

// Unit conversions: GGEMSSystemOfUnits.hh:245-418 (value * unit, in float).
float distance_unit(float v, const std::string& u) {
  if (u == "nm") return v * units::nm;
  if (u == "um") return v * units::um;
  if (u == "mm") return v * units::mm;
  if (u == "cm") return v * units::cm;
  if (u == "m") return v * units::m;
  if (u == "km") return v * units::km;
  if (u == "pc") return v * units::pc;
  throw Error("", "DistanceUnit", "Unknown unit!!! You have choice between: nm, um, mm, cm, m, km, pc");
}
float energy_unit(float v, const std::string& u) {
  if (u == "eV") return v * units::eV;
  if (u == "keV") return v * units::keV;
  if (u == "MeV") return v * units::MeV;
  if (u == "GeV") return v * units::GeV;
  if (u == "TeV") return v * units::TeV;
  if (u == "PeV") return v * units::PeV;
  throw Error("", "EnergyUnit", "Unknown unit!!! You have choice between: eV, keV, MeV, GeV, TeV, PeV");
}
float angle_unit(float v, const std::string& u) {
  if (u == "rad") return v * units::rad;
  if (u == "mrad") return v * units::mrad;
  if (u == "deg") return v * units::deg;
  if (u == "sr") return v * units::sr;
  throw Error("", "AngleUnit", "Unknown unit!!! You have choice between: rad, mrad, deg, sr");
}
float density_unit(float v, const std::string& u) {
  if (u == "g/cm3") return v * units::g / units::cm3;
  if (u == "kg/m3") return v * units::kg / units::m3;
  if (u == "mg/cm3") return v * units::mg / units::cm3;
  throw Error("", "DensityUnit", "Unknown unit!!! You have choice between: g/cm3, kg/m3, mg/cm3");
}

size_t PhysicsData::count(const std::string& name, size_t es) const {
  auto it = arrays.find(name);
  return it == arrays.end() ? 0 : it->second.size() / es;
}

std::string data_directory() {
  if (const char* env = std::getenv("GGEMS_B200_DATA")) return std::string(env) + "/";
  Dl_info info;
  if (dladdr(reinterpret_cast<void*>(&data_directory), &info) && info.dli_fname) {
    // the library's own directory, not that of a link to it (GGEMS's Python
    // module loads libggems.so from beside the module, often a link)
    char resolved[PATH_MAX];
    std::string lib(realpath(info.dli_fname, resolved) ? resolved : info.dli_fname);
    size_t pos = lib.find_last_of('/');
    return (pos == std::string::npos ? std::string("./") : lib.substr(0, pos + 1)) + "data/";
  }
  return "data/";
}

const PhysicsData& physics_data() {
  static std::once_flag once;
  static std::unique_ptr<PhysicsData> pd;
  static std::string error;
  std::call_once(once, []() {
    auto d = std::make_unique<PhysicsData>();
    std::string path = data_directory() + "physics_data.bin";
    std::ifstream f(path, std::ios::binary);
    char magic[8] = {0};
    f.read(magic, 8);
    if (!f || std::memcmp(magic, "GGPHYS01", 8) != 0) {
      error = "cannot read physics data file " + path;
      return;
    }
    uint32_t count = 0;
    f.read(reinterpret_cast<char*>(&count), 4);
    for (uint32_t i = 0; i < count && f; ++i) {
      char name[32];
      uint32_t code = 0, n = 0;
      f.read(name, 32);
      f.read(reinterpret_cast<char*>(&code), 4);
      f.read(reinterpret_cast<char*>(&n), 4);
      size_t es = code == 2 ? 2 : code == 3 ? 1 : 4;
      std::vector<char> buf(es * n);
      f.read(buf.data(), static_cast<std::streamsize>(buf.size()));
      name[31] = 0;
      d->arrays[name] = std::move(buf);
    }
    if (!f) {
      error = "truncated physics data file " + path;
      return;
    }
    pd = std::move(d);
  });
  if (!pd) throw Error("PhysicsData", "Load", error);
  return *pd;
}

// GGEMSTextReader (src/io/GGEMSTextReader.cc:150-185)
void skip_comment(std::istream& in, std::string& line, char comment) {
  while (true) {
    size_t pos = line.find_first_not_of("\t ");
    if (pos == std::string::npos) break;
    if (line[pos] == comment) {
      if (!std::getline(in, line)) {
        line.clear();
        break;
      }
    } else {
      break;
    }
  }
}
bool is_blank(const std::string& line) { return line.find_first_not_of("\t\n ") == std::string::npos; }
void remove_space(std::string& line) {
  for (char c : std::string("\t \n\r\f\v")) line.erase(std::remove(line.begin(), line.end(), c), line.end());
}

// GGEMSMHDImage::Read (src/io/GGEMSMHDImage.cc:129-217)
MHDHeader read_mhd(const std::string& header) {
  std::ifstream in(header);
  if (!in) throw Error("GGEMSFileStream", "CheckInputStream", "Problem reading filename: " + header);
  MHDHeader h;
  size_t dir = header.find_last_of("/\\");
  if (dir != std::string::npos) h.directory = header.substr(0, dir + 1);
  std::string line;
  while (std::getline(in, line)) {
    skip_comment(in, line);
    if (is_blank(line)) continue;
    size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string key = line.substr(line.find_first_not_of("\t "), eq - 1);
    remove_space(key);
    std::istringstream iss(line.substr(eq + 1));
    if (key == "DimSize") iss >> h.dim[0] >> h.dim[1] >> h.dim[2];
    else if (key == "ElementSpacing") iss >> h.spacing[0] >> h.spacing[1] >> h.spacing[2];
    else if (key == "ElementType") iss >> h.type;
    else if (key == "ElementDataFile") iss >> h.raw_file;
  }
  if (h.dim[0] <= 0 || h.dim[1] <= 0 || h.dim[2] <= 0)
    throw Error("GGEMSMHDImage", "Read", "Dimension invalid for the key 'DimSize'!!! The values have to be > 0");
  if (h.spacing[0] == 0.0f || h.spacing[1] == 0.0f || h.spacing[2] == 0.0f)
    throw Error("GGEMSMHDImage", "Read", "Voxel size invalid for the key 'ElementSpacing'!!! The values have to be > 0");
  if (h.raw_file.empty())
    throw Error("GGEMSMHDImage", "Read", "Value invalid for the key 'ElementDataFile'!!! A filename for raw data has to be given");
  return h;
}

namespace {
template <class T>
std::vector<float> read_raw_as_float(const std::string& path, size_t n) {
  std::ifstream in(path, std::ios::binary);
  if (!in) throw Error("GGEMSFileStream", "CheckInputStream", "Problem reading filename: " + path);
  std::vector<T> raw(n);
  in.read(reinterpret_cast<char*>(raw.data()), static_cast<std::streamsize>(n * sizeof(T)));
  if (!in) throw Error("GGEMSMHDImage", "Read", "raw file too short: " + path);
  std::vector<float> out(n);
  for (size_t i = 0; i < n; ++i) out[i] = static_cast<float>(raw[i]);
  return out;
}
}  // namespace

std::vector<float> read_mhd_values(const MHDHeader& h) {
  const size_t n = static_cast<size_t>(h.dim[0]) * h.dim[1] * h.dim[2];
  const std::string path = h.directory + h.raw_file;
  if (h.type == "MET_CHAR") return read_raw_as_float<int8_t>(path, n);
  if (h.type == "MET_UCHAR") return read_raw_as_float<uint8_t>(path, n);
  if (h.type == "MET_SHORT") return read_raw_as_float<int16_t>(path, n);
  if (h.type == "MET_USHORT") return read_raw_as_float<uint16_t>(path, n);
  if (h.type == "MET_INT") return read_raw_as_float<int32_t>(path, n);
  if (h.type == "MET_UINT") return read_raw_as_float<uint32_t>(path, n);
  if (h.type == "MET_FLOAT") return read_raw_as_float<float>(path, n);
  throw Error("GGEMSMHDImage", "Read", "Value invalid for the key 'ElementType'!!! (" + h.type + ")");
}

// GGEMSMHDImage::Write (src/io/GGEMSMHDImage.cc:223-255)
void write_mhd(const std::string& header, const std::string& type, const int32_t dim[3], const float spacing[3],
               const void* data, size_t element_size) {
  std::string base = header;
  size_t dot = base.find_last_of('.');
  if (dot != std::string::npos && base.substr(dot) == ".mhd") base = base.substr(0, dot);
  std::string raw = base + ".raw";
  std::string raw_name = raw.substr(raw.find_last_of("/\\") == std::string::npos ? 0 : raw.find_last_of("/\\") + 1);
  std::ofstream out(base + ".mhd");
  if (!out) throw Error("GGEMSMHDImage", "Write", "cannot write " + base + ".mhd");
  out << "ObjectType = Image\n";
  out << "BinaryDataByteOrderMSB = False\n";
  out << "NDims = 3\n";
  out << "ElementSpacing = " << spacing[0] << " " << spacing[1] << " " << spacing[2] << "\n";
  out << "DimSize = " << dim[0] << " " << dim[1] << " " << dim[2] << "\n";
  out << "ElementType = " << type << "\n";
  out << "ElementDataFile = " << raw_name << "\n";
  std::ofstream r(raw, std::ios::binary);
  r.write(static_cast<const char*>(data),
          static_cast<std::streamsize>(static_cast<size_t>(dim[0]) * dim[1] * dim[2] * element_size));
}

}  // namespace gg
