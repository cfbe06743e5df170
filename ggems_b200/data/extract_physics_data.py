"""Generate ``physics_data.bin``: the physics data tables the photon path needs,
taken from a GGEMS v1.3 checkout so that every value is bit-identical to the
one the reference's own build uses.

The tables are published physics data, not algorithms:

* Sandia photo-absorption fit coefficients, ionisation potentials and Z/A
  ratios (``include/GGEMS/physics/GGEMSSandiaTable.hh:40-1511``), used by the
  photoelectric per-atom cross section (``src/physics/GGEMSPhotoElectricEffect.cc:76-98``);
* Livermore Rayleigh per-atom cross-section table
  (``include/GGEMS/physics/GGEMSRayleighScattering.hh:98-21644``), used by
  ``src/physics/GGEMSRayleighScattering.cc:80-102``;
* the Rayleigh form-factor fit parameters PP0-PP8
  (``include/GGEMS/physics/GGEMSRayleighScatteringModels.hh:36-153``), used by
  the angular sampler;
* the per-element mu/mu_en table (``include/GGEMS/physics/GGEMSMuDataConstants.hh``);
* the chemical element list (name, Z, molar mass, mean excitation energy,
  state) registered by ``src/materials/GGEMSMaterialsDatabaseManager.cc:338-437``.

Decimal-to-float conversion is done by g++ (the same compiler family the
reference is built with), not by Python, so no value can be double-rounded
differently: this script cuts the initialiser text out of the headers, wraps it
into a small C++ program, compiles and runs it.

Usage:  python ggems_b200/data/extract_physics_data.py [reference_checkout]
"""

import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "physics_data.bin")

# (name in the binary, header file, array name in the header, C type)
ARRAYS = [
    ("sandia_ionization_potentials", "include/GGEMS/physics/GGEMSSandiaTable.hh", "kIonizationPotentials", "float"),
    ("sandia_number_of_intervals", "include/GGEMS/physics/GGEMSSandiaTable.hh", "kNumberOfIntervals", "short"),
    ("sandia_cumulative_intervals", "include/GGEMS/physics/GGEMSSandiaTable.hh", "kCumulativeIntervals", "short"),
    ("sandia_z_to_a_ratio", "include/GGEMS/physics/GGEMSSandiaTable.hh", "kZtoARatio", "float"),
    ("sandia_table", "include/GGEMS/physics/GGEMSSandiaTable.hh", "kSandiaTable", "float"),
    ("rayleigh_cs_cumulative", "include/GGEMS/physics/GGEMSRayleighScattering.hh", "kCrossSectionCumulativeIntervals", "int"),
    ("rayleigh_cs_intervals", "include/GGEMS/physics/GGEMSRayleighScattering.hh", "kCrossSectionNumberOfIntervals", "int"),
    ("rayleigh_cross_section", "include/GGEMS/physics/GGEMSRayleighScattering.hh", "kCrossSection", "float"),
    ("mu_nb_energy_bins", "include/GGEMS/physics/GGEMSMuDataConstants.hh", "kMuNbEnergyBins", "int"),
    ("mu_index_energy", "include/GGEMS/physics/GGEMSMuDataConstants.hh", "kMuIndexEnergy", "int"),
    ("mu_data", "include/GGEMS/physics/GGEMSMuDataConstants.hh", "kMuData", "float"),
] + [
    ("rayleigh_pp%d" % i, "include/GGEMS/physics/GGEMSRayleighScatteringModels.hh", "PP%d" % i, "float")
    for i in range(9)
]

DTYPE_CODE = {"float": 0, "int": 1, "short": 2, "uchar": 3}


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def initializer(ref, header, array):
    with open(os.path.join(ref, header)) as f:
        text = strip_comments(f.read())
    m = re.search(r"\b" + re.escape(array) + r"\s*((?:\[\s*\d+\s*\])+)\s*=\s*\{", text)
    if not m:
        raise RuntimeError("array %s not found in %s" % (array, header))
    dims = [int(d) for d in re.findall(r"\d+", m.group(1))]
    depth, i = 1, m.end()
    while depth:
        depth += {"{": 1, "}": -1}.get(text[i], 0)
        i += 1
    return dims, text[m.end() - 1:i]


def elements(ref):
    path = os.path.join(ref, "src/materials/GGEMSMaterialsDatabaseManager.cc")
    with open(path) as f:
        text = strip_comments(f.read())
    pat = re.compile(r'AddChemicalElements\(\s*"(\w+)"\s*,\s*(\d+)\s*,\s*([-+0-9.eE]+f?)\s*,\s*([-+0-9.eE]+f?)\s*,\s*(GAS|SOLID)\s*,\s*(-?\d+)\s*\)')
    out = pat.findall(text)
    if len(out) < 90:
        raise RuntimeError("chemical element list not found")
    return out


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GGEMS_REFERENCE_DIR", "/root/reference")
    lines = ["#include <cstdio>", "#include <cstring>", "#include <cstdint>",
             "static void put(FILE* f, const char* name, unsigned code, unsigned n, const void* p, unsigned es) {",
             "  char nm[32]; std::memset(nm, 0, 32); std::strncpy(nm, name, 31); std::fwrite(nm, 1, 32, f);",
             "  std::fwrite(&code, 4, 1, f); std::fwrite(&n, 4, 1, f); std::fwrite(p, es, n, f); }"]
    for name, header, array, ctype in ARRAYS:
        dims, init = initializer(ref, header, array)
        lines.append("static const %s %s%s = %s;" % (ctype, name, "".join("[%d]" % d for d in dims), init))
    els = elements(ref)
    lines.append("static const char element_names[%d][16] = {%s};" % (len(els), ",".join('"%s"' % e[0] for e in els)))
    lines.append("static const unsigned char element_z[%d] = {%s};" % (len(els), ",".join(e[1] for e in els)))
    lines.append("static const float element_molar_mass[%d] = {%s};" % (len(els), ",".join(e[2] for e in els)))
    lines.append("static const float element_mean_excitation[%d] = {%s};" % (len(els), ",".join(e[3] for e in els)))
    lines.append("static const int element_state[%d] = {%s};" % (len(els), ",".join("1" if e[4] == "GAS" else "0" for e in els)))
    lines.append("static const int element_density_correction[%d] = {%s};" % (len(els), ",".join(e[5] for e in els)))
    body = ["int main(int argc, char** argv) {", "  FILE* f = std::fopen(argv[1], \"wb\");",
            "  std::fwrite(\"GGPHYS01\", 1, 8, f);", "  unsigned count = %d; std::fwrite(&count, 4, 1, f);" % (len(ARRAYS) + 6)]
    sizes = {"float": 4, "int": 4, "short": 2, "uchar": 1}
    for name, _, _, ctype in ARRAYS:
        body.append('  put(f, "%s", %d, sizeof(%s)/%d, %s, %d);' % (name, DTYPE_CODE[ctype], name, sizes[ctype], name, sizes[ctype]))
    body.append('  put(f, "element_names", 3, sizeof(element_names), element_names, 1);')
    body.append('  put(f, "element_z", 3, sizeof(element_z), element_z, 1);')
    body.append('  put(f, "element_molar_mass", 0, sizeof(element_molar_mass)/4, element_molar_mass, 4);')
    body.append('  put(f, "element_mean_excitation", 0, sizeof(element_mean_excitation)/4, element_mean_excitation, 4);')
    body.append('  put(f, "element_state", 1, sizeof(element_state)/4, element_state, 4);')
    body.append('  put(f, "element_density_correction", 1, sizeof(element_density_correction)/4, element_density_correction, 4);')
    body += ["  std::fclose(f);", "  return 0;", "}"]
    with tempfile.TemporaryDirectory() as tmp:
        src = os.path.join(tmp, "gen.cc")
        exe = os.path.join(tmp, "gen")
        with open(src, "w") as f:
            f.write("\n".join(lines + body) + "\n")
        subprocess.check_call(["g++", "-std=c++17", "-O0", "-w", src, "-o", exe])
        subprocess.check_call([exe, OUT])
    print("wrote", OUT, os.path.getsize(OUT), "bytes,", len(els), "elements")


if __name__ == "__main__":
    main()
