"""GGEMS's C++ classes (include/ggems.hh) over libggems.so, without a GPU.

The header declares the extern "C" functions itself with void* handles (it
cannot include ggems_api.h, whose opaque C types carry the GGEMS class names),
so every declaration is checked against ggems_api.h: same name, same argument
types once the opaque handle pointers are read as void*.  Then a C++ program
written the way a GGEMS C++ example is (GGEMS v1.3 examples/*/main.cc: managers
by GetInstance(), sources and navigators by name, SetXxx with units) is
compiled against the header, linked with libggems.so and run: the CBCT
configuration must be accepted, and a bad unit or an unknown data type must
raise std::runtime_error with GGEMS's message.
"""

import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIB = os.path.join(ROOT, "ggems_b200")

_HANDLES = {"GGEMS", "GGEMSXRaySource", "GGEMSVoxelizedSource", "GGEMSVoxelizedPhantom", "GGEMSMeshedPhantom",
            "GGEMSCTSystem", "GGEMSWorld", "GGEMSVolumeCreatorManager", "GGEMSBox", "GGEMSTube", "GGEMSSphere",
            "GGEMSDosimetryCalculator"}


def _strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def _normal_type(t):
    t = re.sub(r"\s+", " ", t.strip())
    t = re.sub(r"\s*\*\s*", "*", t)
    m = re.fullmatch(r"(\w+)\*", t)
    if m and m.group(1) in _HANDLES:
        return "void*"
    return {"size_t": "size_t", "std::size_t": "size_t"}.get(t, t)


def _param_type(p):
    p = p.strip()
    if p in ("", "void"):
        return None
    m = re.fullmatch(r"(.*?[\s\*])(\w+)", p)
    if m and m.group(2) not in ("int", "bool", "float", "char", "void", "double", "size_t") \
            and not m.group(2).endswith("_t"):
        p = m.group(1)
    return _normal_type(p)


def _prototypes(text):
    out = {}
    for ret, name, params in re.findall(r"([\w\s\*]+?)\b(\w+)\s*\(([^()]*)\)\s*;", _strip_comments(text)):
        types = [_param_type(p) for p in params.split(",")]
        out[name] = (_normal_type(ret), tuple(t for t in types if t is not None))
    return out


def test_facade_declarations_match_c_abi():
    api = _prototypes(open(os.path.join(INC, "ggems_api.h")).read())
    hh = open(os.path.join(INC, "ggems.hh")).read()
    block = hh[hh.index('extern "C" {'):hh.index("// Throws the message")]
    mine = _prototypes(block)
    assert len(mine) >= 130
    for name, sig in mine.items():
        assert name in api, name
        assert sig == api[name], (name, sig, api[name])


PROGRAM = r'''
#include "ggems.hh"
#include <cstdio>
#include <cstring>

int main(int argc, char** argv) {
  std::string dir = argv[1];
  GGEMSVerbosity(0);
  GGEMSMaterialsDatabaseManager::GetInstance().SetMaterialsDatabase(argv[2]);
  GGEMSVoxelizedPhantom phantom("phantom");
  phantom.SetPhantomFile(argv[3], argv[4]);
  phantom.SetRotation(0.0f, 0.0f, 0.0f, "deg");
  phantom.SetPosition(0.0f, 0.0f, 0.0f, "mm");
  GGEMSCTSystem ct("flat_panel");
  ct.SetCTSystemType("flat");
  ct.SetNumberOfModules(1, 1);
  ct.SetNumberOfDetectionElementsInsideModule(64, 64, 1);
  ct.SetSizeOfDetectionElements(4.0f, 4.0f, 10.0f, "mm");
  ct.SetMaterialName("GOS");
  ct.SetSourceDetectorDistance(1500.0f, "mm");
  ct.SetSourceIsocenterDistance(1000.0f, "mm");
  ct.SetRotation(0.0f, 0.0f, 0.0f, "deg");
  ct.SetThreshold(10.0f, "keV");
  ct.StoreOutput(dir + "/projection");
  ct.StoreScatter(true);
  GGEMSProcessesManager& pm = GGEMSProcessesManager::GetInstance();
  pm.AddProcess("Compton", "gamma", "all");
  pm.AddProcess("Photoelectric", "gamma", "all");
  pm.AddProcess("Rayleigh", "gamma", "all");
  pm.SetCrossSectionTableNumberOfBins(220);
  pm.SetCrossSectionTableMinimumEnergy(1.0f, "keV");
  pm.SetCrossSectionTableMaximumEnergy(1.0f, "MeV");
  GGEMSRangeCutsManager::GetInstance().SetLengthCut("all", "gamma", 0.1f, "mm");
  GGEMSXRaySource xray("xray");
  xray.SetSourceParticleType("gamma");
  xray.SetNumberOfParticles(1000);
  xray.SetPosition(-1000.0f, 0.0f, 0.0f, "mm");
  xray.SetRotation(0.0f, 0.0f, 0.0f, "deg");
  xray.SetBeamAperture(11.0f, "deg");
  xray.SetFocalSpotSize(0.0f, 0.0f, 0.0f, "mm");
  xray.SetMonoenergy(60.0f, "keV");
  GGEMSDosimetryCalculator dose;
  dose.AttachToNavigator("phantom");
  dose.SetDoselSizes(4.0f, 4.0f, 4.0f, "mm");
  dose.SetOutputDosimetryBasename(dir + "/dose");
  dose.SetEdep(true);
  int caught = 0;
  try {
    xray.SetPosition(1.0f, 2.0f, 3.0f, "furlong");
  } catch (std::runtime_error const& e) {
    std::printf("unit: %s\n", e.what());
    caught += std::strlen(e.what()) > 0;
  }
  try {
    GGEMSVolumeCreatorManager::GetInstance().SetDataType("MET_COMPLEX");
  } catch (std::runtime_error const& e) {
    std::printf("type: %s\n", e.what());
    caught += std::strlen(e.what()) > 0;
  }
  std::printf("caught %d\n", caught);
  return caught == 2 ? 0 : 1;
}
'''


def test_facade_compiles_links_and_throws(tmp_path):
    if not os.path.exists(os.path.join(LIB, "libggems.so")):
        pytest.skip("libggems.so not built")
    from ggems_b200 import workloads
    mhd, rng_file, _ = workloads.cbct_files(str(tmp_path), 32, 8.0, seed=3)
    src = tmp_path / "main.cc"
    src.write_text(PROGRAM)
    exe = tmp_path / "main"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", INC, str(src), "-o", str(exe), "-L", LIB, "-lggems",
                    "-Wl,-rpath," + LIB], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe), str(tmp_path), os.path.join(LIB, "data", "materials.txt"), mhd,
                          rng_file],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "caught 2" in out.stdout
