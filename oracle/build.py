"""Build recipe for the oracle (test infrastructure only).

* ``oracle/_build/libgg_oracle.so`` -- the CPU restatement (gg_oracle.cc),
  built from this repository alone; it is the checker the GPU tests use.
* ``oracle/_ref/libgg_ref.so`` -- GGEMS's own device kernels
  (``src/kernels/*.cl``) compiled straight from a reference checkout through
  ``oracle/ref_shim/ocl_shim.hh``, plus ``gg_ref_driver.cc``.  Only built when
  the checkout exists; it pins the restatement.

Both use ``-ffp-contract=off`` (no fused multiply-add) so float arithmetic
rounds exactly as written.

Usage: python oracle/build.py [--ref /path/to/reference]
"""

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
# The reference checkout: $GGEMS_REFERENCE_DIR, else the path this recipe was
# written against.  Only this recipe (and the scripts that call it) read it.
DEFAULT_REFERENCE = os.environ.get("GGEMS_REFERENCE_DIR", "/root/reference")


def reference_dir():
    """The reference checkout, or None when it is not on this machine."""
    return DEFAULT_REFERENCE if os.path.isdir(os.path.join(DEFAULT_REFERENCE, "src", "kernels")) else None

CXX = ["g++", "-std=c++20", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math"]

# (kernel file, extra defines, symbol renames)
REF_KERNELS = [
    ("GetPrimariesGGEMSXRaySource", [], []),
    ("GetPrimariesGGEMSVoxelizedSource", [], []),
    ("ParticleSolidDistanceGGEMSVoxelizedSolid", [], []),
    ("ParticleSolidDistanceGGEMSSolidBox", [], []),
    ("ProjectToGGEMSVoxelizedSolid", [], []),
    ("ProjectToGGEMSSolidBox", [], []),
    ("TrackThroughGGEMSVoxelizedSolid", [], []),
    ("TrackThroughGGEMSVoxelizedSolid", ["DOSIMETRY"],
     ["track_through_ggems_voxelized_solid=track_through_ggems_voxelized_solid_dosimetry"]),
    ("TrackThroughGGEMSVoxelizedSolid", ["DOSIMETRY", "TLE"],
     ["track_through_ggems_voxelized_solid=track_through_ggems_voxelized_solid_tle"]),
    ("TrackThroughGGEMSSolidBox", ["HISTOGRAM"], []),
    ("ParticleSolidDistanceGGEMSMeshSolid", [], []),
    ("ProjectToGGEMSMeshSolid", [], []),
    ("TrackThroughGGEMSMeshSolid", [], []),
    ("TrackThroughGGEMSMeshSolid", ["DOSIMETRY"],
     ["track_through_ggems_meshed_solid=track_through_ggems_meshed_solid_dosimetry"]),
    ("IsAlive", [], []),
    ("WorldTracking", [], []),
    ("DrawGGEMSBox", ["MET_UCHAR"], []),
    ("DrawGGEMSBox", ["MET_FLOAT"], ["draw_ggems_box=draw_ggems_box_float"]),
    ("DrawGGEMSTube", ["MET_UCHAR"], []),
    ("DrawGGEMSTube", ["MET_FLOAT"], ["draw_ggems_tube=draw_ggems_tube_float"]),
    ("DrawGGEMSSphere", ["MET_UCHAR"], []),
    ("DrawGGEMSSphere", ["MET_FLOAT"], ["draw_ggems_sphere=draw_ggems_sphere_float"]),
]


def run(cmd):
    subprocess.check_call(cmd)


def build_oracle():
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(BUILD, "libgg_oracle.so")
    run(CXX + ["-shared", "-I" + os.path.join(ROOT, "include"), os.path.join(HERE, "gg_oracle.cc"),
               os.path.join(HERE, "gg_oracle_tables.cc"), os.path.join(HERE, "gg_oracle_mesh.cc"),
               os.path.join(HERE, "gg_oracle_volume.cc"), "-o", out, "-lpthread"])
    # the same transport restatement in FP64 (precision reference for the results)
    run(CXX + ["-shared", "-DGG_ORACLE_REAL=double", "-I" + os.path.join(ROOT, "include"),
               os.path.join(HERE, "gg_oracle.cc"), "-o", os.path.join(BUILD, "libgg_oracle_fp64.so"), "-lpthread"])
    return out


def build_ref(reference):
    if not os.path.isdir(os.path.join(reference, "src", "kernels")):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "ref_shim")
    common = CXX + ["-w", "-Wno-narrowing", "-fpermissive", "-include", os.path.join(shim, "ocl_shim.hh"),
                    "-I" + shim, "-I" + os.path.join(reference, "include"), "-I" + os.path.join(ROOT, "include")]
    objs = []
    for name, defines, renames in REF_KERNELS:
        tag = name + ("_" + "_".join(defines) if defines else "")
        obj = os.path.join(REF_OUT, tag + ".o")
        cmd = common + ["-D" + d for d in defines] + ["-D" + r for r in renames]
        run(cmd + ["-x", "c++", "-c", os.path.join(reference, "src", "kernels", name + ".cl"), "-o", obj])
        objs.append(obj)
    drv = os.path.join(REF_OUT, "gg_ref_driver.o")
    run(common + ["-c", os.path.join(HERE, "gg_ref_driver.cc"), "-o", drv])
    out = os.path.join(REF_OUT, "libgg_ref.so")
    run(["g++", "-shared", "-o", out, drv] + objs + ["-lpthread"])
    return out


# GGEMS's host sources the table pin compiles (material database, material
# tables and range cuts, cross sections and the three per-atom formulas,
# attenuations, and the text reader / printing / exception helpers they call).
REF_HOST_SOURCES = [
    "src/materials/GGEMSMaterialsDatabaseManager.cc", "src/materials/GGEMSMaterials.cc",
    "src/materials/GGEMSIonizationParamsMaterial.cc", "src/physics/GGEMSCrossSections.cc",
    "src/physics/GGEMSEMProcess.cc", "src/physics/GGEMSComptonScattering.cc",
    "src/physics/GGEMSPhotoElectricEffect.cc", "src/physics/GGEMSRayleighScattering.cc",
    "src/physics/GGEMSRangeCuts.cc", "src/physics/GGEMSLogEnergyTable.cc", "src/physics/GGEMSProcessesManager.cc",
    "src/physics/GGEMSAttenuations.cc", "src/io/GGEMSTextReader.cc", "src/tools/GGEMSPrint.cc",
    "src/tools/GGEMSTools.cc",
]


def build_ref_tables(reference, extra_flags=(), name="libgg_ref_tables.so"):
    """GGEMS's host table builders, compiled unmodified from the checkout with
    oracle/ref_host (a host stand-in for the OpenCL header and the few
    GGEMSOpenCLManager members they call) into oracle/_ref/<name>."""
    if not os.path.isdir(os.path.join(reference, "src", "physics")):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    host = os.path.join(HERE, "ref_host")
    common = ["g++", "-std=c++17", "-O2", "-fPIC", "-w"] + list(extra_flags) + [
        "-I" + host, "-I" + os.path.join(HERE, "ref_shim"), "-I" + os.path.join(reference, "include")]
    if not extra_flags:
        common += ["-ffp-contract=off", "-fno-fast-math"]
    tag = os.path.splitext(name)[0]
    objs = []
    for src in REF_HOST_SOURCES + [os.path.join(host, "gg_ref_tables.cc")]:
        path = src if os.path.isabs(src) else os.path.join(reference, src)
        obj = os.path.join(REF_OUT, "%s_%s.o" % (tag, os.path.splitext(os.path.basename(path))[0]))
        run(common + ["-c", path, "-o", obj])
        objs.append(obj)
    out = os.path.join(REF_OUT, name)
    run(["g++", "-shared", "-o", out] + objs + ["-lpthread"])
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=DEFAULT_REFERENCE)
    args = ap.parse_args()
    print(build_oracle())
    print(build_ref(args.ref))
    print(build_ref_tables(args.ref))
    # the same sources with the reference's own release flags (CMakeLists.txt:163-164):
    # -O3 -march=native lets g++ contract a*b+c into FMA on hosts that have it
    print(build_ref_tables(args.ref, ("-O3", "-march=native"), "libgg_ref_tables_native.so"))


if __name__ == "__main__":
    sys.exit(main())
