"""Drop-in check with the reference's own Python module: GGEMS's
python_module/*.py, copied unmodified into a temporary directory beside a
link to this build's libggems.so (where the module looks for the library:
python_module/ggems_lib.py:28-36), runs two of the reference's example
scripts unchanged -- 4_Dosimetry_Photon/dosimetry_photon.py (volume creator,
voxelized phantom, dosimetry, polyenergetic X-ray source) and
2_CT_Scanner/ct_scanner.py (46-module curved CT system) -- in copies of their
directories.  Checked here: every class of the module binds its functions
against this library (each __init__ sets argtypes / restype and would fail on
a missing export), and the scripts run through their configuration with no
failure other than the missing device (the volume creator draws on the
device, so the phantom, and with it the scene, needs one).  On a B200 the
same scripts run to completion.  Reading the reference checkout is needed, so
this is a CPU test, skipped without the checkout.
"""

import os
import shutil
import stat
import subprocess
import sys
import textwrap

import pytest

import parity

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "ggems_b200", "libggems.so")


def _stage(tmp_path, ref, example):
    if not os.path.exists(LIB):
        pytest.skip("libggems.so not built")
    stage = tmp_path / "stage"
    stage.mkdir()
    shutil.copytree(os.path.join(ref, "python_module"), stage / "ggems")
    os.symlink(LIB, stage / "libggems.so")
    work = tmp_path / "example"
    shutil.copytree(os.path.join(ref, "examples", example), work)
    for d, dirs, files in os.walk(work):  # the checkout is read-only; the scripts write into data/
        for x in dirs + files:
            p = os.path.join(d, x)
            os.chmod(p, os.stat(p).st_mode | stat.S_IWUSR)
    os.chmod(work, os.stat(work).st_mode | stat.S_IWUSR)
    return stage, work


@pytest.fixture(scope="module")
def reference():
    ref = parity.reference_dir()
    if ref is None:
        pytest.skip("reference checkout not available")
    return ref


# what a GPU-less host may report while running the scripts: the device is
# missing, and everything that needs what it would have made is not initialized
DEVICE_ONLY = ("no such CUDA device", "not initialized", "no CUDA device", "CUDA driver", "no scene")


def _device_only_failures(stderr):
    bad = [line for line in stderr.splitlines() if "EXCEPTION" in line and not any(k in line for k in DEVICE_ONLY)]
    assert "Traceback" not in stderr, stderr[-3000:]
    assert not bad, "\n".join(bad)


def test_every_reference_class_binds(tmp_path, reference):
    """Instantiate every class of the reference's module except the OpenGL
    viewer (no graphics stack here): their constructors bind each function the
    class calls."""
    stage, _ = _stage(tmp_path, reference, "4_Dosimetry_Photon")
    code = textwrap.dedent(r'''
        import sys
        sys.path.insert(0, sys.argv[1])
        import ggems
        made = []
        for name, args in [("GGEMSVerbosity", (0,)), ("GGEMSOpenCLManager", ()), ("GGEMSRAMManager", ()),
                           ("GGEMSMaterialsDatabaseManager", ()), ("GGEMSProcessesManager", ()),
                           ("GGEMSRangeCutsManager", ()), ("GGEMSVolumeCreatorManager", ()),
                           ("GGEMSSourceManager", ()), ("GGEMSProfilerManager", ()), ("GGEMS", ()),
                           ("GGEMSXRaySource", ("s",)), ("GGEMSVoxelizedSource", ("vs",)),
                           ("GGEMSVoxelizedPhantom", ("p",)), ("GGEMSMeshedPhantom", ("m",)), ("GGEMSWorld", ()),
                           ("GGEMSCTSystem", ("ct",)), ("GGEMSDosimetryCalculator", ()),
                           ("GGEMSBox", (1.0, 1.0, 1.0, "mm")), ("GGEMSTube", (1.0, 1.0, 1.0, "mm")),
                           ("GGEMSSphere", (1.0, "mm")), ("GGEMSMaterials", ())]:
            made.append(getattr(ggems, name)(*args))
        m = made[-1]
        made.append(ggems.GGEMSCrossSections(m))
        made.append(ggems.GGEMSAttenuations(m, made[-1]))
        print("bound", len(made))
    ''')
    (tmp_path / "bind.py").write_text(code)
    out = subprocess.run([sys.executable, str(tmp_path / "bind.py"), str(stage)], capture_output=True, text=True,
                         timeout=300, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    assert "bound 23" in out.stdout


@pytest.mark.parametrize("example,script", [("4_Dosimetry_Photon", "dosimetry_photon.py"),
                                            ("2_CT_Scanner", "ct_scanner.py")])
def test_example_scripts_run_unchanged(tmp_path, reference, example, script):
    stage, work = _stage(tmp_path, reference, example)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    out = subprocess.run([sys.executable, script, "-n", "1000"], cwd=str(work), capture_output=True, text=True,
                         env=dict(env, PYTHONPATH=str(stage)), timeout=600)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    _device_only_failures(out.stdout + out.stderr)
