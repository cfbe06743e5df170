"""Phantom volumes on the host side (no GPU): the oracle's range-table label
conversion against a direct numpy statement of ConvertImageToLabel, and the
volume creator API's parameter checks and messages."""

import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np

import scenes
from ggems_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _numpy_labels(image, first, last):
    """include/GGEMS/geometries/GGEMSVoxelizedSolid.hh:162-257: every range line,
    in file order, relabels the voxels it holds; 255 = not converted."""
    v = image.astype(np.float32)
    out = np.full(v.shape, 255, np.uint8)
    for r, (a, b) in enumerate(zip(np.float32(first), np.float32(last))):
        out[((v == a) & (v == b)) | ((v >= a) & (v < b))] = r
    return out


def test_oracle_labels_match_numpy():
    ora = scenes.oracle()
    rng = np.random.default_rng(3)
    cases = [
        (abi.GG_MET_SHORT, rng.integers(-1100, 2000, 5000).astype(np.int16),
         [-1100, -900, -100, 100, 300], [-900, -100, 100, 300, 2000]),
        (abi.GG_MET_UCHAR, rng.integers(0, 6, 4000).astype(np.uint8), [0, 1, 2, 3, 4], [0, 1, 2, 3, 4]),
        (abi.GG_MET_FLOAT, rng.uniform(-2, 2, 3000).astype(np.float32), [-2.0, -0.5, 0.0, 1.0], [-0.5, 0.5, 1.0, 1.5]),
        (abi.GG_MET_INT, rng.integers(-5, 5, 3000).astype(np.int32), [-5, -1, 0, 0], [0, 3, 1, 0]),
    ]
    for met, img, first, last in cases:
        f = np.asarray(first, np.float32)
        l_ = np.asarray(last, np.float32)
        out = np.zeros(img.size, np.uint8)
        missing = C.c_int64()
        assert ora.gg_oracle_labels(img.ctypes.data_as(C.c_void_p), met, img.size, abi.ptr(f, C.c_float),
                                    abi.ptr(l_, C.c_float), len(f), abi.ptr(out, C.c_uint8), C.byref(missing)) == 0
        ref = _numpy_labels(img, f, l_)
        assert np.array_equal(out, ref), met
        assert missing.value == int((ref == 255).sum())
    assert missing.value > 0  # the float case leaves [1.5, 2) unconverted


def test_volume_creator_parameter_checks(tmp_path):
    """GGEMSVolumeCreatorManager::CheckParameters / SetDataType messages, and
    AddLabelAndMaterial refusing a label twice."""
    script = tmp_path / "case.py"
    script.write_text(textwrap.dedent(r'''
        from ggems_b200 import GGEMSVolumeCreatorManager, GGEMSBox, GGEMSError
        from ggems_b200.api import lib
        m = GGEMSVolumeCreatorManager()
        try:
            m.initialize()
            raise SystemExit("no error")
        except GGEMSError as e:
            assert "Phantom dimensions have to be > 0!!!" in str(e), e
        m.set_dimensions(10, 10, 10)
        try:
            m.initialize()
            raise SystemExit("no error")
        except GGEMSError as e:
            assert "Phantom voxel sizes have to be > 0.0!!!" in str(e), e
        m.set_element_sizes(1.0, 1.0, 1.0, "mm")
        try:
            m.initialize()
            raise SystemExit("no error")
        except GGEMSError as e:
            assert "A output image filename has to be done" in str(e), e
        try:
            m.set_data_type("MET_DOUBLE")
            raise SystemExit("no error")
        except GGEMSError as e:
            assert "Your type in not compatible" in str(e), e
        b = GGEMSBox(1.0, 2.0, 3.0, "cm")
        b.set_label_value(2)
        b.set_material("Water")
        c = GGEMSBox(1.0, 2.0, 3.0, "cm")
        c.set_label_value(2)
        try:
            c.set_material("Bone185")
            raise SystemExit("no error")
        except GGEMSError as e:
            assert "The label: 2 already exists..." in str(e), e
        try:
            b.draw()
            raise SystemExit("no error")
        except GGEMSError as e:
            assert "GGEMSBox::Draw" in str(e), e
        print("ok")
    '''))
    env = dict(os.environ, PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, env=env, cwd=str(tmp_path),
                         timeout=300)
    assert out.returncode == 0 and "ok" in out.stdout, out.stdout + out.stderr
