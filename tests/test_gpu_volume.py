"""Phantom volumes on the GPU (gg_volume_*): analytic shapes drawn bit-exactly
as the oracle (itself pinned to GGEMS's Draw kernels) for every MHD element
type, range-table label conversion bit-exactly as the oracle, and the volume
creator API writing the MHD image and the range file."""

import ctypes as C
import os

import numpy as np
import pytest

import scenes
from ggems_b200 import abi

pytestmark = pytest.mark.gpu


def _shape(kind, pos, size, label):
    s = abi.gg_shape()
    s.type = kind
    s.position[:] = [float(v) for v in pos]
    s.size[:] = [float(v) for v in size]
    s.label_value = float(label)
    return s


CASES = [
    ((40, 40, 24), (1.0, 1.0, 2.0), [(abi.GG_SHAPE_BOX, (0, 0, 0), (30, 20, 30), 1),
                                     (abi.GG_SHAPE_TUBE, (3.5, -2.0, 4.0), (9.0, 6.0, 20.0), 2),
                                     (abi.GG_SHAPE_SPHERE, (-8.0, 7.0, -5.0), (6.5, 0, 0), 3)]),
    ((48, 32, 20), (0.5, 0.75, 1.0), [(abi.GG_SHAPE_BOX, (1.0, -1.0, 0.5), (12, 16, 10), 5),
                                      (abi.GG_SHAPE_SPHERE, (0.25, 0.0, 0.0), (7.0, 0, 0), 7)]),
    ((24, 36, 16), (2.0, 2.0, 2.0), [(abi.GG_SHAPE_TUBE, (0, 0, 0), (20.0, 14.0, 24.0), 9),
                                     (abi.GG_SHAPE_SPHERE, (4.0, -6.0, 2.0), (8.0, 0, 0), 11)]),
    ((256, 256, 256), (1.0, 1.0, 1.0), [(abi.GG_SHAPE_TUBE, (0, 0, 0), (110.0, 80.0, 240.0), 1),
                                        (abi.GG_SHAPE_SPHERE, (20.0, -10.0, 5.0), (30.0, 0, 0), 2),
                                        (abi.GG_SHAPE_BOX, (-40.0, 30.0, -50.0), (20.0, 10.0, 30.0), 3)]),
]


def _oracle_draw(met, dims, es, shapes):
    a = np.zeros(int(np.prod(dims)), abi.MET_DTYPES[met])
    d = (C.c_int32 * 3)(*dims)
    e = (C.c_float * 3)(*es)
    for s in shapes:
        assert scenes.oracle().gg_oracle_draw(a.ctypes.data_as(C.c_void_p), met, d, e, C.byref(s)) == 0
    return a


def test_draw_matches_oracle_every_type():
    from ggems_b200._native import Volume
    for dims, es, spec in CASES:
        shapes = [_shape(*t) for t in spec]
        types = range(7) if np.prod(dims) < 10 ** 6 else (abi.GG_MET_UCHAR, abi.GG_MET_FLOAT)
        for met in types:
            v = Volume(met, dims, es)
            v.draw(shapes)
            got = v.download()
            v.close()
            ref = _oracle_draw(met, dims, es, shapes)
            assert np.array_equal(got, ref), (dims, abi.MET_NAMES[met], int((got != ref).sum()))
            assert len(np.unique(ref)) == len(shapes) + 1


def test_labels_match_oracle():
    from ggems_b200._native import Volume
    rng = np.random.default_rng(7)
    dims = (96, 80, 64)
    n = int(np.prod(dims))
    cases = [
        (abi.GG_MET_SHORT, rng.integers(-1100, 2000, n).astype(np.int16),
         [-1100, -900, -100, 100, 300], [-900, -100, 100, 300, 2000]),
        (abi.GG_MET_UCHAR, rng.integers(0, 6, n).astype(np.uint8), [0, 1, 2, 3, 4, 5], [0, 1, 2, 3, 4, 5]),
        (abi.GG_MET_FLOAT, rng.uniform(-2, 2, n).astype(np.float32), [-2.0, -0.5, 0.0, 1.0], [-0.5, 0.5, 1.0, 1.5]),
        (abi.GG_MET_INT, rng.integers(-5, 5, n).astype(np.int32), [-5, -1, 0, 0], [0, 3, 1, 0]),
        (abi.GG_MET_UINT, rng.integers(0, 70000, n).astype(np.uint32), [0, 1000, 60000], [1000, 60000, 70000]),
        (abi.GG_MET_CHAR, rng.integers(-128, 128, n).astype(np.int8), [-128, -20, 0, 50], [-20, 0, 50, 100]),
        (abi.GG_MET_USHORT, rng.integers(0, 65536, n).astype(np.uint16), [0, 100, 30000, 65535],
         [100, 30000, 65535, 65535]),
    ]
    for met, img, first, last in cases:
        v = Volume(met, dims, (1.0, 1.0, 1.0))
        v.upload(img)
        got, missing = v.labels(first, last)
        v.close()
        f = np.asarray(first, np.float32)
        l_ = np.asarray(last, np.float32)
        ref = np.zeros(n, np.uint8)
        m = C.c_int64()
        assert scenes.oracle().gg_oracle_labels(img.ctypes.data_as(C.c_void_p), met, n, abi.ptr(f, C.c_float),
                                                abi.ptr(l_, C.c_float), len(f), abi.ptr(ref, C.c_uint8),
                                                C.byref(m)) == 0
        assert np.array_equal(got, ref), abi.MET_NAMES[met]
        assert missing == m.value


def test_volume_creator_api_writes_mhd_and_ranges(tmp_path):
    """GGEMS's volume-creator script (manager + tube + sphere + box) through the
    Python API: the written image equals the oracle's, the range file lists the
    labels and materials."""
    from ggems_b200 import GGEMSVolumeCreatorManager, GGEMSTube, GGEMSSphere, GGEMSBox
    out = str(tmp_path / "phantom.mhd")
    rng_file = str(tmp_path / "range_phantom.txt")
    m = GGEMSVolumeCreatorManager()
    m.set_dimensions(120, 120, 60)
    m.set_element_sizes(1.0, 1.0, 2.0, "mm")
    m.set_output(out)
    m.set_range_output(rng_file)
    m.set_material("Air")
    m.set_data_type("MET_INT")
    m.initialize()
    tube = GGEMSTube(50.0, 40.0, 100.0, "mm")
    tube.set_position(0.0, 0.0, 0.0, "mm")
    tube.set_label_value(1)
    tube.set_material("Water")
    tube.initialize()
    tube.draw()
    tube.delete()
    sph = GGEMSSphere(1.2, "cm")
    sph.set_position(1.0, -1.5, 0.5, "cm")
    sph.set_label_value(2)
    sph.set_material("Bone185")
    sph.initialize()
    sph.draw()
    sph.delete()
    box = GGEMSBox(10.0, 20.0, 30.0, "mm")
    box.set_position(-20.0, 10.0, 0.0, "mm")
    box.set_label_value(3)
    box.set_material("Lung")
    box.initialize()
    box.draw()
    box.delete()
    m.write()
    m.clean()
    header = open(out).read()
    assert "DimSize = 120 120 60" in header and "ElementType = MET_INT" in header
    raw = np.fromfile(out.replace(".mhd", ".raw"), np.int32)
    cm = np.float32(10.0)  # distance_unit: value * unit, in float
    shapes = [_shape(abi.GG_SHAPE_TUBE, (0, 0, 0), (50, 40, 100), 1),
              _shape(abi.GG_SHAPE_SPHERE, [np.float32(v) * cm for v in (1.0, -1.5, 0.5)],
                     (np.float32(1.2) * cm, 0, 0), 2),
              _shape(abi.GG_SHAPE_BOX, (-20, 10, 0), (10, 20, 30), 3)]
    ref = _oracle_draw(abi.GG_MET_INT, (120, 120, 60), (1.0, 1.0, 2.0), shapes)
    assert np.array_equal(raw, ref)
    assert open(rng_file).read() == "0 0 Air\n1 1 Water\n2 2 Bone185\n3 3 Lung\n"
