"""Pin the CPU oracle against GGEMS's own kernels.

oracle/_ref/libgg_ref.so is GGEMS's device code (src/kernels/*.cl) compiled
unmodified from the reference checkout through an OpenCL-C shim and driven in
the reference's launch order; both run on the same host with the same libm,
so the restatement must agree bit for bit: final particle states, random
streams, histograms and dose tallies.  Skipped where the reference checkout
is not available (it is not shipped).
"""

import ctypes as C
import os

import numpy as np
import pytest

import parity
import scenes
from ggems_b200 import abi

REF = os.path.join(scenes.ROOT, "oracle", "_ref", "libgg_ref.so")


def _ref_lib():
    if not os.path.exists(REF):
        if parity.reference_dir():
            import subprocess
            import sys
            subprocess.check_call([sys.executable, os.path.join(scenes.ROOT, "oracle", "build.py")])
        else:
            pytest.skip("reference checkout not available")
    lib = C.CDLL(REF)
    lib.gg_ref_run.restype = C.c_int
    lib.gg_ref_run.argtypes = scenes.oracle().gg_oracle_run.argtypes
    return lib


def _run_ref(sc, src, n, seed=777):
    st = scenes.seed_states(seed)
    ss = sc.struct()
    P = abi.Particles(min(n, abi.GG_MAXIMUM_PARTICLES))
    T = sc.tallies()
    rc = _ref_lib().gg_ref_run(C.byref(ss), C.byref(src.struct), n, abi.ptr(st, C.c_uint32), C.byref(P.struct),
                               C.byref(T.struct), os.cpu_count())
    assert rc == 0
    return P, T, st


def _assert_identical(a, b):
    Pa, Ta, sa = a
    Pb, Tb, sb = b
    if Ta.world is not None:
        assert np.array_equal(Ta.world["photon_tracking"], Tb.world["photon_tracking"])
        assert Ta.world["photon_tracking"].sum() > 0
        for k in ("energy", "energy_squared", "momentum_x", "momentum_y", "momentum_z"):
            np.testing.assert_allclose(Ta.world[k], Tb.world[k], rtol=1e-12, atol=1e-9)
    exact, _ = parity.history_agreement(Pa, Pb)
    assert exact == 1.0
    assert np.array_equal(sa, sb)
    for x, y in zip(Ta.histograms, Tb.histograms):
        assert np.array_equal(x, y)
    for name in ("hit", "photon_tracking"):
        for x, y in zip(getattr(Ta, name), getattr(Tb, name)):
            assert np.array_equal(x, y)
    for name in ("edep", "edep_squared"):
        for x, y in zip(getattr(Ta, name), getattr(Tb, name)):
            # double sums accumulated in a different order: same terms, last-bit differences only
            np.testing.assert_allclose(x, y, rtol=1e-12, atol=0)


def test_pin_water_box_dosimetry():
    sc = scenes.water_box_scene(photon_tracking=True)
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_cbct_detector_polyenergetic():
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0, focal=(0.6, 0.6, 0.0))
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_rotated_phantom_and_detector():
    """Non-trivial frames: rotated phantom, rotated CT module, rotated source."""
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Air", "Water", "Bone185"], processes=(2, 0, 1)))
    labels = scenes.ellipsoid_phantom(24, 10.0, seed=3, n_bones=4)
    deg = scenes.DEG
    sc.add_voxelized(labels, (10.0, 10.0, 10.0), t,
                     ops=[("rotation", (float(20 * deg), float(-10 * deg), float(35 * deg))),
                          ("translation", (5.0, -12.0, 3.0))])
    td = sc.add_tables(scenes.Tables(["GOS"], processes=(0, 1)))
    sc.add_flat_detector(td, (32, 32, 1), (12.8, 12.8, 10.0), sdd=1500.0, sid=1000.0, threshold=0.0,
                         extra_rotation=(0.0, 0.0, float(15 * deg)))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=12.0,
                            rotation=(0.0, 0.0, float(15 * deg)), order=("position", "rotation"))
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_multiple_batches():
    sc = scenes.cbct_scene(n=16, voxel=16.0, elements=(32, 32, 1), element_size=(12.8, 12.8, 10.0))
    src = scenes.XRaySource(monoenergy=scenes.F(80.0) * scenes.KEV, aperture_deg=11.0)
    n = 2 * 1048576 + 5
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_voxelized_source_in_water_with_dose():
    sc = scenes.water_box_scene(n=32, voxel=4.0, photon_tracking=True)
    src = scenes.VoxelizedSource(scenes.hot_spot_activity(16), (4.0, 4.0, 4.0), position=(8.0, -4.0, 0.0),
                                 monoenergy=scenes.F(140.0) * scenes.KEV)
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_curved_ct_modules():
    """46-module curved detector (the ct_scanner example layout) around a water box."""
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_voxelized(np.zeros((20, 20, 20), np.uint8), (5.0, 5.0, 5.0), t)
    td = sc.add_tables(scenes.Tables(["GOS"]))
    scenes.add_curved_detector(sc, td, (1, 46), (64, 16, 1), (0.6, 0.6, 0.6), 1085.6, 595.0,
                               scenes.F(10.0) * scenes.KEV)
    src = scenes.XRaySource(position=(-595.0, 0.0, 0.0), spectrum=scenes.synthetic_spectrum(), aperture_deg=12.5)
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_tle_dosimetry_water():
    """Track-length-estimator dose (TrackThroughGGEMSVoxelizedSolid.cl built with DOSIMETRY and TLE)."""
    sc = scenes.water_box_scene(photon_tracking=True, tle=True)
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_tle_dosimetry_heterogeneous():
    """TLE in air / water / bone with a polyenergetic beam (mu_en interpolated per material)."""
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Air", "Water", "Bone185"]))
    sc.add_voxelized(scenes.ellipsoid_phantom(32, 8.0, seed=5, n_bones=3), (8.0, 8.0, 8.0), t, dose={"tle": True})
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 30000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_meshed_phantom(tmp_path):
    """GGEMSMeshedPhantom: octree node scan, Moller-Trumbore crossings, parity navigation."""
    sc = scenes.mesh_phantom_scene(str(tmp_path / "body.stl"), subdivisions=2, n_inner=2, depth=3)
    src = scenes.XRaySource(monoenergy=scenes.F(80.0) * scenes.KEV, aperture_deg=8.0)
    n = 20000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_meshed_phantom_dosimetry_rotated(tmp_path):
    """Rotated / translated mesh with a dose map (DOSIMETRY variant of the mesh kernel)."""
    deg = scenes.DEG
    sc = scenes.mesh_phantom_scene(str(tmp_path / "body.stl"), subdivisions=2, n_inner=3, depth=4, dose=True,
                                   ops=[("rotation", (float(90 * deg), float(30 * deg), 0.0)),
                                        ("translation", (10.0, -5.0, 0.0))])
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=8.0)
    n = 20000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def test_pin_world_tracking():
    """GGEMSWorld: photon counts, energy, energy^2 and momentum on a world grid
    (WorldTracking.cl), with a phantom and a CT panel."""
    sc = scenes.cbct_scene(n=32, voxel=8.0, elements=(64, 64, 1), element_size=(6.4, 6.4, 10.0))
    sc.set_world((40, 30, 20), (60.0, 50.0, 40.0))
    src = scenes.XRaySource(spectrum=scenes.synthetic_spectrum(), aperture_deg=11.0)
    n = 20000
    _assert_identical(parity.run_oracle(sc, src, n), _run_ref(sc, src, n))


def _shape(kind, pos, size, label):
    s = abi.gg_shape()
    s.type = kind
    s.position[:] = [float(v) for v in pos]
    s.size[:] = [float(v) for v in size]
    s.label_value = float(label)
    return s


VOLUME_CASES = [
    # dimensions (x, y, z), element sizes, shapes: GGEMS's y-index arithmetic is only
    # right for x == y, so unequal x / y dimensions are included on purpose
    ((40, 40, 24), (1.0, 1.0, 2.0), [(abi.GG_SHAPE_BOX, (0, 0, 0), (30, 20, 30), 1),
                                     (abi.GG_SHAPE_TUBE, (3.5, -2.0, 4.0), (9.0, 6.0, 20.0), 2),
                                     (abi.GG_SHAPE_SPHERE, (-8.0, 7.0, -5.0), (6.5, 0, 0), 3)]),
    ((48, 32, 20), (0.5, 0.75, 1.0), [(abi.GG_SHAPE_BOX, (1.0, -1.0, 0.5), (12, 16, 10), 5),
                                      (abi.GG_SHAPE_SPHERE, (0.25, 0.0, 0.0), (7.0, 0, 0), 7)]),
    ((24, 36, 16), (2.0, 2.0, 2.0), [(abi.GG_SHAPE_TUBE, (0, 0, 0), (20.0, 14.0, 24.0), 9),
                                     (abi.GG_SHAPE_SPHERE, (4.0, -6.0, 2.0), (8.0, 0, 0), 11)]),
]


def test_pin_volume_draw():
    """Volume creator: the oracle draws boxes, tubes and spheres exactly as
    GGEMS's DrawGGEMS{Box,Tube,Sphere}.cl do (uchar and float images)."""
    ref = _ref_lib()
    ref.gg_ref_draw.restype = C.c_int
    ora = scenes.oracle()
    for dims, es, shapes in VOLUME_CASES:
        d = (C.c_int32 * 3)(*dims)
        e = (C.c_float * 3)(*es)
        for met, dt in ((abi.GG_MET_UCHAR, np.uint8), (abi.GG_MET_FLOAT, np.float32)):
            a = np.zeros(int(np.prod(dims)), dt)
            b = np.zeros_like(a)
            for kind, pos, size, label in shapes:
                s = _shape(kind, pos, size, label)
                assert ora.gg_oracle_draw(a.ctypes.data_as(C.c_void_p), met, d, e, C.byref(s)) == 0
                assert ref.gg_ref_draw(b.ctypes.data_as(C.c_void_p), met, d, e, C.byref(s)) == 0
            assert np.array_equal(a, b), (dims, met)
            labels = set(np.unique(a).tolist())
            assert {0} < labels, labels
