"""gg_compute_dose_no_alloc against gg_compute_dose (GPU).

The no-allocation entry point runs the same dose kernel into a fixed device
array instead of per-call allocations, so its outputs must equal
gg_compute_dose's bit for bit (tolerance: exact), on the first call of the
process (which looks the array up) and on the next one (which reuses what the
first left in it).  Dose maps larger than the array are refused.
"""

import ctypes as C

import numpy as np
import pytest

import parity
import scenes
from ggems_b200 import abi

pytestmark = pytest.mark.gpu

MAX_DOSELS = 2097152  # GG_NO_ALLOC_MAX_DOSELS in include/ggems_b200.h


@pytest.fixture(scope="module")
def native():
    from ggems_b200 import _native
    f = _native.lib.gg_compute_dose_no_alloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_int32, C.c_float,
                  C.POINTER(C.c_float), C.POINTER(C.c_float)]
    ctx = _native.Context(0)
    yield _native, ctx
    ctx.close()


def _no_alloc(native, ctx, n, scale, water, min_density, uncertainty=True):
    _native, _ = native
    dose = np.full(n, np.nan, np.float32)
    unc = np.full(n, np.nan, np.float32) if uncertainty else None
    rc = _native.lib.gg_compute_dose_no_alloc(ctx.handle, 0, 0, scale, 1 if water else 0, min_density,
                                               abi.ptr(dose, C.c_float), abi.ptr(unc, C.c_float))
    assert rc == 0, _native.lib.gg_last_error().decode()
    return dose, unc


def test_no_alloc_dose_matches_allocating_entry_point_twice(native):
    _, ctx = native
    sc = scenes.water_box_scene()
    src = scenes.XRaySource(monoenergy=scenes.F(60.0) * scenes.KEV, aperture_deg=10.0)
    parity.run_gpu(ctx, sc, src, 100000)
    n = sc.dose_maps[0].total_number_of_dosels
    ref_dose, ref_unc = ctx.compute_dose(0, 0, n, scale=1.0, water_reference=False, minimum_density=0.0)
    assert np.count_nonzero(ref_dose) > 1000
    for _ in range(2):
        dose, unc = _no_alloc(native, ctx, n, 1.0, False, 0.0)
        np.testing.assert_array_equal(dose, ref_dose)
        np.testing.assert_array_equal(unc, ref_unc)
    # different arguments, and no uncertainty output, on the same array
    ref_dose, _ = ctx.compute_dose(0, 0, n, scale=2.5, water_reference=True, minimum_density=0.0,
                                   uncertainty=False)
    dose, _ = _no_alloc(native, ctx, n, 2.5, True, 0.0, uncertainty=False)
    np.testing.assert_array_equal(dose, ref_dose)


def test_no_alloc_refuses_maps_above_its_limit(native):
    _native, ctx = native
    sc = scenes.water_box_scene(n=129, voxel=1.0)
    n = sc.dose_maps[0].total_number_of_dosels
    assert n > MAX_DOSELS
    ctx.upload_scene(sc.struct())
    dose = np.zeros(n, np.float32)
    rc = _native.lib.gg_compute_dose_no_alloc(ctx.handle, 0, 0, 1.0, 0, 0.0, abi.ptr(dose, C.c_float), None)
    assert rc == 1  # GG_ERROR_INVALID_ARGUMENT
    assert b"at most 2097152" in _native.lib.gg_last_error()
