"""The C-ABI boundary (CPU): libggems.so loads, exports every function that
include/ggems_b200.h and include/ggems_api.h declare, the ctypes structures
match the C layout, and host-side entry points behave without a GPU."""

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import scenes
from ggems_b200 import abi

ROOT = scenes.ROOT


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "sizeof")))


@pytest.fixture(scope="module")
def lib():
    from ggems_b200._native import lib
    return lib


@pytest.mark.parametrize("header", ["ggems_b200.h", "ggems_api.h"])
def test_every_declared_symbol_is_exported(lib, header):
    names = _declared(header)
    assert len(names) > 10
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layouts_match_c():
    """Compile a probe printing sizeof/offsetof of the header's structs and compare with ctypes."""
    probe = r'''
#include <stdio.h>
#include <stddef.h>
#include "ggems_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(gg_obb), sizeof(gg_physics_tables),
         sizeof(gg_solid), sizeof(gg_dose_map), sizeof(gg_scene), sizeof(gg_source), sizeof(gg_particle_buffers),
         sizeof(gg_tally_buffers), offsetof(gg_source, number_of_activity_bins), sizeof(gg_world), sizeof(gg_job),
         sizeof(gg_shape), offsetof(gg_shape, size), sizeof(gg_track_point));
  return 0;
}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "p.c")
        exe = os.path.join(d, "p")
        open(src, "w").write(probe)
        subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), src, "-o", exe])
        sizes = [int(x) for x in subprocess.check_output([exe]).split()]
    ours = [C.sizeof(abi.gg_obb), C.sizeof(abi.gg_physics_tables), C.sizeof(abi.gg_solid), C.sizeof(abi.gg_dose_map),
            C.sizeof(abi.gg_scene), C.sizeof(abi.gg_source), C.sizeof(abi.gg_particle_buffers),
            C.sizeof(abi.gg_tally_buffers), abi.gg_source.number_of_activity_bins.offset, C.sizeof(abi.gg_world),
            C.sizeof(abi.gg_job), C.sizeof(abi.gg_shape), abi.gg_shape.size.offset, C.sizeof(abi.gg_track_point)]
    assert sizes == ours


def test_no_device_reports_error(lib):
    """Without a GPU the device layer fails cleanly with a status code, never a crash."""
    n = C.c_int32(-1)
    rc = lib.gg_device_count(C.byref(n))
    if rc != 0:
        assert n.value == 0
        assert lib.gg_last_error()
        h = C.c_void_p()
        assert lib.gg_context_create(0, C.byref(h)) != 0
        assert not h.value


def test_batch_plan_matches_reference(lib):
    """GGEMSSource::OrganizeParticlesInBatch: float ceil, equal split, remainder first."""
    for n in [1, 1000, 1048576, 1048577, 2 * 1048576 + 5, 10 ** 8, 123456789]:
        cnt = C.c_int64()
        sizes = (C.c_uint64 * 256)()
        assert lib.gg_batch_plan(n, sizes, 256, C.byref(cnt)) == 0
        nb = int(np.ceil(np.float32(n) / np.float32(abi.GG_MAXIMUM_PARTICLES)))
        assert cnt.value == nb
        got = [sizes[i] for i in range(nb)]
        assert sum(got) == n
        assert max(got) - min(got) <= 1 and got == sorted(got, reverse=True)
        assert max(got) <= abi.GG_MAXIMUM_PARTICLES
    cnt = C.c_int64()
    assert lib.gg_batch_plan(10 ** 8, None, 0, C.byref(cnt)) == 0 and cnt.value == 96


def test_invalid_arguments_are_rejected(lib):
    assert lib.gg_upload_scene(None, None) != 0
    assert lib.gg_run_source(None, None, 10) != 0
    assert lib.gg_seed_random_states(None, 10, 1, 0) != 0
