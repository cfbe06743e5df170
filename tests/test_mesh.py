"""Meshed phantom host preparation (CPU).

The product's STL reader, bounding spheres, triangle transform and octree
(ggems_b200/csrc/host/gg_mesh.cc) must equal the oracle's restatement of
GGEMSSTLReader / GGEMSMeshedSolid / GGEMSOctree bit for bit; the octree must
hold every triangle exactly once, inside its node; and the GGEMS Python API
must produce the same meshed solid.
"""

import ctypes as C
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import scenes
from ggems_b200 import abi, workloads


def _product_mesh(path, matrix, depth):
    from ggems_b200._native import lib
    f = lib.ggems_build_mesh
    f.restype = C.c_int
    nt, nn = C.c_int32(), C.c_int32()
    mat = np.ascontiguousarray(matrix.reshape(-1), np.float32)
    assert f(path.encode(), abi.ptr(mat, C.c_float), depth, C.byref(nt), C.byref(nn), None, None, None, None, None,
             None) == 0
    out = dict(triangles=np.zeros(nt.value * abi.GG_TRIANGLE_FLOATS, np.float32), nodes=np.zeros(nn.value * 6, np.float32),
               first=np.zeros(nn.value + 1, np.int32), order=np.zeros(max(nt.value, 1), np.int32),
               bmin=np.zeros(3, np.float32), bmax=np.zeros(3, np.float32))
    assert f(path.encode(), abi.ptr(mat, C.c_float), depth, C.byref(nt), C.byref(nn), abi.ptr(out["triangles"], C.c_float),
             abi.ptr(out["nodes"], C.c_float), abi.ptr(out["first"], C.c_int32), abi.ptr(out["order"], C.c_int32),
             abi.ptr(out["bmin"], C.c_float), abi.ptr(out["bmax"], C.c_float)) == 0
    return out


CASES = [
    (1, (), 1),
    (2, (), 3),
    (2, [("rotation", (1.5707963, 1.5707963, 0.0)), ("translation", (0.0, 0.0, 0.0))], 4),
    (3, [("rotation", (0.3, -0.7, 1.1)), ("translation", (12.5, -40.0, 7.25))], 5),
]


@pytest.mark.parametrize("subdiv,ops,depth", CASES)
def test_mesh_builder_bit_exact(subdiv, ops, depth, tmp_path):
    path = str(tmp_path / "m.stl")
    workloads.write_stl(path, workloads.body_mesh(subdiv, max(subdiv - 1, 0), 4, seed=subdiv))
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_meshed(path, t, ops=ops, depth=depth)
    o = sc.meshes[0]
    p = _product_mesh(path, scenes.geometry_matrix(scenes.PHANTOM_AXIS, ops), depth)
    for k in ("triangles", "nodes", "bmin", "bmax"):
        assert np.array_equal(p[k].view(np.uint32), o[k].view(np.uint32)), k
    assert np.array_equal(p["first"], o["first"])
    assert np.array_equal(p["order"], o["order"])


def test_octree_invariants(tmp_path):
    path = str(tmp_path / "m.stl")
    workloads.write_stl(path, workloads.body_mesh(3, 2, 8, seed=7))
    sc = scenes.Scene()
    t = sc.add_tables(scenes.Tables(["Water"]))
    sc.add_meshed(path, t, depth=4)
    m = sc.meshes[0]
    n = len(m["triangles"]) // abi.GG_TRIANGLE_FLOATS
    assert len(m["nodes"]) // 6 == 585
    assert np.array_equal(np.sort(m["order"][:n]), np.arange(n))  # each triangle in exactly one node
    tri = m["triangles"].reshape(n, abi.GG_TRIANGLE_FLOATS)
    nodes = m["nodes"].reshape(-1, 6)
    for node in range(len(nodes)):
        ids = m["order"][m["first"][node]:m["first"][node + 1]]
        if len(ids) == 0:
            continue
        assert np.all(np.diff(ids) < 0)  # linked list visits the last inserted first
        c, h = nodes[node, :3], nodes[node, 3:]
        v = tri[ids, :9].reshape(-1, 3)
        assert np.all(v >= c - h - 1e-3) and np.all(v <= c + h + 1e-3)  # triangles lie inside their node
    # the OBB is the root node box, grown 2.5 % and rounded to whole mm
    assert np.all(m["bmin"] == np.floor(m["bmin"])) and np.all(m["bmax"] == np.ceil(m["bmax"]))


def test_meshed_phantom_through_the_api(tmp_path):
    """GGEMSMeshedPhantom configured as GGEMS's mesh example does -> the same solid and
    tables as the restatement; dose map on the octree box with the requested dosel size."""
    path = str(tmp_path / "body.stl")
    workloads.write_stl(path, workloads.body_mesh(2, 1, 3, seed=2))
    code = textwrap.dedent(r'''
        import ctypes as C, numpy as np, sys
        import scenes
        from ggems_b200 import abi
        from ggems_b200 import (GGEMSMaterialsDatabaseManager, GGEMSMeshedPhantom, GGEMSDosimetryCalculator,
                                GGEMSProcessesManager, GGEMSRangeCutsManager, GGEMSXRaySource)
        GGEMSMaterialsDatabaseManager().set_materials(scenes.MATERIALS)
        m = GGEMSMeshedPhantom("phantom_mesh")
        m.set_phantom(sys.argv[1])
        m.set_rotation(90.0, 90.0, 0.0, "deg")
        m.set_position(0.0, 0.0, 0.0, "mm")
        m.set_mesh_octree_depth(4)
        m.set_visible(True)
        m.set_material("Water")
        m.set_material_color("Water", color_name="white")
        dose = GGEMSDosimetryCalculator()
        dose.attach_to_navigator("phantom_mesh")
        dose.set_output_basename("dose")
        dose.set_dosel_size(4.0, 4.0, 4.0, "mm")
        dose.uncertainty(True)
        pm = GGEMSProcessesManager()
        for p in ("Compton", "Photoelectric", "Rayleigh"):
            pm.add_process(p, "gamma", "all")
        GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
        s = GGEMSXRaySource("src")
        s.set_source_particle_type("gamma")
        s.set_number_of_particles(1000)
        s.set_position(-1000.0, 0.0, 0.0, "mm")
        s.set_rotation(0.0, 0.0, 0.0, "deg")
        s.set_beam_aperture(8.0, "deg")
        s.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
        s.set_monoenergy(80.0, "keV")
        from ggems_b200.api import lib
        lib.ggems_host_scene.restype = C.POINTER(abi.gg_scene)
        sc = lib.ggems_host_scene().contents
        deg = scenes.DEG
        ref = scenes.Scene()
        t = ref.add_tables(scenes.Tables(["Water"]))
        ref.add_meshed(sys.argv[1], t, ops=[("rotation", (float(90 * deg), float(90 * deg), 0.0)),
                                          ("translation", (0.0, 0.0, 0.0))], depth=4, dose={"dosel_size": (4.0, 4.0, 4.0)})
        r = ref.struct().solids[0]
        a = sc.solids[0]
        assert a.type == abi.GG_SOLID_MESHED and a.number_of_triangles == r.number_of_triangles
        assert a.number_of_nodes == r.number_of_nodes == 585
        n = a.number_of_triangles
        for f, size, ct in (("triangles", n * abi.GG_TRIANGLE_FLOATS, np.uint32), ("nodes", 585 * 6, np.uint32)):
            x = np.ctypeslib.as_array(getattr(a, f), (size,)).view(ct)
            y = np.ctypeslib.as_array(getattr(r, f), (size,)).view(ct)
            assert np.array_equal(x, y), f
        assert np.array_equal(np.ctypeslib.as_array(a.node_first, (586,)), np.ctypeslib.as_array(r.node_first, (586,)))
        assert np.array_equal(np.ctypeslib.as_array(a.node_triangles, (n,)), np.ctypeslib.as_array(r.node_triangles, (n,)))
        assert list(a.obb.border_min) == list(r.obb.border_min) and list(a.obb.border_max) == list(r.obb.border_max)
        assert list(a.obb.matrix) == [1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0, 0, 0, 0, 0, 1.0]
        d, rd = sc.dose_maps[0], ref.dose_maps[0]
        assert list(d.number_of_dosels) == list(rd.number_of_dosels) and d.tle == 0
        print("ok")
    ''')
    (tmp_path / "case.py").write_text(code)
    env = dict(os.environ, PYTHONPATH=scenes.ROOT + os.pathsep + os.path.join(scenes.ROOT, "tests"))
    out = subprocess.run([sys.executable, "case.py", path], capture_output=True, text=True, env=env, cwd=str(tmp_path),
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
