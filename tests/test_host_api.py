"""The GGEMS-compatible Python / C++ host API, without a GPU.

The CBCT workload is configured through the same calls a GGEMS script makes
(materials database, voxelized phantom, CT system, processes, range cuts,
X-ray source) and prepared on the host; the resulting scene must equal the
independent restatement in tests/scenes.py field by field (geometry matrices
bit-exact, tables bit-exact), the labels must follow
GGEMSVoxelizedSolid::ConvertImageToLabel, and errors must surface as
exceptions carrying GGEMS's message.  Each case runs in a fresh process (the
API keeps GGEMS's singletons).
"""

import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(code, tmp_path):
    script = tmp_path / "case.py"
    script.write_text(textwrap.dedent(code))
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.path.join(ROOT, "tests"))
    out = subprocess.run([sys.executable, str(script)], capture_output=True, text=True, env=env, cwd=str(tmp_path),
                         timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return out.stdout


def test_cbct_scene_matches_restatement(tmp_path):
    _run(r'''
        import ctypes as C, numpy as np, os, sys
        sys.path.insert(0, os.environ["PYTHONPATH"].split(os.pathsep)[0])
        import bench, scenes
        from ggems_b200 import workloads, abi
        files = workloads.cbct_files(".", 64, 4.0, seed=5)
        gg = bench._configure(files, 1000)
        from ggems_b200.api import lib
        lib.ggems_host_scene.restype = C.POINTER(abi.gg_scene)
        sc = lib.ggems_host_scene().contents
        ref, rsrc = scenes.cbct_api_scene(64, 4.0, 5)
        rs = ref.struct()
        assert sc.number_of_solids == 2 and sc.number_of_tables == 2 and sc.number_of_histograms == 2
        for i in range(2):
            a, b = sc.solids[i], rs.solids[i]
            for f in ("type", "navigator", "histogram", "scatter_histogram", "dose_map"):
                assert getattr(a, f) == getattr(b, f), (i, f)
            assert np.array_equal(np.array(a.obb.matrix, np.float32).view(np.uint32), np.array(b.obb.matrix, np.float32).view(np.uint32)), i
            for f in ("border_min", "border_max"):
                assert list(getattr(a.obb, f)) == list(getattr(b.obb, f)), (i, f)
            assert list(a.voxel_sizes) == list(b.voxel_sizes) and list(a.number_of_voxels) == list(b.number_of_voxels)
            assert list(a.virtual_element_number) == list(b.virtual_element_number) and list(a.box_size) == list(b.box_size)
            assert a.threshold == b.threshold
        n = 64 ** 3
        assert np.array_equal(np.ctypeslib.as_array(sc.solids[0].labels, (n,)), np.ctypeslib.as_array(rs.solids[0].labels, (n,)))
        for i in range(2):
            a, b = sc.tables[i], rs.tables[i]
            nb, nm = a.number_of_bins, a.number_of_materials
            assert (nb, nm, a.number_of_processes) == (b.number_of_bins, b.number_of_materials, b.number_of_processes)
            for f, size in (("energy_bins", nb), ("cross_sections", 3 * nm * nb), ("density", nm), ("photon_energy_cut", nm)):
                x = np.ctypeslib.as_array(getattr(a, f), (size,)); y = np.ctypeslib.as_array(getattr(b, f), (size,))
                assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), (i, f)
        src = abi.gg_source()
        assert lib.ggems_source_descriptor(0, C.byref(src), None) == 0
        assert np.array_equal(np.array(src.matrix, np.float32), rsrc.matrix.reshape(-1))
        assert np.float32(src.beam_aperture) == np.float32(rsrc.struct.beam_aperture)
        m = src.number_of_energy_bins + 1
        assert np.array_equal(np.ctypeslib.as_array(src.energy_spectrum, (m,)), rsrc.spectrum)
        assert np.array_equal(np.ctypeslib.as_array(src.energy_cdf, (m,)), rsrc.cdf)
        print("ok")
    ''', tmp_path)


def test_label_conversion_ranges(tmp_path):
    """value -> label of the k-th range line when v == first == last or first <= v < last."""
    _run(r'''
        import ctypes as C, numpy as np
        from ggems_b200 import workloads
        from ggems_b200.api import lib
        vals = np.array([[[-1000, -500, 0], [40, 200, 1499]], [[1500, 3000, 12]]], dtype=object)
        v = np.array([-1000, -500, 0, 40, 200, 1499, 1500, 3000, 12, 7, 7, 7], np.int16).reshape(2, 2, 3)
        workloads.write_mhd("p.mhd", v, (1, 1, 1), "MET_SHORT")
        open("r.txt", "w").write("-1000 -100 Air\n0 0 Water\n1 1500 RibBone\n1500 1500 GOS\n2000 4000 Aluminium\n")
        dims = (C.c_int32 * 3)(); lab = np.zeros(12, np.uint8)
        lib.ggems_phantom_labels.restype = C.c_int
        rc = lib.ggems_phantom_labels(b"p.mhd", b"r.txt", dims, None, lab.ctypes.data_as(C.POINTER(C.c_uint8)))
        assert rc == 0 and list(dims) == [3, 2, 2]
        assert list(lab) == [0, 0, 1, 2, 2, 2, 3, 4, 2, 2, 2, 2], list(lab)
        open("bad.txt", "w").write("0 10 Water\n")
        rc = lib.ggems_phantom_labels(b"p.mhd", b"bad.txt", dims, None, lab.ctypes.data_as(C.POINTER(C.c_uint8)))
        assert rc != 0 and b"range data file" in lib.ggems_last_error()
        print("ok")
    ''', tmp_path)


def test_errors_raise_with_ggems_messages(tmp_path):
    _run(r'''
        import ggems_b200 as gg
        src = gg.GGEMSXRaySource("s")
        for call in (lambda: src.set_position(0, 0, 0, "furlong"),
                     lambda: src.set_source_particle_type("neutron"),
                     lambda: gg.GGEMSCTSystem("c").set_ct_type("spiral"),
                     lambda: gg.GGEMSProcessesManager().set_cross_section_table_energy_min(10.0, "eV"),
                     lambda: gg.GGEMSMaterialsDatabaseManager().set_materials("/nonexistent/materials.txt")):
            try:
                call()
            except gg.GGEMSError as e:
                assert "[GGEMS" in str(e), str(e)
            else:
                raise AssertionError("no error raised")
        g = gg.GGEMS()
        try:
            g.initialize(1)
        except gg.GGEMSError as e:
            assert "Materials are not loaded" in str(e)
        else:
            raise AssertionError("initialize without materials did not fail")
        print("ok")
    ''', tmp_path)


def test_polyenergetic_spectrum_file_roundtrip(tmp_path):
    """SetPolyenergy + FillEnergy: cdf normalised, last energy repeated."""
    _run(r'''
        import ctypes as C, numpy as np
        import ggems_b200 as gg
        from ggems_b200 import workloads, abi
        from ggems_b200.api import lib
        path = workloads.write_spectrum("spec.dat")
        gg.GGEMSMaterialsDatabaseManager().set_materials(workloads.MATERIALS)
        s = gg.GGEMSXRaySource("s")
        s.set_source_particle_type("gamma"); s.set_number_of_particles(10)
        s.set_position(-1000, 0, 0, "mm"); s.set_rotation(0, 0, 0, "deg")
        s.set_beam_aperture(5.0, "deg"); s.set_focal_spot_size(0, 0, 0, "mm"); s.set_polyenergy(path)
        gg.GGEMSSourceManager().initialize(1)
        d = abi.gg_source(); assert lib.ggems_source_descriptor(0, C.byref(d), None) == 0
        n = d.number_of_energy_bins
        assert n == 111 and d.is_interp == 1
        cdf = np.ctypeslib.as_array(d.energy_cdf, (n + 1,)); spec = np.ctypeslib.as_array(d.energy_spectrum, (n + 1,))
        assert cdf[0] == 0.0 and cdf[-1] == 1.0 and np.all(np.diff(cdf) >= 0)
        assert spec[-1] == spec[-2] and abs(spec[0] - 0.010) < 1e-9
        print("ok")
    ''', tmp_path)


def test_dosimetry_tle_flag_reaches_the_scene(tmp_path):
    """dose_tle_navigator(True) on a voxelized phantom marks its dose map TLE and
    ships the attenuation tables with the navigator."""
    _run(r'''
        import ctypes as C, numpy as np
        from ggems_b200 import workloads, abi
        from ggems_b200 import (GGEMSMaterialsDatabaseManager, GGEMSVoxelizedPhantom, GGEMSDosimetryCalculator,
                                GGEMSProcessesManager, GGEMSRangeCutsManager, GGEMSXRaySource, GGEMS)
        import scenes
        mhd, rng = workloads.water_files(".", 16, 4.0)
        GGEMSMaterialsDatabaseManager().set_materials(scenes.MATERIALS)
        ph = GGEMSVoxelizedPhantom("phantom")
        ph.set_phantom(mhd, rng)
        ph.set_rotation(0.0, 0.0, 0.0, "deg")
        ph.set_position(0.0, 0.0, 0.0, "mm")
        dose = GGEMSDosimetryCalculator()
        dose.attach_to_navigator("phantom")
        dose.set_output_basename("dose")
        dose.set_tle(True)
        pm = GGEMSProcessesManager()
        for p in ("Compton", "Photoelectric", "Rayleigh"):
            pm.add_process(p, "gamma", "all")
        GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
        s = GGEMSXRaySource("src")
        s.set_source_particle_type("gamma")
        s.set_number_of_particles(1000)
        s.set_position(-1000.0, 0.0, 0.0, "mm")
        s.set_rotation(0.0, 0.0, 0.0, "deg")
        s.set_beam_aperture(10.0, "deg")
        s.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
        s.set_monoenergy(60.0, "keV")
        from ggems_b200.api import lib
        lib.ggems_host_scene.restype = C.POINTER(abi.gg_scene)
        sc = lib.ggems_host_scene().contents
        assert sc.number_of_dose_maps == 1 and sc.dose_maps[0].tle == 1
        t = sc.tables[0]
        bins = np.ctypeslib.as_array(t.attenuation_energy_bins, (abi.GG_ATTENUATION_BINS,))
        ref = scenes.Tables(["Water"])
        assert np.array_equal(bins, ref.attenuation_energy_bins)
        mu_en = np.ctypeslib.as_array(t.mu_en, (abi.GG_ATTENUATION_BINS,))
        assert np.array_equal(mu_en.view(np.uint32), ref.mu_en.view(np.uint32))
        print("ok")
    ''', tmp_path)


def test_world_reaches_the_scene(tmp_path):
    """GGEMSWorld's grid and switches reach the scene in mm; missing
    dimensions raise GGEMSWorld::CheckParameters's message."""
    out = _run(r'''
        import ctypes as C
        from ggems_b200 import workloads, abi
        from ggems_b200 import (GGEMSMaterialsDatabaseManager, GGEMSVoxelizedPhantom, GGEMSProcessesManager,
                                GGEMSRangeCutsManager, GGEMSXRaySource, GGEMSWorld)
        import scenes
        mhd, rng = workloads.water_files(".", 16, 4.0)
        GGEMSMaterialsDatabaseManager().set_materials(scenes.MATERIALS)
        ph = GGEMSVoxelizedPhantom("phantom")
        ph.set_phantom(mhd, rng)
        ph.set_rotation(0.0, 0.0, 0.0, "deg")
        ph.set_position(0.0, 0.0, 0.0, "mm")
        pm = GGEMSProcessesManager()
        pm.add_process("Compton", "gamma", "all")
        GGEMSRangeCutsManager().set_cut("gamma", 0.1, "mm", "all")
        s = GGEMSXRaySource("src")
        s.set_source_particle_type("gamma")
        s.set_number_of_particles(1000)
        s.set_position(-1000.0, 0.0, 0.0, "mm")
        s.set_rotation(0.0, 0.0, 0.0, "deg")
        s.set_beam_aperture(10.0, "deg")
        s.set_focal_spot_size(0.0, 0.0, 0.0, "mm")
        s.set_monoenergy(60.0, "keV")
        from ggems_b200.api import lib
        lib.ggems_host_scene.restype = C.POINTER(abi.gg_scene)
        w = GGEMSWorld()
        lib.ggems_clear_error()
        assert not lib.ggems_host_scene()
        assert b"Dimensions of world have to be set" in lib.ggems_last_error()
        w.set_dimensions(200, 100, 50)
        w.set_element_sizes(1.0, 2.0, 0.5, "cm")
        w.photon_tracking(True)
        w.momentum(True)
        w.set_output_basename("out/w")
        sc = lib.ggems_host_scene().contents
        g = sc.world.contents
        assert list(g.dimensions) == [200, 100, 50]
        assert list(g.sizes) == [10.0, 20.0, 5.0]
        assert (g.photon_tracking, g.energy_tracking, g.energy_squared_tracking, g.momentum) == (1, 0, 0, 1)
        print("ok")
    ''', tmp_path)
    assert "ok" in out
