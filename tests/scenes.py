"""Synthetic scenes for the parity tests, built directly in the C-ABI form
(``include/ggems_b200.h``) with tables from the oracle's table builder.

Geometry matrices follow GGEMSGeometryTransformation
(src/maths/GGEMSGeometryTransformation.cc:143-336): the matrix starts as the
object's axis matrix and each SetRotation / SetTranslation call left-multiplies
it, in float32 with the reference's summation order.  cos/sin come from the
host libm (the functions the reference's host code calls).
"""

import ctypes as C
import ctypes.util
import os

import numpy as np

from ggems_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DATA = os.path.join(ROOT, "ggems_b200", "data")
MATERIALS = os.path.join(DATA, "materials.txt")
PHYSICS = os.path.join(DATA, "physics_data.bin")

_libm = C.CDLL(ctypes.util.find_library("m"))
_libm.cosf.restype = C.c_float
_libm.cosf.argtypes = [C.c_float]
_libm.sinf.restype = C.c_float
_libm.sinf.argtypes = [C.c_float]

F = np.float32
DEG = F(F(3.141592653589793238463) / F(180.0))  # GGEMSSystemOfUnits.hh:80
MEV = F(1.0)
KEV = F(1.0e-3)

SOURCE_AXIS = ((0.0, 0.0, -1.0), (0.0, 1.0, 0.0), (1.0, 0.0, 0.0))    # GGEMSXRaySource.cc:50-56
PHANTOM_AXIS = ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.0, 0.0, 1.0))   # GGEMSVoxelizedSolid.cc:56-62
DETECTOR_AXIS = ((0.0, 0.0, 1.0), (0.0, 1.0, 0.0), (-1.0, 0.0, 0.0))  # GGEMSSolidBox.cc:77-83


def _mat_mul(a, b):
    """GGfloat44MultGGfloat44 in float32, products summed left to right."""
    out = np.zeros((4, 4), np.float32)
    for i in range(4):
        for j in range(4):
            s = F(a[i, 0] * b[0, j])
            s = F(s + F(a[i, 1] * b[1, j]))
            s = F(s + F(a[i, 2] * b[2, j]))
            s = F(s + F(a[i, 3] * b[3, j]))
            out[i, j] = s
    return out


def geometry_matrix(axis, ops):
    """ops: sequence of ("rotation", (rx, ry, rz) rad) / ("translation", (x, y, z) mm) in call order."""
    m = np.eye(4, dtype=np.float32)
    m[:3, :3] = np.array(axis, np.float32)
    for kind, v in ops:
        v = [F(x) for x in v]
        if kind == "translation":
            t = np.eye(4, dtype=np.float32)
            t[:3, 3] = v
            m = _mat_mul(t, m)
        else:
            c, s = F(_libm.cosf(v[0])), F(_libm.sinf(v[0]))
            rx = np.array([[1, 0, 0, 0], [0, c, -s, 0], [0, s, c, 0], [0, 0, 0, 1]], np.float32)
            c, s = F(_libm.cosf(v[1])), F(_libm.sinf(v[1]))
            ry = np.array([[c, 0, s, 0], [0, 1, 0, 0], [-s, 0, c, 0], [0, 0, 0, 1]], np.float32)
            c, s = F(_libm.cosf(v[2])), F(_libm.sinf(v[2]))
            rz = np.array([[c, -s, 0, 0], [s, c, 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], np.float32)
            r = _mat_mul(rz, _mat_mul(ry, rx))
            m = _mat_mul(r, m)
    return m


def _oracle_lib():
    path = os.path.join(ROOT, "oracle", "_build", "libgg_oracle.so")
    if not os.path.exists(path):
        import subprocess
        import sys
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "build.py")])
    lib = C.CDLL(path)
    lib.gg_oracle_run.restype = C.c_int
    lib.gg_oracle_run.argtypes = [C.POINTER(abi.gg_scene), C.POINTER(abi.gg_source), C.c_uint64,
                                  C.POINTER(C.c_uint32), C.POINTER(abi.gg_particle_buffers),
                                  C.POINTER(abi.gg_tally_buffers), C.c_int]
    return lib


_ORACLE = None


def oracle():
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _oracle_lib()
        pp = load_physics()
        arrs = [np.ascontiguousarray(pp["rayleigh_pp%d" % i]) for i in range(9)]
        _ORACLE._pp_keep = arrs
        ptrs = (C.POINTER(C.c_float) * 9)(*[abi.ptr(a, C.c_float) for a in arrs])
        _ORACLE.gg_oracle_set_rayleigh_fit(ptrs)
    return _ORACLE


_ORACLE_FP64 = None


def oracle_fp64():
    """The oracle's transport restatement built in FP64 (libgg_oracle_fp64.so):
    the precision reference the FP32 results are compared with."""
    global _ORACLE_FP64
    if _ORACLE_FP64 is None:
        oracle()  # builds both libraries when missing
        lib = C.CDLL(os.path.join(ROOT, "oracle", "_build", "libgg_oracle_fp64.so"))
        lib.gg_oracle_run.restype = C.c_int
        lib.gg_oracle_run.argtypes = _ORACLE.gg_oracle_run.argtypes
        pp = load_physics()
        arrs = [np.ascontiguousarray(pp["rayleigh_pp%d" % i]) for i in range(9)]
        lib._pp_keep = arrs
        ptrs = (C.POINTER(C.c_float) * 9)(*[abi.ptr(a, C.c_float) for a in arrs])
        lib.gg_oracle_set_rayleigh_fit(ptrs)
        _ORACLE_FP64 = lib
    return _ORACLE_FP64


def load_physics(path=PHYSICS):
    raw = open(path, "rb").read()
    assert raw[:8] == b"GGPHYS01"
    n = int(np.frombuffer(raw, np.uint32, 1, 8)[0])
    off, out = 12, {}
    for _ in range(n):
        name = raw[off:off + 32].split(b"\0")[0].decode()
        code, cnt = np.frombuffer(raw, np.uint32, 2, off + 32)
        off += 40
        dt = {0: np.float32, 1: np.int32, 2: np.int16, 3: np.uint8}[int(code)]
        arr = np.frombuffer(raw, dt, int(cnt), off)
        off += arr.nbytes
        out[name] = arr
    return out


def rayleigh_fit():
    pd = load_physics()
    return np.ascontiguousarray(np.stack([pd["rayleigh_pp%d" % i] for i in range(9)]).astype(np.float32))


class Tables:
    """One navigator's physics tables (oracle restatement of the host builders)."""

    def __init__(self, materials, number_of_bins=220, min_energy=1.0 * KEV, max_energy=1.0 * MEV,
                 processes=(0, 1, 2), photon_cut=0.1, materials_file=MATERIALS, builder="oracle"):
        """builder: "oracle" (the restatement) or "reference" (GGEMS's own host
        code, oracle/_ref/libgg_ref_tables.so; bit-identical, see
        tests/test_tables.py) for the material and cross-section tables."""
        lib = oracle()
        nm, nb = len(materials), number_of_bins
        self.materials = list(materials)
        self.energy_bins = np.zeros(nb, np.float32)
        self.cross_sections = np.zeros(3 * nm * nb, np.float32)
        self.rayleigh = np.zeros(101 * nb, np.float32)
        self.density = np.zeros(nm, np.float32)
        self.photon_cut = np.zeros(nm, np.float32)
        self.n_elements = np.zeros(nm, np.int32)
        self.offset = np.zeros(nm, np.int32)
        self.Z = np.zeros(nm * 32, np.uint8)
        self.atom_density = np.zeros(nm * 32, np.float32)
        total = C.c_int32(0)
        names = (C.c_char_p * nm)(*[m.encode() for m in materials])
        procs = (C.c_int * 3)(*processes)
        if builder == "reference":
            ref = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libgg_ref_tables.so"))
            build = lambda *a: ref.gg_ref_build_tables(a[0], *a[2:])  # noqa: E731  (no physics-data file)
        else:
            build = lib.gg_oracle_build_tables
        rc = build(
            MATERIALS.encode() if materials_file is None else materials_file.encode(), PHYSICS.encode(), names, nm, nb,
            C.c_float(min_energy), C.c_float(max_energy), procs, len(processes), C.c_float(photon_cut),
            abi.ptr(self.energy_bins, C.c_float), abi.ptr(self.cross_sections, C.c_float),
            abi.ptr(self.rayleigh, C.c_float), abi.ptr(self.density, C.c_float), abi.ptr(self.photon_cut, C.c_float),
            abi.ptr(self.n_elements, C.c_int32), abi.ptr(self.offset, C.c_int32), abi.ptr(self.Z, C.c_uint8),
            abi.ptr(self.atom_density, C.c_float), C.byref(total))
        assert rc == 0, "gg_oracle_build_tables failed"
        self.total = total.value
        # GGEMSAttenuations (mu, mu_en on 220 bins), built for every navigator as GGEMS does
        self.attenuation_energy_bins = np.zeros(abi.GG_ATTENUATION_BINS, np.float32)
        self.mu = np.zeros(nm * abi.GG_ATTENUATION_BINS, np.float32)
        self.mu_en = np.zeros(nm * abi.GG_ATTENUATION_BINS, np.float32)
        lib.gg_oracle_build_attenuations.restype = C.c_int
        rc = lib.gg_oracle_build_attenuations(
            MATERIALS.encode() if materials_file is None else materials_file.encode(), PHYSICS.encode(), names, nm,
            abi.ptr(self.attenuation_energy_bins, C.c_float), abi.ptr(self.mu, C.c_float),
            abi.ptr(self.mu_en, C.c_float))
        assert rc == 0, "gg_oracle_build_attenuations failed"
        pid = list(processes) + [0] * (3 - len(processes))
        self.struct = abi.gg_physics_tables(
            nb, nm, len(processes), (C.c_int32 * 3)(*pid), abi.ptr(self.energy_bins, C.c_float),
            abi.ptr(self.cross_sections, C.c_float),
            abi.ptr(self.rayleigh, C.c_float) if 2 in processes else C.cast(None, abi.FP),
            abi.ptr(self.density, C.c_float), abi.ptr(self.photon_cut, C.c_float),
            abi.ptr(self.n_elements, C.c_int32), abi.ptr(self.offset, C.c_int32), abi.ptr(self.Z, C.c_uint8),
            abi.ptr(self.atom_density, C.c_float), self.total, abi.ptr(self.attenuation_energy_bins, C.c_float),
            abi.ptr(self.mu_en, C.c_float))


def _obb(matrix, half):
    o = abi.gg_obb()
    o.matrix[:] = [float(x) for x in matrix.reshape(-1)]
    o.border_min[:] = [float(-h) for h in half]
    o.border_max[:] = [float(h) for h in half]
    return o


class Scene:
    """A gg_scene plus the numpy storage it points into."""

    def __init__(self):
        self.tables = []
        self.solids = []
        self.dose_maps = []
        self.histogram_sizes = []
        self.meshes = []
        self.world = None
        self._keep = []

    def add_tables(self, tables):
        self.tables.append(tables)
        return len(self.tables) - 1

    def add_voxelized(self, labels, voxel_size, navigator, ops=(), dose=None):
        """labels: uint8 array shaped (nz, ny, nx).  dose: dict with dosel size or None."""
        labels = np.ascontiguousarray(labels, np.uint8)
        self._keep.append(labels)
        nz, ny, nx = labels.shape
        vs = [F(v) for v in voxel_size]
        # GGEMSMHDImage::Read (src/io/GGEMSMHDImage.cc:209-213)
        half = [F(F(F(n) * v) * F(0.5)) for n, v in zip((nx, ny, nz), vs)]
        m = geometry_matrix(PHANTOM_AXIS, ops)
        s = abi.gg_solid()
        s.type = abi.GG_SOLID_VOXELIZED
        s.navigator = navigator
        s.obb = _obb(m, half)
        s.threshold = 0.0
        s.number_of_voxels[:] = [nx, ny, nz]
        s.voxel_sizes[:] = [float(v) for v in vs]
        s.labels = abi.ptr(labels, C.c_uint8)
        s.histogram = -1
        s.scatter_histogram = -1
        s.dose_map = -1
        if dose is not None:
            s.dose_map = self._add_dose(s, dose)
        self.solids.append(s)
        return len(self.solids) - 1

    def _add_dose(self, solid, dose):
        # GGEMSDosimetryCalculator::Initialize (src/navigators/GGEMSDosimetryCalculator.cc:435-530)
        d = abi.gg_dose_map()
        size = [F(v) for v in dose.get("dosel_size", list(solid.voxel_sizes))]
        d.size_of_dosels[:] = [float(v) for v in size]
        d.inv_size_of_dosels[:] = [float(F(F(1.0) / v)) for v in size]
        d.border_min[:] = list(solid.obb.border_min)
        d.border_max[:] = list(solid.obb.border_max)
        n = [int(F(F(F(solid.obb.border_max[i]) - F(solid.obb.border_min[i])) / size[i])) for i in range(3)]
        d.number_of_dosels[:] = n
        d.total_number_of_dosels = n[0] * n[1] * n[2]
        d.slice_number_of_dosels = n[0] * n[1]
        d.record_edep_squared = 1
        d.record_hit = 1
        d.record_photon_tracking = 1 if dose.get("photon_tracking") else 0
        d.tle = 1 if dose.get("tle") else 0
        self.dose_maps.append(d)
        return len(self.dose_maps) - 1

    def add_meshed(self, stl_path, navigator, ops=(), depth=4, dose=None):
        """GGEMSMeshedPhantom: STL triangles moved by the solid's transformation (axis
        identity, calls in `ops` order), octree of `depth` levels (oracle restatement of
        GGEMSMeshedSolid / GGEMSOctree).  dose: dict with "dosel_size" (required) or None."""
        lib = oracle()
        nt, nn = C.c_int32(), C.c_int32()
        assert lib.gg_oracle_mesh_counts(stl_path.encode(), depth, C.byref(nt), C.byref(nn)) == 0
        m = geometry_matrix(PHANTOM_AXIS, ops)
        tri = np.zeros(nt.value * abi.GG_TRIANGLE_FLOATS, np.float32)
        nodes = np.zeros(nn.value * 6, np.float32)
        first = np.zeros(nn.value + 1, np.int32)
        order = np.zeros(max(nt.value, 1), np.int32)
        bmin, bmax = np.zeros(3, np.float32), np.zeros(3, np.float32)
        mat = np.ascontiguousarray(m.reshape(-1), np.float32)
        rc = lib.gg_oracle_build_mesh(stl_path.encode(), abi.ptr(mat, C.c_float), depth, abi.ptr(tri, C.c_float),
                                      abi.ptr(nodes, C.c_float), abi.ptr(first, C.c_int32), abi.ptr(order, C.c_int32),
                                      abi.ptr(bmin, C.c_float), abi.ptr(bmax, C.c_float))
        assert rc == 0, "gg_oracle_build_mesh failed"
        self._keep += [tri, nodes, first, order]
        s = abi.gg_solid()
        s.type = abi.GG_SOLID_MESHED
        s.navigator = navigator
        o = abi.gg_obb()
        o.matrix[:] = [float(x) for x in np.eye(4, dtype=np.float32).reshape(-1)]
        o.border_min[:] = [float(x) for x in bmin]
        o.border_max[:] = [float(x) for x in bmax]
        s.obb = o
        s.threshold = 0.0
        s.histogram = -1
        s.scatter_histogram = -1
        s.dose_map = -1
        s.number_of_triangles = nt.value
        s.triangles = abi.ptr(tri, C.c_float)
        s.number_of_nodes = nn.value
        s.nodes = abi.ptr(nodes, C.c_float)
        s.node_first = abi.ptr(first, C.c_int32)
        s.node_triangles = abi.ptr(order, C.c_int32)
        self.meshes.append(dict(triangles=tri, nodes=nodes, first=first, order=order, bmin=bmin, bmax=bmax))
        if dose is not None:
            s.dose_map = self._add_dose(s, dose)
        self.solids.append(s)
        return len(self.solids) - 1

    def add_flat_detector(self, navigator, elements, element_size, sdd, sid, threshold, scatter=True,
                          extra_rotation=None):
        """One-module flat GGEMSCTSystem (src/navigators/GGEMSCTSystem.cc:175-300)."""
        ex, ey, ez = elements
        sx, sy, sz = [F(v) for v in element_size]
        box = [F(F(ex) * sx), F(F(ey) * sy), F(F(ez) * sz)]
        half = [F(b * F(0.5)) for b in box]
        # InitializeFlatGeometry: module (0, 0) of a 1x1 system.
        gx = F(F(sdd) - F(sid))
        gy = F(F(F(ey) * sy) * F(F(0.0) + F(0.5) * F(F(1.0) - F(1.0))))
        gz = F(F(F(ex) * sx) * F(F(0.0) + F(0.5) * F(F(1.0) - F(1.0))))
        ops = [("rotation", (0.0, 0.0, 0.0)), ("translation", (gx, gy, gz))]
        if extra_rotation is not None:
            ops.append(("rotation", extra_rotation))
        m = geometry_matrix(DETECTOR_AXIS, ops)
        s = abi.gg_solid()
        s.type = abi.GG_SOLID_BOX
        s.navigator = navigator
        s.obb = _obb(m, half)
        s.threshold = float(threshold)
        s.virtual_element_number[:] = [ex, ey, ez]
        s.box_size[:] = [float(b) for b in box]
        s.histogram = len(self.histogram_sizes)
        self.histogram_sizes.append(ex * ey)
        s.scatter_histogram = -1
        if scatter:
            s.scatter_histogram = len(self.histogram_sizes)
            self.histogram_sizes.append(ex * ey)
        s.dose_map = -1
        self.solids.append(s)
        return len(self.solids) - 1

    def struct(self):
        self._t = (abi.gg_physics_tables * len(self.tables))(*[t.struct for t in self.tables])
        self._s = (abi.gg_solid * len(self.solids))(*self.solids)
        self._d = (abi.gg_dose_map * max(1, len(self.dose_maps)))(*self.dose_maps)
        self._h = np.array(self.histogram_sizes + [0], np.int32)
        self._pp = rayleigh_fit()
        world = C.pointer(self.world) if self.world is not None else C.cast(None, C.POINTER(abi.gg_world))
        return abi.gg_scene(len(self.tables), self._t, len(self.solids), self._s, len(self.dose_maps), self._d,
                            len(self.histogram_sizes), abi.ptr(self._h, C.c_int32), abi.ptr(self._pp, C.c_float),
                            world)

    def set_world(self, dimensions, sizes, photon=True, energy=True, energy_squared=True, momentum=True):
        """GGEMSWorld grid (centred on the origin)."""
        w = abi.gg_world()
        w.dimensions[:] = list(dimensions)
        w.sizes[:] = [float(F(v)) for v in sizes]
        w.photon_tracking, w.energy_tracking = int(photon), int(energy)
        w.energy_squared_tracking, w.momentum = int(energy_squared), int(momentum)
        self.world = w

    def tallies(self):
        ws = int(np.prod(list(self.world.dimensions))) if self.world is not None else 0
        return abi.Tallies(self.histogram_sizes, [d.total_number_of_dosels for d in self.dose_maps], ws)


class XRaySource:
    """GGEMSXRaySource (src/sources/GGEMSXRaySource.cc) in C-ABI form."""

    def __init__(self, position=(-1000.0, 0.0, 0.0), rotation=(0.0, 0.0, 0.0), aperture_deg=10.0,
                 focal=(0.0, 0.0, 0.0), monoenergy=None, spectrum=None, order=("position", "rotation")):
        ops = []
        for o in order:
            ops.append(("translation", position) if o == "position" else ("rotation", rotation))
        self.matrix = geometry_matrix(SOURCE_AXIS, ops)
        if monoenergy is not None:
            energies, weights, interp = [F(monoenergy)], [1.0], 0
        else:
            energies, weights = spectrum
            energies = [F(e) for e in energies]
            interp = 1
        self.spectrum, self.cdf = fill_energy(energies, weights)
        s = abi.gg_source()
        s.type = abi.GG_SOURCE_XRAY
        s.particle_type = 0
        s.matrix[:] = [float(x) for x in self.matrix.reshape(-1)]
        s.beam_aperture = float(F(F(aperture_deg) * DEG))
        s.focal_spot_size[:] = [float(f) for f in focal]
        s.number_of_energy_bins = len(energies)
        s.energy_spectrum = abi.ptr(self.spectrum, C.c_float)
        s.energy_cdf = abi.ptr(self.cdf, C.c_float)
        s.is_interp = interp
        self.struct = s


def fill_energy(energies, weights):
    """GGEMSSource::FillEnergy (src/sources/GGEMSSource.cc:265-316)."""
    n = len(energies)
    spec = np.zeros(n + 1, np.float32)
    cdf = np.zeros(n + 1, np.float32)
    total = 0.0
    for w in weights:
        total += float(w)
    tmp = [0.0] + [float(w) for w in weights]
    spec[:n] = energies
    spec[n] = spec[n - 1]
    for i in range(1, n + 1):
        tmp[i] = tmp[i] + tmp[i - 1]
        cdf[i] = np.float32(tmp[i] / total)
    cdf[n] = 1.0
    return spec, cdf


def seed_states(seed, slots=abi.GG_MAXIMUM_PARTICLES, skip=0):
    """GGEMSPseudoRandomGenerator::InitializeSeeds with numpy's MT19937 (same
    generator as std::mt19937 for a 32-bit seed)."""
    from numpy.random import MT19937
    bg = MT19937(0)
    bg._legacy_seeding(seed)
    raw = bg.random_raw((skip + slots) * 4)[skip * 4:].astype(np.uint32).reshape(slots, 4)
    st = np.zeros((5, abi.GG_MAXIMUM_PARTICLES), np.uint32)
    st[0, :slots] = raw[:, 0]
    st[1, :slots] = raw[:, 1]
    st[2, :slots] = raw[:, 2]
    st[3, :slots] = raw[:, 3]
    return st


def water_box_scene(n=64, voxel=2.0, dose=True, photon_tracking=False, tle=False):
    """C1: 64^3 water, 2 mm voxels, dose map on the phantom grid."""
    sc = Scene()
    t = sc.add_tables(Tables(["Water"]))
    labels = np.zeros((n, n, n), np.uint8)
    sc.add_voxelized(labels, (voxel, voxel, voxel), t,
                     dose={"photon_tracking": photon_tracking, "tle": tle} if dose else None)
    return sc


def ellipsoid_phantom(n, voxel, seed=1, n_bones=None):
    """C2 generator: air / water ellipsoid / bone ellipsoids, labels (nz, ny, nx)."""
    from ggems_b200 import workloads
    return workloads.cbct_labels(n, voxel, seed, n_bones)


def mesh_phantom_scene(path, subdivisions=2, n_inner=2, depth=3, dose=False, ops=(), seed=1, material="Water"):
    """C4-style meshed phantom (body ellipsoid + inner cavities) written to `path` as STL."""
    from ggems_b200 import workloads
    workloads.write_stl(path, workloads.body_mesh(subdivisions, max(subdivisions - 1, 0), n_inner, seed))
    sc = Scene()
    t = sc.add_tables(Tables([material]))
    sc.add_meshed(path, t, ops=ops, depth=depth, dose={"dosel_size": (10.0, 10.0, 10.0)} if dose else None)
    return sc


def synthetic_spectrum():
    """120 kVp spectrum, 1 keV bins 10-120 keV (ggems_b200.workloads.xray_spectrum),
    with energies rounded through the spectrum file's text format."""
    from ggems_b200 import workloads
    e, w = workloads.xray_spectrum()
    return [F(float("%.6f" % x)) for x in e], [float("%.9e" % x) for x in w]


def cbct_scene(n=256, voxel=1.0, elements=(512, 512, 1), element_size=(0.8, 0.8, 10.0), seed=1):
    """C2: ellipsoid phantom + one-module flat detector at SDD 1500 / SID 1000."""
    sc = Scene()
    t_ph = sc.add_tables(Tables(["Air", "Water", "Bone185"]))
    labels = ellipsoid_phantom(n, voxel, seed)
    sc.add_voxelized(labels, (voxel, voxel, voxel), t_ph)
    t_det = sc.add_tables(Tables(["GOS"]))
    sc.add_flat_detector(t_det, elements, element_size, sdd=1500.0, sid=1000.0, threshold=F(10.0) * KEV)
    return sc


def cbct_api_scene(n=256, voxel=1.0, seed=1, aperture_deg=11.0, builder="oracle"):
    """The CBCT projection exactly as the GGEMS-API configuration builds it
    (phantom rotation then position calls, detector rotation call; 120 kVp
    spectrum through its file format; source at (-1000, 0, 0) mm): (scene,
    source).  tests/test_host_api.py checks it field by field against the
    scene the API prepares."""
    from ggems_b200 import workloads
    sc = Scene()
    t = sc.add_tables(Tables(["Air", "Water", "Bone185"], builder=builder))
    sc.add_voxelized(workloads.cbct_labels(n, voxel, seed), (voxel, voxel, voxel), t,
                     ops=[("rotation", (0.0, 0.0, 0.0)), ("translation", (0.0, 0.0, 0.0))])
    td = sc.add_tables(Tables(["GOS"], builder=builder))
    sc.add_flat_detector(td, (512, 512, 1), (0.8, 0.8, 10.0), 1500.0, 1000.0, F(10.0) * KEV,
                         extra_rotation=(0.0, 0.0, 0.0))
    return sc, XRaySource(spectrum=synthetic_spectrum(), aperture_deg=aperture_deg)


_libm.asinf.restype = C.c_float
_libm.asinf.argtypes = [C.c_float]
_libm.sqrtf.restype = C.c_float
_libm.sqrtf.argtypes = [C.c_float]


def add_curved_detector(sc, navigator, modules, elements, element_size, sdd, sid, threshold, scatter=True,
                        extra_rotation=None):
    """GGEMSCTSystem::InitializeCurvedGeometry (src/navigators/GGEMSCTSystem.cc:131-172) in float32."""
    mx, my = modules
    ex, ey, ez = elements
    sx, sy, sz = [F(v) for v in element_size]
    sdd, sid = F(sdd), F(sid)
    c = F(F(F(ey) * sy) * F(0.5))
    rho = F(_libm.sqrtf(F(F(sdd * sdd) + F(c * c))))
    alpha = F(F(2.0) * F(_libm.asinf(F(c / rho))))
    ox, oy, px, py = F(-sid), F(0.0), F(sdd - sid), F(0.0)
    first = len(sc.solids)
    for j in range(my):
        step = F(alpha * F(F(j) + F(F(0.5) * F(F(1.0) - F(my)))))
        cs, sn = F(_libm.cosf(step)), F(_libm.sinf(step))
        gx = F(F(F(F(px - ox) * cs) - F(F(py - oy) * sn)) + ox)
        gy = F(F(F(F(px - ox) * sn) + F(F(py - oy) * cs)) + oy)
        for i in range(mx):
            gz = F(F(F(F(ex) * sx)) * F(F(i) + F(F(0.5) * F(F(1.0) - F(mx)))))
            ops = [("rotation", (0.0, 0.0, float(step))), ("translation", (float(gx), float(gy), float(gz)))]
            if extra_rotation is not None:
                ops.append(("rotation", extra_rotation))
            m = geometry_matrix(DETECTOR_AXIS, ops)
            box = [F(F(ex) * sx), F(F(ey) * sy), F(F(ez) * sz)]
            half = [F(b * F(0.5)) for b in box]
            s = abi.gg_solid()
            s.type = abi.GG_SOLID_BOX
            s.navigator = navigator
            s.obb = _obb(m, half)
            s.threshold = float(threshold)
            s.virtual_element_number[:] = [ex, ey, ez]
            s.box_size[:] = [float(b) for b in box]
            s.histogram = len(sc.histogram_sizes)
            sc.histogram_sizes.append(ex * ey)
            s.scatter_histogram = -1
            if scatter:
                s.scatter_histogram = len(sc.histogram_sizes)
                sc.histogram_sizes.append(ex * ey)
            s.dose_map = -1
            sc.solids.append(s)
    return first


class VoxelizedSource:
    """GGEMSVoxelizedSource (src/sources/GGEMSVoxelizedSource.cc:287-380) in C-ABI form."""

    def __init__(self, activity, voxel_size, position=(0.0, 0.0, 0.0), monoenergy=None, spectrum=None):
        activity = np.ascontiguousarray(activity, np.float32)
        nz, ny, nx = activity.shape
        flat = activity.reshape(-1)
        active = np.nonzero(flat != 0.0)[0]
        na = len(active)
        self.index = np.zeros(na + 1, np.int32)
        self.index[1:] = active
        self.index[na] = self.index[na - 1]
        tmp = np.zeros(na + 1, np.float32)
        tmp[1:] = flat[active]
        total = F(0.0)
        for v in flat[active]:
            total = F(total + v)
        cum = np.cumsum(tmp, dtype=np.float32)
        self.cdf = (cum / total).astype(np.float32)
        self.cdf[na] = 1.0
        self.matrix = geometry_matrix(PHANTOM_AXIS, [("translation", position)])
        if monoenergy is not None:
            energies, weights, interp = [F(monoenergy)], [1.0], 0
        else:
            energies, weights = spectrum
            interp = 1
        self.spectrum, self.energy_cdf = fill_energy([F(e) for e in energies], weights)
        s = abi.gg_source()
        s.type = abi.GG_SOURCE_VOXELIZED
        s.particle_type = 0
        s.matrix[:] = [float(x) for x in self.matrix.reshape(-1)]
        s.number_of_energy_bins = len(energies)
        s.energy_spectrum = abi.ptr(self.spectrum, C.c_float)
        s.energy_cdf = abi.ptr(self.energy_cdf, C.c_float)
        s.is_interp = interp
        s.number_of_voxels[:] = [nx, ny, nz]
        vs = [F(v) for v in voxel_size]
        s.voxel_sizes[:] = [float(v) for v in vs]
        s.border_min[:] = [float(F(F(-F(n) * v) * F(0.5))) for n, v in zip((nx, ny, nz), vs)]
        s.number_of_activity_bins = na + 1
        s.activity_index = abi.ptr(self.index, C.c_int32)
        s.activity_cdf = abi.ptr(self.cdf, C.c_float)
        self.struct = s


def hot_spot_activity(n=16, seed=2):
    rng = np.random.default_rng(seed)
    a = np.zeros((n, n, n), np.float32)
    c = n // 2
    a[c - 3:c + 3, c - 2:c + 4, c - 4:c + 2] = 1.0
    idx = rng.integers(0, n, (20, 3))
    a[idx[:, 0], idx[:, 1], idx[:, 2]] = rng.uniform(0.5, 4.0, 20).astype(np.float32)
    return a
