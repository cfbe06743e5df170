"""Synthetic inputs for the benchmark workloads, written in GGEMS's file
formats (MHD phantom + range-to-material file, "E_MeV intensity" spectrum).

* ``cbct_phantom``: 256^3 CBCT phantom of 1 mm voxels: air background, a
  water ellipsoid with semi-axes 110/90/120 mm and 6-12 bone-like (1.85
  g/cm3) ellipsoids of semi-axes 5-25 mm with centres inside the body, from a
  seed.  Smaller grids scale the geometry with the grid extent.
* ``water_phantom``: the 64^3 all-water phantom of 2 mm voxels.
* ``xray_spectrum``: 120 kVp, 1 keV bins over 10-120 keV, Kramers-shaped
  ((120 - E)/E) and filtered by 2.5 mm of aluminium with GGEMS's own mu table.
"""

import os

import numpy as np

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
MATERIALS = os.path.join(DATA, "materials.txt")
PHYSICS = os.path.join(DATA, "physics_data.bin")


def load_physics(path=PHYSICS):
    """The arrays of physics_data.bin by name."""
    raw = open(path, "rb").read()
    if raw[:8] != b"GGPHYS01":
        raise ValueError("not a physics data file: " + path)
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


def cbct_labels(n=256, voxel=1.0, seed=1, n_bones=None):
    """uint8 labels (z, y, x): 0 air, 1 water, 2 bone."""
    rng = np.random.default_rng(seed)
    if n_bones is None:
        n_bones = int(rng.integers(6, 13))
    c = ((np.arange(n, dtype=np.float32) + 0.5) * voxel - n * voxel / 2.0).astype(np.float32)
    scale = n * voxel / 256.0
    a, b, cc = 110.0 * scale, 90.0 * scale, 120.0 * scale
    labels = np.zeros((n, n, n), np.uint8)
    zz = (c / cc) ** 2
    yy = (c / b) ** 2
    xx = (c / a) ** 2
    body = (zz[:, None, None] + yy[None, :, None] + xx[None, None, :]) <= 1.0
    labels[body] = 1
    for _ in range(n_bones):
        r = rng.uniform(5, 25, 3) * scale
        while True:
            p = rng.uniform(-1, 1, 3)
            if (p ** 2).sum() <= 1.0:
                break
        ctr = p * np.array([a, b, cc]) * 0.7
        bone = ((((c - ctr[2]) / r[2]) ** 2)[:, None, None] + (((c - ctr[1]) / r[1]) ** 2)[None, :, None] +
                (((c - ctr[0]) / r[0]) ** 2)[None, None, :]) <= 1.0
        labels[bone & body] = 2
    return labels


def write_mhd(path, array, spacing, element_type="MET_UCHAR"):
    """Write an MHD header + raw file (x fastest, array shaped (z, y, x))."""
    base = path[:-4] if path.endswith(".mhd") else path
    raw = base + ".raw"
    nz, ny, nx = array.shape
    with open(base + ".mhd", "w") as f:
        f.write("ObjectType = Image\nBinaryDataByteOrderMSB = False\nNDims = 3\n")
        f.write("ElementSpacing = %g %g %g\n" % tuple(spacing))
        f.write("DimSize = %d %d %d\n" % (nx, ny, nz))
        f.write("ElementType = %s\n" % element_type)
        f.write("ElementDataFile = %s\n" % os.path.basename(raw))
    np.ascontiguousarray(array).tofile(raw)
    return base + ".mhd"


def xray_spectrum():
    """(energies MeV, weights) of the 120 kVp / 2.5 mm Al spectrum."""
    pd = load_physics()
    nb, idx = pd["mu_nb_energy_bins"], pd["mu_index_energy"]
    data = pd["mu_data"].reshape(-1, 3)
    z = 13
    rows = data[idx[z]: idx[z] + nb[z]].astype(np.float64)
    energies = np.arange(10, 121, dtype=np.float64)  # keV
    mu = np.exp(np.interp(np.log(energies * 1e-3), np.log(rows[:, 0]), np.log(rows[:, 1])))
    w = np.clip(120.0 - energies, 0.0, None) / energies * np.exp(-mu * 2.699 * 0.25)
    w = w / w.sum()
    return energies * 1e-3, w


def write_spectrum(path):
    e, w = xray_spectrum()
    with open(path, "w") as f:
        for ei, wi in zip(e, w):
            f.write("%.6f %.9e\n" % (ei, wi))
    return path


def cbct_files(directory, n=256, voxel=1.0, seed=1):
    """Write the CBCT phantom, its range file and the spectrum; return their paths."""
    os.makedirs(directory, exist_ok=True)
    labels = cbct_labels(n, voxel, seed)
    mhd = write_mhd(os.path.join(directory, "cbct_phantom.mhd"), labels, (voxel, voxel, voxel))
    rng_file = os.path.join(directory, "cbct_range.txt")
    with open(rng_file, "w") as f:
        f.write("0 0 Air\n1 1 Water\n2 2 Bone185\n")
    return mhd, rng_file, write_spectrum(os.path.join(directory, "spectrum_120kVp_2.5mmAl.dat"))


def water_files(directory, n=64, voxel=2.0):
    os.makedirs(directory, exist_ok=True)
    mhd = write_mhd(os.path.join(directory, "water_phantom.mhd"), np.zeros((n, n, n), np.uint8), (voxel, voxel, voxel))
    rng_file = os.path.join(directory, "water_range.txt")
    with open(rng_file, "w") as f:
        f.write("0 0 Water\n")
    return mhd, rng_file


# ---- meshed phantom (binary STL) ----

def icosphere(subdivisions):
    """Unit icosphere: (vertices float64 [V, 3], faces int [F, 3]); F = 20 * 4**subdivisions."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    verts = [np.array(p, np.float64) / np.linalg.norm(p) for p in v]
    faces = f
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts), np.array(faces, np.int64)


def ellipsoid_triangles(semi_axes, center=(0.0, 0.0, 0.0), subdivisions=3):
    """Triangles [F, 3, 3] (float32, mm) of an ellipsoid surface."""
    v, f = icosphere(subdivisions)
    v = v * np.asarray(semi_axes, np.float64) + np.asarray(center, np.float64)
    return v[f].astype(np.float32)


def write_stl(path, triangles):
    """Binary STL: 80-byte header, uint32 count, per triangle normal + 3 vertices (float32) + uint16."""
    tri = np.asarray(triangles, np.float32).reshape(-1, 3, 3)
    e1, e2 = tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]
    n = np.cross(e1, e2)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    rec = np.zeros(len(tri), np.dtype([("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")]))
    rec["n"] = n
    rec["v"] = tri.reshape(-1, 9)
    with open(path, "wb") as out:
        out.write(b"ggems-b200 synthetic mesh".ljust(80, b" "))
        out.write(np.uint32(len(tri)).tobytes())
        out.write(rec.tobytes())
    return path


def body_mesh(body_subdivisions=3, inner_subdivisions=2, n_inner=8, seed=1):
    """Body ellipsoid (semi-axes 120/100/150 mm) with n_inner inner ellipsoids (cavities for a
    one-material meshed phantom), seeded; returns triangles [F, 3, 3] float32."""
    rng = np.random.default_rng(seed)
    parts = [ellipsoid_triangles((120.0, 100.0, 150.0), subdivisions=body_subdivisions)]
    for _ in range(n_inner):
        axes = rng.uniform(10.0, 30.0, 3)
        c = rng.uniform(-0.45, 0.45, 3) * np.array([120.0, 100.0, 150.0])
        parts.append(ellipsoid_triangles(axes, c, subdivisions=inner_subdivisions))
    return np.concatenate(parts)


# ---- batched workload: projection angles + phantoms of uneven size ----

def _rotation_z(deg):
    a = np.float32(np.deg2rad(deg))
    c, s = np.float32(np.cos(a)), np.float32(np.sin(a))
    r = np.eye(4, dtype=np.float32)
    r[0, 0], r[0, 1], r[1, 0], r[1, 1] = c, -s, s, c
    return r


class BatchedWorkload:
    """Several source runs for one launch (include/ggems_b200.h, gg_run_jobs):

    * `angles` projection angles of the base scene's source, rotated about z in
      1-degree steps around the isocentre, on the base scene's phantom;
    * `phantoms` phantoms of edge U{96..320} voxels of 1 mm (the ellipsoid
      generator scaled to the cube: air / water / bone 1.85), each scored in a
      dose map of `dosel_mm` dosels, hit by the base source.

    The base scene and source come from the GGEMS API (one voxelized solid with
    a dose map).  `scene` is the gg_scene to upload (base navigators + one for
    the phantoms, base dose map + one per phantom); `jobs` the (gg_source,
    primaries, solids) list.
    """

    def __init__(self, lib, base_scene, base_source, materials_file, angles=360, phantoms=16,
                 primaries=10_000_000, seed=3, dosel_mm=4.0):
        import ctypes as C
        from . import abi
        self._keep = []
        base = base_scene
        if base.number_of_solids != 1 or base.solids[0].type != abi.GG_SOLID_VOXELIZED:
            raise ValueError("the base scene must hold one voxelized solid")
        tables = [base.tables[i] for i in range(base.number_of_tables)]
        dose_maps = [base.dose_maps[i] for i in range(base.number_of_dose_maps)]
        # navigator of the phantoms
        names = ["Air", "Water", "Bone185"]
        nb, nm = 220, len(names)
        t = dict(energy_bins=np.zeros(nb, np.float32), cross_sections=np.zeros(3 * nm * nb, np.float32),
                 rayleigh=np.zeros(101 * nb, np.float32), density=np.zeros(nm, np.float32),
                 photon_cut=np.zeros(nm, np.float32), n_elements=np.zeros(nm, np.int32),
                 offset=np.zeros(nm, np.int32), Z=np.zeros(nm * 32, np.uint8), atom_density=np.zeros(nm * 32, np.float32))
        total = C.c_int32()
        cnames = (C.c_char_p * nm)(*[m.encode() for m in names])
        procs = (C.c_int * 3)(0, 1, 2)
        ctype = {np.float32: C.c_float, np.int32: C.c_int32, np.uint8: C.c_uint8}
        f = lib.ggems_build_tables
        f.restype = C.c_int
        rc = f(materials_file.encode(), cnames, nm, nb, C.c_float(1.0e-3), C.c_float(1.0), procs, 3, C.c_float(0.1),
               *[abi.ptr(t[k], ctype[t[k].dtype.type]) for k in ("energy_bins", "cross_sections", "rayleigh", "density",
                                                                 "photon_cut", "n_elements", "offset", "Z",
                                                                 "atom_density")], C.byref(total))
        if rc != 0:
            raise RuntimeError("ggems_build_tables failed: %s" % lib.ggems_last_error())
        self._keep.append(t)
        pt = abi.gg_physics_tables(nb, nm, 3, (C.c_int32 * 3)(0, 1, 2), abi.ptr(t["energy_bins"], C.c_float),
                                   abi.ptr(t["cross_sections"], C.c_float), abi.ptr(t["rayleigh"], C.c_float),
                                   abi.ptr(t["density"], C.c_float), abi.ptr(t["photon_cut"], C.c_float),
                                   abi.ptr(t["n_elements"], C.c_int32), abi.ptr(t["offset"], C.c_int32),
                                   abi.ptr(t["Z"], C.c_uint8), abi.ptr(t["atom_density"], C.c_float), total.value)
        phantom_nav = len(tables)
        tables.append(pt)
        # jobs
        self.jobs = []
        self.primaries = []
        m0 = np.array(list(base_source.matrix), np.float32).reshape(4, 4)
        for k in range(angles):
            s = abi.gg_source()
            C.pointer(s)[0] = base_source
            s.matrix[:] = [float(x) for x in (_rotation_z(float(k)) @ m0).reshape(-1)]
            self.jobs.append((s, primaries, None))
            self.primaries.append(primaries)
        rng = np.random.default_rng(seed)
        self.phantom_edges = [int(x) for x in rng.integers(96, 321, phantoms)]
        for p, n in enumerate(self.phantom_edges):
            labels = np.ascontiguousarray(cbct_labels(n, 1.0, seed + p), np.uint8)
            self._keep.append(labels)
            half = np.float32(n) * np.float32(0.5)
            sol = abi.gg_solid()
            C.pointer(sol)[0] = base.solids[0]
            sol.navigator = phantom_nav
            sol.obb.matrix[:] = [float(x) for x in np.eye(4, dtype=np.float32).reshape(-1)]
            sol.obb.border_min[:] = [-float(half)] * 3
            sol.obb.border_max[:] = [float(half)] * 3
            sol.number_of_voxels[:] = [n, n, n]
            sol.voxel_sizes[:] = [1.0, 1.0, 1.0]
            sol.labels = abi.ptr(labels, C.c_uint8)
            d = abi.gg_dose_map()
            nd = int(np.float32(n) / np.float32(dosel_mm))
            d.size_of_dosels[:] = [dosel_mm] * 3
            d.inv_size_of_dosels[:] = [float(np.float32(1.0) / np.float32(dosel_mm))] * 3
            d.border_min[:] = [-float(half)] * 3
            d.border_max[:] = [float(half)] * 3
            d.number_of_dosels[:] = [nd] * 3
            d.total_number_of_dosels = nd ** 3
            d.slice_number_of_dosels = nd * nd
            d.record_edep_squared = 1
            d.record_hit = 1
            sol.dose_map = len(dose_maps)
            dose_maps.append(d)
            arr = (abi.gg_solid * 1)(sol)
            self._keep.append(arr)
            self.jobs.append((base_source, primaries, arr))
            self.primaries.append(primaries)
        self._tables = (abi.gg_physics_tables * len(tables))(*tables)
        self._dose = (abi.gg_dose_map * len(dose_maps))(*dose_maps)
        self.scene = abi.gg_scene(len(tables), self._tables, 1, base.solids, len(dose_maps), self._dose,
                                  base.number_of_histograms, base.histogram_sizes, base.rayleigh_fit)
        self.total_primaries = sum(self.primaries)
