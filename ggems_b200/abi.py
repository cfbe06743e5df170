"""ctypes mirror of ``include/ggems_b200.h`` (the B200 transport C ABI).

The structures here must match the header field for field; tests check the
sizes against the compiled library.  Array-valued inputs are numpy arrays
kept alive by the Python objects that own the structures.
"""

import ctypes as C

import numpy as np

GG_ATTENUATION_BINS = 220
GG_TRIANGLE_FLOATS = 13
GG_MAXIMUM_PARTICLES = 1048576
GG_MAX_LOOP = 100
GG_COMPTON_SCATTERING = 0
GG_PHOTOELECTRIC_EFFECT = 1
GG_RAYLEIGH_SCATTERING = 2
GG_SOLID_VOXELIZED = 0
GG_SOLID_BOX = 1
GG_SOLID_MESHED = 2
GG_SOURCE_XRAY = 0
GG_SOURCE_VOXELIZED = 1
# gg_met_type / gg_shape_type (phantom volumes) and the numpy type of each element type
GG_MET_CHAR, GG_MET_UCHAR, GG_MET_SHORT, GG_MET_USHORT, GG_MET_INT, GG_MET_UINT, GG_MET_FLOAT = range(7)
MET_NAMES = ("MET_CHAR", "MET_UCHAR", "MET_SHORT", "MET_USHORT", "MET_INT", "MET_UINT", "MET_FLOAT")
MET_DTYPES = ("int8", "uint8", "int16", "uint16", "int32", "uint32", "float32")
GG_SHAPE_BOX, GG_SHAPE_TUBE, GG_SHAPE_SPHERE = range(3)

STATUS = {0: "GG_OK", 1: "GG_ERROR_INVALID_ARGUMENT", 2: "GG_ERROR_CUDA", 3: "GG_ERROR_NO_DEVICE",
          4: "GG_ERROR_OUT_OF_MEMORY", 5: "GG_ERROR_STATE", 6: "GG_ERROR_TIMEOUT"}

FP = C.POINTER(C.c_float)
IP = C.POINTER(C.c_int32)
UP = C.POINTER(C.c_uint8)


class gg_obb(C.Structure):
    _fields_ = [("matrix", C.c_float * 16), ("border_min", C.c_float * 3), ("border_max", C.c_float * 3)]


class gg_physics_tables(C.Structure):
    _fields_ = [("number_of_bins", C.c_int32), ("number_of_materials", C.c_int32),
                ("number_of_processes", C.c_int32), ("process_id", C.c_int32 * 3),
                ("energy_bins", FP), ("cross_sections", FP), ("rayleigh_per_atom", FP),
                ("density", FP), ("photon_energy_cut", FP), ("number_of_elements", IP),
                ("element_offset", IP), ("atomic_number", UP), ("atomic_number_density", FP),
                ("total_elements", C.c_int32), ("attenuation_energy_bins", FP), ("mu_en", FP)]


class gg_solid(C.Structure):
    _fields_ = [("type", C.c_int32), ("navigator", C.c_int32), ("obb", gg_obb), ("threshold", C.c_float),
                ("number_of_voxels", C.c_int32 * 3), ("voxel_sizes", C.c_float * 3), ("labels", UP),
                ("virtual_element_number", C.c_int32 * 3), ("box_size", C.c_float * 3),
                ("histogram", C.c_int32), ("scatter_histogram", C.c_int32), ("dose_map", C.c_int32),
                ("number_of_triangles", C.c_int32), ("triangles", FP), ("number_of_nodes", C.c_int32),
                ("nodes", FP), ("node_first", IP), ("node_triangles", IP)]


class gg_dose_map(C.Structure):
    _fields_ = [("size_of_dosels", C.c_float * 3), ("inv_size_of_dosels", C.c_float * 3),
                ("border_min", C.c_float * 3), ("border_max", C.c_float * 3),
                ("number_of_dosels", C.c_int32 * 3), ("total_number_of_dosels", C.c_int32),
                ("slice_number_of_dosels", C.c_int32), ("record_edep_squared", C.c_int32),
                ("record_hit", C.c_int32), ("record_photon_tracking", C.c_int32), ("tle", C.c_int32)]


class gg_world(C.Structure):
    _fields_ = [("dimensions", C.c_int32 * 3), ("sizes", C.c_float * 3), ("photon_tracking", C.c_int32),
                ("energy_tracking", C.c_int32), ("energy_squared_tracking", C.c_int32), ("momentum", C.c_int32)]


class gg_scene(C.Structure):
    _fields_ = [("number_of_tables", C.c_int32), ("tables", C.POINTER(gg_physics_tables)),
                ("number_of_solids", C.c_int32), ("solids", C.POINTER(gg_solid)),
                ("number_of_dose_maps", C.c_int32), ("dose_maps", C.POINTER(gg_dose_map)),
                ("number_of_histograms", C.c_int32), ("histogram_sizes", IP), ("rayleigh_fit", FP),
                ("world", C.POINTER(gg_world))]


class gg_source(C.Structure):
    _fields_ = [("type", C.c_int32), ("particle_type", C.c_int32), ("matrix", C.c_float * 16),
                ("beam_aperture", C.c_float), ("focal_spot_size", C.c_float * 3),
                ("number_of_energy_bins", C.c_int32), ("energy_spectrum", FP), ("energy_cdf", FP),
                ("is_interp", C.c_int32), ("number_of_voxels", C.c_int32 * 3), ("voxel_sizes", C.c_float * 3),
                ("border_min", C.c_float * 3), ("number_of_activity_bins", C.c_int64),
                ("activity_index", IP), ("activity_cdf", FP)]


class gg_shape(C.Structure):
    _fields_ = [("type", C.c_int32), ("position", C.c_float * 3), ("label_value", C.c_float), ("size", C.c_float * 3)]


GG_TRACK_PRIMARY, GG_TRACK_ENTER, GG_TRACK_STEP, GG_TRACK_SCATTER, GG_TRACK_LEAVE, GG_TRACK_DEAD = range(6)


class gg_track_point(C.Structure):
    _fields_ = [("kind", C.c_int32), ("solid", C.c_int32), ("process", C.c_int32), ("history", C.c_int32),
                ("E", C.c_float), ("position", C.c_float * 3), ("direction", C.c_float * 3), ("pad", C.c_float)]


class gg_job(C.Structure):
    _fields_ = [("source", gg_source), ("number_of_particles", C.c_uint64), ("solids", C.POINTER(gg_solid))]


GG_TALLY_INT32, GG_TALLY_INT64, GG_TALLY_FP64 = 0, 1, 2


class gg_device_tally(C.Structure):
    _fields_ = [("address", C.c_void_p), ("count", C.c_int64), ("type", C.c_int32)]


class gg_particle_buffers(C.Structure):
    _fields_ = [("E", FP), ("px", FP), ("py", FP), ("pz", FP), ("dx", FP), ("dy", FP), ("dz", FP),
                ("status", C.POINTER(C.c_int8)), ("scatter", C.POINTER(C.c_int8)), ("solid_id", IP)]


class gg_tally_buffers(C.Structure):
    _fields_ = [("histograms", C.POINTER(IP)), ("edep", C.POINTER(C.POINTER(C.c_double))),
                ("edep_squared", C.POINTER(C.POINTER(C.c_double))), ("hit", C.POINTER(IP)),
                ("photon_tracking", C.POINTER(IP)), ("world_photon_tracking", IP),
                ("world_energy", C.POINTER(C.c_double)), ("world_energy_squared", C.POINTER(C.c_double)),
                ("world_momentum_x", C.POINTER(C.c_double)), ("world_momentum_y", C.POINTER(C.c_double)),
                ("world_momentum_z", C.POINTER(C.c_double))]


def ptr(array, ctype):
    """Pointer to a contiguous numpy array (None -> NULL)."""
    if array is None:
        return C.cast(None, C.POINTER(ctype))
    assert array.flags["C_CONTIGUOUS"]
    return array.ctypes.data_as(C.POINTER(ctype))


class Particles:
    """Host SoA buffers for the final per-slot particle states."""

    FIELDS = ("E", "px", "py", "pz", "dx", "dy", "dz")

    def __init__(self, n):
        self.n = n
        for f in self.FIELDS:
            setattr(self, f, np.zeros(n, np.float32))
        self.status = np.zeros(n, np.int8)
        self.scatter = np.zeros(n, np.int8)
        self.solid_id = np.zeros(n, np.int32)
        self.struct = gg_particle_buffers(*[ptr(getattr(self, f), C.c_float) for f in self.FIELDS],
                                          ptr(self.status, C.c_int8), ptr(self.scatter, C.c_int8),
                                          ptr(self.solid_id, C.c_int32))


class Tallies:
    """Host tally buffers matching a scene's histograms and dose maps."""

    def __init__(self, histogram_sizes, dose_sizes, world_size=0, alloc=np.zeros):
        """alloc(n, dtype) makes each zeroed host array (e.g. page-locked memory)."""
        self.histograms = [alloc(n, np.int32) for n in histogram_sizes]
        self.edep = [alloc(n, np.float64) for n in dose_sizes]
        self.edep_squared = [alloc(n, np.float64) for n in dose_sizes]
        self.hit = [alloc(n, np.int32) for n in dose_sizes]
        self.photon_tracking = [alloc(n, np.int32) for n in dose_sizes]

        def arr(lst, ctype):
            a = (C.POINTER(ctype) * max(len(lst), 1))(*[ptr(x, ctype) for x in lst])
            return C.cast(a, C.POINTER(C.POINTER(ctype))), a

        self._h, self._hk = arr(self.histograms, C.c_int32)
        self._e, self._ek = arr(self.edep, C.c_double)
        self._e2, self._e2k = arr(self.edep_squared, C.c_double)
        self._hit, self._hitk = arr(self.hit, C.c_int32)
        self._pt, self._ptk = arr(self.photon_tracking, C.c_int32)
        self.struct = gg_tally_buffers(self._h, self._e, self._e2, self._hit, self._pt)
        self.world = None
        if world_size:
            self.world = dict(photon_tracking=np.zeros(world_size, np.int32),
                              **{k: np.zeros(world_size, np.float64) for k in
                                 ("energy", "energy_squared", "momentum_x", "momentum_y", "momentum_z")})
            self.struct.world_photon_tracking = ptr(self.world["photon_tracking"], C.c_int32)
            for k in ("energy", "energy_squared", "momentum_x", "momentum_y", "momentum_z"):
                setattr(self.struct, "world_" + k, ptr(self.world[k], C.c_double))
