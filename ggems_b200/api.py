"""GGEMS Python API on the B200 transport layer.

Same classes, method names and argument meaning as GGEMS's ``python_module``
(``python_module/__init__.py``, ``ggems_sources.py``, ``ggems_phantoms.py``,
``ggems_systems.py``, ``ggems_dosimetry.py``, ``ggems_processes.py``,
``ggems_materials.py``, ``ggems_opencl.py``), so an existing GGEMS script runs
unchanged after ``from ggems_b200 import *``.  Where GGEMS would abort the
process on an error (a C++ exception escaping through ctypes), these wrappers
raise ``GGEMSError`` with GGEMS's message.
"""

import ctypes as C

from . import abi
from ._native import GGEMSNativeError, lib

__all__ = ["GGEMSError", "GGEMSVerbosity", "GGEMS", "GGEMSOpenCLManager", "GGEMSMaterialsDatabaseManager",
           "GGEMSMaterials", "GGEMSCrossSections", "GGEMSProcessesManager", "GGEMSRangeCutsManager",
           "GGEMSSourceManager", "GGEMSXRaySource", "GGEMSVoxelizedSource", "GGEMSVoxelizedPhantom",
           "GGEMSCTSystem", "GGEMSDosimetryCalculator", "GGEMSProfilerManager", "GGEMSRAMManager", "clean_safely"]


class GGEMSError(GGEMSNativeError):
    pass


vp, f32, u32, u64, i32, b, s = C.c_void_p, C.c_float, C.c_uint32, C.c_uint64, C.c_int, C.c_bool, C.c_char_p

_SIGNATURES = {
    "ggems_last_error": (s, []), "ggems_clear_error": (None, []), "set_ggems_verbose": (None, [i32]),
    "create_ggems": (vp, []), "delete_ggems": (None, [vp]), "initialize_ggems": (None, [vp, u32]),
    "run_ggems": (None, [vp]), "set_opencl_verbose_ggems": (None, [vp, b]),
    "set_material_database_verbose_ggems": (None, [vp, b]), "set_source_ggems": (None, [vp, b]),
    "set_navigator_ggems": (None, [vp, b]), "set_memory_ram_ggems": (None, [vp, b]),
    "set_process_ggems": (None, [vp, b]), "set_range_cuts_ggems": (None, [vp, b]),
    "set_random_ggems": (None, [vp, b]), "set_profiling_ggems": (None, [vp, b]),
    "set_tracking_ggems": (None, [vp, b, i32]),
    "ggems_scene": (C.POINTER(abi.gg_scene), [vp]), "ggems_number_of_devices": (i32, [vp]),
    "ggems_device_context": (vp, [vp, i32]), "ggems_initial_random_states": (C.POINTER(C.c_uint32), [vp, i32]),
    "ggems_last_run": (None, [vp, C.POINTER(f32), C.POINTER(C.c_int64), C.POINTER(u64)]),
    "ggems_number_of_sources": (i32, []),
    "ggems_source_descriptor": (i32, [i32, C.POINTER(abi.gg_source), C.POINTER(u64)]),
    "get_instance_ggems_opencl_manager": (vp, []), "print_infos_opencl_manager": (None, [vp]),
    "set_device_index_ggems_opencl_manager": (None, [vp, u64]),
    "set_device_to_activate_opencl_manager": (None, [vp, s, s]),
    "set_device_balancing_opencl_manager": (None, [vp, s]), "clean_opencl_manager": (None, [vp]),
    "get_instance_materials_manager": (vp, []), "set_materials_ggems_materials_manager": (None, [vp, s]),
    "print_available_chemical_elements_ggems_materials_manager": (None, [vp]),
    "print_available_materials_ggems_materials_manager": (None, [vp]),
    "get_instance_processes_manager": (vp, []), "add_process_processes_manager": (None, [vp, s, s, s]),
    "set_cross_section_table_number_of_bins_processes_manager": (None, [vp, u64]),
    "set_cross_section_table_minimum_energy_processes_manager": (None, [vp, f32, s]),
    "set_cross_section_table_maximum_energy_processes_manager": (None, [vp, f32, s]),
    "print_infos_processes_manager": (None, [vp]), "print_available_processes_manager": (None, [vp]),
    "print_tables_processes_manager": (None, [vp, b]),
    "get_instance_range_cuts_manager": (vp, []), "set_cut_range_cuts_manager": (None, [vp, s, s, f32, s]),
    "get_instance_ggems_source_manager": (vp, []), "initialize_source_manager": (None, [vp, u32]),
    "print_infos_source_manager": (None, [vp]), "clean_source_manager": (None, [vp]),
    "create_ggems_xray_source": (vp, [s]), "set_position_ggems_xray_source": (None, [vp, f32, f32, f32, s]),
    "set_number_of_particles_xray_source": (None, [vp, u64]),
    "set_source_particle_type_ggems_xray_source": (None, [vp, s]),
    "set_beam_aperture_ggems_xray_source": (None, [vp, f32, s]),
    "set_focal_spot_size_ggems_xray_source": (None, [vp, f32, f32, f32, s]),
    "set_rotation_ggems_xray_source": (None, [vp, f32, f32, f32, s]),
    "set_monoenergy_ggems_xray_source": (None, [vp, f32, s]), "set_polyenergy_ggems_xray_source": (None, [vp, s]),
    "set_energy_peak_ggems_xray_source": (None, [vp, f32, s, f32]),
    "create_ggems_voxelized_source": (vp, [s]),
    "set_position_ggems_voxelized_source": (None, [vp, f32, f32, f32, s]),
    "set_rotation_ggems_voxelized_source": (None, [vp, f32, f32, f32, s]),
    "set_number_of_particles_voxelized_source": (None, [vp, u64]),
    "set_source_particle_type_ggems_voxelized_source": (None, [vp, s]),
    "set_monoenergy_ggems_voxelized_source": (None, [vp, f32, s]),
    "set_polyenergy_ggems_voxelized_source": (None, [vp, s]),
    "set_phantom_source_ggems_voxelized_source": (None, [vp, s]),
    "set_energy_peak_ggems_voxelized_source": (None, [vp, f32, s, f32]),
    "create_ggems_voxelized_phantom": (vp, [s]), "set_phantom_file_ggems_voxelized_phantom": (None, [vp, s, s]),
    "set_position_ggems_voxelized_phantom": (None, [vp, f32, f32, f32, s]),
    "set_rotation_ggems_voxelized_phantom": (None, [vp, f32, f32, f32, s]),
    "set_visible_ggems_voxelized_phantom": (None, [vp, b]),
    "set_material_visible_ggems_voxelized_phantom": (None, [vp, s, b]),
    "set_material_color_ggems_voxelized_phantom": (None, [vp, s, C.c_ubyte, C.c_ubyte, C.c_ubyte]),
    "set_material_color_name_ggems_voxelized_phantom": (None, [vp, s, s]),
    "create_ggems_meshed_phantom": (vp, [s]), "set_phantom_file_ggems_meshed_phantom": (None, [vp, s]),
    "set_position_ggems_meshed_phantom": (None, [vp, f32, f32, f32, s]),
    "set_rotation_ggems_meshed_phantom": (None, [vp, f32, f32, f32, s]),
    "set_visible_ggems_meshed_phantom": (None, [vp, b]),
    "set_material_name_ggems_meshed_phantom": (None, [vp, s]),
    "set_material_color_ggems_meshed_phantom": (None, [vp, s, C.c_ubyte, C.c_ubyte, C.c_ubyte]),
    "set_material_color_name_ggems_meshed_phantom": (None, [vp, s, s]),
    "set_mesh_octree_depth_ggems_meshed_phantom": (None, [vp, C.c_int]),
    "create_ggems_world": (vp, []),
    "set_dimension_ggems_world": (None, [vp, C.c_size_t, C.c_size_t, C.c_size_t]),
    "set_size_ggems_world": (None, [vp, f32, f32, f32, s]),
    "photon_tracking_ggems_world": (None, [vp, b]), "energy_tracking_ggems_world": (None, [vp, b]),
    "energy_squared_tracking_ggems_world": (None, [vp, b]), "momentum_ggems_world": (None, [vp, b]),
    "set_output_ggems_world": (None, [vp, s]),
    "get_instance_volume_creator_manager": (vp, []),
    "set_volume_dimension_volume_creator_manager": (None, [vp, C.c_size_t, C.c_size_t, C.c_size_t]),
    "set_element_sizes_volume_creator_manager": (None, [vp, f32, f32, f32, s]),
    "set_output_image_filename_volume_creator_manager": (None, [vp, s]),
    "set_output_range_to_material_filename_volume_creator_manager": (None, [vp, s]),
    "initialize_volume_creator_manager": (None, [vp]), "write_volume_creator_manager": (None, [vp]),
    "set_material_volume_creator_manager": (None, [vp, s]), "set_data_type_volume_creator_manager": (None, [vp, s]),
    "clean_volume_creator_manager": (None, [vp]),
    "create_box": (vp, [f32, f32, f32, s]), "create_tube": (vp, [f32, f32, f32, s]), "create_sphere": (vp, [f32, s]),
    **{f % shape: sig for shape in ("box", "tube", "sphere") for f, sig in (
        ("delete_%s", (None, [vp])), ("set_position_%s", (None, [vp, f32, f32, f32, s])),
        ("set_material_%s", (None, [vp, s])), ("set_label_value_%s", (None, [vp, f32])),
        ("initialize_%s", (None, [vp])), ("draw_%s", (None, [vp])))},
    "create_ggems_ct_system": (vp, [s]), "set_number_of_modules_ggems_ct_system": (None, [vp, u64, u64]),
    "set_ct_system_type_ggems_ct_system": (None, [vp, s]),
    "set_number_of_detection_elements_ggems_ct_system": (None, [vp, u64, u64, u64]),
    "set_size_of_detection_elements_ggems_ct_system": (None, [vp, f32, f32, f32, s]),
    "set_material_name_ggems_ct_system": (None, [vp, s]),
    "set_source_isocenter_distance_ggems_ct_system": (None, [vp, f32, s]),
    "set_source_detector_distance_ggems_ct_system": (None, [vp, f32, s]),
    "set_rotation_ggems_ct_system": (None, [vp, f32, f32, f32, s]), "set_save_ggems_ct_system": (None, [vp, s]),
    "set_threshold_ggems_ct_system": (None, [vp, f32, s]), "store_scatter_ggems_ct_system": (None, [vp, b]),
    "set_global_system_position_ggems_ct_system": (None, [vp, f32, f32, f32, s]),
    "set_visible_ggems_ct_system": (None, [vp, b]),
    "set_material_color_ggems_ct_system": (None, [vp, s, C.c_ubyte, C.c_ubyte, C.c_ubyte]),
    "set_material_color_name_ggems_ct_system": (None, [vp, s, s]),
    "create_ggems_dosimetry_calculator": (vp, []), "delete_dosimetry_calculator": (None, [vp]),
    "scale_factor_dosimetry_calculator": (None, [vp, f32]), "water_reference_dosimetry_calculator": (None, [vp, b]),
    "minimum_density_dosimetry_calculator": (None, [vp, f32, s]),
    "set_dosel_size_dosimetry_calculator": (None, [vp, f32, f32, f32, s]),
    "set_dose_output_dosimetry_calculator": (None, [vp, s]),
    "dose_photon_tracking_dosimetry_calculator": (None, [vp, b]), "dose_edep_dosimetry_calculator": (None, [vp, b]),
    "dose_hit_dosimetry_calculator": (None, [vp, b]), "dose_edep_squared_dosimetry_calculator": (None, [vp, b]),
    "dose_uncertainty_dosimetry_calculator": (None, [vp, b]), "dose_tle_navigator": (None, [vp, b]),
    "attach_to_navigator_dosimetry_calculator": (None, [vp, s]),
    "create_ggems_materials": (vp, []), "add_material_ggems_materials": (None, [vp, s]),
    "initialize_ggems_materials": (None, [vp]), "print_material_properties_ggems_materials": (None, [vp]),
    "get_density_ggems_materials": (f32, [vp, s]), "get_energy_cut_ggems_materials": (f32, [vp, s, s, f32, s]),
    "get_atomic_number_density_ggems_materials": (f32, [vp, s]), "clean_ggems_materials": (None, [vp]),
    "create_ggems_cross_sections": (vp, [vp]), "add_process_ggems_cross_sections": (None, [vp, s, s, b]),
    "initialize_ggems_cross_sections": (None, [vp]), "get_cs_ggems_cross_sections": (f32, [vp, s, s, f32, s]),
    "clean_ggems_cross_sections": (None, [vp]),
    "create_ggems_attenuations": (vp, [vp, vp]), "initialize_ggems_attenuations": (None, [vp]),
    "get_mu_ggems_attenuations": (f32, [vp, s, f32, s]), "get_mu_en_ggems_attenuations": (f32, [vp, s, f32, s]),
    "clean_ggems_attenuations": (None, [vp]),
    "get_instance_profiler_manager": (vp, []), "print_summary_profiler_manager": (None, [vp]),
    "get_instance_ggems_ram_manager": (vp, []), "print_infos_ram_manager": (None, [vp]),
}
for _name, (_res, _args) in _SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args


def _e(x):
    return x.encode("ASCII") if isinstance(x, str) else x


def _call(name, *args):
    lib.ggems_clear_error()
    out = getattr(lib, name)(*args)
    err = lib.ggems_last_error()
    if err:
        raise GGEMSError(err.decode(errors="replace"))
    return out


class GGEMSVerbosity(object):
    """Set the verbosity of infos in GGEMS (ggems_lib.py)."""

    def __init__(self, val):
        _call("set_ggems_verbose", val)


class GGEMS(object):
    """GGEMS class managing the simulation (python_module/__init__.py)."""

    def __init__(self):
        self.obj = _call("create_ggems")

    def delete(self):
        if self.obj:
            _call("delete_ggems", self.obj)
            self.obj = None

    def initialize(self, seed=0):
        _call("initialize_ggems", self.obj, seed)

    def run(self):
        _call("run_ggems", self.obj)

    def opencl_verbose(self, flag):
        _call("set_opencl_verbose_ggems", self.obj, flag)

    def material_database_verbose(self, flag):
        _call("set_material_database_verbose_ggems", self.obj, flag)

    def navigator_verbose(self, flag):
        _call("set_navigator_ggems", self.obj, flag)

    def source_verbose(self, flag):
        _call("set_source_ggems", self.obj, flag)

    def memory_verbose(self, flag):
        _call("set_memory_ram_ggems", self.obj, flag)

    def process_verbose(self, flag):
        _call("set_process_ggems", self.obj, flag)

    def profiling_verbose(self, flag):
        _call("set_profiling_ggems", self.obj, flag)

    def range_cuts_verbose(self, flag):
        _call("set_range_cuts_ggems", self.obj, flag)

    def random_verbose(self, flag):
        _call("set_random_ggems", self.obj, flag)

    def tracking_verbose(self, flag, particle_id):
        _call("set_tracking_ggems", self.obj, flag, particle_id)

    # -- additions: what the run did (no counterpart in GGEMS) --
    def last_run(self):
        """(device milliseconds, kernel launches, primaries) of the last run()."""
        ms, n, p = C.c_float(), C.c_int64(), C.c_uint64()
        lib.ggems_last_run(self.obj, C.byref(ms), C.byref(n), C.byref(p))
        return ms.value, n.value, p.value

    def scene(self):
        """The gg_scene handed to the transport layer (after initialize)."""
        p = lib.ggems_scene(self.obj)
        return p.contents if p else None


class GGEMSOpenCLManager(object):
    """Device selection (ggems_opencl.py); drives the CUDA devices here."""

    def __init__(self):
        self.obj = _call("get_instance_ggems_opencl_manager")

    def print_infos(self):
        _call("print_infos_opencl_manager", self.obj)

    def set_device_index(self, device_id):
        _call("set_device_index_ggems_opencl_manager", self.obj, device_id)

    def set_device_to_activate(self, device_type, device_vendor=""):
        _call("set_device_to_activate_opencl_manager", self.obj, _e(device_type), _e(device_vendor))

    def set_device_balancing(self, device_balancing):
        _call("set_device_balancing_opencl_manager", self.obj, _e(device_balancing))

    def clean(self):
        _call("clean_opencl_manager", self.obj)


class GGEMSMaterialsDatabaseManager(object):
    def __init__(self):
        self.obj = _call("get_instance_materials_manager")

    def set_materials(self, filename):
        _call("set_materials_ggems_materials_manager", self.obj, _e(filename))

    def print_available_chemical_elements(self):
        _call("print_available_chemical_elements_ggems_materials_manager", self.obj)

    def print_available_materials(self):
        _call("print_available_materials_ggems_materials_manager", self.obj)


class GGEMSMaterials(object):
    def __init__(self):
        self.obj = _call("create_ggems_materials")

    def add_material(self, material_name):
        _call("add_material_ggems_materials", self.obj, _e(material_name))

    def initialize(self):
        _call("initialize_ggems_materials", self.obj)

    def print_material_properties(self):
        _call("print_material_properties_ggems_materials", self.obj)

    def get_density(self, material_name):
        return _call("get_density_ggems_materials", self.obj, _e(material_name))

    def get_energy_cut(self, material_name, particle_type, value, unit):
        return _call("get_energy_cut_ggems_materials", self.obj, _e(material_name), _e(particle_type), value, _e(unit))

    def get_atomic_number_density(self, material_name):
        return _call("get_atomic_number_density_ggems_materials", self.obj, _e(material_name))

    def clean(self):
        _call("clean_ggems_materials", self.obj)


class GGEMSCrossSections(object):
    def __init__(self, materials):
        self.obj = _call("create_ggems_cross_sections", materials.obj)

    def add_process(self, process_name, particle_name, is_secondary=False):
        _call("add_process_ggems_cross_sections", self.obj, _e(process_name), _e(particle_name), is_secondary)

    def initialize(self):
        _call("initialize_ggems_cross_sections", self.obj)

    def get_cs(self, process_name, material_name, energy, unit):
        return _call("get_cs_ggems_cross_sections", self.obj, _e(process_name), _e(material_name), energy, _e(unit))

    def clean(self):
        _call("clean_ggems_cross_sections", self.obj)


class GGEMSAttenuations(object):
    """mu / mu_en (cm^-1) of registered materials on GGEMS's 220-bin attenuation table
    (python_module/ggems_attenuation.py)."""

    def __init__(self, materials, cross_sections):
        self.obj = _call("create_ggems_attenuations", materials.obj, cross_sections.obj)

    def initialize(self):
        _call("initialize_ggems_attenuations", self.obj)

    def get_mu(self, material_name, energy, unit):
        return _call("get_mu_ggems_attenuations", self.obj, _e(material_name), energy, _e(unit))

    def get_mu_en(self, material_name, energy, unit):
        return _call("get_mu_en_ggems_attenuations", self.obj, _e(material_name), energy, _e(unit))

    def clean(self):
        _call("clean_ggems_attenuations", self.obj)


class GGEMSProcessesManager(object):
    def __init__(self):
        self.obj = _call("get_instance_processes_manager")

    def set_cross_section_table_number_of_bins(self, number_of_bins):
        _call("set_cross_section_table_number_of_bins_processes_manager", self.obj, number_of_bins)

    def set_cross_section_table_energy_min(self, energy, unit):
        _call("set_cross_section_table_minimum_energy_processes_manager", self.obj, energy, _e(unit))

    def set_cross_section_table_energy_max(self, energy, unit):
        _call("set_cross_section_table_maximum_energy_processes_manager", self.obj, energy, _e(unit))

    def print_available_processes(self):
        _call("print_available_processes_manager", self.obj)

    def print_infos(self):
        _call("print_infos_processes_manager", self.obj)

    def add_process(self, process_name, particle_name, phantom_name="all", is_secondary=False):
        _call("add_process_processes_manager", self.obj, _e(process_name), _e(particle_name), _e(phantom_name))

    def print_tables(self, flag):
        _call("print_tables_processes_manager", self.obj, flag)


class GGEMSRangeCutsManager(object):
    def __init__(self):
        self.obj = _call("get_instance_range_cuts_manager")

    def set_cut(self, particle, value, unit, phantom="all"):
        _call("set_cut_range_cuts_manager", self.obj, _e(phantom), _e(particle), value, _e(unit))


class GGEMSSourceManager(object):
    def __init__(self):
        self.obj = _call("get_instance_ggems_source_manager")

    def initialize(self, seed):
        _call("initialize_source_manager", self.obj, seed)

    def print_infos(self):
        _call("print_infos_source_manager", self.obj)

    def clean(self):
        _call("clean_source_manager", self.obj)


class GGEMSXRaySource(object):
    """X-ray cone-beam source (ggems_sources.py)."""

    def __init__(self, source_name):
        self.obj = _call("create_ggems_xray_source", _e(source_name))

    def set_position(self, x, y, z, unit):
        _call("set_position_ggems_xray_source", self.obj, x, y, z, _e(unit))

    def set_number_of_particles(self, number_of_particles):
        _call("set_number_of_particles_xray_source", self.obj, int(number_of_particles))

    def set_source_particle_type(self, particle_type):
        _call("set_source_particle_type_ggems_xray_source", self.obj, _e(particle_type))

    def set_beam_aperture(self, beam_aperture, unit):
        _call("set_beam_aperture_ggems_xray_source", self.obj, beam_aperture, _e(unit))

    def set_focal_spot_size(self, width, height, depth, unit):
        _call("set_focal_spot_size_ggems_xray_source", self.obj, width, height, depth, _e(unit))

    def set_rotation(self, rx, ry, rz, unit):
        _call("set_rotation_ggems_xray_source", self.obj, rx, ry, rz, _e(unit))

    def set_monoenergy(self, e, unit):
        _call("set_monoenergy_ggems_xray_source", self.obj, e, _e(unit))

    def set_polyenergy(self, file):
        _call("set_polyenergy_ggems_xray_source", self.obj, _e(file))

    def set_energy_peak(self, e, unit, i):
        _call("set_energy_peak_ggems_xray_source", self.obj, e, _e(unit), i)


class GGEMSVoxelizedSource(object):
    """Voxelized (activity map) source (ggems_sources.py)."""

    def __init__(self, source_name):
        self.obj = _call("create_ggems_voxelized_source", _e(source_name))

    def set_position(self, x, y, z, unit):
        _call("set_position_ggems_voxelized_source", self.obj, x, y, z, _e(unit))

    def set_rotation(self, rx, ry, rz, unit):
        _call("set_rotation_ggems_voxelized_source", self.obj, rx, ry, rz, _e(unit))

    def set_number_of_particles(self, number_of_particles):
        _call("set_number_of_particles_voxelized_source", self.obj, int(number_of_particles))

    def set_source_particle_type(self, particle_type):
        _call("set_source_particle_type_ggems_voxelized_source", self.obj, _e(particle_type))

    def set_monoenergy(self, e, unit):
        _call("set_monoenergy_ggems_voxelized_source", self.obj, e, _e(unit))

    def set_polyenergy(self, file):
        _call("set_polyenergy_ggems_voxelized_source", self.obj, _e(file))

    def set_phantom_source(self, file):
        _call("set_phantom_source_ggems_voxelized_source", self.obj, _e(file))

    def set_energy_peak(self, e, unit, i):
        _call("set_energy_peak_ggems_voxelized_source", self.obj, e, _e(unit), i)


class GGEMSVoxelizedPhantom(object):
    """Voxelized phantom navigator (ggems_phantoms.py)."""

    def __init__(self, voxelized_phantom_name):
        self.obj = _call("create_ggems_voxelized_phantom", _e(voxelized_phantom_name))

    def set_phantom(self, phantom_filename, range_data_filename):
        _call("set_phantom_file_ggems_voxelized_phantom", self.obj, _e(phantom_filename), _e(range_data_filename))

    def set_position(self, position_x, position_y, position_z, unit):
        _call("set_position_ggems_voxelized_phantom", self.obj, position_x, position_y, position_z, _e(unit))

    def set_rotation(self, rx, ry, rz, unit):
        _call("set_rotation_ggems_voxelized_phantom", self.obj, rx, ry, rz, _e(unit))

    def set_visible(self, flag):
        _call("set_visible_ggems_voxelized_phantom", self.obj, flag)

    def set_material_visible(self, material_name, flag):
        _call("set_material_visible_ggems_voxelized_phantom", self.obj, _e(material_name), flag)

    def set_material_color(self, material_name, red=0, green=0, blue=0, color_name=""):
        if color_name:
            _call("set_material_color_name_ggems_voxelized_phantom", self.obj, _e(material_name), _e(color_name))
        else:
            _call("set_material_color_ggems_voxelized_phantom", self.obj, _e(material_name), red, green, blue)


class GGEMSMeshedPhantom(object):
    """Meshed (STL) phantom navigator (ggems_phantoms.py)."""

    def __init__(self, meshed_phantom_name):
        self.obj = _call("create_ggems_meshed_phantom", _e(meshed_phantom_name))

    def set_phantom(self, phantom_filename):
        _call("set_phantom_file_ggems_meshed_phantom", self.obj, _e(phantom_filename))

    def set_position(self, pos_x, pos_y, pos_z, unit):
        _call("set_position_ggems_meshed_phantom", self.obj, pos_x, pos_y, pos_z, _e(unit))

    def set_rotation(self, rx, ry, rz, unit):
        _call("set_rotation_ggems_meshed_phantom", self.obj, rx, ry, rz, _e(unit))

    def set_visible(self, flag):
        _call("set_visible_ggems_meshed_phantom", self.obj, flag)

    def set_material(self, material_name):
        _call("set_material_name_ggems_meshed_phantom", self.obj, _e(material_name))

    def set_mesh_octree_depth(self, depth):
        _call("set_mesh_octree_depth_ggems_meshed_phantom", self.obj, depth)

    def set_material_color(self, material_name, red=0, green=0, blue=0, color_name=""):
        if color_name:
            _call("set_material_color_name_ggems_meshed_phantom", self.obj, _e(material_name), _e(color_name))
        else:
            _call("set_material_color_ggems_meshed_phantom", self.obj, _e(material_name), red, green, blue)


class GGEMSWorld(object):
    """World grid recording photon flights between solids (ggems_phantoms.py)."""

    def __init__(self):
        self.obj = _call("create_ggems_world")

    def set_dimensions(self, dim_x, dim_y, dim_z):
        _call("set_dimension_ggems_world", self.obj, dim_x, dim_y, dim_z)

    def set_element_sizes(self, size_x, size_y, size_z, unit):
        _call("set_size_ggems_world", self.obj, size_x, size_y, size_z, _e(unit))

    def photon_tracking(self, activate):
        _call("photon_tracking_ggems_world", self.obj, activate)

    def set_output_basename(self, output):
        _call("set_output_ggems_world", self.obj, _e(output))

    def energy_tracking(self, activate):
        _call("energy_tracking_ggems_world", self.obj, activate)

    def energy_squared_tracking(self, activate):
        _call("energy_squared_tracking_ggems_world", self.obj, activate)

    def momentum(self, activate):
        _call("momentum_ggems_world", self.obj, activate)


class GGEMSVolumeCreatorManager(object):
    """Voxel image of analytic shapes, drawn on the device (ggems_volume_creator.py)."""

    def __init__(self):
        self.obj = _call("get_instance_volume_creator_manager")

    def set_dimensions(self, width, height, depth):
        _call("set_volume_dimension_volume_creator_manager", self.obj, width, height, depth)

    def set_element_sizes(self, width, height, depth, unit):
        _call("set_element_sizes_volume_creator_manager", self.obj, width, height, depth, _e(unit))

    def set_output(self, output):
        _call("set_output_image_filename_volume_creator_manager", self.obj, _e(output))

    def set_range_output(self, output):
        _call("set_output_range_to_material_filename_volume_creator_manager", self.obj, _e(output))

    def initialize(self):
        _call("initialize_volume_creator_manager", self.obj)

    def write(self):
        _call("write_volume_creator_manager", self.obj)

    def set_material(self, material):
        _call("set_material_volume_creator_manager", self.obj, _e(material))

    def set_data_type(self, data_type):
        _call("set_data_type_volume_creator_manager", self.obj, _e(data_type))

    def clean(self):
        _call("clean_volume_creator_manager", self.obj)


class _Shape(object):
    _kind = ""

    def delete(self):
        _call("delete_" + self._kind, self.obj)

    def set_label_value(self, label_value):
        _call("set_label_value_" + self._kind, self.obj, label_value)

    def set_position(self, pos_x, pos_y, pos_z, unit):
        _call("set_position_" + self._kind, self.obj, pos_x, pos_y, pos_z, _e(unit))

    def set_material(self, material):
        _call("set_material_" + self._kind, self.obj, _e(material))

    def initialize(self):
        _call("initialize_" + self._kind, self.obj)

    def draw(self):
        _call("draw_" + self._kind, self.obj)


class GGEMSTube(_Shape):
    """Elliptic tube along z (ggems_volume_creator.py)."""
    _kind = "tube"

    def __init__(self, radius_x, radius_y, height, unit):
        self.obj = _call("create_tube", radius_x, radius_y, height, _e(unit))


class GGEMSBox(_Shape):
    """Box of width (x), height (y), depth (z) (ggems_volume_creator.py)."""
    _kind = "box"

    def __init__(self, width, height, depth, unit):
        self.obj = _call("create_box", width, height, depth, _e(unit))


class GGEMSSphere(_Shape):
    """Sphere (ggems_volume_creator.py)."""
    _kind = "sphere"

    def __init__(self, radius, unit):
        self.obj = _call("create_sphere", radius, _e(unit))


class GGEMSCTSystem(object):
    """CT / CBCT detector navigator (ggems_systems.py)."""

    def __init__(self, ct_system_name):
        self.obj = _call("create_ggems_ct_system", _e(ct_system_name))

    def set_number_of_modules(self, module_x, module_y):
        _call("set_number_of_modules_ggems_ct_system", self.obj, module_x, module_y)

    def set_ct_type(self, ct_system_type):
        _call("set_ct_system_type_ggems_ct_system", self.obj, _e(ct_system_type))

    def set_number_of_detection_elements(self, element_x, element_y, element_z):
        _call("set_number_of_detection_elements_ggems_ct_system", self.obj, element_x, element_y, element_z)

    def set_size_of_detection_elements(self, size_x, size_y, size_z, unit):
        _call("set_size_of_detection_elements_ggems_ct_system", self.obj, size_x, size_y, size_z, _e(unit))

    def set_material(self, material_name):
        _call("set_material_name_ggems_ct_system", self.obj, _e(material_name))

    def set_source_detector_distance(self, sdd, unit):
        _call("set_source_detector_distance_ggems_ct_system", self.obj, sdd, _e(unit))

    def set_source_isocenter_distance(self, sid, unit):
        _call("set_source_isocenter_distance_ggems_ct_system", self.obj, sid, _e(unit))

    def set_rotation(self, rx, ry, rz, unit):
        _call("set_rotation_ggems_ct_system", self.obj, rx, ry, rz, _e(unit))

    def set_global_system_position(self, x, y, z, unit):
        _call("set_global_system_position_ggems_ct_system", self.obj, x, y, z, _e(unit))

    def set_threshold(self, threshold, unit):
        _call("set_threshold_ggems_ct_system", self.obj, threshold, _e(unit))

    def set_visible(self, flag):
        _call("set_visible_ggems_ct_system", self.obj, flag)

    def set_material_color(self, material_name, red=0, green=0, blue=0, color_name=""):
        if color_name:
            _call("set_material_color_name_ggems_ct_system", self.obj, _e(material_name), _e(color_name))
        else:
            _call("set_material_color_ggems_ct_system", self.obj, _e(material_name), red, green, blue)

    def save(self, basename):
        _call("set_save_ggems_ct_system", self.obj, _e(basename))

    def store_scatter(self, flag):
        _call("store_scatter_ggems_ct_system", self.obj, flag)


class GGEMSDosimetryCalculator(object):
    """Dose scoring attached to a voxelized phantom (ggems_dosimetry.py)."""

    def __init__(self):
        self.obj = _call("create_ggems_dosimetry_calculator")

    def set_dosel_size(self, dose_x, dose_y, dose_z, unit):
        _call("set_dosel_size_dosimetry_calculator", self.obj, dose_x, dose_y, dose_z, _e(unit))

    def delete(self):
        if self.obj:
            _call("delete_dosimetry_calculator", self.obj)
            self.obj = None

    def set_output_basename(self, output):
        _call("set_dose_output_dosimetry_calculator", self.obj, _e(output))

    def photon_tracking(self, activate):
        _call("dose_photon_tracking_dosimetry_calculator", self.obj, activate)

    def edep(self, activate):
        _call("dose_edep_dosimetry_calculator", self.obj, activate)

    def hit(self, activate):
        _call("dose_hit_dosimetry_calculator", self.obj, activate)

    def edep_squared(self, activate):
        _call("dose_edep_squared_dosimetry_calculator", self.obj, activate)

    def uncertainty(self, activate):
        _call("dose_uncertainty_dosimetry_calculator", self.obj, activate)

    def set_tle(self, activate):
        _call("dose_tle_navigator", self.obj, activate)

    def scale_factor(self, factor):
        _call("scale_factor_dosimetry_calculator", self.obj, factor)

    def water_reference(self, activate):
        _call("water_reference_dosimetry_calculator", self.obj, activate)

    def minimum_density(self, density, unit):
        _call("minimum_density_dosimetry_calculator", self.obj, density, _e(unit))

    def attach_to_navigator(self, navigator):
        _call("attach_to_navigator_dosimetry_calculator", self.obj, _e(navigator))


class GGEMSProfilerManager(object):
    def __init__(self):
        self.obj = _call("get_instance_profiler_manager")

    def print_summary_profile(self):
        _call("print_summary_profiler_manager", self.obj)


class GGEMSRAMManager(object):
    def __init__(self):
        self.obj = _call("get_instance_ggems_ram_manager")

    def print_infos(self):
        _call("print_infos_ram_manager", self.obj)


def clean_safely():
    """Release the registered sources, navigators and devices (python_module/__init__.py)."""
    GGEMSOpenCLManager().clean()
