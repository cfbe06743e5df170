/*
 * ggems_api.h - the GGEMS-compatible C ABI exported by libggems.so.
 *
 * Same function names, argument order and meaning as GGEMS v1.3's extern "C"
 * functions (declared at the bottom of the reference's headers under
 * include/GGEMS; the file:line of each counterpart is given beside it), so
 * the reference's Python ctypes module binds unchanged.  Objects are opaque
 * handles.  Errors: where GGEMS throws a C++ exception through the C ABI
 * (aborting a ctypes caller), these functions catch it, print the same
 * message and record it for ggems_last_error().
 */
#ifndef GGEMS_API_H
#define GGEMS_API_H

#include <stdbool.h>
#include <stdint.h>

#include "ggems_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct GGEMS GGEMS;
typedef struct GGEMSXRaySource GGEMSXRaySource;
typedef struct GGEMSVoxelizedSource GGEMSVoxelizedSource;
typedef struct GGEMSVoxelizedPhantom GGEMSVoxelizedPhantom;
typedef struct GGEMSMeshedPhantom GGEMSMeshedPhantom;
typedef struct GGEMSCTSystem GGEMSCTSystem;
typedef struct GGEMSWorld GGEMSWorld;
typedef struct GGEMSVolumeCreatorManager GGEMSVolumeCreatorManager;
typedef struct GGEMSBox GGEMSBox;
typedef struct GGEMSTube GGEMSTube;
typedef struct GGEMSSphere GGEMSSphere;
typedef struct GGEMSDosimetryCalculator GGEMSDosimetryCalculator;
typedef struct GGEMSMaterials GGEMSMaterials;
typedef struct GGEMSAttenuations GGEMSAttenuations;
typedef struct GGEMSCrossSections GGEMSCrossSections;

const char* ggems_last_error(void);  /* no counterpart in the reference: B200 build addition */
void ggems_clear_error(void);  /* no counterpart in the reference: B200 build addition */
void set_ggems_verbose(int verbosity);  /* include/GGEMS/tools/GGEMSPrint.hh:266 */
GGEMS* create_ggems(void);  /* include/GGEMS/global/GGEMS.hh:231 */
void delete_ggems(GGEMS* g);  /* include/GGEMS/global/GGEMS.hh:238 */
void initialize_ggems(GGEMS* g, uint32_t seed);  /* include/GGEMS/global/GGEMS.hh:246 */
void run_ggems(GGEMS* g);  /* include/GGEMS/global/GGEMS.hh:334 */
void set_opencl_verbose_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:254 */
void set_material_database_verbose_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:262 */
void set_source_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:270 */
void set_navigator_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:278 */
void set_memory_ram_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:286 */
void set_process_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:294 */
void set_range_cuts_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:302 */
void set_random_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:310 */
void set_profiling_ggems(GGEMS* g, bool v);  /* include/GGEMS/global/GGEMS.hh:318 */
void set_tracking_ggems(GGEMS* g, bool v, int id);  /* include/GGEMS/global/GGEMS.hh:327 */
const gg_scene* ggems_scene(GGEMS* g);  /* no counterpart in the reference: B200 build addition */
int ggems_number_of_devices(GGEMS* g);  /* no counterpart in the reference: B200 build addition */
gg_context* ggems_device_context(GGEMS* g, int d);  /* no counterpart in the reference: B200 build addition */
const uint32_t* ggems_initial_random_states(GGEMS* g, int d);  /* no counterpart in the reference: B200 build addition */
void ggems_last_run(GGEMS* g, float* ms, int64_t* launches, uint64_t* particles);  /* no counterpart in the reference: B200 build addition */
const gg_scene* ggems_host_scene(void);  /* no counterpart in the reference: B200 build addition */
int ggems_number_of_sources(void);  /* no counterpart in the reference: B200 build addition */
int ggems_source_descriptor(int i, gg_source* out, uint64_t* number_of_particles);  /* no counterpart in the reference: B200 build addition */
void* get_instance_ggems_opencl_manager(void);  /* include/GGEMS/global/GGEMSOpenCLManager.hh:794 */
void print_infos_opencl_manager(void*);  /* include/GGEMS/global/GGEMSOpenCLManager.hh:801 */
void set_device_index_ggems_opencl_manager(void*, uint64_t id);  /* include/GGEMS/global/GGEMSOpenCLManager.hh:809 */
void set_device_to_activate_opencl_manager(void*, const char* type, const char* vendor);  /* include/GGEMS/global/GGEMSOpenCLManager.hh:818 */
void set_device_balancing_opencl_manager(void*, const char* balancing);  /* include/GGEMS/global/GGEMSOpenCLManager.hh:833 */
void clean_opencl_manager(void*);  /* include/GGEMS/global/GGEMSOpenCLManager.hh:825 */
void* get_instance_materials_manager(void);  /* include/GGEMS/materials/GGEMSMaterialsDatabaseManager.hh:316 */
void set_materials_ggems_materials_manager(void*, const char* filename);  /* include/GGEMS/materials/GGEMSMaterialsDatabaseManager.hh:324 */
void print_available_chemical_elements_ggems_materials_manager(void*);  /* include/GGEMS/materials/GGEMSMaterialsDatabaseManager.hh:331 */
void print_available_materials_ggems_materials_manager(void*);  /* include/GGEMS/materials/GGEMSMaterialsDatabaseManager.hh:338 */
void* get_instance_processes_manager(void);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:191 */
void add_process_processes_manager(void*, const char* process, const char* particle, const char* phantom);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:201 */
void set_cross_section_table_number_of_bins_processes_manager(void*, uint64_t bins);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:209 */
void set_cross_section_table_minimum_energy_processes_manager(void*, float e, const char* unit);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:218 */
void set_cross_section_table_maximum_energy_processes_manager(void*, float e, const char* unit);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:227 */
void print_infos_processes_manager(void*);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:234 */
void print_available_processes_manager(void*);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:241 */
void print_tables_processes_manager(void*, bool);  /* include/GGEMS/physics/GGEMSProcessesManager.hh:249 */
void* get_instance_range_cuts_manager(void);  /* include/GGEMS/physics/GGEMSRangeCutsManager.hh:127 */
void set_cut_range_cuts_manager(void*, const char* phantom, const char* particle, float value, const char* unit);  /* include/GGEMS/physics/GGEMSRangeCutsManager.hh:138 */
void* get_instance_ggems_source_manager(void);  /* include/GGEMS/sources/GGEMSSourceManager.hh:228 */
void initialize_source_manager(void*, uint32_t);  /* include/GGEMS/sources/GGEMSSourceManager.hh:236 */
void print_infos_source_manager(void*);  /* include/GGEMS/sources/GGEMSSourceManager.hh:243 */
void clean_source_manager(void*);  /* include/GGEMS/sources/GGEMSSourceManager.hh:250 */
GGEMSXRaySource* create_ggems_xray_source(const char* name);  /* include/GGEMS/sources/GGEMSXRaySource.hh:145 */
void set_position_ggems_xray_source(GGEMSXRaySource* s, float x, float y, float z, const char* unit);  /* include/GGEMS/sources/GGEMSXRaySource.hh:156 */
void set_number_of_particles_xray_source(GGEMSXRaySource* s, uint64_t n);  /* include/GGEMS/sources/GGEMSXRaySource.hh:164 */
void set_source_particle_type_ggems_xray_source(GGEMSXRaySource* s, const char* t);  /* include/GGEMS/sources/GGEMSXRaySource.hh:172 */
void set_beam_aperture_ggems_xray_source(GGEMSXRaySource* s, float a, const char* unit);  /* include/GGEMS/sources/GGEMSXRaySource.hh:181 */
void set_focal_spot_size_ggems_xray_source(GGEMSXRaySource* s, float w, float h, float d, const char* unit);  /* include/GGEMS/sources/GGEMSXRaySource.hh:192 */
void set_rotation_ggems_xray_source(GGEMSXRaySource* s, float rx, float ry, float rz, const char* unit);  /* include/GGEMS/sources/GGEMSXRaySource.hh:203 */
void set_monoenergy_ggems_xray_source(GGEMSXRaySource* s, float e, const char* unit);  /* include/GGEMS/sources/GGEMSXRaySource.hh:212 */
void set_polyenergy_ggems_xray_source(GGEMSXRaySource* s, const char* file);  /* include/GGEMS/sources/GGEMSXRaySource.hh:220 */
void set_energy_peak_ggems_xray_source(GGEMSXRaySource* s, float e, const char* unit, float intensity);  /* include/GGEMS/sources/GGEMSXRaySource.hh:230 */
GGEMSVoxelizedSource* create_ggems_voxelized_source(const char* name);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:143 */
void set_position_ggems_voxelized_source(GGEMSVoxelizedSource* s, float x, float y, float z, const char* unit);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:154 */
void set_rotation_ggems_voxelized_source(GGEMSVoxelizedSource* s, float rx, float ry, float rz, const char* unit);  /* no counterpart in the reference: B200 build addition */
void set_number_of_particles_voxelized_source(GGEMSVoxelizedSource* s, uint64_t n);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:162 */
void set_source_particle_type_ggems_voxelized_source(GGEMSVoxelizedSource* s, const char* t);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:170 */
void set_monoenergy_ggems_voxelized_source(GGEMSVoxelizedSource* s, float e, const char* unit);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:179 */
void set_polyenergy_ggems_voxelized_source(GGEMSVoxelizedSource* s, const char* file);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:187 */
void set_phantom_source_ggems_voxelized_source(GGEMSVoxelizedSource* s, const char* file);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:195 */
void set_energy_peak_ggems_voxelized_source(GGEMSVoxelizedSource* s, float e, const char* unit, float intensity);  /* include/GGEMS/sources/GGEMSVoxelizedSource.hh:205 */
GGEMSVoxelizedPhantom* create_ggems_voxelized_phantom(const char* name);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:119 */
void set_phantom_file_ggems_voxelized_phantom(GGEMSVoxelizedPhantom* p, const char* phantom, const char* range);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:128 */
void set_position_ggems_voxelized_phantom(GGEMSVoxelizedPhantom* p, float x, float y, float z, const char* unit);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:139 */
void set_rotation_ggems_voxelized_phantom(GGEMSVoxelizedPhantom* p, float rx, float ry, float rz, const char* unit);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:150 */
void set_visible_ggems_voxelized_phantom(GGEMSVoxelizedPhantom*, bool);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:158 */
void set_material_visible_ggems_voxelized_phantom(GGEMSVoxelizedPhantom*, const char*, bool);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:167 */
void set_material_color_ggems_voxelized_phantom(GGEMSVoxelizedPhantom*, const char*, unsigned char, unsigned char, unsigned char);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:178 */
void set_material_color_name_ggems_voxelized_phantom(GGEMSVoxelizedPhantom*, const char*, const char*);  /* include/GGEMS/navigators/GGEMSVoxelizedPhantom.hh:187 */
GGEMSMeshedPhantom* create_ggems_meshed_phantom(const char* name);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:125 */
void set_phantom_file_ggems_meshed_phantom(GGEMSMeshedPhantom* p, const char* stl_file);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:133 */
void set_position_ggems_meshed_phantom(GGEMSMeshedPhantom* p, float x, float y, float z, const char* unit);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:144 */
void set_rotation_ggems_meshed_phantom(GGEMSMeshedPhantom* p, float rx, float ry, float rz, const char* unit);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:155 */
void set_visible_ggems_meshed_phantom(GGEMSMeshedPhantom* p, bool flag);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:163 */
void set_material_name_ggems_meshed_phantom(GGEMSMeshedPhantom* p, const char* material);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:171 */
void set_material_color_ggems_meshed_phantom(GGEMSMeshedPhantom* p, const char* material, unsigned char r, unsigned char g, unsigned char b);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:182 */
void set_material_color_name_ggems_meshed_phantom(GGEMSMeshedPhantom* p, const char* material, const char* color);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:191 */
void set_mesh_octree_depth_ggems_meshed_phantom(GGEMSMeshedPhantom* p, int depth);  /* include/GGEMS/navigators/GGEMSMeshedPhantom.hh:199 */

/* GGEMSWorld: photon flights between solids recorded on a grid centred on the
 * origin; outputs <basename>_world_photon_tracking / _world_edep /
 * _world_edep_squared / _world_momentum_{x,y,z}.mhd */
GGEMSWorld* create_ggems_world(void);  /* include/GGEMS/navigators/GGEMSWorld.hh:231 */
void set_dimension_ggems_world(GGEMSWorld* w, size_t x, size_t y, size_t z);  /* include/GGEMS/navigators/GGEMSWorld.hh:241 */
void set_size_ggems_world(GGEMSWorld* w, float x, float y, float z, const char* unit);  /* include/GGEMS/navigators/GGEMSWorld.hh:252 */
void photon_tracking_ggems_world(GGEMSWorld* w, bool is_activated);  /* include/GGEMS/navigators/GGEMSWorld.hh:260 */
void energy_tracking_ggems_world(GGEMSWorld* w, bool is_activated);  /* include/GGEMS/navigators/GGEMSWorld.hh:268 */
void energy_squared_tracking_ggems_world(GGEMSWorld* w, bool is_activated);  /* include/GGEMS/navigators/GGEMSWorld.hh:276 */
void set_output_ggems_world(GGEMSWorld* w, const char* basename);  /* include/GGEMS/navigators/GGEMSWorld.hh:284 */
void momentum_ggems_world(GGEMSWorld* w, bool is_activated);  /* include/GGEMS/navigators/GGEMSWorld.hh:292 */

/* Volume creator: analytic shapes drawn into a voxel image on the device,
 * written as MHD plus a label -> material range file. */
GGEMSVolumeCreatorManager* get_instance_volume_creator_manager(void);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:294 */
void set_volume_dimension_volume_creator_manager(GGEMSVolumeCreatorManager* m, size_t width, size_t height, size_t depth);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:304 */
void set_element_sizes_volume_creator_manager(GGEMSVolumeCreatorManager* m, float width, float height, float depth, const char* unit);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:315 */
void set_output_image_filename_volume_creator_manager(GGEMSVolumeCreatorManager* m, const char* filename);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:323 */
void set_output_range_to_material_filename_volume_creator_manager(GGEMSVolumeCreatorManager* m, const char* filename);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:331 */
void initialize_volume_creator_manager(GGEMSVolumeCreatorManager* m);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:338 */
void write_volume_creator_manager(GGEMSVolumeCreatorManager* m);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:345 */
void set_material_volume_creator_manager(GGEMSVolumeCreatorManager* m, const char* material);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:353 */
void set_data_type_volume_creator_manager(GGEMSVolumeCreatorManager* m, const char* data_type);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:361 */
void clean_volume_creator_manager(GGEMSVolumeCreatorManager* m);  /* include/GGEMS/geometries/GGEMSVolumeCreatorManager.hh:368 */
GGEMSBox* create_box(float width, float height, float depth, const char* unit);  /* include/GGEMS/geometries/GGEMSBox.hh:112 */
void delete_box(GGEMSBox* box);  /* include/GGEMS/geometries/GGEMSBox.hh:119 */
void set_position_box(GGEMSBox* box, float x, float y, float z, const char* unit);  /* include/GGEMS/geometries/GGEMSBox.hh:130 */
void set_material_box(GGEMSBox* box, const char* material);  /* include/GGEMS/geometries/GGEMSBox.hh:138 */
void set_label_value_box(GGEMSBox* box, float label_value);  /* include/GGEMS/geometries/GGEMSBox.hh:146 */
void initialize_box(GGEMSBox* box);  /* include/GGEMS/geometries/GGEMSBox.hh:153 */
void draw_box(GGEMSBox* box);  /* include/GGEMS/geometries/GGEMSBox.hh:160 */
GGEMSTube* create_tube(float radius_x, float radius_y, float height, const char* unit);  /* include/GGEMS/geometries/GGEMSTube.hh:112 */
void delete_tube(GGEMSTube* tube);  /* include/GGEMS/geometries/GGEMSTube.hh:119 */
void set_position_tube(GGEMSTube* tube, float x, float y, float z, const char* unit);  /* include/GGEMS/geometries/GGEMSTube.hh:130 */
void set_material_tube(GGEMSTube* tube, const char* material);  /* include/GGEMS/geometries/GGEMSTube.hh:138 */
void set_label_value_tube(GGEMSTube* tube, float label_value);  /* include/GGEMS/geometries/GGEMSTube.hh:146 */
void initialize_tube(GGEMSTube* tube);  /* include/GGEMS/geometries/GGEMSTube.hh:153 */
void draw_tube(GGEMSTube* tube);  /* include/GGEMS/geometries/GGEMSTube.hh:160 */
GGEMSSphere* create_sphere(float radius, const char* unit);  /* include/GGEMS/geometries/GGEMSSphere.hh:106 */
void delete_sphere(GGEMSSphere* sphere);  /* include/GGEMS/geometries/GGEMSSphere.hh:113 */
void set_position_sphere(GGEMSSphere* sphere, float x, float y, float z, const char* unit);  /* include/GGEMS/geometries/GGEMSSphere.hh:124 */
void set_material_sphere(GGEMSSphere* sphere, const char* material);  /* include/GGEMS/geometries/GGEMSSphere.hh:132 */
void set_label_value_sphere(GGEMSSphere* sphere, float label_value);  /* include/GGEMS/geometries/GGEMSSphere.hh:140 */
void initialize_sphere(GGEMSSphere* sphere);  /* include/GGEMS/geometries/GGEMSSphere.hh:147 */
void draw_sphere(GGEMSSphere* sphere);  /* include/GGEMS/geometries/GGEMSSphere.hh:154 */
int ggems_build_mesh(const char* stl, const float* matrix, int depth, int32_t* n_triangles, int32_t* n_nodes, float* triangles, float* nodes, int32_t* node_first, int32_t* node_triangles, float* border_min, float* border_max);  /* no counterpart in the reference: B200 build addition */
GGEMSCTSystem* create_ggems_ct_system(const char* name);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:141 */
void set_number_of_modules_ggems_ct_system(GGEMSCTSystem* c, uint64_t mx, uint64_t my);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:150 */
void set_ct_system_type_ggems_ct_system(GGEMSCTSystem* c, const char* type);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:158 */
void set_number_of_detection_elements_ggems_ct_system(GGEMSCTSystem* c, uint64_t x, uint64_t y, uint64_t z);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:168 */
void set_size_of_detection_elements_ggems_ct_system(GGEMSCTSystem* c, float x, float y, float z, const char* unit);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:179 */
void set_material_name_ggems_ct_system(GGEMSCTSystem* c, const char* material);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:187 */
void set_source_isocenter_distance_ggems_ct_system(GGEMSCTSystem* c, float d, const char* unit);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:196 */
void set_source_detector_distance_ggems_ct_system(GGEMSCTSystem* c, float d, const char* unit);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:205 */
void set_rotation_ggems_ct_system(GGEMSCTSystem* c, float rx, float ry, float rz, const char* unit);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:216 */
void set_save_ggems_ct_system(GGEMSCTSystem* c, const char* basename);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:233 */
void set_threshold_ggems_ct_system(GGEMSCTSystem* c, float t, const char* unit);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:225 */
void store_scatter_ggems_ct_system(GGEMSCTSystem* c, bool s);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:241 */
void set_global_system_position_ggems_ct_system(GGEMSCTSystem* c, float x, float y, float z, const char* unit);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:280 */
void set_visible_ggems_ct_system(GGEMSCTSystem*, bool);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:249 */
void set_material_color_ggems_ct_system(GGEMSCTSystem*, const char*, unsigned char, unsigned char, unsigned char);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:260 */
void set_material_color_name_ggems_ct_system(GGEMSCTSystem*, const char*, const char*);  /* include/GGEMS/navigators/GGEMSCTSystem.hh:269 */
GGEMSDosimetryCalculator* create_ggems_dosimetry_calculator(void);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:318 */
void delete_dosimetry_calculator(GGEMSDosimetryCalculator* d);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:325 */
void scale_factor_dosimetry_calculator(GGEMSDosimetryCalculator* d, float s);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:333 */
void water_reference_dosimetry_calculator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:341 */
void minimum_density_dosimetry_calculator(GGEMSDosimetryCalculator* d, float v, const char* unit);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:350 */
void set_dosel_size_dosimetry_calculator(GGEMSDosimetryCalculator* d, float x, float y, float z, const char* unit);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:361 */
void set_dose_output_dosimetry_calculator(GGEMSDosimetryCalculator* d, const char* f);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:369 */
void dose_photon_tracking_dosimetry_calculator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:377 */
void dose_edep_dosimetry_calculator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:385 */
void dose_hit_dosimetry_calculator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:393 */
void dose_edep_squared_dosimetry_calculator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:401 */
void dose_uncertainty_dosimetry_calculator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:409 */
void dose_tle_navigator(GGEMSDosimetryCalculator* d, bool b);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:417 */
void attach_to_navigator_dosimetry_calculator(GGEMSDosimetryCalculator* d, const char* navigator);  /* include/GGEMS/navigators/GGEMSDosimetryCalculator.hh:425 */
GGEMSMaterials* create_ggems_materials(void);  /* include/GGEMS/materials/GGEMSMaterials.hh:219 */
void add_material_ggems_materials(GGEMSMaterials* m, const char* name);  /* include/GGEMS/materials/GGEMSMaterials.hh:227 */
void initialize_ggems_materials(GGEMSMaterials* m);  /* include/GGEMS/materials/GGEMSMaterials.hh:234 */
void print_material_properties_ggems_materials(GGEMSMaterials* m);  /* include/GGEMS/materials/GGEMSMaterials.hh:241 */
float get_density_ggems_materials(GGEMSMaterials* m, const char* name);  /* include/GGEMS/materials/GGEMSMaterials.hh:250 */
float get_energy_cut_ggems_materials(GGEMSMaterials* m, const char* name, const char* particle, float distance, const char* unit);  /* include/GGEMS/materials/GGEMSMaterials.hh:262 */
float get_atomic_number_density_ggems_materials(GGEMSMaterials* m, const char* name);  /* include/GGEMS/materials/GGEMSMaterials.hh:271 */
void clean_ggems_materials(GGEMSMaterials*);  /* include/GGEMS/materials/GGEMSMaterials.hh:278 */
GGEMSCrossSections* create_ggems_cross_sections(GGEMSMaterials* m);  /* include/GGEMS/physics/GGEMSCrossSections.hh:173 */
void add_process_ggems_cross_sections(GGEMSCrossSections* c, const char* process, const char* particle, bool);  /* include/GGEMS/physics/GGEMSCrossSections.hh:183 */
void initialize_ggems_cross_sections(GGEMSCrossSections* c);  /* include/GGEMS/physics/GGEMSCrossSections.hh:190 */
float get_cs_ggems_cross_sections(GGEMSCrossSections* c, const char* process, const char* material, float energy, const char* unit);  /* include/GGEMS/physics/GGEMSCrossSections.hh:202 */
void clean_ggems_cross_sections(GGEMSCrossSections*);  /* include/GGEMS/physics/GGEMSCrossSections.hh:209 */
GGEMSAttenuations* create_ggems_attenuations(GGEMSMaterials* m, GGEMSCrossSections* c);  /* include/GGEMS/physics/GGEMSAttenuations.hh:157 */
void initialize_ggems_attenuations(GGEMSAttenuations* a);  /* include/GGEMS/physics/GGEMSAttenuations.hh:164 */
float get_mu_ggems_attenuations(GGEMSAttenuations* a, const char* material, float energy, const char* unit);  /* include/GGEMS/physics/GGEMSAttenuations.hh:175 */
float get_mu_en_ggems_attenuations(GGEMSAttenuations* a, const char* material, float energy, const char* unit);  /* include/GGEMS/physics/GGEMSAttenuations.hh:186 */
void clean_ggems_attenuations(GGEMSAttenuations* a);  /* include/GGEMS/physics/GGEMSAttenuations.hh:193 */
void* get_instance_profiler_manager(void);  /* include/GGEMS/tools/GGEMSProfilerManager.hh:138 */
void print_summary_profiler_manager(void*);  /* include/GGEMS/tools/GGEMSProfilerManager.hh:145 */
void* get_instance_ggems_ram_manager(void);  /* include/GGEMS/tools/GGEMSRAMManager.hh:174 */
void print_infos_ram_manager(void*);  /* include/GGEMS/tools/GGEMSRAMManager.hh:181 */
int ggems_build_tables(const char* materials_file, const char* const* material_names, int n_materials, int number_of_bins, float min_energy, float max_energy, const int* process_ids, int n_processes, float photon_distance_cut, float* energy_bins, float* cross_sections, float* rayleigh, float* density, float* photon_cut, int32_t* n_elements, int32_t* element_offset, uint8_t* atomic_number, float* atomic_number_density, int32_t* total_elements);  /* no counterpart in the reference: B200 build addition */
int ggems_phantom_labels(const char* phantom_file, const char* range_file, int32_t* dims, float* spacing, uint8_t* labels);  /* no counterpart in the reference: B200 build addition */

#ifdef __cplusplus
}
#endif

#endif /* GGEMS_API_H */
