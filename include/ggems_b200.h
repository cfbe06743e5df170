/*
 * ggems_b200.h - C ABI of the B200 photon-transport layer.
 *
 * This is the thin device layer that replaces GGEMS's OpenCL manager and
 * command-queue plumbing (include/GGEMS/global/GGEMSOpenCLManager.hh:384-495,
 * src/global/GGEMSOpenCLManager.cc:836-1046) for the photon hot path.  The C++
 * host classes (GGEMS, GGEMSXRaySource, GGEMSVoxelizedPhantom, GGEMSCTSystem,
 * GGEMSDosimetryCalculator, ...) build a scene description out of plain
 * arrays and call these entry points; nothing here exposes CUDA or torch
 * types.  Every function returns a gg_status code; gg_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Units are GGEMS's internal units (include/GGEMS/tools/GGEMSSystemOfUnits.hh):
 * mm, MeV, rad, g = 6.241509704e21.
 */
#ifndef GGEMS_B200_H
#define GGEMS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define GG_API __attribute__((visibility("default")))
#else
#define GG_API
#endif

/* Particle slots per batch: GGEMS's MAXIMUM_PARTICLES (CMakeLists.txt:128-132). */
#define GG_MAXIMUM_PARTICLES 1048576
/* Limits of the reference's fixed-size tables. */
#define GG_MAX_CROSS_SECTION_BINS 2048 /* GGEMSProcessConstants.hh MAX_CROSS_SECTION_TABLE_NUMBER_BINS */
#define GG_MAX_MATERIALS 255           /* GGEMSMaterialTables.hh:44-77 */
#define GG_MAX_LOOP 100                /* src/global/GGEMS.cc:330 */

typedef enum gg_status {
  GG_OK = 0,
  GG_ERROR_INVALID_ARGUMENT = 1,
  GG_ERROR_CUDA = 2,
  GG_ERROR_NO_DEVICE = 3,
  GG_ERROR_OUT_OF_MEMORY = 4,
  GG_ERROR_STATE = 5,
  /* A bounded wait inside a kernel gave up (the transport kernel's table
   * staging, the tensor-core convolution's operand pipeline).  The failing
   * blocks may have exited with copies into their shared memory still in
   * flight: destroy and recreate the context before running on. */
  GG_ERROR_TIMEOUT = 6
} gg_status;

/* Attenuation (mu, mu_en) table size: ATTENUATION_TABLE_NUMBER_BINS
 * (include/GGEMS/physics/GGEMSProcessConstants.hh:62-64). */
#define GG_ATTENUATION_BINS 220

/* Photon process identifiers (include/GGEMS/physics/GGEMSProcessConstants.hh). */
#define GG_COMPTON_SCATTERING 0
#define GG_PHOTOELECTRIC_EFFECT 1
#define GG_RAYLEIGH_SCATTERING 2
#define GG_TRANSPORTATION 99

/* Particle status (include/GGEMS/physics/GGEMSParticleConstants.hh). */
#define GG_ALIVE 0
#define GG_DEAD 1

/* Oriented bounding box: GGEMSOBB (include/GGEMS/geometries/GGEMSPrimitiveGeometries.hh:41-46).
 * matrix = GGfloat44, 4 rows of 4 floats (row-major), local -> global. */
typedef struct gg_obb {
  float matrix[16];
  float border_min[3];
  float border_max[3];
} gg_obb;

/* Per-navigator physics tables: the part of GGEMSParticleCrossSections
 * (include/GGEMS/physics/GGEMSParticleCrossSections.hh:40-58) and of
 * GGEMSMaterialTables (include/GGEMS/materials/GGEMSMaterialTables.hh:41-77)
 * that photon transport reads. */
typedef struct gg_physics_tables {
  int32_t number_of_bins;
  int32_t number_of_materials;
  int32_t number_of_processes;          /* activated photon processes */
  int32_t process_id[3];                /* photon_cs_id_: AddProcess order */
  const float* energy_bins;             /* [number_of_bins] MeV, log spaced */
  const float* cross_sections;          /* [3][number_of_materials*number_of_bins] mm^-1,
                                           indexed [process][bin + number_of_bins*material] */
  const float* rayleigh_per_atom;       /* [101*number_of_bins] mm^2, [bin + number_of_bins*Z];
                                           NULL when Rayleigh is not activated */
  const float* density;                 /* [number_of_materials] internal units */
  const float* photon_energy_cut;       /* [number_of_materials] MeV */
  const int32_t* number_of_elements;    /* [number_of_materials] */
  const int32_t* element_offset;        /* [number_of_materials] index into the element arrays */
  const uint8_t* atomic_number;         /* [total_elements] */
  const float* atomic_number_density;   /* [total_elements] atoms / mm^3 */
  int32_t total_elements;
  /* Track-length-estimator tables: the part of GGEMSMuMuEnData
   * (include/GGEMS/physics/GGEMSMuData.hh:41-52) the TLE dose step reads;
   * NULL when no dose map of this navigator uses TLE. */
  const float* attenuation_energy_bins; /* [GG_ATTENUATION_BINS] MeV, log spaced 1 keV - 1 MeV */
  const float* mu_en;                   /* [number_of_materials*GG_ATTENUATION_BINS] cm^-1,
                                           indexed [bin + GG_ATTENUATION_BINS*material] */
} gg_physics_tables;

typedef enum gg_solid_type {
  GG_SOLID_VOXELIZED = 0,
  GG_SOLID_BOX = 1,
  GG_SOLID_MESHED = 2
} gg_solid_type;

/* One solid.  Solids are listed in GGEMS's registration order, which is
 * also the order of the FindSolid / ProjectToSolid / TrackThroughSolid loops
 * (src/navigators/GGEMSNavigatorManager.cc, GGEMSNavigator.cc:320-530). */
typedef struct gg_solid {
  int32_t type;                 /* gg_solid_type */
  int32_t navigator;            /* index of this solid's gg_physics_tables */
  gg_obb obb;
  float threshold;              /* navigator energy threshold (MeV) */
  /* voxelized solid: GGEMSVoxelizedSolidData */
  int32_t number_of_voxels[3];
  float voxel_sizes[3];
  const uint8_t* labels;        /* [nx*ny*nz] material index, x fastest */
  /* solid box (CT detector module): GGEMSSolidBoxData */
  int32_t virtual_element_number[3];
  float box_size[3];
  int32_t histogram;            /* index of the interaction histogram, -1: none */
  int32_t scatter_histogram;    /* index of the scatter histogram, -1: none */
  /* dosimetry */
  int32_t dose_map;             /* index into gg_scene.dose_maps, -1: none */
  /* meshed solid: GGEMSMeshedSolidData (include/GGEMS/geometries/GGEMSMeshedSolidData.hh:40-49)
   * with its octree (src/geometries/GGEMSOctree.cc).  Triangles are in world
   * coordinates (the solid's rotation and translation already applied) and the
   * OBB is the octree box with an identity matrix, as GGEMS leaves them. */
  int32_t number_of_triangles;
  const float* triangles;       /* [number_of_triangles][GG_TRIANGLE_FLOATS]: vertices p0, p1, p2,
                                   bounding-sphere center, radius */
  int32_t number_of_nodes;      /* (8^depth - 1) / 7 */
  const float* nodes;           /* [number_of_nodes][6]: center xyz, half width xyz */
  const int32_t* node_first;    /* [number_of_nodes + 1]: node n owns node_triangles[node_first[n] .. node_first[n+1]) */
  const int32_t* node_triangles;/* triangle indices, per node in the order GGEMS's linked list visits them */
} gg_solid;

/* Floats per triangle in gg_solid.triangles. */
#define GG_TRIANGLE_FLOATS 13

/* Dose map: GGEMSDoseParams (include/GGEMS/navigators/GGEMSDoseParams.hh:40-49)
 * plus which optional tallies are recorded. */
typedef struct gg_dose_map {
  float size_of_dosels[3];
  float inv_size_of_dosels[3];
  float border_min[3];
  float border_max[3];
  int32_t number_of_dosels[3];
  int32_t total_number_of_dosels;
  int32_t slice_number_of_dosels;
  int32_t record_edep_squared;
  int32_t record_hit;
  int32_t record_photon_tracking;
  int32_t tle;                  /* track-length estimator instead of interaction deposits
                                   (TrackThroughGGEMSVoxelizedSolid.cl:286-301) */
} gg_dose_map;

/* World tracking: GGEMSWorld (src/navigators/GGEMSWorld.cc,
 * src/kernels/WorldTracking.cl) -- a coarse grid centred on the origin that
 * tallies the flight of every photon between solids. */
typedef struct gg_world {
  int32_t dimensions[3];
  float sizes[3];               /* mm */
  int32_t photon_tracking;      /* record crossings (int32) */
  int32_t energy_tracking;      /* record E (MeV) */
  int32_t energy_squared_tracking;
  int32_t momentum;             /* record direction components */
} gg_world;

typedef struct gg_scene {
  int32_t number_of_tables;
  const gg_physics_tables* tables;
  int32_t number_of_solids;
  const gg_solid* solids;
  int32_t number_of_dose_maps;
  const gg_dose_map* dose_maps;
  int32_t number_of_histograms;
  const int32_t* histogram_sizes;   /* elements per histogram */
  const float* rayleigh_fit;        /* [9][101] Livermore form-factor fit PP0..PP8
                                       (GGEMSRayleighScatteringModels.hh:36-153) */
  const gg_world* world;            /* NULL: no world tracking */
} gg_scene;

typedef enum gg_source_type {
  GG_SOURCE_XRAY = 0,
  GG_SOURCE_VOXELIZED = 1
} gg_source_type;

/* A primary source.  X-ray cone source: GGEMSXRaySource
 * (src/sources/GGEMSXRaySource.cc:100-148, src/kernels/GetPrimariesGGEMSXRaySource.cl). */
typedef struct gg_source {
  int32_t type;                  /* gg_source_type */
  int32_t particle_type;         /* 0 photon */
  float matrix[16];              /* source frame, GGfloat44 */
  float beam_aperture;           /* rad */
  float focal_spot_size[3];      /* mm */
  int32_t number_of_energy_bins; /* n; spectrum and cdf hold n+1 values */
  const float* energy_spectrum;  /* [n+1] MeV, last value repeated */
  const float* energy_cdf;       /* [n+1], cdf[0] = 0, cdf[n] = 1 */
  int32_t is_interp;             /* linear interpolation inside the cdf bin */
  /* voxelized source (GGEMSVoxelizedSource): activity CDF over active voxels */
  int32_t number_of_voxels[3];
  float voxel_sizes[3];
  float border_min[3];
  int64_t number_of_activity_bins;  /* entries of activity_index / activity_cdf: active voxels + 1
                                       (the count GGEMSVoxelizedSource.cc:170 passes to the kernel) */
  const int32_t* activity_index;    /* [number_of_activity_bins] voxel index, entry 0 unused (0) */
  const float* activity_cdf;        /* [number_of_activity_bins], cdf[0] = 0 */
} gg_source;

/* Final per-slot particle state (the photon part of GGEMSPrimaryParticles,
 * include/GGEMS/physics/GGEMSPrimaryParticles.hh:40-68), host SoA buffers. */
typedef struct gg_particle_buffers {
  float* E;
  float* px;
  float* py;
  float* pz;
  float* dx;
  float* dy;
  float* dz;
  int8_t* status;
  int8_t* scatter;
  int32_t* solid_id;
} gg_particle_buffers;

/* Host tally buffers, one pointer per histogram / dose map (NULL to skip). */
typedef struct gg_tally_buffers {
  int32_t** histograms;
  double** edep;
  double** edep_squared;
  int32_t** hit;
  int32_t** photon_tracking;
  /* world grid tallies (NULL to skip), dimensions[0]*dimensions[1]*dimensions[2] each */
  int32_t* world_photon_tracking;
  double* world_energy;
  double* world_energy_squared;
  double* world_momentum_x;
  double* world_momentum_y;
  double* world_momentum_z;
} gg_tally_buffers;

typedef struct gg_context gg_context;

/* ---- device selection and context (replaces GGEMSOpenCLManager) ---- */
GG_API int gg_device_count(int32_t* count);
GG_API int gg_context_create(int32_t device_index, gg_context** context);
GG_API int gg_context_destroy(gg_context* context);
GG_API const char* gg_last_error(void);

/* ---- random streams (GGEMSPseudoRandomGenerator) ----
 * states: 5 arrays of number_of_slots uint32 (prng_state_1_ .. prng_state_5_),
 * stored one after the other. */
GG_API int gg_set_random_states(gg_context* context, const uint32_t* states, int64_t number_of_slots);
GG_API int gg_get_random_states(gg_context* context, uint32_t* states, int64_t number_of_slots);
/* JKISS seeding of GGEMSPseudoRandomGenerator::InitializeSeeds
 * (src/randoms/GGEMSPseudoRandomGenerator.cc:140-167): slot j takes four
 * consecutive std::mt19937(seed) outputs, starting after skip_slots*4 draws. */
GG_API int gg_seed_random_states(uint32_t* states, int64_t number_of_slots, uint32_t seed, int64_t skip_slots);

/* ---- scene upload and tallies ---- */
GG_API int gg_upload_scene(gg_context* context, const gg_scene* scene);
GG_API int gg_reset_tallies(gg_context* context);
GG_API int gg_read_tallies(gg_context* context, gg_tally_buffers* tallies);
GG_API int gg_read_particles(gg_context* context, gg_particle_buffers* particles, int64_t number_of_slots);

/* ---- transport ----
 * Runs number_of_particles primaries of one source through the scene,
 * split into batches exactly as GGEMSSource::OrganizeParticlesInBatch
 * (src/sources/GGEMSSource.cc:379-426) and GGEMS::RunOnDevice
 * (src/global/GGEMS.cc:303-363): particle i of every batch uses random
 * slot i.  Asynchronous on the context's stream. */
GG_API int gg_run_source(gg_context* context, const gg_source* source, uint64_t number_of_particles);
GG_API int gg_synchronize(gg_context* context);

/* ---- batched runs (no counterpart in the reference: GGEMS runs sources and
 * geometries one after another) ----
 * A job is one source run with its own geometry: `solids` lists
 * number_of_solids solids of the uploaded scene's layout (same navigators;
 * their matrices, labels, meshes and histogram / dose-map indices are the
 * job's), or NULL for the scene's.  gg_run_jobs runs all jobs in ONE launch
 * and gives exactly what gg_run_source would give for each job in turn with
 * the solids swapped: slot i runs its histories of job 0, then of job 1, ...,
 * its random stream carried from job to job.  Tallies of different jobs are
 * kept apart by giving them different histogram / dose-map indices. */
typedef struct gg_job {
  gg_source source;
  uint64_t number_of_particles;
  const gg_solid* solids;
} gg_job;
GG_API int gg_run_jobs(gg_context* context, const gg_job* jobs, int32_t number_of_jobs);

/* The same batched launch captured once in a CUDA graph (work-queue reset +
 * persistent kernel) and replayed by gg_graph_launch: each replay is another
 * acquisition of the same jobs, the random streams carrying on.  The jobs'
 * device tables live with the graph; a graph stays valid until the context's
 * scene is uploaded again or the graph is destroyed. */
typedef struct gg_graph gg_graph;
GG_API int gg_capture_jobs(gg_context* context, const gg_job* jobs, int32_t number_of_jobs, gg_graph** graph);
GG_API int gg_graph_launch(gg_graph* graph);
GG_API int gg_graph_destroy(gg_graph* graph);

/* Launch shape of the transport kernel (no counterpart in the reference; its
 * GGEMSOpenCLManager::GetBestWorkItem / GetWorkGroupSize pick one work item
 * per photon and a fixed work-group size):
 * - resident blocks per SM (0: as many as fit) and the warp scheduling of the
 *   rare phases (regroup_lanes 1..32, regroup_ratio4 0..128):
 *   gg_set_transport_tuning;
 * - the block size (128, 256 or 512 threads) and the photons per thread, i.e.
 *   the consecutive random slots a lane takes from the work queue at a time
 *   and runs one after another (a power of two, 1..64): gg_set_transport_launch.
 * gg_autotune times short runs of `source` (gg_autotune_jobs: of a batched
 * launch of `jobs`, e.g. a sample of the job mix to run) over a coordinate
 * search of these knobs and the photon stash (gg_set_transport_stash), keeps the fastest and reports its time; it
 * restores the random states and zeroes the tallies afterwards, so call it
 * before the real run.  The results do not depend on the launch shape. */
GG_API int gg_set_transport_tuning(gg_context* context, int32_t blocks_per_sm, int32_t regroup_lanes,
                                   int32_t regroup_ratio4);
GG_API int gg_get_transport_tuning(gg_context* context, int32_t* blocks_per_sm, int32_t* regroup_lanes,
                                   int32_t* regroup_ratio4);
GG_API int gg_set_transport_launch(gg_context* context, int32_t block_threads, int32_t slots_per_claim);
GG_API int gg_get_transport_launch(gg_context* context, int32_t* block_threads, int32_t* slots_per_claim);
/* Photon stash (scenes without a world grid or particle tracking; meshed
 * scenes use it at 80 registers whenever it is on): each warp parks a second set of photons
 * in shared memory and exchanges them with its lanes, so that a lane whose
 * photon waits for a rare phase (new history, FindSolid, Compton / Rayleigh
 * sampling) tracks a parked photon meanwhile, and the rare phases run on full
 * warps.  registers: 0 (off), 64 or 80 per thread (the kernel variant's
 * budget: 4 or 3 resident 256-thread blocks per SM); swap_lanes (1..32): the
 * waiting lanes that start an exchange; round_photons (1..64): the photons of
 * a warp (lanes and records) waiting for a rare phase that start a rare round.
 * Default 80, 4 and 40 (environment overrides at context creation:
 * GGEMS_B200_STASH_REGISTERS, GGEMS_B200_STASH_SWAP, GGEMS_B200_STASH_ROUND).
 * The results do not depend on them. */
GG_API int gg_set_transport_stash(gg_context* context, int32_t registers, int32_t swap_lanes, int32_t round_photons);
GG_API int gg_get_transport_stash(gg_context* context, int32_t* registers, int32_t* swap_lanes,
                                  int32_t* round_photons);
GG_API int gg_autotune(gg_context* context, const gg_source* source, uint64_t number_of_particles,
                       float* best_milliseconds);
GG_API int gg_autotune_jobs(gg_context* context, const gg_job* jobs, int32_t number_of_jobs, float* best_milliseconds);

/* ---- scatter surrogate (no counterpart in the reference) ----
 * A 4-level BF16 U-Net (base 32 channels, FP32 accumulation) mapping a CBCT
 * primary projection and the phantom's line-integral map to the scatter
 * projection, trained and run with this library's own kernels
 * (ggems_b200/csrc/gg_unet.cu, convolutions on tcgen05 in gg_unet_umma.cu).
 * Images are square, side a power of two (>= 64).  A call whose tensor-core
 * convolution gave up waiting for its operands returns GG_ERROR_TIMEOUT.
 * Arrays are DEVICE pointers: input [batch][side][side][2] (primary, line
 * integral), target / output [batch][side][side], all FP32.  Parameters are a
 * flat FP32 vector of gg_unet_parameter_count() values. */
/* Line integral of mu (mm^-1 per material label) along the ray from
 * source_position (world, mm) to the centre of every element of the detector
 * box solid, through the voxelized phantom solid (host labels):
 * out[j * nx + i] for element (i, j), as the detector histogram bins.  No
 * counterpart in the reference: input of the scatter surrogate. */
GG_API int gg_line_integrals(gg_context* context, const gg_solid* phantom, const gg_solid* detector,
                             const float* source_position, const float* mu, int32_t number_of_materials,
                             float* line_integrals);
/* The same for `count` projections of one phantom (a scan): detectors[count]
 * and source_positions[count][3], written as the surrogate network's input,
 * inputs[count][ey][ex][2] = (exp(-L), L) (FP32; a host array, or an array in
 * the context's device memory, which the kernels then write directly).  Returns
 * once the inputs are written. */
GG_API int gg_line_integrals_batch(gg_context* context, const gg_solid* phantom, const gg_solid* detectors,
                                   const float* source_positions, int32_t count, const float* mu,
                                   int32_t number_of_materials, float* inputs);
typedef struct gg_unet gg_unet;
GG_API int gg_unet_create(int32_t batch, int32_t side, uint64_t seed, gg_unet** net);
GG_API int gg_unet_destroy(gg_unet* net);
GG_API int64_t gg_unet_parameter_count(const gg_unet* net);
GG_API int gg_unet_get_parameters(gg_unet* net, float* host_parameters);
GG_API int gg_unet_set_parameters(gg_unet* net, const float* host_parameters);
GG_API int gg_unet_forward(gg_unet* net, const float* input, float* output);
GG_API int gg_unet_gradients(gg_unet* net, const float* input, const float* target, float* loss,
                             float* host_gradients);
GG_API int gg_unet_train_step(gg_unet* net, const float* input, const float* target, float learning_rate,
                              float* loss);
GG_API const char* gg_unet_last_error(void);

/* Batch plan of GGEMSSource::OrganizeParticlesInBatch for one device.
 * Writes at most max_batches sizes; returns the number of batches in *count. */
GG_API int gg_batch_plan(uint64_t number_of_particles, uint64_t* batch_sizes, int64_t max_batches, int64_t* count);

/* ---- device tallies for collectives (no counterpart in the reference:
 * GGEMSSystem::SaveResults and GGEMSDosimetryCalculator read every device's
 * buffers back and sum them on the host) ----
 * The device buffers that hold a context's tallies, in a fixed order
 * (histograms; per dose map edep, edep^2, hit, photon tracking where
 * recorded; world photon count, energy, energy^2, momentum where recorded),
 * so that a multi-GPU run sums them across GPUs in place (one all-reduce per
 * buffer, e.g. NCCL over NVLink) before gg_read_tallies.  Addresses stay
 * valid until the next gg_upload_scene.  edep, world energy and momentum are
 * int64 fixed point (LSB 2^-32 MeV): their sums are exact and do not depend
 * on the order.  With tallies == NULL only *count is set. */
#define GG_TALLY_INT32 0
#define GG_TALLY_INT64 1
#define GG_TALLY_FP64 2
typedef struct gg_device_tally {
  void* address;  /* device address */
  int64_t count;  /* elements */
  int32_t type;   /* GG_TALLY_* */
} gg_device_tally;
GG_API int gg_device_tallies(gg_context* context, gg_device_tally* tallies, int32_t capacity, int32_t* count);

/* ---- dose finalisation (ComputeDoseGGEMSVoxelizedSolid.cl) ----
 * Converts the edep tally of dose_map (recorded inside solid) into Gy and the
 * relative uncertainty of Ma et al.; outputs are host arrays of
 * total_number_of_dosels floats (uncertainty may be NULL). */
GG_API int gg_compute_dose(gg_context* context, int32_t dose_map, int32_t solid, float scale_factor,
                           int32_t is_water_reference, float minimum_density, float* dose, float* uncertainty);

/* Same result as gg_compute_dose, but allocates no device memory: for hosts
 * that must not call cudaMalloc/cudaFree while dose maps are finalised (cudaFree
 * synchronises the whole device and stalls transport running on other
 * streams; a process whose caching allocator holds the free memory may not get
 * any).  No counterpart in the reference.
 * Outputs go through one fixed device array per GPU of 2 x GG_NO_ALLOC_MAX_DOSELS
 * floats (16 MiB), held from library load until process exit; larger dose maps
 * are rejected with GG_ERROR_INVALID_ARGUMENT.  The first call on a device looks
 * up that array's address (once per device), so make it before any stream
 * capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset on a device that has already made a call, this entry point
 * is not supported on that device (the module is reloaded at a new address).
 * All calls on one device share the array: calls that overlap (two threads,
 * or two contexts on the same GPU) race and must be serialised by the
 * caller. */
#define GG_NO_ALLOC_MAX_DOSELS 2097152
GG_API int gg_compute_dose_no_alloc(gg_context* context, int32_t dose_map, int32_t solid, float scale_factor,
                                    int32_t is_water_reference, float minimum_density, float* dose,
                                    float* uncertainty);

/* ---- particle tracking (GGEMS_TRACKING, e.g. TrackThroughGGEMSVoxelizedSolid.cl:184-210) ----
 * The states of one random slot (GGEMS's particle_tracking_id: particle i of
 * every batch) recorded by the transport kernel at each stage of its
 * histories, up to a capacity; read back after a run.  slot < 0 turns it off. */
typedef enum gg_track_kind {
  GG_TRACK_PRIMARY = 0,   /* a new history: global position and direction */
  GG_TRACK_ENTER = 1,     /* projected into a solid (solid-local frame, meshed solids global) */
  GG_TRACK_STEP = 2,      /* a step inside a solid: process (GG_TRANSPORTATION when none) */
  GG_TRACK_SCATTER = 3,   /* after a Compton / Rayleigh interaction */
  GG_TRACK_LEAVE = 4,     /* left the solid (global frame) */
  GG_TRACK_DEAD = 5       /* the history ended */
} gg_track_kind;

typedef struct gg_track_point {
  int32_t kind;           /* gg_track_kind */
  int32_t solid;          /* solid index, -1 outside */
  int32_t process;        /* GG_COMPTON_SCATTERING ... GG_TRANSPORTATION, -1 */
  int32_t history;        /* history of the slot within the run (0, 1, ...) */
  float E;                /* MeV */
  float position[3];      /* mm */
  float direction[3];
  float pad;
} gg_track_point;

GG_API int gg_set_tracking(gg_context* context, int32_t slot, int32_t capacity);
/* Copies up to `capacity` points of the last run; *count = points recorded
 * (may exceed what was stored: the buffer keeps the first ones). */
GG_API int gg_read_tracking(gg_context* context, gg_track_point* points, int32_t capacity, int32_t* count);

/* ---- timing of the last gg_run_source (device time, ms) and launch count ---- */
GG_API int gg_last_run_stats(gg_context* context, float* milliseconds, int64_t* kernel_launches);

/* ---- phantom volumes on the device ----
 * A voxel image of one MHD element type held in device memory: analytic shapes
 * are drawn into it (GGEMSVolumeCreatorManager + GGEMSBox / GGEMSTube /
 * GGEMSSphere, src/geometries/GGEMSVolumeCreatorManager.cc:229-294, kernels
 * src/kernels/DrawGGEMS{Box,Tube,Sphere}.cl), and an image read from an MHD
 * file is converted to material labels by a range table
 * (GGEMSVoxelizedSolid::ConvertImageToLabel,
 * include/GGEMS/geometries/GGEMSVoxelizedSolid.hh:162-257). */
typedef enum gg_met_type {
  GG_MET_CHAR = 0,
  GG_MET_UCHAR = 1,
  GG_MET_SHORT = 2,
  GG_MET_USHORT = 3,
  GG_MET_INT = 4,
  GG_MET_UINT = 5,
  GG_MET_FLOAT = 6
} gg_met_type;

typedef enum gg_shape_type { GG_SHAPE_BOX = 0, GG_SHAPE_TUBE = 1, GG_SHAPE_SPHERE = 2 } gg_shape_type;

typedef struct gg_shape {
  int32_t type;        /* gg_shape_type */
  float position[3];   /* centre, mm, relative to the volume's centre */
  float label_value;   /* written (converted to the element type) into covered voxels */
  float size[3];       /* box: width (x), height (y), depth (z); tube: radius_x, radius_y,
                          height (z); sphere: radius, -, -  (mm) */
} gg_shape;

typedef struct gg_volume gg_volume;
/* Zero-filled volume of dimensions[0]*dimensions[1]*dimensions[2] elements on
 * device device_index (GGEMSVolumeCreatorManager::Initialize). */
GG_API int gg_volume_create(int32_t device_index, int32_t met_type, const int32_t dimensions[3],
                            const float element_sizes[3], gg_volume** volume);
GG_API int gg_volume_destroy(gg_volume* volume);
/* Host <-> device copies of the whole image (bytes = elements * element size). */
GG_API int gg_volume_upload(gg_volume* volume, const void* host_image, uint64_t bytes);
GG_API int gg_volume_download(gg_volume* volume, void* host_image, uint64_t bytes);
/* Draws the shapes in order, one launch each (GGEMSBox::Draw etc.).  GGEMS's
 * voxel-index arithmetic is kept: its y index is (id mod dx*dx) / dx, so a
 * volume whose x and y dimensions differ is drawn exactly as GGEMS draws it. */
GG_API int gg_volume_draw(gg_volume* volume, const gg_shape* shapes, int32_t number_of_shapes);
/* Range table -> uint8 labels (host array of all elements): the label of a
 * voxel is the index of the LAST line whose range holds its value (value ==
 * first == last, or first <= value < last, compared in float); voxels that no
 * line holds keep 255 and are counted in *unconverted. */
GG_API int gg_volume_labels(gg_volume* volume, const float* range_first, const float* range_last,
                            int32_t number_of_ranges, uint8_t* labels, int64_t* unconverted);
/* Device time (CUDA events, ms) of the kernels of the last gg_volume_draw or
 * gg_volume_labels call, copies excluded. */
GG_API int gg_volume_last_kernel_ms(gg_volume* volume, float* milliseconds);

#ifdef __cplusplus
}
#endif

#endif /* GGEMS_B200_H */
