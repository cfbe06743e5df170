// Device-side scene layout shared by the transport kernels and the runtime.
//
// HBM layout (one context = one GPU):
//   * random states: 5 SoA arrays of GG_MAXIMUM_PARTICLES uint32 (JKISS words);
//   * final particle states: SoA float/int8/int32 arrays per slot;
//   * table blob: per navigator, energy bins (float[nbins], 16 B padded),
//     cross sections packed as float4 {Compton, photoelectric, Rayleigh, 0}
//     per (material, bin), and photon energy cuts; copied into shared memory
//     at kernel start when it fits (cp.async.bulk + mbarrier);
//   * element tables and Rayleigh per-atom cross sections stay in HBM (read
//     only on Rayleigh interactions);
//   * labels: uint8 per voxel, x fastest (L2 resident for <= 126 MB volumes);
//   * tallies: int32 histograms, int64 fixed-point edep (LSB 2^-32 MeV),
//     double edep^2, int32 hit / photon-tracking counters.
#ifndef GG_INTERNAL_CUH
#define GG_INTERNAL_CUH

#include <cstdint>

#include <cuda_runtime.h>

#include "ggems_b200.h"

namespace gg {

constexpr int kMaxSolids = 64;
constexpr int kMaxNavigators = 16;
constexpr int kBlockThreads = 256;  // default transport block size (the autotuner tries 128 and 512 too)
// Fixed-point scale of the energy tally: edep is accumulated as int64 multiples of 2^-32 MeV.
constexpr double kEdepScale = 4294967296.0;

struct alignas(16) DevNavigator {
  // read by every tracking step: the first 16 bytes, one vector load
  int32_t number_of_bins;
  uint32_t process_pack;         // number_of_processes | process_id[0] << 8 | process_id[1] << 16 | process_id[2] << 24
  // byte offsets into the table blob (shared memory copy when it fits)
  uint32_t sigma_offset;         // float4[number_of_materials * number_of_bins]
  uint32_t photon_cut_offset;    // float[number_of_materials]
  int32_t number_of_materials;
  int32_t number_of_processes;
  int32_t process_id[3];
  uint32_t energy_bins_offset;   // float[number_of_bins]
  uint32_t attenuation_offset;   // float[GG_ATTENUATION_BINS] energies, then mu_en (TLE navigators only)
  // HBM arrays read on Rayleigh interactions
  const int32_t* number_of_elements;
  const int32_t* element_offset;
  const uint8_t* atomic_number;
  const float* atomic_number_density;
  const float* rayleigh_per_atom;
};

struct DevDoseMap {
  float size_of_dosels[3];
  float inv_size_of_dosels[3];
  float border_min[3];
  float border_max[3];
  int32_t number_of_dosels[3];
  int32_t total_number_of_dosels;
  int32_t slice_number_of_dosels;
  unsigned long long* edep;      // fixed point, LSB 2^-32 MeV
  double* edep_squared;          // nullptr when not recorded
  int32_t* hit;                  // nullptr when not recorded
  int32_t* photon_tracking;      // nullptr when not recorded
};

struct alignas(16) DevSolid {
  // read by every tracking step: the first 80 bytes, five vector loads
  float border_min[3];
  float border_max[3];
  float voxel_sizes[3];
  float inv_voxel_sizes[3];      // exact 2^-k when voxel_pow2
  int32_t number_of_voxels[3];
  int32_t navigator;
  const uint8_t* labels;
  int32_t type;
  int32_t voxel_pow2;            // every voxel size is a power of two
  float matrix[16];
  float threshold;
  int32_t virtual_element_number[3];
  float box_size[3];
  int32_t* histogram;            // nullptr when none
  int32_t* scatter_histogram;    // nullptr when none
  int32_t dose_map;              // -1 when none
  int32_t dose_tle;              // the dose map uses the track-length estimator
  // meshed solid: octree nodes that own triangles, in node order, 2 float4
  // each ({min xyz, max x}, {max y, max z, first, count} with first / count as
  // int bits), and triangles grouped by node, 3 float4 each
  // ({p0 xyz, e1 x}, {e1 yz, e2 xy}, {e2 z, -, -, -}) with e1 = p1 - p0, e2 = p2 - p0.
  // With mesh_bvh set, mesh_nodes is instead a bounding-volume hierarchy in
  // the same 2-float4 form: count > 0 marks a leaf owning triangles
  // [first, first + count), count == 0 an inner node whose children are
  // first and first + 1.
  const float4* mesh_nodes;
  int32_t mesh_node_count;
  const float4* mesh_triangles;
  int32_t mesh_bvh;
};

struct DevSource {
  int32_t type;
  float matrix[16];
  float beam_aperture;
  double new_aperture;             // 1 - cos(aperture), computed on the host in double
  float focal_spot_size[3];
  int32_t number_of_energy_bins;   // n + 1, as passed to the reference kernel
  const float* energy_spectrum;
  const float* energy_cdf;
  int32_t is_interp;
  int32_t number_of_voxels[3];
  float voxel_sizes[3];
  float border_min[3];
  int32_t number_of_activity_bins;
  const int32_t* activity_index;
  const float* activity_cdf;
};

struct DevParticles {
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
};

// One source run of a (possibly batched) launch.  Batch plan of
// GGEMSSource::OrganizeParticlesInBatch: sizes are q+1 for the first r
// batches and q for the others, nb batches; slot i takes part when i < slots.
struct DevJob {
  DevSource source;
  uint64_t q;
  uint64_t r;
  uint32_t nb;
  uint32_t slots;
};

struct TransportParams {
  const DevJob* jobs;           // number_of_jobs runs, done in order by every slot
  int32_t number_of_jobs;
  const DevSolid* job_solids;   // [number_of_jobs][number_of_solids] when number_of_jobs > 1, else NULL
  uint32_t number_of_slots;     // slots touched (largest first batch over the jobs)
  uint32_t* rng;                // 5 * GG_MAXIMUM_PARTICLES words
  DevParticles particles;
  const DevSolid* solids;
  int32_t number_of_solids;
  const DevNavigator* navigators;
  int32_t number_of_navigators;
  const DevDoseMap* dose_maps;
  const unsigned char* table_blob;  // HBM copy of the shared-memory tables
  uint32_t table_bytes;             // multiple of 16
  int32_t tables_in_smem;
  unsigned int* slot_counter;       // work queue head
  int* error;                       // 0 = ok
  // world tracking (GGEMSWorld): grid, tallies (NULL when not recorded);
  // energy and momentum as int64 fixed point (LSB 2^-32), E^2 in FP64
  int32_t world_dimensions[3];
  float world_sizes[3];
  int32_t* world_photon;
  unsigned long long* world_energy;
  double* world_energy_squared;
  unsigned long long* world_momentum;  // [3][cells]
  // particle tracking: the points of slot tracking_slot (-1: off), kFull variant only
  int32_t tracking_slot;
  int32_t tracking_capacity;
  gg_track_point* tracking_points;
  int32_t* tracking_count;
  int32_t regroup_lanes;            // waiting lanes that start a round of the rare phases (1..32)
  int32_t regroup_ratio4;           // ... or 4 x waiting >= regroup_ratio4 x tracking lanes
  uint32_t slots_per_claim;         // consecutive slots a lane takes from the work queue at a time (power of two)
  int32_t stash_swap_lanes;         // stash variant: waiting lanes that start an exchange with ready photons (1..32)
  int32_t stash_round_photons;      // stash variant: waiting photons (lanes + records) that start a rare round
};

// Photon stash of the stash variant: per warp, kStashRecords photon records in
// shared memory, one 32-bit word per field and record (field-major), and a
// 32-entry index table.
constexpr int kStashRecords = 32;
__host__ __device__ constexpr int stash_words(bool batch, bool aux) { return 25 + (batch ? 1 : 0) + (aux ? 1 : 0); }
constexpr size_t stash_bytes_per_warp(bool batch, bool aux) {
  return sizeof(uint32_t) * (static_cast<size_t>(stash_words(batch, aux)) * kStashRecords + kStashRecords);
}

struct DoseParams {
  DevDoseMap map;
  int32_t number_of_voxels[3];
  float voxel_sizes[3];
  float border_min[3];
  const uint8_t* labels;
  const float* density;     // per material
  float scale_factor;
  int32_t is_water_reference;
  float minimum_density;
  float* dose;
  float* uncertainty;
};

void launch_transport(const TransportParams& p, int grid, int threads, size_t smem, void* stream, bool mesh, bool dose,
                      bool aux, int stash);
cudaError_t configure_transport(size_t smem, int threads, int* blocks_per_sm, bool mesh, bool batch, bool dose, bool aux,
                                int stash);
cudaError_t set_rayleigh_fit(const float* pp);
void launch_compute_dose(const DoseParams& p, void* stream);

// Line integrals of mu through a voxelized solid, one ray per detector element
// (source point -> element centre), for the scatter surrogate's inputs.
struct ProjectorParams {
  float phantom_matrix[16];
  float border_min[3], border_max[3];
  int32_t number_of_voxels[3];
  float voxel_sizes[3];
  const uint8_t* labels;
  const float* mu;               // per material, mm^-1
  int32_t number_of_materials;
  float detector_matrix[16];
  float detector_min[3];
  float element_size[3];
  int32_t elements[2];
  float source[3];               // world
  float* out;                    // [elements[1]][elements[0]], or [..][..][2] with network_input
  int32_t network_input;         // 1: write (exp(-L), L) pairs, the surrogate network's input
};
void launch_line_integrals(const ProjectorParams& p, void* stream);

// Records msg as the text of gg_last_error() for this thread; returns code.
int record_error(int code, const char* msg);

}  // namespace gg

#endif
