// Reference driver -- TEST INFRASTRUCTURE ONLY.
//
// Runs GGEMS's own device kernels (src/kernels/*.cl, compiled unmodified
// from the reference checkout through oracle/ref_shim/ocl_shim.hh) on the
// host, in the launch order of GGEMS::RunOnDevice (src/global/GGEMS.cc:303-363)
// and GGEMSNavigator::{ParticleSolidDistance, ProjectToSolid,
// TrackThroughSolid} (src/navigators/GGEMSNavigator.cc:320-530): every stage
// is a parallel loop over the batch's work-items, like an OpenCL NDRange.
//
// Exposes gg_ref_run() with the signature of gg_oracle_run(), so tests can
// pin the oracle restatement against the reference's own kernel code.  Built
// by oracle/build.py into oracle/_ref/ (never committed, never shipped).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "GGEMS/geometries/GGEMSMeshedSolidData.hh"
#include "GGEMS/geometries/GGEMSSolidBoxData.hh"
#include "GGEMS/geometries/GGEMSVoxelizedSolidData.hh"
#include "GGEMS/materials/GGEMSMaterialTables.hh"
#include "GGEMS/navigators/GGEMSDoseParams.hh"
#include "GGEMS/physics/GGEMSMuData.hh"
#include "GGEMS/physics/GGEMSParticleCrossSections.hh"
#include "GGEMS/physics/GGEMSPrimaryParticles.hh"
#include "GGEMS/randoms/GGEMSRandom.hh"
#include "ggems_b200.h"

thread_local size_t gg_shim_global_id = 0;

extern "C" {
void get_primaries_ggems_xray_source(ulong, GGEMSPrimaryParticles*, GGEMSRandom*, char, const float*, const float*, int,
                                     char, float, float3, const GGfloat44*);
void get_primaries_ggems_voxelized_source(ulong, GGEMSPrimaryParticles*, GGEMSRandom*, char, const float*, const float*,
                                          int, char, const int*, const float*, int, const GGEMSVoxelizedSolidData*,
                                          const GGfloat44*);
void particle_solid_distance_ggems_voxelized_solid(ulong, GGEMSPrimaryParticles*, const GGEMSVoxelizedSolidData*);
void particle_solid_distance_ggems_solid_box(ulong, GGEMSPrimaryParticles*, const GGEMSSolidBoxData*);
void project_to_ggems_voxelized_solid(ulong, GGEMSPrimaryParticles*, const GGEMSVoxelizedSolidData*);
void project_to_ggems_solid_box(ulong, GGEMSPrimaryParticles*, const GGEMSSolidBoxData*);
void track_through_ggems_voxelized_solid(ulong, GGEMSPrimaryParticles*, GGEMSRandom*, const GGEMSVoxelizedSolidData*,
                                         const uchar*, const GGEMSParticleCrossSections*, const GGEMSMaterialTables*,
                                         const GGEMSMuMuEnData*, float);
void track_through_ggems_voxelized_solid_dosimetry(ulong, GGEMSPrimaryParticles*, GGEMSRandom*,
                                                   const GGEMSVoxelizedSolidData*, const uchar*,
                                                   const GGEMSParticleCrossSections*, const GGEMSMaterialTables*,
                                                   const GGEMSMuMuEnData*, float, GGEMSDoseParams*, double*, double*,
                                                   int*, int*);
void track_through_ggems_voxelized_solid_tle(ulong, GGEMSPrimaryParticles*, GGEMSRandom*, const GGEMSVoxelizedSolidData*,
                                             const uchar*, const GGEMSParticleCrossSections*, const GGEMSMaterialTables*,
                                             const GGEMSMuMuEnData*, float, GGEMSDoseParams*, double*, double*, int*,
                                             int*);
void track_through_ggems_solid_box(ulong, GGEMSPrimaryParticles*, GGEMSRandom*, const GGEMSSolidBoxData*, const uchar*,
                                   const GGEMSParticleCrossSections*, const GGEMSMaterialTables*, const GGEMSMuMuEnData*,
                                   float, int*, int*);
void particle_solid_distance_ggems_meshed_solid(ulong, GGEMSPrimaryParticles*, const GGEMSMeshedSolidData*);
void project_to_ggems_meshed_solid(ulong, GGEMSPrimaryParticles*, const GGEMSMeshedSolidData*);
void track_through_ggems_meshed_solid(ulong, GGEMSPrimaryParticles*, GGEMSRandom*, const GGEMSMeshedSolidData*,
                                      const uchar*, const GGEMSParticleCrossSections*, const GGEMSMaterialTables*,
                                      const GGEMSMuMuEnData*, float);
void track_through_ggems_meshed_solid_dosimetry(ulong, GGEMSPrimaryParticles*, GGEMSRandom*,
                                                const GGEMSMeshedSolidData*, const uchar*,
                                                const GGEMSParticleCrossSections*, const GGEMSMaterialTables*,
                                                const GGEMSMuMuEnData*, float, GGEMSDoseParams*, double*, double*,
                                                int*, int*);
void is_alive(ulong, GGEMSPrimaryParticles*, int*);
void world_tracking(ulong, GGEMSPrimaryParticles*, int*, double*, double*, double*, double*, double*, ulong, ulong,
                    ulong, float, float, float);
void draw_ggems_box(ulong, float3, int3, float3, float, float, float, float, uchar*);
void draw_ggems_box_float(ulong, float3, int3, float3, float, float, float, float, float*);
void draw_ggems_tube(ulong, float3, int3, float3, float, float, float, float, uchar*);
void draw_ggems_tube_float(ulong, float3, int3, float3, float, float, float, float, float*);
void draw_ggems_sphere(ulong, float3, int3, float3, float, float, uchar*);
void draw_ggems_sphere_float(ulong, float3, int3, float3, float, float, float*);
}

namespace {

// One kernel launch of n work items on `threads` host threads, the way an
// OpenCL CPU runtime runs an NDRange: a pool of worker threads created once per
// process (not per launch) takes the items in chunks from a shared counter, so
// a core that is busy with something else delays only the chunks it holds.
class Pool {
 public:
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(m_);
      stop_ = true;
    }
    wake_.notify_all();
    for (auto& t : workers_) t.join();
  }
  void run(size_t n, int threads, const std::function<void(size_t, size_t)>& body) {
    {
      std::lock_guard<std::mutex> lk(m_);
      while (static_cast<int>(workers_.size()) < threads - 1) {
        const int index = static_cast<int>(workers_.size());
        workers_.emplace_back([this, index, seen = generation_]() { loop(index, seen); });
      }
      body_ = &body;
      n_ = n;
      chunk_ = std::max<size_t>(64, n / (static_cast<size_t>(threads) * 64));
      next_.store(0);
      helpers_ = threads - 1;
      running_ = static_cast<int>(workers_.size());
      ++generation_;
    }
    wake_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(m_);
    done_.wait(lk, [this]() { return running_ == 0; });
  }

 private:
  void work() {
    for (;;) {
      const size_t b = next_.fetch_add(chunk_);
      if (b >= n_) return;
      (*body_)(b, std::min(n_, b + chunk_));
    }
  }
  void loop(int index, uint64_t seen) {
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(m_);
        wake_.wait(lk, [&]() { return stop_ || generation_ != seen; });
        if (stop_) return;
        seen = generation_;
      }
      if (index < helpers_) work();
      std::lock_guard<std::mutex> lk(m_);
      if (--running_ == 0) done_.notify_one();
    }
  }
  std::mutex m_;
  std::condition_variable wake_, done_;
  std::vector<std::thread> workers_;
  const std::function<void(size_t, size_t)>* body_ = nullptr;
  size_t n_ = 0, chunk_ = 1;
  std::atomic<size_t> next_{0};
  uint64_t generation_ = 0;
  int helpers_ = 0, running_ = 0;
  bool stop_ = false;
};

Pool& pool() {
  static Pool p;
  return p;
}

template <class F>
void parallel_for(size_t n, int threads, F f) {
  if (threads <= 1 || n < 4096) {
    for (size_t i = 0; i < n; ++i) {
      gg_shim_global_id = i;
      f();
    }
    return;
  }
  const std::function<void(size_t, size_t)> body = [&f](size_t b, size_t e) {
    for (size_t i = b; i < e; ++i) {
      gg_shim_global_id = i;
      f();
    }
  };
  pool().run(n, threads, body);
}

void set_obb(GGEMSOBB& o, const gg_obb& g) {
  for (int j = 0; j < 4; ++j) {
    o.matrix_transformation_.m0_[j] = g.matrix[j];
    o.matrix_transformation_.m1_[j] = g.matrix[4 + j];
    o.matrix_transformation_.m2_[j] = g.matrix[8 + j];
    o.matrix_transformation_.m3_[j] = g.matrix[12 + j];
  }
  o.border_min_xyz_ = float3(g.border_min[0], g.border_min[1], g.border_min[2]);
  o.border_max_xyz_ = float3(g.border_max[0], g.border_max[1], g.border_max[2]);
}

void set_matrix(GGfloat44& m, const float* g) {
  for (int j = 0; j < 4; ++j) {
    m.m0_[j] = g[j];
    m.m1_[j] = g[4 + j];
    m.m2_[j] = g[8 + j];
    m.m3_[j] = g[12 + j];
  }
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int gg_ref_run(const gg_scene* scene, const gg_source* source,
                                                                 uint64_t number_of_particles, uint32_t* random_states,
                                                                 gg_particle_buffers* particles,
                                                                 gg_tally_buffers* tallies, int threads) {
  if (!scene || !source || !random_states) return GG_ERROR_INVALID_ARGUMENT;
  const size_t S = MAXIMUM_PARTICLES;

  std::unique_ptr<GGEMSPrimaryParticles> pp(new GGEMSPrimaryParticles());
  std::memset(pp.get(), 0, sizeof(GGEMSPrimaryParticles));
  std::unique_ptr<GGEMSRandom> rnd(new GGEMSRandom());
  std::memcpy(rnd->prng_state_1_, random_states, S * 4);
  std::memcpy(rnd->prng_state_2_, random_states + S, S * 4);
  std::memcpy(rnd->prng_state_3_, random_states + 2 * S, S * 4);
  std::memcpy(rnd->prng_state_4_, random_states + 3 * S, S * 4);
  std::memcpy(rnd->prng_state_5_, random_states + 4 * S, S * 4);
  for (size_t i = 0; i < S; ++i) pp->solid_id_[i] = -1;

  // Per-navigator tables in the reference's fixed-size layouts.
  std::vector<std::unique_ptr<GGEMSParticleCrossSections>> cs;
  std::vector<std::unique_ptr<GGEMSMaterialTables>> mt;
  for (int n = 0; n < scene->number_of_tables; ++n) {
    const gg_physics_tables& t = scene->tables[n];
    std::unique_ptr<GGEMSParticleCrossSections> c(new GGEMSParticleCrossSections());
    std::memset(c.get(), 0, sizeof(GGEMSParticleCrossSections));
    c->number_of_bins_ = t.number_of_bins;
    c->number_of_materials_ = t.number_of_materials;
    c->min_energy_ = t.energy_bins[0];
    c->max_energy_ = t.energy_bins[t.number_of_bins - 1];
    for (int i = 0; i < t.number_of_bins; ++i) c->energy_bins_[i] = t.energy_bins[i];
    const size_t block = static_cast<size_t>(t.number_of_materials) * t.number_of_bins;
    for (int p = 0; p < 3; ++p)
      std::memcpy(c->photon_cross_sections_[p], t.cross_sections + p * block, block * sizeof(float));
    if (t.rayleigh_per_atom)
      std::memcpy(c->photon_cross_sections_per_atom_[2], t.rayleigh_per_atom,
                  static_cast<size_t>(101) * t.number_of_bins * sizeof(float));
    c->number_of_activated_photon_processes_ = t.number_of_processes;
    for (int p = 0; p < t.number_of_processes; ++p) c->photon_cs_id_[p] = static_cast<char>(t.process_id[p]);
    cs.push_back(std::move(c));

    std::unique_ptr<GGEMSMaterialTables> m(new GGEMSMaterialTables());
    std::memset(m.get(), 0, sizeof(GGEMSMaterialTables));
    m->number_of_materials_ = t.number_of_materials;
    m->total_number_of_chemical_elements_ = t.total_elements;
    for (int i = 0; i < t.number_of_materials; ++i) {
      m->number_of_chemical_elements_[i] = t.number_of_elements[i];
      m->density_of_material_[i] = t.density[i];
      m->photon_energy_cut_[i] = t.photon_energy_cut[i];
      m->index_of_chemical_elements_[i] = t.element_offset[i];
    }
    for (int e = 0; e < t.total_elements; ++e) {
      m->atomic_number_Z_[e] = t.atomic_number[e];
      m->atomic_number_density_[e] = t.atomic_number_density[e];
    }
    mt.push_back(std::move(m));
  }
  std::unique_ptr<GGEMSMuMuEnData> att(new GGEMSMuMuEnData());
  std::memset(att.get(), 0, sizeof(GGEMSMuMuEnData));
  // Per-navigator GGEMSMuMuEnData for the TLE kernel (energy bins and mu_en).
  std::vector<std::unique_ptr<GGEMSMuMuEnData>> att_nav(scene->number_of_tables);
  for (int n = 0; n < scene->number_of_tables; ++n) {
    const gg_physics_tables& t = scene->tables[n];
    att_nav[n].reset(new GGEMSMuMuEnData());
    std::memset(att_nav[n].get(), 0, sizeof(GGEMSMuMuEnData));
    att_nav[n]->number_of_bins_ = GG_ATTENUATION_BINS;
    att_nav[n]->number_of_materials_ = t.number_of_materials;
    att_nav[n]->energy_min_ = 0.001f;
    att_nav[n]->energy_max_ = 1.0f;
    if (t.attenuation_energy_bins && t.mu_en) {
      std::memcpy(att_nav[n]->energy_bins_, t.attenuation_energy_bins, sizeof(float) * GG_ATTENUATION_BINS);
      std::memcpy(att_nav[n]->mu_en_, t.mu_en, sizeof(float) * GG_ATTENUATION_BINS * t.number_of_materials);
    }
  }

  // Per-solid data structures.
  const int ns = scene->number_of_solids;
  std::vector<GGEMSVoxelizedSolidData> vox(ns);
  std::vector<GGEMSSolidBoxData> box(ns);
  std::vector<GGEMSMeshedSolidData> mesh(ns);
  // Meshed solids: GGEMSNode array with triangle linked lists rebuilt from the
  // per-node index lists (same visiting order).
  std::vector<std::vector<GGEMSTriangle3>> mesh_triangles(ns);
  std::vector<std::vector<GGEMSNode>> mesh_nodes(ns);
  for (int s = 0; s < ns; ++s) {
    const gg_solid& g = scene->solids[s];
    if (g.type != GG_SOLID_MESHED) continue;
    std::vector<GGEMSTriangle3>& tri = mesh_triangles[s];
    tri.resize(g.number_of_triangles);
    for (int t = 0; t < g.number_of_triangles; ++t) {
      const float* f = g.triangles + static_cast<size_t>(t) * GG_TRIANGLE_FLOATS;
      for (int k = 0; k < 3; ++k) {
        tri[t].pts_[k].x_ = f[3 * k];
        tri[t].pts_[k].y_ = f[3 * k + 1];
        tri[t].pts_[k].z_ = f[3 * k + 2];
      }
      tri[t].bounding_sphere_.center_.x_ = f[9];
      tri[t].bounding_sphere_.center_.y_ = f[10];
      tri[t].bounding_sphere_.center_.z_ = f[11];
      tri[t].bounding_sphere_.radius_ = f[12];
      tri[t].next_triangle_ = nullptr;
    }
    std::vector<GGEMSNode>& nodes = mesh_nodes[s];
    nodes.resize(g.number_of_nodes);
    for (int n = 0; n < g.number_of_nodes; ++n) {
      GGEMSNode& nd = nodes[n];
      std::memset(&nd, 0, sizeof(nd));
      nd.center_.x_ = g.nodes[6 * n];
      nd.center_.y_ = g.nodes[6 * n + 1];
      nd.center_.z_ = g.nodes[6 * n + 2];
      for (int k = 0; k < 3; ++k) nd.half_width_[k] = g.nodes[6 * n + 3 + k];
      nd.triangle_list_ = nullptr;
      GGEMSTriangle3* prev = nullptr;
      for (int k = g.node_first[n]; k < g.node_first[n + 1]; ++k) {
        GGEMSTriangle3* t = &tri[g.node_triangles[k]];
        if (prev) prev->next_triangle_ = t;
        else nd.triangle_list_ = t;
        prev = t;
      }
    }
    set_obb(mesh[s].obb_geometry_, g.obb);
    mesh[s].solid_id_ = s;
    mesh[s].nodes_ = nodes.data();
    mesh[s].total_nodes_ = g.number_of_nodes;
  }
  for (int s = 0; s < ns; ++s) {
    const gg_solid& g = scene->solids[s];
    if (g.type == GG_SOLID_VOXELIZED) {
      set_obb(vox[s].obb_geometry_, g.obb);
      vox[s].voxel_sizes_xyz_ = float3(g.voxel_sizes[0], g.voxel_sizes[1], g.voxel_sizes[2]);
      vox[s].number_of_voxels_xyz_ = int3(g.number_of_voxels[0], g.number_of_voxels[1], g.number_of_voxels[2]);
      vox[s].solid_id_ = s;
      vox[s].number_of_voxels_ = g.number_of_voxels[0] * g.number_of_voxels[1] * g.number_of_voxels[2];
    } else if (g.type == GG_SOLID_BOX) {
      set_obb(box[s].obb_geometry_, g.obb);
      for (int k = 0; k < 3; ++k) {
        box[s].virtual_element_number_xyz_[k] = static_cast<GGsize>(g.virtual_element_number[k]);
        box[s].box_size_xyz_[k] = g.box_size[k];
      }
      box[s].solid_id_ = s;
    }
  }
  std::vector<GGEMSDoseParams> dose(scene->number_of_dose_maps);
  for (int d = 0; d < scene->number_of_dose_maps; ++d) {
    const gg_dose_map& g = scene->dose_maps[d];
    dose[d].size_of_dosels_ = float3(g.size_of_dosels[0], g.size_of_dosels[1], g.size_of_dosels[2]);
    dose[d].inv_size_of_dosels_ = float3(g.inv_size_of_dosels[0], g.inv_size_of_dosels[1], g.inv_size_of_dosels[2]);
    dose[d].border_min_xyz_ = float3(g.border_min[0], g.border_min[1], g.border_min[2]);
    dose[d].border_max_xyz_ = float3(g.border_max[0], g.border_max[1], g.border_max[2]);
    dose[d].number_of_dosels_ = int3(g.number_of_dosels[0], g.number_of_dosels[1], g.number_of_dosels[2]);
    dose[d].total_number_of_dosels_ = g.total_number_of_dosels;
    dose[d].slice_number_of_dosels_ = g.slice_number_of_dosels;
  }

  GGfloat44 source_matrix;
  set_matrix(source_matrix, source->matrix);
  GGEMSVoxelizedSolidData source_vox{};
  if (source->type == GG_SOURCE_VOXELIZED) {
    source_vox.number_of_voxels_xyz_ = int3(source->number_of_voxels[0], source->number_of_voxels[1], source->number_of_voxels[2]);
    source_vox.voxel_sizes_xyz_ = float3(source->voxel_sizes[0], source->voxel_sizes[1], source->voxel_sizes[2]);
    source_vox.obb_geometry_.border_min_xyz_ = float3(source->border_min[0], source->border_min[1], source->border_min[2]);
  }

  // Batches (GGEMSSource.cc:403-425, single device).
  const uint64_t nb = static_cast<uint64_t>(std::ceil(static_cast<float>(number_of_particles) / MAXIMUM_PARTICLES));
  std::vector<uint64_t> sizes(nb);
  if (nb == 1) {
    sizes[0] = number_of_particles;
  } else {
    for (uint64_t j = 0; j < nb; ++j) sizes[j] = number_of_particles / nb;
    for (uint64_t j = 0; j < number_of_particles % nb; ++j) sizes[j]++;
  }

  GGEMSPrimaryParticles* P = pp.get();
  GGEMSRandom* R = rnd.get();
  for (uint64_t b = 0; b < nb; ++b) {
    const ulong n = sizes[b];
    if (source->type == GG_SOURCE_XRAY) {
      float3 focal(source->focal_spot_size[0], source->focal_spot_size[1], source->focal_spot_size[2]);
      parallel_for(n, threads, [&]() {
        get_primaries_ggems_xray_source(n, P, R, static_cast<char>(source->particle_type), source->energy_spectrum,
                                        source->energy_cdf, source->number_of_energy_bins + 1,
                                        static_cast<char>(source->is_interp), source->beam_aperture, focal, &source_matrix);
      });
    } else {
      parallel_for(n, threads, [&]() {
        get_primaries_ggems_voxelized_source(n, P, R, static_cast<char>(source->particle_type), source->energy_spectrum,
                                             source->energy_cdf, source->number_of_energy_bins + 1,
                                             static_cast<char>(source->is_interp), source->activity_index,
                                             source->activity_cdf, static_cast<int>(source->number_of_activity_bins),
                                             &source_vox, &source_matrix);
      });
    }
    int loop_counter = 0;
    bool alive = true;
    do {
      for (int s = 0; s < ns; ++s) {
        if (scene->solids[s].type == GG_SOLID_VOXELIZED)
          parallel_for(n, threads, [&]() { particle_solid_distance_ggems_voxelized_solid(n, P, &vox[s]); });
        else if (scene->solids[s].type == GG_SOLID_MESHED)
          parallel_for(n, threads, [&]() { particle_solid_distance_ggems_meshed_solid(n, P, &mesh[s]); });
        else
          parallel_for(n, threads, [&]() { particle_solid_distance_ggems_solid_box(n, P, &box[s]); });
      }
      if (scene->world) {
        const gg_world& w = *scene->world;
        const gg_tally_buffers* o = tallies;
        int* wp = (o && w.photon_tracking) ? o->world_photon_tracking : nullptr;
        double* we = (o && w.energy_tracking) ? o->world_energy : nullptr;
        double* we2 = (o && w.energy_squared_tracking) ? o->world_energy_squared : nullptr;
        double* mx = (o && w.momentum) ? o->world_momentum_x : nullptr;
        double* my = (o && w.momentum) ? o->world_momentum_y : nullptr;
        double* mz = (o && w.momentum) ? o->world_momentum_z : nullptr;
        parallel_for(n, threads, [&]() {
          world_tracking(n, P, wp, we, we2, mx, my, mz, static_cast<ulong>(w.dimensions[0]),
                         static_cast<ulong>(w.dimensions[1]), static_cast<ulong>(w.dimensions[2]), w.sizes[0], w.sizes[1],
                         w.sizes[2]);
        });
      }
      for (int s = 0; s < ns; ++s) {
        if (scene->solids[s].type == GG_SOLID_VOXELIZED)
          parallel_for(n, threads, [&]() { project_to_ggems_voxelized_solid(n, P, &vox[s]); });
        else if (scene->solids[s].type == GG_SOLID_MESHED)
          parallel_for(n, threads, [&]() { project_to_ggems_meshed_solid(n, P, &mesh[s]); });
        else
          parallel_for(n, threads, [&]() { project_to_ggems_solid_box(n, P, &box[s]); });
      }
      for (int s = 0; s < ns; ++s) {
        const gg_solid& g = scene->solids[s];
        const GGEMSParticleCrossSections* C = cs[g.navigator].get();
        const GGEMSMaterialTables* M = mt[g.navigator].get();
        if (g.type == GG_SOLID_VOXELIZED) {
          if (g.dose_map >= 0) {
            const int d = g.dose_map;
            double* edep = tallies && tallies->edep ? tallies->edep[d] : nullptr;
            double* edep2 = tallies && tallies->edep_squared ? tallies->edep_squared[d] : nullptr;
            int* hit = tallies && tallies->hit ? tallies->hit[d] : nullptr;
            int* ptrack = tallies && tallies->photon_tracking ? tallies->photon_tracking[d] : nullptr;
            if (scene->dose_maps[d].tle) {
              const GGEMSMuMuEnData* A = att_nav[g.navigator].get();
              parallel_for(n, threads, [&]() {
                track_through_ggems_voxelized_solid_tle(n, P, R, &vox[s], g.labels, C, M, A, g.threshold, &dose[d],
                                                        edep, edep2, hit, ptrack);
              });
            } else {
              parallel_for(n, threads, [&]() {
                track_through_ggems_voxelized_solid_dosimetry(n, P, R, &vox[s], g.labels, C, M, att.get(),
                                                              g.threshold, &dose[d], edep, edep2, hit, ptrack);
              });
            }
          } else {
            parallel_for(n, threads, [&]() {
              track_through_ggems_voxelized_solid(n, P, R, &vox[s], g.labels, C, M, att.get(), g.threshold);
            });
          }
        } else if (g.type == GG_SOLID_MESHED) {
          if (g.dose_map >= 0) {
            const int d = g.dose_map;
            double* edep = tallies && tallies->edep ? tallies->edep[d] : nullptr;
            double* edep2 = tallies && tallies->edep_squared ? tallies->edep_squared[d] : nullptr;
            int* hit = tallies && tallies->hit ? tallies->hit[d] : nullptr;
            int* ptrack = tallies && tallies->photon_tracking ? tallies->photon_tracking[d] : nullptr;
            parallel_for(n, threads, [&]() {
              track_through_ggems_meshed_solid_dosimetry(n, P, R, &mesh[s], nullptr, C, M, att.get(), g.threshold,
                                                         &dose[d], edep, edep2, hit, ptrack);
            });
          } else {
            parallel_for(n, threads, [&]() {
              track_through_ggems_meshed_solid(n, P, R, &mesh[s], nullptr, C, M, att.get(), g.threshold);
            });
          }
        } else {
          int* h = (tallies && tallies->histograms && g.histogram >= 0) ? tallies->histograms[g.histogram] : nullptr;
          int* sh = (tallies && tallies->histograms && g.scatter_histogram >= 0) ? tallies->histograms[g.scatter_histogram]
                                                                                 : nullptr;
          std::vector<int> dummy;
          if (!h) {
            dummy.assign(static_cast<size_t>(g.virtual_element_number[0]) * g.virtual_element_number[1], 0);
            h = dummy.data();
          }
          parallel_for(n, threads, [&]() {
            track_through_ggems_solid_box(n, P, R, &box[s], nullptr, C, M, att.get(), g.threshold, h, sh);
          });
        }
      }
      ++loop_counter;
      int status = 0;
      for (ulong i = 0; i < n; ++i) {
        gg_shim_global_id = i;
        is_alive(n, P, &status);
      }
      alive = status != static_cast<int>(n);
    } while (alive && loop_counter < GG_MAX_LOOP);
  }

  std::memcpy(random_states, R->prng_state_1_, S * 4);
  std::memcpy(random_states + S, R->prng_state_2_, S * 4);
  std::memcpy(random_states + 2 * S, R->prng_state_3_, S * 4);
  std::memcpy(random_states + 3 * S, R->prng_state_4_, S * 4);
  std::memcpy(random_states + 4 * S, R->prng_state_5_, S * 4);
  if (particles && nb) {
    const uint64_t n = sizes[0];
    for (uint64_t i = 0; i < n; ++i) {
      particles->E[i] = P->E_[i];
      particles->px[i] = P->px_[i];
      particles->py[i] = P->py_[i];
      particles->pz[i] = P->pz_[i];
      particles->dx[i] = P->dx_[i];
      particles->dy[i] = P->dy_[i];
      particles->dz[i] = P->dz_[i];
      particles->status[i] = P->status_[i];
      particles->scatter[i] = P->scatter_[i];
      particles->solid_id[i] = P->solid_id_[i];
    }
  }
  return GG_OK;
}

// GGEMSBox / GGEMSTube / GGEMSSphere::Draw (src/geometries/GGEMSBox.cc, GGEMSTube.cc,
// GGEMSSphere.cc): the reference's draw kernel of the shape over every voxel,
// arguments in the order Draw sets them.  volume: MET_UCHAR or MET_FLOAT image.
extern "C" __attribute__((visibility("default"))) int gg_ref_draw(void* volume, int32_t met_type, const int32_t dim[3],
                                                                  const float es[3], const gg_shape* s) {
  if (met_type != GG_MET_UCHAR && met_type != GG_MET_FLOAT) return GG_ERROR_INVALID_ARGUMENT;
  const ulong n = static_cast<ulong>(dim[0]) * dim[1] * dim[2];
  const float3 sizes(es[0], es[1], es[2]);
  const int3 dims(dim[0], dim[1], dim[2]);
  const float3 pos(s->position[0], s->position[1], s->position[2]);
  const bool u8 = met_type == GG_MET_UCHAR;
  uchar* vu = static_cast<uchar*>(volume);
  float* vf = static_cast<float*>(volume);
  for (ulong i = 0; i < n; ++i) {
    gg_shim_global_id = i;
    if (s->type == GG_SHAPE_BOX) {
      // GGEMSBox::Draw: height_, width_, depth_
      if (u8) draw_ggems_box(n, sizes, dims, pos, s->label_value, s->size[1], s->size[0], s->size[2], vu);
      else draw_ggems_box_float(n, sizes, dims, pos, s->label_value, s->size[1], s->size[0], s->size[2], vf);
    } else if (s->type == GG_SHAPE_TUBE) {
      // GGEMSTube::Draw: height_, radius_x_, radius_y_
      if (u8) draw_ggems_tube(n, sizes, dims, pos, s->label_value, s->size[2], s->size[0], s->size[1], vu);
      else draw_ggems_tube_float(n, sizes, dims, pos, s->label_value, s->size[2], s->size[0], s->size[1], vf);
    } else {
      if (u8) draw_ggems_sphere(n, sizes, dims, pos, s->label_value, s->size[0], vu);
      else draw_ggems_sphere_float(n, sizes, dims, pos, s->label_value, s->size[0], vf);
    }
  }
  return GG_OK;
}
