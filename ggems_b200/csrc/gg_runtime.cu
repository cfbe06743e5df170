// C-ABI runtime of the B200 transport layer (include/ggems_b200.h).
//
// Owns one GPU context: random states, final particle states, the uploaded
// scene (tables, labels, tallies) and the launch of the transport kernel.
// Replaces GGEMSOpenCLManager's Allocate / GetDeviceBuffer / CleanBuffer /
// enqueueNDRangeKernel plumbing (src/global/GGEMSOpenCLManager.cc:836-1046)
// for the photon path.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "gg_internal.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define GG_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t e_ = (call);                                                                       \
    if (e_ != cudaSuccess)                                                                         \
      return fail(e_ == cudaErrorMemoryAllocation ? GG_ERROR_OUT_OF_MEMORY : GG_ERROR_CUDA,        \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                              \
  } while (0)

template <class T>
struct DevArray {
  T* ptr = nullptr;
  size_t n = 0;
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    n = 0;
  }
};

}  // namespace

int gg::record_error(int code, const char* msg) { return fail(code, msg); }

struct gg_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  int sm_count = 0;
  // warp scheduling of the transport kernel (GGEMS_B200_REGROUP_LANES / _RATIO4)
  int regroup_lanes = 32;
  int regroup_ratio4 = 4;
  int blocks_per_sm = 0;  // 0: as many as fit (the autotuner may lower it)
  int block_threads = gg::kBlockThreads;  // transport block size: 128, 256 or 512
  int slots_per_claim = 1;                // photons per thread: slots a lane takes per work-queue grab
  int stash_registers = 80;               // photon stash variant (voxel / detector scenes): 0 off, 64 or 80 registers
  int stash_swap_lanes = 4;               // waiting lanes that start an exchange with the stash
  int stash_round_photons = 40;           // waiting photons of a warp (lanes + records) that start a rare round
  size_t smem_optin = 0;
  uint32_t* rng = nullptr;
  gg::DevParticles particles{};
  std::vector<void*> scene_allocations;  // freed on re-upload / destroy
  // Re-uploads reuse the previous scene's buffers of the same sizes (no
  // cudaFree / cudaMalloc per upload when only the contents change).
  std::map<void*, size_t> scene_bytes;
  std::vector<std::pair<void*, size_t>> scene_spares;
  std::vector<void*> run_allocations;    // source arrays of the last run
  // gg_compute_dose's device outputs, grown on demand and kept: a cudaFree per
  // call would synchronise the whole device
  float* dose_out = nullptr;
  size_t dose_out_floats = 0;
  gg::DevSolid* solids = nullptr;
  int number_of_solids = 0;
  gg::DevNavigator* navigators = nullptr;
  int number_of_navigators = 0;
  gg::DevDoseMap* dose_maps = nullptr;
  std::vector<gg::DevDoseMap> dose_host;
  std::vector<int32_t*> histograms;
  std::vector<int32_t> histogram_sizes;
  std::vector<gg_solid> solid_host;       // host copy (labels pointers replaced by device pointers)
  std::vector<gg::DevSolid> solid_dev_host;  // host copy of the uploaded device solids
  std::vector<char> dose_tle;             // per dose map: track-length estimator
  std::vector<const float*> density_dev;  // per navigator, for dose finalisation
  // particle tracking: slot (-1 off) and its point buffer
  int tracking_slot = -1;
  int tracking_capacity = 0;
  gg_track_point* tracking_points = nullptr;
  int32_t* tracking_count = nullptr;
  // world tracking grid and its device tallies (NULL when not recorded)
  int32_t world_dimensions[3] = {0, 0, 0};
  float world_sizes[3] = {0.0f, 0.0f, 0.0f};
  size_t world_cells = 0;
  int32_t* world_photon = nullptr;
  unsigned long long* world_energy = nullptr;
  double* world_energy_squared = nullptr;
  unsigned long long* world_momentum = nullptr;
  unsigned char* table_blob = nullptr;
  uint32_t table_bytes = 0;
  bool tables_in_smem = false;
  unsigned int* slot_counter = nullptr;
  int* error = nullptr;
  cudaEvent_t start = nullptr, stop = nullptr;
  float last_ms = 0.0f;
  int64_t last_launches = 0;
  bool scene_ready = false;
};

namespace {

template <class T>
int dev_copy_to(gg_context* c, std::vector<void*>& owner, const T* host, size_t n, T** out) {
  *out = nullptr;
  if (n == 0) return GG_OK;
  void* p = nullptr;
  const size_t bytes = n * sizeof(T);
  const bool scene = &owner == &c->scene_allocations;
  if (scene) {
    for (size_t i = 0; i < c->scene_spares.size(); ++i)
      if (c->scene_spares[i].second == bytes) {
        p = c->scene_spares[i].first;
        c->scene_spares.erase(c->scene_spares.begin() + static_cast<std::ptrdiff_t>(i));
        break;
      }
  }
  if (!p) GG_CUDA(cudaMalloc(&p, bytes));
  if (scene) c->scene_bytes[p] = bytes;
  owner.push_back(p);
  if (host) GG_CUDA(cudaMemcpyAsync(p, host, n * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  else GG_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), c->stream));
  *out = static_cast<T*>(p);
  return GG_OK;
}

template <class T>
int dev_copy(gg_context* c, const T* host, size_t n, T** out) {
  return dev_copy_to(c, c->scene_allocations, host, n, out);
}

// keep_buffers: the scene's device buffers become spares for the next upload
// (release_spares() frees what that upload did not reuse).
void release_spares(gg_context* c) {
  for (auto& sp : c->scene_spares) {
    c->scene_bytes.erase(sp.first);
    cudaFree(sp.first);
  }
  c->scene_spares.clear();
}
void free_scene(gg_context* c, bool keep_buffers = false) {
  for (void* p : c->scene_allocations) {
    if (keep_buffers) c->scene_spares.emplace_back(p, c->scene_bytes[p]);
    else {
      c->scene_bytes.erase(p);
      cudaFree(p);
    }
  }
  if (!keep_buffers) release_spares(c);
  c->scene_allocations.clear();
  c->solids = nullptr;
  c->navigators = nullptr;
  c->dose_maps = nullptr;
  c->table_blob = nullptr;
  c->dose_host.clear();
  c->histograms.clear();
  c->histogram_sizes.clear();
  c->solid_host.clear();
  c->solid_dev_host.clear();
  c->dose_tle.clear();
  c->density_dev.clear();
  for (int a = 0; a < 3; ++a) c->world_dimensions[a] = 0;
  c->world_cells = 0;
  c->world_photon = nullptr;
  c->world_energy = nullptr;
  c->world_energy_squared = nullptr;
  c->world_momentum = nullptr;
  c->scene_ready = false;
}

void free_run(gg_context* c) {
  for (void* p : c->run_allocations) cudaFree(p);
  c->run_allocations.clear();
}

uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }

float4 triangle_record(const float* v, int part) {
  const float e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
  const float e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
  if (part == 0) return make_float4(v[0], v[1], v[2], e1[0]);
  if (part == 1) return make_float4(e1[1], e1[2], e2[0], e2[1]);
  return make_float4(e2[2], 0.0f, 0.0f, 0.0f);
}

float int_bits(int x) {
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}

// Bounding-volume hierarchy over the mesh triangles: binned surface-area
// heuristic (12 bins on the widest centroid axis), leaves of at most 4
// triangles, depth at most 48 (the device walk keeps a 64-entry stack).
// Boxes are grown by a relative 1e-5 plus 1e-4 mm so that rounding in the
// slab test never prunes a triangle the ray actually crosses.
void build_bvh(const gg_solid& g, std::vector<float4>* nodes_out, std::vector<float4>* tris_out) {
  const int n = g.number_of_triangles;
  std::vector<float> lo(3 * n), hi(3 * n), cen(3 * n);
  for (int t = 0; t < n; ++t) {
    const float* v = g.triangles + static_cast<size_t>(t) * GG_TRIANGLE_FLOATS;
    for (int a = 0; a < 3; ++a) {
      lo[3 * t + a] = std::min(v[a], std::min(v[3 + a], v[6 + a]));
      hi[3 * t + a] = std::max(v[a], std::max(v[3 + a], v[6 + a]));
      cen[3 * t + a] = 0.5f * (lo[3 * t + a] + hi[3 * t + a]);
    }
  }
  std::vector<int> order(n);
  for (int t = 0; t < n; ++t) order[t] = t;
  struct Item {
    int node, begin, end, depth;
  };
  std::vector<float4>& nodes = *nodes_out;
  nodes.assign(2, make_float4(0, 0, 0, 0));
  std::vector<Item> work{{0, 0, n, 0}};
  auto area = [](const float* b) {
    const float x = b[3] - b[0], y = b[4] - b[1], z = b[5] - b[2];
    return x < 0 ? 0.0f : 2.0f * (x * y + y * z + z * x);
  };
  while (!work.empty()) {
    const Item it = work.back();
    work.pop_back();
    float box[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    float cb[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = it.begin; i < it.end; ++i) {
      const int t = order[i];
      for (int a = 0; a < 3; ++a) {
        box[a] = std::min(box[a], lo[3 * t + a]);
        box[3 + a] = std::max(box[3 + a], hi[3 * t + a]);
        cb[a] = std::min(cb[a], cen[3 * t + a]);
        cb[3 + a] = std::max(cb[3 + a], cen[3 * t + a]);
      }
    }
    for (int a = 0; a < 3; ++a) {
      const float pad = 1.0e-4f + 1.0e-5f * std::max(std::fabs(box[a]), std::fabs(box[3 + a]));
      box[a] -= pad;
      box[3 + a] += pad;
    }
    const int count = it.end - it.begin;
    int split = -1;
    if (count > 4 && it.depth < 47) {
      int axis = 0;
      for (int a = 1; a < 3; ++a)
        if (cb[3 + a] - cb[a] > cb[3 + axis] - cb[axis]) axis = a;
      const float extent = cb[3 + axis] - cb[axis];
      if (extent > 0.0f) {
        constexpr int kBins = 12;
        int bin_count[kBins] = {0};
        float bin_box[kBins][6];
        for (auto& b : bin_box) {
          b[0] = b[1] = b[2] = FLT_MAX;
          b[3] = b[4] = b[5] = -FLT_MAX;
        }
        auto bin_of = [&](int t) {
          int k = static_cast<int>(kBins * (cen[3 * t + axis] - cb[axis]) / extent);
          return k < 0 ? 0 : (k >= kBins ? kBins - 1 : k);
        };
        for (int i = it.begin; i < it.end; ++i) {
          const int t = order[i], k = bin_of(t);
          ++bin_count[k];
          for (int a = 0; a < 3; ++a) {
            bin_box[k][a] = std::min(bin_box[k][a], lo[3 * t + a]);
            bin_box[k][3 + a] = std::max(bin_box[k][3 + a], hi[3 * t + a]);
          }
        }
        float best = FLT_MAX;
        int best_k = -1;
        for (int k = 1; k < kBins; ++k) {
          float l[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX}, r[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
          int nl = 0, nr = 0;
          for (int j = 0; j < kBins; ++j) {
            float* dst = j < k ? l : r;
            (j < k ? nl : nr) += bin_count[j];
            for (int a = 0; a < 3; ++a) {
              dst[a] = std::min(dst[a], bin_box[j][a]);
              dst[3 + a] = std::max(dst[3 + a], bin_box[j][3 + a]);
            }
          }
          if (nl == 0 || nr == 0) continue;
          const float cost = area(l) * nl + area(r) * nr;
          if (cost < best) {
            best = cost;
            best_k = k;
          }
        }
        if (best_k > 0) {
          auto mid = std::partition(order.begin() + it.begin, order.begin() + it.end,
                                    [&](int t) { return bin_of(t) < best_k; });
          split = static_cast<int>(mid - order.begin());
        }
      }
      if (split <= it.begin || split >= it.end) split = it.begin + count / 2;  // degenerate: median
    }
    if (split < 0) {
      nodes[2 * it.node] = make_float4(box[0], box[1], box[2], box[3]);
      nodes[2 * it.node + 1] = make_float4(box[4], box[5], int_bits(it.begin), int_bits(count));
    } else {
      const int left = static_cast<int>(nodes.size() / 2);
      nodes.resize(nodes.size() + 4, make_float4(0, 0, 0, 0));
      nodes[2 * it.node] = make_float4(box[0], box[1], box[2], box[3]);
      nodes[2 * it.node + 1] = make_float4(box[4], box[5], int_bits(left), int_bits(0));
      work.push_back({left, it.begin, split, it.depth + 1});
      work.push_back({left + 1, split, it.end, it.depth + 1});
    }
  }
  tris_out->clear();
  for (int i = 0; i < n; ++i)
    for (int part = 0; part < 3; ++part)
      tris_out->push_back(triangle_record(g.triangles + static_cast<size_t>(order[i]) * GG_TRIANGLE_FLOATS, part));
}

// Whether meshed solids use the hierarchy: GGEMS_B200_MESH_BVH = 0 (never:
// GGEMS's octree scan), 1 (always), unset (meshes above 4096 triangles).
bool use_bvh(int triangles) {
  if (const char* v = std::getenv("GGEMS_B200_MESH_BVH")) return std::atoi(v) != 0;
  return triangles > 4096;
}

// Meshed solid.  Octree form: keep the octree nodes that own triangles (GGEMS
// skips the others), with their boxes as the reference's TestLineNode computes
// them, and the triangles regrouped by node with their two edges precomputed
// (the same float subtractions the Moller-Trumbore test makes).  BVH form for
// large meshes (build_bvh).
int upload_mesh(gg_context* c, const gg_solid& g, gg::DevSolid* d, std::vector<void*>& owner) {
  if (g.number_of_triangles < 1 || !g.triangles || g.number_of_nodes < 1 || !g.nodes || !g.node_first ||
      !g.node_triangles)
    return fail(GG_ERROR_INVALID_ARGUMENT, "meshed solid without triangles or octree");
  std::vector<float4> nodes, tris;
  d->mesh_bvh = use_bvh(g.number_of_triangles) ? 1 : 0;
  if (d->mesh_bvh) {
    build_bvh(g, &nodes, &tris);
    float4* dn;
    float4* dt;
    int rc;
    if ((rc = dev_copy_to(c, owner, nodes.data(), nodes.size(), &dn)) ||
        (rc = dev_copy_to(c, owner, tris.data(), tris.size(), &dt)))
      return rc;
    d->mesh_nodes = dn;
    d->mesh_node_count = static_cast<int32_t>(nodes.size() / 2);
    d->mesh_triangles = dt;
    return GG_OK;
  }
  for (int n = 0; n < g.number_of_nodes; ++n) {
    const int b = g.node_first[n], e = g.node_first[n + 1];
    if (b < 0 || e < b || e > g.number_of_triangles) return fail(GG_ERROR_INVALID_ARGUMENT, "bad octree node list");
    if (b == e) continue;
    const float* nd = g.nodes + 6 * n;
    float mn[3], mx[3];
    for (int a = 0; a < 3; ++a) {
      mn[a] = nd[a] - nd[3 + a];
      mx[a] = nd[a] + nd[3 + a];
    }
    const int first = static_cast<int>(tris.size() / 3), count = e - b;
    float f, k;
    std::memcpy(&f, &first, 4);
    std::memcpy(&k, &count, 4);
    nodes.push_back(make_float4(mn[0], mn[1], mn[2], mx[0]));
    nodes.push_back(make_float4(mx[1], mx[2], f, k));
    for (int i = b; i < e; ++i) {
      const int t = g.node_triangles[i];
      if (t < 0 || t >= g.number_of_triangles) return fail(GG_ERROR_INVALID_ARGUMENT, "bad triangle index");
      const float* v = g.triangles + static_cast<size_t>(t) * GG_TRIANGLE_FLOATS;
      const float e1[3] = {v[3] - v[0], v[4] - v[1], v[5] - v[2]};
      const float e2[3] = {v[6] - v[0], v[7] - v[1], v[8] - v[2]};
      tris.push_back(make_float4(v[0], v[1], v[2], e1[0]));
      tris.push_back(make_float4(e1[1], e1[2], e2[0], e2[1]));
      tris.push_back(make_float4(e2[2], 0.0f, 0.0f, 0.0f));
    }
  }
  float4* dn;
  float4* dt;
  int rc;
  if ((rc = dev_copy_to(c, owner, nodes.data(), nodes.size(), &dn)) ||
      (rc = dev_copy_to(c, owner, tris.data(), tris.size(), &dt)))
    return rc;
  d->mesh_nodes = dn;
  d->mesh_node_count = static_cast<int32_t>(nodes.size() / 2);
  d->mesh_triangles = dt;
  return GG_OK;
}


// Device form of one solid; labels and mesh arrays are uploaded into `owner`
// (once per host array when `labels_seen` is given).
int make_dev_solid(gg_context* c, const gg_solid& g, gg::DevSolid* out, std::vector<void*>& owner,
                   std::map<const void*, const void*>* labels_seen) {
  gg::DevSolid& d = *out;
  d = gg::DevSolid{};
  int rc;
  if (g.navigator < 0 || g.navigator >= c->number_of_navigators)
    return fail(GG_ERROR_INVALID_ARGUMENT, "solid navigator out of range");
  d.type = g.type;
  d.navigator = g.navigator;
  std::memcpy(d.matrix, g.obb.matrix, sizeof(d.matrix));
  std::memcpy(d.border_min, g.obb.border_min, sizeof(d.border_min));
  std::memcpy(d.border_max, g.obb.border_max, sizeof(d.border_max));
  d.threshold = g.threshold;
  std::memcpy(d.number_of_voxels, g.number_of_voxels, sizeof(d.number_of_voxels));
  std::memcpy(d.voxel_sizes, g.voxel_sizes, sizeof(d.voxel_sizes));
  // x / 2^k and x * 2^-k are the same correctly rounded value for every x,
  // so power-of-two voxel sizes let the kernel multiply instead of divide.
  d.voxel_pow2 = 1;
  for (int a = 0; a < 3; ++a) {
    int e = 0;
    const float m = std::frexp(g.voxel_sizes[a], &e);  // v = m * 2^e, m in [0.5, 1)
    const bool pow2 = std::isfinite(g.voxel_sizes[a]) && m == 0.5f && e > -125 && e < 127;
    d.voxel_pow2 &= pow2 ? 1 : 0;
    d.inv_voxel_sizes[a] = pow2 ? std::ldexp(1.0f, 1 - e) : 0.0f;
  }
  std::memcpy(d.virtual_element_number, g.virtual_element_number, sizeof(d.virtual_element_number));
  std::memcpy(d.box_size, g.box_size, sizeof(d.box_size));
  const int nh = static_cast<int>(c->histograms.size()), nd = static_cast<int>(c->dose_host.size());
  d.histogram = (g.histogram >= 0 && g.histogram < nh) ? c->histograms[g.histogram] : nullptr;
  d.scatter_histogram = (g.scatter_histogram >= 0 && g.scatter_histogram < nh) ? c->histograms[g.scatter_histogram] : nullptr;
  d.dose_map = (g.dose_map >= 0 && g.dose_map < nd) ? g.dose_map : -1;
  d.dose_tle = (d.dose_map >= 0 && g.type == GG_SOLID_VOXELIZED && c->dose_tle[d.dose_map]) ? 1 : 0;
  d.labels = nullptr;
  if (g.type == GG_SOLID_VOXELIZED) {
    const size_t nv = static_cast<size_t>(g.number_of_voxels[0]) * g.number_of_voxels[1] * g.number_of_voxels[2];
    if (!g.labels || nv == 0) return fail(GG_ERROR_INVALID_ARGUMENT, "voxelized solid without labels");
    const void* known = nullptr;
    if (labels_seen) {
      auto it = labels_seen->find(g.labels);
      if (it != labels_seen->end()) known = it->second;
    }
    if (known) {
      d.labels = static_cast<const uint8_t*>(known);
    } else {
      uint8_t* lab;
      if ((rc = dev_copy_to(c, owner, g.labels, nv, &lab))) return rc;
      d.labels = lab;
      if (labels_seen) (*labels_seen)[g.labels] = lab;
    }
  } else if (g.type == GG_SOLID_MESHED) {
    if ((rc = upload_mesh(c, g, &d, owner))) return rc;
  } else if (g.type != GG_SOLID_BOX) {
    return fail(GG_ERROR_INVALID_ARGUMENT, "solid type not supported by this build");
  }
  return GG_OK;
}
}  // namespace

extern "C" {

GG_API const char* gg_last_error(void) { return g_last_error.c_str(); }

GG_API int gg_device_count(int32_t* count) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    *count = 0;
    return fail(GG_ERROR_NO_DEVICE, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  }
  *count = n;
  return GG_OK;
}

GG_API int gg_context_create(int32_t device_index, gg_context** context) {
  if (!context) return fail(GG_ERROR_INVALID_ARGUMENT, "context pointer is NULL");
  *context = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return fail(GG_ERROR_NO_DEVICE, "no CUDA device");
  if (device_index < 0 || device_index >= n) return fail(GG_ERROR_INVALID_ARGUMENT, "device index out of range");
  GG_CUDA(cudaSetDevice(device_index));
  cudaDeviceProp prop;
  GG_CUDA(cudaGetDeviceProperties(&prop, device_index));
  if (prop.major < 10) return fail(GG_ERROR_NO_DEVICE, std::string("device is not sm_100 class: ") + prop.name);
  gg_context* c = new gg_context();
  c->device = device_index;
  c->sm_count = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  if (const char* v = std::getenv("GGEMS_B200_REGROUP_LANES")) {
    int r = std::atoi(v);
    if (r >= 1 && r <= 32) c->regroup_lanes = r;
  }
  if (const char* v = std::getenv("GGEMS_B200_REGROUP_RATIO4")) {
    int r = std::atoi(v);
    if (r >= 0 && r <= 128) c->regroup_ratio4 = r;
  }
  if (const char* v = std::getenv("GGEMS_B200_STASH_ROUND")) {
    int r = std::atoi(v);
    if (r >= 1 && r <= 2 * gg::kStashRecords) c->stash_round_photons = r;
  }
  if (const char* v = std::getenv("GGEMS_B200_STASH_REGISTERS")) {
    int r = std::atoi(v);
    if (r == 0 || r == 64 || r == 80) c->stash_registers = r;
  }
  if (const char* v = std::getenv("GGEMS_B200_STASH_SWAP")) {
    int r = std::atoi(v);
    if (r >= 1 && r <= 32) c->stash_swap_lanes = r;
  }
  const size_t S = GG_MAXIMUM_PARTICLES;
  auto cleanup = [&](int code) {
    gg_context_destroy(c);
    return code;
  };
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return cleanup(fail(GG_ERROR_CUDA, "stream"));
  if (cudaMalloc(&c->rng, 5 * S * sizeof(uint32_t)) != cudaSuccess) return cleanup(fail(GG_ERROR_OUT_OF_MEMORY, "rng"));
  cudaMemset(c->rng, 0, 5 * S * sizeof(uint32_t));
  float** fp[7] = {&c->particles.E, &c->particles.px, &c->particles.py, &c->particles.pz,
                   &c->particles.dx, &c->particles.dy, &c->particles.dz};
  for (auto f : fp)
    if (cudaMalloc(reinterpret_cast<void**>(f), S * sizeof(float)) != cudaSuccess)
      return cleanup(fail(GG_ERROR_OUT_OF_MEMORY, "particles"));
  if (cudaMalloc(&c->particles.status, S) != cudaSuccess || cudaMalloc(&c->particles.scatter, S) != cudaSuccess ||
      cudaMalloc(&c->particles.solid_id, S * sizeof(int32_t)) != cudaSuccess)
    return cleanup(fail(GG_ERROR_OUT_OF_MEMORY, "particles"));
  if (cudaMalloc(&c->slot_counter, sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&c->error, sizeof(int)) != cudaSuccess)
    return cleanup(fail(GG_ERROR_OUT_OF_MEMORY, "counters"));
  cudaEventCreate(&c->start);
  cudaEventCreate(&c->stop);
  *context = c;
  return GG_OK;
}

GG_API int gg_context_destroy(gg_context* c) {
  if (!c) return GG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  free_scene(c);
  free_run(c);
  if (c->tracking_points) cudaFree(c->tracking_points);
  if (c->tracking_count) cudaFree(c->tracking_count);
  cudaFree(c->rng);
  cudaFree(c->particles.E);
  cudaFree(c->particles.px);
  cudaFree(c->particles.py);
  cudaFree(c->particles.pz);
  cudaFree(c->particles.dx);
  cudaFree(c->particles.dy);
  cudaFree(c->particles.dz);
  cudaFree(c->particles.status);
  cudaFree(c->particles.scatter);
  cudaFree(c->particles.solid_id);
  cudaFree(c->slot_counter);
  cudaFree(c->error);
  if (c->dose_out) cudaFree(c->dose_out);
  if (c->start) cudaEventDestroy(c->start);
  if (c->stop) cudaEventDestroy(c->stop);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return GG_OK;
}

GG_API int gg_seed_random_states(uint32_t* states, int64_t number_of_slots, uint32_t seed, int64_t skip_slots) {
  if (!states || number_of_slots < 0 || number_of_slots > GG_MAXIMUM_PARTICLES || skip_slots < 0)
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad seeding arguments");
  std::mt19937 mt(seed);
  mt.discard(static_cast<unsigned long long>(skip_slots) * 4ull);
  const size_t S = GG_MAXIMUM_PARTICLES;
  for (int64_t j = 0; j < number_of_slots; ++j) {
    states[j] = static_cast<uint32_t>(mt());
    states[S + j] = static_cast<uint32_t>(mt());
    states[2 * S + j] = static_cast<uint32_t>(mt());
    states[3 * S + j] = static_cast<uint32_t>(mt());
    states[4 * S + j] = 0;
  }
  return GG_OK;
}

GG_API int gg_set_random_states(gg_context* c, const uint32_t* states, int64_t number_of_slots) {
  if (!c || !states || number_of_slots < 0 || number_of_slots > GG_MAXIMUM_PARTICLES)
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad random state arguments");
  GG_CUDA(cudaSetDevice(c->device));
  const size_t S = GG_MAXIMUM_PARTICLES;
  for (int k = 0; k < 5; ++k)
    GG_CUDA(cudaMemcpyAsync(c->rng + k * S, states + k * S, number_of_slots * sizeof(uint32_t), cudaMemcpyHostToDevice,
                            c->stream));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  return GG_OK;
}

GG_API int gg_get_random_states(gg_context* c, uint32_t* states, int64_t number_of_slots) {
  if (!c || !states || number_of_slots < 0 || number_of_slots > GG_MAXIMUM_PARTICLES)
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad random state arguments");
  GG_CUDA(cudaSetDevice(c->device));
  const size_t S = GG_MAXIMUM_PARTICLES;
  for (int k = 0; k < 5; ++k)
    GG_CUDA(cudaMemcpyAsync(states + k * S, c->rng + k * S, number_of_slots * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            c->stream));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  return GG_OK;
}

GG_API int gg_upload_scene(gg_context* c, const gg_scene* sc) {
  if (!c || !sc) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context or scene");
  if (sc->number_of_solids < 0 || sc->number_of_solids > gg::kMaxSolids)
    return fail(GG_ERROR_INVALID_ARGUMENT, "number of solids must be in [0, 64]");
  if (sc->number_of_tables < 0 || sc->number_of_tables > gg::kMaxNavigators)
    return fail(GG_ERROR_INVALID_ARGUMENT, "number of navigators must be in [0, 16]");
  if (!sc->rayleigh_fit) return fail(GG_ERROR_INVALID_ARGUMENT, "scene has no Rayleigh fit table");
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  free_scene(c, true);
  GG_CUDA(gg::set_rayleigh_fit(sc->rayleigh_fit));

  // Navigators that need the TLE attenuation tables.
  std::vector<char> nav_tle(sc->number_of_tables, 0);
  for (int s = 0; s < sc->number_of_solids; ++s) {
    const gg_solid& g = sc->solids[s];
    if (g.type == GG_SOLID_VOXELIZED && g.dose_map >= 0 && g.dose_map < sc->number_of_dose_maps &&
        sc->dose_maps[g.dose_map].tle && g.navigator >= 0 && g.navigator < sc->number_of_tables)
      nav_tle[g.navigator] = 1;
  }

  // ---- tables: shared-memory blob + HBM element data ----
  std::vector<unsigned char> blob;
  std::vector<gg::DevNavigator> navs(sc->number_of_tables);
  c->density_dev.assign(sc->number_of_tables, nullptr);
  for (int n = 0; n < sc->number_of_tables; ++n) {
    const gg_physics_tables& t = sc->tables[n];
    if (t.number_of_bins < 2 || t.number_of_bins > GG_MAX_CROSS_SECTION_BINS || t.number_of_materials < 1 ||
        t.number_of_materials > GG_MAX_MATERIALS || t.number_of_processes < 0 || t.number_of_processes > 3)
      return fail(GG_ERROR_INVALID_ARGUMENT, "bad table dimensions for navigator " + std::to_string(n));
    for (int p = 0; p < t.number_of_processes; ++p)
      if (t.process_id[p] < 0 || t.process_id[p] > 2) return fail(GG_ERROR_INVALID_ARGUMENT, "bad process id");
    gg::DevNavigator& d = navs[n];
    d.number_of_bins = t.number_of_bins;
    d.number_of_materials = t.number_of_materials;
    d.number_of_processes = t.number_of_processes;
    for (int p = 0; p < 3; ++p) d.process_id[p] = t.process_id[p];
    d.process_pack = static_cast<uint32_t>(t.number_of_processes);
    for (int p = 0; p < t.number_of_processes; ++p) d.process_pack |= static_cast<uint32_t>(t.process_id[p]) << (8 * (p + 1));
    const uint32_t nb = t.number_of_bins, nm = t.number_of_materials;
    d.energy_bins_offset = static_cast<uint32_t>(blob.size());
    blob.resize(align16(d.energy_bins_offset + nb * 4), 0);
    std::memcpy(blob.data() + d.energy_bins_offset, t.energy_bins, nb * 4);
    d.sigma_offset = static_cast<uint32_t>(blob.size());
    blob.resize(d.sigma_offset + nm * nb * 16, 0);
    float* sig = reinterpret_cast<float*>(blob.data() + d.sigma_offset);
    const size_t block = static_cast<size_t>(nm) * nb;
    for (uint32_t m = 0; m < nm; ++m)
      for (uint32_t b = 0; b < nb; ++b)
        for (int p = 0; p < 3; ++p) sig[(m * nb + b) * 4 + p] = t.cross_sections[p * block + b + nb * m];
    d.photon_cut_offset = static_cast<uint32_t>(blob.size());
    blob.resize(align16(d.photon_cut_offset + nm * 4), 0);
    std::memcpy(blob.data() + d.photon_cut_offset, t.photon_energy_cut, nm * 4);
    d.attenuation_offset = 0;
    if (nav_tle[n]) {
      if (!t.attenuation_energy_bins || !t.mu_en)
        return fail(GG_ERROR_INVALID_ARGUMENT, "TLE dose map without attenuation tables (navigator " + std::to_string(n) + ")");
      d.attenuation_offset = static_cast<uint32_t>(blob.size());
      const size_t bytes = (1 + static_cast<size_t>(nm)) * GG_ATTENUATION_BINS * 4;
      blob.resize(align16(static_cast<uint32_t>(d.attenuation_offset + bytes)), 0);
      std::memcpy(blob.data() + d.attenuation_offset, t.attenuation_energy_bins, GG_ATTENUATION_BINS * 4);
      std::memcpy(blob.data() + d.attenuation_offset + GG_ATTENUATION_BINS * 4, t.mu_en,
                  static_cast<size_t>(nm) * GG_ATTENUATION_BINS * 4);
    }
    int rc;
    int32_t* ne;
    int32_t* eo;
    uint8_t* z;
    float* ad;
    float* dens;
    if ((rc = dev_copy(c, t.number_of_elements, nm, &ne)) || (rc = dev_copy(c, t.element_offset, nm, &eo)) ||
        (rc = dev_copy(c, t.atomic_number, static_cast<size_t>(t.total_elements), &z)) ||
        (rc = dev_copy(c, t.atomic_number_density, static_cast<size_t>(t.total_elements), &ad)) ||
        (rc = dev_copy(c, t.density, nm, &dens)))
      return rc;
    d.number_of_elements = ne;
    d.element_offset = eo;
    d.atomic_number = z;
    d.atomic_number_density = ad;
    c->density_dev[n] = dens;
    float* ray = nullptr;
    if (t.rayleigh_per_atom) {
      if ((rc = dev_copy(c, t.rayleigh_per_atom, static_cast<size_t>(101) * nb, &ray))) return rc;
    } else {
      bool uses_rayleigh = false;
      for (int p = 0; p < t.number_of_processes; ++p) uses_rayleigh |= t.process_id[p] == GG_RAYLEIGH_SCATTERING;
      if (uses_rayleigh) return fail(GG_ERROR_INVALID_ARGUMENT, "Rayleigh activated without per-atom table");
    }
    d.rayleigh_per_atom = ray;
  }
  blob.resize(align16(static_cast<uint32_t>(blob.size())), 0);
  c->table_bytes = static_cast<uint32_t>(blob.size());
  int rc;
  if ((rc = dev_copy(c, blob.data(), blob.size(), &c->table_blob))) return rc;
  if ((rc = dev_copy(c, navs.data(), navs.size(), &c->navigators))) return rc;
  c->number_of_navigators = sc->number_of_tables;

  // ---- tallies ----
  c->histogram_sizes.assign(sc->histogram_sizes, sc->histogram_sizes + sc->number_of_histograms);
  for (int h = 0; h < sc->number_of_histograms; ++h) {
    int32_t* p;
    if ((rc = dev_copy<int32_t>(c, nullptr, c->histogram_sizes[h], &p))) return rc;
    c->histograms.push_back(p);
  }
  for (int d = 0; d < sc->number_of_dose_maps; ++d) {
    const gg_dose_map& g = sc->dose_maps[d];
    c->dose_tle.push_back(g.tle ? 1 : 0);
    gg::DevDoseMap m{};
    std::memcpy(m.size_of_dosels, g.size_of_dosels, sizeof(m.size_of_dosels));
    std::memcpy(m.inv_size_of_dosels, g.inv_size_of_dosels, sizeof(m.inv_size_of_dosels));
    std::memcpy(m.border_min, g.border_min, sizeof(m.border_min));
    std::memcpy(m.border_max, g.border_max, sizeof(m.border_max));
    std::memcpy(m.number_of_dosels, g.number_of_dosels, sizeof(m.number_of_dosels));
    m.total_number_of_dosels = g.total_number_of_dosels;
    m.slice_number_of_dosels = g.slice_number_of_dosels;
    const size_t n = static_cast<size_t>(g.total_number_of_dosels);
    if ((rc = dev_copy<unsigned long long>(c, nullptr, n, &m.edep))) return rc;
    if (g.record_edep_squared && (rc = dev_copy<double>(c, nullptr, n, &m.edep_squared))) return rc;
    if (g.record_hit && (rc = dev_copy<int32_t>(c, nullptr, n, &m.hit))) return rc;
    if (g.record_photon_tracking && (rc = dev_copy<int32_t>(c, nullptr, n, &m.photon_tracking))) return rc;
    c->dose_host.push_back(m);
  }
  if ((rc = dev_copy(c, c->dose_host.data(), c->dose_host.size(), &c->dose_maps))) return rc;
  if (sc->world) {
    // GGEMSWorld (src/navigators/GGEMSWorld.cc:191-231): one grid, centred on the origin
    const gg_world& w = *sc->world;
    size_t cells = 1;
    for (int a = 0; a < 3; ++a) {
      if (w.dimensions[a] <= 0 || !(w.sizes[a] > 0.0f)) return fail(GG_ERROR_INVALID_ARGUMENT, "world dimensions and sizes must be positive");
      cells *= static_cast<size_t>(w.dimensions[a]);
    }
    std::memcpy(c->world_dimensions, w.dimensions, sizeof(c->world_dimensions));
    std::memcpy(c->world_sizes, w.sizes, sizeof(c->world_sizes));
    c->world_cells = cells;
    if (w.photon_tracking && (rc = dev_copy<int32_t>(c, nullptr, cells, &c->world_photon))) return rc;
    if (w.energy_tracking && (rc = dev_copy<unsigned long long>(c, nullptr, cells, &c->world_energy))) return rc;
    if (w.energy_squared_tracking && (rc = dev_copy<double>(c, nullptr, cells, &c->world_energy_squared))) return rc;
    if (w.momentum && (rc = dev_copy<unsigned long long>(c, nullptr, 3 * cells, &c->world_momentum))) return rc;
  }

  // ---- solids ----
  std::vector<gg::DevSolid> solids(sc->number_of_solids);
  c->solid_host.assign(sc->solids, sc->solids + sc->number_of_solids);
  for (int s = 0; s < sc->number_of_solids; ++s) {
    if ((rc = make_dev_solid(c, sc->solids[s], &solids[s], c->scene_allocations, nullptr))) return rc;
    c->solid_host[s].labels = solids[s].labels;
  }
  c->solid_dev_host = solids;
  if ((rc = dev_copy(c, solids.data(), solids.size(), &c->solids))) return rc;
  c->number_of_solids = sc->number_of_solids;

  // Tables go to shared memory when they fit next to the solid / navigator copies.
  const size_t fixed = sizeof(gg::DevSolid) * c->number_of_solids + sizeof(gg::DevNavigator) * c->number_of_navigators + 16;
  c->tables_in_smem = c->table_bytes + fixed <= 96 * 1024;
  GG_CUDA(cudaStreamSynchronize(c->stream));
  c->scene_ready = true;
  release_spares(c);
  return GG_OK;
}

GG_API int gg_reset_tallies(gg_context* c) {
  if (!c || !c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  GG_CUDA(cudaSetDevice(c->device));
  for (size_t h = 0; h < c->histograms.size(); ++h)
    GG_CUDA(cudaMemsetAsync(c->histograms[h], 0, c->histogram_sizes[h] * sizeof(int32_t), c->stream));
  for (auto& m : c->dose_host) {
    size_t n = static_cast<size_t>(m.total_number_of_dosels);
    GG_CUDA(cudaMemsetAsync(m.edep, 0, n * 8, c->stream));
    if (m.edep_squared) GG_CUDA(cudaMemsetAsync(m.edep_squared, 0, n * 8, c->stream));
    if (m.hit) GG_CUDA(cudaMemsetAsync(m.hit, 0, n * 4, c->stream));
    if (m.photon_tracking) GG_CUDA(cudaMemsetAsync(m.photon_tracking, 0, n * 4, c->stream));
  }
  const size_t w = c->world_cells;
  if (c->world_photon) GG_CUDA(cudaMemsetAsync(c->world_photon, 0, w * 4, c->stream));
  if (c->world_energy) GG_CUDA(cudaMemsetAsync(c->world_energy, 0, w * 8, c->stream));
  if (c->world_energy_squared) GG_CUDA(cudaMemsetAsync(c->world_energy_squared, 0, w * 8, c->stream));
  if (c->world_momentum) GG_CUDA(cudaMemsetAsync(c->world_momentum, 0, 3 * w * 8, c->stream));
  return GG_OK;
}

GG_API int gg_device_tallies(gg_context* c, gg_device_tally* out, int32_t capacity, int32_t* count) {
  if (!c || !count) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context or count");
  if (!c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  std::vector<gg_device_tally> list;
  auto add = [&](void* p, size_t n, int type) {
    if (p && n) list.push_back(gg_device_tally{p, static_cast<int64_t>(n), type});
  };
  for (size_t h = 0; h < c->histograms.size(); ++h) add(c->histograms[h], c->histogram_sizes[h], GG_TALLY_INT32);
  for (auto& m : c->dose_host) {
    const size_t n = static_cast<size_t>(m.total_number_of_dosels);
    add(m.edep, n, GG_TALLY_INT64);
    add(m.edep_squared, n, GG_TALLY_FP64);
    add(m.hit, n, GG_TALLY_INT32);
    add(m.photon_tracking, n, GG_TALLY_INT32);
  }
  const size_t w = c->world_cells;
  add(c->world_photon, w, GG_TALLY_INT32);
  add(c->world_energy, w, GG_TALLY_INT64);
  add(c->world_energy_squared, w, GG_TALLY_FP64);
  add(c->world_momentum, 3 * w, GG_TALLY_INT64);
  *count = static_cast<int32_t>(list.size());
  if (!out) return GG_OK;
  if (capacity < *count) return fail(GG_ERROR_INVALID_ARGUMENT, "capacity below the number of tally buffers");
  std::copy(list.begin(), list.end(), out);
  return GG_OK;
}

GG_API int gg_batch_plan(uint64_t number_of_particles, uint64_t* batch_sizes, int64_t max_batches, int64_t* count) {
  if (!count) return fail(GG_ERROR_INVALID_ARGUMENT, "count is NULL");
  // GGEMSSource::OrganizeParticlesInBatch (src/sources/GGEMSSource.cc:403-425): float ceil.
  uint64_t nb = static_cast<uint64_t>(std::ceil(static_cast<float>(number_of_particles) / GG_MAXIMUM_PARTICLES));
  *count = static_cast<int64_t>(nb);
  if (batch_sizes) {
    for (uint64_t j = 0; j < nb && static_cast<int64_t>(j) < max_batches; ++j) {
      if (nb == 1) batch_sizes[j] = number_of_particles;
      else batch_sizes[j] = number_of_particles / nb + (j < number_of_particles % nb ? 1 : 0);
    }
  }
  return GG_OK;
}

}  // extern "C"

namespace {

// Device copy of a source: spectrum / CDF (and activity) arrays go to `owner`.
int make_dev_source(gg_context* c, const gg_source* src, gg::DevSource* out, std::vector<void*>& owner) {
  if (src->number_of_energy_bins < 1 || !src->energy_spectrum || !src->energy_cdf)
    return fail(GG_ERROR_INVALID_ARGUMENT, "source has no energy spectrum");
  gg::DevSource& s = *out;
  s = gg::DevSource{};
  s.type = src->type;
  std::memcpy(s.matrix, src->matrix, sizeof(s.matrix));
  s.beam_aperture = src->beam_aperture;
  s.new_aperture = 1.0 - std::cos(static_cast<double>(src->beam_aperture));
  std::memcpy(s.focal_spot_size, src->focal_spot_size, sizeof(s.focal_spot_size));
  s.number_of_energy_bins = src->number_of_energy_bins + 1;  // GGEMSXRaySource.cc:133
  s.is_interp = src->is_interp;
  const size_t ne = static_cast<size_t>(src->number_of_energy_bins) + 1;
  float* f;
  int rc;
  if ((rc = dev_copy_to(c, owner, src->energy_spectrum, ne, &f))) return rc;
  s.energy_spectrum = f;
  if ((rc = dev_copy_to(c, owner, src->energy_cdf, ne, &f))) return rc;
  s.energy_cdf = f;
  if (src->type == GG_SOURCE_VOXELIZED) {
    if (src->number_of_activity_bins < 2 || !src->activity_index || !src->activity_cdf)
      return fail(GG_ERROR_INVALID_ARGUMENT, "voxelized source without activity");
    std::memcpy(s.number_of_voxels, src->number_of_voxels, sizeof(s.number_of_voxels));
    std::memcpy(s.voxel_sizes, src->voxel_sizes, sizeof(s.voxel_sizes));
    std::memcpy(s.border_min, src->border_min, sizeof(s.border_min));
    s.number_of_activity_bins = static_cast<int32_t>(src->number_of_activity_bins);
    const size_t na = static_cast<size_t>(src->number_of_activity_bins);
    int32_t* idx;
    if ((rc = dev_copy_to(c, owner, src->activity_index, na, &idx))) return rc;
    s.activity_index = idx;
    if ((rc = dev_copy_to(c, owner, src->activity_cdf, na, &f))) return rc;
    s.activity_cdf = f;
  } else if (src->type != GG_SOURCE_XRAY) {
    return fail(GG_ERROR_INVALID_ARGUMENT, "unknown source type");
  }
  return GG_OK;
}

struct JobLaunch {
  gg::TransportParams params{};
  int grid = 0;
  int threads = gg::kBlockThreads;
  size_t smem = 0;
  bool mesh = false;
  bool dose = false;  // some solid tallies into a dose map
  bool aux = false;   // world grid or particle tracking
  int stash = 0;       // photon stash variant (1: 64 registers, 2: 80)
  bool empty = true;
};

// Device tables of `n` jobs (see gg_run_jobs), allocated into `owner`, and the
// launch shape.
int prepare_jobs(gg_context* c, const gg_job* jobs, int32_t n, std::vector<void*>& owner, JobLaunch* out) {
  if (!c || !jobs || n < 1) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context or no job");
  if (!c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  std::vector<gg::DevJob> dj;
  std::vector<gg::DevSolid> job_solids;
  std::map<const void*, const void*> labels_seen;
  bool mesh = false, own_solids = false;
  for (const gg_solid& g : c->solid_host) mesh |= g.type == GG_SOLID_MESHED;
  uint64_t max_slots = 0;
  int rc;
  for (int j = 0; j < n; ++j) {
    if (jobs[j].number_of_particles == 0) continue;
    int64_t nb64 = 0;
    gg_batch_plan(jobs[j].number_of_particles, nullptr, 0, &nb64);
    const uint64_t nb = static_cast<uint64_t>(nb64), np = jobs[j].number_of_particles;
    if (nb == 0 || nb > 0xffffffffull) return fail(GG_ERROR_INVALID_ARGUMENT, "bad batch plan");
    gg::DevJob J{};
    J.q = nb == 1 ? np : np / nb;
    J.r = nb == 1 ? 0 : np % nb;
    J.nb = static_cast<uint32_t>(nb);
    const uint64_t slots = J.q + (J.r ? 1 : 0);
    if (slots > GG_MAXIMUM_PARTICLES) return fail(GG_ERROR_INVALID_ARGUMENT, "batch larger than the slot count");
    J.slots = static_cast<uint32_t>(slots);
    if (slots > max_slots) max_slots = slots;
    if ((rc = make_dev_source(c, &jobs[j].source, &J.source, owner))) return rc;
    dj.push_back(J);
    for (int s = 0; s < c->number_of_solids; ++s) {
      if (jobs[j].solids) {
        gg::DevSolid d;
        if ((rc = make_dev_solid(c, jobs[j].solids[s], &d, owner, &labels_seen))) return rc;
        mesh |= jobs[j].solids[s].type == GG_SOLID_MESHED;
        own_solids = true;
        job_solids.push_back(d);
      } else {
        job_solids.push_back(c->solid_dev_host[s]);
      }
    }
  }
  if (dj.empty()) return GG_OK;
  bool aux = false;
  bool dose = false;
  for (int s = 0; s < c->number_of_solids; ++s) dose |= c->solid_dev_host[s].dose_map >= 0;
  for (const gg::DevSolid& d : job_solids) dose |= d.dose_map >= 0;
  gg::TransportParams& P = out->params;
  P = gg::TransportParams{};
  gg::DevJob* djd;
  if ((rc = dev_copy_to(c, owner, dj.data(), dj.size(), &djd))) return rc;
  P.jobs = djd;
  P.number_of_jobs = static_cast<int32_t>(dj.size());
  P.solids = c->solids;
  if (dj.size() > 1 || own_solids) {
    gg::DevSolid* js;
    if ((rc = dev_copy_to(c, owner, job_solids.data(), job_solids.size(), &js))) return rc;
    if (dj.size() > 1) P.job_solids = js;
    else P.solids = js;  // a single job's own solids replace the scene's for this launch
  }
  P.number_of_slots = static_cast<uint32_t>(max_slots);
  P.rng = c->rng;
  P.particles = c->particles;
  P.number_of_solids = c->number_of_solids;
  P.navigators = c->navigators;
  P.number_of_navigators = c->number_of_navigators;
  P.dose_maps = c->dose_maps;
  P.table_blob = c->table_blob;
  P.table_bytes = c->table_bytes;
  P.tables_in_smem = c->tables_in_smem ? 1 : 0;
  P.slot_counter = c->slot_counter;
  P.error = c->error;
  P.regroup_lanes = c->regroup_lanes;
  P.regroup_ratio4 = c->regroup_ratio4;
  P.slots_per_claim = static_cast<uint32_t>(c->slots_per_claim);
  P.stash_swap_lanes = c->stash_swap_lanes;
  P.stash_round_photons = c->stash_round_photons;
  P.tracking_slot = -1;
  if (c->tracking_slot >= 0 && c->tracking_points) {
    P.tracking_slot = c->tracking_slot;
    P.tracking_capacity = c->tracking_capacity;
    P.tracking_points = c->tracking_points;
    P.tracking_count = c->tracking_count;
    aux = true;  // recorded by the full kernel variant
  }
  if (c->world_cells) {
    std::memcpy(P.world_dimensions, c->world_dimensions, sizeof(P.world_dimensions));
    std::memcpy(P.world_sizes, c->world_sizes, sizeof(P.world_sizes));
    P.world_photon = c->world_photon;
    P.world_energy = c->world_energy;
    P.world_energy_squared = c->world_energy_squared;
    P.world_momentum = c->world_momentum;
    aux = true;  // the world walk lives in the full kernel variant
  }
  const bool batch = P.number_of_jobs > 1;
  // meshed scenes: the 80-register stash variant only (the mesh variant has 80 registers already)
  const int stash = aux ? 0 : (c->stash_registers == 64 ? (mesh ? 2 : 1) : (c->stash_registers == 80 ? 2 : 0));
  out->smem = (c->tables_in_smem ? c->table_bytes : 0) + sizeof(gg::DevSolid) * c->number_of_solids +
              sizeof(gg::DevNavigator) * c->number_of_navigators + 16;
  if (stash) out->smem += (c->block_threads / 32) * gg::stash_bytes_per_warp(batch, false);
  int blocks_per_sm = 0;
  GG_CUDA(gg::configure_transport(out->smem, c->block_threads, &blocks_per_sm, mesh, batch, dose, aux, stash));
  if (blocks_per_sm < 1) return fail(GG_ERROR_CUDA, "transport kernel does not fit on an SM");
  if (c->blocks_per_sm > 0 && c->blocks_per_sm < blocks_per_sm) blocks_per_sm = c->blocks_per_sm;
  uint64_t grid = static_cast<uint64_t>(blocks_per_sm) * c->sm_count;
  const uint64_t lanes_needed = (max_slots + c->slots_per_claim - 1) / c->slots_per_claim;
  const uint64_t needed = (lanes_needed + c->block_threads - 1) / c->block_threads;
  if (grid > needed) grid = needed;
  out->grid = static_cast<int>(grid);
  out->threads = c->block_threads;
  out->mesh = mesh;
  out->dose = dose;
  out->aux = aux;
  out->stash = stash;
  out->empty = false;
  return GG_OK;
}

// Work-queue reset and the persistent launch, on the context's stream.
int enqueue_jobs(gg_context* c, const JobLaunch& L) {
  GG_CUDA(cudaMemsetAsync(c->slot_counter, 0, sizeof(unsigned int), c->stream));
  if (L.params.tracking_count) GG_CUDA(cudaMemsetAsync(L.params.tracking_count, 0, sizeof(int32_t), c->stream));
  GG_CUDA(cudaMemsetAsync(c->error, 0, sizeof(int), c->stream));
  gg::launch_transport(L.params, L.grid, L.threads, L.smem, c->stream, L.mesh, L.dose, L.aux, L.stash);
  GG_CUDA(cudaGetLastError());
  return GG_OK;
}

// One persistent launch for `n` jobs (see gg_run_jobs).
int launch_jobs(gg_context* c, const gg_job* jobs, int32_t n) {
  if (!c) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context");
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  free_run(c);
  JobLaunch L;
  int rc;
  if ((rc = prepare_jobs(c, jobs, n, c->run_allocations, &L))) return rc;
  if (L.empty) return GG_OK;
  GG_CUDA(cudaEventRecord(c->start, c->stream));
  if ((rc = enqueue_jobs(c, L))) return rc;
  GG_CUDA(cudaEventRecord(c->stop, c->stream));
  c->last_launches = 1;
  return GG_OK;
}

}  // namespace

extern "C" {

GG_API int gg_run_source(gg_context* c, const gg_source* src, uint64_t number_of_particles) {
  if (!c || !src) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context or source");
  if (!c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  if (number_of_particles == 0) return GG_OK;
  gg_job job{};
  job.source = *src;
  job.number_of_particles = number_of_particles;
  job.solids = nullptr;
  return launch_jobs(c, &job, 1);
}

GG_API int gg_run_jobs(gg_context* c, const gg_job* jobs, int32_t number_of_jobs) {
  return launch_jobs(c, jobs, number_of_jobs);
}

}  // extern "C"

struct gg_graph {
  gg_context* context = nullptr;
  std::vector<void*> allocations;  // the jobs' device tables
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

extern "C" {

GG_API int gg_capture_jobs(gg_context* c, const gg_job* jobs, int32_t number_of_jobs, gg_graph** out) {
  if (!c || !out) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  gg_graph* g = new gg_graph();
  g->context = c;
  auto drop = [&](int rc) {
    gg_graph_destroy(g);
    return rc;
  };
  JobLaunch L;
  int rc = prepare_jobs(c, jobs, number_of_jobs, g->allocations, &L);
  if (rc) return drop(rc);
  if (L.empty) return drop(fail(GG_ERROR_INVALID_ARGUMENT, "no primaries in the jobs"));
  cudaError_t e = cudaStreamSynchronize(c->stream);  // the tables' uploads land before capture
  if (e == cudaSuccess) e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return drop(fail(GG_ERROR_CUDA, std::string("begin capture: ") + cudaGetErrorString(e)));
  rc = enqueue_jobs(c, L);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(c->stream, &graph);
  g->graph = graph;
  if (rc) return drop(rc);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) return drop(fail(GG_ERROR_CUDA, std::string("capture: ") + cudaGetErrorString(e)));
  *out = g;
  return GG_OK;
}

GG_API int gg_graph_launch(gg_graph* g) {
  if (!g || !g->exec) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL graph");
  gg_context* c = g->context;
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaEventRecord(c->start, c->stream));
  GG_CUDA(cudaGraphLaunch(g->exec, c->stream));
  GG_CUDA(cudaEventRecord(c->stop, c->stream));
  c->last_launches = 1;
  return GG_OK;
}

GG_API int gg_graph_destroy(gg_graph* g) {
  if (!g) return GG_OK;
  if (g->context) {
    cudaSetDevice(g->context->device);
    cudaStreamSynchronize(g->context->stream);
  }
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (void* p : g->allocations) cudaFree(p);
  delete g;
  return GG_OK;
}

GG_API int gg_synchronize(gg_context* c) {
  if (!c) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context");
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  int err = 0;
  GG_CUDA(cudaMemcpy(&err, c->error, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return fail(GG_ERROR_TIMEOUT, "a bounded wait in the transport kernel timed out");
  cudaEventElapsedTime(&c->last_ms, c->start, c->stop);
  return GG_OK;
}

GG_API int gg_set_transport_tuning(gg_context* c, int32_t blocks_per_sm, int32_t regroup_lanes, int32_t regroup_ratio4) {
  if (!c || blocks_per_sm < 0 || regroup_lanes < 1 || regroup_lanes > 32 || regroup_ratio4 < 0 || regroup_ratio4 > 128)
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad transport tuning");
  c->blocks_per_sm = blocks_per_sm;
  c->regroup_lanes = regroup_lanes;
  c->regroup_ratio4 = regroup_ratio4;
  return GG_OK;
}

GG_API int gg_get_transport_tuning(gg_context* c, int32_t* blocks_per_sm, int32_t* regroup_lanes, int32_t* regroup_ratio4) {
  if (!c) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context");
  if (blocks_per_sm) *blocks_per_sm = c->blocks_per_sm;
  if (regroup_lanes) *regroup_lanes = c->regroup_lanes;
  if (regroup_ratio4) *regroup_ratio4 = c->regroup_ratio4;
  return GG_OK;
}

GG_API int gg_set_transport_launch(gg_context* c, int32_t block_threads, int32_t slots_per_claim) {
  if (!c || (block_threads != 128 && block_threads != 256 && block_threads != 512) || slots_per_claim < 1 ||
      slots_per_claim > 64 || (slots_per_claim & (slots_per_claim - 1)) != 0)
    return fail(GG_ERROR_INVALID_ARGUMENT,
                "bad transport launch (block_threads 128/256/512, slots_per_claim a power of two up to 64)");
  c->block_threads = block_threads;
  c->slots_per_claim = slots_per_claim;
  return GG_OK;
}

GG_API int gg_get_transport_launch(gg_context* c, int32_t* block_threads, int32_t* slots_per_claim) {
  if (!c) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context");
  if (block_threads) *block_threads = c->block_threads;
  if (slots_per_claim) *slots_per_claim = c->slots_per_claim;
  return GG_OK;
}

GG_API int gg_set_transport_stash(gg_context* c, int32_t registers, int32_t swap_lanes, int32_t round_photons) {
  if (!c || (registers != 0 && registers != 64 && registers != 80) || swap_lanes < 1 || swap_lanes > 32 ||
      round_photons < 1 || round_photons > 2 * gg::kStashRecords)
    return fail(GG_ERROR_INVALID_ARGUMENT,
                "bad photon stash (registers 0, 64 or 80; swap_lanes 1..32; round_photons 1..64)");
  c->stash_registers = registers;
  c->stash_swap_lanes = swap_lanes;
  c->stash_round_photons = round_photons;
  return GG_OK;
}

GG_API int gg_get_transport_stash(gg_context* c, int32_t* registers, int32_t* swap_lanes, int32_t* round_photons) {
  if (!c) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context");
  if (registers) *registers = c->stash_registers;
  if (swap_lanes) *swap_lanes = c->stash_swap_lanes;
  if (round_photons) *round_photons = c->stash_round_photons;
  return GG_OK;
}

}  // extern "C"

namespace {

// The launch shape the autotuner varies: the photon stash (off, 64 or 80
// registers), resident blocks per SM, the rare-phase regroup ratio, the block
// size and the photons per thread (slots a lane claims per work-queue grab).
struct LaunchShape {
  int stash_registers, blocks_per_sm, regroup_ratio4, block_threads, slots_per_claim, stash_round_photons;
};

void apply_shape(gg_context* c, const LaunchShape& s) {
  c->stash_registers = s.stash_registers;
  c->stash_round_photons = s.stash_round_photons;
  c->blocks_per_sm = s.blocks_per_sm;
  c->regroup_lanes = 32;
  c->regroup_ratio4 = s.regroup_ratio4;
  c->block_threads = s.block_threads;
  c->slots_per_claim = s.slots_per_claim;
}

// Times `trial` (one launch of the workload to tune on) for each launch shape
// of a coordinate search, restoring the random states before every trial, and
// keeps the fastest:
//   1. photon stash (off, 64, 80 registers) x resident blocks per SM (4..1, as
//      many as the registers allow) x regroup ratio (3/4, 4/4, 6/4) at 256
//      threads, one slot per claim;
//   2. block size 128 and 512 at the same resident threads per SM as the best of 1;
//   3. 2, 4 and 8 slots per claim at the best of 1-2;
//   4. with the stash, 32 and 48 waiting photons per rare round (default 40).
// The tallies are zeroed and the random states restored afterwards.
int autotune(gg_context* c, const std::function<int()>& trial, float* best_ms) {
  GG_CUDA(cudaSetDevice(c->device));
  const size_t bytes = static_cast<size_t>(5) * GG_MAXIMUM_PARTICLES * sizeof(uint32_t);
  void* saved = nullptr;
  GG_CUDA(cudaMalloc(&saved, bytes));
  auto restore = [&]() { return cudaMemcpyAsync(c->rng, saved, bytes, cudaMemcpyDeviceToDevice, c->stream); };
  cudaError_t e = cudaMemcpyAsync(saved, c->rng, bytes, cudaMemcpyDeviceToDevice, c->stream);
  const LaunchShape start{c->stash_registers, c->blocks_per_sm, c->regroup_ratio4, c->block_threads,
                          c->slots_per_claim, c->stash_round_photons};
  const int round0 = c->stash_round_photons;
  LaunchShape best = start;
  float best_time = -1.0f;
  int rc = GG_OK;
  auto run = [&](const LaunchShape& s) {
    if (e != cudaSuccess || rc != GG_OK) return;
    apply_shape(c, s);
    if ((e = restore()) != cudaSuccess) return;
    if ((rc = trial()) != GG_OK) return;
    if ((rc = gg_synchronize(c)) != GG_OK) return;
    if (best_time < 0.0f || c->last_ms < best_time) {
      best_time = c->last_ms;
      best = s;
    }
  };
  for (int stash : {0, 64, 80})
    for (int bps = stash == 80 ? 3 : 4; bps >= 1; --bps)
      for (int r : {3, 4, 6}) run({stash, bps, r, gg::kBlockThreads, 1, round0});
  const LaunchShape stage1 = best;
  for (int threads : {128, 512}) {
    const int bps = stage1.blocks_per_sm * gg::kBlockThreads / threads;
    if (bps >= 1) run({stage1.stash_registers, bps, stage1.regroup_ratio4, threads, 1, round0});
  }
  const LaunchShape stage2 = best;
  for (int k : {2, 4, 8})
    run({stage2.stash_registers, stage2.blocks_per_sm, stage2.regroup_ratio4, stage2.block_threads, k, round0});
  const LaunchShape stage3 = best;
  if (stage3.stash_registers != 0)
    for (int t : {32, 48})
      run({stage3.stash_registers, stage3.blocks_per_sm, stage3.regroup_ratio4, stage3.block_threads,
           stage3.slots_per_claim, t});
  if (e == cudaSuccess) e = restore();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(saved);
  apply_shape(c, best_time < 0.0f ? start : best);
  if (e != cudaSuccess) return fail(GG_ERROR_CUDA, std::string("autotune: ") + cudaGetErrorString(e));
  if (rc != GG_OK) return rc;
  if ((rc = gg_reset_tallies(c)) != GG_OK) return rc;
  if (best_ms) *best_ms = best_time;
  return GG_OK;
}

}  // namespace

extern "C" {

GG_API int gg_autotune(gg_context* c, const gg_source* source, uint64_t number_of_particles, float* best_ms) {
  if (!c || !source || number_of_particles == 0) return fail(GG_ERROR_INVALID_ARGUMENT, "bad autotune arguments");
  if (!c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  return autotune(c, [&]() { return gg_run_source(c, source, number_of_particles); }, best_ms);
}

GG_API int gg_autotune_jobs(gg_context* c, const gg_job* jobs, int32_t number_of_jobs, float* best_ms) {
  if (!c || !jobs || number_of_jobs < 1) return fail(GG_ERROR_INVALID_ARGUMENT, "bad autotune arguments");
  if (!c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  return autotune(c, [&]() { return gg_run_jobs(c, jobs, number_of_jobs); }, best_ms);
}

GG_API int gg_line_integrals(gg_context* c, const gg_solid* phantom, const gg_solid* detector, const float* source_position,
                             const float* mu, int32_t number_of_materials, float* line_integrals) {
  if (!c || !phantom || !detector || !source_position || !mu || !line_integrals || number_of_materials < 1)
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  if (phantom->type != GG_SOLID_VOXELIZED || !phantom->labels || detector->type != GG_SOLID_BOX)
    return fail(GG_ERROR_INVALID_ARGUMENT, "need a voxelized phantom solid (with labels) and a detector box solid");
  for (int a = 0; a < 3; ++a)
    if (phantom->number_of_voxels[a] < 1 || !(phantom->voxel_sizes[a] > 0.0f) || detector->virtual_element_number[a] < 1)
      return fail(GG_ERROR_INVALID_ARGUMENT, "bad phantom or detector dimensions");
  GG_CUDA(cudaSetDevice(c->device));
  gg::ProjectorParams P{};
  std::memcpy(P.phantom_matrix, phantom->obb.matrix, sizeof(P.phantom_matrix));
  std::memcpy(P.border_min, phantom->obb.border_min, sizeof(P.border_min));
  std::memcpy(P.border_max, phantom->obb.border_max, sizeof(P.border_max));
  std::memcpy(P.number_of_voxels, phantom->number_of_voxels, sizeof(P.number_of_voxels));
  std::memcpy(P.voxel_sizes, phantom->voxel_sizes, sizeof(P.voxel_sizes));
  P.number_of_materials = number_of_materials;
  std::memcpy(P.detector_matrix, detector->obb.matrix, sizeof(P.detector_matrix));
  std::memcpy(P.detector_min, detector->obb.border_min, sizeof(P.detector_min));
  for (int a = 0; a < 3; ++a) P.element_size[a] = detector->box_size[a] / static_cast<float>(detector->virtual_element_number[a]);
  P.elements[0] = detector->virtual_element_number[0];
  P.elements[1] = detector->virtual_element_number[1];
  std::memcpy(P.source, source_position, sizeof(P.source));
  const size_t n = static_cast<size_t>(P.elements[0]) * P.elements[1];
  const size_t nv = static_cast<size_t>(phantom->number_of_voxels[0]) * phantom->number_of_voxels[1] * phantom->number_of_voxels[2];
  // stream-ordered buffers (no device-wide synchronisation)
  float *dmu = nullptr, *dout = nullptr;
  uint8_t* dlab = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&dmu), number_of_materials * sizeof(float), c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&dlab), nv, c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&dout), n * sizeof(float), c->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dmu, mu, number_of_materials * sizeof(float), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dlab, phantom->labels, nv, cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) {
    P.mu = dmu;
    P.labels = dlab;
    P.out = dout;
    gg::launch_line_integrals(P, c->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(line_integrals, dout, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  if (dmu) cudaFreeAsync(dmu, c->stream);
  if (dlab) cudaFreeAsync(dlab, c->stream);
  if (dout) cudaFreeAsync(dout, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(GG_ERROR_CUDA, std::string("line integrals: ") + cudaGetErrorString(e));
  return GG_OK;
}

GG_API int gg_line_integrals_batch(gg_context* c, const gg_solid* phantom, const gg_solid* detectors,
                                   const float* source_positions, int32_t count, const float* mu,
                                   int32_t number_of_materials, float* inputs) {
  if (!c || !phantom || !detectors || !source_positions || !mu || !inputs || number_of_materials < 1 || count < 1)
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  if (phantom->type != GG_SOLID_VOXELIZED || !phantom->labels)
    return fail(GG_ERROR_INVALID_ARGUMENT, "need a voxelized phantom solid (with labels)");
  for (int a = 0; a < 3; ++a)
    if (phantom->number_of_voxels[a] < 1 || !(phantom->voxel_sizes[a] > 0.0f))
      return fail(GG_ERROR_INVALID_ARGUMENT, "bad phantom dimensions");
  const int32_t ex = detectors[0].virtual_element_number[0], ey = detectors[0].virtual_element_number[1];
  for (int k = 0; k < count; ++k)
    if (detectors[k].type != GG_SOLID_BOX || detectors[k].virtual_element_number[0] != ex ||
        detectors[k].virtual_element_number[1] != ey || ex < 1 || ey < 1)
      return fail(GG_ERROR_INVALID_ARGUMENT, "detectors must be boxes with the same element grid");
  GG_CUDA(cudaSetDevice(c->device));
  const size_t n = static_cast<size_t>(ex) * ey;
  const size_t nv = static_cast<size_t>(phantom->number_of_voxels[0]) * phantom->number_of_voxels[1] * phantom->number_of_voxels[2];
  // `inputs` in this device's memory: the kernels write it directly
  cudaPointerAttributes pa{};
  const bool on_device = cudaPointerGetAttributes(&pa, inputs) == cudaSuccess &&
                         (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged) && pa.device == c->device;
  cudaGetLastError();  // a host pointer unknown to CUDA is not an error here
  // stream-ordered buffers: no device-wide synchronisation (cudaFree would wait
  // for transport running on other streams)
  float *dmu = nullptr, *dout = nullptr;
  uint8_t* dlab = nullptr;
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&dmu), number_of_materials * sizeof(float), c->stream);
  if (e == cudaSuccess) e = cudaMallocAsync(reinterpret_cast<void**>(&dlab), nv, c->stream);
  if (e == cudaSuccess && !on_device)
    e = cudaMallocAsync(reinterpret_cast<void**>(&dout), 2 * n * count * sizeof(float), c->stream);
  float* const target = on_device ? inputs : dout;
  auto cleanup = [&]() {
    if (dmu) cudaFreeAsync(dmu, c->stream);
    if (dlab) cudaFreeAsync(dlab, c->stream);
    if (dout) cudaFreeAsync(dout, c->stream);
  };
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dmu, mu, number_of_materials * sizeof(float), cudaMemcpyHostToDevice, c->stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dlab, phantom->labels, nv, cudaMemcpyHostToDevice, c->stream);
  for (int k = 0; k < count && e == cudaSuccess; ++k) {
    gg::ProjectorParams P{};
    std::memcpy(P.phantom_matrix, phantom->obb.matrix, sizeof(P.phantom_matrix));
    std::memcpy(P.border_min, phantom->obb.border_min, sizeof(P.border_min));
    std::memcpy(P.border_max, phantom->obb.border_max, sizeof(P.border_max));
    std::memcpy(P.number_of_voxels, phantom->number_of_voxels, sizeof(P.number_of_voxels));
    std::memcpy(P.voxel_sizes, phantom->voxel_sizes, sizeof(P.voxel_sizes));
    P.number_of_materials = number_of_materials;
    const gg_solid& d = detectors[k];
    std::memcpy(P.detector_matrix, d.obb.matrix, sizeof(P.detector_matrix));
    std::memcpy(P.detector_min, d.obb.border_min, sizeof(P.detector_min));
    for (int a = 0; a < 3; ++a) P.element_size[a] = d.box_size[a] / static_cast<float>(d.virtual_element_number[a]);
    P.elements[0] = ex;
    P.elements[1] = ey;
    std::memcpy(P.source, source_positions + 3 * k, sizeof(P.source));
    P.mu = dmu;
    P.labels = dlab;
    P.out = target + 2 * n * k;
    P.network_input = 1;
    gg::launch_line_integrals(P, c->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && !on_device)
    e = cudaMemcpyAsync(inputs, dout, 2 * n * count * sizeof(float), cudaMemcpyDeviceToHost, c->stream);
  cleanup();
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(GG_ERROR_CUDA, std::string("line integrals: ") + cudaGetErrorString(e));
  return GG_OK;
}

GG_API int gg_set_tracking(gg_context* c, int32_t slot, int32_t capacity) {
  if (!c || slot >= GG_MAXIMUM_PARTICLES || (slot >= 0 && capacity < 1))
    return fail(GG_ERROR_INVALID_ARGUMENT, "bad tracking slot or capacity");
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  if (c->tracking_points) cudaFree(c->tracking_points);
  if (c->tracking_count) cudaFree(c->tracking_count);
  c->tracking_points = nullptr;
  c->tracking_count = nullptr;
  c->tracking_slot = -1;
  c->tracking_capacity = 0;
  if (slot < 0) return GG_OK;
  GG_CUDA(cudaMalloc(&c->tracking_points, static_cast<size_t>(capacity) * sizeof(gg_track_point)));
  GG_CUDA(cudaMalloc(&c->tracking_count, sizeof(int32_t)));
  GG_CUDA(cudaMemset(c->tracking_count, 0, sizeof(int32_t)));
  c->tracking_slot = slot;
  c->tracking_capacity = capacity;
  return GG_OK;
}

GG_API int gg_read_tracking(gg_context* c, gg_track_point* points, int32_t capacity, int32_t* count) {
  if (!c || !count || capacity < 0 || (capacity > 0 && !points)) return fail(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  *count = 0;
  if (!c->tracking_points) return GG_OK;
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  int32_t n = 0;
  GG_CUDA(cudaMemcpy(&n, c->tracking_count, sizeof(n), cudaMemcpyDeviceToHost));
  *count = n;
  const int32_t stored = std::min(std::min(n, c->tracking_capacity), capacity);
  if (stored > 0)
    GG_CUDA(cudaMemcpy(points, c->tracking_points, static_cast<size_t>(stored) * sizeof(gg_track_point),
                       cudaMemcpyDeviceToHost));
  return GG_OK;
}

GG_API int gg_last_run_stats(gg_context* c, float* milliseconds, int64_t* kernel_launches) {
  if (!c) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL context");
  if (milliseconds) *milliseconds = c->last_ms;
  if (kernel_launches) *kernel_launches = c->last_launches;
  return GG_OK;
}

}  // extern "C"

namespace {
// n int64 fixed-point tallies (LSB 2^-32 MeV) into the caller's doubles: the
// integers land in the caller's array itself (same size), whose page-locked
// memory the copy then uses if it is, and are converted in place.
cudaError_t read_fixed_point(double* dst, const unsigned long long* src, size_t n) {
  cudaError_t e = cudaMemcpy(dst, src, n * 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return e;
  long long* q = reinterpret_cast<long long*>(dst);
  for (size_t i = 0; i < n; ++i) {
    long long v;
    std::memcpy(&v, q + i, sizeof(v));
    dst[i] = static_cast<double>(v) / gg::kEdepScale;
  }
  return cudaSuccess;
}
}  // namespace

extern "C" {

GG_API int gg_read_tallies(gg_context* c, gg_tally_buffers* t) {
  if (!c || !t) return fail(GG_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (!c->scene_ready) return fail(GG_ERROR_STATE, "no scene uploaded");
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  for (size_t h = 0; h < c->histograms.size(); ++h)
    if (t->histograms && t->histograms[h])
      GG_CUDA(cudaMemcpy(t->histograms[h], c->histograms[h], c->histogram_sizes[h] * 4, cudaMemcpyDeviceToHost));
  for (size_t d = 0; d < c->dose_host.size(); ++d) {
    const gg::DevDoseMap& m = c->dose_host[d];
    const size_t n = static_cast<size_t>(m.total_number_of_dosels);
    if (t->edep && t->edep[d]) GG_CUDA(read_fixed_point(t->edep[d], m.edep, n));
    if (t->edep_squared && t->edep_squared[d] && m.edep_squared)
      GG_CUDA(cudaMemcpy(t->edep_squared[d], m.edep_squared, n * 8, cudaMemcpyDeviceToHost));
    if (t->hit && t->hit[d] && m.hit) GG_CUDA(cudaMemcpy(t->hit[d], m.hit, n * 4, cudaMemcpyDeviceToHost));
    if (t->photon_tracking && t->photon_tracking[d] && m.photon_tracking)
      GG_CUDA(cudaMemcpy(t->photon_tracking[d], m.photon_tracking, n * 4, cudaMemcpyDeviceToHost));
  }
  const size_t w = c->world_cells;
  auto read_fixed = [&](double* dst, const unsigned long long* src) { return read_fixed_point(dst, src, w); };
  if (t->world_photon_tracking && c->world_photon)
    GG_CUDA(cudaMemcpy(t->world_photon_tracking, c->world_photon, w * 4, cudaMemcpyDeviceToHost));
  if (t->world_energy && c->world_energy) GG_CUDA(read_fixed(t->world_energy, c->world_energy));
  if (t->world_energy_squared && c->world_energy_squared)
    GG_CUDA(cudaMemcpy(t->world_energy_squared, c->world_energy_squared, w * 8, cudaMemcpyDeviceToHost));
  if (c->world_momentum) {
    double* m[3] = {t->world_momentum_x, t->world_momentum_y, t->world_momentum_z};
    for (int a = 0; a < 3; ++a)
      if (m[a]) GG_CUDA(read_fixed(m[a], c->world_momentum + a * w));
  }
  return GG_OK;
}

GG_API int gg_read_particles(gg_context* c, gg_particle_buffers* b, int64_t n) {
  if (!c || !b || n < 0 || n > GG_MAXIMUM_PARTICLES) return fail(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  GG_CUDA(cudaSetDevice(c->device));
  GG_CUDA(cudaStreamSynchronize(c->stream));
  const gg::DevParticles& p = c->particles;
  float* dst[7] = {b->E, b->px, b->py, b->pz, b->dx, b->dy, b->dz};
  float* src[7] = {p.E, p.px, p.py, p.pz, p.dx, p.dy, p.dz};
  for (int k = 0; k < 7; ++k)
    if (dst[k]) GG_CUDA(cudaMemcpy(dst[k], src[k], n * 4, cudaMemcpyDeviceToHost));
  if (b->status) GG_CUDA(cudaMemcpy(b->status, p.status, n, cudaMemcpyDeviceToHost));
  if (b->scatter) GG_CUDA(cudaMemcpy(b->scatter, p.scatter, n, cudaMemcpyDeviceToHost));
  if (b->solid_id) GG_CUDA(cudaMemcpy(b->solid_id, p.solid_id, n * 4, cudaMemcpyDeviceToHost));
  return GG_OK;
}

GG_API int gg_compute_dose(gg_context* c, int32_t dose_map, int32_t solid, float scale_factor,
                           int32_t is_water_reference, float minimum_density, float* dose, float* uncertainty) {
  if (!c || !c->scene_ready || !dose) return fail(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  if (dose_map < 0 || dose_map >= static_cast<int>(c->dose_host.size()) || solid < 0 ||
      solid >= static_cast<int>(c->solid_host.size()) ||
      (c->solid_host[solid].type != GG_SOLID_VOXELIZED && c->solid_host[solid].type != GG_SOLID_MESHED))
    return fail(GG_ERROR_INVALID_ARGUMENT, "dose map or solid out of range");
  GG_CUDA(cudaSetDevice(c->device));
  const gg_solid& s = c->solid_host[solid];
  gg::DoseParams P{};
  P.map = c->dose_host[dose_map];
  std::memcpy(P.number_of_voxels, s.number_of_voxels, sizeof(P.number_of_voxels));
  std::memcpy(P.voxel_sizes, s.voxel_sizes, sizeof(P.voxel_sizes));
  std::memcpy(P.border_min, s.obb.border_min, sizeof(P.border_min));
  P.labels = s.labels;
  P.density = c->density_dev[s.navigator];
  P.scale_factor = scale_factor;
  P.is_water_reference = is_water_reference;
  P.minimum_density = minimum_density;
  const size_t n = static_cast<size_t>(P.map.total_number_of_dosels);
  if (c->dose_out_floats < 2 * n) {  // grow once; later calls reuse the buffer
    GG_CUDA(cudaStreamSynchronize(c->stream));
    if (c->dose_out) cudaFree(c->dose_out);
    c->dose_out = nullptr;
    c->dose_out_floats = 0;
    if (cudaMalloc(&c->dose_out, 2 * n * sizeof(float)) != cudaSuccess)
      return fail(GG_ERROR_OUT_OF_MEMORY, "dose output buffer");
    c->dose_out_floats = 2 * n;
  }
  P.dose = c->dose_out;
  P.uncertainty = uncertainty ? c->dose_out + n : nullptr;
  gg::launch_compute_dose(P, c->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dose, P.dose, n * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && uncertainty) e = cudaMemcpyAsync(uncertainty, P.uncertainty, n * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(GG_ERROR_CUDA, std::string("compute dose: ") + cudaGetErrorString(e));
  return GG_OK;
}

}  // extern "C"

// ---- dose finalisation without device allocation ----
//
// gg_compute_dose allocates its two device output arrays per call and frees
// them afterwards; cudaFree synchronises the whole device, so a host that
// finalises dose maps while transport keeps running on another stream stalls,
// and a process whose caching allocator already holds the free HBM may not be
// able to allocate at all.  gg_compute_dose_no_alloc writes into this fixed
// array instead.  It is created with the library's device code on every GPU
// that loads the library and is held until the process exits:
// 2 x GG_NO_ALLOC_MAX_DOSELS floats (16 MiB).  In host code g_dose_scratch is
// only the symbol handed to cudaGetSymbolAddress, never a device address.
namespace {

static __device__ __align__(256) float g_dose_scratch[2 * GG_NO_ALLOC_MAX_DOSELS];

constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_mutex;
float* g_scratch_address[kMaxScratchDevices] = {};

// Looks the array's device address up once per device, with that device
// current (the caller has made it current).
int scratch_for_device(int device, float** out) {
  if (device < 0 || device >= kMaxScratchDevices) return fail(GG_ERROR_INVALID_ARGUMENT, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_address[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dose_scratch);
    if (e != cudaSuccess || !p)
      return fail(GG_ERROR_CUDA, std::string("cudaGetSymbolAddress(dose scratch): ") + cudaGetErrorString(e));
    g_scratch_address[device] = static_cast<float*>(p);
  }
  *out = g_scratch_address[device];
  return GG_OK;
}

}  // namespace

extern "C" {

GG_API int gg_compute_dose_no_alloc(gg_context* c, int32_t dose_map, int32_t solid, float scale_factor,
                                    int32_t is_water_reference, float minimum_density, float* dose,
                                    float* uncertainty) {
  if (!c || !c->scene_ready || !dose) return fail(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  if (dose_map < 0 || dose_map >= static_cast<int>(c->dose_host.size()) || solid < 0 ||
      solid >= static_cast<int>(c->solid_host.size()) ||
      (c->solid_host[solid].type != GG_SOLID_VOXELIZED && c->solid_host[solid].type != GG_SOLID_MESHED))
    return fail(GG_ERROR_INVALID_ARGUMENT, "dose map or solid out of range");
  const size_t n = static_cast<size_t>(c->dose_host[dose_map].total_number_of_dosels);
  if (n > static_cast<size_t>(GG_NO_ALLOC_MAX_DOSELS))
    return fail(GG_ERROR_INVALID_ARGUMENT, "dose map has " + std::to_string(n) +
                                               " dosels; gg_compute_dose_no_alloc handles at most " +
                                               std::to_string(GG_NO_ALLOC_MAX_DOSELS) + " (use gg_compute_dose)");
  GG_CUDA(cudaSetDevice(c->device));
  float* scratch = nullptr;
  if (int rc = scratch_for_device(c->device, &scratch)) return rc;
  const gg_solid& s = c->solid_host[solid];
  gg::DoseParams P{};
  P.map = c->dose_host[dose_map];
  std::memcpy(P.number_of_voxels, s.number_of_voxels, sizeof(P.number_of_voxels));
  std::memcpy(P.voxel_sizes, s.voxel_sizes, sizeof(P.voxel_sizes));
  std::memcpy(P.border_min, s.obb.border_min, sizeof(P.border_min));
  P.labels = s.labels;
  P.density = c->density_dev[s.navigator];
  P.scale_factor = scale_factor;
  P.is_water_reference = is_water_reference;
  P.minimum_density = minimum_density;
  // The kernel writes every one of the n dose (and uncertainty) entries, so
  // nothing left in the array by an earlier call is read back.
  P.dose = scratch;
  P.uncertainty = uncertainty ? scratch + GG_NO_ALLOC_MAX_DOSELS : nullptr;
  gg::launch_compute_dose(P, c->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(dose, P.dose, n * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess && uncertainty)
    e = cudaMemcpyAsync(uncertainty, P.uncertainty, n * 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(GG_ERROR_CUDA, std::string("compute dose (no alloc): ") + cudaGetErrorString(e));
  return GG_OK;
}

}  // extern "C"
