// Photon transport kernels for sm_100a.
//
// One persistent kernel runs the whole GGEMS photon loop for every history:
// primary generation (X-ray cone or voxelized source), FindSolid /
// ProjectToSolid over all solids, and the per-step tracking through the
// current solid (voxelized phantom or CT detector box), with Compton,
// photoelectric and Rayleigh sampling from GGEMS's tables and the dose /
// histogram tallies.  It replaces the reference's host loop of
// 2*S+2 launches per iteration (src/global/GGEMS.cc:303-363,
// src/navigators/GGEMSNavigator.cc:320-530) and its is_alive round trip.
//
// Design:
//  * each lane owns one random slot (JKISS state in registers) and runs that
//    slot's histories in batch order, so every history draws exactly the
//    random numbers the reference's slot would; lanes fetch slots from a
//    device work counter;
//  * a lane advances one "step" per loop iteration (a voxel step, a box step,
//    or a FindSolid/ProjectToSolid round), and starts its next history as
//    soon as one ends, so lanes never idle while others finish long histories;
//  * the per-navigator cross-section tables (float4 per material and energy
//    bin), energy bins and photon cuts are staged into shared memory with
//    cp.async.bulk completing on an mbarrier (bounded wait);
//  * tallies: int32 histogram counts, int64 fixed-point energy deposits
//    (order independent), double energy^2.
//
// Arithmetic follows the reference operation by operation in float (double
// where it uses double) and the file is compiled with -fmad=false so that no
// multiply-add is contracted; the CPU oracle does the same.
#include <cfloat>
#include <cstdint>
#include <type_traits>

#include "gg_internal.cuh"

namespace gg {
namespace {

constexpr float kTwoPi = 6.283185307179586f;             // GGEMSConstants.hh:39
constexpr float kElectronMassC2 = 0.510998910f;           // GGEMSConstants.hh:52
constexpr float kTolerance = 5.0e-04f;                    // GGEMSGeometryConstants.hh:39
constexpr float kEps6 = 1.0e-06f;                         // GGEMSGeometryConstants.hh:38
constexpr float kOutOfWorld = FLT_MAX;                    // GGEMSParticleConstants.hh:44
constexpr int kNoProcess = 99;
constexpr float kRayleighFactor = 32526509815670243328.0f;  // GGEMSRayleighScatteringModels.hh:36
// KissUniform's (float)((double)x / 4294967295.0 * (1 - 2^-23)) equals, for
// every float x = (float)(uint32), the single-precision fused multiply-add
// fma(x, kKissCorrection, x * 2^-32): x * 2^-32 is exact and
// x * kKissCorrection + x * 2^-32 = x * 2^-32 * (1 - 2^-23 + 2^-32) is rounded
// once, which lands on the same float as the reference's double arithmetic for
// all 83,886,080 such x (checked exhaustively in tests/test_rng.py, against
// the division and against the double product).
constexpr float kKissTwoToMinus32 = 0x1p-32f;
constexpr float kKissCorrection = -0x1.ffp-56f;  // -(2^-23 - 2^-32) * 2^-32, exact in float

enum Phase : int { kNewHistory = 0, kFind = 1, kTrackVoxel = 2, kTrackBox = 3, kTrackMesh = 4, kInteract = 5, kDone = 6 };

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 divv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
__device__ __forceinline__ V3 scale(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 normalize3(V3 v) { return scale(v, 1.0f / sqrtf(dot3(v, v))); }

// GGfloat44 (row-major) products, GGEMSMatrixOperations.hh:46-125.
__device__ __forceinline__ V3 m_point(const float* m, V3 p) {
  return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3] * 1.0f, m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7] * 1.0f,
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11] * 1.0f);
}
__device__ __forceinline__ V3 m33(const float* m, V3 p) {
  return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z, m[4] * p.x + m[5] * p.y + m[6] * p.z, m[8] * p.x + m[9] * p.y + m[10] * p.z);
}
__device__ __forceinline__ V3 m33t(const float* m, V3 p) {
  return v3(m[0] * p.x + m[4] * p.y + m[8] * p.z, m[1] * p.x + m[5] * p.y + m[9] * p.z, m[2] * p.x + m[6] * p.y + m[10] * p.z);
}
// GGEMSReferentialTransformation.hh:80-141
__device__ __forceinline__ V3 g2l_pos(const float* m, V3 p) { return m33t(m, v3(p.x - m[3], p.y - m[7], p.z - m[11])); }
__device__ __forceinline__ V3 l2g_pos(const float* m, V3 p) { return m_point(m, p); }
__device__ __forceinline__ V3 g2l_dir(const float* m, V3 d) { return normalize3(m33t(m, d)); }
__device__ __forceinline__ V3 l2g_dir(const float* m, V3 d) { return normalize3(m33(m, d)); }

// RotateUnitZ, GGEMSReferentialTransformation.hh:44-70
__device__ __forceinline__ V3 rotate_uz(V3 v, V3 u) {
  float up = u.x * u.x + u.y * u.y;
  if (up > 0) {
    up = sqrtf(up);
    float px = v.x, py = v.y, pz = v.z;
    v.x = (u.x * u.z * px - u.y * py) / up + u.x * pz;
    v.y = (u.y * u.z * px + u.x * py) / up + u.y * pz;
    v.z = -up * px + u.z * pz;
  } else if (u.z < 0.0f) {
    v.x = -v.x;
    v.z = -v.z;
  }
  return v;
}

// BinarySearch / LinearInterpolation, GGEMSMathAlgorithms.hh:46-86
__device__ __forceinline__ int binary_search(float key, const float* a, int size) {
  int low = 0, high = size - 1;
  while (high - low > 1) {
    int mid = (high + low) / 2;
    float v = a[mid];
    if (v == key) return mid;
    if (v < key) low = mid;
    else high = mid;
  }
  return low;
}
__device__ __forceinline__ float lerp_ref(float xa, float ya, float xb, float yb, float x) {
  if (xa > xb) return yb;
  if (xa >= x) return ya;
  if (xb <= x) return yb;
  return ya + (x - xa) * (yb - ya) / (xb - xa);
}

// Ray tracing, GGEMSRayTracing.hh:60-326
__device__ __forceinline__ float safety_in(float p, float mn, float mx) {
  float a = fabsf(p - mn), b = fabsf(p - mx);
  p = (a < kTolerance) ? mn + kTolerance : p;
  return (b < kTolerance) ? mx - kTolerance : p;
}
__device__ __forceinline__ float safety_out(float p, float mn, float mx) {
  float a = fabsf(p - mn), b = fabsf(p - mx);
  p = (a < kTolerance) ? mn - kTolerance : p;
  return (b < kTolerance) ? mx + kTolerance : p;
}
__device__ __forceinline__ V3 safety_inside(V3 p, V3 mn, V3 mx) {
  return v3(safety_in(p.x, mn.x, mx.x), safety_in(p.y, mn.y, mx.y), safety_in(p.z, mn.z, mx.z));
}
__device__ __forceinline__ V3 safety_outside(V3 p, V3 mn, V3 mx) {
  return v3(safety_out(p.x, mn.x, mx.x), safety_out(p.y, mn.y, mx.y), safety_out(p.z, mn.z, mx.z));
}
__device__ __forceinline__ bool in_aabb(V3 p, V3 mn, V3 mx) {
  if (p.x < (mn.x + kTolerance) || p.x > (mx.x - kTolerance)) return false;
  if (p.y < (mn.y + kTolerance) || p.y > (mx.y - kTolerance)) return false;
  if (p.z < (mn.z + kTolerance) || p.z > (mx.z - kTolerance)) return false;
  return true;
}
// inv holds 1.0f / d per axis (used only where |d| >= 1e-6, as the reference
// computes it there), so a direction's reciprocals can be computed once.
__device__ __forceinline__ float distance_to_aabb(V3 p, V3 d, V3 inv, V3 mn, V3 mx) {
  float tmin = FLT_MIN, tmax = FLT_MAX;
  if (fabsf(d.x) < kEps6) {
    if (p.x < mn.x || p.x > mx.x) return kOutOfWorld;
  } else {
    float id = inv.x;
    tmin = (mn.x - p.x) * id;
    tmax = (mx.x - p.x) * id;
    if (tmin > tmax) {
      float t = tmin;
      tmin = tmax;
      tmax = t;
    }
  }
  if (fabsf(d.y) < kEps6) {
    if (p.y < mn.y || p.y > mx.y) return kOutOfWorld;
  } else {
    float id = inv.y;
    float lo = (mn.y - p.y) * id, hi = (mx.y - p.y) * id;
    if (lo > hi) {
      float t = lo;
      lo = hi;
      hi = t;
    }
    if (lo > tmin) tmin = lo;
    if (hi < tmax) tmax = hi;
    if (tmin > tmax) return kOutOfWorld;
  }
  if (fabsf(d.z) < kEps6) {
    if (p.z < mn.z || p.z > mx.z) return kOutOfWorld;
  } else {
    float id = inv.z;
    float lo = (mn.z - p.z) * id, hi = (mx.z - p.z) * id;
    if (lo > hi) {
      float t = lo;
      lo = hi;
      hi = t;
    }
    if (lo > tmin) tmin = lo;
    if (hi < tmax) tmax = hi;
    if (tmin > tmax) return kOutOfWorld;
  }
  if (tmin < 0.0f && (tmax < 0.0f || tmax == 0.0f)) return kOutOfWorld;
  if (static_cast<double>(tmax - tmin) < (2.0 * static_cast<double>(kTolerance))) return kOutOfWorld;
  if (tmin <= kEps6) return tmax;
  return tmin;
}

__device__ __forceinline__ V3 reciprocal(V3 d) { return v3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z); }
__device__ __forceinline__ float distance_to_aabb(V3 p, V3 d, V3 mn, V3 mx) {
  return distance_to_aabb(p, d, reciprocal(d), mn, mx);
}

// JKISS32, GGEMSKissEngine.hh:50-75
struct Kiss {
  uint32_t s1, s2, s3, s4, s5;
  __device__ __forceinline__ float uniform() {
    s2 ^= (s2 << 5);
    s2 ^= (s2 >> 7);
    s2 ^= (s2 << 22);
    int t = static_cast<int>(s3 + s4 + s5);
    s3 = s4;
    s5 = t < 0;
    s4 = static_cast<uint32_t>(t) & 2147483647u;
    s1 += 1411392427u;
    const float x = __uint2float_rn(s1 + s2 + s4);
    return __fmaf_rn(x, kKissCorrection, x * kKissTwoToMinus32);
  }
};

struct Photon {
  V3 p, d;          // global outside solids, local while tracking inside one
  float E;
  float psd;        // particle_solid_distance_
  int solid_id;
  int8_t status;
  int8_t scatter;
};

// Tables (shared memory when they fit, otherwise the HBM blob).
struct Tab {
  const unsigned char* base;
  const DevNavigator* nav;
  __device__ __forceinline__ const float* energy_bins(int n) const {
    return reinterpret_cast<const float*>(base + nav[n].energy_bins_offset);
  }
  __device__ __forceinline__ const float4* sigma(int n) const {
    return reinterpret_cast<const float4*>(base + nav[n].sigma_offset);
  }
  __device__ __forceinline__ const float* photon_cut(int n) const {
    return reinterpret_cast<const float*>(base + nav[n].photon_cut_offset);
  }
  // TLE tables: GG_ATTENUATION_BINS energies followed by mu_en per material
  __device__ __forceinline__ const float* attenuation(int n) const {
    return reinterpret_cast<const float*>(base + nav[n].attenuation_offset);
  }
};

__device__ __forceinline__ float pick(float4 s, int pid) { return pid == 0 ? s.x : (pid == 1 ? s.y : s.z); }

// GetPhotonNextInteraction, GGEMSPhotonNavigator.hh:57-93.  Returns the
// distance, writes the process; energy_id is the cached BinarySearch result,
// process_pack the navigator's process count and ids (DevNavigator).
__device__ __forceinline__ float next_interaction(Kiss& rng, int number_of_bins, uint32_t process_pack,
                                                  const float4* sig, int energy_id, int material, int& proc) {
  float4 s = sig[material * number_of_bins + energy_id];
  float nid = kOutOfWorld;
  proc = kNoProcess;
  const int n = static_cast<int>(process_pack & 0xffu);
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (i >= n) break;
    const int pid = static_cast<int>((process_pack >> (8 * (i + 1))) & 0xffu);
    float dist = -logf(rng.uniform()) / pick(s, pid);
    if (dist < nid) {
      nid = dist;
      proc = pid;
    }
  }
  return nid;
}

// 16-byte shared-memory (or global) loads of a struct's leading fields.
__device__ __forceinline__ float4 load4f(const void* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ int4 load4i(const void* p) { return *reinterpret_cast<const int4*>(p); }

// State handed to and returned by the (out-of-line) interaction samplers.
// Passed by value so that the photon and its random state stay in registers
// in the transport loop (a reference would force them into local memory).
struct Interaction {
  float E;
  V3 d;
  Kiss rng;
  int dead;
};

// KleinNishinaComptonSampleSecondaries, GGEMSComptonScatteringModels.hh:47-132
__device__ __noinline__ Interaction compton(Interaction in) {
  Kiss rng = in.rng;
  float E0 = in.E;
  float E0m = E0 / kElectronMassC2;
  V3 gd = in.d;
  float eps0 = 1.0f / (1.0f + 2.0f * E0m);
  float eps0sq = eps0 * eps0;
  float alpha1 = -logf(eps0);
  float alpha2 = alpha1 + 0.5f * (1.0f - eps0sq);
  float eps, epssq, onecost, sint2, greject, r3;
  int nloop = 0;
  do {
    ++nloop;
    if (nloop > 1000) {
      in.rng = rng;
      return in;
    }
    float r1 = rng.uniform();
    float r2 = rng.uniform();
    r3 = rng.uniform();
    if (alpha1 > alpha2 * r1) {
      eps = expf(-alpha1 * r2);
      epssq = eps * eps;
    } else {
      epssq = eps0sq + (1.0f - eps0sq) * r2;
      eps = sqrtf(epssq);
    }
    onecost = (1.0f - eps) / (eps * E0m);
    sint2 = onecost * (2.0f - onecost);
    greject = 1.0f - eps * sint2 / (1.0f + epssq);
  } while (greject < r3);
  if (sint2 < 0.0f) sint2 = 0.0f;
  float cost = 1.0f - onecost;
  float sint = sqrtf(sint2);
  float phi = rng.uniform() * kTwoPi;
  V3 g = v3(sint * cosf(phi), sint * sinf(phi), cost);
  g = normalize3(rotate_uz(g, gd));
  in.E = E0 * eps;
  in.d = g;
  in.rng = rng;
  return in;
}

__constant__ float c_rayleigh_pp[9][101];

__device__ __forceinline__ float rayleigh_w(float x, float n) {
  return (x < 0.02f) ? n * x * (1.0f - 0.5f * (n - 1.0f) * x * (1.0f - (n - 2.0f) * x / 3.0f))
                     : 1.0f - expf(-n * logf(1.0f + x));
}

// LivermoreRayleighSampleSecondaries, GGEMSRayleighScatteringModels.hh:169-316
__device__ __noinline__ Interaction rayleigh(Interaction in, const DevNavigator& nv, const float* ebins,
                                             const float4* sig, int material, int energy_id) {
  float E0 = in.E;
  if (E0 <= 250.0e-6f) {
    in.dead = 1;
    return in;
  }
  Kiss rng = in.rng;
  V3 gd = in.d;
  const int nb = nv.number_of_bins;
  int n_minus_one = static_cast<int8_t>(nv.number_of_elements[material] - 1);
  int mixture = nv.element_offset[material];
  int z = nv.atomic_number[mixture + n_minus_one];
  if (n_minus_one > 0) {
    float kcs = lerp_ref(ebins[energy_id], sig[material * nb + energy_id].z, ebins[energy_id + 1],
                         sig[material * nb + energy_id + 1].z, E0);
    float x = rng.uniform() * kcs;
    float cs = 0.0f;
    for (int i = 0; i < n_minus_one; ++i) {
      int zi = nv.atomic_number[mixture + i];
      const float* pa = nv.rayleigh_per_atom + nb * zi;
      cs += nv.atomic_number_density[mixture + i] *
            lerp_ref(ebins[energy_id], pa[energy_id], ebins[energy_id + 1], pa[energy_id + 1], E0);
      if (x < cs) {
        z = zi;
        break;
      }
    }
  }
  float xx = kRayleighFactor * E0 * E0;
  float n0 = c_rayleigh_pp[6][z] - 1.0f, n1 = c_rayleigh_pp[7][z] - 1.0f, n2 = c_rayleigh_pp[8][z] - 1.0f;
  float b0 = c_rayleigh_pp[3][z], b1 = c_rayleigh_pp[4][z], b2 = c_rayleigh_pp[5][z];
  float w0 = rayleigh_w(2.0f * xx * b0, n0);
  float w1 = rayleigh_w(2.0f * xx * b1, n1);
  float w2 = rayleigh_w(2.0f * xx * b2, n2);
  float x0 = w0 * c_rayleigh_pp[0][z] / (b0 * n0);
  float x1 = w1 * c_rayleigh_pp[1][z] / (b1 * n1);
  float x2 = w2 * c_rayleigh_pp[2][z] / (b2 * n2);
  float cost;
  do {
    float w = w0, n = n0, b = b0;
    float x = rng.uniform() * (x0 + x1 + x2);
    if (x > x0) {
      x -= x0;
      if (x <= x1) {
        w = w1; n = n1; b = b1;
      } else {
        w = w2; n = n2; b = b2;
      }
    }
    n = 1.0f / n;
    float y = rng.uniform() * w;
    if (y < 0.02f) x = y * n * (1.0f + 0.5f * (n + 1.0f) * y * (1.0f - (n + 2.0f) * y / 3.0f));
    else x = expf(-n * logf(1.0f - y)) - 1.0f;
    cost = 1.0f - x / (b * xx);
  } while (2.0f * rng.uniform() > 1.0f + cost * cost || cost < -1.0f);
  float phi = kTwoPi * rng.uniform();
  float sint = sqrtf((1.0f - cost) * (1.0f + cost));
  V3 g = v3(sint * cosf(phi), sint * sinf(phi), cost);
  in.d = normalize3(rotate_uz(g, gd));
  in.rng = rng;
  return in;
}

// Compton or Rayleigh interaction of the photon (proc is one of the two).
__device__ __forceinline__ void scatter(Photon& ph, Kiss& rng, int proc, const DevNavigator& nv, const float* ebins,
                                        const float4* sig, int material, int energy_id) {
  Interaction in{ph.E, ph.d, rng, 0};
  in = proc == GG_COMPTON_SCATTERING ? compton(in) : rayleigh(in, nv, ebins, sig, material, energy_id);
  ph.E = in.E;
  ph.d = in.d;
  rng = in.rng;
  if (in.dead) ph.status = GG_DEAD;
}

// dose_record_standard / dose_photon_tracking, GGEMSDoseRecording.hh:65-118
__device__ __forceinline__ int dosel(const DevDoseMap& dm, V3 p) {
  if (p.x < dm.border_min[0] + kEps6 || p.x > dm.border_max[0] - kEps6) return -1;
  if (p.y < dm.border_min[1] + kEps6 || p.y > dm.border_max[1] - kEps6) return -1;
  if (p.z < dm.border_min[2] + kEps6 || p.z > dm.border_max[2] - kEps6) return -1;
  int ix = __float2int_rz((p.x - dm.border_min[0]) * dm.inv_size_of_dosels[0]);
  int iy = __float2int_rz((p.y - dm.border_min[1]) * dm.inv_size_of_dosels[1]);
  int iz = __float2int_rz((p.z - dm.border_min[2]) * dm.inv_size_of_dosels[2]);
  if (ix < 0 || ix >= dm.number_of_dosels[0]) return -1;
  if (iy < 0 || iy >= dm.number_of_dosels[1]) return -1;
  if (iz < 0 || iz >= dm.number_of_dosels[2]) return -1;
  return ix + iy * dm.number_of_dosels[0] + iz * dm.number_of_dosels[0] * dm.number_of_dosels[1];
}
__device__ __forceinline__ void dose_record(const DevDoseMap& dm, float edep, V3 p) {
  int id = dosel(dm, p);
  if (id < 0) return;
  if (dm.hit) atomicAdd(dm.hit + id, 1);
  long long q = __double2ll_rn(static_cast<double>(edep) * kEdepScale);
  atomicAdd(dm.edep + id, static_cast<unsigned long long>(q));
  if (dm.edep_squared) atomicAdd(dm.edep_squared + id, static_cast<double>(edep) * static_cast<double>(edep));
}

// get_primaries_ggems_xray_source, GetPrimariesGGEMSXRaySource.cl:52-143
__device__ void xray_primary(Photon& ph, Kiss& rng, const DevSource& s, double new_aperture) {
  double phi = rng.uniform();
  double theta = rng.uniform();
  phi *= static_cast<double>(kTwoPi);
  theta = acos(1.0 - new_aperture * theta);
  double st = sin(theta);
  V3 rot = v3(static_cast<float>(cos(phi) * st), static_cast<float>(sin(phi) * st), static_cast<float>(cos(theta)));
  V3 gp = l2g_pos(s.matrix, v3(0.0f, 0.0f, 0.0f));
  V3 dir = normalize3(sub(v3(0.0f, 0.0f, 0.0f), gp));
  dir = normalize3(rotate_uz(rot, dir));
  gp.x = s.focal_spot_size[0] * (rng.uniform() - 0.5f);
  gp.y = s.focal_spot_size[1] * (rng.uniform() - 0.5f);
  gp.z = s.focal_spot_size[2] * (rng.uniform() - 0.5f);
  gp = l2g_pos(s.matrix, gp);
  int index = 0;
  float rnd = 0.0f;
  if (s.number_of_energy_bins != 1) {
    rnd = rng.uniform();
    index = binary_search(rnd, s.energy_cdf, s.number_of_energy_bins + 1);
  }
  ph.E = !s.is_interp ? s.energy_spectrum[index]
                      : lerp_ref(s.energy_cdf[index], s.energy_spectrum[index], s.energy_cdf[index + 1],
                                 s.energy_spectrum[index + 1], rnd);
  ph.p = gp;
  ph.d = dir;
}

// get_primaries_ggems_voxelized_source, GetPrimariesGGEMSVoxelizedSource.cl:57-150
__device__ void voxelized_primary(Photon& ph, Kiss& rng, const DevSource& s) {
  double phi = rng.uniform();
  double theta = rng.uniform();
  phi *= static_cast<double>(kTwoPi);
  theta = acos(1.0 - 2.0 * theta);
  double st = sin(theta);
  V3 dir = v3(static_cast<float>(cos(phi) * st), static_cast<float>(sin(phi) * st), static_cast<float>(cos(theta)));
  float rnd_act = rng.uniform();
  int ia = binary_search(rnd_act, s.activity_cdf, s.number_of_activity_bins);
  int vox = s.activity_index[ia];
  int nx = s.number_of_voxels[0], slice = nx * s.number_of_voxels[1];
  int iz = vox / slice;
  int ix = (vox - iz * slice) % nx;
  int iy = (vox - iz * slice) / nx;
  V3 bmin = v3(s.border_min[0], s.border_min[1], s.border_min[2]);
  V3 vs = v3(s.voxel_sizes[0], s.voxel_sizes[1], s.voxel_sizes[2]);
  V3 vmin = add(bmin, mul(v3(static_cast<float>(ix), static_cast<float>(iy), static_cast<float>(iz)), vs));
  V3 vmax = add(vmin, vs);
  V3 p;
  p.x = bmin.x + (static_cast<float>(ix) + rng.uniform()) * vs.x;
  p.y = bmin.y + (static_cast<float>(iy) + rng.uniform()) * vs.y;
  p.z = bmin.z + (static_cast<float>(iz) + rng.uniform()) * vs.z;
  p = safety_inside(p, vmin, vmax);
  ph.p = l2g_pos(s.matrix, p);
  int index = 0;
  float rnd = 0.0f;
  if (s.number_of_energy_bins != 1) {
    rnd = rng.uniform();
    index = binary_search(rnd, s.energy_cdf, s.number_of_energy_bins + 1);
  }
  ph.E = !s.is_interp ? s.energy_spectrum[index]
                      : lerp_ref(s.energy_cdf[index], s.energy_spectrum[index], s.energy_cdf[index + 1],
                                 s.energy_spectrum[index + 1], rnd);
  ph.d = dir;
}

// Track-length-estimator deposit of one voxel step
// (TrackThroughGGEMSVoxelizedSolid.cl:286-301): E * mu_en(E, material) * step
// (mm -> cm), with mu_en interpolated in the 220-bin attenuation table.
// A new primary out of line (it runs once per history, in the warp's rare
// round): keeps its FP64 cone sampling out of the tracking loop's
// instruction footprint; state in and out by value, so nothing goes to the
// stack.  Measured +0.8 % on the CBCT projection.
struct PrimaryOut {
  V3 p, d;
  float E;
  Kiss rng;
};
__device__ __noinline__ PrimaryOut new_primary(Kiss rng, const DevSource& s) {
  Photon ph{};
  if (s.type == GG_SOURCE_XRAY) xray_primary(ph, rng, s, s.new_aperture);
  else voxelized_primary(ph, rng, s);
  return PrimaryOut{ph.p, ph.d, ph.E, rng};
}

__device__ __forceinline__ float tle_edep(const float* att, int material, float energy, float step) {
  const float* me = att + GG_ATTENUATION_BINS * (1 + material);
  int e_index = binary_search(energy, att, GG_ATTENUATION_BINS);
  float mu_en = e_index == 0 ? me[0] : lerp_ref(att[e_index - 1], me[e_index - 1], att[e_index], me[e_index], energy);
  return energy * mu_en * step * 0.1f;
}

// ---- meshed solid (TrackThroughGGEMSMeshSolid.cl) ----
constexpr int kMaxMeshCrossings = 16;  // MAX_TRIANGLE_INTERACTION

struct MeshCrossings {
  V3 first, second;  // nearest and second nearest crossing
  int count;
};

__device__ __forceinline__ V3 cross3(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

// GetMeshIOPositions (l.249-318): every octree node that owns triangles, in
// node order, is slab-tested (TestLineNode, l.182-230, with the direction's
// reciprocals) and its triangles are intersected with the Moller-Trumbore test
// (l.121-170).  GGEMS keeps up to 16 crossings sorted by squared distance (a
// new crossing goes after equal ones) but only reads the first two, so only
// those two are kept here, with the same ordering rule; the search ends at 16
// crossings (GGEMS writes past its array beyond that).
// Moller-Trumbore test of triangle k (l.121-170) and GGEMS's crossing
// ordering: a new crossing goes before the kept ones only when strictly
// nearer (squared distance, l.276-303).  Returns true once 16 crossings were
// counted.
struct CrossingState {
  float d0, d1;
  bool have0, have1;
};
__device__ __forceinline__ bool add_crossing(V3 p, V3 d, const float4* tris, int k, MeshCrossings& out, CrossingState& c) {
  const float4 t0 = __ldg(tris + 3 * k), t1 = __ldg(tris + 3 * k + 1), t2 = __ldg(tris + 3 * k + 2);
  const V3 p0 = v3(t0.x, t0.y, t0.z), e1 = v3(t0.w, t1.x, t1.y), e2 = v3(t1.z, t1.w, t2.x);
  const V3 h = cross3(d, e2);
  const float det = dot3(e1, h);
  if (det > -kEps6 && det < kEps6) return false;
  const float f = 1.0f / det;
  const V3 sv = sub(p, p0);
  const float u = f * dot3(sv, h);
  if (u < 0.0f || u > 1.0f) return false;
  const V3 q = cross3(sv, e1);
  const float v = f * dot3(q, d);
  if (v < 0.0f || u + v > 1.0f) return false;
  const float t = f * dot3(q, e2);
  if (!(t > kEps6)) return false;
  const V3 x = v3(p.x + d.x * t, p.y + d.y * t, p.z + d.z * t);
  const float dx = x.x - p.x, dy = x.y - p.y, dz = x.z - p.z;
  const float d2 = dx * dx + dy * dy + dz * dz;
  if (!c.have0 || d2 < c.d0) {
    if (c.have0) {
      out.second = out.first;
      c.d1 = c.d0;
      c.have1 = true;
    }
    out.first = x;
    c.d0 = d2;
    c.have0 = true;
  } else if (!c.have1 || d2 < c.d1) {
    out.second = x;
    c.d1 = d2;
    c.have1 = true;
  }
  return ++out.count == kMaxMeshCrossings;
}

// Slab test of the ray [0, inf) against a box (TestLineNode, l.182-230).
__device__ __forceinline__ bool ray_hits_box(const float pos[3], const float dir[3], const float ood[3],
                                             const float mn[3], const float mx[3]) {
  float tmin = 0.0f, tmax = FLT_MAX;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (fabsf(dir[i]) < kEps6) {
      if (pos[i] < mn[i] || pos[i] > mx[i]) return false;
    } else {
      float t1 = (mn[i] - pos[i]) * ood[i], t2 = (mx[i] - pos[i]) * ood[i];
      if (t1 > t2) {
        float t = t2;
        t2 = t1;
        t1 = t;
      }
      if (t1 > tmin) tmin = t1;
      if (t2 < tmax) tmax = t2;
      if (tmin > tmax) return false;
    }
  }
  return true;
}

// GetMeshIOPositions (l.249-318).  GGEMS keeps up to 16 crossings sorted by
// squared distance but only reads the first two and the count (whose parity
// says inside / outside), so only those are kept here, with the same ordering
// rule; the search ends at 16 crossings (GGEMS writes past its array beyond
// that).  Octree form: every node that owns triangles, in node order, is
// slab-tested and its triangles intersected, exactly GGEMS's scan.  BVH form
// (large meshes): the hierarchy is walked with a stack; each triangle test is
// the same arithmetic, so the crossings found are the same set and only their
// discovery order (hence exact ties) can differ from the scan's.
__device__ __noinline__ MeshCrossings mesh_crossings(V3 p, V3 d, V3 inv, const float4* nodes, int node_count,
                                                     const float4* tris, int bvh) {
  MeshCrossings out;
  out.count = 0;
  out.first = out.second = p;
  CrossingState c{FLT_MAX, FLT_MAX, false, false};
  const float dir[3] = {d.x, d.y, d.z}, pos[3] = {p.x, p.y, p.z}, ood[3] = {inv.x, inv.y, inv.z};
  if (!bvh) {
    for (int n = 0; n < node_count; ++n) {
      const float4 a = __ldg(nodes + 2 * n), b = __ldg(nodes + 2 * n + 1);
      const float mn[3] = {a.x, a.y, a.z}, mx[3] = {a.w, b.x, b.y};
      if (!ray_hits_box(pos, dir, ood, mn, mx)) continue;
      const int first = __float_as_int(b.z), count = __float_as_int(b.w);
      for (int k = first; k < first + count; ++k)
        if (add_crossing(p, d, tris, k, out, c)) return out;
    }
    return out;
  }
  constexpr int kStack = 64;
  int stack[kStack];
  int sp = 0, node = 0;
  for (;;) {
    const float4 a = __ldg(nodes + 2 * node), b = __ldg(nodes + 2 * node + 1);
    const float mn[3] = {a.x, a.y, a.z}, mx[3] = {a.w, b.x, b.y};
    if (ray_hits_box(pos, dir, ood, mn, mx)) {
      const int first = __float_as_int(b.z), count = __float_as_int(b.w);
      if (count > 0) {
        for (int k = first; k < first + count; ++k)
          if (add_crossing(p, d, tris, k, out, c)) return out;
      } else if (sp < kStack) {
        stack[sp++] = first + 1;
        node = first;
        continue;
      }
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
  return out;
}

// world_tracking (WorldTracking.cl:54-162): the flight from the photon's
// position to the solid FindSolid chose (10 m when none) sampled in steps of
// the world element size along the dominant axis.
__device__ __noinline__ void world_track(V3 p1, V3 dir, float E, float psd, const TransportParams& P) {
  float distance = psd == kOutOfWorld ? 10000.0f : psd;
  if (distance <= kTolerance) return;
  const V3 size = v3(P.world_sizes[0], P.world_sizes[1], P.world_sizes[2]);
  const int nx = P.world_dimensions[0], ny = P.world_dimensions[1], nz = P.world_dimensions[2];
  const V3 p2 = add(p1, scale(dir, distance));
  const V3 lo = v3(size.x * static_cast<float>(nx) * -0.5f, size.y * static_cast<float>(ny) * -0.5f,
                   size.z * static_cast<float>(nz) * -0.5f);
  V3 q = divv(sub(p1, lo), size);
  int ix = __float2int_rz(q.x), iy = __float2int_rz(q.y), iz = __float2int_rz(q.z);
  const V3 diff = sub(p2, p1);
  float length = fabsf(diff.x), main_size = size.x;
  if (fabsf(diff.y) > length) {
    length = fabsf(diff.y);
    main_size = size.y;
  } else if (fabsf(diff.z) > length) {
    length = fabsf(diff.z);
    main_size = size.z;
  }
  const float inv_length = 1.0f / length;
  const V3 increment = v3(inv_length * diff.x, inv_length * diff.y, inv_length * diff.z);
  const int steps = static_cast<int>(1.0f + (length / main_size));
  const size_t cells = static_cast<size_t>(nx) * ny * nz;
  const long long e_fixed = __double2ll_rn(static_cast<double>(E) * kEdepScale);
  const long long m_fixed[3] = {__double2ll_rn(static_cast<double>(dir.x) * kEdepScale),
                                __double2ll_rn(static_cast<double>(dir.y) * kEdepScale),
                                __double2ll_rn(static_cast<double>(dir.z) * kEdepScale)};
  for (int i = 0; i < steps; ++i) {
    if (ix < 0 || ix >= nx || iy < 0 || iy >= ny || iz < 0 || iz >= nz) break;
    const size_t g = ix + static_cast<size_t>(iy) * nx + static_cast<size_t>(iz) * nx * ny;
    if (P.world_photon) atomicAdd(P.world_photon + g, 1);
    if (P.world_energy) atomicAdd(P.world_energy + g, static_cast<unsigned long long>(e_fixed));
    if (P.world_energy_squared) atomicAdd(P.world_energy_squared + g, static_cast<double>(E) * static_cast<double>(E));
    if (P.world_momentum)
      for (int a = 0; a < 3; ++a) atomicAdd(P.world_momentum + a * cells + g, static_cast<unsigned long long>(m_fixed[a]));
    p1 = add(p1, scale(increment, main_size));
    q = divv(sub(p1, lo), size);
    ix = __float2int_rz(q.x);
    iy = __float2int_rz(q.y);
    iz = __float2int_rz(q.z);
  }
}

// One point of the tracked slot's trajectory (gg_track_point).
__device__ __noinline__ void track_point(gg_track_point* points, int32_t* count, int capacity, int kind, int solid,
                                         int process, int history, V3 p, V3 d, float E) {
  const int i = atomicAdd(count, 1);
  if (i >= capacity) return;
  gg_track_point& t = points[i];
  t.kind = kind;
  t.solid = solid;
  t.process = process;
  t.history = history;
  t.E = E;
  t.position[0] = p.x;
  t.position[1] = p.y;
  t.position[2] = p.z;
  t.direction[0] = d.x;
  t.direction[1] = d.y;
  t.direction[2] = d.z;
  t.pad = 0.0f;
}

// Histogram of interaction sites in a CT detector module (the HISTOGRAM part of
// TrackThroughGGEMSSolidBox.cl:214-236), with the scatter histogram.
__device__ __forceinline__ void box_histogram(const DevSolid& so, const Photon& ph) {
  if (!so.histogram) return;
  V3 bmin = v3(so.border_min[0], so.border_min[1], so.border_min[2]);
  V3 es = divv(v3(so.box_size[0], so.box_size[1], so.box_size[2]),
               v3(static_cast<float>(so.virtual_element_number[0]), static_cast<float>(so.virtual_element_number[1]),
                  static_cast<float>(so.virtual_element_number[2])));
  V3 q = divv(sub(ph.p, bmin), es);
  int ix = __float2int_rz(q.x), iy = __float2int_rz(q.y);
  if (ix >= 0 && iy >= 0 && ix < so.virtual_element_number[0] && iy < so.virtual_element_number[1]) {
    int idx = ix + iy * so.virtual_element_number[0];
    atomicAdd(so.histogram + idx, 1);
    if (so.scatter_histogram && ph.scatter == 1) atomicAdd(so.scatter_histogram + idx, 1);
  }
}

// ---- shared-memory staging with bounded waits ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Copies `bytes` (multiple of 16) from HBM into shared memory with
// cp.async.bulk and waits on an mbarrier for at most 2^22 polls (far longer
// than a 15 KB copy takes).  Returns false (and sets *error) when the copy did
// not complete in time; the CTA then exits, possibly with the copy still in
// flight, so the run reports GG_ERROR_TIMEOUT and the context must be
// recreated (include/ggems_b200.h).  Extra wait code here, even out of line,
// changes the register allocation of the whole kernel (more spills).
__device__ bool stage_tables(unsigned char* dst, const unsigned char* src, uint32_t bytes, uint64_t* bar, int* error) {
  constexpr uint32_t kChunk = 16384;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    for (uint32_t off = 0; off < bytes; off += kChunk) {
      uint32_t n = bytes - off < kChunk ? bytes - off : kChunk;
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_u32(dst + off)),
          "l"(src + off), "r"(n), "r"(smem_u32(bar))
          : "memory");
    }
  }
  uint32_t done = 0;
  for (int i = 0; i < (1 << 22) && !done; ++i) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(smem_u32(bar))
        : "memory");
  }
  if (!done) atomicExch(error, 1);
  return __syncthreads_and(done) != 0;
}

extern __shared__ __align__(16) unsigned char g_smem[];

// Masks over a warp's stash records (one bit per record).
using StashMask = std::conditional_t<(kStashRecords > 32), unsigned long long, unsigned>;
__device__ __forceinline__ int stash_popc(unsigned m) { return __popc(m); }
__device__ __forceinline__ int stash_popc(unsigned long long m) { return __popcll(m); }
// 32-bit part h of a mask, and a 32-bit part placed at h
__device__ __forceinline__ unsigned stash_part(StashMask m, int h) {
  if constexpr (kStashRecords > 32) return static_cast<unsigned>(m >> (32 * h));
  else return m;
}
__device__ __forceinline__ StashMask stash_mask(unsigned part, int h) {
  if constexpr (kStashRecords > 32) return static_cast<StashMask>(part) << (32 * h);
  else return part;
}

// Register budget of a variant: what 256-thread blocks need to keep `blocks`
// of them resident per SM (64, 80 or 128 registers), fixed per kernel so that
// the block size stays a launch parameter (128, 256 or 512 threads).
constexpr int transport_registers(int blocks) { return (65536 / (kBlockThreads * blocks)) & ~7; }

// kFull: the scene has a meshed solid, a world grid or a tracked particle;
// kAux: the world walk and particle tracking are compiled in.  Scenes without
// them run variants compiled without that code, so its instructions and
// registers stay out of the voxel / detector (or mesh) hot loop.
// kDose: some solid tallies into a dose map.
// kBatch: several jobs (source runs) in one launch, each with its own solids.
// kStash: each warp keeps a second set of photons in shared memory and
// exchanges them with its lanes, so that lanes waiting for a rare phase track
// a parked photon meanwhile and rare rounds run on full warps.

template <bool kFull, bool kBatch, bool kDose, bool kAux, int kStash>
__global__ void __maxnreg__(transport_registers(kAux ? 2 : (kFull ? 3 : ((kBatch && kDose) || kStash == 2 ? 3 : 4))))
    transport_kernel(TransportParams P) {
  // shared memory: [tables][solids][navigators][mbarrier][stash]
  unsigned char* tables = g_smem;
  DevSolid* scene_solids = reinterpret_cast<DevSolid*>(g_smem + (P.tables_in_smem ? P.table_bytes : 0));
  DevNavigator* navs = reinterpret_cast<DevNavigator*>(scene_solids + P.number_of_solids);
  uint64_t* bar = reinterpret_cast<uint64_t*>(navs + P.number_of_navigators);
  for (int i = threadIdx.x; i < P.number_of_solids; i += blockDim.x) scene_solids[i] = P.solids[i];
  for (int i = threadIdx.x; i < P.number_of_navigators; i += blockDim.x) navs[i] = P.navigators[i];
  Tab tab{P.table_blob, navs};
  if (P.tables_in_smem) {
    if (!stage_tables(tables, P.table_blob, P.table_bytes, bar, P.error)) return;
    tab.base = tables;
  } else {
    __syncthreads();
  }

  const size_t S = GG_MAXIMUM_PARTICLES;
  // Solids of the lane's current job: the shared-memory copy for a single
  // run, the job's own array (global memory) in a batched launch.
  const DevSolid* solids = scene_solids;
  int job = 0;
  const int number_of_jobs = kBatch ? P.number_of_jobs : 1;

  Kiss rng{0, 0, 0, 0, 0};
  Photon ph{};
  ph.solid_id = -1;
  uint32_t slot = ~0u;
  uint32_t histories_left = 0;
  int rounds = 0;
  int phase = kDone;
  int energy_id = 0;
  float cached_E = -1.0f;
  int cached_nav = -1;
  int pending = 0;  // deferred interaction: process << 8 | material
  V3 inv_d = v3(0.0f, 0.0f, 0.0f);  // reciprocal(ph.d) while tracking inside a solid
  int history_number = -1;           // particle tracking: histories of the slot so far
  // particle tracking (full variant only): a point of this lane's photon when
  // its slot is the tracked one
  auto trk = [&](int kind, int solid, int process) {
    if (kAux && P.tracking_points && static_cast<int>(slot) == P.tracking_slot)
      track_point(P.tracking_points, P.tracking_count, P.tracking_capacity, kind, solid, process, history_number, ph.p,
                  ph.d, ph.E);
  };

  // A slot runs its histories of job 0, then of job 1, ... (each job is one
  // GGEMS source run; the slot's random stream carries over from run to run).
  // Returns false when the slot takes part in no job from `from` on.
  auto enter_job = [&](int from) -> bool {
    for (int j = from; j < number_of_jobs; ++j) {
      const DevJob& J = P.jobs[j];
      const uint32_t h = slot < J.q ? J.nb : (slot < J.q + 1 && J.r > 0 ? static_cast<uint32_t>(J.r) : 0u);
      if (h > 0) {
        if (kBatch) {
          job = j;
          solids = P.job_solids + static_cast<size_t>(j) * P.number_of_solids;
        }
        histories_left = h;
        ph.solid_id = -1;
        return true;
      }
    }
    return false;
  };
  // Grab the next slot: the lane takes slots_per_claim consecutive slots from
  // the work queue at a time and runs their photons one after another.  The
  // queue hands out runs starting at multiples of slots_per_claim (a power of
  // two), so the run is used up when the next slot is such a multiple (slot
  // starts at ~0u: the first call claims).
  auto next_slot = [&]() -> bool {
    if ((++slot & (P.slots_per_claim - 1)) == 0) slot = atomicAdd(P.slot_counter, P.slots_per_claim);
    if (slot >= P.number_of_slots) return false;
    rng = Kiss{P.rng[slot], P.rng[S + slot], P.rng[2 * S + slot], P.rng[3 * S + slot], P.rng[4 * S + slot]};
    return enter_job(0);
  };
  auto finish_slot = [&]() {
    P.rng[slot] = rng.s1;
    P.rng[S + slot] = rng.s2;
    P.rng[2 * S + slot] = rng.s3;
    P.rng[3 * S + slot] = rng.s4;
    P.rng[4 * S + slot] = rng.s5;
    if (P.particles.E) {
      P.particles.E[slot] = ph.E;
      P.particles.px[slot] = ph.p.x;
      P.particles.py[slot] = ph.p.y;
      P.particles.pz[slot] = ph.p.z;
      P.particles.dx[slot] = ph.d.x;
      P.particles.dy[slot] = ph.d.y;
      P.particles.dz[slot] = ph.d.z;
      P.particles.status[slot] = ph.status;
      P.particles.scatter[slot] = ph.scatter;
      P.particles.solid_id[slot] = ph.solid_id;
    }
  };

  auto end_history = [&]() {
    if (--histories_left > 0 || (kBatch && enter_job(job + 1))) {
      phase = kNewHistory;
    } else {
      finish_slot();
      phase = next_slot() ? kNewHistory : kDone;
    }
  };
  // End of track_through_*: back to the global frame; the history goes on
  // (FindSolid) unless the photon died.
  auto leave_solid = [&](const DevSolid& so, bool dead) {
    if (kFull && so.type == GG_SOLID_MESHED) {
      // A meshed solid tracks in world coordinates and, on leaving (dead or
      // not), carries the photon to its OBB boundary (TrackThroughGGEMSMeshSolid.cl:521-533).
      V3 mn = v3(so.border_min[0], so.border_min[1], so.border_min[2]);
      V3 mx = v3(so.border_max[0], so.border_max[1], so.border_max[2]);
      float dist = distance_to_aabb(g2l_pos(so.matrix, ph.p), g2l_dir(so.matrix, ph.d), mn, mx);
      float step = dist + kTolerance;
      ph.p = v3(ph.p.x + ph.d.x * step, ph.p.y + ph.d.y * step, ph.p.z + ph.d.z * step);
    } else {
      ph.p = l2g_pos(so.matrix, ph.p);
      ph.d = l2g_dir(so.matrix, ph.d);
    }
    trk(dead ? GG_TRACK_DEAD : GG_TRACK_LEAVE, -1, -1);
    if (dead) end_history();
    else phase = kFind;
  };
  auto track_phase = [](int type) {
    return type == GG_SOLID_VOXELIZED ? kTrackVoxel : (kFull && type == GG_SOLID_MESHED) ? kTrackMesh : kTrackBox;
  };

  // ---- photon stash (kStash) ----
  // Per warp, kStashRecords photon records in shared memory (field f of record
  // r at w_stash[f * 32 + r]: a lane's accesses hit 32 different banks) and
  // three warp-uniform masks saying which records hold a photon ready to track
  // (st_ready), waiting for an interaction (st_int) or for a new history /
  // FindSolid round (st_find); a record in none of them is empty.  A photon
  // carries its whole state, slot and random stream included, so moving it
  // between a lane and a record never changes what its slot computes.
  constexpr int kWords = stash_words(kBatch, kAux);
  const int lane = threadIdx.x & 31;
  const unsigned lanes_below = (1u << lane) - 1u;
  uint32_t* w_stash = nullptr;
  int* w_index = nullptr;
  StashMask st_ready = 0, st_int = 0, st_find = 0;
  if (kStash) {
    uint32_t* base = reinterpret_cast<uint32_t*>(bar + 2);
    w_stash = base + (threadIdx.x >> 5) * (kWords * kStashRecords + kStashRecords);
    w_index = reinterpret_cast<int*>(w_stash + kWords * kStashRecords);
  }
  // Exchanges this lane's photon with record r.
  auto swap_record = [&](int r) {
    uint32_t* q = w_stash + r;
    auto xu = [&](int f, uint32_t& v) {
      const uint32_t t = q[f * kStashRecords];
      q[f * kStashRecords] = v;
      v = t;
    };
    auto xf = [&](int f, float& v) {
      const uint32_t t = q[f * kStashRecords];
      q[f * kStashRecords] = __float_as_uint(v);
      v = __uint_as_float(t);
    };
    auto xi = [&](int f, int& v) {
      const uint32_t t = q[f * kStashRecords];
      q[f * kStashRecords] = static_cast<uint32_t>(v);
      v = static_cast<int>(t);
    };
    xu(0, rng.s1);
    xu(1, rng.s2);
    xu(2, rng.s3);
    xu(3, rng.s4);
    xu(4, rng.s5);
    xf(5, ph.p.x);
    xf(6, ph.p.y);
    xf(7, ph.p.z);
    xf(8, ph.d.x);
    xf(9, ph.d.y);
    xf(10, ph.d.z);
    xf(11, ph.E);
    xf(12, ph.psd);
    xi(13, ph.solid_id);
    uint32_t packed = static_cast<uint32_t>(static_cast<uint8_t>(ph.status)) |
                      (static_cast<uint32_t>(static_cast<uint8_t>(ph.scatter)) << 8) |
                      (static_cast<uint32_t>(phase) << 16);
    xu(14, packed);
    ph.status = static_cast<int8_t>(packed & 0xffu);
    ph.scatter = static_cast<int8_t>((packed >> 8) & 0xffu);
    phase = static_cast<int>(packed >> 16);
    xu(15, slot);
    xu(16, histories_left);
    xi(17, rounds);
    xi(18, pending);
    xf(19, inv_d.x);
    xf(20, inv_d.y);
    xf(21, inv_d.z);
    xi(22, energy_id);
    xf(23, cached_E);
    xi(24, cached_nav);
    if (kBatch) {
      xi(25, job);
      solids = P.job_solids + static_cast<size_t>(job) * P.number_of_solids;
    }
    if (kAux) xi(kWords - 1, history_number);
  };
  // The k-th lane of `lanes` (in lane order) gets the k-th record of
  // `records`; -1 for the other lanes.  Called by the whole warp.
  auto match = [&](unsigned lanes, StashMask records) -> int {
    int ranked = 0;
#pragma unroll
    for (int h = 0; h < kStashRecords / 32; ++h) {
      const unsigned part = stash_part(records, h);
      if ((part >> lane) & 1u) w_index[ranked + __popc(part & lanes_below)] = lane + 32 * h;
      ranked += __popc(part);
    }
    __syncwarp();
    int r = -1;
    if ((lanes >> lane) & 1u) {
      const int k = __popc(lanes & lanes_below);
      if (k < ranked) r = w_index[k];
    }
    __syncwarp();
    return r;
  };
  auto is_rare = [](int ph_phase) { return ph_phase == kNewHistory || ph_phase == kFind || ph_phase == kInteract; };
  // Lanes of `lanes` exchange their photons with records of `records`; the
  // masks then say what each touched record holds.  Called by the whole warp.
  auto exchange = [&](unsigned lanes, StashMask records) {
    const int r = match(lanes, records);
    const int old = phase;
    if (r >= 0) swap_record(r);
    StashMask moved = 0, to_int = 0, to_find = 0, to_empty = 0;
#pragma unroll
    for (int h = 0; h < kStashRecords / 32; ++h) {
      const unsigned bit = (r >= 32 * h && r < 32 * h + 32) ? (1u << (r - 32 * h)) : 0u;
      moved |= stash_mask(__reduce_or_sync(0xffffffffu, bit), h);
      to_int |= stash_mask(__reduce_or_sync(0xffffffffu, old == kInteract ? bit : 0u), h);
      to_find |= stash_mask(__reduce_or_sync(0xffffffffu, (old == kNewHistory || old == kFind) ? bit : 0u), h);
      to_empty |= stash_mask(__reduce_or_sync(0xffffffffu, old == kDone ? bit : 0u), h);
    }
    st_int = (st_int & ~moved) | to_int;
    st_find = (st_find & ~moved) | to_find;
    st_ready = (st_ready & ~moved) | (moved & ~(to_int | to_find | to_empty));
  };

  if (kStash) {
    // Fill the records first: each lane claims a slot (a run of its own) for
    // records lane, lane + 32, ..., then one for itself.
#pragma unroll 1
    for (int h = 0; h < kStashRecords / 32; ++h) {
    phase = next_slot() ? kNewHistory : kDone;
    st_find |= stash_mask(__ballot_sync(0xffffffffu, phase == kNewHistory), h);
    swap_record(lane + 32 * h);  // the lane receives whatever the record held before: reset below
    slot = ~0u;
    histories_left = 0;
    rounds = 0;
    pending = 0;
    energy_id = 0;
    cached_E = -1.0f;
    cached_nav = -1;
    history_number = -1;
    ph = Photon{};
    ph.solid_id = -1;
    inv_d = v3(0.0f, 0.0f, 0.0f);
    if (kBatch) {
      job = 0;
      solids = scene_solids;
    }
    phase = kDone;
    }
  }
  if (next_slot()) phase = kNewHistory;

  // Warp-level phase scheduling.  Tracking steps (voxel or detector box) are
  // ~98 % of all steps; new histories, FindSolid/ProjectToSolid rounds and
  // Compton/Rayleigh sampling are rare but long.  Running every lane's phase
  // each iteration would execute the rare code for one or two lanes in most
  // iterations; instead the rare phases wait until regroup_lanes lanes need
  // them, or until they are at least regroup_ratio4/4 times as many as the
  // tracking lanes, and then run together.  A waiting lane draws no random
  // number and touches no tally, so waiting changes when it computes, never
  // what.
  const int regroup = P.regroup_lanes;
  const int ratio4 = P.regroup_ratio4;
  const int swap_lanes = P.stash_swap_lanes;
  const int round_photons = P.stash_round_photons;
  for (;;) {
    bool round = false, serve_interact = false;
    if (kStash) {
      unsigned active = __ballot_sync(0xffffffffu, phase != kDone);
      if (active == 0 && (st_ready | st_int | st_find) == 0) break;
      unsigned waiting = __ballot_sync(0xffffffffu, is_rare(phase));
      // Lanes waiting for a rare phase, and lanes without a photon, take
      // ready photons from the stash (once enough of them wait: an exchange
      // costs the warp two shared-memory accesses per word).
      const unsigned want = waiting | ~active;
      if (st_ready != 0 && __popc(want) >= min(swap_lanes, stash_popc(st_ready))) {
        exchange(want, st_ready);
        active = __ballot_sync(0xffffffffu, phase != kDone);
        waiting = __ballot_sync(0xffffffffu, is_rare(phase));
      }
      // A round of one kind of rare work when a full warp of it is waiting
      // (lanes and records), or when the waiting lanes are many against the
      // tracking ones and no ready photon is left to replace them.
      const unsigned w_int = __ballot_sync(0xffffffffu, phase == kInteract);
      const int n_int = __popc(w_int) + stash_popc(st_int);
      const int n_find = __popc(waiting & ~w_int) + stash_popc(st_find);
      const int n_wait = __popc(waiting), n_track = __popc(active & ~waiting);
      round = n_int + n_find > 0 &&
              (n_int >= 32 || n_find >= 32 || n_int + n_find >= round_photons || n_track == 0 ||
               (n_wait > 0 && (n_wait >= regroup || 4 * n_wait >= ratio4 * n_track)));
      if (round) {
        serve_interact = n_int >= 32 ? (n_find < 32 || n_int >= n_find) : (n_find < 32 && n_int >= n_find);
        // gather: lanes without a photon of the served kind take one from the stash
        const unsigned kind_lanes = serve_interact ? w_int : (waiting & ~w_int);
        const StashMask kind_records = serve_interact ? st_int : st_find;
        if (kind_records != 0 && kind_lanes != 0xffffffffu) exchange(~kind_lanes, kind_records);
      }
    } else {
      const unsigned active = __ballot_sync(0xffffffffu, phase != kDone);
      if (active == 0) break;
      const unsigned tracking =
          __ballot_sync(0xffffffffu, phase == kTrackVoxel || phase == kTrackBox || (kFull && phase == kTrackMesh));
      const int n_other = __popc(active & ~tracking);
      round = n_other > 0 && (n_other >= regroup || 4 * n_other >= ratio4 * __popc(tracking));
      // A round serves one kind of rare work: the interaction samplers, or the
      // new-history / FindSolid chain, whichever more lanes wait for; the
      // others wait for the next round (their code paths stay out of this
      // one).  Measured +1.4 % on the CBCT projection.
      if (round) serve_interact = 2 * __popc(__ballot_sync(0xffffffffu, phase == kInteract)) >= n_other;
    }
    // A step or an interaction that ends the photon's stay in its solid sets
    // `leave` (1: alive, 2: dead) and `leaving`, and jumps to the one copy of
    // the exit code at the end of the loop body.
    int leave = 0;
    const DevSolid* leaving = nullptr;
    if (round) {
      if ((phase == kInteract) != serve_interact) continue;
      if (phase == kInteract) {
        // The Compton / Rayleigh part of a tracking step (the tail of
        // track_through_*): sample the interaction, then tally as the step would.
        const DevSolid& so = solids[ph.solid_id];
        const int nav = so.navigator;
        const int material = pending & 0xff;
        const int proc = pending >> 8;
        float e0 = ph.E;
        scatter(ph, rng, proc, navs[nav], tab.energy_bins(nav), tab.sigma(nav), material, energy_id);
        trk(GG_TRACK_SCATTER, ph.solid_id, proc);
        if (so.type != GG_SOLID_BOX) {
          // voxelized and meshed solids flag scattering; boxes do not
          // (TrackThroughGGEMSVoxelizedSolid.cl:253, TrackThroughGGEMSMeshSolid.cl:484)
          ph.scatter = 1;
          if ((kDose && so.dose_map >= 0) && !so.dose_tle) dose_record(P.dose_maps[so.dose_map], e0 - ph.E, ph.p);
          if (ph.E <= tab.photon_cut(nav)[material]) {
            if ((kDose && so.dose_map >= 0)) dose_record(P.dose_maps[so.dose_map], ph.E, ph.p);
            ph.status = GG_DEAD;
          }
        } else if (proc == GG_COMPTON_SCATTERING) {
          box_histogram(so, ph);
        }
        if (ph.status == GG_DEAD) {
          leave = 2;
          leaving = &so;
          goto exit_solid;
        }
        inv_d = reciprocal(ph.d);
        phase = track_phase(so.type);
        continue;
      }
      if (phase == kNewHistory) {
        const DevSource& source = P.jobs[job].source;
        const PrimaryOut o = new_primary(rng, source);
        ph.p = o.p;
        ph.d = o.d;
        ph.E = o.E;
        rng = o.rng;
        ph.scatter = 0;
        ph.status = GG_ALIVE;
        ph.psd = kOutOfWorld;
        rounds = 0;
        phase = kFind;
        if (kAux) {
          ++history_number;
          trk(GG_TRACK_PRIMARY, -1, -1);
        }
      }
      if (phase != kFind) continue;
      bool end = rounds >= GG_MAX_LOOP;
      if (!end && P.number_of_solids == 0) {
        ++rounds;  // no navigator: the reference loop only counts iterations
      } else if (!end) {
        ++rounds;
        // particle_solid_distance_* (ParticleSolidDistanceGGEMS*.cl:43-108)
        for (int s = 0; s < P.number_of_solids; ++s) {
          if (ph.status == GG_DEAD || ph.psd == 0.0f) break;
          const DevSolid& so = solids[s];
          V3 mn = v3(so.border_min[0], so.border_min[1], so.border_min[2]);
          V3 mx = v3(so.border_max[0], so.border_max[1], so.border_max[2]);
          V3 lp = g2l_pos(so.matrix, ph.p);
          if (in_aabb(lp, mn, mx)) {
            ph.psd = 0.0f;
            ph.solid_id = s;
            break;
          }
          float dist = distance_to_aabb(lp, g2l_dir(so.matrix, ph.d), mn, mx);
          if (dist < ph.psd) {
            ph.psd = dist;
            ph.solid_id = s;
          }
        }
        if (kAux && P.world_dimensions[0] > 0 && ph.status != GG_DEAD) world_track(ph.p, ph.d, ph.E, ph.psd, P);
        // project_to_* (ProjectToGGEMS*.cl:44-129)
        if (ph.solid_id == -1) ph.status = GG_DEAD;
        if (ph.psd == kOutOfWorld) {
          ph.solid_id = -1;
          ph.status = GG_DEAD;
        } else if (ph.status != GG_DEAD) {
          const DevSolid& so = solids[ph.solid_id];
          ph.p = add(ph.p, scale(ph.d, ph.psd + kTolerance));
          V3 lp = g2l_pos(so.matrix, ph.p);
          lp = safety_inside(lp, v3(so.border_min[0], so.border_min[1], so.border_min[2]),
                             v3(so.border_max[0], so.border_max[1], so.border_max[2]));
          ph.p = l2g_pos(so.matrix, lp);
          ph.psd = 0.0f;
        }
        if (ph.status == GG_DEAD) {
          end = true;
          trk(GG_TRACK_DEAD, -1, -1);
        } else {
          // Enter the solid: switch to local coordinates (a meshed solid's
          // triangles are already in world coordinates).
          const DevSolid& so = solids[ph.solid_id];
          if (!kFull || so.type != GG_SOLID_MESHED) {
            ph.p = g2l_pos(so.matrix, ph.p);
            ph.d = g2l_dir(so.matrix, ph.d);
          }
          trk(GG_TRACK_ENTER, ph.solid_id, -1);
          inv_d = reciprocal(ph.d);
          phase = track_phase(so.type);
        }
      }
      if (end) end_history();
      continue;
    }
    if (phase != kTrackVoxel && phase != kTrackBox && !(kFull && phase == kTrackMesh)) continue;
    {

    // ---- one tracking step inside solid ph.solid_id ----
    // the solid's and navigator's per-step fields in six 16-byte loads
    // (DevSolid / DevNavigator lead with them)
    const DevSolid& so = solids[ph.solid_id];
    const float4 s0 = load4f(&so.border_min[0]);     // border_min xyz, border_max x
    const float4 s1 = load4f(&so.border_max[1]);     // border_max yz, voxel_sizes xy
    const float4 s2 = load4f(&so.voxel_sizes[2]);    // voxel_sizes z, inv_voxel_sizes xyz
    const int4 s3 = load4i(&so.number_of_voxels[0]);  // number_of_voxels xyz, navigator
    const int4 s4 = load4i(&so.labels);               // labels (2 words), type, voxel_pow2
    const int nav = s3.w;
    const int4 n0 = load4i(&navs[nav]);               // number_of_bins, process_pack, sigma / cut offsets
    const float4* sig = reinterpret_cast<const float4*>(tab.base + static_cast<uint32_t>(n0.z));
    V3 bmin = v3(s0.x, s0.y, s0.z);
    V3 bmax = v3(s0.w, s1.x, s1.y);
    if (ph.E != cached_E || nav != cached_nav) {
      energy_id = binary_search(ph.E, tab.energy_bins(nav), n0.x);
      cached_E = ph.E;
      cached_nav = nav;
    }

    leaving = &so;
    if (!kFull || phase != kTrackMesh) do {
      // One step through a voxelized solid (track_through_ggems_voxelized_solid,
      // TrackThroughGGEMSVoxelizedSolid.cl:133-310) or a detector box
      // (track_through_ggems_solid_box, TrackThroughGGEMSSolidBox.cl:122-248):
      // the same sampling and slab test against the current voxel or the whole
      // box (material 0), then each solid's own tail.
      const bool voxel = phase == kTrackVoxel;
      V3 vmin = bmin, vmax = bmax;
      int material = 0;
      if (voxel) {
        V3 vs = v3(s1.z, s1.w, s2.x);
        V3 q = sub(ph.p, bmin);
        q = s4.w ? mul(q, v3(s2.y, s2.z, s2.w)) : divv(q, vs);
        int ix = __float2int_rz(q.x), iy = __float2int_rz(q.y), iz = __float2int_rz(q.z);
        const int nx = s3.x, ny = s3.y, nz = s3.z;
        if (ix >= nx || iy >= ny || iz >= nz || ix < 0 || iy < 0 || iz < 0) {
          ph.psd = kOutOfWorld;
          ph.solid_id = -1;
          leave = 1;
          break;
        }
        const uint8_t* labels = reinterpret_cast<const uint8_t*>(
            (static_cast<unsigned long long>(static_cast<uint32_t>(s4.y)) << 32) | static_cast<uint32_t>(s4.x));
        material = __ldg(labels + (ix + iy * nx + iz * nx * ny));
        vmin = add(bmin, mul(v3(static_cast<float>(ix), static_cast<float>(iy), static_cast<float>(iz)), vs));
        vmax = add(vmin, vs);
      }
      int proc;
      float nid = next_interaction(rng, n0.x, static_cast<uint32_t>(n0.y), sig, energy_id, material, proc);
      ph.p = safety_inside(ph.p, vmin, vmax);
      float dtb = distance_to_aabb(ph.p, ph.d, inv_d, vmin, vmax);
      if (dtb <= nid) {
        nid = dtb + kTolerance;
        proc = GG_TRANSPORTATION;
        if (kDose && voxel && so.dose_map >= 0) {
          const DevDoseMap& dm = P.dose_maps[so.dose_map];
          if (dm.photon_tracking) {
            int id = dosel(dm, ph.p);
            if (id >= 0) atomicAdd(dm.photon_tracking + id, 1);
          }
        }
      }
      ph.p = safety_outside(add(ph.p, scale(ph.d, nid)), vmin, vmax);
      if (!in_aabb(ph.p, bmin, bmax)) {
        ph.psd = kOutOfWorld;
        ph.solid_id = -1;
        leave = 1;
        break;
      }
      if (!voxel) {
        if (ph.E < so.threshold) ph.status = GG_DEAD;
      } else if (kDose && so.dose_tle) {
        // The step's deposit depends only on the energy before the interaction,
        // so it is recorded here even when the interaction itself is deferred.
        dose_record(P.dose_maps[so.dose_map], tle_edep(tab.attenuation(nav), material, ph.E, nid), ph.p);
      }
      trk(GG_TRACK_STEP, ph.solid_id, proc);
      if (proc == GG_COMPTON_SCATTERING || proc == GG_RAYLEIGH_SCATTERING) {
        pending = (proc << 8) | material;
        phase = kInteract;
        continue;
      }
      if (!voxel) {
        if (proc == GG_PHOTOELECTRIC_EFFECT) {
          ph.status = GG_DEAD;
          ph.E = 0.0f;
          box_histogram(so, ph);
        }
      } else {
        if (proc == GG_PHOTOELECTRIC_EFFECT) {
          if (kDose && so.dose_map >= 0 && !so.dose_tle) dose_record(P.dose_maps[so.dose_map], ph.E, ph.p);
          ph.status = GG_DEAD;
          ph.E = 0.0f;
        }
        if (ph.E <= reinterpret_cast<const float*>(tab.base + static_cast<uint32_t>(n0.w))[material]) {
          if (kDose && so.dose_map >= 0) dose_record(P.dose_maps[so.dose_map], ph.E, ph.p);
          ph.status = GG_DEAD;
        }
      }
      if (ph.status == GG_DEAD) leave = 2;
    } while (0);
    else if (kFull && phase == kTrackMesh) do {
      // track_through_ggems_meshed_solid, TrackThroughGGEMSMeshSolid.cl:385-518:
      // the parity of the crossing count says whether the photon is inside the
      // mesh; outside, it jumps to the first crossing.  Material 0.
      const MeshCrossings x =
          mesh_crossings(ph.p, ph.d, inv_d, so.mesh_nodes, so.mesh_node_count, so.mesh_triangles, so.mesh_bvh);
      if (x.count == 0) {
        ph.psd = kOutOfWorld;
        ph.solid_id = -1;
        leave = 1;
        break;
      }
      V3 next = x.first;
      if ((x.count & 1) == 0) {
        ph.p = x.first;
        next = x.second;
      }
      int proc;
      float nid = next_interaction(rng, n0.x, static_cast<uint32_t>(n0.y), sig, energy_id, 0, proc);
      const float dx = next.x - ph.p.x, dy = next.y - ph.p.y, dz = next.z - ph.p.z;
      const float to_next = sqrtf(dx * dx + dy * dy + dz * dz);
      if (to_next <= nid) {
        nid = to_next + kTolerance;
        proc = GG_TRANSPORTATION;
        if ((kDose && so.dose_map >= 0)) {
          const DevDoseMap& dm = P.dose_maps[so.dose_map];
          if (dm.photon_tracking) {
            int id = dosel(dm, ph.p);
            if (id >= 0) atomicAdd(dm.photon_tracking + id, 1);
          }
        }
      }
      ph.p = add(ph.p, scale(ph.d, nid));
      trk(GG_TRACK_STEP, ph.solid_id, proc);
      if (proc == GG_COMPTON_SCATTERING || proc == GG_RAYLEIGH_SCATTERING) {
        pending = proc << 8;
        phase = kInteract;
        continue;
      }
      if (proc == GG_PHOTOELECTRIC_EFFECT) {
        if ((kDose && so.dose_map >= 0)) dose_record(P.dose_maps[so.dose_map], ph.E, ph.p);
        ph.status = GG_DEAD;
        ph.E = 0.0f;
      }
      if (ph.E <= reinterpret_cast<const float*>(tab.base + static_cast<uint32_t>(n0.w))[0]) {
        if ((kDose && so.dose_map >= 0)) dose_record(P.dose_maps[so.dose_map], ph.E, ph.p);
        ph.status = GG_DEAD;
      }
      if (ph.status == GG_DEAD) leave = 2;
    } while (0);
    }
  exit_solid:
    if (leave) leave_solid(*leaving, leave == 2);
  }
}

// compute_dose_ggems_{voxelized,meshed}_solid, ComputeDoseGGEMSVoxelizedSolid.cl:53-121,
// ComputeDoseGGEMSMeshSolid.cl:53-114
__global__ void compute_dose_kernel(DoseParams P) {
  const DevDoseMap& dm = P.map;
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= dm.total_number_of_dosels) return;
  int z = id / dm.slice_number_of_dosels;
  int x = (id - z * dm.slice_number_of_dosels) % dm.number_of_dosels[0];
  int y = (id - z * dm.slice_number_of_dosels) / dm.number_of_dosels[0];
  float px = static_cast<float>(x) * dm.size_of_dosels[0] +
             static_cast<float>(dm.number_of_dosels[0] - 1) * (-0.5f * dm.size_of_dosels[0]);
  float py = static_cast<float>(y) * dm.size_of_dosels[1] +
             static_cast<float>(dm.number_of_dosels[1] - 1) * (-0.5f * dm.size_of_dosels[1]);
  float pz = static_cast<float>(z) * dm.size_of_dosels[2] +
             static_cast<float>(dm.number_of_dosels[2] - 1) * (-0.5f * dm.size_of_dosels[2]);
  int material = 0;  // meshed solids (ComputeDoseGGEMSMeshSolid.cl:90): material 0, no labels
  if (P.labels) {
    int vx = __float2int_rz((px - P.border_min[0]) / P.voxel_sizes[0]);
    int vy = __float2int_rz((py - P.border_min[1]) / P.voxel_sizes[1]);
    int vz = __float2int_rz((pz - P.border_min[2]) / P.voxel_sizes[2]);
    material = P.labels[vx + vy * P.number_of_voxels[0] + vz * P.number_of_voxels[0] * P.number_of_voxels[1]];
  }
  float vol = dm.size_of_dosels[0] * dm.size_of_dosels[1] * dm.size_of_dosels[2];
  constexpr float kGCm3 = 6.241509704e+21f / 1.e3f;  // g/cm3
  constexpr float kGy = 1.0e-12f;
  float density = P.is_water_reference ? 1.0f * kGCm3 : P.density[material];
  double edep = static_cast<double>(static_cast<long long>(dm.edep[id])) / kEdepScale;
  P.dose[id] = density < P.minimum_density
                   ? 0.0f
                   : static_cast<float>(static_cast<double>(P.scale_factor) * edep / static_cast<double>(density) /
                                        static_cast<double>(vol) / static_cast<double>(kGy));
  if (P.uncertainty) {
    int hit = dm.hit ? dm.hit[id] : 0;
    if (hit > 1 && edep != 0.0) {
      double e2 = dm.edep_squared ? dm.edep_squared[id] : 0.0;
      double sum2 = edep * edep;
      P.uncertainty[id] = static_cast<float>(sqrt((hit * e2 - sum2) / ((hit - 1) * sum2)));
    } else {
      P.uncertainty[id] = 1.0f;
    }
  }
}

}  // namespace

namespace {
using TransportKernel = void (*)(TransportParams);
// kFull: meshed solids, world grid or particle tracking (dose code always in),
// kAux: world grid or particle tracking; otherwise the dose-map code is
// compiled in only for scenes that tally dose.
// kStash: the photon stash (voxel / detector scenes without world grid or
// particle tracking).
TransportKernel transport_variant(bool mesh, bool batch, bool dose, bool aux, int stash) {
  if (aux) return batch ? transport_kernel<true, true, true, true, 0> : transport_kernel<true, false, true, true, 0>;
  if (mesh) {
    if (stash) return batch ? transport_kernel<true, true, true, false, 2> : transport_kernel<true, false, true, false, 2>;
    return batch ? transport_kernel<true, true, true, false, 0> : transport_kernel<true, false, true, false, 0>;
  }
  if (stash == 1) {
    if (dose) return batch ? transport_kernel<false, true, true, false, 1> : transport_kernel<false, false, true, false, 1>;
    return batch ? transport_kernel<false, true, false, false, 1> : transport_kernel<false, false, false, false, 1>;
  }
  if (stash == 2) {
    if (dose) return batch ? transport_kernel<false, true, true, false, 2> : transport_kernel<false, false, true, false, 2>;
    return batch ? transport_kernel<false, true, false, false, 2> : transport_kernel<false, false, false, false, 2>;
  }
  if (dose) return batch ? transport_kernel<false, true, true, false, 0> : transport_kernel<false, false, true, false, 0>;
  return batch ? transport_kernel<false, true, false, false, 0> : transport_kernel<false, false, false, false, 0>;
}
}  // namespace

void launch_transport(const TransportParams& p, int grid, int threads, size_t smem, void* stream, bool mesh, bool dose,
                      bool aux, int stash) {
  const bool batch = p.number_of_jobs > 1;
  transport_variant(mesh, batch, dose, aux, stash)<<<grid, threads, smem, static_cast<cudaStream_t>(stream)>>>(p);
}

namespace {

// Siddon-style ray march (Amanatides-Woo voxel walk) from the source to the
// centre of detector element (i, j), in the phantom's frame: sum of
// mu[label] x chord length.  Element centres follow the detector histogram's
// binning (element (i, j) covers [bmin + i es, bmin + (i+1) es) in x, y).
__global__ void line_integral_kernel(ProjectorParams P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i >= P.elements[0] || j >= P.elements[1]) return;
  const V3 local_pixel = v3(P.detector_min[0] + (static_cast<float>(i) + 0.5f) * P.element_size[0],
                            P.detector_min[1] + (static_cast<float>(j) + 0.5f) * P.element_size[1], 0.0f);
  const V3 pixel = l2g_pos(P.detector_matrix, local_pixel);
  const V3 s = g2l_pos(P.phantom_matrix, v3(P.source[0], P.source[1], P.source[2]));
  const V3 e = g2l_pos(P.phantom_matrix, pixel);
  const float dv[3] = {e.x - s.x, e.y - s.y, e.z - s.z};
  const float sv[3] = {s.x, s.y, s.z};
  float t0 = 0.0f, t1 = 1.0f;
  for (int a = 0; a < 3; ++a) {
    if (fabsf(dv[a]) < 1e-12f) {
      if (sv[a] < P.border_min[a] || sv[a] > P.border_max[a]) t1 = -1.0f;
    } else {
      float ta = (P.border_min[a] - sv[a]) / dv[a], tb = (P.border_max[a] - sv[a]) / dv[a];
      if (ta > tb) {
        float t = ta;
        ta = tb;
        tb = t;
      }
      t0 = fmaxf(t0, ta);
      t1 = fminf(t1, tb);
    }
  }
  float sum = 0.0f;
  if (t1 > t0) {
    const float length = sqrtf(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
    int idx[3], step[3];
    float tmax[3], tdelta[3];
    const float tm = 0.5f * (t0 + t1);
    for (int a = 0; a < 3; ++a) {
      // start voxel: the one containing the entry point (nudged inside)
      const float pa = sv[a] + fminf(t0 + 1e-6f * (t1 - t0), tm) * dv[a];
      int k = static_cast<int>(floorf((pa - P.border_min[a]) / P.voxel_sizes[a]));
      idx[a] = min(max(k, 0), P.number_of_voxels[a] - 1);
      if (dv[a] > 0.0f) {
        step[a] = 1;
        tmax[a] = (P.border_min[a] + (idx[a] + 1) * P.voxel_sizes[a] - sv[a]) / dv[a];
        tdelta[a] = P.voxel_sizes[a] / dv[a];
      } else if (dv[a] < 0.0f) {
        step[a] = -1;
        tmax[a] = (P.border_min[a] + idx[a] * P.voxel_sizes[a] - sv[a]) / dv[a];
        tdelta[a] = -P.voxel_sizes[a] / dv[a];
      } else {
        step[a] = 0;
        tmax[a] = FLT_MAX;
        tdelta[a] = FLT_MAX;
      }
    }
    float t = t0;
    const int nx = P.number_of_voxels[0], nxy = nx * P.number_of_voxels[1];
    for (int guard = 0; guard < 4 * (P.number_of_voxels[0] + P.number_of_voxels[1] + P.number_of_voxels[2]); ++guard) {
      const int a = (tmax[0] < tmax[1]) ? (tmax[0] < tmax[2] ? 0 : 2) : (tmax[1] < tmax[2] ? 1 : 2);
      const float tn = fminf(tmax[a], t1);
      const int m = P.labels[idx[0] + idx[1] * nx + idx[2] * nxy];
      if (m < P.number_of_materials) sum += P.mu[m] * (tn - t) * length;
      t = tn;
      if (t >= t1) break;
      idx[a] += step[a];
      if (idx[a] < 0 || idx[a] >= P.number_of_voxels[a]) break;
      tmax[a] += tdelta[a];
    }
  }
  const size_t o = static_cast<size_t>(j) * P.elements[0] + i;
  if (P.network_input) {
    P.out[2 * o] = expf(-sum);
    P.out[2 * o + 1] = sum;
  } else {
    P.out[o] = sum;
  }
}

}  // namespace

void launch_line_integrals(const ProjectorParams& p, void* stream) {
  dim3 grid((p.elements[0] + 127) / 128, p.elements[1]);
  line_integral_kernel<<<grid, 128, 0, static_cast<cudaStream_t>(stream)>>>(p);
}

void launch_compute_dose(const DoseParams& p, void* stream) {
  int n = p.map.total_number_of_dosels;
  compute_dose_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(p);
}

cudaError_t configure_transport(size_t smem, int threads, int* blocks_per_sm, bool mesh, bool batch, bool dose,
                                bool aux, int stash) {
  auto kernel = transport_variant(mesh, batch, dose, aux, stash);
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kernel, threads, smem);
}

cudaError_t set_rayleigh_fit(const float* pp /* 9*101 */) {
  return cudaMemcpyToSymbol(c_rayleigh_pp, pp, sizeof(float) * 9 * 101);
}

}  // namespace gg
