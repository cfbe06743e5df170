// CPU oracle for the GGEMS photon path -- TEST INFRASTRUCTURE ONLY.
//
// A plain C++ restatement of GGEMS v1.3's photon transport (sources, solid
// navigation, Compton / photoelectric / Rayleigh sampling, dose and CT
// histogram tallies), one history at a time per random slot.  It exists to
// check the CUDA product against; only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg load it, and the product never links it.
//
// Each function cites the reference file:line it follows.  Arithmetic is
// kept in the reference's order and precision (float unless the reference
// uses double); build with -ffp-contract=off so a*b+c is never fused.
//
// The restatement is pinned against the reference's own kernels, compiled
// from the reference checkout through oracle/ref_shim (oracle/_ref), by
// tests/test_oracle_pin.py.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "ggems_b200.h"

// Arithmetic type of the restatement: float (the reference's precision, pinned
// bit for bit against its kernels) or, built with -DGG_ORACLE_REAL=double, the
// same algorithm in FP64 (the reference's float constants kept) -- the FP64
// oracle the CUDA results' precision is measured against.
#ifndef GG_ORACLE_REAL
#define GG_ORACLE_REAL float
#endif

namespace {

using Real = GG_ORACLE_REAL;

constexpr Real kTwoPi = 6.283185307179586f;            // GGEMSConstants.hh:39
constexpr Real kElectronMassC2 = 0.510998910f;          // GGEMSConstants.hh:52
constexpr Real kGeometryTolerance = 5.0e-04f;           // GGEMSGeometryConstants.hh:39
constexpr Real kEpsilon6 = 1.0e-06f;                    // GGEMSGeometryConstants.hh:38
constexpr Real kOutOfWorld = FLT_MAX;                   // GGEMSParticleConstants.hh:44
constexpr int8_t kNoProcess = 99;                        // GGEMSProcessConstants.hh:37
constexpr Real kRayleighFactor = 32526509815670243328.0f;  // GGEMSRayleighScatteringModels.hh:36

struct V3 {
  Real x, y, z;
};
inline V3 v3(Real x, Real y, Real z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 divv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 scale(V3 a, Real s) { return v3(a.x * s, a.y * s, a.z * s); }
inline Real dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// normalize: v * (1 / sqrt(dot(v, v))), the convention fixed for OpenCL's builtin.
inline V3 normalize3(V3 v) { return scale(v, 1.0f / std::sqrt(dot3(v, v))); }

// Row-major GGfloat44 helpers (GGEMSMatrixOperations.hh:46-125).
inline V3 mat_mul_point(const float* m, V3 p) {  // GGfloat44MultGGfloat3
  return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3] * 1.0f,
            m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7] * 1.0f,
            m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11] * 1.0f);
}
inline V3 mat33_mul(const float* m, V3 p) {  // GGfloat33MultGGfloat3
  return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z, m[4] * p.x + m[5] * p.y + m[6] * p.z,
            m[8] * p.x + m[9] * p.y + m[10] * p.z);
}
inline V3 mat33_transpose_mul(const float* m, V3 p) {  // GGfloat33TransposeMultGGfloat3
  return v3(m[0] * p.x + m[4] * p.y + m[8] * p.z, m[1] * p.x + m[5] * p.y + m[9] * p.z,
            m[2] * p.x + m[6] * p.y + m[10] * p.z);
}
// GGEMSReferentialTransformation.hh:80-141
inline V3 global_to_local_position(const float* m, V3 p) {
  return mat33_transpose_mul(m, v3(p.x - m[3], p.y - m[7], p.z - m[11]));
}
inline V3 local_to_global_position(const float* m, V3 p) { return mat_mul_point(m, p); }
inline V3 global_to_local_direction(const float* m, V3 d) { return normalize3(mat33_transpose_mul(m, d)); }
inline V3 local_to_global_direction(const float* m, V3 d) { return normalize3(mat33_mul(m, d)); }

// RotateUnitZ (GGEMSReferentialTransformation.hh:44-70, CLHEP rotateUz).
inline V3 rotate_unit_z(V3 v, V3 u) {
  Real up = u.x * u.x + u.y * u.y;
  if (up > 0) {
    up = std::sqrt(up);
    Real px = v.x, py = v.y, pz = v.z;
    v.x = (u.x * u.z * px - u.y * py) / up + u.x * pz;
    v.y = (u.y * u.z * px + u.x * py) / up + u.y * pz;
    v.z = -up * px + u.z * pz;
  } else if (u.z < 0.) {
    v.x = -v.x;
    v.z = -v.z;
  }
  return v;
}

// BinarySearch / LinearInterpolation (GGEMSMathAlgorithms.hh:46-86).
inline int binary_search(Real key, const float* a, int size) {
  int low = 0, mid = 0, high = size - 1;
  while (high - low > 1) {
    mid = (high + low) / 2;
    if (a[mid] == key) return mid;
    if (a[mid] < key) low = mid;
    else high = mid;
  }
  return low;
}
inline Real linear_interpolation(Real xa, Real ya, Real xb, Real yb, Real x) {
  if (xa > xb) return yb;
  if (xa >= x) return ya;
  if (xb <= x) return yb;
  return ya + (x - xa) * (yb - ya) / (xb - xa);
}

// Ray tracing (GGEMSRayTracing.hh:60-326).
inline void safety_inside_aabb(V3& p, V3 mn, V3 mx) {
  Real a = std::fabs(p.x - mn.x), b = std::fabs(p.x - mx.x);
  p.x = (a < kGeometryTolerance) ? mn.x + kGeometryTolerance : p.x;
  p.x = (b < kGeometryTolerance) ? mx.x - kGeometryTolerance : p.x;
  a = std::fabs(p.y - mn.y); b = std::fabs(p.y - mx.y);
  p.y = (a < kGeometryTolerance) ? mn.y + kGeometryTolerance : p.y;
  p.y = (b < kGeometryTolerance) ? mx.y - kGeometryTolerance : p.y;
  a = std::fabs(p.z - mn.z); b = std::fabs(p.z - mx.z);
  p.z = (a < kGeometryTolerance) ? mn.z + kGeometryTolerance : p.z;
  p.z = (b < kGeometryTolerance) ? mx.z - kGeometryTolerance : p.z;
}
inline void safety_outside_aabb(V3& p, V3 mn, V3 mx) {
  Real a = std::fabs(p.x - mn.x), b = std::fabs(p.x - mx.x);
  p.x = (a < kGeometryTolerance) ? mn.x - kGeometryTolerance : p.x;
  p.x = (b < kGeometryTolerance) ? mx.x + kGeometryTolerance : p.x;
  a = std::fabs(p.y - mn.y); b = std::fabs(p.y - mx.y);
  p.y = (a < kGeometryTolerance) ? mn.y - kGeometryTolerance : p.y;
  p.y = (b < kGeometryTolerance) ? mx.y + kGeometryTolerance : p.y;
  a = std::fabs(p.z - mn.z); b = std::fabs(p.z - mx.z);
  p.z = (a < kGeometryTolerance) ? mn.z - kGeometryTolerance : p.z;
  p.z = (b < kGeometryTolerance) ? mx.z + kGeometryTolerance : p.z;
}
inline bool in_aabb(V3 p, V3 mn, V3 mx) {
  if (p.x < (mn.x + kGeometryTolerance) || p.x > (mx.x - kGeometryTolerance)) return false;
  if (p.y < (mn.y + kGeometryTolerance) || p.y > (mx.y - kGeometryTolerance)) return false;
  if (p.z < (mn.z + kGeometryTolerance) || p.z > (mx.z - kGeometryTolerance)) return false;
  return true;
}
inline Real distance_to_aabb(V3 p, V3 d, V3 mn, V3 mx) {
  Real tmin = FLT_MIN, tmax = FLT_MAX, t1, t2, tmp;
  if (std::fabs(d.x) < kEpsilon6) {
    if (p.x < mn.x || p.x > mx.x) return kOutOfWorld;
  } else {
    Real id = 1.0f / d.x;
    tmin = (mn.x - p.x) * id;
    tmax = (mx.x - p.x) * id;
    if (tmin > tmax) { tmp = tmin; tmin = tmax; tmax = tmp; }
    if (tmin > tmax) return kOutOfWorld;
  }
  if (std::fabs(d.y) < kEpsilon6) {
    if (p.y < mn.y || p.y > mx.y) return kOutOfWorld;
  } else {
    Real id = 1.0f / d.y;
    t1 = (mn.y - p.y) * id;
    t2 = (mx.y - p.y) * id;
    if (t1 > t2) { tmp = t1; t1 = t2; t2 = tmp; }
    if (t1 > tmin) tmin = t1;
    if (t2 < tmax) tmax = t2;
    if (tmin > tmax) return kOutOfWorld;
  }
  if (std::fabs(d.z) < kEpsilon6) {
    if (p.z < mn.z || p.z > mx.z) return kOutOfWorld;
  } else {
    Real id = 1.0f / d.z;
    t1 = (mn.z - p.z) * id;
    t2 = (mx.z - p.z) * id;
    if (t1 > t2) { tmp = t1; t1 = t2; t2 = tmp; }
    if (t1 > tmin) tmin = t1;
    if (t2 < tmax) tmax = t2;
    if (tmin > tmax) return kOutOfWorld;
  }
  if (tmin < 0.0f && (tmax < 0.0f || tmax == 0.0f)) return kOutOfWorld;
  if ((tmax - tmin) < (2.0 * kGeometryTolerance)) return kOutOfWorld;  // double compare, as the reference
  if (tmin <= kEpsilon6) return tmax;
  return tmin;
}

inline V3 obb_min(const gg_obb& o) { return v3(o.border_min[0], o.border_min[1], o.border_min[2]); }
inline V3 obb_max(const gg_obb& o) { return v3(o.border_max[0], o.border_max[1], o.border_max[2]); }

// ---------------------------------------------------------------------------
// JKISS32 (GGEMSKissEngine.hh:50-75).
// ---------------------------------------------------------------------------
struct Kiss {
  uint32_t s1, s2, s3, s4, s5;
  Real uniform() {
    s2 ^= (s2 << 5);
    s2 ^= (s2 >> 7);
    s2 ^= (s2 << 22);
    int32_t t = static_cast<int32_t>(s3 + s4 + s5);
    s3 = s4;
    s5 = t < 0;
    s4 = static_cast<uint32_t>(t) & 2147483647u;
    s1 += 1411392427u;
    return static_cast<Real>((static_cast<Real>(s1 + s2 + s4) / 4294967295.0) * (1.0f - 1.0f / (1 << 23)));
  }
};

// ---------------------------------------------------------------------------
// Particle state: the photon fields of GGEMSPrimaryParticles.
// ---------------------------------------------------------------------------
struct Photon {
  Real E;
  V3 p, d;
  int8_t scatter, status, next_process;
  int32_t E_index, solid_id;
  Real psd;  // particle_solid_distance_
  Real nid;  // next_interaction_distance_
};

struct Tallies {
  const gg_scene* scene;
  gg_tally_buffers* out;
};

// Event counts for the algorithmic-byte model of the benchmark: voxel steps,
// box steps, dose deposits, histogram increments, primaries.
thread_local uint64_t t_counts[5];
std::atomic<uint64_t> g_counts[5];

void atomic_add_double(double* addr, double v) {
  std::atomic_ref<double> a(*addr);
  double cur = a.load(std::memory_order_relaxed);
  while (!a.compare_exchange_weak(cur, cur + v, std::memory_order_relaxed)) {
  }
}
void atomic_add_int(int32_t* addr, int32_t v) { __atomic_fetch_add(addr, v, __ATOMIC_RELAXED); }

// Squared-count tallies of the detector histograms (statistical tests only):
// when registered, every history's increments are collected per (histogram,
// bin) and k^2 is added for each bin the history counted k times in, so that
// sum k^2 - (sum k)^2 / n estimates each bin's variance over n primaries.  A
// primary can count more than once in one bin (a Compton site then a
// photoelectric site in the same detector element), so the bins are not
// Poisson.  Not part of the reference's algorithm; off by default.
int64_t* const* g_histogram_squares = nullptr;
thread_local std::vector<std::pair<int, int>> t_history_counts;

void record_histogram(int histogram, int index) {
  if (g_histogram_squares && g_histogram_squares[histogram]) t_history_counts.emplace_back(histogram, index);
}

void flush_history_counts() {
  auto& v = t_history_counts;
  if (v.empty()) return;
  std::sort(v.begin(), v.end());
  for (size_t i = 0; i < v.size();) {
    size_t j = i;
    while (j < v.size() && v[j] == v[i]) ++j;
    const int64_t k = static_cast<int64_t>(j - i);
    __atomic_fetch_add(&g_histogram_squares[v[i].first][v[i].second], k * k, __ATOMIC_RELAXED);
    i = j;
  }
  v.clear();
}

// dose_record_standard / dose_photon_tracking (GGEMSDoseRecording.hh:65-118).
bool dosel_index(const gg_dose_map& dm, V3 p, int* gid) {
  if (p.x < dm.border_min[0] + kEpsilon6 || p.x > dm.border_max[0] - kEpsilon6) return false;
  if (p.y < dm.border_min[1] + kEpsilon6 || p.y > dm.border_max[1] - kEpsilon6) return false;
  if (p.z < dm.border_min[2] + kEpsilon6 || p.z > dm.border_max[2] - kEpsilon6) return false;
  V3 q = mul(sub(p, v3(dm.border_min[0], dm.border_min[1], dm.border_min[2])),
             v3(dm.inv_size_of_dosels[0], dm.inv_size_of_dosels[1], dm.inv_size_of_dosels[2]));
  int ix = static_cast<int>(q.x), iy = static_cast<int>(q.y), iz = static_cast<int>(q.z);
  *gid = ix + iy * dm.number_of_dosels[0] + iz * dm.number_of_dosels[0] * dm.number_of_dosels[1];
  if (ix < 0 || ix >= dm.number_of_dosels[0]) return false;
  if (iy < 0 || iy >= dm.number_of_dosels[1]) return false;
  if (iz < 0 || iz >= dm.number_of_dosels[2]) return false;
  return true;
}
void dose_record(const Tallies& t, int map, Real edep, V3 p) {
  const gg_dose_map& dm = t.scene->dose_maps[map];
  int gid;
  if (!dosel_index(dm, p, &gid)) return;
  ++t_counts[2];
  if (t.out->hit && t.out->hit[map]) atomic_add_int(&t.out->hit[map][gid], 1);
  if (t.out->edep && t.out->edep[map]) atomic_add_double(&t.out->edep[map][gid], static_cast<double>(edep));
  if (t.out->edep_squared && t.out->edep_squared[map])
    atomic_add_double(&t.out->edep_squared[map][gid], static_cast<double>(edep) * static_cast<double>(edep));
}
void photon_tracking_record(const Tallies& t, int map, V3 p) {
  const gg_dose_map& dm = t.scene->dose_maps[map];
  int gid;
  if (!dosel_index(dm, p, &gid)) return;
  if (t.out->photon_tracking && t.out->photon_tracking[map]) atomic_add_int(&t.out->photon_tracking[map][gid], 1);
}

// GetPhotonNextInteraction (GGEMSPhotonNavigator.hh:57-93).
void next_interaction(Photon& ph, Kiss& rng, const gg_physics_tables& tb, int material) {
  int energy_id = binary_search(ph.E, tb.energy_bins, tb.number_of_bins);
  Real nid = kOutOfWorld;
  int8_t proc = kNoProcess;
  for (int i = 0; i < tb.number_of_processes; ++i) {
    int pid = tb.process_id[i];
    Real dist = -std::log(rng.uniform()) /
                 tb.cross_sections[static_cast<size_t>(pid) * tb.number_of_materials * tb.number_of_bins +
                                   energy_id + tb.number_of_bins * material];
    if (dist < nid) {
      nid = dist;
      proc = static_cast<int8_t>(pid);
    }
  }
  ph.E_index = energy_id;
  ph.nid = nid;
  ph.next_process = proc;
}

// KleinNishinaComptonSampleSecondaries (GGEMSComptonScatteringModels.hh:47-132).
void compton(Photon& ph, Kiss& rng) {
  Real E0 = ph.E;
  Real E0_mec2 = E0 / kElectronMassC2;
  V3 gd = ph.d;
  Real eps0 = 1.0f / (1.0f + 2.0f * E0_mec2);
  Real eps0sq = eps0 * eps0;
  Real alpha1 = -std::log(eps0);
  Real alpha2 = alpha1 + 0.5f * (1.0f - eps0sq);
  Real r1, r2, r3, epsilon, epsilonsq, onecost, sint2, greject;
  int nloop = 0;
  do {
    ++nloop;
    if (nloop > 1000) return;
    r1 = rng.uniform();
    r2 = rng.uniform();
    r3 = rng.uniform();
    if (alpha1 > alpha2 * r1) {
      epsilon = std::exp(-alpha1 * r2);
      epsilonsq = epsilon * epsilon;
    } else {
      epsilonsq = eps0sq + (1.0f - eps0sq) * r2;
      epsilon = std::sqrt(epsilonsq);
    }
    onecost = (1.0f - epsilon) / (epsilon * E0_mec2);
    sint2 = onecost * (2.0f - onecost);
    greject = 1.0f - epsilon * sint2 / (1.0f + epsilonsq);
  } while (greject < r3);
  if (sint2 < 0.0f) sint2 = 0.0f;
  Real costheta = 1.0f - onecost;
  Real sintheta = std::sqrt(sint2);
  Real phi = rng.uniform() * kTwoPi;
  V3 g = v3(sintheta * std::cos(phi), sintheta * std::sin(phi), costheta);
  g = rotate_unit_z(g, gd);
  g = normalize3(g);
  ph.E = E0 * epsilon;
  ph.d = g;
}

// LivermoreRayleighSampleSecondaries (GGEMSRayleighScatteringModels.hh:169-316).
struct RayleighFit {
  const float* pp[9];
};
RayleighFit g_rayleigh_fit;

Real rayleigh_w(Real x, Real n) {
  return (x < 0.02f) ? n * x * (1.0f - 0.5f * (n - 1.0f) * x * (1.0f - (n - 2.0f) * x / 3.0f))
                     : 1.0f - std::exp(-n * std::log(1.0f + x));
}

void rayleigh(Photon& ph, Kiss& rng, const gg_physics_tables& tb, int material) {
  Real E0 = ph.E;
  if (E0 <= 250.0e-6f) {
    ph.status = GG_DEAD;
    return;
  }
  V3 gd = ph.d;
  int nbins = tb.number_of_bins;
  int8_t n_minus_one = static_cast<int8_t>(tb.number_of_elements[material] - 1);
  int mixture = tb.element_offset[material];
  int energy_id = ph.E_index;
  uint8_t z = tb.atomic_number[mixture + n_minus_one];
  if (n_minus_one > 0) {
    const float* cs = tb.cross_sections + static_cast<size_t>(GG_RAYLEIGH_SCATTERING) * tb.number_of_materials * nbins;
    Real kcs = linear_interpolation(tb.energy_bins[energy_id], cs[energy_id + nbins * material],
                                     tb.energy_bins[energy_id + 1], cs[energy_id + 1 + nbins * material], E0);
    Real x = rng.uniform() * kcs;
    Real cross_section = 0.0f;
    uint8_t i = 0;
    while (i < n_minus_one) {
      uint8_t zi = tb.atomic_number[mixture + i];
      cross_section += tb.atomic_number_density[mixture + i] *
                       linear_interpolation(tb.energy_bins[energy_id], tb.rayleigh_per_atom[energy_id + nbins * zi],
                                            tb.energy_bins[energy_id + 1], tb.rayleigh_per_atom[energy_id + 1 + nbins * zi],
                                            E0);
      if (x < cross_section) {
        z = zi;
        break;
      }
      ++i;
    }
  }
  const float* const* P = g_rayleigh_fit.pp;
  Real xx = kRayleighFactor * E0 * E0;
  Real n0 = P[6][z] - 1.0f, n1 = P[7][z] - 1.0f, n2 = P[8][z] - 1.0f;
  Real b0 = P[3][z], b1 = P[4][z], b2 = P[5][z];
  Real w0 = rayleigh_w(2.0f * xx * b0, n0);
  Real w1 = rayleigh_w(2.0f * xx * b1, n1);
  Real w2 = rayleigh_w(2.0f * xx * b2, n2);
  Real x0 = w0 * P[0][z] / (b0 * n0);
  Real x1 = w1 * P[1][z] / (b1 * n1);
  Real x2 = w2 * P[2][z] / (b2 * n2);
  Real costheta = 0.0f, x;
  do {
    Real w = w0, n = n0, b = b0;
    x = rng.uniform() * (x0 + x1 + x2);
    if (x > x0) {
      x -= x0;
      if (x <= x1) {
        w = w1; n = n1; b = b1;
      } else {
        w = w2; n = n2; b = b2;
      }
    }
    n = 1.0f / n;
    Real y = rng.uniform() * w;
    if (y < 0.02f) {
      x = y * n * (1.0f + 0.5f * (n + 1.0f) * y * (1.0f - (n + 2.0f) * y / 3.0f));
    } else {
      x = std::exp(-n * std::log(1.0f - y)) - 1.0f;
    }
    costheta = 1.0f - x / (b * xx);
  } while (2.0f * rng.uniform() > 1.0f + costheta * costheta || costheta < -1.0f);
  Real phi = kTwoPi * rng.uniform();
  Real sintheta = std::sqrt((1.0f - costheta) * (1.0f + costheta));
  V3 g = v3(sintheta * std::cos(phi), sintheta * std::sin(phi), costheta);
  g = rotate_unit_z(g, gd);
  g = normalize3(g);
  ph.d = g;
}

// PhotonDiscreteProcess (GGEMSPhotonNavigator.hh:107-131).
void discrete_process(Photon& ph, Kiss& rng, const gg_physics_tables& tb, int material) {
  if (ph.next_process == GG_COMPTON_SCATTERING) {
    compton(ph, rng);
  } else if (ph.next_process == GG_PHOTOELECTRIC_EFFECT) {
    ph.status = GG_DEAD;  // StandardPhotoElectricSampleSecondaries (GGEMSPhotoElectricEffectModels.hh:46-53)
    ph.E = 0.0f;
  } else if (ph.next_process == GG_RAYLEIGH_SCATTERING) {
    rayleigh(ph, rng, tb, material);
  }
}

// get_primaries_ggems_xray_source (GetPrimariesGGEMSXRaySource.cl:52-143).
void xray_primary(Photon& ph, Kiss& rng, const gg_source& src) {
  double phi = rng.uniform();
  double theta = rng.uniform();
  phi *= static_cast<double>(kTwoPi);
  double new_aperture = 1.0 - std::cos(static_cast<double>(src.beam_aperture));
  theta = std::acos(1.0 - new_aperture * theta);
  V3 rotation = v3(static_cast<Real>(std::cos(phi) * std::sin(theta)), static_cast<Real>(std::sin(phi) * std::sin(theta)),
                   static_cast<Real>(std::cos(theta)));
  V3 gp = local_to_global_position(src.matrix, v3(0.0f, 0.0f, 0.0f));
  V3 dir = normalize3(sub(v3(0.0f, 0.0f, 0.0f), gp));
  dir = rotate_unit_z(rotation, dir);
  dir = normalize3(dir);
  gp.x = src.focal_spot_size[0] * (rng.uniform() - 0.5f);
  gp.y = src.focal_spot_size[1] * (rng.uniform() - 0.5f);
  gp.z = src.focal_spot_size[2] * (rng.uniform() - 0.5f);
  gp = local_to_global_position(src.matrix, gp);
  int nbins = src.number_of_energy_bins + 1;  // GGEMSXRaySource.cc:133 passes n+1
  int index = 0;
  Real rnd = 0.0f;
  if (nbins != 1) {
    rnd = rng.uniform();
    index = binary_search(rnd, src.energy_cdf, nbins + 1);
  }
  ph.E = !src.is_interp ? src.energy_spectrum[index]
                        : linear_interpolation(src.energy_cdf[index], src.energy_spectrum[index], src.energy_cdf[index + 1],
                                               src.energy_spectrum[index + 1], rnd);
  ph.p = gp;
  ph.d = dir;
  ph.scatter = 0;
  ph.status = GG_ALIVE;
  ph.psd = kOutOfWorld;
  ph.next_process = kNoProcess;
  ph.nid = 0.0f;
}

// get_primaries_ggems_voxelized_source (GetPrimariesGGEMSVoxelizedSource.cl:57-150).
void voxelized_primary(Photon& ph, Kiss& rng, const gg_source& src) {
  double phi = rng.uniform();
  double theta = rng.uniform();
  phi *= static_cast<double>(kTwoPi);
  theta = std::acos(1.0 - 2.0 * theta);
  V3 dir = v3(static_cast<Real>(std::cos(phi) * std::sin(theta)), static_cast<Real>(std::sin(phi) * std::sin(theta)),
              static_cast<Real>(std::cos(theta)));
  double rnd_act = rng.uniform();
  // number_of_activity_bins is the count passed to the kernel (active voxels + 1,
  // GGEMSVoxelizedSource.cc:170); the cdf and index arrays hold that many entries.
  int index_act = binary_search(static_cast<Real>(rnd_act), src.activity_cdf, static_cast<int>(src.number_of_activity_bins));
  int32_t vox = src.activity_index[index_act];
  int nx = src.number_of_voxels[0], ny = src.number_of_voxels[1];
  int slice = nx * ny;
  int iz = vox / slice;
  int ix = (vox - iz * slice) % nx;
  int iy = (vox - iz * slice) / nx;
  V3 bmin = v3(src.border_min[0], src.border_min[1], src.border_min[2]);
  V3 vs = v3(src.voxel_sizes[0], src.voxel_sizes[1], src.voxel_sizes[2]);
  V3 vmin = add(bmin, mul(v3(static_cast<Real>(ix), static_cast<Real>(iy), static_cast<Real>(iz)), vs));
  V3 vmax = add(vmin, vs);
  V3 p;
  p.x = bmin.x + (static_cast<Real>(ix) + rng.uniform()) * vs.x;
  p.y = bmin.y + (static_cast<Real>(iy) + rng.uniform()) * vs.y;
  p.z = bmin.z + (static_cast<Real>(iz) + rng.uniform()) * vs.z;
  safety_inside_aabb(p, vmin, vmax);
  p = local_to_global_position(src.matrix, p);
  int nbins = src.number_of_energy_bins + 1;
  int index = 0;
  Real rnd = 0.0f;
  if (nbins != 1) {
    rnd = rng.uniform();
    index = binary_search(rnd, src.energy_cdf, nbins + 1);
  }
  ph.E = !src.is_interp ? src.energy_spectrum[index]
                        : linear_interpolation(src.energy_cdf[index], src.energy_spectrum[index], src.energy_cdf[index + 1],
                                               src.energy_spectrum[index + 1], rnd);
  ph.p = p;
  ph.d = dir;
  ph.scatter = 0;
  ph.status = GG_ALIVE;
  ph.psd = kOutOfWorld;
  ph.next_process = kNoProcess;
  ph.nid = 0.0f;
}

// particle_solid_distance_* (ParticleSolidDistanceGGEMS*.cl:43-108).
void solid_distance(Photon& ph, const gg_solid& s, int solid_index) {
  if (ph.status == GG_DEAD) return;
  if (ph.psd == 0.0f) return;
  const float* m = s.obb.matrix;
  V3 local = global_to_local_position(m, ph.p);
  if (in_aabb(local, obb_min(s.obb), obb_max(s.obb))) {
    ph.psd = 0.0f;
    ph.solid_id = solid_index;
    return;
  }
  V3 ld = global_to_local_direction(m, ph.d);
  Real distance = distance_to_aabb(local, ld, obb_min(s.obb), obb_max(s.obb));
  if (distance < ph.psd) {
    ph.psd = distance;
    ph.solid_id = solid_index;
  }
}

// project_to_* (ProjectToGGEMS*.cl:44-129).
void project_to(Photon& ph, const gg_solid& s, int solid_index) {
  if (ph.solid_id == -1) ph.status = GG_DEAD;
  if (ph.psd == kOutOfWorld) {
    ph.solid_id = -1;
    ph.status = GG_DEAD;
    return;
  }
  if (ph.solid_id != solid_index) return;
  if (ph.status == GG_DEAD) return;
  ph.p = add(ph.p, scale(ph.d, ph.psd + kGeometryTolerance));
  // TransportGetSafetyInsideOBB (GGEMSRayTracing.hh:94-116)
  V3 local = global_to_local_position(s.obb.matrix, ph.p);
  safety_inside_aabb(local, obb_min(s.obb), obb_max(s.obb));
  ph.p = local_to_global_position(s.obb.matrix, local);
  ph.psd = 0.0f;
}

// track_through_ggems_voxelized_solid (TrackThroughGGEMSVoxelizedSolid.cl:58-323).
void track_voxelized(Photon& ph, Kiss& rng, const gg_scene& sc, const gg_solid& s, int solid_index, const Tallies& t) {
  if (ph.solid_id != solid_index) return;
  if (ph.status == GG_DEAD) return;
  const gg_physics_tables& tb = sc.tables[s.navigator];
  const float* m = s.obb.matrix;
  V3 lp = global_to_local_position(m, ph.p);
  V3 ld = global_to_local_direction(m, ph.d);
  ph.d = ld;
  V3 bmin = obb_min(s.obb), bmax = obb_max(s.obb);
  V3 vs = v3(s.voxel_sizes[0], s.voxel_sizes[1], s.voxel_sizes[2]);
  int nx = s.number_of_voxels[0], ny = s.number_of_voxels[1], nz = s.number_of_voxels[2];
  const int dm = s.dose_map;
  const bool tle = dm >= 0 && sc.dose_maps[dm].tle && tb.attenuation_energy_bins && tb.mu_en;
  do {
    V3 q = divv(sub(lp, bmin), vs);
    int ix = static_cast<int>(q.x), iy = static_cast<int>(q.y), iz = static_cast<int>(q.z);
    if (ix >= nx || iy >= ny || iz >= nz) {
      ph.psd = kOutOfWorld;
      ph.solid_id = -1;
      break;
    }
    int material = s.labels[ix + iy * nx + iz * nx * ny];
    ++t_counts[0];
    next_interaction(ph, rng, tb, material);
    Real nid = ph.nid;
    int8_t proc = ph.next_process;
    V3 vmin = add(bmin, mul(v3(static_cast<Real>(ix), static_cast<Real>(iy), static_cast<Real>(iz)), vs));
    V3 vmax = add(vmin, vs);
    safety_inside_aabb(lp, vmin, vmax);
    Real dtb = distance_to_aabb(lp, ld, vmin, vmax);
    if (dtb <= nid) {
      nid = dtb + kGeometryTolerance;
      proc = GG_TRANSPORTATION;
      if (dm >= 0) photon_tracking_record(t, dm, lp);
    }
    lp = add(lp, scale(ld, nid));
    safety_outside_aabb(lp, vmin, vmax);
    if (!in_aabb(lp, bmin, bmax)) {
      ph.psd = kOutOfWorld;
      ph.solid_id = -1;
      break;
    }
    ph.p = lp;
    Real initial_energy = ph.E;
    if (proc != GG_TRANSPORTATION) {
      discrete_process(ph, rng, tb, material);
      if (proc == GG_COMPTON_SCATTERING || proc == GG_RAYLEIGH_SCATTERING) ph.scatter = 1;
      if (dm >= 0 && !tle) dose_record(t, dm, initial_energy - ph.E, lp);
      ld = ph.d;
    }
    if (tle) {
      // Track-length estimator (TrackThroughGGEMSVoxelizedSolid.cl:286-301).
      const float* eb = tb.attenuation_energy_bins;
      const float* me = tb.mu_en + static_cast<size_t>(material) * GG_ATTENUATION_BINS;
      int e_index = binary_search(initial_energy, eb, GG_ATTENUATION_BINS);
      Real mu_en = e_index == 0 ? me[0]
                                 : linear_interpolation(eb[e_index - 1], me[e_index - 1], eb[e_index], me[e_index],
                                                        initial_energy);
      dose_record(t, dm, initial_energy * mu_en * nid * 0.1f, lp);
    }
    if (ph.E <= tb.photon_energy_cut[material]) {
      if (dm >= 0) dose_record(t, dm, ph.E, lp);
      ph.status = GG_DEAD;
    }
  } while (ph.status == GG_ALIVE);
  ph.p = local_to_global_position(m, lp);
  ph.d = local_to_global_direction(m, ld);
}

// track_through_ggems_solid_box (TrackThroughGGEMSSolidBox.cl:56-261), HISTOGRAM variant.
void track_box(Photon& ph, Kiss& rng, const gg_scene& sc, const gg_solid& s, int solid_index, const Tallies& t) {
  if (ph.solid_id != solid_index) return;
  if (ph.status == GG_DEAD) return;
  const gg_physics_tables& tb = sc.tables[s.navigator];
  const float* m = s.obb.matrix;
  V3 lp = global_to_local_position(m, ph.p);
  V3 ld = global_to_local_direction(m, ph.d);
  ph.d = ld;
  V3 bmin = obb_min(s.obb), bmax = obb_max(s.obb);
  V3 box = v3(s.box_size[0], s.box_size[1], s.box_size[2]);
  int vx = s.virtual_element_number[0], vy = s.virtual_element_number[1], vz = s.virtual_element_number[2];
  do {
    ++t_counts[1];
    next_interaction(ph, rng, tb, 0);
    Real nid = ph.nid;
    int8_t proc = ph.next_process;
    safety_inside_aabb(lp, bmin, bmax);
    Real dtb = distance_to_aabb(lp, ld, bmin, bmax);
    if (dtb <= nid) {
      nid = dtb + kGeometryTolerance;
      proc = GG_TRANSPORTATION;
    }
    lp = add(lp, scale(ld, nid));
    safety_outside_aabb(lp, bmin, bmax);
    if (!in_aabb(lp, bmin, bmax)) {
      ph.psd = kOutOfWorld;
      ph.solid_id = -1;
      break;
    }
    ph.p = lp;
    if (ph.E < s.threshold) ph.status = GG_DEAD;
    if (proc != GG_TRANSPORTATION) {
      discrete_process(ph, rng, tb, 0);
      ld = ph.d;
      if (s.histogram >= 0 && (proc == GG_PHOTOELECTRIC_EFFECT || proc == GG_COMPTON_SCATTERING)) {
        V3 es = divv(box, v3(static_cast<Real>(vx), static_cast<Real>(vy), static_cast<Real>(vz)));
        V3 q = divv(sub(lp, bmin), es);
        int ix = static_cast<int>(q.x), iy = static_cast<int>(q.y);
        int index = ix + iy * vx;
        ++t_counts[3];
        if (t.out->histograms && t.out->histograms[s.histogram]) {
          atomic_add_int(&t.out->histograms[s.histogram][index], 1);
          record_histogram(s.histogram, index);
        }
        if (s.scatter_histogram >= 0 && ph.scatter == 1 && t.out->histograms && t.out->histograms[s.scatter_histogram]) {
          atomic_add_int(&t.out->histograms[s.scatter_histogram][index], 1);
          record_histogram(s.scatter_histogram, index);
        }
      }
    }
  } while (ph.status == GG_ALIVE);
  ph.p = local_to_global_position(m, lp);
  ph.d = local_to_global_direction(m, ld);
}

// ---- meshed solid (TrackThroughGGEMSMeshSolid.cl:53-534) ----
constexpr int kMaxMeshHits = 16;  // MAX_TRIANGLE_INTERACTION

inline V3 cross3(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }

// MollerTrumboreRayTriangle (l.121-170); tri = p0, p1, p2, ...
bool moller_trumbore(V3 p, V3 d, const float* tri, V3* hit) {
  V3 p0 = v3(tri[0], tri[1], tri[2]);
  V3 e1 = v3(tri[3] - tri[0], tri[4] - tri[1], tri[5] - tri[2]);
  V3 e2 = v3(tri[6] - tri[0], tri[7] - tri[1], tri[8] - tri[2]);
  V3 h = cross3(d, e2);
  Real a = dot3(e1, h);
  if (a > -kEpsilon6 && a < kEpsilon6) return false;
  Real f = 1.0f / a;
  V3 s = sub(p, p0);
  Real u = f * dot3(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  V3 q = cross3(s, e1);
  Real v = f * dot3(q, d);
  if (v < 0.0f || u + v > 1.0f) return false;
  Real t = f * dot3(q, e2);
  if (!(t > kEpsilon6)) return false;
  *hit = v3(p.x + d.x * t, p.y + d.y * t, p.z + d.z * t);
  return true;
}

// TestLineNode (l.182-230): slab test of the ray against a node box.
bool line_hits_node(V3 p, V3 d, const float* node) {
  const Real pos[3] = {p.x, p.y, p.z}, dir[3] = {d.x, d.y, d.z};
  Real tmin = 0.0f, tmax = FLT_MAX;
  for (int i = 0; i < 3; ++i) {
    Real mn = node[i] - node[3 + i], mx = node[i] + node[3 + i];
    if (std::fabs(dir[i]) < kEpsilon6) {
      if (pos[i] < mn || pos[i] > mx) return false;
    } else {
      Real ood = 1.0f / dir[i];
      Real t1 = (mn - pos[i]) * ood, t2 = (mx - pos[i]) * ood;
      if (t1 > t2) std::swap(t1, t2);
      if (t1 > tmin) tmin = t1;
      if (t2 < tmax) tmax = t2;
      if (tmin > tmax) return false;
    }
  }
  return true;
}

// GetMeshIOPositions (l.240-318): crossings of the ray with the mesh, nearest
// first (insertion sort on squared distance, ties keep discovery order).  The
// reference stops a node's triangle loop at 16 crossings and goes on to the
// next node, writing past its 16-entry array if that node has crossings too;
// here the search ends at 16.
int mesh_crossings(V3 p, V3 d, const gg_solid& s, V3 out[kMaxMeshHits]) {
  Real dist2[kMaxMeshHits];
  int n = 0;
  for (int node = 0; node < s.number_of_nodes; ++node) {
    const int b = s.node_first[node], e = s.node_first[node + 1];
    if (b == e) continue;
    if (!line_hits_node(p, d, s.nodes + 6 * node)) continue;
    for (int k = b; k < e; ++k) {
      V3 hit;
      if (!moller_trumbore(p, d, s.triangles + static_cast<size_t>(s.node_triangles[k]) * GG_TRIANGLE_FLOATS, &hit))
        continue;
      Real d2 = (hit.x - p.x) * (hit.x - p.x) + (hit.y - p.y) * (hit.y - p.y) + (hit.z - p.z) * (hit.z - p.z);
      int at = n;
      while (at > 0 && d2 < dist2[at - 1]) {
        out[at] = out[at - 1];
        dist2[at] = dist2[at - 1];
        --at;
      }
      out[at] = hit;
      dist2[at] = d2;
      if (++n == kMaxMeshHits) return n;
    }
  }
  return n;
}

// track_through_ggems_meshed_solid (l.330-534): no frame change (triangles are
// in world coordinates), material 0, parity of the crossing count decides
// inside / outside; on leaving, the photon is carried to the OBB boundary.
void track_meshed(Photon& ph, Kiss& rng, const gg_scene& sc, const gg_solid& s, int solid_index, const Tallies& t) {
  if (ph.solid_id != solid_index) return;
  if (ph.status == GG_DEAD) return;
  const gg_physics_tables& tb = sc.tables[s.navigator];
  const int dm = s.dose_map;
  V3 lp = ph.p, ld = ph.d;
  V3 hits[kMaxMeshHits];
  do {
    ++t_counts[1];
    const int n = mesh_crossings(lp, ld, s, hits);
    if (n == 0) {
      ph.psd = kOutOfWorld;
      ph.solid_id = -1;
      break;
    }
    V3 next;
    if (n % 2 == 0) {
      lp = hits[0];
      next = hits[1];
    } else {
      next = hits[0];
    }
    ph.p = lp;
    ph.d = ld;
    next_interaction(ph, rng, tb, 0);
    Real nid = ph.nid;
    int8_t proc = ph.next_process;
    Real dx = next.x - lp.x, dy = next.y - lp.y, dz = next.z - lp.z;
    Real to_next = std::sqrt(dx * dx + dy * dy + dz * dz);
    if (to_next <= nid) {
      nid = to_next + kGeometryTolerance;
      proc = GG_TRANSPORTATION;
      if (dm >= 0) photon_tracking_record(t, dm, lp);
    }
    lp = add(lp, scale(ld, nid));
    ph.p = lp;
    Real initial_energy = ph.E;
    if (proc != GG_TRANSPORTATION) {
      discrete_process(ph, rng, tb, 0);
      if (proc == GG_COMPTON_SCATTERING || proc == GG_RAYLEIGH_SCATTERING) ph.scatter = 1;
      if (dm >= 0) dose_record(t, dm, initial_energy - ph.E, lp);
      ld = ph.d;
    }
    if (ph.E <= tb.photon_energy_cut[0]) {
      if (dm >= 0) dose_record(t, dm, ph.E, lp);
      ph.status = GG_DEAD;
    }
  } while (ph.status == GG_ALIVE);
  const float* m = s.obb.matrix;
  Real dist = distance_to_aabb(global_to_local_position(m, lp), global_to_local_direction(m, ld), obb_min(s.obb),
                                obb_max(s.obb));
  ph.p = v3(lp.x + ld.x * (dist + kGeometryTolerance), lp.y + ld.y * (dist + kGeometryTolerance),
            lp.z + ld.z * (dist + kGeometryTolerance));
  ph.d = ld;
}

// world_tracking (WorldTracking.cl:54-162): the photon's flight from its
// position to the solid FindSolid chose (10 m when none) is sampled in steps
// of the world element size along the dominant axis.
void world_tracking(const Photon& ph, const gg_world& w, const Tallies& t) {
  if (ph.status == GG_DEAD) return;
  Real distance = ph.psd == kOutOfWorld ? 10000.0f : ph.psd;
  if (distance <= kGeometryTolerance) return;
  V3 p1 = ph.p;
  const V3 dir = ph.d;
  const V3 size = v3(w.sizes[0], w.sizes[1], w.sizes[2]);
  const int dim[3] = {w.dimensions[0], w.dimensions[1], w.dimensions[2]};
  V3 p2 = add(p1, scale(dir, distance));
  const V3 lo = v3(size.x * static_cast<Real>(dim[0]) * -0.5f, size.y * static_cast<Real>(dim[1]) * -0.5f,
                   size.z * static_cast<Real>(dim[2]) * -0.5f);
  auto index_of = [&](V3 p, int idx[3]) {
    V3 q = divv(sub(p, lo), size);
    idx[0] = static_cast<int>(q.x);
    idx[1] = static_cast<int>(q.y);
    idx[2] = static_cast<int>(q.z);
  };
  int idx[3];
  index_of(p1, idx);
  V3 diff = sub(p2, p1);
  V3 len = v3(std::fabs(diff.x), std::fabs(diff.y), std::fabs(diff.z));
  Real length = len.x, main_size = size.x;
  if (len.y > length) {
    length = len.y;
    main_size = size.y;
  } else if (len.z > length) {
    length = len.z;
    main_size = size.z;
  }
  Real inv_length = 1.0f / length;
  V3 increment = v3(inv_length * diff.x, inv_length * diff.y, inv_length * diff.z);
  int steps = static_cast<int>(1.0f + (length / main_size));
  const double E = ph.E;
  for (int i = 0; i < steps; ++i) {
    if (idx[0] < 0 || idx[0] >= dim[0] || idx[1] < 0 || idx[1] >= dim[1] || idx[2] < 0 || idx[2] >= dim[2]) break;
    const size_t g = idx[0] + static_cast<size_t>(idx[1]) * dim[0] + static_cast<size_t>(idx[2]) * dim[0] * dim[1];
    const gg_tally_buffers* o = t.out;
    if (o && w.photon_tracking && o->world_photon_tracking) atomic_add_int(&o->world_photon_tracking[g], 1);
    if (o && w.energy_tracking && o->world_energy) atomic_add_double(&o->world_energy[g], E);
    if (o && w.energy_squared_tracking && o->world_energy_squared) atomic_add_double(&o->world_energy_squared[g], E * E);
    if (o && w.momentum && o->world_momentum_x) {
      atomic_add_double(&o->world_momentum_x[g], static_cast<double>(dir.x));
      atomic_add_double(&o->world_momentum_y[g], static_cast<double>(dir.y));
      atomic_add_double(&o->world_momentum_z[g], static_cast<double>(dir.z));
    }
    p1 = add(p1, scale(increment, main_size));
    index_of(p1, idx);
  }
}

// One history, following GGEMS::RunOnDevice's inner loop (src/global/GGEMS.cc:326-345):
// FindSolid, ProjectToSolid, TrackThroughSolid over all solids in order,
// until the particle is dead or GG_MAX_LOOP iterations were made.
void transport(Photon& ph, Kiss& rng, const gg_scene& sc, const Tallies& t) {
  for (int loop = 0; loop < GG_MAX_LOOP; ++loop) {
    for (int s = 0; s < sc.number_of_solids; ++s) solid_distance(ph, sc.solids[s], s);
    if (sc.world) world_tracking(ph, *sc.world, t);
    for (int s = 0; s < sc.number_of_solids; ++s) project_to(ph, sc.solids[s], s);
    for (int s = 0; s < sc.number_of_solids; ++s) {
      const gg_solid& solid = sc.solids[s];
      if (solid.type == GG_SOLID_VOXELIZED) track_voxelized(ph, rng, sc, solid, s, t);
      else if (solid.type == GG_SOLID_BOX) track_box(ph, rng, sc, solid, s, t);
      else if (solid.type == GG_SOLID_MESHED) track_meshed(ph, rng, sc, solid, s, t);
    }
    if (ph.status == GG_DEAD) break;
  }
}

uint64_t batch_count(uint64_t n) {
  // GGEMSSource.cc:403 (float division, as in the reference)
  return static_cast<uint64_t>(std::ceil(static_cast<float>(n) / GG_MAXIMUM_PARTICLES));
}

}  // namespace

extern "C" {

// Event counts accumulated by gg_oracle_run since the last reset:
// [voxel steps, box steps, dose deposits, histogram increments, primaries].
__attribute__((visibility("default"))) void gg_oracle_counts(uint64_t* out, int reset) {
  for (int k = 0; k < 5; ++k) {
    if (out) out[k] = g_counts[k].load();
    if (reset) g_counts[k] = 0;
  }
}

// Register (or, with NULL, drop) the squared-count tallies of the detector
// histograms: one int64 array per histogram of the scene (NULL entries skip a
// histogram), summed into by every following run.
__attribute__((visibility("default"))) void gg_oracle_set_histogram_squares(int64_t* const* squares) {
  g_histogram_squares = squares;
}

// Register the Rayleigh form-factor fit tables PP0..PP8 (101 floats each).
__attribute__((visibility("default"))) void gg_oracle_set_rayleigh_fit(const float* const* pp) {
  for (int i = 0; i < 9; ++i) g_rayleigh_fit.pp[i] = pp[i];
}

// Run number_of_particles primaries of `source` through `scene`, batching as
// GGEMSSource::OrganizeParticlesInBatch for one device.  random_states holds
// 5 arrays of GG_MAXIMUM_PARTICLES words (in/out).  Final particle states are
// written for the slots of the last batch that touched them.
__attribute__((visibility("default"))) int gg_oracle_run(const gg_scene* scene, const gg_source* source,
                                                         uint64_t number_of_particles, uint32_t* random_states,
                                                         gg_particle_buffers* particles, gg_tally_buffers* tallies,
                                                         int threads) {
  if (!scene || !source || !random_states) return GG_ERROR_INVALID_ARGUMENT;
  const uint64_t nb = batch_count(number_of_particles);
  std::vector<uint64_t> sizes(nb);
  if (nb == 1) {
    sizes[0] = number_of_particles;
  } else {
    for (uint64_t j = 0; j < nb; ++j) sizes[j] = number_of_particles / nb;
    for (uint64_t j = 0; j < number_of_particles % nb; ++j) sizes[j]++;
  }
  const uint64_t slots = nb ? sizes[0] : 0;
  if (scene->rayleigh_fit)
    for (int i = 0; i < 9; ++i) g_rayleigh_fit.pp[i] = scene->rayleigh_fit + 101 * i;
  Tallies t{scene, tallies};
  const size_t S = GG_MAXIMUM_PARTICLES;
  auto worker = [&](uint64_t begin, uint64_t end) {
    for (auto& c : t_counts) c = 0;
    struct Flush {
      ~Flush() {
        for (int k = 0; k < 5; ++k) g_counts[k] += t_counts[k];
      }
    } flush;
    for (uint64_t slot = begin; slot < end; ++slot) {
      Kiss rng{random_states[slot], random_states[S + slot], random_states[2 * S + slot], random_states[3 * S + slot],
               random_states[4 * S + slot]};
      Photon ph{};
      ph.solid_id = -1;
      for (uint64_t b = 0; b < nb; ++b) {
        if (slot >= sizes[b]) break;
        ++t_counts[4];
        if (source->type == GG_SOURCE_XRAY) xray_primary(ph, rng, *source);
        else voxelized_primary(ph, rng, *source);
        transport(ph, rng, *scene, t);
        flush_history_counts();
      }
      random_states[slot] = rng.s1;
      random_states[S + slot] = rng.s2;
      random_states[2 * S + slot] = rng.s3;
      random_states[3 * S + slot] = rng.s4;
      random_states[4 * S + slot] = rng.s5;
      if (particles) {
        particles->E[slot] = ph.E;
        particles->px[slot] = ph.p.x;
        particles->py[slot] = ph.p.y;
        particles->pz[slot] = ph.p.z;
        particles->dx[slot] = ph.d.x;
        particles->dy[slot] = ph.d.y;
        particles->dz[slot] = ph.d.z;
        particles->status[slot] = ph.status;
        particles->scatter[slot] = ph.scatter;
        particles->solid_id[slot] = ph.solid_id;
      }
    }
  };
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  for (int i = 0; i < threads; ++i) {
    uint64_t b = slots * i / threads, e = slots * (i + 1) / threads;
    pool.emplace_back(worker, b, e);
  }
  for (auto& th : pool) th.join();
  return GG_OK;
}

}  // extern "C"
