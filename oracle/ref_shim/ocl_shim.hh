// Test infrastructure only (oracle pin): an OpenCL-C-to-C++ shim that lets
// g++ compile the reference's device kernels (src/kernels/*.cl and the
// __OPENCL_C_VERSION__ halves of include/GGEMS/**) unmodified, straight from
// the reference checkout, so the oracle restatement can be checked against
// the reference's own kernel code run on the host.
//
// Nothing in the product links this file.  It is force-included (g++ -include)
// before each .cl translation unit by oracle/build.py (build_ref).
//
// Semantics chosen where OpenCL leaves them to the runtime (and mirrored
// exactly by the product kernels and the oracle restatement):
//   * dot(a, b)       = a.x*b.x + a.y*b.y + a.z*b.z (+ a.w*b.w), left to right,
//                       no contraction (-ffp-contract=off);
//   * normalize(v)    = v * (1.0f / sqrt(dot(v, v)));
//   * convert_int3(v) = truncation toward zero (the OpenCL default _rtz mode);
//   * log/exp/sin/cos/acos/sqrt = the host libm overloads of the same precision.
#ifndef GG_ORACLE_OCL_SHIM_HH
#define GG_ORACLE_OCL_SHIM_HH

// Standard headers the driver needs are pulled in before the qualifier
// macros below (`global`, `constant`, `kernel`) are defined.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

// Device-side precision switches the reference is built with by default
// (CMakeLists.txt: DOSIMETRY_DOUBLE_PRECISION=ON).
#define __OPENCL_C_VERSION__ 300
#define DOSIMETRY_DOUBLE_PRECISION 1
#define cl_khr_fp64 1
#define cl_khr_int64_base_atomics 1

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef unsigned long ulong;

using std::acos;
using std::cos;
using std::exp;
using std::fabs;
using std::log;
using std::log10;
using std::pow;
using std::sin;
using std::sqrt;

// ---------------------------------------------------------------------------
// Vector types.  Members are `mutable` because the reference writes through
// `GGfloat3 const*` (include/GGEMS/geometries/GGEMSRayTracing.hh:60-82,
// 130-152), which OpenCL C accepts and C++ does not.  float3/int3 occupy 16
// bytes like cl_float3/cl_int3.
// ---------------------------------------------------------------------------
struct float3 {
  mutable float x, y, z;
  float w_pad_;
  float3() : x(0.0f), y(0.0f), z(0.0f), w_pad_(0.0f) {}
  float3(float s) : x(s), y(s), z(s), w_pad_(0.0f) {}
  float3(float a, float b, float c) : x(a), y(b), z(c), w_pad_(0.0f) {}
};

struct float4 {
  float x, y, z, w;
};

struct int3 {
  int x, y, z;
  int w_pad_;
  int3() : x(0), y(0), z(0), w_pad_(0) {}
  int3(int a, int b, int c) : x(a), y(b), z(c), w_pad_(0) {}
};

#define s0 x
#define s1 y
#define s2 z

inline float3 operator+(float3 const& a, float3 const& b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 const& a, float3 const& b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 const& a, float3 const& b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 const& a, float3 const& b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator*(float3 const& a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float s, float3 const& a) { return float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator/(float3 const& a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
inline float3& operator+=(float3& a, float3 const& b) { a = a + b; return a; }
inline float3& operator-=(float3& a, float3 const& b) { a = a - b; return a; }
inline int3 operator-(int3 const& a, int s) { return int3(a.x - s, a.y - s, a.z - s); }

inline float dot(float3 const& a, float3 const& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float4 const& a, float4 const& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float3 normalize(float3 const& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline float3 fabs(float3 const& v) { return float3(std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)); }

inline int3 convert_int3(float3 const& v) { return int3(static_cast<int>(v.x), static_cast<int>(v.y), static_cast<int>(v.z)); }
inline float3 convert_float3(int3 const& v) { return float3(static_cast<float>(v.x), static_cast<float>(v.y), static_cast<float>(v.z)); }

// ---------------------------------------------------------------------------
// Work-item index: the oracle driver sets it before calling a kernel body.
// ---------------------------------------------------------------------------
extern thread_local size_t gg_shim_global_id;
inline size_t get_global_id(int) { return gg_shim_global_id; }

// ---------------------------------------------------------------------------
// Atomics (OpenCL 1.x names used by the reference).
// ---------------------------------------------------------------------------
inline int atomic_add(volatile int* p, int v) { return __atomic_fetch_add(const_cast<int*>(p), v, __ATOMIC_RELAXED); }
inline uint atomic_cmpxchg(volatile uint* p, uint cmp, uint val) {
  uint expected = cmp;
  __atomic_compare_exchange_n(const_cast<uint*>(p), &expected, val, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
  return expected;
}
inline ulong atom_cmpxchg(volatile ulong* p, ulong cmp, ulong val) {
  ulong expected = cmp;
  __atomic_compare_exchange_n(const_cast<ulong*>(p), &expected, val, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED);
  return expected;
}

// ---------------------------------------------------------------------------
// Address-space and function qualifiers.
// ---------------------------------------------------------------------------
#define __global
#define global
#define __private
#define __local
#define __constant static const
#define constant static const
#define __kernel extern "C"
#define kernel extern "C"

#endif  // GG_ORACLE_OCL_SHIM_HH
