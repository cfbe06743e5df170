// Test infrastructure only (host-table pin): a host-side stand-in for the
// OpenCL C++ header, with just enough of its types for the reference's host
// headers (include/GGEMS/**) and table-building sources to compile with g++.
// A "device buffer" here is plain host memory: mapping it returns its
// address, so the reference's GetDeviceBuffer / ReleaseDeviceBuffer pairs read
// and write ordinary arrays.  Nothing in the product includes this file.
#ifndef GG_ORACLE_REF_HOST_CL_HPP
#define GG_ORACLE_REF_HOST_CL_HPP

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

typedef int8_t cl_char;
typedef uint8_t cl_uchar;
typedef int16_t cl_short;
typedef uint16_t cl_ushort;
typedef int32_t cl_int;
typedef uint32_t cl_uint;
typedef int64_t cl_long;
typedef uint64_t cl_ulong;
typedef float cl_float;
typedef double cl_double;
typedef uint32_t cl_bool;

// Vector types: the element array s[] plus x/y/z/w names, as the OpenCL host
// headers give them (cl_T3 has the size of cl_T4).
#define GG_CL_VEC(T, N)                      \
  typedef union {                            \
    T s[N];                                  \
    struct {                                 \
      T x, y, z, w;                          \
    };                                       \
    struct {                                 \
      T s0, s1, s2, s3;                      \
    };                                       \
  } T##N;
#define GG_CL_VEC2(T)  \
  typedef union {      \
    T s[2];            \
    struct {           \
      T x, y;          \
    };                 \
    struct {           \
      T s0, s1;        \
    };                 \
  } T##2;
#define GG_CL_VECN(T, N) \
  typedef union {        \
    T s[N];              \
    struct {             \
      T x, y, z, w;      \
    };                   \
  } T##N;
#define GG_CL_TYPES(T)   \
  GG_CL_VEC2(T)          \
  GG_CL_VEC(T, 4)        \
  typedef T##4 T##3;     \
  GG_CL_VECN(T, 8)       \
  GG_CL_VECN(T, 16)
GG_CL_TYPES(cl_char)
GG_CL_TYPES(cl_uchar)
GG_CL_TYPES(cl_short)
GG_CL_TYPES(cl_ushort)
GG_CL_TYPES(cl_int)
GG_CL_TYPES(cl_uint)
GG_CL_TYPES(cl_long)
GG_CL_TYPES(cl_ulong)
GG_CL_TYPES(cl_float)
GG_CL_TYPES(cl_double)
#undef GG_CL_TYPES
#undef GG_CL_VEC
#undef GG_CL_VEC2
#undef GG_CL_VECN

typedef cl_ulong cl_bitfield;
typedef cl_bitfield cl_map_flags;
typedef cl_bitfield cl_mem_flags;
typedef cl_bitfield cl_svm_mem_flags;
typedef cl_bitfield cl_device_type;
typedef cl_bitfield cl_device_fp_config;
typedef cl_bitfield cl_device_exec_capabilities;
typedef cl_bitfield cl_device_svm_capabilities;
typedef cl_bitfield cl_device_affinity_domain;
typedef cl_bitfield cl_command_queue_properties;
typedef cl_uint cl_device_mem_cache_type;
typedef cl_uint cl_device_local_mem_type;
typedef cl_uint cl_profiling_info;
typedef struct _cl_event* cl_event;
typedef struct _cl_context* cl_context;
typedef struct _cl_command_queue* cl_command_queue;
typedef struct _cl_mem* cl_mem;
typedef struct _cl_kernel* cl_kernel;

#define CL_SUCCESS 0
#define CL_FALSE 0
#define CL_TRUE 1
#define CL_COMPLETE 0x0
#define CL_MAP_READ (1 << 0)
#define CL_MAP_WRITE (1 << 1)
#define CL_MEM_READ_WRITE (1 << 0)
#define CL_MEM_WRITE_ONLY (1 << 1)
#define CL_MEM_READ_ONLY (1 << 2)
#define CL_MEM_USE_HOST_PTR (1 << 3)
#define CL_MEM_ALLOC_HOST_PTR (1 << 4)
#define CL_MEM_COPY_HOST_PTR (1 << 5)
#define CL_MEM_SVM_FINE_GRAIN_BUFFER (1 << 10)
#define CL_DEVICE_TYPE_CPU (1 << 1)
#define CL_DEVICE_TYPE_GPU (1 << 2)
#define CL_DEVICE_TYPE_ACCELERATOR (1 << 3)
#define CL_PROFILING_COMMAND_START 0x1282
#define CL_PROFILING_COMMAND_END 0x1283

// Declared so that the reference's header templates (SVM helpers, never
// instantiated by the table builders) name-check; not defined.
void* clSVMAlloc(cl_context, cl_svm_mem_flags, size_t, cl_uint);
void clSVMFree(cl_context, void*);
cl_int clEnqueueSVMMap(cl_command_queue, cl_bool, cl_map_flags, void*, size_t, cl_uint, const cl_event*, cl_event*);
cl_int clEnqueueSVMUnmap(cl_command_queue, void*, cl_uint, const cl_event*, cl_event*);

namespace cl {

class Event {
 public:
  cl_int wait() const { return CL_SUCCESS; }
  cl_int setCallback(cl_int, void (*)(cl_event, cl_int, void*), void* = nullptr) { return CL_SUCCESS; }
  template <typename T>
  cl_int getProfilingInfo(cl_profiling_info, T* v) const {
    *v = T();
    return CL_SUCCESS;
  }
  cl_event operator()() const { return nullptr; }
};

// Host memory standing in for a device buffer.
class Buffer {
 public:
  Buffer() = default;
  explicit Buffer(size_t size) : bytes_(size) {}
  void* data() { return bytes_.data(); }
  size_t size() const { return bytes_.size(); }

 private:
  std::vector<unsigned char> bytes_;
};

class Context {
 public:
  cl_context operator()() const { return nullptr; }
};

class Device {};
class Platform {};
class Program {};
class Kernel {};
class NDRange {
 public:
  NDRange() = default;
  explicit NDRange(size_t) {}
};

class CommandQueue {
 public:
  void* enqueueMapBuffer(Buffer& buffer, cl_bool, cl_map_flags, size_t offset, size_t, const std::vector<Event>*,
                         Event*, cl_int* err) {
    if (err) *err = CL_SUCCESS;
    return static_cast<unsigned char*>(buffer.data()) + offset;
  }
  cl_int enqueueUnmapMemObject(Buffer&, void*, const std::vector<Event>*, Event*) { return CL_SUCCESS; }
  cl_int finish() { return CL_SUCCESS; }
  cl_command_queue operator()() const { return nullptr; }
};

}  // namespace cl

#endif
