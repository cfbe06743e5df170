// Phantom volumes on the device (include/ggems_b200.h, "phantom volumes"):
// the volume creator's analytic shapes drawn into a voxel image
// (GGEMSVolumeCreatorManager, src/geometries/GGEMSVolumeCreatorManager.cc;
// GGEMSBox / GGEMSTube / GGEMSSphere::Draw; kernels
// src/kernels/DrawGGEMS{Box,Tube,Sphere}.cl) and the range-table conversion
// of an MHD image into material labels
// (GGEMSVoxelizedSolid::ConvertImageToLabel,
// include/GGEMS/geometries/GGEMSVoxelizedSolid.hh:162-257).
//
// Both are one pass over the image, one thread per element, grid-stride: pure
// HBM streams (the draw kernels write only covered voxels; the label kernel
// reads the image once and writes one byte per voxel).  Built with
// -fmad=false so every voxel-centre and inside test rounds like GGEMS's
// single-precision expressions.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>

#include "gg_internal.cuh"

struct gg_volume {
  int device = 0;
  int met_type = GG_MET_FLOAT;
  int32_t dimensions[3] = {0, 0, 0};
  float element_sizes[3] = {0.0f, 0.0f, 0.0f};
  uint64_t elements = 0;
  size_t element_bytes = 4;
  void* data = nullptr;
  cudaStream_t stream = nullptr;
  // label conversion buffers, allocated on first use
  uint8_t* labels = nullptr;
  float* table = nullptr;  // [255] first, [255] last
  uint8_t* lut = nullptr;  // label of every value of an 8- or 16-bit element type
  unsigned long long* missing = nullptr;
  cudaEvent_t start = nullptr, stop = nullptr;
  float last_ms = 0.0f;  // device time of the last draw / label kernels
};

namespace {

int check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return GG_OK;
  return gg::record_error(e == cudaErrorMemoryAllocation ? GG_ERROR_OUT_OF_MEMORY : GG_ERROR_CUDA,
                          (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}
#define VOL_CUDA(call)                         \
  do {                                         \
    int rc_ = check((call), #call);            \
    if (rc_ != GG_OK) return rc_;              \
  } while (0)

size_t met_bytes(int t) {
  switch (t) {
    case GG_MET_CHAR:
    case GG_MET_UCHAR: return 1;
    case GG_MET_SHORT:
    case GG_MET_USHORT: return 2;
    case GG_MET_INT:
    case GG_MET_UINT:
    case GG_MET_FLOAT: return 4;
    default: return 0;
  }
}

struct DrawParams {
  uint64_t elements;
  int32_t dim[3];
  float es[3];
  float pos[3];
  float label;
  float size[3];
};

// Voxel centre relative to the shape, with GGEMS's index arithmetic
// (DrawGGEMSBox.cl:82-89): y = (id mod dx*dx) / dx, x = id mod (dx*dy) - y*dx
// (size_t arithmetic, then int), z = id / (dx*dy); centre =
// (es/2) * ((1 - dim) + 2*index) - position.
// Volumes below 2^32 elements (all practical ones) take the same arithmetic in
// 32 bits, where every intermediate fits and the results are identical.
__device__ __forceinline__ void voxel_centre(const DrawParams& p, uint64_t id, float c[3]) {
  const int dx = p.dim[0], dy = p.dim[1];
  int ix, iy, iz;
  if (p.elements <= 0xffffffffull) {
    const uint32_t i = static_cast<uint32_t>(id);
    const uint32_t sq = static_cast<uint32_t>(dx * dx), plane = static_cast<uint32_t>(dx * dy);
    iy = static_cast<int>((i % sq) / static_cast<uint32_t>(dx));
    ix = static_cast<int>(static_cast<uint64_t>(i % plane) - static_cast<uint64_t>(static_cast<int64_t>(iy * dx)));
    iz = static_cast<int>(i / plane);
  } else {
    const uint64_t sq = static_cast<uint64_t>(static_cast<int64_t>(dx * dx));
    const uint64_t plane = static_cast<uint64_t>(static_cast<int64_t>(dx * dy));
    iy = static_cast<int>((id % sq) / static_cast<uint64_t>(static_cast<int64_t>(dx)));
    ix = static_cast<int>((id % plane) - static_cast<uint64_t>(static_cast<int64_t>(iy * dx)));
    iz = static_cast<int>(id / plane);
  }
  const int idx[3] = {ix, iy, iz};
  for (int a = 0; a < 3; ++a) {
    const float half = p.es[a] / 2.0f;
    const float f = (1.0f - static_cast<float>(p.dim[a])) + 2.0f * static_cast<float>(idx[a]);
    c[a] = half * f - p.pos[a];
  }
}

template <class T, int kShape>
__global__ void draw_kernel(T* __restrict__ volume, DrawParams p) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t id = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; id < p.elements; id += stride) {
    float c[3];
    voxel_centre(p, id, c);
    bool inside;
    if (kShape == GG_SHAPE_BOX) {
      // DrawGGEMSBox.cl:74-97: |z| <= depth/2, |y| <= height/2, |x| <= width/2
      const float hw = p.size[0] / 2.0f, hh = p.size[1] / 2.0f, hd = p.size[2] / 2.0f;
      inside = c[2] <= hd && c[2] >= -hd && c[1] <= hh && c[1] >= -hh && c[0] <= hw && c[0] >= -hw;
    } else if (kShape == GG_SHAPE_TUBE) {
      // DrawGGEMSTube.cl:89-91: |z| <= height/2 and x^2/rx^2 + y^2/ry^2 <= 1
      const float h2 = p.size[2] / 2.0f;
      inside = c[2] <= h2 && c[2] >= -h2 &&
               (c[0] * c[0] / (p.size[0] * p.size[0]) + c[1] * c[1] / (p.size[1] * p.size[1])) <= 1.0f;
    } else {
      // DrawGGEMSSphere.cl:86: x^2 + y^2 + z^2 <= r^2
      inside = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] <= p.size[0] * p.size[0];
    }
    if (inside) volume[id] = static_cast<T>(p.label);
  }
}

// The LAST range line holding the value gives the label (the reference
// rewrites the whole image once per line, in file order); 255 = none.
__device__ __forceinline__ int range_label(float v, const float* table, int ranges) {
  for (int r = ranges - 1; r >= 0; --r) {
    const float a = table[r], b = table[ranges + r];
    if ((v == a && v == b) || (v >= a && v < b)) return r;
  }
  return 255;
}

// Each thread converts chunks of 16 elements: sizeof(T) 16-byte streaming
// loads in, one 16-byte store of labels out (the image and the labels are
// touched once, so both bypass L2 residency with the .cs hint); the last
// elements % 16 go one per thread.  Both arrays come from cudaMalloc, so every
// chunk is 16-byte aligned.
template <class T>
__global__ void labels_kernel(const T* __restrict__ image, uint64_t elements, const float* __restrict__ first,
                              const float* __restrict__ last, int ranges, uint8_t* __restrict__ labels,
                              unsigned long long* __restrict__ unconverted) {
  extern __shared__ float table[];  // [ranges] first, [ranges] last
  for (int i = threadIdx.x; i < ranges; i += blockDim.x) {
    table[i] = first[i];
    table[ranges + i] = last[i];
  }
  __syncthreads();
  unsigned long long missing = 0;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t chunks = elements / 16;
  for (uint64_t c = tid; c < chunks; c += stride) {
    union {
      uint4 q[sizeof(T)];
      T e[16];
    } in;
    const uint4* src = reinterpret_cast<const uint4*>(image + c * 16);
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(T)); ++k) in.q[k] = __ldcs(src + k);
    union {
      uint4 q;
      uint8_t b[16];
    } out;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int label = range_label(static_cast<float>(in.e[j]), table, ranges);
      out.b[j] = static_cast<uint8_t>(label);
      missing += label == 255;
    }
    __stcs(reinterpret_cast<uint4*>(labels + c * 16), out.q);
  }
  for (uint64_t i = chunks * 16 + tid; i < elements; i += stride) {
    const int label = range_label(static_cast<float>(image[i]), table, ranges);
    labels[i] = static_cast<uint8_t>(label);
    missing += label == 255;
  }
  for (int o = 16; o > 0; o >>= 1) missing += __shfl_down_sync(0xffffffffu, missing, o);
  if ((threadIdx.x & 31) == 0 && missing) atomicAdd(unconverted, missing);
}

template <class T>
__host__ __device__ constexpr int lowest_value() {
  return std::is_signed<T>::value ? -(1 << (8 * sizeof(T) - 1)) : 0;
}

// 8- and 16-bit images: the label of every representable value is computed
// once (range_label on its float value, as above), and the image pass is a
// table lookup in shared memory.
template <class T>
__global__ void label_table_kernel(const float* __restrict__ first, const float* __restrict__ last, int ranges,
                                   uint8_t* __restrict__ lut) {
  __shared__ float table[2 * 255];
  for (int i = threadIdx.x; i < ranges; i += blockDim.x) {
    table[i] = first[i];
    table[ranges + i] = last[i];
  }
  __syncthreads();
  constexpr int kValues = 1 << (8 * sizeof(T));
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kValues) return;
  // index i holds value i + lowest (two's complement offset for signed types)
  const T value = static_cast<T>(i + lowest_value<T>());
  lut[i] = static_cast<uint8_t>(range_label(static_cast<float>(value), table, ranges));
}

// Two 16-element chunks per thread and iteration, so that 2 * 16 * sizeof(T)
// bytes per thread are in flight before the lookups.
template <class T>
__global__ void __launch_bounds__(512) labels_lut_kernel(const T* __restrict__ image, uint64_t elements,
                                                          const uint8_t* __restrict__ lut, uint8_t* __restrict__ labels,
                                                          unsigned long long* __restrict__ unconverted) {
  constexpr int kValues = 1 << (8 * sizeof(T));
  extern __shared__ uint4 lut_words[];
  uint8_t* table = reinterpret_cast<uint8_t*>(lut_words);
  for (int i = threadIdx.x; i < kValues / 16; i += blockDim.x) lut_words[i] = reinterpret_cast<const uint4*>(lut)[i];
  __syncthreads();
  constexpr int kLowest = lowest_value<T>();
  unsigned long long missing = 0;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t chunks = elements / 16;
  union Chunk {
    uint4 q[sizeof(T)];
    T e[16];
  };
  union Out {
    uint4 q;
    uint8_t b[16];
  };
  for (uint64_t c = tid; c < chunks; c += 2 * stride) {
    const bool two = c + stride < chunks;
    Chunk in0, in1;
    const uint4* s0 = reinterpret_cast<const uint4*>(image + c * 16);
#pragma unroll
    for (int k = 0; k < static_cast<int>(sizeof(T)); ++k) in0.q[k] = __ldcs(s0 + k);
    if (two) {
      const uint4* s1 = reinterpret_cast<const uint4*>(image + (c + stride) * 16);
#pragma unroll
      for (int k = 0; k < static_cast<int>(sizeof(T)); ++k) in1.q[k] = __ldcs(s1 + k);
    }
    Out o0, o1;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      o0.b[j] = table[static_cast<int>(in0.e[j]) - kLowest];
      missing += o0.b[j] == 255;
    }
    __stcs(reinterpret_cast<uint4*>(labels + c * 16), o0.q);
    if (two) {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        o1.b[j] = table[static_cast<int>(in1.e[j]) - kLowest];
        missing += o1.b[j] == 255;
      }
      __stcs(reinterpret_cast<uint4*>(labels + (c + stride) * 16), o1.q);
    }
  }
  for (uint64_t i = chunks * 16 + tid; i < elements; i += stride) {
    const uint8_t l = table[static_cast<int>(image[i]) - kLowest];
    labels[i] = l;
    missing += l == 255;
  }
  for (int o = 16; o > 0; o >>= 1) missing += __shfl_down_sync(0xffffffffu, missing, o);
  if ((threadIdx.x & 31) == 0 && missing) atomicAdd(unconverted, missing);
}

int grid_for(const gg_volume* v) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v->device);
  const uint64_t blocks = (v->elements / 16 + 255) / 256;
  const uint64_t cap = static_cast<uint64_t>(sms) * 8;
  return static_cast<int>(blocks < cap ? (blocks ? blocks : 1) : cap);
}

template <class T>
void launch_draw(gg_volume* v, const DrawParams& p, int shape) {
  T* out = static_cast<T*>(v->data);
  const int g = grid_for(v);
  if (shape == GG_SHAPE_BOX) draw_kernel<T, GG_SHAPE_BOX><<<g, 256, 0, v->stream>>>(out, p);
  else if (shape == GG_SHAPE_TUBE) draw_kernel<T, GG_SHAPE_TUBE><<<g, 256, 0, v->stream>>>(out, p);
  else draw_kernel<T, GG_SHAPE_SPHERE><<<g, 256, 0, v->stream>>>(out, p);
}

template <class T>
void launch_labels(gg_volume* v, const float* first, const float* last, int ranges, uint8_t* labels,
                   unsigned long long* missing) {
  if constexpr (sizeof(T) <= 2) {
    constexpr int kValues = 1 << (8 * sizeof(T));
    label_table_kernel<T><<<(kValues + 255) / 256, 256, 0, v->stream>>>(first, last, ranges, v->lut);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v->device);
    const uint64_t blocks = (v->elements / 32 + 511) / 512;
    const int grid = static_cast<int>(blocks < static_cast<uint64_t>(2 * sms) ? (blocks ? blocks : 1) : 2 * sms);
    cudaFuncSetAttribute(labels_lut_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kValues);
    labels_lut_kernel<T><<<grid, 512, kValues, v->stream>>>(static_cast<const T*>(v->data), v->elements, v->lut, labels,
                                                             missing);
    return;
  }
  labels_kernel<T><<<grid_for(v), 256, 2 * ranges * sizeof(float), v->stream>>>(
      static_cast<const T*>(v->data), v->elements, first, last, ranges, labels, missing);
}

}  // namespace

extern "C" {

GG_API int gg_volume_create(int32_t device_index, int32_t met_type, const int32_t dimensions[3],
                            const float element_sizes[3], gg_volume** out) {
  if (!out || !dimensions || !element_sizes) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "NULL argument");
  *out = nullptr;
  const size_t eb = met_bytes(met_type);
  if (!eb) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "unknown MHD element type");
  uint64_t n = 1;
  for (int a = 0; a < 3; ++a) {
    if (dimensions[a] <= 0) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "volume dimensions must be positive");
    n *= static_cast<uint64_t>(dimensions[a]);
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device_index < 0 || device_index >= count)
    return gg::record_error(GG_ERROR_NO_DEVICE, "no such CUDA device");
  VOL_CUDA(cudaSetDevice(device_index));
  gg_volume* v = new gg_volume();
  v->device = device_index;
  v->met_type = met_type;
  std::memcpy(v->dimensions, dimensions, sizeof(v->dimensions));
  std::memcpy(v->element_sizes, element_sizes, sizeof(v->element_sizes));
  v->elements = n;
  v->element_bytes = eb;
  int rc = check(cudaStreamCreateWithFlags(&v->stream, cudaStreamNonBlocking), "cudaStreamCreateWithFlags");
  if (rc == GG_OK) rc = check(cudaEventCreate(&v->start), "cudaEventCreate");
  if (rc == GG_OK) rc = check(cudaEventCreate(&v->stop), "cudaEventCreate");
  if (rc == GG_OK) rc = check(cudaMalloc(&v->data, n * eb), "cudaMalloc");
  if (rc == GG_OK) rc = check(cudaMemsetAsync(v->data, 0, n * eb, v->stream), "cudaMemsetAsync");
  if (rc == GG_OK) rc = check(cudaStreamSynchronize(v->stream), "cudaStreamSynchronize");
  if (rc != GG_OK) {
    gg_volume_destroy(v);
    return rc;
  }
  *out = v;
  return GG_OK;
}

GG_API int gg_volume_destroy(gg_volume* v) {
  if (!v) return GG_OK;
  cudaSetDevice(v->device);
  if (v->stream) cudaStreamSynchronize(v->stream);
  if (v->data) cudaFree(v->data);
  if (v->labels) cudaFree(v->labels);
  if (v->table) cudaFree(v->table);
  if (v->lut) cudaFree(v->lut);
  if (v->missing) cudaFree(v->missing);
  if (v->start) cudaEventDestroy(v->start);
  if (v->stop) cudaEventDestroy(v->stop);
  if (v->stream) cudaStreamDestroy(v->stream);
  delete v;
  return GG_OK;
}

GG_API int gg_volume_upload(gg_volume* v, const void* host, uint64_t bytes) {
  if (!v || !host) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (bytes != v->elements * v->element_bytes) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "image size mismatch");
  VOL_CUDA(cudaSetDevice(v->device));
  VOL_CUDA(cudaMemcpyAsync(v->data, host, bytes, cudaMemcpyHostToDevice, v->stream));
  VOL_CUDA(cudaStreamSynchronize(v->stream));
  return GG_OK;
}

GG_API int gg_volume_download(gg_volume* v, void* host, uint64_t bytes) {
  if (!v || !host) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "NULL argument");
  if (bytes != v->elements * v->element_bytes) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "image size mismatch");
  VOL_CUDA(cudaSetDevice(v->device));
  VOL_CUDA(cudaMemcpyAsync(host, v->data, bytes, cudaMemcpyDeviceToHost, v->stream));
  VOL_CUDA(cudaStreamSynchronize(v->stream));
  return GG_OK;
}

GG_API int gg_volume_draw(gg_volume* v, const gg_shape* shapes, int32_t n) {
  if (!v || (n > 0 && !shapes) || n < 0) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "bad arguments");
  VOL_CUDA(cudaSetDevice(v->device));
  VOL_CUDA(cudaEventRecord(v->start, v->stream));
  for (int32_t k = 0; k < n; ++k) {
    const gg_shape& s = shapes[k];
    if (s.type < GG_SHAPE_BOX || s.type > GG_SHAPE_SPHERE) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "unknown shape");
    DrawParams p{};
    p.elements = v->elements;
    std::memcpy(p.dim, v->dimensions, sizeof(p.dim));
    std::memcpy(p.es, v->element_sizes, sizeof(p.es));
    std::memcpy(p.pos, s.position, sizeof(p.pos));
    p.label = s.label_value;
    std::memcpy(p.size, s.size, sizeof(p.size));
    switch (v->met_type) {
      case GG_MET_CHAR: launch_draw<int8_t>(v, p, s.type); break;
      case GG_MET_UCHAR: launch_draw<uint8_t>(v, p, s.type); break;
      case GG_MET_SHORT: launch_draw<int16_t>(v, p, s.type); break;
      case GG_MET_USHORT: launch_draw<uint16_t>(v, p, s.type); break;
      case GG_MET_INT: launch_draw<int32_t>(v, p, s.type); break;
      case GG_MET_UINT: launch_draw<uint32_t>(v, p, s.type); break;
      default: launch_draw<float>(v, p, s.type); break;
    }
    VOL_CUDA(cudaGetLastError());
  }
  VOL_CUDA(cudaEventRecord(v->stop, v->stream));
  VOL_CUDA(cudaStreamSynchronize(v->stream));
  VOL_CUDA(cudaEventElapsedTime(&v->last_ms, v->start, v->stop));
  return GG_OK;
}

GG_API int gg_volume_labels(gg_volume* v, const float* range_first, const float* range_last, int32_t ranges,
                            uint8_t* labels, int64_t* unconverted) {
  if (!v || !labels || ranges < 0 || ranges > 255 || (ranges > 0 && (!range_first || !range_last)))
    return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "bad arguments (at most 255 ranges)");
  VOL_CUDA(cudaSetDevice(v->device));
  if (!v->labels) {
    VOL_CUDA(cudaMalloc(&v->labels, v->elements));
    VOL_CUDA(cudaMalloc(&v->table, 2 * 255 * sizeof(float)));
    VOL_CUDA(cudaMalloc(&v->missing, sizeof(unsigned long long)));
    VOL_CUDA(cudaMalloc(&v->lut, 65536));
  }
  float* first = v->table;
  float* last = v->table + ranges;
  if (ranges > 0) {
    VOL_CUDA(cudaMemcpyAsync(first, range_first, ranges * sizeof(float), cudaMemcpyHostToDevice, v->stream));
    VOL_CUDA(cudaMemcpyAsync(last, range_last, ranges * sizeof(float), cudaMemcpyHostToDevice, v->stream));
  }
  VOL_CUDA(cudaMemsetAsync(v->missing, 0, sizeof(unsigned long long), v->stream));
  VOL_CUDA(cudaEventRecord(v->start, v->stream));
  switch (v->met_type) {
    case GG_MET_CHAR: launch_labels<int8_t>(v, first, last, ranges, v->labels, v->missing); break;
    case GG_MET_UCHAR: launch_labels<uint8_t>(v, first, last, ranges, v->labels, v->missing); break;
    case GG_MET_SHORT: launch_labels<int16_t>(v, first, last, ranges, v->labels, v->missing); break;
    case GG_MET_USHORT: launch_labels<uint16_t>(v, first, last, ranges, v->labels, v->missing); break;
    case GG_MET_INT: launch_labels<int32_t>(v, first, last, ranges, v->labels, v->missing); break;
    case GG_MET_UINT: launch_labels<uint32_t>(v, first, last, ranges, v->labels, v->missing); break;
    default: launch_labels<float>(v, first, last, ranges, v->labels, v->missing); break;
  }
  VOL_CUDA(cudaGetLastError());
  VOL_CUDA(cudaEventRecord(v->stop, v->stream));
  unsigned long long m = 0;
  VOL_CUDA(cudaMemcpyAsync(labels, v->labels, v->elements, cudaMemcpyDeviceToHost, v->stream));
  VOL_CUDA(cudaMemcpyAsync(&m, v->missing, sizeof(m), cudaMemcpyDeviceToHost, v->stream));
  VOL_CUDA(cudaStreamSynchronize(v->stream));
  VOL_CUDA(cudaEventElapsedTime(&v->last_ms, v->start, v->stop));
  if (unconverted) *unconverted = static_cast<int64_t>(m);
  return GG_OK;
}

GG_API int gg_volume_last_kernel_ms(gg_volume* v, float* milliseconds) {
  if (!v || !milliseconds) return gg::record_error(GG_ERROR_INVALID_ARGUMENT, "NULL argument");
  *milliseconds = v->last_ms;
  return GG_OK;
}

}  // extern "C"
