// 3x3 "same" convolutions of the scatter-surrogate U-Net on the 5th-generation
// tensor cores (tcgen05), one implicit GEMM per launch:
//
//   D[pixel][co] = sum over taps t and input channels c of X[pixel + offset(t)][c] * W[t][co][c]
//
// rows = 128 pixels per CTA (M = 128), columns = an output-channel tile
// (N <= 256), reduction = 9 taps x input channels in chunks of Kc = 16/32/64.
//
//   * operands: TMA (cp.async.bulk.tensor, no multicast) brings per (tap,
//     chunk) the 128 x Kc activation tile -- the box of a 4-D NHWC tensor map
//     at the tap's shifted (x, y), whose out-of-range rows and columns TMA
//     fills with zeros, which is exactly the convolution's zero padding -- and
//     the N x Kc weight tile, both K-major with the 128/64/32-byte swizzle of
//     their row length, into a ring of shared-memory stages;
//   * one thread issues tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) into a
//     TMEM accumulator and frees each stage with tcgen05.commit;
//   * all four warps read their 32 TMEM lanes (= 32 pixels) with tcgen05.ld
//     and store: mode 0 adds the bias, applies ReLU and writes BF16 (the
//     forward activations), mode 1 writes FP32 (data gradients, no bias).
//
// Every mbarrier wait is bounded; a wait that gives up sets *error, the CTA
// stops issuing work, waits (bounded) for the copies it started, frees its
// TMEM and returns.  The shared-memory and instruction descriptors are
// encoded by gg_umma_desc.cuh (the PTX ISA's bit layout).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "gg_umma_desc.cuh"

#include "gg_unet_umma.cuh"

namespace gg_umma {
namespace {

constexpr int kThreads = 128;
constexpr uint64_t kWaitNs = 2000000000ull;  // a wait gives up after 2 s of device time

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Waits for the phase of parity `parity` of the mbarrier at `bar`; gives up
// after kWaitNs, or as soon as another CTA of the launch has given up (*error).
__device__ __forceinline__ bool wait_parity(uint32_t bar, uint32_t parity, const int* error) {
  uint32_t done = 0;
  const uint64_t t0 = global_ns();
  for (uint32_t i = 0; !done; ++i) {
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (!done && (i & 255) == 255 && (global_ns() - t0 > kWaitNs || *reinterpret_cast<const volatile int*>(error)))
      break;
  }
  return done != 0;
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{ .reg .pred p; setp.ne.b32 p, %4, 0; tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p; }" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 lanes x 32 columns of FP32 from TMEM into 32 registers per thread.
__device__ __forceinline__ void tmem_load_32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// K-major operand tile of `rows` rows of `row_bytes` (32, 64 or 128) bytes,
// swizzled over the row length, 8-row groups `8 * row_bytes` apart.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, int row_bytes) {
  // leading byte offset unused by swizzled K-major tiles (encoded as 1 unit)
  return gg::umma_smem_desc(addr, 16, 8 * row_bytes, gg::umma_row_swizzle(row_bytes));
}

template <int kMode>
__global__ void __launch_bounds__(kThreads, 1) conv_umma_kernel(const __grid_constant__ CUtensorMap tmx,
                                                             const __grid_constant__ CUtensorMap tmw, ConvArgs a) {
  extern __shared__ unsigned char smem_raw[];
  // 1024-byte alignment for the 128-byte swizzle
  unsigned char* smem = smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023);
  const int S = a.stages;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + static_cast<size_t>(S) * a.stage_bytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + S;
  uint64_t* acc = bars + 2 * S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc + 1);
  __shared__ int cta_error;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * 128;
  const int n0 = blockIdx.y * a.n_tile;
  // the tile's first pixel: image b0, row y0, column x0 (boxes of whole rows / images)
  const int hw = a.height * a.width;
  const int b0 = m0 / hw, rem = m0 - b0 * hw, y0 = rem / a.width, x0 = rem - y0 * a.width;

  if (threadIdx.x == 0) {
    cta_error = 0;
    for (int i = 0; i < 2 * S + 1; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + i)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int chunks = a.cin / a.kc;
  const int iters = 9 * chunks;
  const uint32_t tx_bytes = static_cast<uint32_t>(a.a_bytes + a.b_bytes);
  if (warp == 0 && lane == 0) {
    // ---- producer: TMA loads of (tap, chunk) operand tiles ----
    int issued = 0;
    for (int it = 0; it < iters; ++it) {
      const int s = it % S;
      if (it >= S && !wait_parity(smem_addr(empty + s), ((it / S) + 1) & 1, a.error)) {
        atomicExch(&cta_error, 1);
        break;
      }
      const int tap = it / chunks, c0 = (it - tap * chunks) * a.kc;
      const int ky = tap / 3, kx = tap - 3 * ky;
      unsigned char* st = smem + static_cast<size_t>(s) * a.stage_bytes;
      const uint32_t bar = smem_addr(full + s);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx_bytes) : "memory");
      tma_load_4d(smem_addr(st), &tmx, c0, x0 + kx - 1, y0 + ky - 1, b0, bar);
      tma_load_3d(smem_addr(st + a.a_tile_bytes), &tmw, c0, n0, tap, bar);
      ++issued;
    }
    // copies still in flight land before the CTA can end (no-op when all were consumed)
    for (int it = issued > S ? issued - S : 0; it < issued; ++it)
      if (!wait_parity(smem_addr(full + it % S), (it / S) & 1, a.error)) atomicExch(&cta_error, 1);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    bool ok = true;
    for (int it = 0; it < iters && ok; ++it) {
      const int s = it % S;
      if (!wait_parity(smem_addr(full + s), (it / S) & 1, a.error)) {
        atomicExch(&cta_error, 1);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* st = smem + static_cast<size_t>(s) * a.stage_bytes;
      const uint64_t ad = smem_desc(smem_addr(st), a.kc * 2);
      const uint64_t bd = smem_desc(smem_addr(st + a.a_tile_bytes), a.kc * 2);
      for (int k = 0; k < a.kc / 16; ++k)  // 16 elements = 32 bytes = 2 descriptor units
        umma_f16(tmem, ad + 2 * k, bd + 2 * k, a.idesc, (it > 0 || k > 0) ? 1u : 0u);
      umma_commit(smem_addr(empty + s));
    }
    if (ok) umma_commit(smem_addr(acc));
  }
  __syncwarp();

  // ---- epilogue: TMEM lanes 32*warp .. +31 = pixels, columns = output channels ----
  const bool ready = wait_parity(smem_addr(acc), 0, a.error);
  if (!ready) atomicExch(&cta_error, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (!cta_error) {
    const int row = warp * 32 + lane;
    const long long pixel = static_cast<long long>(m0) + row;
    const bool valid = pixel < a.pixels;
    for (int cb = 0; cb < a.n_tile / 32; ++cb) {
      float v[32];
      tmem_load_32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cb * 32, v);
      if (!valid) continue;
      const int co = n0 + cb * 32;
      if (kMode == 0) {
        __align__(16) __nv_bfloat162 h[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const float x0v = fmaxf(v[2 * j] + a.bias[co + 2 * j], 0.0f);
          const float x1v = fmaxf(v[2 * j + 1] + a.bias[co + 2 * j + 1], 0.0f);
          h[j] = __floats2bfloat162_rn(x0v, x1v);
        }
        uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.y) + pixel * a.cout + co);
        const uint4* src = reinterpret_cast<const uint4*>(h);
#pragma unroll
        for (int j = 0; j < 4; ++j) dst[j] = src[j];
      } else {
        float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.y) + pixel * a.cout + co);
#pragma unroll
        for (int j = 0; j < 8; ++j) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
  if (threadIdx.x == 0 && cta_error) atomicExch(a.error, 1);
}

// Row-streaming 3x3 convolution for images whose width is a multiple of 128.
// A CTA owns `rows` (R) consecutive output rows of one 128-pixel row segment
// and keeps one TMEM accumulator (128 lanes x N columns) per output row.  Per
// input-channel chunk it loads the chunk's weights of all 9 taps once (one
// 3-D TMA box, double-buffered across chunks), then streams the input rows
// y0-1 .. y0+R, each as ONE 130-pixel tile (pixels x0-1 .. x0+128; TMA's zero
// fill supplies the padding outside the image).  The three x-taps of a row
// are the same tile addressed 0, 1 and 2 pixel rows in: the shared-memory
// swizzle is a function of the absolute address, so a K-major descriptor may
// start at any 128/64/32-byte row of a tile written by TMA (matrix base offset
// 0); the tile is padded to 136 rows so that every read stays inside it.
// Each input row feeds the up-to-three output rows it touches (y-taps), so an
// activation tile is written (R+2)/R times per output row instead of 9 times.
// An MMA costs max(N/2, operand bytes / 128) cycles here, so the single
// issuing thread keeps per-MMA work to a few adds on precomputed descriptors.
template <int kMode, int KC>
__global__ void __launch_bounds__(kThreads, 1) conv_rows_kernel(const __grid_constant__ CUtensorMap tmx,
                                                             const __grid_constant__ CUtensorMap tmw, ConvArgs a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023);
  const int S = a.stages, R = a.rows, N = a.n_tile;
  unsigned char* wbuf = smem;                                        // 2 x w_bytes
  unsigned char* ring = smem + 2 * static_cast<size_t>(a.w_bytes);  // S x a_tile_bytes
  uint64_t* bars = reinterpret_cast<uint64_t*>(ring + static_cast<size_t>(S) * a.a_tile_bytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + S;
  uint64_t* wfull = bars + 2 * S;
  uint64_t* wempty = bars + 2 * S + 2;
  uint64_t* acc = bars + 2 * S + 4;  // one per output row: its accumulator is complete
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc + R);
  __shared__ int cta_error;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int segs = a.width / 128, groups = a.height / R;
  const int seg = blockIdx.x % segs, t = blockIdx.x / segs;
  const int grp = t % groups, b0 = t / groups;
  const int x0 = seg * 128, y0 = grp * R;
  const int n0 = blockIdx.y * N;

  if (threadIdx.x == 0) {
    cta_error = 0;
    for (int i = 0; i < 2 * S + 4 + R; ++i)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + i)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int per_chunk = R + 2;  // input rows per chunk
  const uint32_t a_tx = static_cast<uint32_t>(a.a_bytes);
  const uint32_t w_tx = static_cast<uint32_t>(9 * N * KC * 2);
  if (warp == 0 && lane == 0) {
    // ---- producer: per chunk the 9-tap weight box, then the input rows ----
    int issued = 0, w_issued = 0;
    bool ok = true;
    for (int c = 0; c < a.chunks && ok; ++c) {
      const int wb = c & 1;
      if (c >= 2 && !wait_parity(smem_addr(wempty + wb), ((c >> 1) + 1) & 1, a.error)) {
        ok = false;
        break;
      }
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(wfull + wb)), "r"(w_tx)
                   : "memory");
      tma_load_3d(smem_addr(wbuf + wb * static_cast<size_t>(a.w_bytes)), &tmw, c * KC, n0, 0, smem_addr(wfull + wb));
      ++w_issued;
      for (int j = 0; j < per_chunk; ++j) {
        const int it = c * per_chunk + j;
        const int s = it % S;
        if (it >= S && !wait_parity(smem_addr(empty + s), ((it / S) + 1) & 1, a.error)) {
          ok = false;
          break;
        }
        const uint32_t bar = smem_addr(full + s);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(a_tx) : "memory");
        tma_load_4d(smem_addr(ring + static_cast<size_t>(s) * a.a_tile_bytes), &tmx, c * KC, x0 - 1, y0 - 1 + j, b0,
                    bar);
        ++issued;
      }
    }
    if (!ok) atomicExch(&cta_error, 1);
    // copies still in flight land before the CTA can end
    for (int it = issued > S ? issued - S : 0; it < issued; ++it)
      if (!wait_parity(smem_addr(full + it % S), (it / S) & 1, a.error)) atomicExch(&cta_error, 1);
    for (int c = w_issued > 2 ? w_issued - 2 : 0; c < w_issued; ++c)
      if (!wait_parity(smem_addr(wfull + (c & 1)), (c >> 1) & 1, a.error)) atomicExch(&cta_error, 1);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer ----
    // descriptors advance by constant steps (start address field = address / 16)
    const uint64_t ring_desc = smem_desc(smem_addr(ring), KC * 2);
    const uint64_t w_desc[2] = {smem_desc(smem_addr(wbuf), KC * 2),
                                smem_desc(smem_addr(wbuf + a.w_bytes), KC * 2)};
    const uint64_t stage_step = static_cast<uint64_t>(a.a_tile_bytes >> 4);
    const uint64_t tap_step = static_cast<uint64_t>((N * KC * 2) >> 4);
    constexpr uint64_t kRowStep = (KC * 2) >> 4;  // one pixel row of the tile
    bool ok = true;
    for (int c = 0; c < a.chunks && ok; ++c) {
      const int wb = c & 1;
      if (!wait_parity(smem_addr(wfull + wb), (c >> 1) & 1, a.error)) {
        ok = false;
        break;
      }
      const uint64_t wd = w_desc[wb];
      for (int j = 0; j < per_chunk; ++j) {
        const int it = c * per_chunk + j;
        const int s = it % S;
        if (!wait_parity(smem_addr(full + s), (it / S) & 1, a.error)) {
          ok = false;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint64_t ad = ring_desc + static_cast<uint64_t>(s) * stage_step;
#pragma unroll
        for (int ky = 0; ky < 3; ++ky) {
          const int r = j - ky;  // output row y0 + r takes input row y0 - 1 + j through y-tap ky
          if (r < 0 || r >= R) continue;
          const uint32_t d = tmem + static_cast<uint32_t>(r * N);
          const uint32_t fresh = (c == 0 && ky == 0) ? 1u : 0u;  // this row's first MMA starts its accumulator
#pragma unroll
          for (int kx = 0; kx < 3; ++kx) {
            const uint64_t bd = wd + static_cast<uint64_t>(3 * ky + kx) * tap_step;
            const uint64_t axd = ad + static_cast<uint64_t>(kx) * kRowStep;
#pragma unroll
            for (int k = 0; k < KC / 16; ++k)
              umma_f16(d, axd + 2 * k, bd + 2 * k, a.idesc, (fresh && kx == 0 && k == 0) ? 0u : 1u);
          }
        }
        umma_commit(smem_addr(empty + s));
        // In the last chunk, input row j brings output row j - 2 its last tap:
        // that row's accumulator is complete once these MMAs are, and its
        // epilogue can run while the later rows still load and multiply.
        if (c == a.chunks - 1 && j >= 2) umma_commit(smem_addr(acc + (j - 2)));
      }
      umma_commit(smem_addr(wempty + wb));
    }
    if (!ok) atomicExch(&cta_error, 1);
  }
  __syncwarp();

  // ---- epilogue, row by row as the rows complete: TMEM lanes 32*warp .. +31 =
  // pixels x0 + 32*warp + lane; columns r*N .. = row y0 + r ----
  {
    const int x = x0 + warp * 32 + lane;
    for (int r = 0; r < R; ++r) {
      // warp-uniform, so that the warp's tcgen05.ld below stays converged
      if (!__all_sync(0xffffffffu, wait_parity(smem_addr(acc + r), 0, a.error))) {
        atomicExch(&cta_error, 1);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const long long pixel = (static_cast<long long>(b0) * a.height + (y0 + r)) * a.width + x;
      for (int cb = 0; cb < N / 32; ++cb) {
        float v[32];
        tmem_load_32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(r * N + cb * 32), v);
        const int co = n0 + cb * 32;
        if (kMode == 0) {
          __align__(16) __nv_bfloat162 h[16];
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const float lo = fmaxf(v[2 * q] + a.bias[co + 2 * q], 0.0f);
            const float hi = fmaxf(v[2 * q + 1] + a.bias[co + 2 * q + 1], 0.0f);
            h[q] = __floats2bfloat162_rn(lo, hi);
          }
          uint4* dst = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.y) + pixel * a.cout + co);
          const uint4* src = reinterpret_cast<const uint4*>(h);
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = src[q];
        } else {
          float4* dst = reinterpret_cast<float4*>(static_cast<float*>(a.y) + pixel * a.cout + co);
#pragma unroll
          for (int q = 0; q < 8; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
  if (threadIdx.x == 0 && cta_error) atomicExch(a.error, 1);
}

// 32 lanes x 16 columns of FP32 from TMEM into 16 registers per thread.
__device__ __forceinline__ void tmem_load_16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// MN-major operand tile: 64 pixel rows (the reduction) of `atom` channels
// (32/64/128-byte rows, swizzled over that length), 8-row groups 16 * atom
// bytes apart, successive channel atoms `lbo` bytes apart.
__device__ __forceinline__ uint64_t smem_desc_mn(uint32_t addr, int atom, uint32_t lbo) {
  return gg::umma_smem_desc(addr, lbo, 8 * atom * 2, gg::umma_row_swizzle(2 * atom));
}

constexpr int kChunk = 64;               // pixels per reduction chunk
constexpr int kWgradATileBytes = 128 * kChunk * 2;

// Weight gradient: D[(tap, co)][ci] = sum over the CTA's pixels q of
// dY[q - offset(tap)][co] * X[q][ci].  The dY boxes are loaded at the shifted
// position (TMA zero-fills what falls outside the image, which is the
// convolution's zero padding seen from the other side), the X boxes at q.
__global__ void __launch_bounds__(kThreads, 1) wgrad_umma_kernel(const __grid_constant__ CUtensorMap tmdy,
                                                              const __grid_constant__ CUtensorMap tmx, WgradArgs a) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = smem_raw + ((1024 - (smem_addr(smem_raw) & 1023)) & 1023);
  const int S = a.stages;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + static_cast<size_t>(S) * a.stage_bytes);
  uint64_t* full = bars;
  uint64_t* empty = bars + S;
  uint64_t* acc = bars + 2 * S;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acc + 1);
  __shared__ int cta_error;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tap0 = (blockIdx.x / a.co_blocks) * a.taps_per_tile;
  const int co0 = (blockIdx.x % a.co_blocks) * a.co_tile;
  const int n0 = blockIdx.y * a.n_tile;
  const int c_begin = blockIdx.z * a.chunks_per_split;
  const int c_end = min(a.chunks, c_begin + a.chunks_per_split);
  const int iters = c_end - c_begin;
  const int taps_here = min(a.taps_per_tile, 9 - tap0);
  const int boxes_per_tap = a.co_tile / a.a_atom;
  const int a_boxes = taps_here * boxes_per_tap;
  const int b_boxes = a.n_tile / a.b_atom;
  const uint32_t tx_bytes = static_cast<uint32_t>(a_boxes * a.a_bytes_per_box + a.b_bytes);
  const int hw = a.height * a.width;

  if (threadIdx.x == 0) {
    cta_error = 0;
    for (int i = 0; i < 2 * S + 1; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + i)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                 "r"(a.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---- producer: per 64-pixel chunk, the shifted dY boxes of the tile's taps and the X boxes ----
    int issued = 0;
    for (int it = 0; it < iters; ++it) {
      const int s = it % S;
      if (it >= S && !wait_parity(smem_addr(empty + s), ((it / S) + 1) & 1, a.error)) {
        atomicExch(&cta_error, 1);
        break;
      }
      const int p0 = (c_begin + it) * kChunk;
      const int b0 = p0 / hw, rem = p0 - b0 * hw, y0 = rem / a.width, x0 = rem - y0 * a.width;
      unsigned char* st = smem + static_cast<size_t>(s) * a.stage_bytes;
      const uint32_t bar = smem_addr(full + s);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(tx_bytes) : "memory");
      for (int j = 0; j < a_boxes; ++j) {
        const int t = j / boxes_per_tap, cb = j - t * boxes_per_tap;
        const int tap = tap0 + t, ky = tap / 3, kx = tap - 3 * ky;
        tma_load_4d(smem_addr(st + j * a.a_bytes_per_box), &tmdy, co0 + cb * a.a_atom, x0 - (kx - 1), y0 - (ky - 1),
                    b0, bar);
      }
      for (int j = 0; j < b_boxes; ++j)
        tma_load_4d(smem_addr(st + kWgradATileBytes + j * a.b_atom * kChunk * 2), &tmx, n0 + j * a.b_atom, x0, y0, b0,
                    bar);
      ++issued;
    }
    for (int it = issued > S ? issued - S : 0; it < issued; ++it)
      if (!wait_parity(smem_addr(full + it % S), (it / S) & 1, a.error)) atomicExch(&cta_error, 1);
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: 4 x K=16 per chunk; K advances by two 8-row groups ----
    bool ok = true;
    const uint32_t a_step = (2 * 8 * a.a_atom * 2) >> 4, b_step = (2 * 8 * a.b_atom * 2) >> 4;
    for (int it = 0; it < iters && ok; ++it) {
      const int s = it % S;
      if (!wait_parity(smem_addr(full + s), (it / S) & 1, a.error)) {
        atomicExch(&cta_error, 1);
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* st = smem + static_cast<size_t>(s) * a.stage_bytes;
      const uint64_t ad = smem_desc_mn(smem_addr(st), a.a_atom, static_cast<uint32_t>(a.a_bytes_per_box));
      const uint64_t bd =
          smem_desc_mn(smem_addr(st + kWgradATileBytes), a.b_atom, static_cast<uint32_t>(a.b_atom * kChunk * 2));
      for (int k = 0; k < kChunk / 16; ++k)
        umma_f16(tmem, ad + k * a_step, bd + k * b_step, a.idesc, (it > 0 || k > 0) ? 1u : 0u);
      umma_commit(smem_addr(empty + s));
    }
    if (ok) umma_commit(smem_addr(acc));
  }
  __syncwarp();

  // ---- epilogue: TMEM lane = (tap, co) row, columns = input channels; add to dW ----
  const bool ready = wait_parity(smem_addr(acc), 0, a.error);
  if (!ready) atomicExch(&cta_error, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  __syncthreads();
  if (!cta_error && iters > 0) {
    const int row = warp * 32 + lane;
    const int t = row / a.co_tile;
    const bool valid = t < taps_here;
    const int tap = tap0 + t, co = co0 + row - t * a.co_tile;
    float* out = a.dw + (static_cast<size_t>(valid ? tap : 0) * a.cout + co) * a.cin + n0;
    for (int cb = 0; cb < a.n_tile / 16; ++cb) {
      float v[16];
      tmem_load_16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cb * 16, v);
      if (!valid) continue;
      float4* dst = reinterpret_cast<float4*>(out + cb * 16);
#pragma unroll
      for (int j = 0; j < 4; ++j) atomicAdd(dst + j, make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols));
  if (threadIdx.x == 0 && cta_error) atomicExch(a.error, 1);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

CUtensorMapSwizzle swizzle_for(int row_bytes) {
  return row_bytes == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
         : row_bytes == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                           : CU_TENSOR_MAP_SWIZZLE_32B;
}

int pow2_at_least(int v, int lo) {
  int p = lo;
  while (p < v) p <<= 1;
  return p;
}

bool is_pow2(int v) { return v > 0 && (v & (v - 1)) == 0; }

// Plan of the row-streaming kernel (width a multiple of 128).  Rows per CTA:
// R x N TMEM columns <= 256 so that two CTAs fit an SM (knob
// GGEMS_B200_CONV_ROWS: rows per CTA, a power of two; 0 selects the tile
// kernel); chunks of 64 / 32 / 16 channels, the widest whose two weight buffers
// and a ring of at least 3 row tiles fit two CTAs per SM (one if none does).
const char* make_rows_plan(ConvPlan* p, const void* x, const void* w, int batch, int height, int width, int cin,
                           int cout, int rows_knob, PFN_cuTensorMapEncodeTiled_v12000 fn) {
  ConvArgs& a = p->args;
  a.n_tile = cout <= 256 ? cout : (cout % 128 == 0 ? 128 : 64);
  if (cout % a.n_tile != 0 || a.n_tile % 32 != 0) return "unsupported output channel count";
  const int N = a.n_tile;
  int R = rows_knob > 0 ? rows_knob : 256 / N;
  while (R > 1 && R * N > 512) R >>= 1;
  if (R < 1) R = 1;
  if (R > height) R = height;
  if ((R & (R - 1)) != 0 || R * N > 512) return "rows per CTA must be a power of two with rows x channels <= 512";
  a.rows = R;
  a.tmem_cols = pow2_at_least(R * N, 32);
  auto w_bytes = [&](int kc) { return ((9 * N * kc * 2 + 1023) / 1024) * 1024; };
  auto tile_bytes = [&](int kc) { return ((136 * kc * 2 + 1023) / 1024) * 1024; };
  const int budgets[2] = {110 * 1024, 200 * 1024};  // two CTAs per SM, else one
  a.kc = 0;
  for (int budget : budgets) {
    for (int kc : {64, 32, 16}) {
      if (cin % kc != 0) continue;
      if (2 * w_bytes(kc) + 3 * tile_bytes(kc) <= budget) {
        a.kc = kc;
        break;
      }
    }
    if (a.kc) {
      a.stages = (budget - 2 * w_bytes(a.kc)) / tile_bytes(a.kc);
      break;
    }
  }
  if (a.kc == 0) return "weights of a chunk do not fit in shared memory";
  if (a.stages > 8) a.stages = 8;
  a.chunks = cin / a.kc;
  a.w_bytes = w_bytes(a.kc);
  a.a_tile_bytes = tile_bytes(a.kc);
  a.a_bytes = 130 * a.kc * 2;  // the 130 pixels TMA writes
  a.b_bytes = 9 * N * a.kc * 2;
  a.stage_bytes = a.a_tile_bytes;
  p->smem = 2 * static_cast<size_t>(a.w_bytes) + static_cast<size_t>(a.stages) * a.a_tile_bytes +
            (2 * a.stages + 4 + R) * 8 + 16 + 1024;
  const size_t tmem_cap_smem = 228 * 1024 / (512 / a.tmem_cols + 1) + 1;
  if (p->smem < tmem_cap_smem) p->smem = tmem_cap_smem;
  if (p->smem > 227 * 1024) return "row kernel does not fit in shared memory";
  a.idesc = gg::umma_idesc_bf16_f32(128, N, false, false);
  cuuint32_t ones[4] = {1, 1, 1, 1};
  cuuint64_t xd[4] = {static_cast<cuuint64_t>(cin), static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(height),
                      static_cast<cuuint64_t>(batch)};
  cuuint64_t xs[3] = {static_cast<cuuint64_t>(cin) * 2, static_cast<cuuint64_t>(width) * cin * 2,
                      static_cast<cuuint64_t>(height) * width * cin * 2};
  cuuint32_t xbox[4] = {static_cast<cuuint32_t>(a.kc), 130, 1, 1};
  if (fn(&p->tmap_x, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), xd, xs, xbox, ones,
         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(a.kc * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return "activation tensor map rejected";
  cuuint64_t wd[3] = {static_cast<cuuint64_t>(cin), static_cast<cuuint64_t>(cout), 9};
  cuuint64_t ws[2] = {static_cast<cuuint64_t>(cin) * 2, static_cast<cuuint64_t>(cout) * cin * 2};
  cuuint32_t wbox[3] = {static_cast<cuuint32_t>(a.kc), static_cast<cuuint32_t>(N), 9};
  if (fn(&p->tmap_w, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(w), wd, ws, wbox, ones,
         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(a.kc * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return "weight tensor map rejected";
  p->grid_m = batch * (height / R) * (width / 128);
  p->grid_n = cout / N;
  return nullptr;
}

}  // namespace

const char* make_plan(ConvPlan* p, const void* x, const void* w, int batch, int height, int width, int cin, int cout) {
  std::memset(p, 0, sizeof(*p));
  if (!is_pow2(width) || !is_pow2(height) || batch < 1) return "image sides must be powers of two";
  if (cin % 16 != 0 || cout % 32 != 0) return "channel counts must be multiples of 16 (in) and 32 (out)";
  auto fn = encode_fn();
  if (!fn) return "cuTensorMapEncodeTiled is not available";
  ConvArgs& a = p->args;
  a.height = height;
  a.width = width;
  a.cin = cin;
  a.cout = cout;
  a.pixels = static_cast<long long>(batch) * height * width;
  static const int rows_knob = [] {
    const char* e = std::getenv("GGEMS_B200_CONV_ROWS");
    return e ? std::atoi(e) : -1;
  }();
  if (width % 128 == 0 && rows_knob != 0) return make_rows_plan(p, x, w, batch, height, width, cin, cout, rows_knob, fn);
  a.kc = cin % 64 == 0 ? 64 : (cin % 32 == 0 ? 32 : 16);
  a.n_tile = cout <= 256 ? cout : (cout % 128 == 0 ? 128 : 64);
  if (cout > 256 && cout % a.n_tile != 0) return "unsupported output channel count";
  // small images: thinner output-channel tiles until about two CTAs per SM exist
  // (the 32^2 bottleneck has only 64 pixel tiles)
  {
    const long long m_tiles = (a.pixels + 127) / 128;
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    while (m_tiles * (cout / a.n_tile) < 2LL * sms && a.n_tile > 64 && (a.n_tile / 2) % 32 == 0 &&
           cout % (a.n_tile / 2) == 0)
      a.n_tile /= 2;
  }
  a.tmem_cols = pow2_at_least(a.n_tile, 32);
  a.a_tile_bytes = 128 * a.kc * 2;
  const int b_tile = a.n_tile * a.kc * 2;
  a.a_bytes = a.a_tile_bytes;
  a.b_bytes = b_tile;
  a.stage_bytes = a.a_tile_bytes + ((b_tile + 1023) / 1024) * 1024;
  // a ring of ~32 KB (at least 2 stages): several CTAs per SM, whose TMA
  // round trips and epilogues overlap, beat deeper rings in fewer CTAs
  // (measured on the 256^2 U-Net forward: 1.15 ms at 32 KB, 1.18 ms at 50 KB,
  // 1.40 ms at 100 KB)
  static const int ring_kb = [] {
    const char* e = std::getenv("GGEMS_B200_CONV_RING_KB");  // tuning knob, default 32
    const int v = e ? std::atoi(e) : 0;
    return v >= 16 && v <= 200 ? v : 32;
  }();
  a.stages = ring_kb * 1024 / a.stage_bytes;
  if (a.stages > 8) a.stages = 8;
  if (a.stages < 2) a.stages = 2;
  if (static_cast<size_t>(a.stages) * a.stage_bytes > 200 * 1024) return "operand tiles do not fit in shared memory";
  p->smem = static_cast<size_t>(a.stages) * a.stage_bytes + (2 * a.stages + 1) * 8 + 16 + 1024;
  // no more CTAs per SM than the 512 TMEM columns hold: shared memory caps residency
  const size_t tmem_cap_smem = 228 * 1024 / (512 / a.tmem_cols + 1) + 1;
  if (p->smem < tmem_cap_smem) p->smem = tmem_cap_smem;
  // instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128, N = n_tile
  a.idesc = gg::umma_idesc_bf16_f32(128, a.n_tile, false, false);
  // activation boxes: 128 pixels as whole rows, or whole images
  const int bw = width < 128 ? width : 128;
  const int bh = (128 / bw) < height ? 128 / bw : height;
  const int bb = 128 / (bw * bh);
  cuuint64_t xd[4] = {static_cast<cuuint64_t>(cin), static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(height),
                      static_cast<cuuint64_t>(batch)};
  cuuint64_t xs[3] = {static_cast<cuuint64_t>(cin) * 2, static_cast<cuuint64_t>(width) * cin * 2,
                      static_cast<cuuint64_t>(height) * width * cin * 2};
  cuuint32_t xbox[4] = {static_cast<cuuint32_t>(a.kc), static_cast<cuuint32_t>(bw), static_cast<cuuint32_t>(bh),
                        static_cast<cuuint32_t>(bb)};
  cuuint32_t ones[4] = {1, 1, 1, 1};
  if (fn(&p->tmap_x, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), xd, xs, xbox, ones,
         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(a.kc * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return "activation tensor map rejected";
  cuuint64_t wd[3] = {static_cast<cuuint64_t>(cin), static_cast<cuuint64_t>(cout), 9};
  cuuint64_t ws[2] = {static_cast<cuuint64_t>(cin) * 2, static_cast<cuuint64_t>(cout) * cin * 2};
  cuuint32_t wbox[3] = {static_cast<cuuint32_t>(a.kc), static_cast<cuuint32_t>(a.n_tile), 1};
  if (fn(&p->tmap_w, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(w), wd, ws, wbox, ones,
         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(a.kc * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return "weight tensor map rejected";
  p->grid_m = static_cast<int>((a.pixels + 127) / 128);
  p->grid_n = cout / a.n_tile;
  return nullptr;
}

cudaError_t launch(const ConvPlan& p, int mode, const float* bias, void* y, int* error, cudaStream_t stream) {
  ConvArgs a = p.args;
  a.bias = bias;
  a.y = y;
  a.error = error;
  dim3 grid(p.grid_m, p.grid_n);
  if (a.rows > 0) {
    using K = void (*)(const CUtensorMap, const CUtensorMap, ConvArgs);
    K k = nullptr;
    if (a.kc == 64) k = mode == 0 ? conv_rows_kernel<0, 64> : conv_rows_kernel<1, 64>;
    else if (a.kc == 32) k = mode == 0 ? conv_rows_kernel<0, 32> : conv_rows_kernel<1, 32>;
    else k = mode == 0 ? conv_rows_kernel<0, 16> : conv_rows_kernel<1, 16>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(p.smem));
    k<<<grid, kThreads, p.smem, stream>>>(p.tmap_x, p.tmap_w, a);
  } else if (mode == 0) {
    cudaFuncSetAttribute(conv_umma_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(p.smem));
    conv_umma_kernel<0><<<grid, kThreads, p.smem, stream>>>(p.tmap_x, p.tmap_w, a);
  } else {
    cudaFuncSetAttribute(conv_umma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(p.smem));
    conv_umma_kernel<1><<<grid, kThreads, p.smem, stream>>>(p.tmap_x, p.tmap_w, a);
  }
  return cudaGetLastError();
}

const char* make_wgrad_plan(WgradPlan* p, const void* x, const void* dy, int batch, int height, int width, int cin,
                            int cout) {
  std::memset(p, 0, sizeof(*p));
  if (!is_pow2(width) || !is_pow2(height) || batch < 1 || width * height < kChunk)
    return "image sides must be powers of two with at least 64 pixels per image";
  if (cin % 16 != 0) return "input channels must be a multiple of 16";
  if (!(cout == 32 || cout == 64 || cout % 128 == 0)) return "output channels must be 32, 64 or a multiple of 128";
  auto fn = encode_fn();
  if (!fn) return "cuTensorMapEncodeTiled is not available";
  WgradArgs& a = p->args;
  a.height = height;
  a.width = width;
  a.cin = cin;
  a.cout = cout;
  a.co_tile = cout < 128 ? cout : 128;
  a.taps_per_tile = 128 / a.co_tile;
  a.co_blocks = cout / a.co_tile;
  a.a_atom = a.co_tile < 64 ? a.co_tile : 64;
  a.n_tile = cin <= 256 ? cin : (cin % 128 == 0 ? 128 : (cin % 64 == 0 ? 64 : 0));
  if (a.n_tile == 0) return "unsupported input channel count";
  a.b_atom = a.n_tile % 64 == 0 ? 64 : (a.n_tile % 32 == 0 ? 32 : 16);
  a.tmem_cols = pow2_at_least(a.n_tile, 32);
  a.a_bytes_per_box = a.a_atom * kChunk * 2;
  a.b_bytes = a.n_tile * kChunk * 2;
  a.stage_bytes = kWgradATileBytes + ((a.b_bytes + 1023) / 1024) * 1024;
  a.stages = 96 * 1024 / a.stage_bytes;
  if (a.stages > 6) a.stages = 6;
  if (a.stages < 2) a.stages = 2;
  p->smem = static_cast<size_t>(a.stages) * a.stage_bytes + (2 * a.stages + 1) * 8 + 16 + 1024;
  const size_t tmem_cap_smem = 228 * 1024 / (512 / a.tmem_cols + 1) + 1;
  if (p->smem < tmem_cap_smem) p->smem = tmem_cap_smem;
  if (p->smem > 227 * 1024) return "operand tiles do not fit in shared memory";
  // MN-major: channels contiguous, pixels (the reduction) strided
  a.idesc = gg::umma_idesc_bf16_f32(128, a.n_tile, true, true);
  // 64-pixel boxes: a run of one row, or whole rows
  const int bw = width < kChunk ? width : kChunk;
  const int bh = (kChunk / bw) < height ? kChunk / bw : height;
  const int bb = kChunk / (bw * bh);
  cuuint32_t ones[4] = {1, 1, 1, 1};
  cuuint64_t dd[4] = {static_cast<cuuint64_t>(cout), static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(height),
                      static_cast<cuuint64_t>(batch)};
  cuuint64_t ds[3] = {static_cast<cuuint64_t>(cout) * 2, static_cast<cuuint64_t>(width) * cout * 2,
                      static_cast<cuuint64_t>(height) * width * cout * 2};
  cuuint32_t dbox[4] = {static_cast<cuuint32_t>(a.a_atom), static_cast<cuuint32_t>(bw), static_cast<cuuint32_t>(bh),
                        static_cast<cuuint32_t>(bb)};
  if (fn(&p->tmap_dy, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(dy), dd, ds, dbox, ones,
         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(a.a_atom * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return "gradient tensor map rejected";
  cuuint64_t xd[4] = {static_cast<cuuint64_t>(cin), static_cast<cuuint64_t>(width), static_cast<cuuint64_t>(height),
                      static_cast<cuuint64_t>(batch)};
  cuuint64_t xs[3] = {static_cast<cuuint64_t>(cin) * 2, static_cast<cuuint64_t>(width) * cin * 2,
                      static_cast<cuuint64_t>(height) * width * cin * 2};
  cuuint32_t xbox[4] = {static_cast<cuuint32_t>(a.b_atom), static_cast<cuuint32_t>(bw), static_cast<cuuint32_t>(bh),
                        static_cast<cuuint32_t>(bb)};
  if (fn(&p->tmap_x, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(x), xd, xs, xbox, ones,
         CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle_for(a.b_atom * 2), CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return "activation tensor map rejected";
  a.chunks = static_cast<int>(static_cast<long long>(batch) * height * width / kChunk);
  p->grid_m = ((9 + a.taps_per_tile - 1) / a.taps_per_tile) * a.co_blocks;
  p->grid_n = cin / a.n_tile;
  // split the pixels so that about two CTAs per SM exist; partial tiles are added to dW
  int sms = 148, dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = p->grid_m * p->grid_n;
  int splits = (2 * sms + tiles - 1) / tiles;
  if (splits > a.chunks) splits = a.chunks;
  if (splits < 1) splits = 1;
  a.chunks_per_split = (a.chunks + splits - 1) / splits;
  p->splits = (a.chunks + a.chunks_per_split - 1) / a.chunks_per_split;
  return nullptr;
}

cudaError_t launch_wgrad(const WgradPlan& p, float* dw, int* error, cudaStream_t stream) {
  if (reinterpret_cast<uintptr_t>(dw) & 15) return cudaErrorMisalignedAddress;
  WgradArgs a = p.args;
  a.dw = dw;
  a.error = error;
  cudaFuncSetAttribute(wgrad_umma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(p.smem));
  wgrad_umma_kernel<<<dim3(p.grid_m, p.grid_n, p.splits), kThreads, p.smem, stream>>>(p.tmap_dy, p.tmap_x, a);
  return cudaGetLastError();
}

}  // namespace gg_umma
