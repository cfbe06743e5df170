// tcgen05 implicit-GEMM 3x3 convolution of the scatter-surrogate U-Net
// (gg_unet_umma.cu).  A plan holds the two TMA tensor maps (NHWC BF16
// activations, [tap][cout][cin] BF16 weights) and the tile configuration of one
// convolution; it is made once per layer and direction and launched as often
// as needed (the tensors it points to must stay where they are).
#ifndef GG_UNET_UMMA_CUH
#define GG_UNET_UMMA_CUH

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace gg_umma {

struct ConvArgs {
  int height, width, cin, cout;
  long long pixels;   // batch * height * width
  int kc;             // input channels per reduction chunk (16, 32 or 64)
  int n_tile;         // output channels per CTA
  int tmem_cols;      // TMEM columns allocated (power of two >= n_tile)
  int stages;         // shared-memory ring depth
  int a_tile_bytes, a_bytes, b_bytes, stage_bytes;
  uint32_t idesc;     // tcgen05.mma instruction descriptor
  // row-streaming kernel (rows > 0, images at least 128 pixels wide): a CTA
  // computes `rows` output rows of one 128-pixel row segment
  int rows;           // output rows per CTA (0: the tile kernel)
  int chunks;         // cin / kc
  int w_bytes;        // one weight buffer: 9 taps x n_tile x kc BF16 (1024-aligned)
  const float* bias;  // mode 0 only
  void* y;            // mode 0: BF16 [pixels][cout]; mode 1: FP32 [pixels][cout]
  int* error;         // set to 1 when a wait gave up
};

struct ConvPlan {
  CUtensorMap tmap_x;
  CUtensorMap tmap_w;
  ConvArgs args;
  size_t smem;
  int grid_m, grid_n;
};

// x: [batch][height][width][cin] BF16, w: [9][cout][cin] BF16 (device).
// Images whose width is a multiple of 128 use the row-streaming kernel, the
// others the tile kernel.  Returns NULL, or why the shape is not supported.
const char* make_plan(ConvPlan* plan, const void* x, const void* w, int batch, int height, int width, int cin, int cout);

// mode 0: y = relu(conv + bias) as BF16; mode 1: y = conv as FP32.
cudaError_t launch(const ConvPlan& plan, int mode, const float* bias, void* y, int* error, cudaStream_t stream);

// Weight gradient of one 3x3 convolution on tcgen05:
//   dW[tap][co][ci] += sum over pixels q of dY[q - offset(tap)][co] * X[q][ci]
// rows = (tap, output channel) pairs (128 per tile: 1, 2 or 4 taps of 128, 64
// or 32 channels), columns = an input-channel tile, reduction = pixels in
// chunks of 64, split over CTAs whose partial tiles are added to dW (FP32).
struct WgradArgs {
  int height, width, cin, cout;
  int co_tile;        // output channels per tap in a tile (32, 64 or 128)
  int taps_per_tile;  // 128 / co_tile
  int co_blocks;      // cout / co_tile
  int a_atom, b_atom; // channels per TMA box of dY / X (16, 32 or 64)
  int n_tile;         // input channels per tile
  int tmem_cols;
  int stages, a_bytes_per_box, b_bytes, stage_bytes;
  int chunks, chunks_per_split;  // 64-pixel chunks in all, per CTA
  uint32_t idesc;
  float* dw;          // FP32 [9][cout][cin], accumulated into
  int* error;
};

struct WgradPlan {
  CUtensorMap tmap_dy;
  CUtensorMap tmap_x;
  WgradArgs args;
  size_t smem;
  int grid_m, grid_n, splits;
};

// x: [batch][height][width][cin] BF16 (layer input), dy: [batch][height][width][cout]
// BF16 (gradient before the ReLU).  Returns NULL, or why the shape is not supported.
const char* make_wgrad_plan(WgradPlan* plan, const void* x, const void* dy, int batch, int height, int width, int cin,
                            int cout);
cudaError_t launch_wgrad(const WgradPlan& plan, float* dw, int* error, cudaStream_t stream);

}  // namespace gg_umma

#endif
