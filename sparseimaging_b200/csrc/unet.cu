// Learned warm start for MFISTA: a U-Net (4 levels, 16-32-64-128 channels,
// BF16 weights, FP32 activations and accumulation) that maps the dirty
// image and the dirty beam of a problem to an initial image (clamped >= 0).
// It has no counterpart in the reference; MFISTA always runs from its output
// to the reference's own stopping rule, which alone decides when it stops.
//
// Everything runs on the GPU with the kernels of this file: 3x3 convolutions
// (forward; backward-data as the forward kernel over flipped, transposed
// weights; backward-weights as per-tile partial sums reduced in a fixed
// order, so training is deterministic), 2x2 max pooling, nearest 2x
// upsampling folded into the convolution that follows it, skip
// concatenation folded into the convolution's input, a 1x1 output layer
// fused with the loss, and Adam on FP32 master weights that are rounded to
// the BF16 copies the forward pass reads.
//
// Layout: activations NCHW float; weights [cout][cin][3][3].
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mfista_b200.h"

namespace unet {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define UN_CK(x)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (x);                                                               \
    if (e_ != cudaSuccess)                                                              \
      throw Error(e_ == cudaErrorMemoryAllocation ? MFISTA_ERR_NOMEM : MFISTA_ERR_CUDA, \
                  std::string(#x) + ": " + cudaGetErrorString(e_));                     \
  } while (0)
#define UN_LAUNCH() UN_CK(cudaGetLastError())

__host__ __device__ inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

// ---------------------------------------------------------------------------
// 3x3 convolution, stride 1, zero padding 1.
//   input channels [0, ca) come from `a` ([n][ca][ha][wa]; when a_up, ha =
//   H/2 and the input is a's nearest 2x upsampling), channels [ca, ca+cb)
//   from `b` ([n][cb][H][W]); when `amask` is set, a's values are multiplied
//   by (amask > 0) (the ReLU derivative in the backward pass; amask has a's
//   shape); out[n][co][y][x] (+)= bias[co] + sum w[co][ci][ky][kx] *
//   in[ci][y+ky-1][x+kx-1], ReLU when relu, added to out when accumulate.
// Block: a 16 x 16 output tile, 128 threads with two vertically adjacent
// pixels each, 16 output channels; input channels in chunks of 16 staged
// (with halo) in shared memory with their weights.
// ---------------------------------------------------------------------------
struct ConvArgs {
  const float* a;
  const float* amask;
  int ca, a_up;
  const float* b;
  int cb;
  const __nv_bfloat16* w;  // [cout][ca+cb][3][3]
  const float* bias;       // [cout] or null
  float* out;
  int cout, H, W, relu, accumulate;
};

constexpr int kCT = 16;  // tile edge
constexpr int kCO = 16;  // output channels per block
constexpr int kCI = 16;  // input channels per staged chunk

__global__ void __launch_bounds__(128) k_conv3x3(ConvArgs g) {
  __shared__ float s_in[kCI][kCT + 2][kCT + 3];
  __shared__ __align__(16) float s_w[kCI][9][kCO];
  const int tiles_x = cdiv(g.W, kCT);
  const int tx0 = (blockIdx.x % tiles_x) * kCT, ty0 = (blockIdx.x / tiles_x) * kCT;
  const int co0 = blockIdx.y * kCO, n = blockIdx.z;
  const int cin = g.ca + g.cb;
  const int lx = threadIdx.x & 15, ly = (threadIdx.x >> 4) * 2;  // pixels (lx, ly), (lx, ly + 1)
  float acc[2][kCO];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int c = 0; c < kCO; ++c) acc[p][c] = 0.f;
  const int ha = g.a_up ? g.H / 2 : g.H, wa = g.a_up ? g.W / 2 : g.W;
  for (int c0 = 0; c0 < cin; c0 += kCI) {
    const int nc = min(kCI, cin - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < kCI * (kCT + 2) * (kCT + 2); t += blockDim.x) {
      const int ci = t / ((kCT + 2) * (kCT + 2));
      const int r = t - ci * (kCT + 2) * (kCT + 2);
      const int yy = r / (kCT + 2), xx = r - yy * (kCT + 2);
      const int y = ty0 + yy - 1, x = tx0 + xx - 1;
      float v = 0.f;
      if (ci < nc && y >= 0 && y < g.H && x >= 0 && x < g.W) {
        const int c = c0 + ci;
        if (c < g.ca) {
          const int sy = g.a_up ? y >> 1 : y, sx = g.a_up ? x >> 1 : x;
          const size_t idx = (((size_t)n * g.ca + c) * ha + sy) * wa + sx;
          v = g.a[idx];
          if (g.amask && !(g.amask[idx] > 0.f)) v = 0.f;
        } else {
          v = g.b[(((size_t)n * g.cb + (c - g.ca)) * g.H + y) * g.W + x];
        }
      }
      s_in[ci][yy][xx] = v;
    }
    for (int t = threadIdx.x; t < kCI * 9 * kCO; t += blockDim.x) {
      const int ci = t / (9 * kCO);
      const int r = t - ci * 9 * kCO;
      const int k = r / kCO, co = r - k * kCO;
      float v = 0.f;
      if (ci < nc && co0 + co < g.cout) v = __bfloat162float(g.w[((size_t)(co0 + co) * cin + c0 + ci) * 9 + k]);
      s_w[ci][k][co] = v;
    }
    __syncthreads();
    for (int ci = 0; ci < nc; ++ci) {
      float in[4][3];
#pragma unroll
      for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) in[r][c] = s_in[ci][ly + r][lx + c];
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        const int ky = k / 3, kx = k - ky * 3;
        const float i0 = in[ky][kx], i1 = in[ky + 1][kx];
        const float4* wp = reinterpret_cast<const float4*>(&s_w[ci][k][0]);
#pragma unroll
        for (int q = 0; q < kCO / 4; ++q) {
          const float4 w4 = wp[q];
          acc[0][4 * q + 0] += w4.x * i0;
          acc[0][4 * q + 1] += w4.y * i0;
          acc[0][4 * q + 2] += w4.z * i0;
          acc[0][4 * q + 3] += w4.w * i0;
          acc[1][4 * q + 0] += w4.x * i1;
          acc[1][4 * q + 1] += w4.y * i1;
          acc[1][4 * q + 2] += w4.z * i1;
          acc[1][4 * q + 3] += w4.w * i1;
        }
      }
    }
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const int y = ty0 + ly + p, x = tx0 + lx;
    if (y >= g.H || x >= g.W) continue;
#pragma unroll
    for (int c = 0; c < kCO; ++c) {
      const int co = co0 + c;
      if (co >= g.cout) break;
      float v = acc[p][c] + (g.bias ? g.bias[co] : 0.f);
      if (g.relu) v = fmaxf(v, 0.f);
      float* o = g.out + (((size_t)n * g.cout + co) * g.H + y) * g.W + x;
      *o = g.accumulate ? *o + v : v;
    }
  }
}

// ---------------------------------------------------------------------------
// The same 3x3 convolution as an implicit GEMM on the tensor cores
// (mma.sync m16n8k16, BF16 operands, FP32 accumulation):
//   out[co][pix] = sum_{tap, ci} W[co][ci][tap] X[ci][pix + tap]
// with K ordered tap-major (one k16 step = one tap x 16 input channels).
// The weights are BF16 already; an FP32 activation x enters as the two BF16
// planes hi = bf16(x), lo = bf16(x - hi), whose sum is x to 2^-18 relative,
// so every product is W hi + W lo, two MMAs, accumulated in FP32.
// Block: a 16 x 16 output tile and 16 * MT output channels, 8 warps; warp w
// owns output rows 2w, 2w + 1 (four n8 tiles of 8 pixels).  Per chunk of 16
// input channels the halo tile (18 x 18 pixels, channel-minor, both planes)
// and the chunk's weights ([tap][co][ci]) are staged in shared memory with
// 24 BF16 per row, which makes the fragment loads bank-conflict free.
// Deterministic: the MMA sequence is fixed.
// ---------------------------------------------------------------------------
constexpr int kTcRow = 12;                       // 32-bit words per staged pixel / weight row (16 used)
constexpr int kTcHalo = (kCT + 2) * (kCT + 2);   // 324 halo pixels

__device__ __forceinline__ void mma_bf16_16816(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int MT>
__global__ void __launch_bounds__(256) k_conv3x3_tc(ConvArgs g) {
  constexpr int CO = 16 * MT;
  extern __shared__ __align__(16) uint32_t s_tc[];
  uint32_t* s_x = s_tc;                                  // [2][324][kTcRow]
  uint32_t* s_w = s_tc + 2 * kTcHalo * kTcRow;           // [9][CO][kTcRow]
  __nv_bfloat16* s_x16 = reinterpret_cast<__nv_bfloat16*>(s_x);
  __nv_bfloat16* s_w16 = reinterpret_cast<__nv_bfloat16*>(s_w);
  const int tiles_x = cdiv(g.W, kCT);
  const int tx0 = (blockIdx.x % tiles_x) * kCT, ty0 = (blockIdx.x / tiles_x) * kCT;
  const int co0 = blockIdx.y * CO, n = blockIdx.z;
  const int cin = g.ca + g.cb;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gid = lane >> 2, tig = lane & 3;
  float acc[MT][4][4];
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[m][j][e] = 0.f;
  const int ha = g.a_up ? g.H / 2 : g.H, wa = g.a_up ? g.W / 2 : g.W;
  for (int c0 = 0; c0 < cin; c0 += kCI) {
    __syncthreads();  // the previous chunk's fragments have been read
    for (int t = threadIdx.x; t < kCI * kTcHalo; t += blockDim.x) {
      const int ci = t / kTcHalo, pix = t - ci * kTcHalo;
      const int yy = pix / (kCT + 2), xx = pix - yy * (kCT + 2);
      const int y = ty0 + yy - 1, x = tx0 + xx - 1;
      const int c = c0 + ci;
      float v = 0.f;
      if (c < cin && y >= 0 && y < g.H && x >= 0 && x < g.W) {
        if (c < g.ca) {
          const int sy = g.a_up ? y >> 1 : y, sx = g.a_up ? x >> 1 : x;
          const size_t idx = (((size_t)n * g.ca + c) * ha + sy) * wa + sx;
          v = g.a[idx];
          if (g.amask && !(g.amask[idx] > 0.f)) v = 0.f;
        } else {
          v = g.b[(((size_t)n * g.cb + (c - g.ca)) * g.H + y) * g.W + x];
        }
      }
      const __nv_bfloat16 hi = __float2bfloat16_rn(v);
      const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
      s_x16[(size_t)pix * (2 * kTcRow) + ci] = hi;
      s_x16[(size_t)(kTcHalo + pix) * (2 * kTcRow) + ci] = lo;
    }
    for (int t = threadIdx.x; t < 9 * CO * kCI; t += blockDim.x) {
      const int ci = t % kCI, r = t / kCI, co = r % CO, tap = r / CO;
      __nv_bfloat16 w = __float2bfloat16_rn(0.f);
      if (co0 + co < g.cout && c0 + ci < cin) w = g.w[((size_t)(co0 + co) * cin + c0 + ci) * 9 + tap];
      s_w16[(size_t)(tap * CO + co) * (2 * kTcRow) + ci] = w;
    }
    __syncthreads();
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
      const int ky = tap / 3, kx = tap - ky * 3;
      uint32_t a[MT][4];
#pragma unroll
      for (int m = 0; m < MT; ++m) {
        const uint32_t* w0 = s_w + (size_t)(tap * CO + m * 16 + gid) * kTcRow + tig;
        const uint32_t* w8 = w0 + 8 * kTcRow;
        a[m][0] = w0[0];
        a[m][1] = w8[0];
        a[m][2] = w0[4];
        a[m][3] = w8[4];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int row = 2 * warp + (j >> 1), x0 = (j & 1) * 8;
        const int hp = (row + ky) * (kCT + 2) + x0 + gid + kx;
#pragma unroll
        for (int pl = 0; pl < 2; ++pl) {
          const uint32_t* bx = s_x + (size_t)(pl * kTcHalo + hp) * kTcRow + tig;
          const uint32_t b0 = bx[0], b1 = bx[4];
#pragma unroll
          for (int m = 0; m < MT; ++m) mma_bf16_16816(acc[m][j], a[m], b0, b1);
        }
      }
    }
  }
#pragma unroll
  for (int m = 0; m < MT; ++m)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int y = ty0 + 2 * warp + (j >> 1);
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int co = co0 + m * 16 + gid + (e >> 1) * 8;
        const int x = tx0 + (j & 1) * 8 + tig * 2 + (e & 1);
        if (co >= g.cout || y >= g.H || x >= g.W) continue;
        float v = acc[m][j][e] + (g.bias ? g.bias[co] : 0.f);
        if (g.relu) v = fmaxf(v, 0.f);
        float* o = g.out + (((size_t)n * g.cout + co) * g.H + y) * g.W + x;
        *o = g.accumulate ? *o + v : v;
      }
    }
}

template <int MT> constexpr size_t conv_tc_smem() { return sizeof(uint32_t) * (2 * kTcHalo + 9 * 16 * MT) * kTcRow; }

// weights of the backward-data convolution: wt[ci][co][k] = w[co][ci][8 - k]
__global__ void k_flip_transpose(const __nv_bfloat16* __restrict__ w, int cout, int cin,
                                 __nv_bfloat16* __restrict__ wt) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cout * cin * 9) return;
  int co = t / (cin * 9), r = t - co * cin * 9, ci = r / 9, k = r - ci * 9;
  wt[((size_t)ci * cout + co) * 9 + (8 - k)] = w[t];
}

// ---------------------------------------------------------------------------
// weight gradient: dw[co][ci][k] = sum_{n,y,x} g[n][co][y][x] m * in[n][ci][y+ky-1][x+kx-1]
// with g masked by (gmask > 0) and in = concat(up?(a), b) as in k_conv3x3.
// Block: one 16 x 16 pixel tile of one image, 16 output x 16 input
// channels; thread (co, ci) keeps 9 sums; partials [tile][cout][cin][9] are
// reduced in tile order by k_reduce_partials (deterministic).
// ---------------------------------------------------------------------------
struct WgradArgs {
  const float* g;
  const float* gmask;
  const float* a;
  int ca, a_up;
  const float* b;
  int cb;
  float* part;  // [ntiles][cout][cin][9]
  int cout, H, W;
};

__global__ void __launch_bounds__(256) k_conv3x3_wgrad(WgradArgs g) {
  __shared__ float s_g[kCO][kCT * kCT];
  __shared__ float s_in[kCI][kCT + 2][kCT + 3];
  const int tiles_x = cdiv(g.W, kCT), tiles_y = cdiv(g.H, kCT);
  const int tile = blockIdx.x;  // over n * tiles
  const int n = tile / (tiles_x * tiles_y), tr = tile - n * tiles_x * tiles_y;
  const int tx0 = (tr % tiles_x) * kCT, ty0 = (tr / tiles_x) * kCT;
  const int co0 = blockIdx.y * kCO, ci0 = blockIdx.z * kCI;
  const int cin = g.ca + g.cb;
  const int ha = g.a_up ? g.H / 2 : g.H, wa = g.a_up ? g.W / 2 : g.W;
  for (int t = threadIdx.x; t < kCO * kCT * kCT; t += blockDim.x) {
    const int co = t / (kCT * kCT), p = t - co * kCT * kCT;
    const int y = ty0 + p / kCT, x = tx0 + p % kCT;
    float v = 0.f;
    if (co0 + co < g.cout && y < g.H && x < g.W) {
      const size_t idx = (((size_t)n * g.cout + co0 + co) * g.H + y) * g.W + x;
      v = g.g[idx];
      if (g.gmask && !(g.gmask[idx] > 0.f)) v = 0.f;
    }
    s_g[co][p] = v;
  }
  for (int t = threadIdx.x; t < kCI * (kCT + 2) * (kCT + 2); t += blockDim.x) {
    const int ci = t / ((kCT + 2) * (kCT + 2));
    const int r = t - ci * (kCT + 2) * (kCT + 2);
    const int yy = r / (kCT + 2), xx = r - yy * (kCT + 2);
    const int y = ty0 + yy - 1, x = tx0 + xx - 1;
    const int c = ci0 + ci;
    float v = 0.f;
    if (c < cin && y >= 0 && y < g.H && x >= 0 && x < g.W) {
      if (c < g.ca) {
        const int sy = g.a_up ? y >> 1 : y, sx = g.a_up ? x >> 1 : x;
        v = g.a[(((size_t)n * g.ca + c) * ha + sy) * wa + sx];
      } else {
        v = g.b[(((size_t)n * g.cb + (c - g.ca)) * g.H + y) * g.W + x];
      }
    }
    s_in[ci][yy][xx] = v;
  }
  __syncthreads();
  const int co = threadIdx.x >> 4, ci = threadIdx.x & 15;
  float s[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) s[k] = 0.f;
  for (int p = 0; p < kCT * kCT; ++p) {
    const int py = p / kCT, px = p - py * kCT;
    const float gv = s_g[co][p];
#pragma unroll
    for (int k = 0; k < 9; ++k) s[k] += gv * s_in[ci][py + k / 3][px + k % 3];
  }
  if (co0 + co < g.cout && ci0 + ci < cin) {
    float* o = g.part + (((size_t)tile * g.cout + co0 + co) * cin + ci0 + ci) * 9;
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = s[k];
  }
}

// The weight gradient on the tensor cores: per 16 x 16 pixel tile,
//   part[tile][co][ci][tap] = sum_{pix} G[co][pix] X[ci][pix + tap],
// a GEMM with M = 16 output channels, N = 16 input channels per tap and
// K = the tile's 256 pixels (16 k16 steps, one pixel row each).  G (the
// masked output gradient) and X (the input, as in k_conv3x3) are FP32 and
// enter as BF16 hi/lo planes; the three products hi*hi + hi*lo + lo*hi are
// accumulated in FP32 (lo*lo, ~2^-18 of the rest, is left out).  Nine warps,
// one per tap; the partials go to the same layout as k_conv3x3_wgrad's and
// are reduced over tiles in tile order by k_reduce_partials.
constexpr int kWgG = 132;  // 32-bit words per staged G row (256 pixels + pad)
constexpr int kWgX = 164;  // 32-bit words per staged X channel (324 halo pixels + pad)

__global__ void __launch_bounds__(288) k_conv3x3_wgrad_tc(WgradArgs g) {
  extern __shared__ __align__(16) uint32_t s_wg[];
  uint32_t* s_g = s_wg;                   // [2][16][kWgG]
  uint32_t* s_x = s_wg + 2 * 16 * kWgG;   // [2][16][kWgX]
  __nv_bfloat16* s_g16 = reinterpret_cast<__nv_bfloat16*>(s_g);
  __nv_bfloat16* s_x16 = reinterpret_cast<__nv_bfloat16*>(s_x);
  const int tiles_x = cdiv(g.W, kCT), tiles_y = cdiv(g.H, kCT);
  const int tile = blockIdx.x;  // over n * tiles
  const int n = tile / (tiles_x * tiles_y), tr = tile - n * tiles_x * tiles_y;
  const int tx0 = (tr % tiles_x) * kCT, ty0 = (tr / tiles_x) * kCT;
  const int co0 = blockIdx.y * 16, ci0 = blockIdx.z * kCI;
  const int cin = g.ca + g.cb;
  const int ha = g.a_up ? g.H / 2 : g.H, wa = g.a_up ? g.W / 2 : g.W;
  for (int t = threadIdx.x; t < 16 * kCT * kCT; t += blockDim.x) {
    const int co = t / (kCT * kCT), p = t - co * kCT * kCT;
    const int y = ty0 + p / kCT, x = tx0 + p % kCT;
    float v = 0.f;
    if (co0 + co < g.cout && y < g.H && x < g.W) {
      const size_t idx = (((size_t)n * g.cout + co0 + co) * g.H + y) * g.W + x;
      v = g.g[idx];
      if (g.gmask && !(g.gmask[idx] > 0.f)) v = 0.f;
    }
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    s_g16[(size_t)co * (2 * kWgG) + p] = hi;
    s_g16[(size_t)(16 + co) * (2 * kWgG) + p] = __float2bfloat16_rn(v - __bfloat162float(hi));
  }
  for (int t = threadIdx.x; t < kCI * kTcHalo; t += blockDim.x) {
    const int ci = t / kTcHalo, pix = t - ci * kTcHalo;
    const int yy = pix / (kCT + 2), xx = pix - yy * (kCT + 2);
    const int y = ty0 + yy - 1, x = tx0 + xx - 1;
    const int c = ci0 + ci;
    float v = 0.f;
    if (c < cin && y >= 0 && y < g.H && x >= 0 && x < g.W) {
      if (c < g.ca) {
        const int sy = g.a_up ? y >> 1 : y, sx = g.a_up ? x >> 1 : x;
        v = g.a[(((size_t)n * g.ca + c) * ha + sy) * wa + sx];
      } else {
        v = g.b[(((size_t)n * g.cb + (c - g.ca)) * g.H + y) * g.W + x];
      }
    }
    const __nv_bfloat16 hi = __float2bfloat16_rn(v);
    s_x16[(size_t)ci * (2 * kWgX) + pix] = hi;
    s_x16[(size_t)(16 + ci) * (2 * kWgX) + pix] = __float2bfloat16_rn(v - __bfloat162float(hi));
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, tap = threadIdx.x >> 5;  // warp = tap
  const int gid = lane >> 2, tig = lane & 3;
  const int ky = tap / 3, kx = tap - ky * 3;
  float acc[2][4];
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) acc[j][e] = 0.f;
  auto pack = [](__nv_bfloat16 lo16, __nv_bfloat16 hi16) -> uint32_t {
    return (uint32_t)__bfloat16_as_ushort(lo16) | ((uint32_t)__bfloat16_as_ushort(hi16) << 16);
  };
#pragma unroll 1
  for (int py = 0; py < kCT; ++py) {  // k16 step: pixels (py, 0..15)
    uint32_t a[2][4];                   // G planes: rows co = gid (+8), k = pixel
#pragma unroll
    for (int pl = 0; pl < 2; ++pl) {
      const uint32_t* r0 = s_g + (size_t)(pl * 16 + gid) * kWgG + py * (kCT / 2) + tig;
      const uint32_t* r8 = r0 + 8 * kWgG;
      a[pl][0] = r0[0];
      a[pl][1] = r8[0];
      a[pl][2] = r0[4];
      a[pl][3] = r8[4];
    }
    const int hrow = (py + ky) * (kCT + 2) + kx;  // halo index of pixel (py, 0) shifted by the tap
#pragma unroll
    for (int j = 0; j < 2; ++j) {  // n8 tiles: input channels 8j .. 8j+7
      uint32_t b[2][2];
#pragma unroll
      for (int pl = 0; pl < 2; ++pl) {
        const __nv_bfloat16* xr = s_x16 + (size_t)(pl * 16 + 8 * j + gid) * (2 * kWgX) + hrow;
        b[pl][0] = pack(xr[tig * 2], xr[tig * 2 + 1]);
        b[pl][1] = pack(xr[tig * 2 + 8], xr[tig * 2 + 9]);
      }
      mma_bf16_16816(acc[j], a[0], b[0][0], b[0][1]);  // hi * hi
      mma_bf16_16816(acc[j], a[0], b[1][0], b[1][1]);  // hi * lo
      mma_bf16_16816(acc[j], a[1], b[0][0], b[0][1]);  // lo * hi
    }
  }
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int co = co0 + gid + (e >> 1) * 8, ci = ci0 + 8 * j + tig * 2 + (e & 1);
      if (co < g.cout && ci < cin)
        g.part[(((size_t)tile * g.cout + co) * cin + ci) * 9 + tap] = acc[j][e];
    }
}

constexpr size_t kWgradTcSmem = sizeof(uint32_t) * (2 * 16 * kWgG + 2 * 16 * kWgX);

// out[i] = sum_t part[t][i] (t ascending), i < len
__global__ void k_reduce_partials(const float* __restrict__ part, int ntiles, long len, float* __restrict__ out) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= len) return;
  float s = 0.f;
  for (int t = 0; t < ntiles; ++t) s += part[(size_t)t * len + i];
  out[i] = s;
}

// bias gradient: db[co] = sum_{n,y,x} g m (one block per channel, fixed order)
__global__ void k_bias_grad(const float* __restrict__ g, const float* __restrict__ gmask, int n, int cout, int hw,
                            float* __restrict__ db) {
  __shared__ float sh[256];
  const int co = blockIdx.x;
  float s = 0.f;
  for (int i = 0; i < n; ++i) {
    const float* gp = g + ((size_t)i * cout + co) * hw;
    const float* mp = gmask ? gmask + ((size_t)i * cout + co) * hw : nullptr;
    for (int p = threadIdx.x; p < hw; p += blockDim.x) {
      float v = gp[p];
      if (mp && !(mp[p] > 0.f)) v = 0.f;
      s += v;
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[co] = sh[0];
}

// 2x2 max pooling (H, W even) and its gradient (to the first maximum)
__global__ void k_maxpool(const float* __restrict__ in, int nc, int H, int W, float* __restrict__ out) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int h = H / 2, w = W / 2;
  if (t >= (long)nc * h * w) return;
  const int c = (int)(t / (h * w)), r = (int)(t - (long)c * h * w), y = r / w, x = r - y * w;
  const float* p = in + ((size_t)c * H + 2 * y) * W + 2 * x;
  out[t] = fmaxf(fmaxf(p[0], p[1]), fmaxf(p[W], p[W + 1]));
}

__global__ void k_maxpool_grad(const float* __restrict__ in, const float* __restrict__ gout, int nc, int H, int W,
                               float* __restrict__ gin) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int h = H / 2, w = W / 2;
  if (t >= (long)nc * h * w) return;
  const int c = (int)(t / (h * w)), r = (int)(t - (long)c * h * w), y = r / w, x = r - y * w;
  const size_t base = ((size_t)c * H + 2 * y) * W + 2 * x;
  const float v[4] = {in[base], in[base + 1], in[base + W], in[base + W + 1]};
  int am = 0;
  for (int k = 1; k < 4; ++k)
    if (v[k] > v[am]) am = k;
  const size_t off[4] = {0, 1, (size_t)W, (size_t)W + 1};
  for (int k = 0; k < 4; ++k) gin[base + off[k]] += (k == am) ? gout[t] : 0.f;
}

// gradient of a nearest 2x upsampling: glow[c][y][x] = sum of the 2x2 block
__global__ void k_upsample_grad(const float* __restrict__ ghigh, int nc, int h, int w, float* __restrict__ glow) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nc * h * w) return;
  const int c = (int)(t / (h * w)), r = (int)(t - (long)c * h * w), y = r / w, x = r - y * w;
  const float* p = ghigh + ((size_t)c * 2 * h + 2 * y) * (2 * w) + 2 * x;
  glow[t] = p[0] + p[1] + p[2 * w] + p[2 * w + 1];
}

// output layer: s = b + sum_c w[c] h[c], out = max(0, s) (the initial image
// is clamped); with a target, the loss is the mean squared error of the
// unclamped s (so the gradient never dies at the clamp): per-pixel squared
// error, d loss / d s and d loss / d h
__global__ void k_head(const float* __restrict__ h, int n, int c16, int hw, const __nv_bfloat16* __restrict__ w,
                       const float* __restrict__ bias, float* __restrict__ out, const float* __restrict__ target,
                       float* __restrict__ sq, float* __restrict__ gh, float* __restrict__ gpre) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n * hw) return;
  const int i = (int)(t / hw), p = (int)(t - (long)i * hw);
  float s = bias[0];
  for (int c = 0; c < c16; ++c) s += __bfloat162float(w[c]) * h[((size_t)i * c16 + c) * hw + p];
  out[t] = fmaxf(s, 0.f);
  if (target) {
    const float d = s - target[t];
    sq[t] = d * d;
    const float gp = 2.f * d / (float)((long)n * hw);  // d loss / d s
    gpre[t] = gp;
    for (int c = 0; c < c16; ++c) gh[((size_t)i * c16 + c) * hw + p] = gp * __bfloat162float(w[c]);
  }
}

// head weight gradients: dw[c] = sum gpre h[c], db = sum gpre (fixed order)
__global__ void k_head_wgrad(const float* __restrict__ h, const float* __restrict__ gpre, int n, int c16, int hw,
                             float* __restrict__ dw, float* __restrict__ db) {
  __shared__ float sh[256];
  const int c = blockIdx.x;  // c16 blocks for weights, one more for the bias
  float s = 0.f;
  for (int i = 0; i < n; ++i)
    for (int p = threadIdx.x; p < hw; p += blockDim.x) {
      const float gp = gpre[(size_t)i * hw + p];
      s += c < c16 ? gp * h[((size_t)i * c16 + c) * hw + p] : gp;
    }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) (c < c16 ? dw[c] : db[0]) = sh[0];
}

__global__ void k_sum(const float* __restrict__ v, long n, float* __restrict__ out) {
  __shared__ float sh[256];
  float s = 0.f;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

__global__ void k_add(float* __restrict__ dst, const float* __restrict__ src, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] += src[i];
}

// Adam on FP32 master parameters; refreshes the BF16 weight copies
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m,
                       float* __restrict__ v, long n, float lr, float b1, float b2, float eps, float c1, float c2,
                       __nv_bfloat16* __restrict__ wbf, const int* __restrict__ wmap) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = gr[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = pi;
  if (wmap[i] >= 0) wbf[wmap[i]] = __float2bfloat16(pi);
}

// master parameters -> BF16 weight copies
__global__ void k_round_weights(const float* __restrict__ p, long n, __nv_bfloat16* __restrict__ wbf,
                                const int* __restrict__ wmap) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && wmap[i] >= 0) wbf[wmap[i]] = __float2bfloat16(p[i]);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
struct Mem {
  void* p = nullptr;
  size_t bytes = 0;
  Mem() {}
  Mem(const Mem&) = delete;
  Mem& operator=(const Mem&) = delete;
  Mem(Mem&& o) noexcept : p(o.p), bytes(o.bytes) {
    o.p = nullptr;
    o.bytes = 0;
  }
  ~Mem() {
    if (p) cudaFree(p);
  }
  void alloc(size_t n) {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = n;
    if (n) UN_CK(cudaMalloc(&p, n));
  }
  template <typename U> U* as() const { return reinterpret_cast<U*>(p); }
};

// one 3x3 convolution layer of the graph
struct Conv {
  int cout, ca, cb, a_up;
  int level;          // resolution level (0 = full)
  long w_off, b_off;  // offsets into the FP32 parameter vector
  long wbf_off;       // offset into the BF16 weights
};

// input a of conv i: -1 the network input, -2..-4 pool outputs 0..2,
// k >= 1 the output of conv k - 1 (act[k]); the concatenated b input of
// convs 9, 12, 15 is e3, e2, e1 (act 6, 4, 2)
constexpr int kSrcA[17] = {-1, 1, -2, 3, -3, 5, -4, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16};

inline int src_b(int i) { return i == 9 ? 6 : i == 12 ? 4 : i == 15 ? 2 : -1; }

// The network: the fixed U-Net described at the top of the file.
struct Net {
  int H = 0, W = 0, nmax = 0;
  std::vector<Conv> convs;
  long nparam = 0, nweights = 0;
  long head_w = 0, head_b = 0, head_wbf = 0;
  Mem p, g, m, v, wbf, wmap, wt, part;
  std::vector<Mem> act, gact;  // act[0] input, act[i + 1] output of conv i (post-ReLU)
  Mem pool[3], gpool[3], gup, gin_tmp, out, sq, gpre, lossv, tgt;
  cudaStream_t s = nullptr;
  long step = 0;
  bool cuda_cores = false;  // FP32 CUDA-core convolutions instead of the tensor cores

  int lvH(int l) const { return H >> l; }
  int lvW(int l) const { return W >> l; }

  Net(int H_, int W_, int nmax_) : H(H_), W(W_), nmax(nmax_) {
    if (H < 16 || W < 16 || H % 8 || W % 8 || nmax < 1)
      throw Error(MFISTA_ERR_ARG, "U-Net needs H, W multiples of 8 (>= 16) and a batch >= 1");
    auto add = [&](int cout, int ca, int cb, int up, int lv) { convs.push_back(Conv{cout, ca, cb, up, lv, 0, 0, 0}); };
    add(16, 2, 0, 0, 0);     // 0  e1a
    add(16, 16, 0, 0, 0);    // 1  e1
    add(32, 16, 0, 0, 1);    // 2  e2a  (input pool(e1))
    add(32, 32, 0, 0, 1);    // 3  e2
    add(64, 32, 0, 0, 2);    // 4  e3a  (pool(e2))
    add(64, 64, 0, 0, 2);    // 5  e3
    add(128, 64, 0, 0, 3);   // 6  e4a  (pool(e3))
    add(128, 128, 0, 0, 3);  // 7  e4
    add(64, 128, 0, 1, 2);   // 8  u3 = conv(up(e4))
    add(64, 64, 64, 0, 2);   // 9  d3a = conv(cat(u3, e3))
    add(64, 64, 0, 0, 2);    // 10 d3
    add(32, 64, 0, 1, 1);    // 11 u2 = conv(up(d3))
    add(32, 32, 32, 0, 1);   // 12 d2a = conv(cat(u2, e2))
    add(32, 32, 0, 0, 1);    // 13 d2
    add(16, 32, 0, 1, 0);    // 14 u1 = conv(up(d2))
    add(16, 16, 16, 0, 0);   // 15 d1a = conv(cat(u1, e1))
    add(16, 16, 0, 0, 0);    // 16 d1
    long off = 0, wo = 0;
    for (Conv& c : convs) {
      c.w_off = off;
      c.wbf_off = wo;
      const long nw = (long)c.cout * (c.ca + c.cb) * 9;
      off += nw;
      wo += nw;
      c.b_off = off;
      off += c.cout;
    }
    head_w = off;
    head_wbf = wo;
    off += 16;
    wo += 16;
    head_b = off;
    off += 1;
    nparam = off;
    nweights = wo;
    p.alloc(sizeof(float) * nparam);
    g.alloc(sizeof(float) * nparam);
    m.alloc(sizeof(float) * nparam);
    v.alloc(sizeof(float) * nparam);
    UN_CK(cudaMemset(g.p, 0, g.bytes));
    wbf.alloc(sizeof(__nv_bfloat16) * nweights);
    std::vector<int> map(nparam, -1);
    for (const Conv& c : convs)
      for (long i = 0; i < (long)c.cout * (c.ca + c.cb) * 9; ++i) map[c.w_off + i] = (int)(c.wbf_off + i);
    for (int i = 0; i < 16; ++i) map[head_w + i] = (int)(head_wbf + i);
    wmap.alloc(sizeof(int) * nparam);
    UN_CK(cudaMemcpy(wmap.p, map.data(), sizeof(int) * nparam, cudaMemcpyHostToDevice));
    long maxw = 0;
    size_t maxpart = 0;
    for (const Conv& c : convs) {
      maxw = std::max(maxw, (long)c.cout * (c.ca + c.cb) * 9);
      const size_t tiles = (size_t)nmax * cdiv(lvH(c.level), kCT) * cdiv(lvW(c.level), kCT);
      maxpart = std::max(maxpart, tiles * (size_t)c.cout * (c.ca + c.cb) * 9);
    }
    wt.alloc(sizeof(__nv_bfloat16) * maxw);
    part.alloc(sizeof(float) * maxpart);
    act.resize(convs.size() + 1);
    gact.resize(convs.size() + 1);
    act[0].alloc(sizeof(float) * (size_t)nmax * 2 * H * W);  // the input
    for (size_t i = 0; i < convs.size(); ++i) {
      const Conv& c = convs[i];
      const size_t n = (size_t)nmax * c.cout * lvH(c.level) * lvW(c.level);
      act[i + 1].alloc(sizeof(float) * n);
      gact[i + 1].alloc(sizeof(float) * n);
    }
    for (int l = 0; l < 3; ++l) {
      const size_t n = (size_t)nmax * (16 << l) * lvH(l + 1) * lvW(l + 1);  // pool(e1) 16 ch, pool(e2) 32, pool(e3) 64
      pool[l].alloc(sizeof(float) * n);
      gpool[l].alloc(sizeof(float) * n);
    }
    // largest input gradient of one conv: 32 channels at full resolution
    // (u1 and d1a), i.e. 128 channels at a quarter of the pixels
    gup.alloc(sizeof(float) * (size_t)nmax * 32 * H * W);
    gin_tmp.alloc(sizeof(float) * (size_t)nmax * 32 * H * W);
    out.alloc(sizeof(float) * (size_t)nmax * H * W);
    sq.alloc(sizeof(float) * (size_t)nmax * H * W);
    gpre.alloc(sizeof(float) * (size_t)nmax * H * W);
    tgt.alloc(sizeof(float) * (size_t)nmax * H * W);
    lossv.alloc(sizeof(float));
    UN_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const char* cc = getenv("MFISTA_UNET_CUDA_CORES");
    cuda_cores = cc && cc[0] == '1';
    UN_CK(cudaDeviceSynchronize());  // the set-up above ran on the legacy stream
    init_params(1234);
  }
  ~Net() {
    if (s) cudaStreamDestroy(s);
  }

  // He-normal initial weights (deterministic LCG + Box-Muller), zero biases
  void init_params(uint64_t seed) {
    std::vector<float> h(nparam, 0.f);
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
      st = st * 6364136223846793005ull + 1442695040888963407ull;
      return ((st >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() {
      const double u1 = uni(), u2 = uni();
      return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
    };
    for (const Conv& c : convs) {
      const double sd = sqrt(2.0 / (9.0 * (c.ca + c.cb)));
      for (long i = 0; i < (long)c.cout * (c.ca + c.cb) * 9; ++i) h[c.w_off + i] = (float)(sd * normal());
    }
    for (int i = 0; i < 16; ++i) h[head_w + i] = (float)(sqrt(2.0 / 16.0) * normal());
    set_params(h.data());
  }

  void set_params(const float* hp) {
    UN_CK(cudaMemcpyAsync(p.p, hp, sizeof(float) * nparam, cudaMemcpyHostToDevice, s));
    k_round_weights<<<cdiv(nparam, 256), 256, 0, s>>>(p.as<float>(), nparam, wbf.as<__nv_bfloat16>(),
                                                      wmap.as<int>());
    UN_LAUNCH();
    UN_CK(cudaMemsetAsync(m.p, 0, m.bytes, s));
    UN_CK(cudaMemsetAsync(v.p, 0, v.bytes, s));
    step = 0;
    UN_CK(cudaStreamSynchronize(s));
  }

  const __nv_bfloat16* wb(const Conv& c) const { return wbf.as<__nv_bfloat16>() + c.wbf_off; }

  const float* src_a_ptr(int i) const {
    const int sa = kSrcA[i];
    return sa == -1 ? act[0].as<float>() : sa <= -2 ? pool[-sa - 2].as<float>() : act[sa].as<float>();
  }
  float* src_a_grad(int i) const { return kSrcA[i] <= -2 ? gpool[-kSrcA[i] - 2].as<float>() : gact[kSrcA[i]].as<float>(); }
  const float* src_b_ptr(int i) const { return src_b(i) >= 0 ? act[src_b(i)].as<float>() : nullptr; }

  // a 3x3 convolution on the tensor cores (32 output channels per CTA, 16
  // when cout is 16); MFISTA_UNET_CUDA_CORES=1 selects the FP32 CUDA-core
  // kernel instead (comparison runs)
  void conv(const ConvArgs& a, int n) {
    dim3 grid(cdiv(a.W, kCT) * cdiv(a.H, kCT), 1, n);
    if (cuda_cores) {
      grid.y = cdiv(a.cout, kCO);
      k_conv3x3<<<grid, 128, 0, s>>>(a);
    } else if (a.cout % 32 == 0) {
      grid.y = a.cout / 32;
      k_conv3x3_tc<2><<<grid, 256, conv_tc_smem<2>(), s>>>(a);
    } else {
      grid.y = cdiv(a.cout, 16);
      k_conv3x3_tc<1><<<grid, 256, conv_tc_smem<1>(), s>>>(a);
    }
    UN_LAUNCH();
  }

  void conv_forward(int i, int n) {
    const Conv& c = convs[i];
    ConvArgs ga{src_a_ptr(i), nullptr, c.ca, c.a_up, src_b_ptr(i), c.cb, wb(c), p.as<float>() + c.b_off,
                act[i + 1].as<float>(), c.cout, lvH(c.level), lvW(c.level), 1, 0};
    conv(ga, n);
  }

  void pool_forward(int l, int n) {  // pool l of e_{l+1} = act[2 + 2 l]
    const int c = 16 << l;
    const long cnt = (long)n * c * lvH(l + 1) * lvW(l + 1);
    k_maxpool<<<cdiv(cnt, 256), 256, 0, s>>>(act[2 + 2 * l].as<float>(), n * c, lvH(l), lvW(l), pool[l].as<float>());
    UN_LAUNCH();
  }

  void forward(int n, const float* target) {
    for (int i = 0; i < 17; ++i) {
      if (i == 2) pool_forward(0, n);
      if (i == 4) pool_forward(1, n);
      if (i == 6) pool_forward(2, n);
      conv_forward(i, n);
    }
    const long hw = (long)H * W;
    k_head<<<cdiv(n * hw, 256), 256, 0, s>>>(act[17].as<float>(), n, 16, (int)hw,
                                             wbf.as<__nv_bfloat16>() + head_wbf, p.as<float>() + head_b,
                                             out.as<float>(), target, sq.as<float>(), gact[17].as<float>(),
                                             gpre.as<float>());
    UN_LAUNCH();
    if (target) {
      k_sum<<<1, 256, 0, s>>>(sq.as<float>(), n * hw, lossv.as<float>());
      UN_LAUNCH();
    }
  }

  void add_into(float* dst, const float* src, long cnt) {
    k_add<<<cdiv(cnt, 256), 256, 0, s>>>(dst, src, cnt);
    UN_LAUNCH();
  }

  // gradient of conv i given gact[i+1] (w.r.t. its post-ReLU output):
  // weight and bias gradients into g, input gradients added to the
  // producers' gradient buffers
  void conv_backward(int i, int n) {
    const Conv& c = convs[i];
    const int Hl = lvH(c.level), Wl = lvW(c.level), cin = c.ca + c.cb;
    const float* go = gact[i + 1].as<float>();
    const float* mask = act[i + 1].as<float>();  // ReLU: the gradient passes where the output > 0
    const int ntiles = n * cdiv(Hl, kCT) * cdiv(Wl, kCT);
    WgradArgs wa{go, mask, src_a_ptr(i), c.ca, c.a_up, src_b_ptr(i), c.cb, part.as<float>(), c.cout, Hl, Wl};
    if (cuda_cores)
      k_conv3x3_wgrad<<<dim3(ntiles, cdiv(c.cout, kCO), cdiv(cin, kCI)), 256, 0, s>>>(wa);
    else
      k_conv3x3_wgrad_tc<<<dim3(ntiles, cdiv(c.cout, 16), cdiv(cin, kCI)), 288, kWgradTcSmem, s>>>(wa);
    UN_LAUNCH();
    const long len = (long)c.cout * cin * 9;
    k_reduce_partials<<<cdiv(len, 256), 256, 0, s>>>(part.as<float>(), ntiles, len, g.as<float>() + c.w_off);
    UN_LAUNCH();
    k_bias_grad<<<c.cout, 256, 0, s>>>(go, mask, n, c.cout, Hl * Wl, g.as<float>() + c.b_off);
    UN_LAUNCH();
    if (i == 0) return;  // no gradient for the network input
    // data: the transposed convolution of the masked gradient
    k_flip_transpose<<<cdiv(len, 256), 256, 0, s>>>(wb(c), c.cout, cin, wt.as<__nv_bfloat16>());
    UN_LAUNCH();
    float* gi = c.a_up ? gup.as<float>() : gin_tmp.as<float>();  // w.r.t. the (upsampled) concat input
    ConvArgs gd{go, mask, c.cout, 0, nullptr, 0, wt.as<__nv_bfloat16>(), nullptr, gi, cin, Hl, Wl, 0, 0};
    conv(gd, n);
    float* ga_dst = src_a_grad(i);
    const size_t hw = (size_t)Hl * Wl;
    if (c.a_up) {  // sum the 2x2 blocks into a's half-resolution gradient
      const int h = Hl / 2, w = Wl / 2;
      for (int k = 0; k < n; ++k) {
        k_upsample_grad<<<cdiv((long)c.ca * h * w, 256), 256, 0, s>>>(gi + (size_t)k * cin * hw, c.ca, h, w,
                                                                      gin_tmp.as<float>() + (size_t)k * c.ca * h * w);
        UN_LAUNCH();
      }
      add_into(ga_dst, gin_tmp.as<float>(), (long)n * c.ca * h * w);
      return;
    }
    for (int k = 0; k < n; ++k) {  // channels [0, ca) to a's producer, [ca, cin) to b's
      add_into(ga_dst + (size_t)k * c.ca * hw, gi + (size_t)k * cin * hw, (long)c.ca * hw);
      if (c.cb)
        add_into(gact[src_b(i)].as<float>() + (size_t)k * c.cb * hw, gi + ((size_t)k * cin + c.ca) * hw,
                 (long)c.cb * hw);
    }
  }

  void pool_backward(int l, int n) {
    const int c = 16 << l;
    const long cnt = (long)n * c * lvH(l + 1) * lvW(l + 1);
    k_maxpool_grad<<<cdiv(cnt, 256), 256, 0, s>>>(act[2 + 2 * l].as<float>(), gpool[l].as<float>(), n * c, lvH(l),
                                                   lvW(l), gact[2 + 2 * l].as<float>());
    UN_LAUNCH();
  }

  void backward(int n) {
    for (size_t i = 1; i + 1 < gact.size(); ++i) UN_CK(cudaMemsetAsync(gact[i].p, 0, gact[i].bytes, s));
    for (int l = 0; l < 3; ++l) UN_CK(cudaMemsetAsync(gpool[l].p, 0, gpool[l].bytes, s));
    const long hw = (long)H * W;
    k_head_wgrad<<<17, 256, 0, s>>>(act[17].as<float>(), gpre.as<float>(), n, 16, (int)hw, g.as<float>() + head_w,
                                   g.as<float>() + head_b);
    UN_LAUNCH();
    for (int i = 16; i >= 0; --i) {
      conv_backward(i, n);
      // once the consumer of a pool output is done, route the pool gradient
      if (i == 6) pool_backward(2, n);
      if (i == 4) pool_backward(1, n);
      if (i == 2) pool_backward(0, n);
    }
  }

  void upload(const float* in, const float* target, int n) {
    UN_CK(cudaMemcpyAsync(act[0].p, in, sizeof(float) * (size_t)n * 2 * H * W, cudaMemcpyHostToDevice, s));
    if (target)
      UN_CK(cudaMemcpyAsync(tgt.p, target, sizeof(float) * (size_t)n * H * W, cudaMemcpyHostToDevice, s));
  }

  float loss(int n) {
    float sum = 0.f;
    UN_CK(cudaMemcpyAsync(&sum, lossv.p, sizeof(float), cudaMemcpyDeviceToHost, s));
    UN_CK(cudaStreamSynchronize(s));
    return sum / (float)((long)n * H * W);
  }
};

thread_local int g_status = 0;
thread_local std::string g_msg;

int fail(const Error& e) {
  g_status = e.status;
  g_msg = e.what();
  return e.status;
}

Net* checked(void* net, int n, bool need_n) {
  Net* N = static_cast<Net*>(net);
  if (!N) throw Error(MFISTA_ERR_ARG, "null network");
  if (need_n && (n < 1 || n > N->nmax)) throw Error(MFISTA_ERR_ARG, "batch must be 1..batch_max");
  return N;
}

}  // namespace unet

using unet::Error;
using unet::Net;

extern "C" {

void* mfista_unet_create(int H, int W, int batch_max) {
  try {
    unet::g_status = 0;
    return new Net(H, W, batch_max);
  } catch (const Error& e) {
    unet::fail(e);
    return nullptr;
  }
}

void mfista_unet_destroy(void* net) { delete static_cast<Net*>(net); }

long mfista_unet_param_count(void* net) { return net ? static_cast<Net*>(net)->nparam : 0; }

int mfista_unet_get_params(void* net, float* out) {
  try {
    Net* N = unet::checked(net, 0, false);
    if (!out) throw Error(MFISTA_ERR_ARG, "null argument");
    UN_CK(cudaMemcpyAsync(out, N->p.p, sizeof(float) * N->nparam, cudaMemcpyDeviceToHost, N->s));
    UN_CK(cudaStreamSynchronize(N->s));
    return MFISTA_OK;
  } catch (const Error& e) {
    return unet::fail(e);
  }
}

int mfista_unet_set_params(void* net, const float* in) {
  try {
    Net* N = unet::checked(net, 0, false);
    if (!in) throw Error(MFISTA_ERR_ARG, "null argument");
    N->set_params(in);
    return MFISTA_OK;
  } catch (const Error& e) {
    return unet::fail(e);
  }
}

int mfista_unet_forward(void* net, const float* in, int n, float* out) {
  try {
    Net* N = unet::checked(net, n, true);
    if (!in || !out) throw Error(MFISTA_ERR_ARG, "null argument");
    N->upload(in, nullptr, n);
    N->forward(n, nullptr);
    UN_CK(cudaMemcpyAsync(out, N->out.p, sizeof(float) * (size_t)n * N->H * N->W, cudaMemcpyDeviceToHost, N->s));
    UN_CK(cudaStreamSynchronize(N->s));
    return MFISTA_OK;
  } catch (const Error& e) {
    return unet::fail(e);
  }
}

int mfista_unet_grad(void* net, const float* in, const float* target, int n, float* loss, float* grad) {
  try {
    Net* N = unet::checked(net, n, true);
    if (!in || !target) throw Error(MFISTA_ERR_ARG, "null argument");
    N->upload(in, target, n);
    N->forward(n, N->tgt.as<float>());
    N->backward(n);
    if (grad) UN_CK(cudaMemcpyAsync(grad, N->g.p, sizeof(float) * N->nparam, cudaMemcpyDeviceToHost, N->s));
    const float l = N->loss(n);
    if (loss) *loss = l;
    return MFISTA_OK;
  } catch (const Error& e) {
    return unet::fail(e);
  }
}

int mfista_unet_train_step(void* net, const float* in, const float* target, int n, float lr, float* loss) {
  try {
    Net* N = unet::checked(net, n, true);
    if (!in || !target) throw Error(MFISTA_ERR_ARG, "null argument");
    N->upload(in, target, n);
    N->forward(n, N->tgt.as<float>());
    N->backward(n);
    N->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)N->step), c2 = 1.f - powf(b2, (float)N->step);
    unet::k_adam<<<unet::cdiv(N->nparam, 256), 256, 0, N->s>>>(
        N->p.as<float>(), N->g.as<float>(), N->m.as<float>(), N->v.as<float>(), N->nparam, lr, b1, b2, 1e-8f, c1,
        c2, N->wbf.as<__nv_bfloat16>(), N->wmap.as<int>());
    UN_LAUNCH();
    const float l = N->loss(n);
    if (loss) *loss = l;
    return MFISTA_OK;
  } catch (const Error& e) {
    return unet::fail(e);
  }
}

int mfista_unet_last_status(void) { return unet::g_status; }
const char* mfista_unet_last_error(void) { return unet::g_msg.c_str(); }

}  // extern "C"
