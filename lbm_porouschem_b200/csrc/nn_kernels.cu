// nn_kernels.cu -- kernels of the warm-start surrogate (a small 2D U-Net).
//
// Activations are NHWC bf16 (channels fastest, channel counts multiples of 8),
// weights bf16 [Cout][taps][Cin], accumulation FP32 on the tensor cores
// (mma.sync m16n8k16, bf16 x bf16 -> f32).  A convolution is an implicit GEMM:
//   out[p, n] = sum_{t, c} in[p + off(t), c] * w[n][t][c]      (M = pixels, N = Cout,
//                                                                K = taps * Cin)
// with the im2col gather done while staging tiles in shared memory (zero outside
// the image).  Channel offset/stride arguments let a layer read or write a slice
// of a wider buffer, so the U-Net's skip concatenation needs no copy.  The input
// gradient of a convolution is the same GEMM on the flipped, transposed weights
// (nn_flip_weights); the weight gradient is a second GEMM over pixels
// (nn_conv_wgrad, split over pixel ranges, FP32 atomics).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "lbm_nn.h"

namespace lbm {
namespace capi {
int fail(int code, const std::string& msg);
}
}  // namespace lbm

namespace {

using bf16 = __nv_bfloat16;
constexpr int kBM = 64, kBN = 64, kBK = 32, kPad = 8;  // block tile; row pad (bf16) against bank conflicts

struct ConvArgs {
  const bf16* in;
  int in_cstride, in_coff;   // channel stride of the input buffer, first channel read
  const bf16* w;             // [Cout][taps][Cin]
  const float* bias;         // [Cout] or null
  const bf16* gate;          // out *= (gate > 0) when not null (same layout as out)
  bf16* out;                 // bf16 output, or
  float* out_f32;            // FP32 output (one of the two)
  int out_cstride, out_coff;
  int B, D, H, W, Cin, Cout, ks;  // ks = 1 or 3; D = 1 in 2D
  int nd;                         // spatial dimensions: 2 (taps ks^2) or 3 (taps ks^3)
  int relu, accumulate;           // accumulate: out += result (bf16 / f32)
};

// Input pixel that tap `tap` of output pixel p reads (NDHWC, x fastest; taps in
// z, y, x order, x fastest); false where the tap falls outside (zero padding).
__device__ __forceinline__ bool tap_pixel(int p, int tap, int D, int H, int W, int ks, int nd, size_t& q) {
  const int half = ks / 2;
  const int x = p % W, y = (p / W) % H, zb = p / (W * H);
  const int z = zb % D, b = zb / D;
  const int xx = x + tap % ks - half, yy = y + (tap / ks) % ks - half;
  const int zz = nd == 3 ? z + tap / (ks * ks) - half : z;
  if (xx < 0 || xx >= W || yy < 0 || yy >= H || zz < 0 || zz >= D) return false;
  q = ((size_t)(b * D + zz) * H + yy) * W + xx;
  return true;
}

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp tile 32 x 32 of a 64 x 64 block tile: 2 (m16) x 4 (n8) mma tiles.  As[m][k],
// Bs[n][k] (row stride kBK + kPad).  Fragment layout of m16n8k16 (PTX ISA): lane =
// 4 g + t; A: rows g / g+8, columns 2t, 2t+1 (+8); B: column g, rows 2t, 2t+1 (+8);
// C: rows g / g+8, columns 2t, 2t+1.
__device__ __forceinline__ void warp_tile_mma(const bf16 (*As)[kBK + kPad], const bf16 (*Bs)[kBK + kPad], int wm,
                                              int wn, int lane, float acc[2][4][4]) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int kk = 0; kk < kBK; kk += 16) {
    uint32_t a[2][4], b[4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = wm + i * 16 + g;
      a[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 2 * t]);
      a[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 2 * t]);
      a[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][kk + 8 + 2 * t]);
      a[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][kk + 8 + 2 * t]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = wn + j * 8 + g;
      b[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 2 * t]);
      b[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[n][kk + 8 + 2 * t]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], a[i], b[j]);
  }
}

// Convolution as implicit GEMM.  Grid (ceil(B*H*W / 64), ceil(Cout / 64)), 128 threads.
__global__ void __launch_bounds__(128) conv_igemm(const ConvArgs a) {
  __shared__ __align__(16) bf16 As[kBM][kBK + kPad];
  __shared__ __align__(16) bf16 Bs[kBN][kBK + kPad];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int P = a.B * a.D * a.H * a.W;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
  const int taps = a.nd == 3 ? a.ks * a.ks * a.ks : a.ks * a.ks;
  const int K = taps * a.Cin;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  for (int k0 = 0; k0 < K; k0 += kBK) {
    // A: 64 pixels x 32 k as 256 chunks of 8 channels (Cin % 8 == 0, so a chunk
    // never straddles two taps)
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int q = tid + r * 128;
      const int mi = q >> 2, kc = (q & 3) * 8;
      const int p = m0 + mi, k = k0 + kc;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p < P && k < K) {
        const int tap = k / a.Cin, c = k - tap * a.Cin;
        size_t q;
        if (tap_pixel(p, tap, a.D, a.H, a.W, a.ks, a.nd, q))
          v = *reinterpret_cast<const uint4*>(a.in + q * a.in_cstride + a.in_coff + c);
      }
      *reinterpret_cast<uint4*>(&As[mi][kc]) = v;
    }
    // B: 64 output channels x 32 k
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int q = tid + r * 128;
      const int ni = q >> 2, kc = (q & 3) * 8;
      const int n = n0 + ni, k = k0 + kc;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (n < a.Cout && k < K) v = *reinterpret_cast<const uint4*>(a.w + (size_t)n * K + k);
      *reinterpret_cast<uint4*>(&Bs[ni][kc]) = v;
    }
    __syncthreads();
    warp_tile_mma(As, Bs, wm, wn, lane, acc);
    __syncthreads();
  }
  // epilogue: bias, ReLU, gate, store (pairs of channels)
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = m0 + wm + i * 16 + g + h * 8;
      if (p >= P) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int n = n0 + wn + j * 8 + 2 * t + e;
          if (n >= a.Cout) continue;
          float v = acc[i][j][h * 2 + e];
          if (a.bias) v += a.bias[n];
          if (a.relu) v = fmaxf(v, 0.f);
          const size_t o = (size_t)p * a.out_cstride + a.out_coff + n;
          if (a.gate && !(__bfloat162float(a.gate[o]) > 0.f)) v = 0.f;
          if (a.out_f32) {
            a.out_f32[o] = a.accumulate ? a.out_f32[o] + v : v;
          } else {
            if (a.accumulate) v += __bfloat162float(a.out[o]);
            a.out[o] = __float2bfloat16_rn(v);
          }
        }
      }
    }
}

// Weight gradient dw[n][t][c] += sum_p dout[p][n] * in[p + off(t)][c] over the
// pixel range of blockIdx.z.  M = Cout (n), N = taps * Cin, K = pixels.
struct WgradArgs {
  const bf16* in;
  int in_cstride, in_coff;
  const bf16* dout;
  int dout_cstride, dout_coff;
  float* dw;
  int B, D, H, W, Cin, Cout, ks, nd;
  int pix_per_split;
};

__global__ void __launch_bounds__(128) conv_wgrad(const WgradArgs a) {
  __shared__ __align__(16) bf16 As[kBM][kBK + kPad];  // [n][pixel]
  __shared__ __align__(16) bf16 Bs[kBN][kBK + kPad];  // [tap*Cin + c][pixel]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  const int P = a.B * a.D * a.H * a.W;
  const int taps = a.nd == 3 ? a.ks * a.ks * a.ks : a.ks * a.ks, Kc = taps * a.Cin;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
  const int p_begin = blockIdx.z * a.pix_per_split;
  const int p_end = min(P, p_begin + a.pix_per_split);
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  for (int p0 = p_begin; p0 < p_end; p0 += kBK) {
    // A: dout for 32 pixels x 64 output channels, transposed into As[n][pixel]
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int q = tid + r * 128;
      const int pi = q >> 3, nc = (q & 7) * 8;
      const int p = p0 + pi, n = m0 + nc;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p < p_end && n < a.Cout)
        v = *reinterpret_cast<const uint4*>(a.dout + (size_t)p * a.dout_cstride + a.dout_coff + n);
      const bf16* e8 = reinterpret_cast<const bf16*>(&v);
#pragma unroll
      for (int e = 0; e < 8; ++e) As[nc + e][pi] = e8[e];
    }
    // B: im2col rows of 32 pixels x 64 (tap, c) columns, transposed into Bs[col][pixel]
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int q = tid + r * 128;
      const int pi = q >> 3, kc = (q & 7) * 8;
      const int p = p0 + pi, k = n0 + kc;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p < p_end && k < Kc) {
        const int tap = k / a.Cin, c = k - tap * a.Cin;
        size_t q;
        if (tap_pixel(p, tap, a.D, a.H, a.W, a.ks, a.nd, q))
          v = *reinterpret_cast<const uint4*>(a.in + q * a.in_cstride + a.in_coff + c);
      }
      const bf16* e8 = reinterpret_cast<const bf16*>(&v);
#pragma unroll
      for (int e = 0; e < 8; ++e) Bs[kc + e][pi] = e8[e];
    }
    __syncthreads();
    warp_tile_mma(As, Bs, wm, wn, lane, acc);
    __syncthreads();
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int n = m0 + wm + i * 16 + g + h * 8;
      if (n >= a.Cout) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int k = n0 + wn + j * 8 + 2 * t + e;
          if (k < Kc) atomicAdd(&a.dw[(size_t)n * Kc + k], acc[i][j][h * 2 + e]);
        }
    }
}

// dbias[n] += sum_p dout[p][n]; grid (ceil(Cout/32), splits), 256 threads.
__global__ void __launch_bounds__(256) bias_grad(const bf16* dout, int cstride, int coff, int P, int Cout,
                                                 float* dbias) {
  __shared__ float s[8][32];
  const int n = blockIdx.x * 32 + (threadIdx.x & 31);
  const int row = threadIdx.x >> 5;
  float v = 0.f;
  if (n < Cout)
    for (int p = blockIdx.y * 8 + row; p < P; p += gridDim.y * 8) v += __bfloat162float(dout[(size_t)p * cstride + coff + n]);
  s[row][threadIdx.x & 31] = v;
  __syncthreads();
  if (row == 0 && n < Cout) {
    float t = 0.f;
#pragma unroll
    for (int r = 0; r < 8; ++r) t += s[r][threadIdx.x & 31];
    atomicAdd(&dbias[n], t);
  }
}

// wt[c][flip(t)][n] = w[n][t][c]: the input gradient of a convolution is the
// convolution of the output gradient with these weights.
__global__ void flip_weights(const bf16* w, bf16* wt, int Cout, int taps, int Cin) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Cout * taps * Cin) return;
  const int c = i % Cin, t = (i / Cin) % taps, n = i / (Cin * taps);
  wt[((size_t)c * taps + (taps - 1 - t)) * Cout + n] = w[i];
}

// Pixel (b, z, y, x) of a B x D x H x W grid (x fastest).
struct Pix {
  int b, z, y, x;
  __device__ __forceinline__ Pix(size_t p, int D, int H, int W) {
    x = (int)(p % W);
    y = (int)((p / W) % H);
    const size_t zb = p / ((size_t)W * H);
    z = (int)(zb % D);
    b = (int)(zb / D);
  }
};
__device__ __forceinline__ size_t pix(int b, int z, int y, int x, int D, int H, int W) {
  return ((size_t)(b * D + z) * H + y) * W + x;
}

// 2x2 (3D: 2x2x2) average pooling of a channel slice (D, H, W even; D = 1 in 2D).
__global__ void avgpool2(const bf16* in, int in_cstride, int in_coff, bf16* out, int B, int D, int H, int W, int C,
                         int nd) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int Do = nd == 3 ? D / 2 : D, Ho = H / 2, Wo = W / 2, nz = nd == 3 ? 2 : 1;
  if (i >= (size_t)B * Do * Ho * Wo * C) return;
  const int c = (int)(i % C);
  const Pix o(i / C, Do, Ho, Wo);
  float s = 0.f;
  for (int dz = 0; dz < nz; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx)
        s += __bfloat162float(
            in[pix(o.b, nz * o.z + dz, 2 * o.y + dy, 2 * o.x + dx, D, H, W) * in_cstride + in_coff + c]);
  out[i] = __float2bfloat16_rn(s / (4.0f * nz));
}

// Gradient of avgpool2: every input pixel receives its share of its window's
// gradient; accumulate adds it to what the slice holds.
__global__ void avgpool2_bwd(const bf16* dout, bf16* din, int din_cstride, int din_coff, int B, int D, int H, int W,
                             int C, int nd, int accumulate) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * D * H * W * C) return;
  const int c = (int)(i % C);
  const size_t p = i / C;
  const Pix q(p, D, H, W);
  const int nz = nd == 3 ? 2 : 1;
  const float g = __bfloat162float(dout[pix(q.b, q.z / nz, q.y / 2, q.x / 2, D / nz, H / 2, W / 2) * C + c]) /
                  (4.0f * nz);
  const size_t o = p * din_cstride + din_coff + c;
  din[o] = __float2bfloat16_rn(accumulate ? __bfloat162float(din[o]) + g : g);
}

// Nearest 2x upsampling (3D: in z too) into a channel slice, and its gradient
// (sums over each 2x2 / 2x2x2 block).
__global__ void upsample2(const bf16* in, bf16* out, int out_cstride, int out_coff, int B, int D, int H, int W, int C,
                          int nd) {
  const int nz = nd == 3 ? 2 : 1;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // over the output
  if (i >= (size_t)B * nz * D * 4 * H * W * C) return;
  const int c = (int)(i % C);
  const size_t p = i / C;
  const Pix o(p, nz * D, 2 * H, 2 * W);
  out[p * out_cstride + out_coff + c] = in[pix(o.b, o.z / nz, o.y / 2, o.x / 2, D, H, W) * C + c];
}
__global__ void upsample2_bwd(const bf16* dout, int dout_cstride, int dout_coff, bf16* din, int B, int D, int H, int W,
                              int C, int nd) {
  const int nz = nd == 3 ? 2 : 1;
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // over din
  if (i >= (size_t)B * D * H * W * C) return;
  const int c = (int)(i % C);
  const Pix q(i / C, D, H, W);
  float s = 0.f;
  for (int dz = 0; dz < nz; ++dz)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dx = 0; dx < 2; ++dx)
        s += __bfloat162float(dout[pix(q.b, nz * q.z + dz, 2 * q.y + dy, 2 * q.x + dx, nz * D, 2 * H, 2 * W) *
                                       dout_cstride + dout_coff + c]);
  din[i] = __float2bfloat16_rn(s);
}

// Masked mean-squared error over the first `C` channels of pred (f32, stride C)
// against target (f32): per-block partial sums, and the gradient as bf16.
__global__ void mse_loss(const float* pred, const float* target, const float* weight, size_t n, float scale,
                         bf16* grad, float* partial) {
  __shared__ float s[256];
  float acc = 0.f;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float wgt = weight ? weight[i] : 1.f;
    const float d = pred[i] - target[i];
    acc += wgt * d * d;
    grad[i] = __float2bfloat16_rn(2.f * scale * wgt * d);
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// Adam on FP32 master weights; writes the bf16 copy the kernels read.
__global__ void adam_step(float* w, const float* g, float* m, float* v, bf16* wb, size_t n, float lr, float b1,
                          float b2, float eps, float c1, float c2, float wd) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] + wd * w[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = __float2bfloat16_rn(wi);
}

// ReLU gradient: dy = 0 where y <= 0 (channel slices of equal shape).
__global__ void relu_bwd(bf16* dy, int dy_cstride, int dy_coff, const bf16* y, int y_cstride, int y_coff, size_t P,
                         int C) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= P * C) return;
  const int c = (int)(i % C);
  const size_t p = i / C;
  if (!(__bfloat162float(y[p * y_cstride + y_coff + c]) > 0.f)) dy[p * dy_cstride + dy_coff + c] = __float2bfloat16_rn(0.f);
}

__global__ void to_bf16(const float* x, bf16* y, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

unsigned blocks_for(size_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lbm::capi::fail(LBM_NN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  return 0;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

int conv_nd(const void* in, int32_t in_cstride, int32_t in_coff, const void* w, const float* bias, const void* gate,
            void* out_bf16, float* out_f32, int32_t out_cstride, int32_t out_coff, int32_t B, int32_t D, int32_t H,
            int32_t W, int32_t Cin, int32_t Cout, int32_t ksize, int32_t relu, int32_t accumulate, int nd,
            void* stream) {
  if (!in || !w || (!out_bf16 && !out_f32) || (out_bf16 && out_f32))
    return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv: in, w and exactly one output are required");
  if (ksize != 1 && ksize != 3) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv: ksize must be 1 or 3");
  if (Cin % 8 || in_cstride % 8 || in_coff % 8 || B < 1 || D < 1 || H < 1 || W < 1 || Cout < 1 ||
      in_coff + Cin > in_cstride || out_coff + Cout > out_cstride)
    return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv: channel counts/offsets must be multiples of 8 and fit");
  if ((double)B * D * H * W >= 2147483647.0) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv: too many pixels");
  if (!aligned16(in) || !aligned16(w)) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv: in and w must be 16-byte aligned");
  ConvArgs a{(const bf16*)in, in_cstride, in_coff, (const bf16*)w, bias, (const bf16*)gate, (bf16*)out_bf16, out_f32,
             out_cstride, out_coff, B, D, H, W, Cin, Cout, ksize, nd, relu, accumulate};
  const size_t P = (size_t)B * D * H * W;
  const dim3 grid((unsigned)((P + kBM - 1) / kBM), (unsigned)((Cout + kBN - 1) / kBN));
  conv_igemm<<<grid, 128, 0, (cudaStream_t)stream>>>(a);
  return check_launch("conv_igemm");
}

int wgrad_nd(const void* in, int32_t in_cstride, int32_t in_coff, const void* dout, int32_t dout_cstride,
             int32_t dout_coff, float* dw, int32_t B, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
             int32_t ksize, int nd, void* stream) {
  if (!in || !dout || !dw) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv_wgrad: NULL argument");
  if (ksize != 1 && ksize != 3) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv_wgrad: ksize must be 1 or 3");
  if (Cin % 8 || Cout % 8 || in_cstride % 8 || in_coff % 8 || dout_cstride % 8 || dout_coff % 8 ||
      in_coff + Cin > in_cstride || dout_coff + Cout > dout_cstride || B < 1 || D < 1 || H < 1 || W < 1)
    return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv_wgrad: channel counts/offsets must be multiples of 8 and fit");
  if ((double)B * D * H * W >= 2147483647.0) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv_wgrad: too many pixels");
  if (!aligned16(in) || !aligned16(dout)) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_conv_wgrad: 16-byte alignment");
  const int P = B * D * H * W;
  const int Kc = (nd == 3 ? ksize * ksize * ksize : ksize * ksize) * Cin;
  const int mt = (Cout + kBM - 1) / kBM, nt = (Kc + kBN - 1) / kBN;
  // enough pixel splits to fill the GPU (about 4 blocks per SM), each a multiple of 32 pixels
  int splits = std::max(1, 148 * 4 / std::max(1, mt * nt));
  int pps = (P + splits - 1) / splits;
  pps = (pps + kBK - 1) / kBK * kBK;
  splits = (P + pps - 1) / pps;
  WgradArgs a{(const bf16*)in, in_cstride, in_coff, (const bf16*)dout, dout_cstride, dout_coff, dw, B, D, H, W, Cin,
              Cout, ksize, nd, pps};
  conv_wgrad<<<dim3(mt, nt, splits), 128, 0, (cudaStream_t)stream>>>(a);
  return check_launch("conv_wgrad");
}

int pool_nd(const void* in, int32_t in_cstride, int32_t in_coff, void* out, int32_t B, int32_t D, int32_t H, int32_t W,
            int32_t C, int nd, void* stream) {
  if (H % 2 || W % 2 || (nd == 3 && D % 2)) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_avgpool2: sizes must be even");
  const size_t n = (size_t)B * (nd == 3 ? D / 2 : D) * (H / 2) * (W / 2) * C;
  avgpool2<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)in, in_cstride, in_coff, (bf16*)out, B, D,
                                                                 H, W, C, nd);
  return check_launch("avgpool2");
}

int pool_bwd_nd(const void* dout, void* din, int32_t din_cstride, int32_t din_coff, int32_t B, int32_t D, int32_t H,
                int32_t W, int32_t C, int32_t accumulate, int nd, void* stream) {
  if (H % 2 || W % 2 || (nd == 3 && D % 2)) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_avgpool2_bwd: sizes must be even");
  const size_t n = (size_t)B * D * H * W * C;
  avgpool2_bwd<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)dout, (bf16*)din, din_cstride,
                                                                     din_coff, B, D, H, W, C, nd, accumulate);
  return check_launch("avgpool2_bwd");
}

int up_nd(const void* in, void* out, int32_t out_cstride, int32_t out_coff, int32_t B, int32_t D, int32_t H, int32_t W,
          int32_t C, int nd, void* stream) {
  const size_t n = (size_t)B * (nd == 3 ? 2 * D : D) * 4 * H * W * C;
  upsample2<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)in, (bf16*)out, out_cstride, out_coff, B,
                                                                   D, H, W, C, nd);
  return check_launch("upsample2");
}

int up_bwd_nd(const void* dout, int32_t dout_cstride, int32_t dout_coff, void* din, int32_t B, int32_t D, int32_t H,
              int32_t W, int32_t C, int nd, void* stream) {
  const size_t n = (size_t)B * D * H * W * C;
  upsample2_bwd<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)dout, dout_cstride, dout_coff,
                                                                      (bf16*)din, B, D, H, W, C, nd);
  return check_launch("upsample2_bwd");
}

}  // namespace

extern "C" {

int32_t lbm_nn_conv(const void* in, int32_t in_cstride, int32_t in_coff, const void* w, const float* bias,
                    const void* gate, void* out_bf16, float* out_f32, int32_t out_cstride, int32_t out_coff,
                    int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout, int32_t ksize, int32_t relu,
                    int32_t accumulate, void* stream) {
  return conv_nd(in, in_cstride, in_coff, w, bias, gate, out_bf16, out_f32, out_cstride, out_coff, B, 1, H, W, Cin,
                 Cout, ksize, relu, accumulate, 2, stream);
}

int32_t lbm_nn_conv3d(const void* in, int32_t in_cstride, int32_t in_coff, const void* w, const float* bias,
                      const void* gate, void* out_bf16, float* out_f32, int32_t out_cstride, int32_t out_coff,
                      int32_t B, int32_t D, int32_t H, int32_t W, int32_t Cin, int32_t Cout, int32_t ksize,
                      int32_t relu, int32_t accumulate, void* stream) {
  return conv_nd(in, in_cstride, in_coff, w, bias, gate, out_bf16, out_f32, out_cstride, out_coff, B, D, H, W, Cin,
                 Cout, ksize, relu, accumulate, 3, stream);
}

int32_t lbm_nn_conv_wgrad(const void* in, int32_t in_cstride, int32_t in_coff, const void* dout, int32_t dout_cstride,
                          int32_t dout_coff, float* dw, int32_t B, int32_t H, int32_t W, int32_t Cin, int32_t Cout,
                          int32_t ksize, void* stream) {
  return wgrad_nd(in, in_cstride, in_coff, dout, dout_cstride, dout_coff, dw, B, 1, H, W, Cin, Cout, ksize, 2, stream);
}

int32_t lbm_nn_conv3d_wgrad(const void* in, int32_t in_cstride, int32_t in_coff, const void* dout,
                            int32_t dout_cstride, int32_t dout_coff, float* dw, int32_t B, int32_t D, int32_t H,
                            int32_t W, int32_t Cin, int32_t Cout, int32_t ksize, void* stream) {
  return wgrad_nd(in, in_cstride, in_coff, dout, dout_cstride, dout_coff, dw, B, D, H, W, Cin, Cout, ksize, 3, stream);
}

int32_t lbm_nn_bias_grad(const void* dout, int32_t cstride, int32_t coff, int32_t P, int32_t Cout, float* dbias,
                         void* stream) {
  if (!dout || !dbias) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_bias_grad: NULL argument");
  const int splits = std::min(256, std::max(1, P / 256));
  bias_grad<<<dim3((Cout + 31) / 32, splits), 256, 0, (cudaStream_t)stream>>>((const bf16*)dout, cstride, coff, P, Cout,
                                                                             dbias);
  return check_launch("bias_grad");
}

int32_t lbm_nn_flip_weights(const void* w, void* wt, int32_t Cout, int32_t taps, int32_t Cin, void* stream) {
  const size_t n = (size_t)Cout * taps * Cin;
  flip_weights<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((const bf16*)w, (bf16*)wt, Cout, taps, Cin);
  return check_launch("flip_weights");
}

int32_t lbm_nn_avgpool2(const void* in, int32_t in_cstride, int32_t in_coff, void* out, int32_t B, int32_t H, int32_t W,
                        int32_t C, void* stream) {
  return pool_nd(in, in_cstride, in_coff, out, B, 1, H, W, C, 2, stream);
}
int32_t lbm_nn_avgpool2_3d(const void* in, int32_t in_cstride, int32_t in_coff, void* out, int32_t B, int32_t D,
                           int32_t H, int32_t W, int32_t C, void* stream) {
  return pool_nd(in, in_cstride, in_coff, out, B, D, H, W, C, 3, stream);
}

int32_t lbm_nn_avgpool2_bwd(const void* dout, void* din, int32_t din_cstride, int32_t din_coff, int32_t B, int32_t H,
                            int32_t W, int32_t C, int32_t accumulate, void* stream) {
  return pool_bwd_nd(dout, din, din_cstride, din_coff, B, 1, H, W, C, accumulate, 2, stream);
}
int32_t lbm_nn_avgpool2_3d_bwd(const void* dout, void* din, int32_t din_cstride, int32_t din_coff, int32_t B, int32_t D,
                               int32_t H, int32_t W, int32_t C, int32_t accumulate, void* stream) {
  return pool_bwd_nd(dout, din, din_cstride, din_coff, B, D, H, W, C, accumulate, 3, stream);
}

int32_t lbm_nn_upsample2(const void* in, void* out, int32_t out_cstride, int32_t out_coff, int32_t B, int32_t H,
                         int32_t W, int32_t C, void* stream) {
  return up_nd(in, out, out_cstride, out_coff, B, 1, H, W, C, 2, stream);
}
int32_t lbm_nn_upsample2_3d(const void* in, void* out, int32_t out_cstride, int32_t out_coff, int32_t B, int32_t D,
                            int32_t H, int32_t W, int32_t C, void* stream) {
  return up_nd(in, out, out_cstride, out_coff, B, D, H, W, C, 3, stream);
}

int32_t lbm_nn_upsample2_bwd(const void* dout, int32_t dout_cstride, int32_t dout_coff, void* din, int32_t B, int32_t H,
                             int32_t W, int32_t C, void* stream) {
  return up_bwd_nd(dout, dout_cstride, dout_coff, din, B, 1, H, W, C, 2, stream);
}
int32_t lbm_nn_upsample2_3d_bwd(const void* dout, int32_t dout_cstride, int32_t dout_coff, void* din, int32_t B,
                                int32_t D, int32_t H, int32_t W, int32_t C, void* stream) {
  return up_bwd_nd(dout, dout_cstride, dout_coff, din, B, D, H, W, C, 3, stream);
}

int32_t lbm_nn_mse(const float* pred, const float* target, const float* weight, size_t n, float scale, void* grad,
                   float* partial, int32_t nblocks, void* stream) {
  if (nblocks < 1 || nblocks > 4096) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_mse: 1..4096 blocks");
  mse_loss<<<nblocks, 256, 0, (cudaStream_t)stream>>>(pred, target, weight, n, scale, (bf16*)grad, partial);
  return check_launch("mse_loss");
}

int32_t lbm_nn_adam(float* w, const float* g, float* m, float* v, void* w_bf16, size_t n, float lr, float beta1,
                    float beta2, float eps, int32_t step, float weight_decay, void* stream) {
  if (step < 1) return lbm::capi::fail(LBM_NN_ERR_ARG, "lbm_nn_adam: step counts from 1");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_step<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (bf16*)w_bf16, n, lr, beta1, beta2, eps, c1,
                                                                   c2, weight_decay);
  return check_launch("adam_step");
}

int32_t lbm_nn_relu_bwd(void* dy, int32_t dy_cstride, int32_t dy_coff, const void* y, int32_t y_cstride,
                        int32_t y_coff, int32_t P, int32_t C, void* stream) {
  const size_t n = (size_t)P * C;
  relu_bwd<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>((bf16*)dy, dy_cstride, dy_coff, (const bf16*)y, y_cstride,
                                                                 y_coff, (size_t)P, C);
  return check_launch("relu_bwd");
}

int32_t lbm_nn_to_bf16(const float* x, void* y, size_t n, void* stream) {
  to_bf16<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(x, (bf16*)y, n);
  return check_launch("to_bf16");
}

}  // extern "C"
