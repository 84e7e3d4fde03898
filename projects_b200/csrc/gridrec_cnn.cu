// Learned correction for narrow-kernel gridrec: a 3-layer, 16-channel, 3x3
// residual CNN on the reconstructed slice,
//   h1 = relu(conv1(x)), h2 = relu(conv2(h1)), y = x + conv3(h2),
// conv1: 1 -> 16, conv2: 16 -> 16, conv3: 16 -> 1, zero padding, biases.
// Hidden activations are stored in BF16, channels last (16 per pixel); every
// sum accumulates in FP32.  conv2 -- 2304 of the 2592 multiply-adds per pixel --
// runs on the tensor cores (mma.sync m16n8k16, BF16 in, FP32 accumulate), in the
// forward pass and, with flipped and transposed weights, for the gradient with
// respect to its input; the thin 1 -> 16 and 16 -> 1 layers and the weight
// gradients (sums over all pixels) run on the CUDA cores with fixed-order
// partial sums, so training is deterministic.
//
// Parameters: one float32 array of kCnnParams entries:
//   w1[tap][co] (144), b1 (16), w2[tap][co][ci] (2304), b2 (16), w3[tap][ci] (144), b3 (1)
// with tap = (dy + 1) * 3 + (dx + 1) and conv(x)[p] = b + sum_tap w[tap] x[p + (dy, dx)].
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "gr_device.cuh"
#include "gr_internal.h"

namespace gr {
namespace {

constexpr int kC = 16;
constexpr int kW1 = 0, kB1 = 144, kW2 = 160, kB2 = 2464, kW3 = 2480, kB3 = 2624;
constexpr int kCnnParams = 2625;

__device__ __forceinline__ int tap_dy(int tap) { return tap / 3 - 1; }
__device__ __forceinline__ int tap_dx(int tap) { return tap % 3 - 1; }

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}
__device__ __forceinline__ float2 unpack_bf16(unsigned u) {
  const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&u);
  return __bfloat1622float2(v);
}

// ---------------------------------------------------------------- conv1 (1 -> 16)
__global__ void cnn_conv1_kernel(const float* params, const float* x, __nv_bfloat16* h1, int h,
                                 int w) {
  __shared__ float sp[kB1 + kC];  // w1, b1
  for (int i = threadIdx.x; i < kB1 + kC; i += blockDim.x) sp[i] = params[i];
  __syncthreads();
  const int xi = blockIdx.x * blockDim.x + threadIdx.x, yi = blockIdx.y, im = blockIdx.z;
  if (xi >= w) return;
  const float* xm = x + (size_t)im * h * w;
  float in[9];
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    const int yy = yi + tap_dy(tap), xx = xi + tap_dx(tap);
    in[tap] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? xm[(size_t)yy * w + xx] : 0.f;
  }
  unsigned o[kC / 2];
#pragma unroll
  for (int c = 0; c < kC; c += 2) {
    float z0 = sp[kB1 + c], z1 = sp[kB1 + c + 1];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      z0 = fmaf(sp[kW1 + tap * kC + c], in[tap], z0);
      z1 = fmaf(sp[kW1 + tap * kC + c + 1], in[tap], z1);
    }
    o[c / 2] = pack_bf16(fmaxf(z0, 0.f), fmaxf(z1, 0.f));
  }
  uint4* out = reinterpret_cast<uint4*>(h1 + (((size_t)im * h + yi) * w + xi) * kC);
  out[0] = make_uint4(o[0], o[1], o[2], o[3]);
  out[1] = make_uint4(o[4], o[5], o[6], o[7]);
}

// ---------------------------------------------------------------- conv2 (16 -> 16), tensor cores
// One warp: 16 consecutive pixels of a row (the M = 16 rows of the mma) x 16
// output channels (two n = 8 tiles); K = 16 input channels per tap, 9 taps.
// Fragments of mma.m16n8k16 (g = lane / 4, t = lane % 4): A rows g, g + 8 and
// columns 2t, 2t + 1, 2t + 8, 2t + 9 (pixel, input channel); B rows (input
// channels) 2t, 2t + 1, 2t + 8, 2t + 9 of column g (output channel); D rows g,
// g + 8, columns 2t, 2t + 1.
// backward = 0: out = relu(conv2(in) + b2).  backward = 1: the gradient with
// respect to conv2's input, conv with w'[tap][ci][co] = w2[8 - tap][co][ci]
// (no bias), times (mask > 0) -- the ReLU of h1.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0,
                                         unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

constexpr int kConv2Tiles = 4;  // 16-pixel tiles per warp

__global__ void __launch_bounds__(128) cnn_conv2_kernel(const float* params,
                                                        const __nv_bfloat16* in,
                                                        const __nv_bfloat16* mask,
                                                        __nv_bfloat16* out, int h, int w,
                                                        int backward) {
  // B fragments (packed BF16 pairs) of all taps and both output-channel tiles,
  // built once per block from the FP32 weights: sb[tap][nt][half][lane]
  __shared__ unsigned sb[9 * 2 * 2 * 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < 9 * 2 * 2 * 32; e += blockDim.x) {
    const int ln = e & 31, half = (e >> 5) & 1, nt = (e >> 6) & 1, tap = e >> 7;
    const int n = nt * 8 + (ln >> 2);       // output channel
    const int k = 2 * (ln & 3) + 8 * half;  // input channels k, k + 1
    float w0, w1;
    if (!backward) {
      w0 = params[kW2 + (tap * kC + n) * kC + k];
      w1 = params[kW2 + (tap * kC + n) * kC + k + 1];
    } else {
      w0 = params[kW2 + ((8 - tap) * kC + k) * kC + n];
      w1 = params[kW2 + ((8 - tap) * kC + k + 1) * kC + n];
    }
    sb[e] = pack_bf16(w0, w1);
  }
  __syncthreads();
  const int g = lane >> 2, t = lane & 3;
  const int yi = blockIdx.y, im = blockIdx.z;
  for (int mt = 0; mt < kConv2Tiles; ++mt) {
  const int x0 = ((blockIdx.x * 4 + warp) * kConv2Tiles + mt) * 16;
  if (x0 >= w) return;
  const unsigned* in32 = reinterpret_cast<const unsigned*>(in) + (size_t)im * h * w * (kC / 2);
  float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    const int yy = yi + tap_dy(tap);
    const int xa = x0 + g + tap_dx(tap), xb = xa + 8;
    const bool row_ok = yy >= 0 && yy < h;
    const bool oka = row_ok && xa >= 0 && xa < w, okb = row_ok && xb >= 0 && xb < w;
    const size_t pa = ((size_t)yy * w + xa) * (kC / 2), pb = ((size_t)yy * w + xb) * (kC / 2);
    unsigned a[4];
    a[0] = oka ? __ldg(&in32[pa + t]) : 0u;      // row g, channels 2t, 2t+1
    a[1] = okb ? __ldg(&in32[pb + t]) : 0u;      // row g + 8
    a[2] = oka ? __ldg(&in32[pa + t + 4]) : 0u;  // row g, channels 2t+8, 2t+9
    a[3] = okb ? __ldg(&in32[pb + t + 4]) : 0u;
    const unsigned* b = sb + tap * 128 + lane;
    mma_bf16(acc[0], a, b[0], b[32]);
    mma_bf16(acc[1], a, b[64], b[96]);
  }
  unsigned* out32 = reinterpret_cast<unsigned*>(out) + (size_t)im * h * w * (kC / 2);
  const unsigned* m32 =
      mask ? reinterpret_cast<const unsigned*>(mask) + (size_t)im * h * w * (kC / 2) : nullptr;
#pragma unroll
  for (int nt = 0; nt < 2; ++nt) {
    const int c = nt * 8 + 2 * t;  // output channels c, c + 1
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      const int xi = x0 + g + 8 * half;
      if (xi >= w) continue;
      float z0 = acc[nt][2 * half], z1 = acc[nt][2 * half + 1];
      const size_t po = ((size_t)yi * w + xi) * (kC / 2) + c / 2;
      if (!backward) {
        z0 = fmaxf(z0 + __ldg(&params[kB2 + c]), 0.f);
        z1 = fmaxf(z1 + __ldg(&params[kB2 + c + 1]), 0.f);
      } else {
        const float2 m = unpack_bf16(__ldg(&m32[po]));
        z0 = m.x > 0.f ? z0 : 0.f;
        z1 = m.y > 0.f ? z1 : 0.f;
      }
      out32[po] = pack_bf16(z0, z1);
    }
  }
  }  // tiles
}

// ---------------------------------------------------------------- conv3 (16 -> 1) + residual
__global__ void cnn_conv3_kernel(const float* params, const float* x, const __nv_bfloat16* h2,
                                 float* y, int h, int w) {
  __shared__ float sp[9 * kC + 1];  // w3, b3
  for (int i = threadIdx.x; i < 9 * kC + 1; i += blockDim.x) sp[i] = params[kW3 + i];
  __syncthreads();
  const int xi = blockIdx.x * blockDim.x + threadIdx.x, yi = blockIdx.y, im = blockIdx.z;
  if (xi >= w) return;
  const uint4* h128 = reinterpret_cast<const uint4*>(h2) + (size_t)im * h * w * 2;
  float z = sp[9 * kC];
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    const int yy = yi + tap_dy(tap), xx = xi + tap_dx(tap);
    if (yy < 0 || yy >= h || xx < 0 || xx >= w) continue;
    const uint4* p = h128 + ((size_t)yy * w + xx) * 2;
    const uint4 q0 = __ldg(&p[0]), q1 = __ldg(&p[1]);
    const unsigned u[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
    for (int c = 0; c < kC; c += 2) {
      const float2 v = unpack_bf16(u[c / 2]);
      z = fmaf(sp[tap * kC + c], v.x, z);
      z = fmaf(sp[tap * kC + c + 1], v.y, z);
    }
  }
  const size_t o = ((size_t)im * h + yi) * w + xi;
  y[o] = x[o] + z;
}

// ---------------------------------------------------------------- backward pieces
// loss = mean (y - target)^2; gy = 2 (y - target) / N; per-block loss partials.
__global__ void cnn_loss_kernel(const float* y, const float* target, float* gy, double* part,
                                long n) {
  __shared__ double red[8];
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float d = y[i] - target[i];
    gy[i] = 2.f * d / (float)n;
    s += (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    part[blockIdx.x] = t;
  }
}

// g_z2[p][c] = (h2[p][c] > 0) * sum_tap w3[tap][c] gy[p - (dy, dx)]
__global__ void cnn_conv3_bwd_kernel(const float* params, const float* gy,
                                     const __nv_bfloat16* h2, __nv_bfloat16* gz2, int h, int w) {
  const int xi = blockIdx.x * blockDim.x + threadIdx.x, yi = blockIdx.y, im = blockIdx.z;
  if (xi >= w) return;
  const float* gm = gy + (size_t)im * h * w;
  float gin[9];
#pragma unroll
  for (int tap = 0; tap < 9; ++tap) {
    const int yy = yi - tap_dy(tap), xx = xi - tap_dx(tap);
    gin[tap] = (yy >= 0 && yy < h && xx >= 0 && xx < w) ? gm[(size_t)yy * w + xx] : 0.f;
  }
  const size_t p = ((size_t)im * h + yi) * w + xi;
  const unsigned* h32 = reinterpret_cast<const unsigned*>(h2) + p * (kC / 2);
  unsigned* g32 = reinterpret_cast<unsigned*>(gz2) + p * (kC / 2);
#pragma unroll
  for (int c = 0; c < kC; c += 2) {
    float z0 = 0.f, z1 = 0.f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      z0 = fmaf(__ldg(&params[kW3 + tap * kC + c]), gin[tap], z0);
      z1 = fmaf(__ldg(&params[kW3 + tap * kC + c + 1]), gin[tap], z1);
    }
    const float2 m = unpack_bf16(__ldg(&h32[c / 2]));
    g32[c / 2] = pack_bf16(m.x > 0.f ? z0 : 0.f, m.y > 0.f ? z1 : 0.f);
  }
}

// Weight gradients of all three layers over one row segment of kSeg pixels:
// partial sums of the kCnnParams gradient entries, written to part[segment].
constexpr int kSeg = 128;

__global__ void __launch_bounds__(256) cnn_wgrad_kernel(const float* x, const float* gy,
                                                        const __nv_bfloat16* h1,
                                                        const __nv_bfloat16* h2,
                                                        const __nv_bfloat16* gz1,
                                                        const __nv_bfloat16* gz2, float* part,
                                                        int h, int w, int segs_per_row) {
  extern __shared__ float sm[];
  const int W2 = kSeg + 2;
  float* s_x = sm;                       // [3][W2]
  float* s_h1 = s_x + 3 * W2;            // [3][W2][16]
  float* s_h2 = s_h1 + 3 * W2 * kC;      // [3][W2][16]
  float* s_gz1 = s_h2 + 3 * W2 * kC;     // [kSeg][16]
  float* s_gz2 = s_gz1 + kSeg * kC;      // [kSeg][16]
  float* s_gy = s_gz2 + kSeg * kC;       // [kSeg]
  const int seg = blockIdx.x % segs_per_row, yi = blockIdx.x / segs_per_row, im = blockIdx.y;
  const int x0 = seg * kSeg;
  const size_t img = (size_t)im * h * w;
  for (int i = threadIdx.x; i < 3 * W2; i += blockDim.x) {
    const int r = i / W2, c = i % W2;
    const int yy = yi + r - 1, xx = x0 + c - 1;
    const bool ok = yy >= 0 && yy < h && xx >= 0 && xx < w;
    const size_t p = img + (size_t)yy * w + xx;
    s_x[i] = ok ? x[p] : 0.f;
    for (int ch = 0; ch < kC; ++ch) {
      s_h1[i * kC + ch] = ok ? __bfloat162float(h1[p * kC + ch]) : 0.f;
      s_h2[i * kC + ch] = ok ? __bfloat162float(h2[p * kC + ch]) : 0.f;
    }
  }
  for (int i = threadIdx.x; i < kSeg; i += blockDim.x) {
    const int xx = x0 + i;
    const bool ok = xx < w;
    const size_t p = img + (size_t)yi * w + xx;
    s_gy[i] = ok ? gy[p] : 0.f;
    for (int ch = 0; ch < kC; ++ch) {
      s_gz1[i * kC + ch] = ok ? __bfloat162float(gz1[p * kC + ch]) : 0.f;
      s_gz2[i * kC + ch] = ok ? __bfloat162float(gz2[p * kC + ch]) : 0.f;
    }
  }
  __syncthreads();
  float* out = part + ((size_t)im * gridDim.x + blockIdx.x) * kCnnParams;
  const int tid = threadIdx.x;
  // dW2[tap][co][ci] = sum_p gz2[p][co] h1[p + off][ci]; thread = (co, ci), all taps
  {
    const int co = tid / kC, ci = tid % kC;
    float a[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < kSeg; ++i) {
      const float gv = s_gz2[i * kC + co];
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int r = tap / 3, c = i + tap % 3;
        a[tap] = fmaf(gv, s_h1[(r * W2 + c) * kC + ci], a[tap]);
      }
    }
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) out[kW2 + (tap * kC + co) * kC + ci] = a[tap];
  }
  if (tid < kC) {  // dW1[tap][co] = sum_p gz1[p][co] x[p + off]; db1
    float a[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, b = 0.f;
    for (int i = 0; i < kSeg; ++i) {
      const float gv = s_gz1[i * kC + tid];
      b += gv;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) a[tap] = fmaf(gv, s_x[(tap / 3) * W2 + i + tap % 3], a[tap]);
    }
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) out[kW1 + tap * kC + tid] = a[tap];
    out[kB1 + tid] = b;
  } else if (tid < 2 * kC) {  // db2
    const int c = tid - kC;
    float b = 0.f;
    for (int i = 0; i < kSeg; ++i) b += s_gz2[i * kC + c];
    out[kB2 + c] = b;
  } else if (tid < 3 * kC) {  // dW3[tap][ci] = sum_p gy[p] h2[p + off][ci]
    const int ci = tid - 2 * kC;
    float a[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < kSeg; ++i) {
      const float gv = s_gy[i];
#pragma unroll
      for (int tap = 0; tap < 9; ++tap)
        a[tap] = fmaf(gv, s_h2[((tap / 3) * W2 + i + tap % 3) * kC + ci], a[tap]);
    }
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) out[kW3 + tap * kC + ci] = a[tap];
  } else if (tid == 3 * kC) {
    float b = 0.f;
    for (int i = 0; i < kSeg; ++i) b += s_gy[i];
    out[kB3] = b;
  }
}

// grads[k] = sum over segments (fixed order) of part[seg][k]
__global__ void cnn_reduce_kernel(const float* part, long nseg, float* grads) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= kCnnParams) return;
  double s = 0.0;
  for (long i = 0; i < nseg; ++i) s += part[i * kCnnParams + k];
  grads[k] = (float)s;
}

__global__ void cnn_adam_kernel(float* params, const float* grads, float* m, float* v, int n,
                                float lr, float b1, float b2, float eps, float c1, float c2) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float g = grads[k];
  const float mk = b1 * m[k] + (1.f - b1) * g;
  const float vk = b2 * v[k] + (1.f - b2) * g * g;
  m[k] = mk;
  v[k] = vk;
  params[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

// ---------------------------------------------------------------- fused inference, tcgen05
// One CTA (kFThreads / 32 warps) computes output tiles of kFTh x kFTw pixels.  The tile's x region
// ((kFTh + 6) x (kFTw + 6) pixels), its h1 and h2 and conv3's per-tap partials stay in
// shared memory; only x is read from HBM and y written.  Positions of the x region are
// flattened with row stride kFWt, so a 3x3 tap (dy, dx) is the constant offset
// dy kFWt + dx: conv2 on a block of 128 consecutive positions is nine tcgen05 MMAs whose
// A operand is the same activation plane started dy kFWt + dx positions later -- no
// im2col copy.  The layers:
//  * conv1 (1 -> 16): a tcgen05 MMA per block of 128 positions on a 16-wide im2col of x
//    (the nine taps and seven zeros, BF16) built in shared memory, against w1 in BF16,
//    on the rows conv2 reads (rows 1..kFTh+4 of the x region); the im2col is dead once
//    the MMAs are done, and h1 = relu(conv1 + b1) in BF16 is written over it;
//  * conv2 (16 -> 16): tcgen05.mma kind::f16, BF16 operands from shared memory (A: 128
//    positions x 16 input channels, K-major, two 8-channel planes; B: the tap's 16 x 16
//    weights), FP32 accumulator in tensor memory (M = 128, N = 16, K = 16; one MMA per
//    tap), then bias, ReLU and BF16 on the way back to shared memory;
//  * conv3 (16 -> 1): a 1x1 tcgen05 MMA to the nine per-tap partials
//    Z[p][tap] = sum_ci w3[tap][ci] h2[p][ci] (w3 in BF16; N = 16, taps 9..15 zero), then
//    y[p] = x[p] + (b3 + sum_tap Z[p + (dy, dx)][tap]) in FP32 on the CUDA cores.  (Nine
//    shifted MMAs into one column would drop the partials, but every N = 16 MMA reads its
//    4 KB A operand from shared memory, about 30 cycles of the SM's shared-memory
//    bandwidth: eight more of them per block cost more than the partials' stores and loads.)
// Positions outside the image hold zero x, h1 and h2 (the network's zero padding); the
// wrap-around columns of the flattened rows produce values only at positions that no
// kept output reads.  One thread issues the MMAs; completion is a tcgen05.commit on an
// mbarrier with bounded waits (timeout: error word, early exit).  Each CTA holds
// kFTmemCols tensor-memory columns; its dynamic shared memory (kFSmemLaunch) admits at
// most kFCtas CTAs per SM, whose allocations fit the SM's 512 columns together, so an
// allocation never waits on another CTA.

constexpr int kFTh = 8, kFTw = 64;
constexpr int kFThreads = 128, kFCtas = 4;                     // 4 warps, 4 CTAs per SM
constexpr int kFGroups = kFThreads / 128;                      // warp groups sharing the blocks
constexpr int kFWt = kFTw + 6;                                 // flattened row stride
constexpr int kFRows = kFTh + 6;
constexpr int kFPos = kFRows * kFWt;                           // positions of the x region
constexpr int kFQ1 = kFWt, kFQ1e = (kFTh + 5) * kFWt;          // conv1: rows 1..kFTh+4
constexpr int kFQ2 = 2 * kFWt;                                 // first conv2 / conv3 position
constexpr int kFBlocks = ((kFTh + 4) * kFWt - kFQ2 + 127) / 128;  // 128-position blocks
constexpr int kFBlocks1 = (kFQ1e - kFQ1 + 127) / 128;           // conv1's blocks from kFQ1
constexpr int kFZ = 128 * kFBlocks;                            // partials per tap
constexpr int kFPlane = ((kFQ1 + 128 * kFBlocks1 > kFQ2 + kFZ + kFWt + 1 ? kFQ1 + 128 * kFBlocks1
                                                                         : kFQ2 + kFZ + kFWt + 1) +
                         127) / 128 * 128;                     // positions per activation plane
constexpr int kFXOff = 72;                                     // x buffer: reads at q - 71 .. q + 71
constexpr int kFXLen = kFPos + 2 * kFXOff;
constexpr int kFTmemNeed = 16 * (kFBlocks1 > kFBlocks ? kFBlocks1 : kFBlocks);
constexpr int kFTmemCols = kFTmemNeed <= 32 ? 32 : kFTmemNeed <= 64 ? 64 : kFTmemNeed <= 128 ? 128
                                                                                                : 256;
constexpr int kFParams = 177;                                  // w1, b1, b2, b3 in FP32
// shared memory: activation planes | B2 (9 taps) | B3 | B1 | x | FP32 params | mbarrier, tmem slot
constexpr int kFSmAct = 0, kFSmB2 = 2 * kFPlane * 16, kFSmB3 = kFSmB2 + 9 * 512;
constexpr int kFSmB1 = kFSmB3 + 512;
constexpr int kFSmX = kFSmB1 + 512, kFSmP = kFSmX + kFXLen * 4;
constexpr int kFSmBar = (kFSmP + kFParams * 4 + 15) & ~15;
constexpr int kFSmUsed = kFSmBar + 16;
constexpr int kFSmemLaunch = (228 * 1024 / kFCtas - 1024) & ~1023;
static_assert(kFQ2 + kFZ + kFWt + 1 <= kFPlane, "conv2's shifted reads stay inside the planes");
static_assert(kFQ1 + 128 * kFBlocks1 <= kFPlane, "conv1's blocks fit the planes");
static_assert(kFTmemNeed <= kFTmemCols && kFCtas * kFTmemCols <= 512,
              "accumulators fit the tensor-memory allocation, and every CTA of an SM gets one");
static_assert(9 * kFZ * 4 <= 2 * kFPlane * 16, "conv3's partials fit the activation buffer");
static_assert(kFSmUsed <= kFSmemLaunch && (kFCtas + 1) * (kFSmemLaunch + 1024) > 228 * 1024,
              "at most kFCtas CTAs per SM");

__device__ __forceinline__ uint64_t cnn_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  // start >> 4 [0,14), leading-dimension offset >> 4 [16,30), stride offset >> 4
  // [32,46), version 1 [46,48); no swizzle, base offset 0 (K-major core matrices of
  // 8 rows x 16 bytes)
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// instruction descriptor: D f32 [4,6) = 1, A bf16 [7,10) = 1, B bf16 [10,13) = 1, both
// K-major, N = 16 [17,23) = 16 >> 3, M = 128 [24,29) = 128 >> 4
constexpr uint32_t kCnnIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                               ((128u >> 4) << 24);

__device__ __forceinline__ void cnn_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(kCnnIdesc), "r"(acc));
}
__device__ __forceinline__ void cnn_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
// relu(v + b) of two channels in BF16 (packed FP32 add, then one converting relu)
__device__ __forceinline__ unsigned relu_bias_pack(float v0, float v1, float b0, float b1) {
  unsigned long long s;
  asm("{\n .reg .b64 x, y;\n mov.b64 x, {%1, %2};\n mov.b64 y, {%3, %4};\n"
      " add.rn.f32x2 %0, x, y;\n}" : "=l"(s) : "f"(v0), "f"(v1), "f"(b0), "f"(b1));
  unsigned r;
  asm("{\n .reg .f32 lo, hi;\n mov.b64 {lo, hi}, %1;\n cvt.rn.relu.bf16x2.f32 %0, hi, lo;\n}"
      : "=r"(r) : "l"(s));
  return r;
}
// 16 accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void cnn_tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

__global__ void __launch_bounds__(kFThreads, kFCtas) cnn_fused_kernel(const float* params, const float* x,
                                                                       float* y, const float* scale,
                                                                       int n_img, int h, int w,
                                                                       int* err) {
  extern __shared__ __align__(1024) unsigned char smf[];
  uint4* act = reinterpret_cast<uint4*>(smf + kFSmAct);  // plane g: act[g kFPlane + q] = 8 BF16 channels
  unsigned short* b2s = reinterpret_cast<unsigned short*>(smf + kFSmB2);
  unsigned short* b3s = reinterpret_cast<unsigned short*>(smf + kFSmB3);
  unsigned short* b1s = reinterpret_cast<unsigned short*>(smf + kFSmB1);
  float* xs = reinterpret_cast<float*>(smf + kFSmX) + kFXOff;
  float* pw = reinterpret_cast<float*>(smf + kFSmP);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smf + kFSmBar);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smf + kFSmBar + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // B operands in BF16, K-major core matrices [ci / 8][n][ci % 8]: conv2's taps (n = co)
  // and conv3's 1x1 matrix (n = tap, taps 9..15 zero); FP32 w1, b1, b2, b3
  for (int e = tid; e < 9 * 256; e += kFThreads) {
    const int t = e >> 8, g = (e >> 7) & 1, co = (e >> 3) & 15, k8 = e & 7;
    const __nv_bfloat16 v = __float2bfloat16_rn(params[kW2 + (t * kC + co) * kC + g * 8 + k8]);
    b2s[e] = *reinterpret_cast<const unsigned short*>(&v);
  }
  for (int e = tid; e < 256; e += kFThreads) {
    const int g = e >> 7, n = (e >> 3) & 15, k8 = e & 7;
    const __nv_bfloat16 v = __float2bfloat16_rn(n < 9 ? params[kW3 + n * kC + g * 8 + k8] : 0.f);
    b3s[e] = *reinterpret_cast<const unsigned short*>(&v);
  }
  for (int e = tid; e < 256; e += kFThreads) {  // conv1: n = co, k = tap (taps 9..15 zero)
    const int g = e >> 7, co = (e >> 3) & 15, k = g * 8 + (e & 7);
    const __nv_bfloat16 v = __float2bfloat16_rn(k < 9 ? params[kW1 + k * kC + co] : 0.f);
    b1s[e] = *reinterpret_cast<const unsigned short*>(&v);
  }
  for (int i = tid; i < kFParams; i += kFThreads)
    pw[i] = i < kB1 + kC ? params[i] : (i < kB1 + 2 * kC ? params[kB2 + i - kB1 - kC] : params[kB3]);
  for (int i = tid; i < kFXLen; i += kFThreads) xs[i - kFXOff] = 0.f;
  for (int i = tid; i < 2 * kFPlane; i += kFThreads) act[i] = make_uint4(0u, 0u, 0u, 0u);
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tslot)), "n"(kFTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_proxy_async();  // the B operands and zeroed planes, before the tensor core reads them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  // descriptors: a position offset q adds q to the start-address field (16-byte units)
  const uint64_t da = cnn_smem_desc(smem_u32(act), kFPlane * 16, 128);
  const uint64_t db1 = cnn_smem_desc(smem_u32(b1s), 256, 128);
  const uint64_t db2 = cnn_smem_desc(smem_u32(b2s), 256, 128);
  const uint64_t db3 = cnn_smem_desc(smem_u32(b3s), 256, 128);
  const float b3 = pw[kB1 + 2 * kC];
  float bias1[kC], bias2[kC];
#pragma unroll
  for (int c = 0; c < kC; ++c) {
    bias1[c] = pw[kB1 + c];
    bias2[c] = pw[kB1 + kC + c];
  }
  const int tiles_x = (w + kFTw - 1) / kFTw, tiles_y = (h + kFTh - 1) / kFTh;
  const long n_tiles = (long)n_img * tiles_x * tiles_y;
  const int lq = warp & 3;  // this warp's quarter of the tensor-memory lanes
  unsigned phase = 0;
  bool ok = true;
  // the x region of a tile (zero outside the image), this thread's positions
  // tid + k kFThreads; loaded one tile ahead into registers, so that the loads' latency
  // passes during the previous tile's work
  constexpr int kXPer = (kFPos + kFThreads - 1) / kFThreads;
  float xr[kXPer], x_inv = 1.f;
  const int r_tid = tid / kFWt, c_tid = tid - r_tid * kFWt;
  auto load_x = [&](long t) {
    const int im = (int)(t / ((long)tiles_x * tiles_y));
    const int rem = (int)(t - (long)im * tiles_x * tiles_y);
    const int ty0 = (rem / tiles_x) * kFTh, tx0 = (rem % tiles_x) * kFTw;
    const bool all_in = t < n_tiles && ty0 >= 3 && tx0 >= 3 && ty0 + kFTh + 3 <= h &&
                        tx0 + kFTw + 3 <= w;
    const float* xm = x + (size_t)im * h * w;
    // the image's 1 / scale, applied when the values are stored to shared memory (a
    // product here would wait on the loads)
    x_inv = scale && t < n_tiles ? 1.f / __ldg(&scale[im]) : 1.f;
    int r = r_tid, c = c_tid;  // position tid + k kFThreads = (r, c)
#pragma unroll
    for (int k = 0; k < kXPer; ++k) {
      const int iy = ty0 - 3 + r, ix = tx0 - 3 + c;
      const bool in = tid + k * kFThreads < kFPos &&
                      (all_in || (t < n_tiles && iy >= 0 && iy < h && ix >= 0 && ix < w));
      xr[k] = in ? __ldg(&xm[(size_t)iy * w + ix]) : 0.f;
      r += kFThreads / kFWt;
      c += kFThreads % kFWt;
      if (c >= kFWt) {
        c -= kFWt;
        ++r;
      }
    }
  };
  load_x(blockIdx.x);
  for (long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    const int im = (int)(tile / ((long)tiles_x * tiles_y));
    const int rem = (int)(tile - (long)im * tiles_x * tiles_y);
    const int y0 = (rem / tiles_x) * kFTh, x0 = (rem % tiles_x) * kFTw;
    // a tile whose x region lies inside the image needs no zero padding
    const bool all_in = y0 >= 3 && x0 >= 3 && y0 + kFTh + 3 <= h && x0 + kFTw + 3 <= w;
    auto inside = [&](int q) {
      if (all_in) return true;
      const int r = q / kFWt, c = q - (q / kFWt) * kFWt;
      const int iy = y0 - 3 + r, ix = x0 - 3 + c;
      return iy >= 0 && iy < h && ix >= 0 && ix < w;
    };
#pragma unroll
    for (int k = 0; k < kXPer; ++k)
      if (tid + k * kFThreads < kFPos) xs[tid + k * kFThreads] = xr[k] * x_inv;
    __syncthreads();
    load_x(tile + gridDim.x);  // the next tile's x, in flight during this tile
    // conv1's im2col (BF16): plane 0 holds taps 0..7 of position q, plane 1 tap 8 and
    // zeros; conv1's blocks cover [kFQ1, kFQ1 + 128 kFBlocks1)
    for (int q = kFQ1 + tid; q < kFQ1 + 128 * kFBlocks1; q += kFThreads) {
      float in[9];
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) in[tap] = xs[q + tap_dy(tap) * kFWt + tap_dx(tap)];
      act[q] = make_uint4(pack_bf16(in[0], in[1]), pack_bf16(in[2], in[3]),
                          pack_bf16(in[4], in[5]), pack_bf16(in[6], in[7]));
      act[kFPlane + q] = make_uint4(pack_bf16(in[8], 0.f), 0u, 0u, 0u);
    }
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int b = 0; b < kFBlocks1; ++b) cnn_mma(tmem + 16 * b, da + (kFQ1 + 128 * b), db1, 0u);
      cnn_commit(bar);
    }
    bool got = warp == 0 ? mbar_wait(bar, phase) : true;
    if (__syncthreads_or(!got)) {
      ok = false;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    // h1 = relu(conv1 + b1) in BF16 over the im2col (every MMA reading it is done); zero
    // outside the image and beyond conv1's rows; the planes' other positions are
    // cleared of the previous tile's values
    for (int b = warp >> 2; b < kFBlocks1; b += kFGroups) {
      float v[16];
      cnn_tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + 16 * b, v);
      const int q = kFQ1 + 128 * b + 32 * lq + lane;
      uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
      if (q < kFQ1e && inside(q)) {
        unsigned o[kC / 2];
#pragma unroll
        for (int c = 0; c < kC; c += 2) o[c / 2] = relu_bias_pack(v[c], v[c + 1], bias1[c], bias1[c + 1]);
        lo = make_uint4(o[0], o[1], o[2], o[3]);
        hi = make_uint4(o[4], o[5], o[6], o[7]);
      }
      act[q] = lo;
      act[kFPlane + q] = hi;
    }
    for (int i = tid; i < kFPlane - 128 * kFBlocks1; i += kFThreads) {
      const int q = i < kFQ1 ? i : i + 128 * kFBlocks1;
      act[q] = act[kFPlane + q] = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    // conv2: nine MMAs per block of 128 positions, A shifted by the tap's offset
    if (tid == 0) {
      tc_fence_after();
#pragma unroll 2
      for (int b = 0; b < kFBlocks; ++b)
#pragma unroll
        for (int t = 0; t < 9; ++t)
          cnn_mma(tmem + 16 * b, da + (kFQ2 + 128 * b + tap_dy(t) * kFWt + tap_dx(t)),
                  db2 + 32 * t, t > 0 ? 1u : 0u);
      cnn_commit(bar);
    }
    // one warp polls the barrier; the others wait at the CTA barrier (no issue slots)
    got = warp == 0 ? mbar_wait(bar, phase) : true;
    if (__syncthreads_or(!got)) {
      ok = false;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    // h2 = relu(conv2 + b2) in BF16 over h1's planes (every MMA reading h1 is done);
    // warp group g (4 warps, one per quarter of the lanes) takes blocks g, g + kFGroups, ...
    for (int b = warp >> 2; b < kFBlocks; b += kFGroups) {
      float v[16];
      cnn_tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + 16 * b, v);
      const int q = kFQ2 + 128 * b + 32 * lq + lane;
      uint4 lo = make_uint4(0u, 0u, 0u, 0u), hi = lo;
      if (inside(q)) {
        unsigned o[kC / 2];
#pragma unroll
        for (int c = 0; c < kC; c += 2) o[c / 2] = relu_bias_pack(v[c], v[c + 1], bias2[c], bias2[c + 1]);
        lo = make_uint4(o[0], o[1], o[2], o[3]);
        hi = make_uint4(o[4], o[5], o[6], o[7]);
      }
      act[q] = lo;
      act[kFPlane + q] = hi;
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    // conv3's 1x1 MMA: Z[q][tap] for every block
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int b = 0; b < kFBlocks; ++b) cnn_mma(tmem + 16 * b, da + (kFQ2 + 128 * b), db3, 0u);
      cnn_commit(bar);
    }
    got = warp == 0 ? mbar_wait(bar, phase) : true;
    if (__syncthreads_or(!got)) {
      ok = false;
      break;
    }
    phase ^= 1u;
    tc_fence_after();
    // partials into the activation buffer (h2 is consumed): z_s[tap][q - kFQ2]
    float* zs = reinterpret_cast<float*>(smf + kFSmAct);
    for (int b = warp >> 2; b < kFBlocks; b += kFGroups) {
      float v[16];
      cnn_tmem_ld16(tmem + ((uint32_t)(32 * lq) << 16) + 16 * b, v);
      const int qi = 128 * b + 32 * lq + lane;
#pragma unroll
      for (int t = 0; t < 9; ++t) zs[t * kFZ + qi] = v[t];
    }
    tc_fence_before();
    __syncthreads();
    // y = x + (b3 + sum_tap Z[p + (dy, dx)][tap])
    float* ym = y + (size_t)im * h * w;
    const float sc = scale ? __ldg(&scale[im]) : 1.f;
    for (int k = tid; k < kFTh * kFTw; k += kFThreads) {
      const int ry = k / kFTw, rx = k - ry * kFTw;
      const int iy = y0 + ry, ix = x0 + rx;
      if (iy >= h || ix >= w) continue;
      const int q = (ry + 3) * kFWt + rx + 3;
      float z = b3;
#pragma unroll
      for (int t = 0; t < 9; ++t) z += zs[t * kFZ + q + tap_dy(t) * kFWt + tap_dx(t) - kFQ2];
      ym[(size_t)iy * w + ix] = (xs[q] + z) * sc;
    }
    __syncthreads();  // x and the partials are read before the next tile overwrites them
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // the MMAs in flight finish before the tensor memory is released
    if (warp == 0) mbar_wait(bar, phase);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "n"(kFTmemCols)
                 : "memory");
}

int cnn_check(int n_img, int h, int w) {
  if (n_img < 1 || h < 1 || w < 1 || n_img > 65535 || h > 65535)
    return fail(GR_ERR_ARG, "cnn: need 1 <= n_img, h <= 65535 and w >= 1");
  return GR_OK;
}

}  // namespace
}  // namespace gr

using namespace gr;

extern "C" {

int gr_cnn_param_count(void) { return kCnnParams; }

size_t gr_cnn_workspace_bytes(int n_img, int h, int w) {
  const size_t px = (size_t)n_img * h * w;
  const long segs = (long)n_img * h * ((w + kSeg - 1) / kSeg);
  // h1, h2, gz1, gz2 (bf16 x 16) + gy (f32) + segment partials + loss partials
  return 4 * px * kC * 2 + px * 4 + (size_t)segs * kCnnParams * 4 + 1024 * 8 + 1024;
}

size_t gr_cnn_forward_workspace_bytes(int n_img, int h, int w) {
  return 2 * (size_t)n_img * h * w * kC * 2;  // h1, h2 (BF16 x 16)
}

int gr_cnn_forward(const float* params, const float* x, float* y, int n_img, int h, int w,
                   void* workspace, void* stream) {
  int rc = cnn_check(n_img, h, w);
  if (rc) return rc;
  if (!params || !x || !y || !workspace) return fail(GR_ERR_ARG, "cnn forward: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t px = (size_t)n_img * h * w;
  __nv_bfloat16* h1 = static_cast<__nv_bfloat16*>(workspace);
  __nv_bfloat16* h2 = h1 + px * kC;
  const dim3 gp((w + 127) / 128, h, n_img);
  cnn_conv1_kernel<<<gp, 128, 0, st>>>(params, x, h1, h, w);
  cnn_conv2_kernel<<<dim3((w + 64 * kConv2Tiles - 1) / (64 * kConv2Tiles), h, n_img), 128, 0, st>>>(params, h1, nullptr, h2, h, w, 0);
  cnn_conv3_kernel<<<gp, 128, 0, st>>>(params, x, h2, y, h, w);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GR_OK : fail(GR_ERR_CUDA, "cnn forward: %s", cudaGetErrorString(e));
}

int gr_cnn_backward(const float* params, const float* x, const float* y, const float* target,
                    int n_img, int h, int w, float* grads, double* loss, void* workspace,
                    void* stream) {
  int rc = cnn_check(n_img, h, w);
  if (rc) return rc;
  if (!params || !x || !y || !target || !grads || !workspace)
    return fail(GR_ERR_ARG, "cnn backward: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const size_t px = (size_t)n_img * h * w;
  __nv_bfloat16* h1 = static_cast<__nv_bfloat16*>(workspace);
  __nv_bfloat16* h2 = h1 + px * kC;
  __nv_bfloat16* gz1 = h2 + px * kC;
  __nv_bfloat16* gz2 = gz1 + px * kC;
  float* gy = reinterpret_cast<float*>(gz2 + px * kC);
  const int segs_row = (w + kSeg - 1) / kSeg;
  const long segs = (long)n_img * h * segs_row;
  float* part = gy + px;
  double* lpart = reinterpret_cast<double*>(part + (size_t)segs * kCnnParams);
  lpart = reinterpret_cast<double*>(((uintptr_t)lpart + 7) & ~(uintptr_t)7);
  const int lblocks = 1024;
  cnn_loss_kernel<<<lblocks, 256, 0, st>>>(y, target, gy, lpart, (long)px);
  const dim3 gp((w + 127) / 128, h, n_img);
  cnn_conv3_bwd_kernel<<<gp, 128, 0, st>>>(params, gy, h2, gz2, h, w);
  cnn_conv2_kernel<<<dim3((w + 64 * kConv2Tiles - 1) / (64 * kConv2Tiles), h, n_img), 128, 0, st>>>(params, gz2, h1, gz1, h, w, 1);
  const int smem = (3 * (kSeg + 2) * (1 + 2 * kC) + kSeg * (2 * kC + 1)) * (int)sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(cnn_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       smem);
  if (e != cudaSuccess) return fail(GR_ERR_CUDA, "cnn wgrad smem: %s", cudaGetErrorString(e));
  cnn_wgrad_kernel<<<dim3(h * segs_row, n_img), 256, smem, st>>>(x, gy, h1, h2, gz1, gz2, part, h,
                                                                 w, segs_row);
  cnn_reduce_kernel<<<(kCnnParams + 255) / 256, 256, 0, st>>>(part, segs, grads);
  if (loss) {
    double lp[lblocks];
    e = cudaMemcpyAsync(lp, lpart, sizeof(lp), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(GR_ERR_CUDA, "cnn loss: %s", cudaGetErrorString(e));
    double s = 0.0;
    for (int i = 0; i < lblocks; ++i) s += lp[i];
    *loss = s / (double)px;
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? GR_OK : fail(GR_ERR_CUDA, "cnn backward: %s", cudaGetErrorString(e));
}

size_t gr_cnn_infer_workspace_bytes(void) { return 256; }

int gr_cnn_infer(const float* params, const float* x, float* y, const float* scale, int n_img,
                 int h, int w, void* workspace, void* stream) {
  int rc = cnn_check(n_img, h, w);
  if (rc) return rc;
  if (!params || !x || !y || !workspace) return fail(GR_ERR_ARG, "cnn infer: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(cnn_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kFSmemLaunch);
  if (e != cudaSuccess) return fail(GR_ERR_CUDA, "cnn infer: %s", cudaGetErrorString(e));
  const long tiles = (long)n_img * ((h + kFTh - 1) / kFTh) * ((w + kFTw - 1) / kFTw);
  const int blocks = (int)std::min<long>(tiles, (long)kFCtas * sms);
  cnn_fused_kernel<<<blocks, kFThreads, kFSmemLaunch, st>>>(params, x, y, scale, n_img, h, w,
                                                            static_cast<int*>(workspace));
  e = cudaGetLastError();
  return e == cudaSuccess ? GR_OK : fail(GR_ERR_CUDA, "cnn infer: %s", cudaGetErrorString(e));
}

int gr_cnn_infer_status(void* workspace, void* stream) {
  if (!workspace) return fail(GR_ERR_ARG, "cnn infer status: null workspace");
  cudaStream_t st = (cudaStream_t)stream;
  int flag = 0;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(&flag, workspace, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && flag) e = cudaMemset(workspace, 0, sizeof(int));
  if (e != cudaSuccess) return fail(GR_ERR_CUDA, "cnn infer status: %s", cudaGetErrorString(e));
  return flag ? fail(GR_ERR_TIMEOUT, "cnn infer: a bounded device wait ran out") : GR_OK;
}

int gr_cnn_adam(float* params, const float* grads, float* m, float* v, int step, float lr,
                float beta1, float beta2, float eps, void* stream) {
  if (!params || !grads || !m || !v || step < 1) return fail(GR_ERR_ARG, "cnn adam: bad arguments");
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  cnn_adam_kernel<<<(kCnnParams + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      params, grads, m, v, kCnnParams, lr, beta1, beta2, eps, c1, c2);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GR_OK : fail(GR_ERR_CUDA, "cnn adam: %s", cudaGetErrorString(e));
}

}  // extern "C"
