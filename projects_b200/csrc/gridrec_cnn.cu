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
