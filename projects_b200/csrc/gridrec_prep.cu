// Slice-pipeline steps around gridrec, on the device (decarlof/projects):
//   ring suppression        RingCorrectionSinogram  gridrec/GPU/tomo_recon.cpp:3905-3968
//   sub-pixel shift + pad   GridRecSlices           gridrec/GPU/tomo_recon.cpp:3708-3810
//                           (same code in find_shift/src/main/find_shift.cpp:1729-1808)
//   centre crop             GridRecSlices           gridrec/GPU/tomo_recon.cpp:3855-3862
//   circular crop           output stage            gridrec/GPU/tomo_recon.cpp:2150-2165
//   histogram entropy       entropy()               find_shift/src/main/find_shift.cpp:2078-2115
//   centre search           entropy refinement      find_shift/src/main/find_shift.cpp:1653-1900
// Sinograms are n_ang rows of n_det floats, slices contiguous.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "gr_internal.h"

namespace gr {
namespace {

constexpr int kPrepThreads = 256;
constexpr int kMaxBins = 50000;

__device__ __forceinline__ float block_sum(float v, float* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float s = 0.f;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  return s;  // valid in thread 0
}

__device__ __forceinline__ double block_sum_d(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x < 32) {
    s = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  return s;
}

// ---------------------------------------------------------------------------
// Ring suppression.  Each of `iterations` rounds, per slice:
//   r_i = mean_j x_ij,  g = mean_i r_i,  v_ij = x_ij g / r_i   (rows with r_i = 0 kept)
//   c_j = mean_i v_ij,  t_j = c_j - (c_{j-1} + c_j + c_{j+1}) / 3   (t_0 = t_{n-1} = 0)
//   x_ij <- v_ij - coeff t_j  where positive, else 0
// Two launches per round: the row update fused with the next round's row means
// and column partial sums over chunks of rows, then the column means.  The
// first round's partials come from a column pass over the input.  The
// renormalised value is formed as (x g) / r in float, the reference's expression.

// Rows per chunk of the column passes (32: measured fastest of 4..32 at
// 16 x 2048 x 1500; more row chunks add partial-sum traffic, fewer leave SMs idle).
constexpr int kRingRows = 32;

int ring_chunks(int n_ang) { return (n_ang + kRingRows - 1) / kRingRows; }

__global__ void ring_rowmean_kernel(const float* data, float* rowmean, int n_det, int n_ang) {
  __shared__ float red[32];
  const int i = blockIdx.x, s = blockIdx.y;
  const float* row = data + ((size_t)s * n_ang + i) * n_det;
  float acc = 0.f;
  for (int j = threadIdx.x; j < n_det; j += blockDim.x) acc += row[j];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) rowmean[(size_t)s * n_ang + i] = acc / n_det;
}

__device__ __forceinline__ float slice_gmean(const float* rm, int n_ang, float* red) {
  __shared__ float g_s;
  float acc = 0.f;
  for (int i = threadIdx.x; i < n_ang; i += blockDim.x) acc += rm[i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) g_s = acc / n_ang;
  __syncthreads();
  return g_s;
}

__global__ void ring_colpart_kernel(const float* data, const float* rowmean, float* part,
                                    float* gmean, int n_det, int n_ang, int rows_per_chunk) {
  __shared__ float red[32];
  const int r = blockIdx.y, s = blockIdx.z, R = gridDim.y;
  const float* rm = rowmean + (size_t)s * n_ang;
  const float g = slice_gmean(rm, n_ang, red);
  if (threadIdx.x == 0 && blockIdx.x == 0 && r == 0) gmean[s] = g;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n_det) return;
  const int i0 = r * rows_per_chunk, i1 = min(n_ang, i0 + rows_per_chunk);
  const float* x = data + (size_t)s * n_ang * n_det + j;
  float acc = 0.f;
  for (int i = i0; i < i1; ++i) {
    const float ri = rm[i];
    const float v = x[(size_t)i * n_det];
    acc += ri != 0.f ? __fdiv_rn(__fmul_rn(v, g), ri) : v;
  }
  part[((size_t)s * R + r) * n_det + j] = acc;
}

// Column means c_j = g / n_ang * sum_q part[q][j] (32 columns x 8 chunk
// strides per block).  scaled = 1: partials already include g (first round,
// sums of v); scaled = 0: partials are sums of x / r_i and g, the mean of the
// row means, is formed here and recorded for the next update.
__global__ void __launch_bounds__(256) ring_colmean_kernel(const float* part, const float* rowmean,
                                                          float* colmean, float* gmean, int n_det,
                                                          int n_ang, int R, int scaled) {
  __shared__ float red[32];
  __shared__ float acc_s[8][33];
  const int s = blockIdx.y;
  float g = 1.f;
  if (!scaled) {
    g = slice_gmean(rowmean + (size_t)s * n_ang, n_ang, red);
    if (threadIdx.x == 0 && threadIdx.y == 0 && blockIdx.x == 0) gmean[s] = g;
  }
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int j = blockIdx.x * 32 + tx;
  float acc = 0.f;
  if (j < n_det) {
    const float* p = part + (size_t)s * R * n_det + j;
    for (int q = ty; q < R; q += 8) acc += p[(size_t)q * n_det];
  }
  acc_s[ty][tx] = acc;
  __syncthreads();
  if (ty == 0 && j < n_det) {
    float c = 0.f;
    for (int q = 0; q < 8; ++q) c += acc_s[q][tx];
    colmean[(size_t)s * n_det + j] = c * g / n_ang;
  }
}

// One round on rows [r * rows_per_chunk, ...) of slice s, all columns, fused
// with the next round's column partials:
//   t_j = c_j - (c_{j-1} + c_j + c_{j+1}) / 3 (0 at both edges),
//   x <- max((x g) / r_i - coeff t_j, 0),  r_i <- mean of the new row,
//   part[j] = sum over the chunk of x_new / r_i.
// After a round every value is >= 0, so a row with r_i = 0 is all zeros and
// adds nothing whether scaled or not.  KPT columns per thread, RB rows per
// barrier (warp partials double-buffered).
template <int KPT, int RB>
__global__ void __launch_bounds__(kPrepThreads) ring_round_kernel(
    float* data, float* rowmean, const float* colmean, const float* gmean, float* part, int n_det,
    int n_ang, int rows_per_chunk, float coeff) {
  constexpr int NW = kPrepThreads / 32;
  __shared__ float red[2][RB][NW];
  const int r = blockIdx.x, s = blockIdx.y, R = gridDim.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const float g = gmean[s];
  const float* c = colmean + (size_t)s * n_det;
  float d[KPT], acc[KPT];
#pragma unroll
  for (int k = 0; k < KPT; ++k) {
    const int j = threadIdx.x + k * kPrepThreads;
    float t = 0.f;
    if (j > 0 && j < n_det - 1) t = c[j] - (c[j - 1] + c[j] + c[j + 1]) / 3.f;
    d[k] = __fmul_rn(t, coeff);
    acc[k] = 0.f;
  }
  float* rm = rowmean + (size_t)s * n_ang;
  const int i0 = r * rows_per_chunk, i1 = min(n_ang, i0 + rows_per_chunk);
  int buf = 0;
  for (int ib = i0; ib < i1; ib += RB, buf ^= 1) {
    float y[RB][KPT];
    float ri[RB], sum[RB];
    // all loads of the RB rows first, so they are in flight together
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int i = ib + b;
      ri[b] = i < i1 ? rm[i] : 0.f;
      const float* row = data + ((size_t)s * n_ang + i) * n_det;
#pragma unroll
      for (int k = 0; k < KPT; ++k) {
        const int j = threadIdx.x + k * kPrepThreads;
        y[b][k] = (i < i1 && j < n_det) ? row[j] : 0.f;
      }
    }
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      const int i = ib + b;
      sum[b] = 0.f;
      float* row = data + ((size_t)s * n_ang + i) * n_det;
#pragma unroll
      for (int k = 0; k < KPT; ++k) {
        const int j = threadIdx.x + k * kPrepThreads;
        if (i < i1 && j < n_det) {
          const float x = y[b][k];
          // A zero sample skips the division: for finite g its quotient is +-0,
          // and +-0 - d rounds to the same float for either sign, so the result
          // is the same.  Zeros are common after a round's clamp, and warps
          // holding some of them ran up to 25 % slower through the division
          // (measured on phantom sinograms).
          const float v = (ri[b] != 0.f && x != 0.f) ? __fdiv_rn(__fmul_rn(x, g), ri[b]) : x;
          y[b][k] = __fsub_rn(v, d[k]) > 0.f ? __fsub_rn(v, d[k]) : 0.f;
          row[j] = y[b][k];
        }
        sum[b] += y[b][k];
      }
    }
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      float v = sum[b];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) red[buf][b][w] = v;
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < RB; ++b) {
      float tot = 0.f;
#pragma unroll
      for (int q = 0; q < NW; ++q) tot += red[buf][b][q];
      const float rn = tot / n_det;
      const int i = ib + b;
      if (i < i1) {
        if (threadIdx.x == 0) rm[i] = rn;
        if (rn != 0.f) {
          const float inv = 1.f / rn;
#pragma unroll
          for (int k = 0; k < KPT; ++k) acc[k] += y[b][k] * inv;
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < KPT; ++k) {
    const int j = threadIdx.x + k * kPrepThreads;
    if (j < n_det) part[((size_t)s * R + r) * n_det + j] = acc[k];
  }
}

__global__ void ring_update_kernel(float* data, float* rowmean, const float* colmean,
                                   const float* gmean, int n_det, int n_ang, float coeff) {
  __shared__ float red[32];
  const int i = blockIdx.x, s = blockIdx.y;
  float* row = data + ((size_t)s * n_ang + i) * n_det;
  const float* c = colmean + (size_t)s * n_det;
  const float ri = rowmean[(size_t)s * n_ang + i];
  const float g = gmean[s];
  float acc = 0.f;
  for (int j = threadIdx.x; j < n_det; j += blockDim.x) {
    const float t = (j > 0 && j < n_det - 1) ? c[j] - (c[j - 1] + c[j] + c[j + 1]) / 3.f : 0.f;
    const float x = row[j];
    const float v = (ri != 0.f && x != 0.f) ? __fdiv_rn(__fmul_rn(x, g), ri) : x;  // as above
    const float d = __fmul_rn(t, coeff);
    const float y = __fsub_rn(v, d) > 0.f ? __fsub_rn(v, d) : 0.f;
    row[j] = y;
    acc += y;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) rowmean[(size_t)s * n_ang + i] = acc / n_det;
}

// ---------------------------------------------------------------------------
// Sub-pixel shift and half padding.  Output slice s reads input slice
// (s % in_mod) and shift xoff[s / off_div] (x_const when xoff is null).  Column k of the input row maps to
// kp = k + pad (pad = n_det / 2) and takes
//   kk = k - x0,  n = floor(kk),  in[clamp(n)] (n + 1 - kk) + in[clamp(n + 1)] (kk - n)
// with indices clamped to [0, n_det); columns left of pad repeat column pad,
// the pad columns right of pad + n_det repeat column pad + n_det - 1, and any
// remaining column (odd n_det) is zero.  Float operations in the reference's
// order without contraction, so the result equals its float arithmetic.
// kStaged: the input row is first copied to shared memory in one coalesced pass
// (16-byte loads where the row is 16-byte aligned), so the two taps of every
// output read shared memory; rows longer than kShiftStageMax read their taps
// from global memory.  Outputs are written strided by the block size (each warp
// store one contiguous 128-byte run).
constexpr int kShiftStageMax = 12288;  // 48 KB of dynamic shared memory

template <bool kStaged>
__global__ void __launch_bounds__(kPrepThreads) shift_pad_kernel(
    const float* in, long in_slice, int in_mod, const float* xoff, int off_div, float x_const,
    float* out, int n_det, int n_ang, int out_width) {
  extern __shared__ float srow[];
  const int i = blockIdx.x, s = blockIdx.y;
  const float* r = in + (size_t)(s % in_mod) * in_slice + (size_t)i * n_det;
  float* o = out + ((size_t)s * n_ang + i) * out_width;
  const float x0 = xoff ? xoff[s / off_div] : x_const;
  const int pad = n_det / 2;
  if (kStaged) {
    int q0 = 0;
    if ((reinterpret_cast<uintptr_t>(r) & 15) == 0) {
      const int n4 = n_det >> 2;
      for (int q = threadIdx.x; q < n4; q += blockDim.x)
        reinterpret_cast<float4*>(srow)[q] = __ldg(reinterpret_cast<const float4*>(r) + q);
      q0 = 4 * n4;
    }
    for (int q = q0 + threadIdx.x; q < n_det; q += blockDim.x) srow[q] = __ldg(&r[q]);
    __syncthreads();
  }
  // Integer-valued floats below 2^24 are exact, so (float)k is kept as a float
  // counter clamped in float, and (float)nk, (float)(nk + 1) are floor(kk) and
  // floor(kk) + 1 (the sum rounds like the int-to-float conversion of nk + 1):
  // the same bits as the reference's expressions with two conversions per output
  // instead of five (the conversion pipe bounded this kernel).
  const int lim = 2 * pad + n_det;
  const float fmax_k = (float)(n_det - 1), fstep = (float)blockDim.x;
  float fkm = (float)((int)threadIdx.x - pad);  // (float)(kp - pad)
#pragma unroll 4
  for (int kp = threadIdx.x; kp < out_width; kp += blockDim.x, fkm += fstep) {
    if (kp >= lim) {
      o[kp] = 0.f;
      continue;
    }
    const float fk = fminf(fmaxf(fkm, 0.f), fmax_k);  // (float)min(max(kp - pad, 0), n_det - 1)
    const float kk = __fsub_rn(fk, x0);
    const float fl = floorf(kk);
    const int nk = (int)fl;
    const int a = min(max(nk, 0), n_det - 1);
    const int b = min(max(nk + 1, 0), n_det - 1);
    const float wa = __fsub_rn(__fadd_rn(fl, 1.f), kk);
    const float wb = __fsub_rn(kk, fl);
    const float va = kStaged ? srow[a] : __ldg(&r[a]);
    const float vb = kStaged ? srow[b] : __ldg(&r[b]);
    o[kp] = __fadd_rn(__fmul_rn(va, wa), __fmul_rn(vb, wb));
  }
}

// One block per (row, output slice); the staged form when the row fits.  128
// threads: blocks alternate between staging a row and writing it, and more
// blocks per SM overlap those phases better (16 x 2048 x 1500 to 4096-wide rows,
// us per slice: 256 threads 11.2, 128 threads 9.9, 64 threads 10.9).
constexpr int kShiftThreads = 128;

void launch_shift_pad(int n_ang, int n_out, cudaStream_t st, const float* in, long in_slice,
                      int in_mod, const float* xoff, int off_div, float x_const, float* out,
                      int n_det, int out_width) {
  const dim3 grid(n_ang, n_out);
  if (n_det <= kShiftStageMax)
    shift_pad_kernel<true><<<grid, kShiftThreads, (size_t)n_det * sizeof(float), st>>>(
        in, in_slice, in_mod, xoff, off_div, x_const, out, n_det, n_ang, out_width);
  else
    shift_pad_kernel<false><<<grid, kShiftThreads, 0, st>>>(in, in_slice, in_mod, xoff, off_div,
                                                             x_const, out, n_det, n_ang, out_width);
}

// ---------------------------------------------------------------------------
// Window copy rows [offset, offset + n) x cols [offset, offset + n); with
// radius > 0, pixels with (k - n/2)^2 + (j - n/2)^2 >= radius^2 become 0.
__global__ void crop_kernel(const float* rec, long rec_stride, long rec_slice, float* out,
                            long out_stride, long out_slice, int n, int offset, int radius) {
  const int j = blockIdx.x, s = blockIdx.y;
  const float* src = rec + (size_t)s * rec_slice + (size_t)(j + offset) * rec_stride + offset;
  float* dst = out + (size_t)s * out_slice + (size_t)j * out_stride;
  const long long r2 = (long long)radius * radius;
  const int h = n / 2;
  const long long dj = (long long)(j - h) * (j - h);
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    float v = src[k];
    if (radius > 0 && (long long)(k - h) * (k - h) + dj >= r2) v = 0.f;
    dst[k] = v;
  }
}

// ---------------------------------------------------------------------------
// Output thresholds and 8-bit slices of the reference's BMP/TIFF writer
// (gridrec/GPU/tomo_recon.cpp:2282-2361).  lo / hi: min / max over every pixel
// of the given slices (start 1e10 / -1e10; NaN compares false and is skipped),
// then capped by the configured upper / raised to the configured lower value.
// Min and max do not depend on the order of evaluation, so the block partials
// give the reference's values exactly.
constexpr int kMinMaxBlocks = 1024;

__global__ void __launch_bounds__(kPrepThreads) minmax_partial_kernel(
    const float* img, int n_slices, int rows, int cols, long row_stride, long slice_stride,
    float2* part) {
  float lo = 1e10f, hi = -1e10f;
  const long per_slice = (long)rows * cols;
  const long total = per_slice * n_slices;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const long s = i / per_slice, r = (i - s * per_slice) / cols;
    const long c = i - s * per_slice - r * cols;
    const float p = img[s * slice_stride + r * row_stride + c];
    if (hi < p) hi = p;
    if (lo > p) lo = p;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = fminf(lo, l2);
    hi = fmaxf(hi, h2);
  }
  __shared__ float2 s_part[kPrepThreads / 32];
  if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = make_float2(lo, hi);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kPrepThreads / 32; ++w) {
      lo = fminf(lo, s_part[w].x);
      hi = fmaxf(hi, s_part[w].y);
    }
    part[blockIdx.x] = make_float2(lo, hi);
  }
}

__global__ void minmax_final_kernel(const float2* part, int n, float lower_clamp, float upper_clamp,
                                    float* lohi) {
  float lo = 1e10f, hi = -1e10f;
  for (int i = 0; i < n; ++i) {
    lo = fminf(lo, part[i].x);
    hi = fmaxf(hi, part[i].y);
  }
  if (hi > upper_clamp) hi = upper_clamp;
  if (lo < lower_clamp) lo = lower_clamp;
  lohi[0] = lo;
  lohi[1] = hi;
}

// 0 below lo, 255 above hi, else (unsigned char)(255 * (p - lo) / (hi - lo)) in
// float left to right (a NaN value, which the reference's cast leaves undefined,
// gives 0); with radius > 0, pixels with (x - cols/2)^2 + (y - rows/2)^2 > radius^2
// are 0 (the writer's cropped copy keeps the boundary, unlike crop_kernel).
__global__ void to_u8_kernel(const float* img, int cols, int rows, long row_stride,
                             long slice_stride, const float* lohi, int radius, unsigned char* out,
                             long out_row_stride, long out_slice_stride) {
  const int y = blockIdx.x, s = blockIdx.y;
  const float lo = lohi[0], hi = lohi[1];
  const float* src = img + (size_t)s * slice_stride + (size_t)y * row_stride;
  unsigned char* dst = out + (size_t)s * out_slice_stride + (size_t)y * out_row_stride;
  const long long r2 = (long long)radius * radius;
  const long long dy = (long long)(y - rows / 2) * (y - rows / 2);
  for (int x = threadIdx.x; x < cols; x += blockDim.x) {
    const float p = src[x];
    unsigned char v;
    if (p < lo) v = 0;
    else if (p > hi) v = 255;
    else {
      const float q = __fdiv_rn(__fmul_rn(255.f, __fsub_rn(p, lo)), __fsub_rn(hi, lo));
      v = (q == q) ? (unsigned char)q : 0;
    }
    if (radius > 0 && (long long)(x - cols / 2) * (x - cols / 2) + dy > r2) v = 0;
    dst[x] = v;
  }
}

// ---------------------------------------------------------------------------
// Histogram entropy of a group of image windows: nbins + 1 bins of width
// inv = (vmax - vmin) / nbins, bin = (int)((x - vmin) / inv) in float
// (truncation toward zero, values outside [0, nbins] ignored), entropy =
// -sum p log2 p with p = count / (pixels in the group).
struct Window {
  const float* base;
  long row_stride, image_stride, group_stride;
  int rows, cols, group;
};

__global__ void hist_kernel(Window w, float vmin, float inv, int nbins, unsigned* ghist) {
  extern __shared__ unsigned hist[];
  for (int b = threadIdx.x; b <= nbins; b += blockDim.x) hist[b] = 0u;
  __syncthreads();
  const int g = blockIdx.y;
  const int total_rows = w.rows * w.group;
  for (int q = blockIdx.x; q < total_rows; q += gridDim.x) {
    const int im = q / w.rows, r = q - im * w.rows;
    const float* row = w.base + (size_t)g * w.group_stride + (size_t)im * w.image_stride +
                       (size_t)r * w.row_stride;
    for (int k = threadIdx.x; k < w.cols; k += blockDim.x) {
      const float f = __fdiv_rn(__fsub_rn(row[k], vmin), inv);
      const int ind = (int)f;  // NaN is skipped (a host cast gives INT_MIN for it)
      if (f == f && ind >= 0 && ind <= nbins) atomicAdd(&hist[ind], 1u);
    }
  }
  __syncthreads();
  unsigned* gh = ghist + (size_t)g * (nbins + 1);
  for (int b = threadIdx.x; b <= nbins; b += blockDim.x)
    if (hist[b]) atomicAdd(&gh[b], hist[b]);
}

__global__ void entropy_final_kernel(const unsigned* ghist, int nbins, double n, float* out) {
  __shared__ double red[32];
  const unsigned* gh = ghist + (size_t)blockIdx.x * (nbins + 1);
  double acc = 0.0;
  for (int b = threadIdx.x; b <= nbins; b += blockDim.x)
    if (gh[b]) {
      const double p = (double)gh[b] / n;
      acc += -p * log(p) / log(2.0);
    }
  acc = block_sum_d(acc, red);
  if (threadIdx.x == 0) out[blockIdx.x] = (float)acc;
}

int launch_entropy(const Window& w, int n_groups, float vmin, float vmax, int nbins,
                   unsigned* ghist, float* out, cudaStream_t st) {
  const float inv = (vmax - vmin) / (float)nbins;
  const int smem = (nbins + 1) * (int)sizeof(unsigned);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem);
    if (e != cudaSuccess) return fail(GR_ERR_CUDA, "hist smem: %s", cudaGetErrorString(e));
  }
  cudaError_t e =
      cudaMemsetAsync(ghist, 0, (size_t)n_groups * (nbins + 1) * sizeof(unsigned), st);
  if (e != cudaSuccess) return fail(GR_ERR_CUDA, "hist memset: %s", cudaGetErrorString(e));
  const int total_rows = w.rows * w.group;
  const int bx = std::max(1, std::min(total_rows, (4 * 148 + n_groups - 1) / n_groups));
  hist_kernel<<<dim3(bx, n_groups), 512, smem, st>>>(w, vmin, inv, nbins, ghist);
  entropy_final_kernel<<<n_groups, 256, 0, st>>>(ghist, nbins,
                                                 (double)w.rows * w.cols * w.group, out);
  e = cudaGetLastError();
  return e == cudaSuccess ? GR_OK : fail(GR_ERR_CUDA, "entropy: %s", cudaGetErrorString(e));
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(GR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GR_OK : fail(GR_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Carves 256-byte aligned pieces out of one scratch allocation.
struct Carve {
  size_t off = 0;
  char* base = nullptr;
  template <class T> T* take(size_t count) {
    off = (off + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};

// ---------------------------------------------------------------------------
// Rotation-axis search by cross-correlation (find_shift's brute-force path:
// data_interp + cross_correlation, find_shift/src/main/find_shift.cpp:1975-2076,
// the CPU twin of cross_correlation.cu:19-413).  For translation (tx, ty) the
// match image is sampled at (nx - tx, ny - ty) for every ROI pixel by bilinear
// interpolation over the in-image neighbours, normalised by their weight
// (0 when the weight is <= 1e-5); M_avg is the ROI mean of the samples, and
//   score = sum (T - T_avg)(M - M_avg) / (T_rms sqrt(sum (M - M_avg)^2))
// (0 when T_rms or the second sum is <= 1e-5), T_rms = sqrt(sum (T - T_avg)^2).
// All arithmetic in double, as the reference's; two passes per translation
// (mean, then centred sums), block partials summed in a fixed order.
struct XcorrArgs {
  const float* templ;   // roi_h x roi_w
  const float* match;   // height x width
  int width, height, x0, y0, roi_w, roi_h;
  double tx0, ty0, dtx, dty;
  int n_tx;
  int rows_per_block;
  double* part;         // [trans][block][2]
  const double* mavg;   // [trans] (second pass)
  const double* tavg;   // template mean
};

__device__ __forceinline__ double xcorr_sample(const XcorrArgs& a, double x, double y) {
  const double fx = floor(x), fy = floor(y);
  const int nxx = (int)fx, nyy = (int)fy;
  double pix = 0.0, wsum = 0.0;
  const double ax = (double)(nxx + 1) - x, bx = x - (double)nxx;
  const double ay = (double)(nyy + 1) - y, by = y - (double)nyy;
  const bool x0ok = nxx >= 0 && nxx < a.width, x1ok = nxx + 1 >= 0 && nxx + 1 < a.width;
  const bool y0ok = nyy >= 0 && nyy < a.height, y1ok = nyy + 1 >= 0 && nyy + 1 < a.height;
  const float* m = a.match;
  if (x0ok && y0ok) {
    pix += (double)__ldg(&m[(size_t)nyy * a.width + nxx]) * ax * ay;
    wsum += ax * ay;
  }
  if (x1ok && y0ok) {
    pix += (double)__ldg(&m[(size_t)nyy * a.width + nxx + 1]) * bx * ay;
    wsum += bx * ay;
  }
  if (x0ok && y1ok) {
    pix += (double)__ldg(&m[(size_t)(nyy + 1) * a.width + nxx]) * ax * by;
    wsum += ax * by;
  }
  if (x1ok && y1ok) {
    pix += (double)__ldg(&m[(size_t)(nyy + 1) * a.width + nxx + 1]) * bx * by;
    wsum += bx * by;
  }
  return wsum > 1e-5 ? pix / wsum : 0.0;
}

// pass 0: sum of samples; pass 1: sum (T - T_avg)(M - M_avg) and sum (M - M_avg)^2
template <int PASS>
__global__ void __launch_bounds__(256) xcorr_kernel(XcorrArgs a) {
  __shared__ double red[2][8];
  const int blk = blockIdx.x, tr = blockIdx.y;
  const double tx = a.tx0 + (tr % a.n_tx) * a.dtx;
  const double ty = a.ty0 + (tr / a.n_tx) * a.dty;
  const double mavg = PASS == 1 ? a.mavg[tr] : 0.0;
  const double tavg = PASS == 1 ? *a.tavg : 0.0;
  double s0 = 0.0, s1 = 0.0;
  const int r0 = blk * a.rows_per_block, r1 = min(a.roi_h, r0 + a.rows_per_block);
  for (int r = r0; r < r1; ++r) {
    const double y = (double)(a.y0 + r) - ty;
    for (int c = threadIdx.x; c < a.roi_w; c += blockDim.x) {
      const double m = xcorr_sample(a, (double)(a.x0 + c) - tx, y);
      if (PASS == 0) {
        s0 += m;
      } else {
        const double dm = m - mavg;
        s0 += ((double)__ldg(&a.templ[(size_t)r * a.roi_w + c]) - tavg) * dm;
        s1 += dm * dm;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = s0;
    red[1][w] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      t0 += red[0][k];
      t1 += red[1][k];
    }
    double* p = a.part + ((size_t)tr * gridDim.x + blk) * 2;
    p[0] = t0;
    p[1] = t1;
  }
}

// One thread per translation sums its block partials in order.  mode 0: mean
// of the samples; mode 1: the score.
__global__ void xcorr_finish_kernel(const double* part, int nblk, int n_trans, double area,
                                    double* mavg, const double* trms, double* score, int mode) {
  const int tr = blockIdx.x * blockDim.x + threadIdx.x;
  if (tr >= n_trans) return;
  double t0 = 0.0, t1 = 0.0;
  for (int b = 0; b < nblk; ++b) {
    t0 += part[((size_t)tr * nblk + b) * 2];
    t1 += part[((size_t)tr * nblk + b) * 2 + 1];
  }
  if (mode == 0) {
    mavg[tr] = t0 / area;
  } else {
    const double r = *trms;
    score[tr] = (fabs(r) > 1e-5 && fabs(t1) > 1e-5) ? t0 / (r * sqrt(t1)) : 0.0;
  }
}

// Template mean and T_rms = sqrt(sum (T - T_avg)^2), one block, fixed order.
__global__ void __launch_bounds__(256) xcorr_template_kernel(const float* t, long n, double* out) {
  __shared__ double red[8];
  __shared__ double mean_s;
  double s = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) s += (double)t[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < 8; ++k) m += red[k];
    mean_s = m / (double)n;
    out[0] = mean_s;
  }
  __syncthreads();
  const double mean = mean_s;
  double q = 0.0;
  for (long i = threadIdx.x; i < n; i += blockDim.x) {
    const double d = (double)t[i] - mean;
    q += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) q += __shfl_xor_sync(0xffffffffu, q, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = q;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < 8; ++k) m += red[k];
    out[1] = sqrt(m);
  }
}

}  // namespace
}  // namespace gr

namespace gr {
namespace {
template <int KPT, int RB>
void launch_ring_round(dim3 grid, cudaStream_t st, float* x, float* rm, const float* c,
                       const float* g, float* part, int n_det, int n_ang, float coeff) {
  ring_round_kernel<KPT, RB><<<grid, kPrepThreads, 0, st>>>(x, rm, c, g, part, n_det, n_ang,
                                                            kRingRows, coeff);
}
}  // namespace
}  // namespace gr

using namespace gr;

extern "C" {

size_t gr_ring_workspace_bytes(int n_slices, int n_det, int n_ang) {
  if (n_slices < 1 || n_det < 1 || n_ang < 1) return 0;
  const int R = ring_chunks(n_ang);
  const size_t floats = (size_t)n_slices * ((size_t)n_ang + (size_t)R * n_det + n_det + 1);
  return floats * sizeof(float);
}


int gr_ring_removal(float* sinos, int n_slices, int n_det, int n_ang, float ring_coeff,
                    int iterations, void* workspace, void* stream) {
  if (!sinos || !workspace) return fail(GR_ERR_ARG, "ring removal: null pointer");
  if (n_slices < 1 || n_det < 3 || n_ang < 1 || iterations < 0)
    return fail(GR_ERR_ARG, "ring removal: need n_slices >= 1, n_det >= 3, n_ang >= 1, "
                            "iterations >= 0");
  if (iterations == 0) return GR_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const int R = ring_chunks(n_ang);
  float* rowmean = static_cast<float*>(workspace);
  float* part = rowmean + (size_t)n_slices * n_ang;
  float* colmean = part + (size_t)n_slices * R * n_det;
  float* gmean = colmean + (size_t)n_slices * n_det;
  const int bx = (n_det + kPrepThreads - 1) / kPrepThreads;
  const int cx = (n_det + 31) / 32;
  const int kpt = bx <= 1 ? 1 : bx <= 2 ? 2 : bx <= 4 ? 4 : bx <= 8 ? 8 : 16;
  const bool fused = bx <= 16;
  {
    const int ns = n_slices;
    float* x = sinos;
    float* rm = rowmean;
    float* pt = part;
    float* cm = colmean;
    float* gm = gmean;
    ring_rowmean_kernel<<<dim3(n_ang, ns), kPrepThreads, 0, st>>>(x, rm, n_det, n_ang);
    ring_colpart_kernel<<<dim3(bx, R, ns), kPrepThreads, 0, st>>>(x, rm, pt, gm, n_det, n_ang,
                                                                  kRingRows);
    ring_colmean_kernel<<<dim3(cx, ns), 256, 0, st>>>(pt, rm, cm, gm, n_det, n_ang, R, 1);
    for (int m = 0; m < iterations; ++m) {
      if (fused) {
        const dim3 grid(R, ns);
        switch (kpt) {
          case 1: launch_ring_round<1, 4>(grid, st, x, rm, cm, gm, pt, n_det, n_ang, ring_coeff); break;
          case 2: launch_ring_round<2, 4>(grid, st, x, rm, cm, gm, pt, n_det, n_ang, ring_coeff); break;
          case 4: launch_ring_round<4, 4>(grid, st, x, rm, cm, gm, pt, n_det, n_ang, ring_coeff); break;
          case 8: launch_ring_round<8, 4>(grid, st, x, rm, cm, gm, pt, n_det, n_ang, ring_coeff); break;
          default: launch_ring_round<16, 2>(grid, st, x, rm, cm, gm, pt, n_det, n_ang, ring_coeff);
        }
        if (m + 1 < iterations)
          ring_colmean_kernel<<<dim3(cx, ns), 256, 0, st>>>(pt, rm, cm, gm, n_det, n_ang, R, 0);
      } else {
        // Rows wider than 4096: separate update and column passes.
        if (m > 0) {
          ring_colpart_kernel<<<dim3(bx, R, ns), kPrepThreads, 0, st>>>(x, rm, pt, gm, n_det,
                                                                        n_ang, kRingRows);
          ring_colmean_kernel<<<dim3(cx, ns), 256, 0, st>>>(pt, rm, cm, gm, n_det, n_ang, R, 1);
        }
        ring_update_kernel<<<dim3(n_ang, ns), kPrepThreads, 0, st>>>(x, rm, cm, gm, n_det, n_ang,
                                                                     ring_coeff);
      }
    }
  }
  return check_launch("ring removal");
}

int gr_shift_pad(const float* in, float* out, int n_slices, int n_det, int n_ang,
                 const float* xoffsets, int out_width, void* stream) {
  if (!in || !out || !xoffsets) return fail(GR_ERR_ARG, "shift/pad: null pointer");
  if (n_slices < 1 || n_det < 1 || n_ang < 1 || out_width < n_det)
    return fail(GR_ERR_ARG, "shift/pad: need n_slices, n_det, n_ang >= 1 and out_width >= n_det");
  launch_shift_pad(n_ang, n_slices, (cudaStream_t)stream, in, (long)n_ang * n_det, n_slices,
                   xoffsets, 1, 0.f, out, n_det, out_width);
  return check_launch("shift/pad");
}

int gr_crop_center(const float* recon, long recon_stride, long recon_slice_elems, float* out,
                   long out_stride, long out_slice_elems, int n_slices, int n, int offset,
                   int radius, void* stream) {
  if (!recon || !out) return fail(GR_ERR_ARG, "crop: null pointer");
  if (n_slices < 1 || n < 1 || offset < 0 || out_stride < n || recon_stride < n + offset ||
      radius < 0)
    return fail(GR_ERR_ARG, "crop: bad sizes (n=%d offset=%d recon_stride=%ld out_stride=%ld)", n,
                offset, recon_stride, out_stride);
  crop_kernel<<<dim3(n, n_slices), kPrepThreads, 0, (cudaStream_t)stream>>>(
      recon, recon_stride, recon_slice_elems, out, out_stride, out_slice_elems, n, offset, radius);
  return check_launch("crop");
}

size_t gr_threshold_workspace_bytes(void) { return kMinMaxBlocks * sizeof(float2); }

int gr_threshold_range(const float* images, int n_slices, int rows, int cols, long row_stride,
                       long slice_stride, float lower_clamp, float upper_clamp, float* lohi,
                       void* workspace, void* stream) {
  if (!images || !lohi || !workspace) return fail(GR_ERR_ARG, "threshold: null pointer");
  if (n_slices < 1 || rows < 1 || cols < 1 || row_stride < cols ||
      (n_slices > 1 && slice_stride < (long)rows * row_stride))
    return fail(GR_ERR_ARG, "threshold: bad sizes (rows=%d cols=%d row_stride=%ld)", rows, cols,
                row_stride);
  const long total = (long)n_slices * rows * cols;
  const int blocks = (int)std::min<long>(kMinMaxBlocks, (total + kPrepThreads - 1) / kPrepThreads);
  cudaStream_t st = (cudaStream_t)stream;
  float2* part = static_cast<float2*>(workspace);
  minmax_partial_kernel<<<blocks, kPrepThreads, 0, st>>>(images, n_slices, rows, cols, row_stride,
                                                         slice_stride, part);
  int rc = check_launch("threshold: min/max");
  if (rc) return rc;
  minmax_final_kernel<<<1, 1, 0, st>>>(part, blocks, lower_clamp, upper_clamp, lohi);
  return check_launch("threshold: final");
}

int gr_to_u8(const float* images, int n_slices, int rows, int cols, long row_stride,
             long slice_stride, const float* lohi, int radius, unsigned char* out,
             long out_row_stride, long out_slice_stride, void* stream) {
  if (!images || !lohi || !out) return fail(GR_ERR_ARG, "to_u8: null pointer");
  if (n_slices < 1 || n_slices > 65535 || rows < 1 || cols < 1 || row_stride < cols ||
      out_row_stride < cols || radius < 0)
    return fail(GR_ERR_ARG, "to_u8: bad sizes (rows=%d cols=%d)", rows, cols);
  to_u8_kernel<<<dim3(rows, n_slices), kPrepThreads, 0, (cudaStream_t)stream>>>(
      images, cols, rows, row_stride, slice_stride, lohi, radius, out, out_row_stride,
      out_slice_stride);
  return check_launch("to_u8");
}

size_t gr_entropy_workspace_bytes(int n_groups, int nbins) {
  if (n_groups < 1 || nbins < 1) return 0;
  return (size_t)n_groups * (nbins + 1) * sizeof(unsigned);
}

int gr_entropy(const float* images, int n_groups, int group, int rows, int cols, long row_stride,
               long image_stride, long group_stride, float vmin, float vmax, int nbins,
               float* entropies, void* workspace, void* stream) {
  if (!images || !entropies || !workspace) return fail(GR_ERR_ARG, "entropy: null pointer");
  if (n_groups < 1 || n_groups > 65535 || group < 1 || rows < 1 || cols < 1 ||
      row_stride < cols || nbins < 1 || nbins > kMaxBins || !(vmax > vmin))
    return fail(GR_ERR_ARG, "entropy: bad sizes or range (nbins in [1, %d], vmax > vmin)",
                kMaxBins);
  Window w{images, row_stride, image_stride, group_stride, rows, cols, group};
  return launch_entropy(w, n_groups, vmin, vmax, nbins, static_cast<unsigned*>(workspace),
                        entropies, (cudaStream_t)stream);
}

int gr_reconstruct_padded(gr_plan* plan, const float* sinos, int n_slices, int n_det, int n_ang,
                          float xoffset, float* outs, long out_stride, void* stream) {
  int pn, pa, M0, max_pairs, dev;
  int rc = plan_shape(plan, &pn, &pa, &M0, &max_pairs, &dev);
  if (rc) return rc;
  if (!sinos || !outs) return fail(GR_ERR_ARG, "padded: null pointer");
  if (n_slices < 1 || pa != n_ang || pn < n_det + 2 * (n_det / 2) || out_stride < n_det)
    return fail(GR_ERR_ARG, "padded: plan must be %d angles and >= %d wide (is %d x %d)", n_ang,
                n_det + 2 * (n_det / 2), pa, pn);
  const int off = n_det / 2;
  if (off + n_det > M0)
    return fail(GR_ERR_ARG, "padded: crop window [%d, %d) exceeds the image size %d", off,
                off + n_det, M0);
  DeviceGuard guard(dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int chunk = std::min(n_slices, 2 * max_pairs);
  Carve c;
  c.take<float>((size_t)chunk * n_ang * pn);
  c.take<float>((size_t)chunk * M0 * M0);
  if ((rc = plan_scratch(plan, c.off + 256, (void**)&c.base))) return rc;
  c.off = 0;
  float* sp = c.take<float>((size_t)chunk * n_ang * pn);
  float* rec = c.take<float>((size_t)chunk * M0 * M0);
  for (int s0 = 0; s0 < n_slices; s0 += chunk) {
    const int ns = std::min(chunk, n_slices - s0);
    launch_shift_pad(n_ang, ns, st, sinos + (size_t)s0 * n_ang * n_det, (long)n_ang * n_det, ns,
                     nullptr, 1, xoffset, sp, n_det, pn);
    if ((rc = check_launch("padded: shift/pad"))) return rc;
    gr_batch_desc b{};
    b.n_slices = ns;
    b.dtype = GR_DTYPE_F32;
    b.sinos = sp;
    b.outs = rec;
    b.out_stride = M0;
    if ((rc = gr_reconstruct_batch(plan, &b, st))) return rc;
    crop_kernel<<<dim3(n_det, ns), kPrepThreads, 0, st>>>(
        rec, M0, (long)M0 * M0, outs + (size_t)s0 * n_det * out_stride, out_stride,
        (long)n_det * out_stride, n_det, off, 0);
    if ((rc = check_launch("padded: crop"))) return rc;
  }
  return GR_OK;
}

int gr_center_search(gr_plan* plan, const float* sino1, const float* sino2, int n_det, int n_ang,
                     const float* shifts, int n_cand, float hist_lo, float hist_hi, int nbins,
                     float* scores, int* best, float* best_images, void* stream) {
  int pn, pa, M0, max_pairs, dev;
  int rc = plan_shape(plan, &pn, &pa, &M0, &max_pairs, &dev);
  if (rc) return rc;
  if (!sino1 || !sino2 || !shifts || !scores) return fail(GR_ERR_ARG, "centre search: null pointer");
  if (n_cand < 1 || pa != n_ang || pn < n_det + 2 * (n_det / 2))
    return fail(GR_ERR_ARG, "centre search: plan must be %d angles and >= %d wide (is %d x %d)",
                n_ang, n_det + 2 * (n_det / 2), pa, pn);
  if (nbins < 1 || nbins > kMaxBins || !(hist_hi > hist_lo))
    return fail(GR_ERR_ARG, "centre search: nbins in [1, %d] and hist_hi > hist_lo", kMaxBins);
  const int off = n_det / 2;
  if (off + n_det > M0)
    return fail(GR_ERR_ARG, "centre search: crop window [%d, %d) exceeds the image size %d", off,
                off + n_det, M0);
  DeviceGuard guard(dev);
  cudaStream_t st = (cudaStream_t)stream;
  const int chunk = std::min(n_cand, max_pairs);  // candidates per batch (one pair each)
  const long slice_in = (long)n_ang * n_det;
  const long slice_rec = (long)M0 * M0;
  Carve c;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      if ((rc = plan_scratch(plan, c.off + 256, (void**)&c.base))) return rc;
      c.off = 0;
    }
    c.take<float>(2 * slice_in);
    c.take<float>((size_t)2 * chunk * n_ang * pn);
    c.take<float>((size_t)2 * chunk * slice_rec);
    c.take<float>(n_cand);
    c.take<unsigned>((size_t)chunk * (nbins + 1));
    c.take<float>(n_cand);
  }
  c.off = 0;
  float* pr = c.take<float>(2 * slice_in);
  float* sp = c.take<float>((size_t)2 * chunk * n_ang * pn);
  float* rec = c.take<float>((size_t)2 * chunk * slice_rec);
  float* xo = c.take<float>(n_cand);
  unsigned* gh = c.take<unsigned>((size_t)chunk * (nbins + 1));
  float* sc = c.take<float>(n_cand);
  cudaError_t e = cudaMemcpyAsync(pr, sino1, slice_in * sizeof(float), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(pr + slice_in, sino2, slice_in * sizeof(float), cudaMemcpyDeviceToDevice,
                        st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(xo, shifts, n_cand * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail(e, "centre search: copies");
  for (int c0 = 0; c0 < n_cand; c0 += chunk) {
    const int nc = std::min(chunk, n_cand - c0);
    launch_shift_pad(n_ang, 2 * nc, st, pr, slice_in, 2, xo + c0, 2, 0.f, sp, n_det, pn);
    if ((rc = check_launch("centre search: shift/pad"))) return rc;
    gr_batch_desc b{};
    b.n_slices = 2 * nc;
    b.dtype = GR_DTYPE_F32;
    b.sinos = sp;
    b.outs = rec;
    b.out_stride = M0;
    if ((rc = gr_reconstruct_batch(plan, &b, st))) return rc;
    Window w{rec + (size_t)off * M0 + off, M0, slice_rec, 2 * slice_rec, n_det, n_det, 2};
    if ((rc = launch_entropy(w, nc, hist_lo, hist_hi, nbins, gh, sc + c0, st))) return rc;
  }
  e = cudaMemcpyAsync(scores, sc, n_cand * sizeof(float), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "centre search: scores");
  // First strict minimum, as the reference's `entropy_cur < entropy_optim` scan.
  int bi = 0;
  for (int k = 1; k < n_cand; ++k)
    if (scores[k] < scores[bi]) bi = k;
  if (best) *best = bi;
  if (best_images) {
    launch_shift_pad(n_ang, 2, st, pr, slice_in, 2, xo + bi, 2, 0.f, sp, n_det, pn);
    if ((rc = check_launch("centre search: shift/pad"))) return rc;
    gr_batch_desc b{};
    b.n_slices = 2;
    b.dtype = GR_DTYPE_F32;
    b.sinos = sp;
    b.outs = rec;
    b.out_stride = M0;
    if ((rc = gr_reconstruct_batch(plan, &b, st))) return rc;
    crop_kernel<<<dim3(n_det, 2), kPrepThreads, 0, st>>>(rec, M0, slice_rec, best_images, n_det,
                                                         (long)n_det * n_det, n_det, off, 0);
    if ((rc = check_launch("centre search: crop"))) return rc;
  }
  return GR_OK;
}

int gr_xcorr_scores(const float* templ_roi, const float* match, int width, int height, int roi_x0,
                    int roi_x1, int roi_y0, int roi_y1, double tx0, double ty0, double dtx,
                    double dty, int n_tx, int n_ty, double* scores, void* stream) {
  if (!templ_roi || !match || !scores) return fail(GR_ERR_ARG, "xcorr: null pointer");
  if (width < 1 || height < 1 || n_tx < 1 || n_ty < 1 || roi_x0 < 0 || roi_y0 < 0 ||
      roi_x1 < roi_x0 || roi_y1 < roi_y0 || roi_x1 >= width || roi_y1 >= height)
    return fail(GR_ERR_ARG, "xcorr: bad image, ROI or translation grid");
  if ((long)n_tx * n_ty > 65535) return fail(GR_ERR_ARG, "xcorr: at most 65535 translations");
  cudaStream_t st = (cudaStream_t)stream;
  const int roi_w = roi_x1 - roi_x0 + 1, roi_h = roi_y1 - roi_y0 + 1;
  const int n_trans = n_tx * n_ty;
  // enough blocks to fill the GPU: split the ROI rows when translations are few
  const int want_blocks = 4 * 148;
  int nblk = std::max(1, std::min(roi_h, (want_blocks + n_trans - 1) / n_trans));
  const int rows_per = (roi_h + nblk - 1) / nblk;
  nblk = (roi_h + rows_per - 1) / rows_per;
  double* d = nullptr;
  const size_t nd = (size_t)n_trans * nblk * 2 + n_trans * 2 + 2;
  cudaError_t e = cudaMallocAsync(&d, nd * sizeof(double), st);
  if (e != cudaSuccess) return fail(GR_ERR_NOMEM, "xcorr: %s", cudaGetErrorString(e));
  double* part = d;
  double* mavg = part + (size_t)n_trans * nblk * 2;
  double* sc = mavg + n_trans;
  double* tstat = sc + n_trans;  // T_avg, T_rms
  XcorrArgs a{templ_roi, match, width, height, roi_x0, roi_y0, roi_w, roi_h,
              tx0, ty0, dtx, dty, n_tx, rows_per, part, mavg, tstat};
  const int fin = (n_trans + 255) / 256;
  xcorr_template_kernel<<<1, 256, 0, st>>>(templ_roi, (long)roi_w * roi_h, tstat);
  xcorr_kernel<0><<<dim3(nblk, n_trans), 256, 0, st>>>(a);
  xcorr_finish_kernel<<<fin, 256, 0, st>>>(part, nblk, n_trans, (double)roi_w * roi_h, mavg,
                                           tstat + 1, sc, 0);
  xcorr_kernel<1><<<dim3(nblk, n_trans), 256, 0, st>>>(a);
  xcorr_finish_kernel<<<fin, 256, 0, st>>>(part, nblk, n_trans, (double)roi_w * roi_h, mavg,
                                           tstat + 1, sc, 1);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(scores, sc, n_trans * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? GR_OK : cuda_fail(e, "xcorr");
}

}  // extern "C"
