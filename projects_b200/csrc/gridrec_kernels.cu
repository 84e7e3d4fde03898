// sm_100a kernels of the gridrec pipeline.
//
//   phase_kernel    per pair: filter x centre phase ramps P_j, Q_j (FP64 -> FP32)
//   spectra_kernel  per (pair, angle): load (f32/f16/bf16/u16 raw with fused
//                   flat/dark + log), pack slice 1 + i*slice 2, zero-pad to
//                   pdim, shared-memory Stockham FFT exp(+i), filter/phase
//                   multiply -> filtered samples C1_j, C2_j
//                   (gridrec/GPU/gridrec.cu:500-538)
//   grid_kernel     per (tile work item, pair): binned gather of all samples
//                   whose PSWF footprint meets a 32x32 tile of the M x M grid,
//                   accumulated in shared memory, tile written once
//                   (gridrec.cu:540-576; no global atomics)
//   cols_kernel     per (column group, pair): Stockham FFT exp(-i) along the
//                   first grid axis, in place (first half of gridrec.cu:641-646)
//   rows_kernel     per (grid row, pair): Stockham FFT exp(-i) along the second
//                   axis fused with deapodisation winv[j]*winv[k], the
//                   four-corner crop and the split into two real images
//                   (gridrec.cu:641-646 + 691-719)
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <type_traits>
#include <mutex>
#include <vector>

#include "gr_device.cuh"
#include "gr_internal.h"

namespace gr {

// ------------------------------------------------------------------ complex helpers

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * (S * i)
template <int S>
__device__ __forceinline__ float2 mul_si(float2 a) {
  return S > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// a * exp(S * 2 pi i m / 16) for the compile-time constant m used by dft16/dft8
template <int S, int m>
__device__ __forceinline__ float2 tw16(float2 a) {
  constexpr float c1 = 0.92387953251128676f, c2 = 0.70710678118654752f, c3 = 0.38268343236508977f;
  constexpr float cs[10] = {1.f, c1, c2, c3, 0.f, -c3, -c2, -c1, -1.f, -c1};
  constexpr float sn[10] = {0.f, c3, c2, c1, 1.f, c1, c2, c3, 0.f, -c3};
  if constexpr (m == 0) {
    return a;
  } else if constexpr (m == 4) {
    return mul_si<S>(a);
  } else if constexpr (m == 8) {
    return make_float2(-a.x, -a.y);
  } else {
    return cmul(a, make_float2(cs[m], S * sn[m]));
  }
}


// ------------------------------------------------------------------ in-register DFTs
// Natural order in and out: v[k] <- sum_n v[n] exp(S 2 pi i n k / R).

template <int S>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int S>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  float2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = mul_si<S>(csub(a1, a3));
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd(t1, t3);
  a3 = csub(t1, t3);
}

template <int S>
__device__ __forceinline__ void dft4(float2* v) { dft4<S>(v[0], v[1], v[2], v[3]); }

// R = 8 as 2 x 4: n = 2 n2 + n1, k = k1 + 4 k2.
template <int S>
__device__ __forceinline__ void dft8(float2* v) {
  dft4<S>(v[0], v[2], v[4], v[6]);  // n1 = 0 -> Y0[k1] at v[2 k1]
  dft4<S>(v[1], v[3], v[5], v[7]);  // n1 = 1 -> Y1[k1] at v[2 k1 + 1]
  float2 y1[4] = {v[1], tw16<S, 2>(v[3]), tw16<S, 4>(v[5]), tw16<S, 6>(v[7])};
  float2 y0[4] = {v[0], v[2], v[4], v[6]};
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    v[k1] = cadd(y0[k1], y1[k1]);
    v[k1 + 4] = csub(y0[k1], y1[k1]);
  }
}

// R = 16 as 4 x 4: n = 4 n2 + n1, k = k1 + 4 k2.
template <int S>
__device__ __forceinline__ void dft16(float2* v) {
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) dft4<S>(v[n1], v[4 + n1], v[8 + n1], v[12 + n1]);
  // Y[n1][k1] sits at v[4 k1 + n1]; twiddle by W16^(n1 k1)
  v[5] = tw16<S, 1>(v[5]);
  v[6] = tw16<S, 2>(v[6]);
  v[7] = tw16<S, 3>(v[7]);
  v[9] = tw16<S, 2>(v[9]);
  v[10] = tw16<S, 4>(v[10]);
  v[11] = tw16<S, 6>(v[11]);
  v[13] = tw16<S, 3>(v[13]);
  v[14] = tw16<S, 6>(v[14]);
  v[15] = tw16<S, 9>(v[15]);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) dft4<S>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // now v[4 k1 + k2] = X[k1 + 4 k2]: transpose the 4 x 4 register block
  float2 t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1)
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[4 * k1 + k2];
}

template <int R, int S>
__device__ __forceinline__ void dftR(float2* v) {
  if constexpr (R == 16) dft16<S>(v);
  else if constexpr (R == 8) dft8<S>(v);
  else if constexpr (R == 4) dft4<S>(v);
  else dft2<S>(v);
}

// ------------------------------------------------------------------ register/shared Stockham FFT
// One line of N = 2^m (m >= 4) complex values, transformed by nthr = N/16
// threads holding 16 values each.  On entry thread tid holds
// x[tid + r N/16] (r = 0..15) -- exactly the inputs of its first radix-16
// butterfly -- so the caller loads straight from global memory into
// registers.  Pass with radix R and span Ns (product of earlier radices):
// butterfly j reads x[j + r N/R], twiddles by exp(S 2 pi i r k /(Ns R)) with
// k = j mod Ns, and writes x[(j - k) R + k + r Ns].  Intermediate passes
// exchange through shared memory (XOR-swizzled, bank-conflict-free for
// these access patterns); the last pass leaves X[tid + nthr (i + r 16/R)] in
// v[i R + r], natural order across threads, for the caller to store.
// Twiddles exp(S 2 pi i e/N) = lo[e & 63] * hi[e >> 6] from a two-level table
// of exp(+2 pi i e/N) in shared memory.

__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 4) & 15); }
// swz(x + d) = swz_at(x, d) + d for d a multiple of 16: the XOR mask of the low 4 bits
// moves by d / 16 (mod 16), the rest of d passes through.  With d a compile-time
// multiple of 16 the mask takes few distinct values across a pass's r (one when d is
// a multiple of 256), so the bases are computed once and d becomes an immediate offset.
__device__ __forceinline__ int swz_at(int x, int d) { return x ^ (((x >> 4) + (d >> 4)) & 15); }

template <int S>
__device__ __forceinline__ float2 twiddle(const float2* lo, const float2* hi, int e) {
  float2 w = cmul(lo[e & 63], hi[e >> 6]);
  if (S < 0) w.y = -w.y;
  return w;
}

template <int R, int S>
__device__ __forceinline__ void fft_pass(float2 (&v)[16], float2* buf, int N, int Ns, int tid,
                                         int nthr, const float2* lo, const float2* hi, bool last) {
  constexpr int B = 16 / R;
  const int NR = N / R;
#pragma unroll
  for (int i = 0; i < B; ++i) {
    const int j = tid + i * nthr;
#pragma unroll
    for (int r = 0; r < R; ++r) v[i * R + r] = buf[swz(j + r * NR)];
  }
  const int tstep = N / (Ns * R);
#pragma unroll
  for (int i = 0; i < B; ++i) {
    const int j = tid + i * nthr;
    const int k = j & (Ns - 1);
    const int e = k * tstep;
    // w^r from the bases w, w^2, w^4, w^8, multiplied in just in time so
    // that few twiddles are live at once
    const float2 w1 = twiddle<S>(lo, hi, e);
    v[i * R + 1] = cmul(v[i * R + 1], w1);
    if constexpr (R >= 4) {
      const float2 w2 = twiddle<S>(lo, hi, 2 * e);
      const float2 w3 = cmul(w1, w2);
      v[i * R + 2] = cmul(v[i * R + 2], w2);
      v[i * R + 3] = cmul(v[i * R + 3], w3);
      if constexpr (R >= 8) {
        const float2 w4 = twiddle<S>(lo, hi, 4 * e);
        v[i * R + 4] = cmul(v[i * R + 4], w4);
        v[i * R + 5] = cmul(v[i * R + 5], cmul(w1, w4));
        v[i * R + 6] = cmul(v[i * R + 6], cmul(w2, w4));
        v[i * R + 7] = cmul(v[i * R + 7], cmul(w3, w4));
        if constexpr (R >= 16) {
          const float2 w8 = twiddle<S>(lo, hi, 8 * e);
          const float2 w12 = cmul(w4, w8);
          v[i * R + 8] = cmul(v[i * R + 8], w8);
          v[i * R + 9] = cmul(v[i * R + 9], cmul(w1, w8));
          v[i * R + 10] = cmul(v[i * R + 10], cmul(w2, w8));
          v[i * R + 11] = cmul(v[i * R + 11], cmul(w3, w8));
          v[i * R + 12] = cmul(v[i * R + 12], w12);
          v[i * R + 13] = cmul(v[i * R + 13], cmul(w1, w12));
          v[i * R + 14] = cmul(v[i * R + 14], cmul(w2, w12));
          v[i * R + 15] = cmul(v[i * R + 15], cmul(w3, w12));
        }
      }
    }
    dftR<R, S>(&v[i * R]);
  }
  if (last) return;
  __syncthreads();  // every thread has read buf
#pragma unroll
  for (int i = 0; i < B; ++i) {
    const int j = tid + i * nthr;
    const int k = j & (Ns - 1);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) buf[swz(base + r * Ns)] = v[i * R + r];
  }
  __syncthreads();
}

// Radix of the last pass for N = 2^m.
__device__ __forceinline__ int last_radix(int N) {
  const int m = (31 - __clz(N)) & 3;
  return m == 0 ? 16 : (1 << m);
}

// Index m of X[tid + nthr * m] held in v[idx] after fft_reg.
__device__ __forceinline__ int out_index(int idx, int Rl) {
  return idx / Rl + (idx % Rl) * (16 / Rl);
}

template <int S>
__device__ __forceinline__ void fft_reg(float2 (&v)[16], float2* buf, int N, int tid, int nthr,
                                        const float2* lo, const float2* hi) {
  dft16<S>(v);  // first pass: R = 16, Ns = 1 (no twiddles)
  int m = (31 - __clz(N)) - 4;
  if (m == 0) return;
#pragma unroll
  for (int r = 0; r < 16; ++r) buf[swz(tid * 16 + r)] = v[r];
  __syncthreads();
  int Ns = 16;
  while (m > 0) {
    const int R = m >= 4 ? 16 : (1 << m);
    m -= (R == 16 ? 4 : (R == 8 ? 3 : (R == 4 ? 2 : 1)));
    const bool last = (m == 0);
    if (R == 16) fft_pass<16, S>(v, buf, N, Ns, tid, nthr, lo, hi, last);
    else if (R == 8) fft_pass<8, S>(v, buf, N, Ns, tid, nthr, lo, hi, last);
    else if (R == 4) fft_pass<4, S>(v, buf, N, Ns, tid, nthr, lo, hi, last);
    else fft_pass<2, S>(v, buf, N, Ns, tid, nthr, lo, hi, last);
    Ns *= R;
  }
}

// The same transform with N a compile-time constant: pass radices, strides,
// twiddle steps and swizzle offsets fold into constants (fft_reg computes them
// at run time).  Instantiated for N = 256 .. 8192.
template <int R, int S, int N, int Ns, bool LAST>
__device__ __forceinline__ void fft_pass_t(float2 (&v)[16], float2* buf, int tid, const float2* lo,
                                           const float2* hi) {
  constexpr int B = 16 / R, NR = N / R, nthr = N / 16, tstep = N / (Ns * R);
  static_assert(NR % 16 == 0 && Ns % 16 == 0, "offsets that keep the swizzle's low bits");
#pragma unroll
  for (int i = 0; i < B; ++i) {
    const int j = tid + i * nthr;
#pragma unroll
    for (int r = 0; r < R; ++r) v[i * R + r] = buf[swz_at(j, r * NR) + r * NR];
  }
#pragma unroll
  for (int i = 0; i < B; ++i) {
    const int j = tid + i * nthr;
    const int k = j & (Ns - 1);
    const int e = k * tstep;
    const float2 w1 = twiddle<S>(lo, hi, e);
    v[i * R + 1] = cmul(v[i * R + 1], w1);
    if constexpr (R >= 4) {
      const float2 w2 = twiddle<S>(lo, hi, 2 * e);
      const float2 w3 = cmul(w1, w2);
      v[i * R + 2] = cmul(v[i * R + 2], w2);
      v[i * R + 3] = cmul(v[i * R + 3], w3);
      if constexpr (R >= 8) {
        const float2 w4 = twiddle<S>(lo, hi, 4 * e);
        v[i * R + 4] = cmul(v[i * R + 4], w4);
        v[i * R + 5] = cmul(v[i * R + 5], cmul(w1, w4));
        v[i * R + 6] = cmul(v[i * R + 6], cmul(w2, w4));
        v[i * R + 7] = cmul(v[i * R + 7], cmul(w3, w4));
        if constexpr (R >= 16) {
          const float2 w8 = twiddle<S>(lo, hi, 8 * e);
          const float2 w12 = cmul(w4, w8);
          v[i * R + 8] = cmul(v[i * R + 8], w8);
          v[i * R + 9] = cmul(v[i * R + 9], cmul(w1, w8));
          v[i * R + 10] = cmul(v[i * R + 10], cmul(w2, w8));
          v[i * R + 11] = cmul(v[i * R + 11], cmul(w3, w8));
          v[i * R + 12] = cmul(v[i * R + 12], w12);
          v[i * R + 13] = cmul(v[i * R + 13], cmul(w1, w12));
          v[i * R + 14] = cmul(v[i * R + 14], cmul(w2, w12));
          v[i * R + 15] = cmul(v[i * R + 15], cmul(w3, w12));
        }
      }
    }
    dftR<R, S>(&v[i * R]);
  }
  if constexpr (!LAST) {
    __syncthreads();
#pragma unroll
    for (int i = 0; i < B; ++i) {
      const int j = tid + i * nthr;
      const int k = j & (Ns - 1);
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[swz_at(base, r * Ns) + r * Ns] = v[i * R + r];
    }
    __syncthreads();
  }
}

template <int S, int N, int Ns>
__device__ __forceinline__ void fft_passes_t(float2 (&v)[16], float2* buf, int tid,
                                             const float2* lo, const float2* hi) {
  if constexpr (Ns < N) {
    constexpr int rem = N / Ns;
    constexpr int R = rem >= 16 ? 16 : rem;
    fft_pass_t<R, S, N, Ns, Ns * R == N>(v, buf, tid, lo, hi);
    fft_passes_t<S, N, Ns * R>(v, buf, tid, lo, hi);
  }
}

template <int S, int N>
__device__ __forceinline__ void fft_reg_t(float2 (&v)[16], float2* buf, int tid, const float2* lo,
                                          const float2* hi) {
  dft16<S>(v);
  if constexpr (N > 16) {
#pragma unroll
    for (int r = 0; r < 16; ++r) buf[swz(tid * 16 + r)] = v[r];
    __syncthreads();
    fft_passes_t<S, N, 16>(v, buf, tid, lo, hi);
  }
}

constexpr int last_radix_c(int N) {
  return ((N == 16 || N == 256 || N == 4096) ? 16
          : (N == 32 || N == 512 || N == 8192) ? 2
          : (N == 64 || N == 1024) ? 4 : 8);
}

// One line of N points (NT = N known at compile time, or NT = 0: N at run time).
template <int S, int NT>
__device__ __forceinline__ void fft_line(float2 (&v)[16], float2* buf, int N, int tid, int nthr,
                                         const float2* lo, const float2* hi) {
  if constexpr (NT > 0) fft_reg_t<S, NT>(v, buf, tid, lo, hi);
  else fft_reg<S>(v, buf, N, tid, nthr, lo, hi);
}

template <int NT>
__device__ __forceinline__ int line_last_radix(int N) {
  if constexpr (NT > 0) return last_radix_c(NT);
  else return last_radix(N);
}

// Copies the two-level twiddle table (64 + max(1, N/64) entries) to shared memory.
__device__ __forceinline__ void load_twiddles(float2* dst, const float2* src, int N) {
  const int n = 64 + max(1, N >> 6);
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(&src[i]);
}

constexpr int kTwSlots = 64 + 128;  // table slots reserved in shared memory (N <= 8192)

// ------------------------------------------------------------------ bulk copies + mbarriers
// (the 1-D bulk copy, mbarrier and tcgen05 fence helpers are in gr_device.cuh)

// Tiled 2-D TMA load of one box at (x, y) (x: innermost, in elements) into
// shared memory, completed on `bar`.  x * element size must be a multiple of 16.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
// ------------------------------------------------------------------ phase ramps

__global__ void phase_kernel(PhaseArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int pair = blockIdx.y;
  if (j >= a.J) return;
  const int s1 = a.slice_base + 2 * pair;
  const int s2 = s1 + 1;
  double c1 = a.centers ? (double)a.centers[s1] : (double)a.center_default;
  double c2 = (a.centers && (2 * pair + 1) < a.n_slices_valid) ? (double)a.centers[s2] : c1;
  // e_k = exp(-2 pi i j c_k / pdim) in FP64
  double sn1, cs1, sn2, cs2;
  sincospi(-2.0 * (double)j * c1 / (double)a.pdim, &sn1, &cs1);
  sincospi(-2.0 * (double)j * c2 / (double)a.pdim, &sn2, &cs2);
  const double f = 0.5 * (double)a.filt[j];
  a.pq[(size_t)pair * a.J + j] =
      make_float4((float)(f * (cs1 + cs2)), (float)(f * (sn1 + sn2)), (float)(f * (cs1 - cs2)),
                  (float)(f * (sn1 - sn2)));
}

// ------------------------------------------------------------------ spectra (K1)

template <typename T>
__device__ __forceinline__ float load_sino(const T* row, int k, const float*, const float*);
template <>
__device__ __forceinline__ float load_sino<float>(const float* row, int k, const float*, const float*) {
  return __ldg(&row[k]);
}
// 16-bit inputs go through the read-only path as their raw bits (a plain dereference
// of these pointers compiles to loads the compiler cannot treat as read-only global
// ones: measured 1.5x the f32 path's spectra time at half the bytes)
__device__ __forceinline__ unsigned short ldg_u16(const void* row, int k) {
  return __ldg(static_cast<const unsigned short*>(row) + k);
}
template <>
__device__ __forceinline__ float load_sino<__half>(const __half* row, int k, const float*, const float*) {
  return __half2float(__ushort_as_half(ldg_u16(row, k)));
}
template <>
__device__ __forceinline__ float load_sino<__nv_bfloat16>(const __nv_bfloat16* row, int k,
                                                          const float*, const float*) {
  return __bfloat162float(__ushort_as_bfloat16(ldg_u16(row, k)));
}
// Raw uint16 counts with flat/dark: the normalisation of
// gridrec/GPU/tomo_recon.cpp:1533-1541 (log((flat-dark)/(raw-dark)), 0 when
// raw <= dark or the ratio is not positive), as the difference of two fast
// logarithms (no division; ~1e-6 absolute on line integrals of a few units):
// the load runs inside the issue-bound spectra FFT kernel.
template <>
__device__ __forceinline__ float load_sino<uint16_t>(const uint16_t* row, int k, const float* flat,
                                                     const float* dark) {
  const float d = __ldg(&dark[k]);
  const float v = (float)ldg_u16(row, k) - d;
  const float fd = __ldg(&flat[k]) - d;
  return (v > 0.f && fd > 0.f) ? __logf(fd) - __logf(v) : 0.f;
}
// Raw uint16 counts, linear normalisation of the HDF5 path of
// gridrec/GPU/tomo_recon.cpp:1871-1877 and :2019: 1 - (raw - dark) / (flat - dark)
// in float, in that order (flat = 0.5 white1 + 0.5 white2 gives the reference's
// denominator bit for bit; no guard, as there).
struct U16Linear {
  uint16_t v;
};
template <>
__device__ __forceinline__ float load_sino<U16Linear>(const U16Linear* row, int k,
                                                      const float* flat, const float* dark) {
  const float d = __ldg(&dark[k]);
  return __fsub_rn(1.f, __fdiv_rn(__fsub_rn((float)ldg_u16(row, k), d), __fsub_rn(__ldg(&flat[k]), d)));
}

// Lines of up to 4096 points run 64-register variants (several CTAs per SM);
// 8192-point lines need 512 threads and use the MAXT = 512 variants.
// Raw u16 counts with the slice's precomputed {dark, log(flat - dark) or NaN}: the
// value of load_sino<uint16_t> (same operations, same order) from one 8-byte load and
// one logarithm.
__device__ __forceinline__ float raw_log(unsigned short raw, const float2* dl, int k) {
  const float2 q = __ldg(&dl[k]);
  const float v = (float)raw - q.x;
  return (v > 0.f && q.y == q.y) ? q.y - __logf(v) : 0.f;
}

// {dark, log(flat - dark)} of the chunk's slices (NaN where flat - dark is not
// positive, which makes raw_log return 0 as the per-sample form does).
__global__ void dark_log_kernel(const float* flat, const float* dark, long flat_stride,
                                int slice_base, int n_det, float2* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (k >= n_det) return;
  const long fo = (long)(slice_base + s) * flat_stride;
  const float d = __ldg(&dark[fo + k]);
  const float fd = __ldg(&flat[fo + k]) - d;
  out[(size_t)s * n_det + k] = make_float2(d, fd > 0.f ? __logf(fd) : __int_as_float(0x7fc00000));
}

cudaError_t launch_dark_log(const float* flat, const float* dark, long flat_stride, int slice_base,
                            int n_valid, int n_det, float2* out, cudaStream_t s) {
  dim3 grid((n_det + 255) / 256, n_valid);
  dark_log_kernel<<<grid, 256, 0, s>>>(flat, dark, flat_stride, slice_base, n_det, out);
  return cudaGetLastError();
}

// Element type of the staged row (the 16-bit types as their bits).
template <typename T>
struct StagedType {
  using U = unsigned short;
};
template <>
struct StagedType<float> {
  using U = float;
};
template <typename T>
__device__ __forceinline__ float from_staged(const typename StagedType<T>::U* row, int k,
                                             const float* flat, const float* dark);
template <>
__device__ __forceinline__ float from_staged<float>(const float* row, int k, const float*,
                                                    const float*) {
  return row[k];
}
template <>
__device__ __forceinline__ float from_staged<__half>(const unsigned short* row, int k,
                                                     const float*, const float*) {
  return __half2float(__ushort_as_half(row[k]));
}
template <>
__device__ __forceinline__ float from_staged<__nv_bfloat16>(const unsigned short* row, int k,
                                                            const float*, const float*) {
  return __bfloat162float(__ushort_as_bfloat16(row[k]));
}
template <>
__device__ __forceinline__ float from_staged<uint16_t>(const unsigned short* row, int k,
                                                       const float* flat, const float* dark) {
  const float d = __ldg(&dark[k]);
  const float v = (float)row[k] - d;
  const float fd = __ldg(&flat[k]) - d;
  return (v > 0.f && fd > 0.f) ? __logf(fd) - __logf(v) : 0.f;
}
template <>
__device__ __forceinline__ float from_staged<U16Linear>(const unsigned short* row, int k,
                                                        const float* flat, const float* dark) {
  const float d = __ldg(&dark[k]);
  return __fsub_rn(1.f, __fdiv_rn(__fsub_rn((float)row[k], d), __fsub_rn(__ldg(&flat[k]), d)));
}

template <typename T, int MAXT, int NT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT) spectra_kernel(SpectraArgs a) {
  extern __shared__ __align__(16) float2 sm[];
  __shared__ uint64_t in_bar;
  float2* tw = sm;
  float2* buf = sm + kTwSlots;
  // wide layouts: pairs vary fastest, so the 16 or 32 pairs sharing each 512- or
  // 1024-byte span of the interleaved spectra write it at about the same time
  const int n = a.wide ? blockIdx.y : blockIdx.x, pair = a.wide ? blockIdx.x : blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  load_twiddles(tw, a.tw, a.pdim);
  const T* r1 = static_cast<const T*>(a.s1) + pair * a.pair_stride + (long)n * a.n_det;
  const T* r2 = (2 * pair + 1 < a.n_slices_valid)
                    ? static_cast<const T*>(a.s2) + pair * a.pair_stride + (long)n * a.n_det
                    : nullptr;
  const long fo = (long)(a.slice_base + 2 * pair) * a.flat_stride;  // slice 1's flat/dark row
  const float* f1 = a.flat ? a.flat + fo : nullptr;
  const float* d1 = a.dark ? a.dark + fo : nullptr;
  const float* f2 = f1 ? f1 + a.flat_stride : nullptr;
  const float* d2 = d1 ? d1 + a.flat_stride : nullptr;
  constexpr bool kRaw = std::is_same<T, uint16_t>::value;
  const float2* q1 = kRaw && a.dl ? a.dl + (size_t)(2 * pair) * a.n_det : nullptr;
  const float2* q2 = q1 ? q1 + a.n_det : nullptr;
  float2 v[16];
  // The pair's two rows are contiguous: with an error word and 16-byte-aligned rows,
  // two 1-D bulk copies land them in the exchange buffer (2 n_det elements <= 8 pdim
  // bytes) on an mbarrier, instead of 16 strided loads per row and thread whose
  // latency the kernel cannot hide (bounded wait: on a timeout the error word is
  // set and the inputs read as zeros).  Same values either way.
  using U = typename StagedType<T>::U;
  const unsigned row_bytes = (unsigned)a.n_det * (unsigned)sizeof(U);
  const bool staged = a.err && (row_bytes & 15u) == 0 && ((uintptr_t)r1 & 15u) == 0 &&
                      (!r2 || ((uintptr_t)r2 & 15u) == 0);
  if (staged) {
    U* st1 = reinterpret_cast<U*>(buf);
    U* st2 = st1 + a.n_det;
    if (tid == 0) {
      mbar_init(&in_bar, 1);
      fence_mbar_init();
      mbar_expect_tx(&in_bar, r2 ? 2u * row_bytes : row_bytes);
      bulk_g2s(st1, r1, row_bytes, &in_bar);
      if (r2) bulk_g2s(st2, r2, row_bytes, &in_bar);
    }
    __syncthreads();  // the barrier is initialised before any thread polls it
    const bool ok = mbar_wait(&in_bar, 0u);
    if (!ok && tid == 0) atomicExch(a.err, 1);
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int k = tid + r * nthr;
      float x = 0.f, y = 0.f;
      if (ok && k < a.n_det) {
        if constexpr (kRaw) {
          if (q1) {
            x = raw_log(st1[k], q1, k);
            if (r2) y = raw_log(st2[k], q2, k);
          } else {
            x = from_staged<T>(st1, k, f1, d1);
            if (r2) y = from_staged<T>(st2, k, f2, d2);
          }
        } else {
          x = from_staged<T>(st1, k, f1, d1);
          if (r2) y = from_staged<T>(st2, k, f2, d2);
        }
      }
      v[r] = make_float2(x, y);
    }
    if (__syncthreads_or(!ok) && tid == 0) mbar_wait(&in_bar, 0u);  // copies done before reuse
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
      const int k = tid + r * nthr;
      float x = 0.f, y = 0.f;
      if (k < a.n_det) {
        if constexpr (kRaw) {
          if (q1) {
            x = raw_log(ldg_u16(r1, k), q1, k);
            if (r2) y = raw_log(ldg_u16(r2, k), q2, k);
          } else {
            x = load_sino<T>(r1, k, f1, d1);
            if (r2) y = load_sino<T>(r2, k, f2, d2);
          }
        } else {
          x = load_sino<T>(r1, k, f1, d1);
          if (r2) y = load_sino<T>(r2, k, f2, d2);
        }
      }
      v[r] = make_float2(x, y);
    }
  }
  __syncthreads();  // twiddle table ready; the staged rows read before buf is reused
  fft_line<+1, NT>(v, buf, a.pdim, tid, nthr, tw, tw + 64);
  // F[j] and F[pdim - j] meet through shared memory
  const int Rl = line_last_radix<NT>(a.pdim);
  __syncthreads();
  // offsets d = multiples of nthr = pdim / 16: when nthr is a multiple of 16 (pdim >=
  // 256, always for the compile-time lengths) swz(tid + d) = swz_at(tid, d) + d
  const bool d16 = NT > 0 || (nthr & 15) == 0;
#pragma unroll
  for (int idx = 0; idx < 16; ++idx) {
    const int d = nthr * out_index(idx, Rl);
    buf[d16 ? swz_at(tid, d) + d : swz(tid + d)] = v[idx];
  }
  __syncthreads();
  const float4* pq = a.pq + (size_t)pair * a.J;
  // plain: [pair][dir][j]; wide (G = 16 or 32 pairs): [pair / G][dir][j / 4][pair % G][j % 4],
  // so each pair still writes whole 32-byte sectors and the gridding kernel stages a
  // run of G pairs as one contiguous range.  For G = 32 the two 16-byte halves of
  // pair p's chunk are swapped when (p / 4) is odd (sample j at position
  // (j % 4) ^ (2 ((p / 4) % 2))): the 32-pair kernel's lanes then read their chunks
  // with two conflict-free 16-byte loads.
  float2* o1;
  float2* o2;
  int qshift, qmask, qlog, rot = 0;
  if (a.wide) {
    const int G = a.wide;
    qlog = G == 32 ? 7 : 6;  // float2 per quad: 4 samples x G pairs
    const size_t per_dir = (size_t)(a.J >> 2) << qlog;
    o1 = a.spec + ((size_t)(pair / G) * 2 * a.n_ang + 2 * n) * per_dir + (pair % G) * 4;
    o2 = o1 + per_dir;
    qshift = 2;
    qmask = 3;
    if (G == 32) rot = ((pair >> 2) & 1) << 1;
  } else {
    o1 = a.spec + ((size_t)pair * a.n_ang + n) * 2 * a.J;
    o2 = o1 + a.J;
    qshift = 30;
    qmask = 0x3fffffff;
    qlog = 6;
  }
  // J = pdim / 2 = 8 nthr: thread tid takes j = tid + i nthr, i < 8; the swizzled
  // addresses of j and pdim - j follow from tid and pdim - tid by swz_at
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int j = tid + i * nthr;
    if (j >= a.J) break;
    const int oj = ((j >> qshift) << qlog) + ((j & qmask) ^ rot);
    float2 c1 = make_float2(0.f, 0.f), c2 = make_float2(0.f, 0.f);
    if (j > 0) {
      const int d = i * nthr;
      const float2 F = buf[d16 ? swz_at(tid, d) + d : swz(j)];
      const float2 G = buf[d16 ? swz_at(a.pdim - tid, -d) - d : swz(a.pdim - j)];
      const float4 q = __ldg(&pq[j]);  // P = (x, y), Q = (z, w)
      // C1 = P F + Q conj(G);  C2 = conj(P) G + conj(Q) conj(F)
      c1.x = q.x * F.x - q.y * F.y + q.z * G.x + q.w * G.y;
      c1.y = q.x * F.y + q.y * F.x - q.z * G.y + q.w * G.x;
      c2.x = q.x * G.x + q.y * G.y + q.z * F.x - q.w * F.y;
      c2.y = q.x * G.y - q.y * G.x - q.z * F.y - q.w * F.x;
      if (a.roi_off) {  // ROI offset: C1 exp(-i j off), C2 exp(+i j off) (GridrecCPP)
        double sn, cs;
        sincos((double)j * a.roi_off[n], &sn, &cs);
        const float pr = (float)cs, pi = (float)-sn;
        c1 = make_float2(c1.x * pr - c1.y * pi, c1.x * pi + c1.y * pr);
        c2 = make_float2(c2.x * pr + c2.y * pi, c2.y * pr - c2.x * pi);
      }
    }
    o1[oj] = c1;
    o2[oj] = c2;
  }
}

// ------------------------------------------------------------------ gridding (K2)
// Gather over binned work items: each work item is one kTile x kTile tile of
// H plus the runs of samples (consecutive j along one direction, built on the
// host from the exact ray/tile geometry) whose footprint can reach the tile.
// Each sample adds w(|u - iu|) w(|v - iv|) C to every cell within L/2 in both
// coordinates -- the tap set and nearest-neighbour table index of
// gridrec.cu:546-566.  The second half of the reference's scatter
// (H[M-iu][M-iv] += w C2) is the direction d = 2n+1 at the mirrored position.
// Cells in row 0 or column 0 stay zero (the reference clamps taps to [1, M-1]).
//
// Execution: a persistent grid of warps pulls (work item, pair group) entries
// from a queue.  A warp accumulates the tile of PG slice pairs (their
// cells interleaved as float4) in a private shared-memory tile, NT lanes per
// sample (lane t owns footprint row t; column weights are exchanged by
// shuffles), so the geometry -- positions, table lookups -- is computed once
// for both pairs.  The samples of one step are taken P apart along the run
// with P * max(|du|,|dv|) > L, so no two of them share a valid tap (taps lie
// within L/2 of their sample; P per run comes from the host), so
// plain read-modify-write needs no atomics, and the summation order is fixed,
// so the result is bitwise reproducible.  Tap positions and table indices are
// FP64, as the FP64 restatement of the algorithm forms them: FP32 positions put some taps on
// the other side of a table-bin boundary (a position error of 2^-12 at
// |u| ~ 2048 moves the index when |u - c| * tblspcg lies that close to a
// half-integer), which alone costs ~5e-4 relative L2.  Tiles split over several items
// leave partial tiles in scratch, summed in slot order by split_reduce_kernel.

constexpr int kTileStride = kTile + 1;
constexpr int kGridWarps = 4;

// (int)(d * ts + 0.5) for d >= 0 -- the nearest-neighbour table index of
// gridrec.h:53 -- in FP64 with the product and the sum rounded separately, as
// the FP64 restatement forms them; capped so that far taps stay in int range
// (callers clamp to the table length and zero taps beyond L/2).
__device__ __forceinline__ int table_index64(double d, double ts) {
  return (int)fmin(__dadd_rn(__dmul_rn(d, ts), 0.5), 2.0e9);
}

// A cell of PG pairs gridded together: float4 (C_A, C_B) for two, float2 for one.
template <int PG>
struct GridCell;
template <>
struct GridCell<2> {
  using T = float4;
  static __device__ __forceinline__ float4 zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  static __device__ __forceinline__ float4 make(float2 A, float2 B) {
    return make_float4(A.x, A.y, B.x, B.y);
  }
  static __device__ __forceinline__ float4 scale(float w, float4 c) {
    return make_float4(w * c.x, w * c.y, w * c.z, w * c.w);
  }
  static __device__ __forceinline__ void fma(float w, float4 c, float4& h) {
    h.x = fmaf(w, c.x, h.x);
    h.y = fmaf(w, c.y, h.y);
    h.z = fmaf(w, c.z, h.z);
    h.w = fmaf(w, c.w, h.w);
  }
  static __device__ __forceinline__ float2 pairA(float4 c) { return make_float2(c.x, c.y); }
  static __device__ __forceinline__ float2 pairB(float4 c) { return make_float2(c.z, c.w); }
};
template <>
struct GridCell<1> {
  using T = float2;
  static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
  static __device__ __forceinline__ float2 make(float2 A, float2) { return A; }
  static __device__ __forceinline__ float2 scale(float w, float2 c) {
    return make_float2(w * c.x, w * c.y);
  }
  static __device__ __forceinline__ void fma(float w, float2 c, float2& h) {
    h.x = fmaf(w, c.x, h.x);
    h.y = fmaf(w, c.y, h.y);
  }
  static __device__ __forceinline__ float2 pairA(float2 c) { return c; }
  static __device__ __forceinline__ float2 pairB(float2) { return make_float2(0.f, 0.f); }
};

// PG = 2: two pairs per warp from one set of weights (chunks of two or more pairs);
// PG = 1: a lone pair, with half the tile memory and read-modify-write traffic.  Pair
// A's arithmetic is the same in both, so a pair's cells are bitwise equal.
template <int NT, int PG>
__global__ void __launch_bounds__(kGridWarps * 32) grid_kernel(GridArgs a) {
  using CellOps = GridCell<PG>;
  using Cell = typename CellOps::T;
  constexpr int SPW = 32 / NT;  // samples per step
  extern __shared__ float4 smem4[];
  float* s_wtbl = reinterpret_cast<float*>(smem4);
  Cell* tiles = reinterpret_cast<Cell*>(smem4 + 257);  // table: up to 1028 floats
  for (int i = threadIdx.x; i <= a.ltbl; i += blockDim.x) s_wtbl[i] = __ldg(&a.wtbl[i]);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cell* tile = tiles + warp * (kTile * kTileStride);
  // the current run's samples of the PG pairs: stage[j - jlo] = (C_A[, C_B])
  Cell* stage = tiles + kGridWarps * (kTile * kTileStride) + warp * kRunMax;
  const int slot_k = lane / NT;          // sample slot of this lane
  const int t = lane - slot_k * NT;      // footprint row of this lane
  const int lane0 = slot_k * NT;         // first lane of this sample
  const bool lane_used = slot_k < SPW;
  const double L2d = a.L2, tsd = a.tblspcg;
  const int ltbl = a.ltbl;
  const int groups = (a.pairs + PG - 1) / PG;
  const unsigned total = (unsigned)a.n_items * (unsigned)groups;
  const size_t spec_pair = (size_t)a.n_ang * 2 * a.J;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(a.queue, 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= total) break;
    const int grp = (int)(w / (unsigned)a.n_items);
    const Item it = a.items[w - (unsigned)grp * (unsigned)a.n_items];
    const int pA = grp * PG;
    const bool hasB = PG == 2 && pA + 1 < a.pairs;
    const int tu = it.tile / a.tiles_v;
    const int tv = it.tile - tu * a.tiles_v;
    const int p0 = tu * kTile, q0 = tv * kTile;
    for (int i = lane; i < kTile * kTileStride; i += 32) tile[i] = CellOps::zero();
    __syncwarp();
    const double offu = (double)(a.M / 2 - p0), offv = (double)(a.M / 2 - q0);
    const float2* specA = a.spec + (size_t)pA * spec_pair;
    const float2* specB = hasB ? specA + spec_pair : specA;
    // Software pipeline over runs: the samples of run r+1 are loaded into
    // registers (lane l holds j = jlo + l and jlo + l + 32) while run r is
    // gridded from the shared staging buffer.
    // The run record and its direction travel with the prefetch too, so no
    // dependent global load sits at the start of a run.
    float2 nA0 = make_float2(0.f, 0.f), nA1 = nA0, nB0 = nA0, nB1 = nA0;
    Run nrun{0, 0, -1, 1};
    double2 ndir = make_double2(0.0, 0.0);
    auto prefetch = [&](int rr) {
      if (rr >= it.run_end) return;
      nrun = a.runs[rr];
      ndir = __ldg(&a.dir[nrun.dir]);
      const float2* pa = specA + (size_t)nrun.dir * a.J;
      const float2* pb = specB + (size_t)nrun.dir * a.J;
      if (nrun.jlo + lane <= nrun.jhi) {
        nA0 = __ldg(&pa[nrun.jlo + lane]);
        if (PG == 2) nB0 = __ldg(&pb[nrun.jlo + lane]);
      }
      if (nrun.jlo + 32 + lane <= nrun.jhi) {
        nA1 = __ldg(&pa[nrun.jlo + 32 + lane]);
        if (PG == 2) nB1 = __ldg(&pb[nrun.jlo + 32 + lane]);
      }
    };
    prefetch(it.run_begin);
    for (int r = it.run_begin; r < it.run_end; ++r) {
      const Run run = nrun;
      const double2 d = ndir;
      stage[lane] = CellOps::make(nA0, nB0);
      stage[32 + lane] = CellOps::make(nA1, nB1);
      __syncwarp();
      prefetch(r + 1);
      // run.P: samples P apart never share a valid tap (P * max(|du|,|dv|)
      // > L with margin), chosen on the host to minimise the steps
      const int P = run.P;
      for (int blk = run.jlo; blk <= run.jhi; blk += SPW * P) {
        for (int ph = 0; ph < P && blk + ph <= run.jhi; ++ph) {
          const int j = blk + ph + P * slot_k;
          const bool active = lane_used && j <= run.jhi;
          // positions, taps and table indices in FP64 (tile-relative, exact
          // offsets), as the float64 algorithm forms them
          const double fj = (double)j;
          const double u = fma(fj, d.x, offu), v = fma(fj, d.y, offv);
          const int iu0 = (int)ceil(u - L2d), iv0 = (int)ceil(v - L2d);
          const int row = iu0 + t;
          const int col = iv0 + t;
          const double du = fabs(u - (double)row);
          const double dv = fabs(v - (double)col);
          const float wtu = s_wtbl[min(table_index64(du, tsd), ltbl)];
          const float wtv = s_wtbl[min(table_index64(dv, tsd), ltbl)];
          const float wu = (active && du <= L2d && (unsigned)row < (unsigned)kTile) ? wtu : 0.f;
          const float wvt = (active && dv <= L2d && (unsigned)col < (unsigned)kTile) ? wtv : 0.f;
          Cell cc = CellOps::zero();
          if (wu != 0.f) cc = stage[j - run.jlo];
          const Cell c4 = CellOps::scale(wu, cc);
          float wv[NT];
#pragma unroll
          for (int s2 = 0; s2 < NT; ++s2) wv[s2] = __shfl_sync(0xffffffffu, wvt, lane0 + s2);
          Cell* cell = tile + row * kTileStride + iv0;
          Cell h[NT];
#pragma unroll
          for (int s2 = 0; s2 < NT; ++s2)
            if (wu != 0.f && wv[s2] != 0.f) h[s2] = cell[s2];
#pragma unroll
          for (int s2 = 0; s2 < NT; ++s2) CellOps::fma(wv[s2], c4, h[s2]);
#pragma unroll
          for (int s2 = 0; s2 < NT; ++s2)
            if (wu != 0.f && wv[s2] != 0.f) cell[s2] = h[s2];
          __syncwarp();
        }
      }
    }
    const int np = min(kTile, a.M - p0), nq = min(kTile, a.M - q0);
    if (it.slot < 0) {
      const size_t MM = (size_t)a.M * a.M;
      float2* HA = a.H + (size_t)pA * MM;
      float2* HB = HA + MM;
      if (lane < nq) {
        const int q = q0 + lane;
        for (int pr = 0; pr < np; ++pr) {
          const int p = p0 + pr;
          Cell val = tile[pr * kTileStride + lane];
          if (p == 0 || q == 0) val = CellOps::zero();
          HA[(size_t)p * a.M + q] = CellOps::pairA(val);
          if (hasB) HB[(size_t)p * a.M + q] = CellOps::pairB(val);
        }
      }
    } else {
      // partial tile of a split tile: summed later by split_reduce_kernel
      Cell* part = reinterpret_cast<Cell*>(a.scratch) + ((size_t)grp * a.n_slots + it.slot) * (kTile * kTile);
      for (int pr = 0; pr < kTile; ++pr) part[pr * kTile + lane] = tile[pr * kTileStride + lane];
    }
    __syncwarp();
  }
}

// Sums the partial tiles of every split tile in slot order and writes H.
// Grid: (split tiles, pair groups); 256 threads over the tile's cells.
template <int PG>
__global__ void __launch_bounds__(256) split_reduce_kernel(GridArgs a) {
  using CellOps = GridCell<PG>;
  using Cell = typename CellOps::T;
  const int4 sp = a.split_list[blockIdx.x];  // (tile, slot0, nsplit, -)
  const int grp = blockIdx.y;
  const int pA = grp * PG;
  const bool hasB = PG == 2 && pA + 1 < a.pairs;
  const int tu = sp.x / a.tiles_v, tv = sp.x - (sp.x / a.tiles_v) * a.tiles_v;
  const int p0 = tu * kTile, q0 = tv * kTile;
  const int np = min(kTile, a.M - p0), nq = min(kTile, a.M - q0);
  const Cell* base = reinterpret_cast<const Cell*>(a.scratch) + ((size_t)grp * a.n_slots + sp.y) * (kTile * kTile);
  const size_t MM = (size_t)a.M * a.M;
  float2* HA = a.H + (size_t)pA * MM;
  float2* HB = HA + MM;
  for (int i = threadIdx.x; i < kTile * kTile; i += blockDim.x) {
    const int pr = i / kTile, qc = i - (i / kTile) * kTile;
    if (pr >= np || qc >= nq) continue;
    Cell sum = CellOps::zero();
    for (int k = 0; k < sp.z; ++k) CellOps::fma(1.f, __ldg(&base[(size_t)k * (kTile * kTile) + i]), sum);
    const int p = p0 + pr, q = q0 + qc;
    if (p == 0 || q == 0) sum = CellOps::zero();
    HA[(size_t)p * a.M + q] = CellOps::pairA(sum);
    if (hasB) HB[(size_t)p * a.M + q] = CellOps::pairB(sum);
  }
}

// ------------------------------------------------------------------ gridding, 16 pairs per warp
// The same gather as grid_kernel -- the work-list geometry, tap set and
// nearest-neighbour weights of gridrec.cu:546-566 -- organised for chunks of
// many slice pairs.  Lane l of a warp carries component l & 1 (re, im) of pair
// l >> 1 of a group of kWidePairs pairs, so all lanes apply the same taps, each
// to its own value:
// * the geometry and weights of a sample are warp-uniform and shared by all
//   16 pairs; they depend on the geometry only, so wide_weights_kernel
//   computes them once per work list, with each run's column-pair range, and
//   the kernel copies them in beside the values;
// * a work item is one kWideRows x kWideCols sub-tile whose cells stay in registers
//   for all its runs: no shared-memory read-modify-write and no atomics.
// Every sample carries one weight per sub-tile row and per column,
// w(|u - row|) and w(|v - col|), zero where the distance exceeds L/2 -- the
// test that selects the taps -- and is applied to the register tile with
// packed FP32x2 FMAs over the column pairs its run reaches: no per-sample
// branches or offsets.  A tap adds wv * (wu * value), the rounding
// of grid_kernel, at positions formed as grid_kernel forms them, so the two
// kernels differ only in summation order.  Each cell sums its taps in a fixed
// order (runs in work-list order, samples in j order; split sub-tiles by
// slot): results are bitwise reproducible.  The run's values for the 16 pairs
// are one contiguous range of the interleaved spectra layout
// ([group][dir][j / 4][pair][j % 4]), staged by 16-byte cp.async two runs ahead
// and then moved sample-major (one 32-value row per sample) into a second
// buffer, so the FMA loop reads a sample's values with one conflict-free load
// at a fixed stride.

constexpr int kWideWarps = 4;
// staging: up to kRunMaxW samples span kWideQuads quads of 4 j x 16 pairs
constexpr int kWideQuads = (kRunMaxW + 3) / 4 + 1;
constexpr int kWideStage = kWideQuads * 16 * 4 * 2;  // floats of one staged run
// sample-major rows: 32 values + 8 pad floats, so the rows a restaging store
// writes at once (t and t + 2 of a quad) fall on disjoint banks
constexpr int kWideRowStride = 40;
constexpr int kWideSamp = kWideQuads * 4 * kWideRowStride;
// per warp: staging [2][kWideStage] + sample rows [kWideSamp] + weights [3][kRunMaxW][kWideRec]
// (copies run two runs ahead: values of runs r+1, r+2 in flight or landed
// while run r is applied)
constexpr int kWideWarpFloats = 2 * kWideStage + kWideSamp + 3 * kRunMaxW * kWideRec;

__device__ __forceinline__ void cp_async16(float* dst_smem, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long v) {
  float2 r;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
  return r;
}
// acc += a * b elementwise on packed float pairs (one rounding per element)
__device__ __forceinline__ void ffma2(unsigned long long& acc, unsigned long long a,
                                      unsigned long long b) {
  asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(acc) : "l"(a), "l"(b));
}

// Applies the n samples of one restaged run to the 4 x 8 register tile, over
// column pairs C0..C1 only.  sv points at this lane's value of the run's
// first sample (rows kWideRowStride floats apart); rec holds per sample
// kWideRec floats: 4 row weights, then 8 column weights.
template <int C0, int C1>
__device__ __forceinline__ void wide_apply_run(unsigned long long (&acc)[kWideRows][kWideCols / 2],
                                               const float* sv, const float* rec, int n) {
  static_assert(kWideRows == 4 && kWideCols == 8 && kWideRec == 12, "weight record layout");
  for (int s = 0; s < n; ++s) {
    const float val = sv[s * kWideRowStride];
    const float4 wr = *reinterpret_cast<const float4*>(rec + s * kWideRec);
    const float wrs[4] = {wr.x, wr.y, wr.z, wr.w};
    const float4 wc0 = *reinterpret_cast<const float4*>(rec + s * kWideRec + 4);
    const float4 wc1 = *reinterpret_cast<const float4*>(rec + s * kWideRec + 8);
    const unsigned long long wc[4] = {pack2(wc0.x, wc0.y), pack2(wc0.z, wc0.w),
                                      pack2(wc1.x, wc1.y), pack2(wc1.z, wc1.w)};
#pragma unroll
    for (int rr = 0; rr < kWideRows; ++rr) {
      const float x = wrs[rr] * val;  // wu * value
      const unsigned long long x2 = pack2(x, x);
#pragma unroll
      for (int c = C0; c <= C1; ++c) ffma2(acc[rr][c], wc[c], x2);  // += wv * (wu * value)
    }
  }
}

// The weights of every (run, sample) of the 16-pair work list, computed once
// per work list: they depend on the geometry only.  Thread r takes run r of
// sub-tile meta[r].y (tile index) and writes, for each of its samples, the 4
// row and 8 column weights w(|u - row|), w(|v - col|) -- zero where a distance
// exceeds L/2 -- at wts + meta[r].x * kWideRec, with positions formed as
// grid_kernel forms them (FP64, relative to the enclosing 32 x 32 tile, moved
// to the sub-tile by an integer).  It then replaces meta[r].y by the range of
// column pairs some sample reaches, c2lo * 4 + c2hi, or kWideNoReach.
__global__ void __launch_bounds__(128) wide_weights_kernel(GridArgs a, int n_runs, float* wts,
                                                           int2* meta) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_runs) return;
  const Run run = a.runs[r];
  const int2 m = meta[r];
  const int tu = m.y / a.tiles_v, tv = m.y - (m.y / a.tiles_v) * a.tiles_v;
  const int p0 = tu * kWideRows, q0 = tv * kWideCols;
  const double offu = (double)(a.M / 2 - (p0 & ~(kTile - 1))), subu = (double)(p0 & (kTile - 1));
  const double offv = (double)(a.M / 2 - (q0 & ~(kTile - 1))), subv = (double)(q0 & (kTile - 1));
  const double2 d = a.dir[run.dir];
  const double L2d = a.L2, tsd = a.tblspcg;
  float* w = wts + (size_t)m.x * kWideRec;
  unsigned cols = 0;
  for (int j = run.jlo; j <= run.jhi; ++j, w += kWideRec) {
    const double u = fma((double)j, d.x, offu) - subu, v = fma((double)j, d.y, offv) - subv;
    float4 o[3];
    float* of = reinterpret_cast<float*>(o);
#pragma unroll
    for (int k = 0; k < kWideRows; ++k) {
      const double dd = fabs(u - (double)k);
      of[k] = dd <= L2d ? __ldg(&a.wtbl[min(table_index64(dd, tsd), a.ltbl)]) : 0.f;
    }
#pragma unroll
    for (int k = 0; k < kWideCols; ++k) {
      const double dd = fabs(v - (double)k);
      of[kWideRows + k] = dd <= L2d ? __ldg(&a.wtbl[min(table_index64(dd, tsd), a.ltbl)]) : 0.f;
      if (dd <= L2d) cols |= 1u << k;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) reinterpret_cast<float4*>(w)[k] = o[k];
  }
  meta[r].y = cols ? ((__ffs(cols) - 1) >> 1) * 4 + ((31 - __clz(cols)) >> 1) : kWideNoReach;
}

// kWideMinBlocks CTAs per SM (registers capped accordingly, no spills)
__global__ void __launch_bounds__(kWideWarps * 32, kWideMinBlocks) grid_wide_kernel(GridArgs a) {
  constexpr int TR = kWideRows, TC = kWideCols;
  extern __shared__ float4 smw4[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* wbase = reinterpret_cast<float*>(smw4) + warp * kWideWarpFloats;
  float* stages = wbase;                    // [2][kWideQuads][16][4][2] as copied
  float* samp = wbase + 2 * kWideStage;     // [kWideQuads * 4][kWideRowStride]
  float* recs = samp + kWideSamp;           // [3][kRunMaxW][kWideRec] weights
  const int groups = (a.pairs + kWidePairs - 1) / kWidePairs;
  const unsigned total = (unsigned)a.n_items * (unsigned)groups;
  const size_t per_dir = (size_t)(a.J >> 2) * 64;  // float2 per direction and group
  const size_t MM = (size_t)a.M * a.M;
  const int pl = lane >> 1, cl = lane & 1;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(a.queue, 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= total) break;
    const int grp = (int)(w / (unsigned)a.n_items);
    const Item it = a.items[w - (unsigned)grp * (unsigned)a.n_items];
    const int pg0 = grp * kWidePairs;
    const int np = min(kWidePairs, a.pairs - pg0);
    const int tu = it.tile / a.tiles_v;
    const int tv = it.tile - tu * a.tiles_v;
    const int p0 = tu * TR, q0 = tv * TC;
    const float2* specg = a.spec + (size_t)grp * 2 * a.n_ang * per_dir;
    unsigned long long acc[TR][TC / 2];  // (cell c, cell c + 1) of row r
#pragma unroll
    for (int r = 0; r < TR; ++r)
#pragma unroll
      for (int c = 0; c < TC / 2; ++c) acc[r][c] = 0ull;
    // run rn's quads -> staging buffer vb, its weights -> weight buffer b
    auto stage_run = [&](const Run& rn, int2 mn, int vb, int b) {
      const int nq = (rn.jhi >> 2) - (rn.jlo >> 2) + 1;
      const float2* src = specg + (size_t)rn.dir * per_dir + (size_t)(rn.jlo >> 2) * 64;
      float* vdst = stages + vb * kWideStage;
      for (int i = lane; i < nq * 32; i += 32) cp_async16(vdst + i * 4, src + i * 2);
      const float* wsrc = a.wts + (size_t)mn.x * kWideRec;
      float* wdst = recs + b * (kRunMaxW * kWideRec);
      for (int i = lane; i < (rn.jhi - rn.jlo + 1) * (kWideRec / 4); i += 32)
        cp_async16(wdst + i * 4, wsrc + i * 4);
    };
    // copies run two runs ahead (one cp.async group per run); run records are
    // read one run before their copies are issued.  A tile that no sample
    // reaches has an empty item (rb == re, possibly one past the last run):
    // nothing is read and its cells are written as zeros
    const int rb = it.run_begin, re = it.run_end;
    Run runA{0, 1, 0, 1}, runB = runA, runC = runA;  // runs r, r + 1, r + 2
    int2 metaA = make_int2(0, kWideNoReach), metaB = metaA, metaC = metaA;
    if (rb < re) {
      runA = a.runs[rb];
      metaA = __ldg(&a.wmeta[rb]);
      stage_run(runA, metaA, 0, 0);
    }
    cp_async_commit();
    if (rb + 1 < re) {
      runB = a.runs[rb + 1];
      metaB = __ldg(&a.wmeta[rb + 1]);
      stage_run(runB, metaB, 1, 1);
    }
    cp_async_commit();
    if (rb + 2 < re) {
      runC = a.runs[rb + 2];
      metaC = __ldg(&a.wmeta[rb + 2]);
    }
    int wb = 0;  // weight buffer of run r: (r - rb) % 3
    for (int r = rb; r < re; ++r) {
      const Run run = runA;
      const int2 meta = metaA;
      const int vb = (r - rb) & 1;
      cp_async_wait<1>();  // run r's group has landed (run r + 1's may be in flight)
      __syncwarp();
      // sample-major rows: lane (p, h) moves its 16-byte piece of each quad --
      // samples 2h and 2h + 1 of pair p, (re, im) each -- to rows 4q + 2h and
      // 4q + 2h + 1, columns 2p and 2p + 1
      const float* stage = stages + vb * kWideStage;
      const int nq = (run.jhi >> 2) - (run.jlo >> 2) + 1;
      for (int q = 0; q < nq; ++q) {
        const float4 c = *reinterpret_cast<const float4*>(stage + q * 128 + lane * 4);
        float* dst = samp + (q * 4 + 2 * (lane & 1)) * kWideRowStride + pl * 2;
        *reinterpret_cast<float2*>(dst) = make_float2(c.x, c.y);
        *reinterpret_cast<float2*>(dst + kWideRowStride) = make_float2(c.z, c.w);
      }
      __syncwarp();  // staging buffer read and rows written before it is refilled
      const int wb2 = wb == 0 ? 2 : wb - 1;  // (r + 2 - rb) % 3
      if (r + 2 < re) stage_run(runC, metaC, vb, wb2);  // overlaps runs r and r + 1
      cp_async_commit();  // possibly empty: keeps one group per run
      runA = runB;
      metaA = metaB;
      runB = runC;
      metaB = metaC;
      if (r + 3 < re) {
        runC = a.runs[r + 3];
        metaC = __ldg(&a.wmeta[r + 3]);
      }
      // the run's samples over the column pairs some sample reaches (the
      // other pairs would only add zero products)
      const int n = run.jhi - run.jlo + 1;
      const float* sv = samp + (run.jlo & 3) * kWideRowStride + lane;  // first sample's row
      const float* rec = recs + wb * (kRunMaxW * kWideRec);
      switch (meta.y) {
        case 0: wide_apply_run<0, 0>(acc, sv, rec, n); break;
        case 1: wide_apply_run<0, 1>(acc, sv, rec, n); break;
        case 2: wide_apply_run<0, 2>(acc, sv, rec, n); break;
        case 3: wide_apply_run<0, 3>(acc, sv, rec, n); break;
        case 5: wide_apply_run<1, 1>(acc, sv, rec, n); break;
        case 6: wide_apply_run<1, 2>(acc, sv, rec, n); break;
        case 7: wide_apply_run<1, 3>(acc, sv, rec, n); break;
        case 10: wide_apply_run<2, 2>(acc, sv, rec, n); break;
        case 11: wide_apply_run<2, 3>(acc, sv, rec, n); break;
        case 15: wide_apply_run<3, 3>(acc, sv, rec, n); break;
        default: break;  // kWideNoReach: no sample reaches the sub-tile
      }
      wb = wb == 2 ? 0 : wb + 1;
      __syncwarp();
    }
    cp_async_wait<0>();
    if (it.slot < 0) {
      // lane pairs trade halves so each lane stores one complex cell:
      // lane 2p+0 stores cell (r, c), lane 2p+1 cell (r, c+1)
      float2* Hp = a.H + (size_t)(pg0 + min(pl, np - 1)) * MM;
#pragma unroll
      for (int r = 0; r < TR; ++r) {
#pragma unroll
        for (int c2 = 0; c2 < TC / 2; ++c2) {
          const float2 v = unpack2(acc[r][c2]);  // cells (r, 2 c2), (r, 2 c2 + 1)
          const float give = cl ? v.x : v.y;
          const float got = __shfl_xor_sync(0xffffffffu, give, 1);
          float2 val = cl ? make_float2(got, v.y) : make_float2(v.x, got);
          const int p = p0 + r, q = q0 + 2 * c2 + cl;
          if (p == 0 || q == 0) val = make_float2(0.f, 0.f);
          if (pl < np) Hp[(size_t)p * a.M + q] = val;
        }
      }
    } else {
      // partial sub-tile of a split sub-tile: [cell][lane], summed by split_reduce_wide_kernel
      float* part = reinterpret_cast<float*>(a.scratch) +
                    ((size_t)grp * a.n_slots + it.slot) * (TR * TC * 32);
#pragma unroll
      for (int r = 0; r < TR; ++r)
#pragma unroll
        for (int c2 = 0; c2 < TC / 2; ++c2) {
          const float2 v = unpack2(acc[r][c2]);
          part[(r * TC + 2 * c2) * 32 + lane] = v.x;
          part[(r * TC + 2 * c2 + 1) * 32 + lane] = v.y;
        }
    }
    __syncwarp();
  }
}

// Sums the partial sub-tiles of every split sub-tile in slot order and writes H.
// Grid: (split sub-tiles, pair groups of 16); 256 threads over (cell, lane).
__global__ void __launch_bounds__(256) split_reduce_wide_kernel(GridArgs a) {
  constexpr int TR = kWideRows, TC = kWideCols;
  const int4 sp = a.split_list[blockIdx.x];  // (tile, slot0, nsplit, -)
  const int grp = blockIdx.y;
  const int pg0 = grp * kWidePairs;
  const int np = min(kWidePairs, a.pairs - pg0);
  const int tu = sp.x / a.tiles_v, tv = sp.x - (sp.x / a.tiles_v) * a.tiles_v;
  const int p0 = tu * TR, q0 = tv * TC;
  const float* base = reinterpret_cast<const float*>(a.scratch) +
                      ((size_t)grp * a.n_slots + sp.y) * (TR * TC * 32);
  const size_t MM = (size_t)a.M * a.M;
  for (int i = threadIdx.x; i < TR * TC * 32; i += blockDim.x) {
    const int cell = i >> 5, l = i & 31;
    if ((l >> 1) >= np) continue;
    float sum = 0.f;
    for (int k = 0; k < sp.z; ++k) sum += __ldg(&base[(size_t)k * (TR * TC * 32) + i]);
    const int p = p0 + cell / TC, q = q0 + cell % TC;
    if (p == 0 || q == 0) sum = 0.f;
    float* Hf = reinterpret_cast<float*>(a.H + (size_t)(pg0 + (l >> 1)) * MM);
    Hf[((size_t)p * a.M + q) * 2 + (l & 1)] = sum;
  }
}

// ------------------------------------------------------------------ gridding, 32 pairs per warp
// The gather of grid_wide_kernel (same work list, taps, weights and positions)
// with one complex value per lane: lane p carries (re, im) of pair p of a group
// of kW32Pairs pairs, and each cell's accumulator is one packed (re, im) register
// pair.  Per sample the row products x_r = w(|u - r|) value take one packed
// multiply with the row weight doubled, and each cell adds w(|v - c|) x_r with
// one packed FMA with the column weight doubled.  Per element that is the
// rounding and the summation order of grid_wide_kernel, whose output this
// kernel reproduces bit for bit from the same work list, for twice the pairs
// per instruction and per unit of run and item bookkeeping.
// Per run one lane issues two 1-D bulk copies (cp.async.bulk global -> shared,
// completed on the buffer's mbarrier; no multicast): the run's spectra quads,
// 1 KB each (4 samples x 32 pairs, each pair's 4 samples one 32-byte chunk whose
// halves the spectra kernel swaps for every other group of 4 pairs), and its
// 16-bit table indices.  Each lane then loads its pair's 4 samples of a quad with
// two conflict-free 16-byte loads and applies them from registers.  Copies run
// kW32Bufs - 1 runs ahead (kW32Bufs buffers per warp).
// The lanes expand the run's indices once, through a shared copy of the table
// with a zero entry appended, into doubled weights.  Every wait is bounded: on
// a timeout the warp records it in the error word, waits a second bounded time
// for its copies and returns.  At the end of an item the warp transposes its
// 32 cells x 32 pairs through shared memory, so each store writes whole 64-byte
// row segments of H.

constexpr int kW32Bufs = 2;
constexpr int kW32QuadBytes = 4 * kW32Pairs * 8;                      // 1 KB
constexpr int kW32ValBytes = kWideQuads * kW32QuadBytes;              // a run spans <= 5 quads
constexpr int kW32IdxBytes = (kRunMaxW * kWideRec * 2 + 15) & ~15;    // 384
constexpr int kW32BufBytes = kW32ValBytes + kW32IdxBytes;
constexpr int kW32DblBytes = kRunMaxW * kWideRec * 8;                 // doubled weights of a run
constexpr int kW32RowBytes = (kWideRows * kWideCols + 2) * 8;         // transposition row per pair
constexpr int kW32WarpBytes = kW32Bufs * kW32BufBytes + kW32DblBytes;
static_assert(kW32Pairs * kW32RowBytes <= kW32WarpBytes, "the transposition fits the warp's buffers");
static_assert(kW32WarpBytes % 16 == 0 && kW32BufBytes % 16 == 0 && kW32ValBytes % 16 == 0,
              "bulk-copy destinations are 16-byte aligned");
static_assert(kWideRows == 4 && kWideCols == 8 && kWideRec == 12, "index record layout");

__host__ __device__ constexpr int w32_table_bytes(int ltbl) { return ((ltbl + 2) * 4 + 15) & ~15; }

__device__ __forceinline__ unsigned long long fmul2(unsigned long long a, unsigned long long b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}

// One sample: x_r = w_r * value (packed (re, im)), then every cell of column pairs
// C0..C1 adds w_c * x_r; d: the sample's 6 x 16 bytes of doubled weights, rows
// 0..3 then columns 0..7.
template <int C0, int C1>
__device__ __forceinline__ void w32_apply_sample(unsigned long long (&acc)[kWideRows][kWideCols],
                                                 unsigned long long v, const ulonglong2* d) {
  const ulonglong2 r01 = d[0], r23 = d[1];
  const unsigned long long x[kWideRows] = {fmul2(r01.x, v), fmul2(r01.y, v), fmul2(r23.x, v),
                                           fmul2(r23.y, v)};  // wu * value, (re, im)
#pragma unroll
  for (int c2 = C0; c2 <= C1; ++c2) {
    const ulonglong2 w = d[2 + c2];  // (wv_c, wv_c), (wv_c+1, wv_c+1)
#pragma unroll
    for (int rr = 0; rr < kWideRows; ++rr) {
      ffma2(acc[rr][2 * c2], w.x, x[rr]);
      ffma2(acc[rr][2 * c2 + 1], w.y, x[rr]);
    }
  }
}

// Applies the n samples of one run, at positions t0 .. t0 + n - 1 of its staged
// quads, to the 4 x 8 register tile over column pairs C0..C1.  qa, qb: this
// lane's 16-byte halves with samples (0, 1) and (2, 3) of the run's first quad
// (quads 64 x 16 bytes apart); dbl: the run's doubled weights, 6 x 16 bytes per
// sample.
template <int C0, int C1>
__device__ __forceinline__ void w32_apply_run(unsigned long long (&acc)[kWideRows][kWideCols],
                                              const ulonglong2* qa, const ulonglong2* qb,
                                              const ulonglong2* dbl, int n, int t0) {
  const int tend = t0 + n;
  for (int q = 0; 4 * q < tend; ++q) {
    const ulonglong2 va = qa[q * 64], vb = qb[q * 64];
    const unsigned long long v[4] = {va.x, va.y, vb.x, vb.y};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int t = 4 * q + k;
      if (t >= t0 && t < tend) w32_apply_sample<C0, C1>(acc, v[k], dbl + (t - t0) * 6);
    }
  }
}

// The 16-bit table indices of every (run, sample) of the 16-pair work list, once
// per list: min((int)(|u - r| tblspcg + 0.5), ltbl) for the 4 rows and 8 columns
// of the run's sub-tile where the distance is within L/2, else the zero entry
// ltbl + 1, at the positions grid_wide_kernel's weights use.  Thread r takes run
// r (rinfo[r] = {index block in 16-byte units, sub-tile}) and writes its record
// {first quad (direction * J / 4 + jlo / 4), index block, n | (jlo % 4) << 5 |
// column-pair range << 12}.
__global__ void __launch_bounds__(128) w32_index_kernel(GridArgs a, int n_runs, const int2* rinfo,
                                                        unsigned short* idx, int4* xmeta) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_runs) return;
  const Run run = a.runs[r];
  const int2 ri = rinfo[r];
  const int tu = ri.y / a.tiles_v, tv = ri.y - (ri.y / a.tiles_v) * a.tiles_v;
  const int p0 = tu * kWideRows, q0 = tv * kWideCols;
  const double offu = (double)(a.M / 2 - (p0 & ~(kTile - 1))), subu = (double)(p0 & (kTile - 1));
  const double offv = (double)(a.M / 2 - (q0 & ~(kTile - 1))), subv = (double)(q0 & (kTile - 1));
  const double2 d = a.dir[run.dir];
  const double L2d = a.L2, tsd = a.tblspcg;
  const unsigned short zero = (unsigned short)(a.ltbl + 1);
  unsigned short* w = idx + (size_t)ri.x * 8;
  unsigned cols = 0;
  for (int j = run.jlo; j <= run.jhi; ++j, w += kWideRec) {
    const double u = fma((double)j, d.x, offu) - subu, v = fma((double)j, d.y, offv) - subv;
#pragma unroll
    for (int k = 0; k < kWideRows; ++k) {
      const double dd = fabs(u - (double)k);
      w[k] = dd <= L2d ? (unsigned short)min(table_index64(dd, tsd), a.ltbl) : zero;
    }
#pragma unroll
    for (int k = 0; k < kWideCols; ++k) {
      const double dd = fabs(v - (double)k);
      w[kWideRows + k] = dd <= L2d ? (unsigned short)min(table_index64(dd, tsd), a.ltbl) : zero;
      if (dd <= L2d) cols |= 1u << k;
    }
  }
  const int n = run.jhi - run.jlo + 1;
  const int code = cols ? ((__ffs(cols) - 1) >> 1) * 4 + ((31 - __clz(cols)) >> 1) : kWideNoReach;
  xmeta[r] = make_int4(run.dir * (a.J >> 2) + (run.jlo >> 2), ri.x,
                       n | ((run.jlo & 3) << 5) | (code << 12), 0);
}

__global__ void __launch_bounds__(kWideWarps * 32, kW32MinBlocks) grid_w32_kernel(GridArgs a) {
  extern __shared__ __align__(128) unsigned char smx[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tbl_bytes = w32_table_bytes(a.ltbl);
  float* tbl = reinterpret_cast<float*>(smx);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smx + tbl_bytes) + warp * kW32Bufs;
  unsigned char* wbuf = smx + tbl_bytes + kWideWarps * kW32Bufs * 8 + warp * kW32WarpBytes;
  ulonglong2* dbl = reinterpret_cast<ulonglong2*>(wbuf + kW32Bufs * kW32BufBytes);
  for (int i = threadIdx.x; i <= a.ltbl; i += blockDim.x) tbl[i] = __ldg(&a.wtbl[i]);
  if (threadIdx.x == 0) tbl[a.ltbl + 1] = 0.f;
  if (lane == 0) {
    for (int b = 0; b < kW32Bufs; ++b) mbar_init(&bars[b], 1);
    fence_mbar_init();
  }
  __syncthreads();  // table and barriers ready before any use
  const int groups = (a.pairs + kW32Pairs - 1) / kW32Pairs;
  const unsigned total = (unsigned)a.n_items * (unsigned)groups;
  const size_t group_bytes = (size_t)a.n_ang * 2 * a.J * kW32Pairs * 8;
  // this lane's halves of its pair's 32-byte chunk: samples (0, 1), then (2, 3)
  const int swap16 = ((lane >> 2) & 1) * 16;
  const int off_a = lane * 32 + swap16, off_b = lane * 32 + (16 - swap16);
  const size_t MM = (size_t)a.M * a.M;
  const unsigned char* idxb = reinterpret_cast<const unsigned char*>(a.xidx);
  unsigned phase = 0;     // bit b: parity of bars[b]'s next phase
  unsigned inflight = 0;  // bit b: a copy into buffer b is issued and not yet consumed
  int cur = 0;            // buffer of the next run to consume
  bool failed = false;
  for (;;) {
    unsigned w = 0;
    if (lane == 0) w = atomicAdd(a.queue, 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    if (w >= total) break;
    const int grp = (int)(w / (unsigned)a.n_items);
    const Item it = a.items[w - (unsigned)grp * (unsigned)a.n_items];
    const int pg0 = grp * kW32Pairs;
    const int np = min(kW32Pairs, a.pairs - pg0);
    const int tu = it.tile / a.tiles_v;
    const int tv = it.tile - tu * a.tiles_v;
    const int p0 = tu * kWideRows, q0 = tv * kWideCols;
    const unsigned char* specg = reinterpret_cast<const unsigned char*>(a.spec) + (size_t)grp * group_bytes;
    unsigned long long acc[kWideRows][kWideCols];
#pragma unroll
    for (int r = 0; r < kWideRows; ++r)
#pragma unroll
      for (int c = 0; c < kWideCols; ++c) acc[r][c] = 0ull;
    // run m's quads and indices into buffer b (one lane issues, all lanes track)
    auto issue = [&](const int4& m, int b) {
      if (lane == 0) {
        const unsigned n = (unsigned)m.z & 31u, t0 = ((unsigned)m.z >> 5) & 3u;
        const unsigned vbytes = ((t0 + n + 3u) >> 2) * kW32QuadBytes;
        const unsigned ibytes = (n * (kWideRec * 2) + 15u) & ~15u;
        unsigned char* dst = wbuf + b * kW32BufBytes;
        fence_proxy_async();  // this warp's earlier shared accesses before the copy's writes
        mbar_expect_tx(&bars[b], vbytes + ibytes);
        bulk_g2s(dst, specg + (size_t)m.x * kW32QuadBytes, vbytes, &bars[b]);
        bulk_g2s(dst + kW32ValBytes, idxb + (size_t)m.y * 16, ibytes, &bars[b]);
      }
      inflight |= 1u << b;
    };
    // A sub-tile that no sample reaches has an empty item (rb == re): nothing is
    // read and its cells are written as zeros.
    const int rb = it.run_begin, re = it.run_end;
    int4 mq[kW32Bufs];  // records of runs r .. r + kW32Bufs - 1 (the runs in flight)
#pragma unroll
    for (int k = 0; k < kW32Bufs; ++k) {
      mq[k] = make_int4(0, 0, 0, 0);
      if (rb + k < re) {
        mq[k] = __ldg(&a.xmeta[rb + k]);
        issue(mq[k], cur + k < kW32Bufs ? cur + k : cur + k - kW32Bufs);
      }
    }
    for (int r = rb; r < re; ++r) {
      int4 mn = make_int4(0, 0, 0, 0);
      if (r + kW32Bufs < re) mn = __ldg(&a.xmeta[r + kW32Bufs]);  // read early: issued after run r
      const int4 mA = mq[0];
      const int b = cur;
      const bool ok = mbar_wait(&bars[b], (phase >> b) & 1u);
      if (__any_sync(0xffffffffu, !ok)) {
        failed = true;
        break;
      }
      phase ^= 1u << b;
      inflight &= ~(1u << b);
      const unsigned char* vb = wbuf + b * kW32BufBytes;
      const unsigned short* ib = reinterpret_cast<const unsigned short*>(vb + kW32ValBytes);
      const int n = mA.z & 31;
      float2* d2 = reinterpret_cast<float2*>(dbl);
      {  // up to kRunMaxW * kWideRec = 192 entries, 6 per lane: all index loads, then
         // all table loads, then all stores, so the six chains overlap
        constexpr int kE = (kRunMaxW * kWideRec + 31) / 32;
        const int ne = n * kWideRec;
        unsigned short ix[kE];
#pragma unroll
        for (int e = 0; e < kE; ++e) ix[e] = lane + 32 * e < ne ? ib[lane + 32 * e] : (unsigned short)0;
        float wv[kE];
#pragma unroll
        for (int e = 0; e < kE; ++e) wv[e] = tbl[ix[e]];
#pragma unroll
        for (int e = 0; e < kE; ++e)
          if (lane + 32 * e < ne) d2[lane + 32 * e] = make_float2(wv[e], wv[e]);
      }
      __syncwarp();
      const ulonglong2* qa = reinterpret_cast<const ulonglong2*>(vb + off_a);
      const ulonglong2* qb = reinterpret_cast<const ulonglong2*>(vb + off_b);
      const int t0 = (mA.z >> 5) & 3;
      // the run's samples over the column pairs some sample reaches (the other pairs
      // would only add zero products): runs within columns 0..3 or 4..7 get their own
      // loops, the rest take all four column pairs -- few loop bodies keep the
      // instruction fetch warm
      switch ((mA.z >> 12) & 31) {
        case 0: case 1: case 5: w32_apply_run<0, 1>(acc, qa, qb, dbl, n, t0); break;
        case 10: case 11: case 15: w32_apply_run<2, 3>(acc, qa, qb, dbl, n, t0); break;
        case kWideNoReach: break;  // no sample reaches the sub-tile
        default: w32_apply_run<0, 3>(acc, qa, qb, dbl, n, t0); break;
      }
      __syncwarp();  // buffer b and the weights read by every lane before they are refilled
      if (r + kW32Bufs < re) issue(mn, b);
#pragma unroll
      for (int k = 0; k + 1 < kW32Bufs; ++k) mq[k] = mq[k + 1];
      mq[kW32Bufs - 1] = mn;
      cur = cur + 1 == kW32Bufs ? 0 : cur + 1;
    }
    if (failed) break;
    // no copy is in flight now: the transposition reuses the warp's buffers
    if (it.slot < 0) {
      unsigned char* tr = wbuf;
#pragma unroll
      for (int rr = 0; rr < kWideRows; ++rr)
#pragma unroll
        for (int c2 = 0; c2 < kWideCols / 2; ++c2)
          *reinterpret_cast<ulonglong2*>(tr + lane * kW32RowBytes + (rr * kWideCols + 2 * c2) * 8) =
              make_ulonglong2(acc[rr][2 * c2], acc[rr][2 * c2 + 1]);
      __syncwarp();
      // chunk k * 32 + lane: pair P, row rr, cells 2h and 2h + 1
#pragma unroll 4
      for (int k = 0; k < kW32Pairs * kWideRows * (kWideCols / 2) / 32; ++k) {
        const int ch = k * 32 + lane;
        const int P = ch >> 4, rr = (ch >> 2) & 3, h = ch & 3;
        float4 v = *reinterpret_cast<const float4*>(tr + P * kW32RowBytes + (rr * kWideCols + 2 * h) * 8);
        const int p = p0 + rr, q = q0 + 2 * h;
        if (p == 0) v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (q == 0) v.x = v.y = 0.f;
        if (P < np) *reinterpret_cast<float4*>(a.H + (size_t)(pg0 + P) * MM + (size_t)p * a.M + q) = v;
      }
      __syncwarp();  // the transposition area is read before copies land in it again
    } else {
      // partial sub-tile of a split sub-tile: [cell][lane] complex, summed by split_reduce_w32_kernel
      unsigned long long* part = reinterpret_cast<unsigned long long*>(a.scratch) +
                                 ((size_t)grp * a.n_slots + it.slot) * (kWideRows * kWideCols * 32);
#pragma unroll
      for (int rr = 0; rr < kWideRows; ++rr)
#pragma unroll
        for (int c = 0; c < kWideCols; ++c) part[(rr * kWideCols + c) * 32 + lane] = acc[rr][c];
    }
  }
  if (failed) {
    if (lane == 0) atomicExch(a.err, 1);
    // let the copies in flight land before the CTA's shared memory is released
    for (int b = 0; b < kW32Bufs; ++b)
      if ((inflight >> b) & 1u) mbar_wait(&bars[b], (phase >> b) & 1u);
  }
}

// Sums the partial sub-tiles of every split sub-tile in slot order and writes H.
// Grid: (split sub-tiles, pair groups of 32); 256 threads over (cell, pair).
__global__ void __launch_bounds__(256) split_reduce_w32_kernel(GridArgs a) {
  const int4 sp = a.split_list[blockIdx.x];  // (tile, slot0, nsplit, -)
  const int grp = blockIdx.y;
  const int pg0 = grp * kW32Pairs;
  const int np = min(kW32Pairs, a.pairs - pg0);
  const int tu = sp.x / a.tiles_v, tv = sp.x - (sp.x / a.tiles_v) * a.tiles_v;
  const int p0 = tu * kWideRows, q0 = tv * kWideCols;
  const float2* base = reinterpret_cast<const float2*>(a.scratch) +
                       ((size_t)grp * a.n_slots + sp.y) * (kWideRows * kWideCols * 32);
  const size_t MM = (size_t)a.M * a.M;
  for (int i = threadIdx.x; i < kWideRows * kWideCols * 32; i += blockDim.x) {
    const int cell = i >> 5, l = i & 31;
    if (l >= np) continue;
    float2 sum = make_float2(0.f, 0.f);
    for (int k = 0; k < sp.z; ++k) {
      const float2 v = __ldg(&base[(size_t)k * (kWideRows * kWideCols * 32) + i]);
      sum.x += v.x;
      sum.y += v.y;
    }
    const int p = p0 + cell / kWideCols, q = q0 + cell % kWideCols;
    if (p == 0 || q == 0) sum = make_float2(0.f, 0.f);
    a.H[(size_t)(pg0 + l) * MM + (size_t)p * a.M + q] = sum;
  }
}

// ------------------------------------------------------------------ gridding on the tensor cores
// The gather of grid_wide_kernel as a dense product per work item.  For a
// kTcRows x kTcCols sub-tile (128 cells) and the item's samples s,
//   H[cell][value] = sum_s A[cell][s] B[s][value],
//   A[(r, c)][s] = w(|u_s - r|) w(|v_s - c|)   (zero where a distance exceeds L/2),
//   B[s][2 p + re/im] = spectrum of pair p at sample s,
// so each tcgen05.mma (kind::tf32, M = 128 cells, N = 32 values, K = 8
// samples) applies eight samples to the whole sub-tile for 16 pairs.  The
// accumulator stays in tensor memory for the whole item.  FP32 accuracy comes
// from three TF32 products per step, A_hi B_hi + A_hi B_lo + A_lo B_hi with
// x_hi = x with the low 13 mantissa bits cleared and x_lo = x - x_hi (exact),
// so each term keeps ~22 bits.  Positions, distances and table indices are
// those of grid_kernel (positions relative to the enclosing 32 x 32 tile,
// moved by exact integers).  A CTA of 128 threads handles one item at a time:
// thread t owns cell t of A, one weight, and two values of B per step; the
// operands are double-buffered and each buffer is released by tcgen05.commit
// on its own mbarrier (bounded waits, device error word on timeout).  Items
// list their samples as one flat array of (direction << 13 | j) codes padded
// to a multiple of 8 with j = 0, whose spectrum is zero.  Operands use the
// no-swizzle K-major layout: 8-row x 16-byte core matrices, the two K halves
// 128 bytes apart (LBO), 8-row groups 256 bytes apart (SBO).

constexpr int kTcThreads = 128;
constexpr int kTcStages = 2;                    // operand buffers in flight
constexpr int kTcStage = 2 * 4096 + 2 * 1024;  // A_hi, A_lo (128 x 8), B_hi, B_lo (32 x 8) bytes
constexpr int kTcSmem = 4224 + kTcStages * kTcStage + 16 * 8 * 4 + 8 * 8 * 4 + 8 * kTcStages + 16;

__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
  // start >> 4 [0,14), LBO 128 >> 4 [16,30), SBO 256 >> 4 [32,46), version 1 [46,48), no swizzle
  return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}
// instruction descriptor: D f32, A/B tf32, both K-major, N = 32, M = 128
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(kTcIdesc), "r"(acc));
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

__global__ void __launch_bounds__(kTcThreads) grid_tc_kernel(GridArgs a) {
  constexpr int TR = kTcRows, TC = kTcCols;
  extern __shared__ __align__(128) unsigned char smt[];
  float* s_wtbl = reinterpret_cast<float*>(smt);                  // up to 1028 floats
  unsigned char* stg = smt + 4224;                                // [kTcStages][kTcStage]
  float* s_wu = reinterpret_cast<float*>(stg + kTcStages * kTcStage);  // [TR][8]: row weights
  float* s_wv = s_wu + TR * 8;                                    // [TC][8]
  uint64_t* bar = reinterpret_cast<uint64_t*>(s_wv + TC * 8);     // [kTcStages]
  unsigned* s_misc = reinterpret_cast<unsigned*>(bar + kTcStages);  // [0] tmem base, [1] item
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i <= a.ltbl; i += kTcThreads) s_wtbl[i] = __ldg(&a.wtbl[i]);
  if (tid == 0) {
    for (int b = 0; b < kTcStages; ++b) mbar_init(&bar[b], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(
                     smem_u32(&s_misc[0]))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_misc[0];
  const double L2d = a.L2, tsd = a.tblspcg;
  const int ltbl = a.ltbl;
  const int groups = (a.pairs + kWidePairs - 1) / kWidePairs;
  const unsigned total = (unsigned)a.n_items * (unsigned)groups;
  const size_t per_dir = (size_t)(a.J >> 2) * 64;
  const size_t MM = (size_t)a.M * a.M;
  const unsigned* codes = a.codes;
  // roles: weights (thread -> sample k = tid >> 4, row tid & 15; tid < 64 also
  // sample tid >> 3, column tid & 7); B (value n = tid >> 2, samples kb, kb + 1);
  // A (cell tid = r * TC + c)
  const int wk = tid >> 4, wr = tid & 15, vk = (tid >> 3) & 7, vc = tid & 7;
  const int bn = tid >> 2, bk = (tid & 3) * 2;
  const int bp = bn >> 1, bc = bn & 1;
  unsigned uses[kTcStages] = {};
  int last_buf = -1;
  bool ok = true;
  for (;;) {
    if (tid == 0) s_misc[1] = atomicAdd(a.queue, 1u);
    __syncthreads();
    const unsigned w = s_misc[1];
    if (w >= total) break;
    const int grp = (int)(w / (unsigned)a.n_items);
    const Item it = a.items[w - (unsigned)grp * (unsigned)a.n_items];
    const int pg0 = grp * kWidePairs;
    const int np = min(kWidePairs, a.pairs - pg0);
    const int tu = it.tile / a.tiles_v, tv = it.tile - (it.tile / a.tiles_v) * a.tiles_v;
    const int p0 = tu * TR, q0 = tv * TC;
    // FP64 positions formed as grid_kernel forms them (see grid_wide_kernel)
    const double offu = (double)(a.M / 2 - (p0 & ~(kTile - 1))), offv = (double)(a.M / 2 - (q0 & ~(kTile - 1)));
    const double subu = (double)(p0 & (kTile - 1)), subv = (double)(q0 & (kTile - 1));
    const float* specg = reinterpret_cast<const float*>(a.spec + (size_t)grp * 2 * a.n_ang * per_dir);
    const int nchunk = (it.run_end - it.run_begin) >> 3;
    // a step's codes (this thread's weight samples and its two B samples) are
    // loaded two steps ahead, its B values one step ahead
    struct Codes { unsigned w, v, b0, b1; };
    auto load_codes = [&](int ch) {
      Codes c{0u, 0u, 0u, 0u};
      if (ch < nchunk) {
        const unsigned* cs = codes + it.run_begin + ch * 8;
        c = Codes{__ldg(&cs[wk]), __ldg(&cs[vk]), __ldg(&cs[bk]), __ldg(&cs[bk + 1])};
      }
      return c;
    };
    auto load_val = [&](unsigned code) {
      const int j = code & 8191;
      return __ldg(&specg[(((code >> 13) * per_dir + (j >> 2) * 64 + bp * 4 + (j & 3)) << 1) + bc]);
    };
    Codes cur = load_codes(0), nxt = load_codes(1);
    float b0 = load_val(cur.b0), b1 = load_val(cur.b1);
    double dwx = __ldg(&a.dir[cur.w >> 13].x), dvy = __ldg(&a.dir[cur.v >> 13].y);
    for (int ch = 0; ch < nchunk && ok; ++ch) {
      const int buf = ch % kTcStages;
      const unsigned cw = cur.w, cv = cur.v;
      const double cdx = dwx, cdy = dvy;
      unsigned char* sb = stg + buf * kTcStage;
      // the MMAs that last read this buffer are done
      bool got = true;
      if (uses[buf] > 0) got = mbar_wait(&bar[buf], (uses[buf] - 1) & 1);
      // weights of this step's samples
      {
        const double u = fma((double)(cw & 8191), cdx, offu) - subu;
        const double dd = fabs(u - (double)wr);
        const float wt = s_wtbl[min(table_index64(dd, tsd), ltbl)];
        s_wu[wr * 8 + wk] = dd <= L2d ? wt : 0.f;
        if (tid < 64) {
          const double v = fma((double)(cv & 8191), cdy, offv) - subv;
          const double ddv = fabs(v - (double)vc);
          const float wtv = s_wtbl[min(table_index64(ddv, tsd), ltbl)];
          s_wv[vc * 8 + vk] = ddv <= L2d ? wtv : 0.f;
        }
      }
      // B (K-major: value n's 4 samples per 16-byte row), hi and lo parts
      {
        const int off = (bn >> 3) * 256 + (bk >> 2) * 128 + (bn & 7) * 16 + (bk & 3) * 4;
        const float h0 = tf32_hi(b0), h1 = tf32_hi(b1);
        *reinterpret_cast<float2*>(sb + 8192 + off) = make_float2(h0, h1);
        *reinterpret_cast<float2*>(sb + 9216 + off) = make_float2(b0 - h0, b1 - h1);
      }
      // next step's values (codes loaded a step ago), codes of the step after
      const float nb0 = load_val(nxt.b0), nb1 = load_val(nxt.b1);
      dwx = __ldg(&a.dir[nxt.w >> 13].x);
      dvy = __ldg(&a.dir[nxt.v >> 13].y);
      cur = nxt;
      nxt = load_codes(ch + 2);
      if (__syncthreads_or(!got)) {
        ok = false;
        break;
      }
      // A: cell tid = (r, c), its 8 products, hi and lo parts
      {
        const int r = tid >> 3, c = tid & 7;
        const float4 u0 = *reinterpret_cast<const float4*>(s_wu + r * 8);
        const float4 u1 = *reinterpret_cast<const float4*>(s_wu + r * 8 + 4);
        const float4 v0 = *reinterpret_cast<const float4*>(s_wv + c * 8);
        const float4 v1 = *reinterpret_cast<const float4*>(s_wv + c * 8 + 4);
        const float4 p0v = make_float4(u0.x * v0.x, u0.y * v0.y, u0.z * v0.z, u0.w * v0.w);
        const float4 p1v = make_float4(u1.x * v1.x, u1.y * v1.y, u1.z * v1.z, u1.w * v1.w);
        const float4 h0 = make_float4(tf32_hi(p0v.x), tf32_hi(p0v.y), tf32_hi(p0v.z), tf32_hi(p0v.w));
        const float4 h1 = make_float4(tf32_hi(p1v.x), tf32_hi(p1v.y), tf32_hi(p1v.z), tf32_hi(p1v.w));
        const int off = (tid >> 3) * 256 + (tid & 7) * 16;
        *reinterpret_cast<float4*>(sb + off) = h0;
        *reinterpret_cast<float4*>(sb + off + 128) = h1;
        *reinterpret_cast<float4*>(sb + 4096 + off) =
            make_float4(p0v.x - h0.x, p0v.y - h0.y, p0v.z - h0.z, p0v.w - h0.w);
        *reinterpret_cast<float4*>(sb + 4096 + off + 128) =
            make_float4(p1v.x - h1.x, p1v.y - h1.y, p1v.z - h1.z, p1v.w - h1.w);
      }
      // generic-proxy writes -> visible to the tensor core (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t base = smem_u32(sb);
        const uint64_t a_hi = tc_desc(base), a_lo = tc_desc(base + 4096);
        const uint64_t b_hi = tc_desc(base + 8192), b_lo = tc_desc(base + 9216);
        tc_mma(tmem, a_lo, b_hi, ch > 0 ? 1u : 0u);
        tc_mma(tmem, a_hi, b_lo, 1u);
        tc_mma(tmem, a_hi, b_hi, 1u);
        tc_commit(&bar[buf]);
      }
      uses[buf]++;
      last_buf = buf;
      b0 = nb0;
      b1 = nb1;
    }
    if (!ok) break;
    float v[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = 0.f;
    if (nchunk > 0) {  // a tile that no sample reaches has an empty item: zeros
      // all MMAs of the item are done: the last commit covers the earlier ones
      const bool got = mbar_wait(&bar[last_buf], (uses[last_buf] - 1) & 1);
      if (__syncthreads_or(!got)) {
        ok = false;
        break;
      }
      tc_fence_after();
      unsigned r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
            "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
            "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
            "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
    }
    const int cr = tid >> 3, cc = tid & 7;  // this thread's cell
    if (it.slot < 0) {
      const int p = p0 + cr, q = q0 + cc;
      const bool zero = p == 0 || q == 0;
#pragma unroll
      for (int pp = 0; pp < kWidePairs; ++pp)
        if (pp < np)
          a.H[(size_t)(pg0 + pp) * MM + (size_t)p * a.M + q] =
              zero ? make_float2(0.f, 0.f) : make_float2(v[2 * pp], v[2 * pp + 1]);
    } else {
      float4* part = reinterpret_cast<float4*>(a.scratch) +
                     (((size_t)grp * a.n_slots + it.slot) * (TR * TC) + tid) * 8;
#pragma unroll
      for (int k = 0; k < 8; ++k) part[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    }
    // every thread has read the accumulator before the next item overwrites it
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (!ok) {
    if (tid == 0) atomicExch(a.err, 1);
    // let MMAs in flight finish before the tensor memory is released
    if (last_buf >= 0) mbar_wait(&bar[last_buf], (uses[last_buf] - 1) & 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tmem) : "memory");
}

// Sums the partial sub-tiles of every split sub-tile of grid_tc_kernel in slot order.
__global__ void __launch_bounds__(256) split_reduce_tc_kernel(GridArgs a) {
  constexpr int TR = kTcRows, TC = kTcCols;
  const int4 sp = a.split_list[blockIdx.x];  // (tile, slot0, nsplit, -)
  const int grp = blockIdx.y;
  const int pg0 = grp * kWidePairs;
  const int np = min(kWidePairs, a.pairs - pg0);
  const int tu = sp.x / a.tiles_v, tv = sp.x - (sp.x / a.tiles_v) * a.tiles_v;
  const int p0 = tu * TR, q0 = tv * TC;
  const float* base = reinterpret_cast<const float*>(a.scratch) +
                      ((size_t)grp * a.n_slots + sp.y) * (TR * TC * 32);
  const size_t MM = (size_t)a.M * a.M;
  for (int i = threadIdx.x; i < TR * TC * 32; i += blockDim.x) {
    const int cell = i >> 5, l = i & 31;
    if ((l >> 1) >= np) continue;
    float sum = 0.f;
    for (int k = 0; k < sp.z; ++k) sum += __ldg(&base[(size_t)k * (TR * TC * 32) + i]);
    const int p = p0 + cell / TC, q = q0 + cell % TC;
    if (p == 0 || q == 0) sum = 0.f;
    float* Hf = reinterpret_cast<float*>(a.H + (size_t)(pg0 + (l >> 1)) * MM);
    Hf[((size_t)p * a.M + q) * 2 + (l & 1)] = sum;
  }
}

// ------------------------------------------------------------------ 2-D FFT, first axis (K3)
// G columns of H per CTA: thread t works on column g = t % G (so a warp's
// loads cover G adjacent columns of several rows) and line position t / G.
// Each column's exchange buffer has stride M + 16/G, which keeps the G lines
// on distinct banks.

template <int MAXT, int NT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT) cols_kernel(ColArgs a, int G) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  const int M = NT ? NT : a.M;
  const int nthr = M >> 4;
  const int g = threadIdx.x % G, tid = threadIdx.x / G;
  float2* buf = sm + kTwSlots + g * (M + 16 / G);
  const int q0 = blockIdx.x * G, pair = blockIdx.y;
  load_twiddles(tw, a.tw, M);
  float2* Hp = a.H + (size_t)pair * M * M + q0 + g;
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = Hp[(size_t)(tid + r * nthr) * M];
  __syncthreads();
  fft_line<-1, NT>(v, buf, M, tid, nthr, tw, tw + 64);
  const int Rl = line_last_radix<NT>(M);
#pragma unroll
  for (int idx = 0; idx < 16; ++idx) Hp[(size_t)(tid + nthr * out_index(idx, Rl)) * M] = v[idx];
}

// TMA-fed variant: one thread loads the CTA's G columns x M rows with
// M / box_rows tiled tensor copies (boxes of G complex x box_rows rows, rows
// of the box contiguous in shared memory), the other threads fetch the
// twiddle table meanwhile.  The landing buffer then serves as the FFT
// exchange buffers.  The wait is bounded; a timeout sets *err and the CTA
// returns after giving the copies a second bounded wait.
template <int MAXT, int NT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT)
    cols_tma_kernel(const __grid_constant__ CUtensorMap tmap, ColArgs a, int G, int box_rows) {
  extern __shared__ __align__(128) float2 sm[];
  const int M = NT ? NT : a.M;
  const int nthr = M >> 4;
  float2* tw = sm;
  float2* land = sm + kTwSlots;  // [row][g], G * M values (+ 16 for exchange stride)
  uint64_t* bar = reinterpret_cast<uint64_t*>(land + G * M + 16);
  const int g = threadIdx.x % G, tid = threadIdx.x / G;
  const int q0 = blockIdx.x * G, pair = blockIdx.y;
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();  // the barrier is initialised before any thread polls it
  if (threadIdx.x == 0) {
    mbar_expect_tx(bar, (unsigned)(G * M) * (unsigned)sizeof(float2));
    for (int b = 0; b < M; b += box_rows)
      tma_load_2d(land + (size_t)b * G, &tmap, 2 * q0, pair * M + b, bar);
  }
  load_twiddles(tw, a.tw, M);
  const bool ok = mbar_wait(bar, 0u);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicExch(a.err, 1);
      mbar_wait(bar, 0u);
    }
    __syncthreads();
    return;
  }
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = land[(tid + r * nthr) * G + g];
  __syncthreads();  // inputs read before the landing buffer becomes the exchange buffer
  fft_line<-1, NT>(v, land + g * (M + 16 / G), M, tid, nthr, tw, tw + 64);
  float2* Hp = a.H + (size_t)pair * M * M + q0 + g;
  const int Rl = line_last_radix<NT>(M);
#pragma unroll
  for (int idx = 0; idx < 16; ++idx) Hp[(size_t)(tid + nthr * out_index(idx, Rl)) * M] = v[idx];
}

// The column FFT with persistent CTAs (as many as fit per SM): strip s = blockIdx.x + i gridDim.x
// of G columns lands by TMA in buffer i % 2 while the previous strip is transformed
// from the other, so the copy latency that the one-strip kernel waits out is hidden.
// A buffer is refilled once every thread is done with it (its FFT exchange writes are
// ordered before the copy by a proxy fence and a barrier).  Waits are bounded: on a
// timeout the CTA records the error word, waits (bounded) for its copies in flight and
// leaves.  Same transform, same results as cols_tma_kernel.
template <int MAXT, int NT>
__global__ void __launch_bounds__(MAXT, 512 / MAXT > 0 ? 512 / MAXT : 1)
    cols_ring_kernel(const __grid_constant__ CUtensorMap tmap, ColArgs a, int G, int box_rows) {
  extern __shared__ __align__(128) float2 sm[];
  const int M = NT ? NT : a.M;
  const int nthr = M >> 4;
  const int per_pair = M / G, total = per_pair * a.pairs;
  const int lstride = G * M + 16;  // landing buffer: [row][g], + 16 for the exchange stride
  float2* tw = sm;
  float2* land0 = sm + kTwSlots;
  uint64_t* bar = reinterpret_cast<uint64_t*>(land0 + 2 * lstride);
  const int g = threadIdx.x % G, tid = threadIdx.x / G;
  const unsigned bytes = (unsigned)(G * M) * (unsigned)sizeof(float2);
  auto issue = [&](int s, int b) {  // one thread
    const int pair = s / per_pair, q0 = (s - pair * per_pair) * G;
    mbar_expect_tx(&bar[b], bytes);
    for (int r = 0; r < M; r += box_rows)
      tma_load_2d(land0 + (size_t)b * lstride + (size_t)r * G, &tmap, 2 * q0, pair * M + r, &bar[b]);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();  // the barriers are initialised before any thread polls them
  if (threadIdx.x == 0) {
    if ((int)blockIdx.x < total) issue(blockIdx.x, 0);
    if ((int)(blockIdx.x + gridDim.x) < total) issue(blockIdx.x + gridDim.x, 1);
  }
  load_twiddles(tw, a.tw, M);
  const int Rl = line_last_radix<NT>(M);
  int i = 0;
  for (int s = blockIdx.x; s < total; s += gridDim.x, ++i) {
    const int b = i & 1;
    const unsigned ph = (unsigned)(i >> 1) & 1u;
    float2* land = land0 + (size_t)b * lstride;
    const bool ok = mbar_wait(&bar[b], ph);
    if (__syncthreads_or(!ok)) {
      if (threadIdx.x == 0) {
        atomicExch(a.err, 1);
        mbar_wait(&bar[b], ph);  // this strip's copy
        if (s + (int)gridDim.x < total) mbar_wait(&bar[b ^ 1], (unsigned)((i + 1) >> 1) & 1u);
      }
      __syncthreads();
      return;
    }
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = land[(tid + r * nthr) * G + g];
    __syncthreads();  // inputs read before the landing buffer becomes the exchange buffer
    fft_line<-1, NT>(v, land + g * (M + 16 / G), M, tid, nthr, tw, tw + 64);
    const int pair = s / per_pair, q0 = (s - pair * per_pair) * G;
    float2* Hp = a.H + (size_t)pair * M * M + q0 + g;
#pragma unroll
    for (int idx = 0; idx < 16; ++idx) Hp[(size_t)(tid + nthr * out_index(idx, Rl)) * M] = v[idx];
    // every thread's exchange accesses of this buffer come before the copy that refills it
    fence_proxy_async();
    __syncthreads();
    if (threadIdx.x == 0 && s + 2 * (int)gridDim.x < total) issue(s + 2 * gridDim.x, b);
  }
}

// ------------------------------------------------------------------ second axis + deapod (K4)

template <int MAXT, int NT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT) rows_kernel(RowArgs a) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* buf = sm + kTwSlots;
  const int M = NT ? NT : a.M;
  const int iu = blockIdx.x, pair = blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  load_twiddles(tw, a.tw, M);
  const float2* row = a.H + ((size_t)pair * M + iu) * M;
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = row[tid + r * nthr];
  __syncthreads();
  fft_line<-1, NT>(v, buf, M, tid, nthr, tw, tw + 64);
  // iu = (j - M02) mod M  (gridrec.cu:694-719)
  int j = iu + a.M02;
  if (j >= M) j -= M;
  if (j >= a.M0) return;
  const float wj = __ldg(&a.winv[j]);
  float* o1 = a.out1 + pair * a.pair_stride + (long)j * a.out_stride;
  float* o2 = (2 * pair + 1 < a.n_slices_valid) ? a.out2 + pair * a.pair_stride + (long)j * a.out_stride
                                                : nullptr;
  const int Rl = line_last_radix<NT>(M);
#pragma unroll
  for (int idx = 0; idx < 16; ++idx) {
    const int iv = tid + nthr * out_index(idx, Rl);
    int k = iv + a.M02;
    if (k >= M) k -= M;
    if (k < a.M0) {
      const float c = wj * __ldg(&a.winv[k]);
      o1[k] = c * v[idx].x;
      if (o2) o2[k] = c * v[idx].y;
    }
  }
}

// Self-test of the bounded-wait path: one thread arms an mbarrier that no
// copy or thread ever completes, polls it `limit` times, and records the
// timeout in *err.  No fault, trap or hang is involved.
__global__ void wait_timeout_probe(int* err, int limit) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  fence_mbar_init();
  bool done = false;
  for (int it = 0; it < limit && !done; ++it) done = mbar_try_wait(&bar, 0u);
  *err = done ? 0 : 1;
}

cudaError_t launch_wait_probe(int* err, int limit, cudaStream_t s) {
  wait_timeout_probe<<<1, 32, 0, s>>>(err, limit);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ launchers

static int fft_smem_bytes(int N) { return (kTwSlots + N) * (int)sizeof(float2); }

// Calls CALL(NT) with NT = N for the compiled line lengths, 0 (run-time N) otherwise.
#define GR_DISPATCH_N(N, CALL)  \
  switch (N) {                  \
    case 256: CALL(256); break;   \
    case 512: CALL(512); break;   \
    case 1024: CALL(1024); break; \
    case 2048: CALL(2048); break; \
    case 4096: CALL(4096); break; \
    case 8192: CALL(8192); break; \
    default: CALL(0);             \
  }

// ------------------------------------------------------------------ FBP comparator filter
// OptimizedFBP (gridrec/GPU/filteredbackprojection.cpp:280-300): each projection
// row, gated to (-5, 5), goes through an FFT exp(+i), bin k times lut[k] =
// 1 - sqrt(|k - n/2| / (n/2)), and an unnormalised FFT exp(-i), keeping the real
// part.  lut[k] = lut[n - k] is real, so two rows packed as re + i im are
// filtered together and come apart as the real and imaginary parts.
// Grid: (row pairs, slices); n/16 threads.

__device__ __forceinline__ float fbp_gate(float v) { return (v > -5.f && v < 5.f) ? v : 0.f; }

template <int MAXT, int NT>
__global__ void __launch_bounds__(MAXT, 1024 / MAXT) fbp_filter_kernel(FbpFilterArgs a) {
  extern __shared__ float2 sm[];
  float2* tw = sm;
  float2* buf = sm + kTwSlots;
  const int pr = blockIdx.x, s = blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int n = NT ? NT : a.n;
  load_twiddles(tw, a.tw, n);
  const int ra = 2 * pr, rb = 2 * pr + 1;
  const float* xa = a.sino + ((size_t)s * a.n_ang + ra) * n;
  const float* xb = rb < a.n_ang ? xa + n : nullptr;
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) {
    const int k = tid + r * nthr;
    v[r] = make_float2(fbp_gate(__ldg(&xa[k])), xb ? fbp_gate(__ldg(&xb[k])) : 0.f);
  }
  __syncthreads();
  fft_line<+1, NT>(v, buf, n, tid, nthr, tw, tw + 64);
  const int Rl = line_last_radix<NT>(n);
  __syncthreads();
#pragma unroll
  for (int idx = 0; idx < 16; ++idx) {
    const int k = tid + nthr * out_index(idx, Rl);
    const float w = __ldg(&a.lut[k]);
    buf[swz(k)] = make_float2(v[idx].x * w, v[idx].y * w);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = buf[swz(tid + r * nthr)];
  __syncthreads();
  fft_line<-1, NT>(v, buf, n, tid, nthr, tw, tw + 64);
  float* ya = a.filt + ((size_t)s * a.n_ang + ra) * n;
#pragma unroll
  for (int idx = 0; idx < 16; ++idx) {
    const int k = tid + nthr * out_index(idx, Rl);
    ya[k] = v[idx].x;
    if (xb) ya[n + k] = v[idx].y;
  }
}

cudaError_t launch_fbp_filter(const FbpFilterArgs& a, cudaStream_t s) {
  const int smem = fft_smem_bytes(a.n);
  dim3 grid((a.n_ang + 1) / 2, a.slices);
#define GR_FBP(NT)                                                                   \
  if (a.n <= 4096) fbp_filter_kernel<256, NT><<<grid, a.n / 16, smem, s>>>(a);      \
  else fbp_filter_kernel<(NT > 4096 || NT == 0) ? 512 : 256, NT><<<grid, a.n / 16, smem, s>>>(a)
  GR_DISPATCH_N(a.n, GR_FBP)
#undef GR_FBP
  return cudaGetLastError();
}

// Every FFT kernel instantiation for line length NT (both block-size variants:
// the launchers choose by run-time N for NT = 0 and by the column group width).
template <int NT>
void add_fft_kernels(std::vector<const void*>& f) {
  f.push_back((const void*)spectra_kernel<float, 256, NT>);
  f.push_back((const void*)spectra_kernel<__half, 256, NT>);
  f.push_back((const void*)spectra_kernel<__nv_bfloat16, 256, NT>);
  f.push_back((const void*)spectra_kernel<uint16_t, 256, NT>);
  f.push_back((const void*)spectra_kernel<U16Linear, 256, NT>);
  f.push_back((const void*)spectra_kernel<float, 512, NT>);
  f.push_back((const void*)spectra_kernel<__half, 512, NT>);
  f.push_back((const void*)spectra_kernel<__nv_bfloat16, 512, NT>);
  f.push_back((const void*)spectra_kernel<uint16_t, 512, NT>);
  f.push_back((const void*)spectra_kernel<U16Linear, 512, NT>);
  f.push_back((const void*)cols_kernel<256, NT>);
  f.push_back((const void*)cols_kernel<512, NT>);
  f.push_back((const void*)cols_tma_kernel<256, NT>);
  f.push_back((const void*)cols_tma_kernel<512, NT>);
  f.push_back((const void*)cols_tma_kernel<1024, NT>);
  f.push_back((const void*)cols_ring_kernel<256, NT>);
  f.push_back((const void*)cols_ring_kernel<512, NT>);
  f.push_back((const void*)cols_ring_kernel<1024, NT>);
  f.push_back((const void*)rows_kernel<256, NT>);
  f.push_back((const void*)rows_kernel<512, NT>);
  f.push_back((const void*)fbp_filter_kernel<256, NT>);
  f.push_back((const void*)fbp_filter_kernel<512, NT>);
}

// Allows the dynamic-shared-memory kernels the device's opt-in maximum; called
// once per device at plan creation so that launches need no attribute calls
// (and can be captured in a CUDA graph).
cudaError_t init_kernel_attributes() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  std::vector<const void*> fns;
  add_fft_kernels<0>(fns);
  add_fft_kernels<256>(fns);
  add_fft_kernels<512>(fns);
  add_fft_kernels<1024>(fns);
  add_fft_kernels<2048>(fns);
  add_fft_kernels<4096>(fns);
  add_fft_kernels<8192>(fns);
  fns.push_back((const void*)grid_kernel<3, 2>);
  fns.push_back((const void*)grid_kernel<4, 2>);
  fns.push_back((const void*)grid_kernel<kMaxTaps, 2>);
  fns.push_back((const void*)grid_kernel<3, 1>);
  fns.push_back((const void*)grid_kernel<4, 1>);
  fns.push_back((const void*)grid_kernel<kMaxTaps, 1>);
  fns.push_back((const void*)grid_wide_kernel);
  fns.push_back((const void*)grid_tc_kernel);
  fns.push_back((const void*)grid_w32_kernel);
  for (const void* f : fns) {
    if (e != cudaSuccess) break;
    // the opt-in limit covers static and dynamic shared memory together
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, f);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               optin - (int)fa.sharedSizeBytes);
  }
  return e;
}

cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t s) {
  dim3 grid((a.J + 255) / 256, a.pairs);
  phase_kernel<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <typename T>
static cudaError_t launch_spectra_t(const SpectraArgs& a, cudaStream_t s) {
  const int smem = fft_smem_bytes(a.pdim);
  const dim3 grid = a.wide ? dim3(a.pairs, a.n_ang) : dim3(a.n_ang, a.pairs);
#define GR_SPEC(NT)                                                                  \
  if (a.pdim <= 4096) spectra_kernel<T, 256, NT><<<grid, a.pdim / 16, smem, s>>>(a); \
  else spectra_kernel<T, (NT > 4096 || NT == 0) ? 512 : 256, NT><<<grid, a.pdim / 16, smem, s>>>(a)
  GR_DISPATCH_N(a.pdim, GR_SPEC)
#undef GR_SPEC
  return cudaGetLastError();
}

cudaError_t launch_spectra(const SpectraArgs& a, gr_dtype dt, cudaStream_t s) {
  switch (dt) {
    case GR_DTYPE_F32: return launch_spectra_t<float>(a, s);
    case GR_DTYPE_F16: return launch_spectra_t<__half>(a, s);
    case GR_DTYPE_BF16: return launch_spectra_t<__nv_bfloat16>(a, s);
    case GR_DTYPE_U16_RAW: return launch_spectra_t<uint16_t>(a, s);
    case GR_DTYPE_U16_LINEAR: return launch_spectra_t<U16Linear>(a, s);
  }
  return cudaErrorInvalidValue;
}

static int grid_smem_bytes(int pg) {
  return 257 * (int)sizeof(float4) + kGridWarps * (kTile * kTileStride + kRunMax) * pg * (int)sizeof(float2);
}

template <int PG>
static cudaError_t launch_grid_pg(const GridArgs& a, int ntaps, cudaStream_t s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int smem = grid_smem_bytes(PG);
  int per_sm = 0;
  if (ntaps <= 3) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_kernel<3, PG>, kGridWarps * 32, smem);
  } else if (ntaps <= 4) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_kernel<4, PG>, kGridWarps * 32, smem);
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_kernel<kMaxTaps, PG>, kGridWarps * 32,
                                                  smem);
  }
  const long groups = (a.pairs + PG - 1) / PG;
  const long want = ((long)a.n_items * groups + kGridWarps - 1) / kGridWarps;
  const int blocks = (int)std::min<long>(want, (long)std::max(per_sm, 1) * sms);
  if (ntaps <= 3) grid_kernel<3, PG><<<blocks, kGridWarps * 32, smem, s>>>(a);
  else if (ntaps <= 4) grid_kernel<4, PG><<<blocks, kGridWarps * 32, smem, s>>>(a);
  else grid_kernel<kMaxTaps, PG><<<blocks, kGridWarps * 32, smem, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || a.n_split_tiles == 0) return e;
  dim3 rgrid(a.n_split_tiles, (unsigned)groups);
  split_reduce_kernel<PG><<<rgrid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

// A chunk of one pair runs the one-pair variant; larger chunks grid two pairs per warp.
cudaError_t launch_grid(const GridArgs& a, int ntaps, cudaStream_t s) {
  if (a.n_items == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  return a.pairs == 1 ? launch_grid_pg<1>(a, ntaps, s) : launch_grid_pg<2>(a, ntaps, s);
}

static int grid_wide_smem_bytes() {
  return kWideWarps * kWideWarpFloats * (int)sizeof(float);
}

cudaError_t launch_wide_weights(const GridArgs& a, int n_runs, float* wts, int2* meta,
                                cudaStream_t s) {
  if (n_runs == 0) return cudaSuccess;
  wide_weights_kernel<<<(n_runs + 127) / 128, 128, 0, s>>>(a, n_runs, wts, meta);
  return cudaGetLastError();
}

cudaError_t launch_grid_wide(const GridArgs& a, cudaStream_t s) {
  if (a.n_items == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int smem = grid_wide_smem_bytes();
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_wide_kernel, kWideWarps * 32, smem);
  const long groups = (a.pairs + kWidePairs - 1) / kWidePairs;
  const long want = ((long)a.n_items * groups + kWideWarps - 1) / kWideWarps;
  const int blocks = (int)std::min<long>(want, (long)std::max(per_sm, 1) * sms);
  grid_wide_kernel<<<blocks, kWideWarps * 32, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess || a.n_split_tiles == 0) return e;
  dim3 rgrid(a.n_split_tiles, (unsigned)groups);
  split_reduce_wide_kernel<<<rgrid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

static int grid_w32_smem_bytes(int ltbl) {
  return w32_table_bytes(ltbl) + kWideWarps * kW32Bufs * 8 + kWideWarps * kW32WarpBytes;
}

cudaError_t launch_w32_index(const GridArgs& a, int n_runs, const int2* rinfo,
                             unsigned short* idx, int4* xmeta, cudaStream_t s) {
  if (n_runs == 0) return cudaSuccess;
  w32_index_kernel<<<(n_runs + 127) / 128, 128, 0, s>>>(a, n_runs, rinfo, idx, xmeta);
  return cudaGetLastError();
}

cudaError_t launch_grid_w32(const GridArgs& a, cudaStream_t s) {
  if (a.n_items == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int smem = grid_w32_smem_bytes(a.ltbl);
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, grid_w32_kernel, kWideWarps * 32, smem);
  const long groups = (a.pairs + kW32Pairs - 1) / kW32Pairs;
  const long want = ((long)a.n_items * groups + kWideWarps - 1) / kWideWarps;
  const int blocks = (int)std::min<long>(want, (long)std::max(per_sm, 1) * sms);
  grid_w32_kernel<<<blocks, kWideWarps * 32, smem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess || a.n_split_tiles == 0) return e;
  dim3 rgrid(a.n_split_tiles, (unsigned)groups);
  split_reduce_w32_kernel<<<rgrid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_grid_tc(const GridArgs& a, cudaStream_t s) {
  if (a.n_items == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // CTAs per SM from its shared memory (1 KB reserved per CTA) and tensor
  // memory (32 of the 512 columns each); 128 threads and 56 registers allow more
  int smem_sm = 0;
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  int per_sm = std::min(smem_sm / (kTcSmem + 1024), 16);
  per_sm = std::max(per_sm, 1);
  const long groups = (a.pairs + kWidePairs - 1) / kWidePairs;
  const long want = (long)a.n_items * groups;
  const int blocks = (int)std::min<long>(want, (long)per_sm * sms);
  grid_tc_kernel<<<blocks, kTcThreads, kTcSmem, s>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess || a.n_split_tiles == 0) return e;
  dim3 rgrid(a.n_split_tiles, (unsigned)groups);
  split_reduce_tc_kernel<<<rgrid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

int cols_group(int M) {
  int g = 8192 / M;  // G * M / 16 <= 512 threads; G = 4 (32-byte rows) at M = 2048
  return g < 1 ? 1 : (g > 8 ? 8 : g);
}

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    else
      cudaGetLastError();
  });
  return fn;
}

cudaError_t launch_cols(const ColArgs& a, cudaStream_t s) {
  const int G = a.G > 0 ? a.G : cols_group(a.M);
  const int threads = G * (a.M / 16);
  PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
  if (a.err && encode && G >= 2 && a.M >= 16 && ((uintptr_t)a.H % 16) == 0) {
    // H as a 2-D float array: 2*M floats per row, pairs*M rows
    CUtensorMap map;
    const int box_rows = a.M < 256 ? a.M : 256;
    cuuint64_t dims[2] = {(cuuint64_t)2 * a.M, (cuuint64_t)a.pairs * a.M};
    cuuint64_t strides[1] = {(cuuint64_t)2 * a.M * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)(2 * G), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)a.H, dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    int optin = 0, dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int ring_smem = (kTwSlots + 2 * (G * a.M + 16)) * (int)sizeof(float2) + 2 * (int)sizeof(uint64_t);
    if (r == CUDA_SUCCESS && a.ring && ring_smem <= optin) {
      const int total = (a.M / G) * a.pairs;
      // persistent: as many CTAs as fit on the SMs at once
#define GR_COLR(NT)                                                                              \
  {                                                                                              \
    const void* fn = threads <= 256 ? (const void*)cols_ring_kernel<256, NT>                     \
                     : threads <= 512 ? (const void*)cols_ring_kernel<512, NT>                   \
                                      : (const void*)cols_ring_kernel<1024, NT>;                 \
    int per_sm = 0;                                                                              \
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, ring_smem);              \
    const int blocks = std::min(total, std::max(per_sm, 1) * std::max(sms, 1));                  \
    if (threads <= 256) cols_ring_kernel<256, NT><<<blocks, threads, ring_smem, s>>>(map, a, G, box_rows); \
    else if (threads <= 512) cols_ring_kernel<512, NT><<<blocks, threads, ring_smem, s>>>(map, a, G, box_rows); \
    else cols_ring_kernel<1024, NT><<<blocks, threads, ring_smem, s>>>(map, a, G, box_rows);      \
  }
      GR_DISPATCH_N(a.M, GR_COLR)
#undef GR_COLR
      return cudaGetLastError();
    }
    if (r == CUDA_SUCCESS) {
      const int smem = (kTwSlots + G * a.M + 16) * (int)sizeof(float2) + (int)sizeof(uint64_t);
      dim3 grid(a.M / G, a.pairs);
#define GR_COLT(NT)                                                                      \
  if (threads <= 256) cols_tma_kernel<256, NT><<<grid, threads, smem, s>>>(map, a, G, box_rows); \
  else if (threads <= 512) cols_tma_kernel<512, NT><<<grid, threads, smem, s>>>(map, a, G, box_rows); \
  else cols_tma_kernel<1024, NT><<<grid, threads, smem, s>>>(map, a, G, box_rows)
      GR_DISPATCH_N(a.M, GR_COLT)
#undef GR_COLT
      return cudaGetLastError();
    }
  }
  // the plain kernel takes at most 512 threads: narrower column groups if needed
  int Gp = G;
  while (Gp > 1 && Gp * (a.M / 16) > 512) Gp >>= 1;
  const int smem = (kTwSlots + Gp * (a.M + 16 / Gp)) * (int)sizeof(float2);
  dim3 grid(a.M / Gp, a.pairs);
#define GR_COL(NT)                                                                         \
  if (Gp * (a.M / 16) <= 256) cols_kernel<256, NT><<<grid, Gp * (a.M / 16), smem, s>>>(a, Gp); \
  else cols_kernel<512, NT><<<grid, Gp * (a.M / 16), smem, s>>>(a, Gp)
  GR_DISPATCH_N(a.M, GR_COL)
#undef GR_COL
  return cudaGetLastError();
}

cudaError_t launch_rows(const RowArgs& a, cudaStream_t s) {
  const int smem = fft_smem_bytes(a.M);
  dim3 grid(a.M, a.pairs);
#define GR_ROW(NT)                                                                   \
  if (a.M <= 4096) rows_kernel<256, NT><<<grid, a.M / 16, smem, s>>>(a);            \
  else rows_kernel<(NT > 4096 || NT == 0) ? 512 : 256, NT><<<grid, a.M / 16, smem, s>>>(a)
  GR_DISPATCH_N(a.M, GR_ROW)
#undef GR_ROW
  return cudaGetLastError();
}

}  // namespace gr
