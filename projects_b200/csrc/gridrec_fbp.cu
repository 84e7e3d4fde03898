// FBP comparator: the reference's OptimizedFBP reconstruction class
// (gridrec/GPU/filteredbackprojection.cpp:190-330, a ReconAlgorithm like GridRec)
// on the device.  Row filter: fbp_filter_kernel (gridrec_kernels.cu).  Here:
// pixel-driven backprojection and the C ABI.
//
// Backprojection of pixel (x, y) of the n x n image (row y), as the reference:
//   x = (col - n/2) / (n/2), y = (row - n/2) / (n/2), r = x cos_a + y sin_a,
//   image += filtered[a][(int)((r + 1) n/2)] for -1 <= r < 1, angles in order,
// in float with the reference's operation order (no contraction), so the sample
// chosen for every (pixel, angle) is the reference's (except an index that
// rounds to n, which is clamped to n - 1 instead of reading outside the row).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "gr_internal.h"

namespace gr {
namespace {

constexpr int kBpX = 32, kBpY = 8;

__global__ void __launch_bounds__(kBpX * kBpY) fbp_backproject_kernel(const float* filt,
                                                                     const float2* cs,
                                                                     float* recon, int n,
                                                                     int n_ang) {
  extern __shared__ float2 s_cs[];
  const int tid = threadIdx.y * kBpX + threadIdx.x;
  for (int i = tid; i < n_ang; i += kBpX * kBpY) s_cs[i] = cs[i];
  __syncthreads();
  const int xi = blockIdx.x * kBpX + threadIdx.x, yi = blockIdx.y * kBpY + threadIdx.y;
  const int s = blockIdx.z;
  if (xi >= n || yi >= n) return;
  const float h = (float)n / 2.0f;
  const float x = __fdiv_rn(__fsub_rn((float)xi, h), h);
  const float y = __fdiv_rn(__fsub_rn((float)yi, h), h);
  const float* f = filt + (size_t)s * n_ang * n;
  float acc = 0.f;
  for (int a = 0; a < n_ang; ++a) {
    const float2 c = s_cs[a];  // (cos, sin)
    const float r = __fadd_rn(__fmul_rn(x, c.x), __fmul_rn(y, c.y));
    if (r >= -1.f && r < 1.f) {
      // r just below 1 can round (r + 1) n/2 up to n; the reference then reads
      // the next row (or past its buffer), here the last sample of the row
      const int k = min((int)__fmul_rn(__fadd_rn(r, 1.f), h), n - 1);
      acc = __fadd_rn(acc, __ldg(&f[(size_t)a * n + k]));
    }
  }
  recon[((size_t)s * n + yi) * n + xi] = acc;
}

}  // namespace
}  // namespace gr

struct gr_fbp {
  int device = 0, n = 0, n_ang = 0, max_slices = 1;
  float* d_lut = nullptr;
  float2* d_tw = nullptr;
  float2* d_cs = nullptr;
  float* d_filt = nullptr;
};

using namespace gr;

extern "C" {

int gr_fbp_destroy(gr_fbp* f) {
  if (!f) return GR_OK;
  DeviceGuard g(f->device);
  cudaFree(f->d_lut);
  cudaFree(f->d_tw);
  cudaFree(f->d_cs);
  cudaFree(f->d_filt);
  delete f;
  return GR_OK;
}

int gr_fbp_create(int n_det, int n_ang, const float* theta_deg, int max_slices, int device,
                  gr_fbp** out) {
  if (!out || !theta_deg) return fail(GR_ERR_ARG, "fbp: null argument");
  *out = nullptr;
  if (n_det < 16 || n_det > 8192 || (n_det & (n_det - 1)) || n_ang < 1 || max_slices < 1)
    return fail(GR_ERR_ARG, "fbp: n_det a power of two in [16, 8192], n_ang >= 1, max_slices >= 1");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
    return fail(GR_ERR_ARG, "fbp: device %d not available", device);
  DeviceGuard g(device);
  const int n = n_det;
  // Tables as the reference computes them: the degree list to radians as
  // (theta * PI) / 180 stored in float (PI of gridrec/GPU/fft.h:5), sin/cos of
  // that float; the filter 1 - sqrt(|t|) with t = (k - n/2) / (n/2) in float.
  const double kPiRef = 3.1415926535897932385;
  std::vector<float2> cs(n_ang);
  for (int a = 0; a < n_ang; ++a) {
    const float th = (float)((theta_deg[a] * kPiRef) / 180.0);
    cs[a] = make_float2((float)std::cos((double)th), (float)std::sin((double)th));
  }
  std::vector<float> lut(n);
  for (int k = 0; k < n; ++k) {
    const float t = (float)(k - (float)(n / 2)) / ((float)(n / 2));
    lut[k] = (float)(1 - std::sqrt(std::fabs((double)t)));
  }
  const int nhi = std::max(1, n / 64);
  std::vector<float2> tw(64 + nhi);
  for (int e = 0; e < 64; ++e) {
    const double a = 2.0 * M_PI * e / n;
    tw[e] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  for (int f = 0; f < nhi; ++f) {
    const double a = 2.0 * M_PI * 64.0 * f / n;
    tw[64 + f] = make_float2((float)std::cos(a), (float)std::sin(a));
  }
  gr_fbp* p = new gr_fbp;
  p->device = device;
  p->n = n;
  p->n_ang = n_ang;
  p->max_slices = max_slices;
  cudaError_t e = cudaMalloc(&p->d_lut, n * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_tw, tw.size() * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_cs, n_ang * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_filt, (size_t)max_slices * n_ang * n * sizeof(float));
  if (e == cudaSuccess) e = cudaMemcpy(p->d_lut, lut.data(), n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(p->d_cs, cs.data(), n_ang * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = init_kernel_attributes();
  if (e != cudaSuccess) {
    gr_fbp_destroy(p);
    cudaGetLastError();
    return fail(GR_ERR_NOMEM, "fbp create: %s", cudaGetErrorString(e));
  }
  *out = p;
  return GR_OK;
}

int gr_fbp_reconstruct(gr_fbp* f, const float* sinos, int n_slices, float* recons, void* stream) {
  if (!f || !sinos || !recons || n_slices < 1) return fail(GR_ERR_ARG, "fbp: bad arguments");
  DeviceGuard g(f->device);
  cudaStream_t st = (cudaStream_t)stream;
  const int n = f->n;
  const size_t slice_in = (size_t)f->n_ang * n, slice_out = (size_t)n * n;
  const int smem_bp = f->n_ang * (int)sizeof(float2);
  if (smem_bp > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(fbp_backproject_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bp);
    if (e != cudaSuccess) return fail(GR_ERR_UNSUPPORTED, "fbp: %d angles: %s", f->n_ang,
                                      cudaGetErrorString(e));
  }
  for (int s0 = 0; s0 < n_slices; s0 += f->max_slices) {
    const int ns = std::min(f->max_slices, n_slices - s0);
    FbpFilterArgs fa{sinos + s0 * slice_in, f->d_filt, f->d_lut, f->d_tw, n, f->n_ang, ns};
    cudaError_t e = launch_fbp_filter(fa, st);
    if (e != cudaSuccess) return fail(GR_ERR_CUDA, "fbp filter: %s", cudaGetErrorString(e));
    dim3 grid((n + kBpX - 1) / kBpX, (n + kBpY - 1) / kBpY, ns);
    fbp_backproject_kernel<<<grid, dim3(kBpX, kBpY), smem_bp, st>>>(
        f->d_filt, f->d_cs, recons + s0 * slice_out, n, f->n_ang);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(GR_ERR_CUDA, "fbp backprojection: %s", cudaGetErrorString(e));
  }
  return GR_OK;
}

}  // extern "C"
