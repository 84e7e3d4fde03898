// Test infrastructure: C wrappers around the reference's own slice-pipeline
// code, compiled by build_ref.sh from line ranges of the reference sources
// that it writes to a temporary directory (nothing of the reference is kept in
// this repository):
//   ring_ref.inc      RingCorrectionSinogram   gridrec/GPU/tomo_recon.cpp:3905-3972
//   entropy_ref.inc   entropy()                find_shift/src/main/find_shift.cpp:2078-2115
//   shiftpad_ref.inc  shift + half-padding     gridrec/GPU/tomo_recon.cpp:3708-3807
//                     (body of GridRecSlices; expects the locals declared below)
//   xcorr_ref.inc     data_interp + cross_correlation (brute-force axis search)
//                                              find_shift/src/main/find_shift.cpp:1975-2076
#include <cmath>
#include <cstdlib>
#include <vector>
using namespace std;  // the reference translation units see std names unqualified

#include "ring_ref.inc"
#include "entropy_ref.inc"
#include "xcorr_ref.inc"

extern "C" {

// 20 rounds, as the reference hard-codes.
void ref_ring_removal(float* data, int n_det, int n_ang, float ring_coeff) {
  vector<float> mv(n_ang), ms(n_det), lp(n_det);
  RingCorrectionSinogram(data, ring_coeff, n_det, n_ang, mv.data(), ms.data(), lp.data());
}

float ref_entropy(float* data, float vmin, float vmax, int nbins, int xm, int ym) {
  return entropy(data, vmin, vmax, nbins, xm, ym);
}

// sino1, sino2: n_ang x n_det; sinogram: 2 x n_ang x (2 n_det), the layout of
// GridRecSlices' padded pair.
void ref_shift_pad(const float* sino1, const float* sino2, int n_det, int n_ang, float xoffset,
                   float* sinogram) {
  struct {
    float* h_input_data;
  } plan_s;
  vector<float> in(2 * (size_t)n_ang * n_det);
  for (int a = 0; a < n_ang; ++a)
    for (int d = 0; d < n_det; ++d) {
      in[((size_t)a * 2 + 0) * n_det + d] = sino1[(size_t)a * n_det + d];
      in[((size_t)a * 2 + 1) * n_det + d] = sino2[(size_t)a * n_det + d];
    }
  plan_s.h_input_data = in.data();
  auto* plan = &plan_s;
  const unsigned int num_ray = n_det, num_proj = n_ang, num_elevation = 2;
  const int num_ray_half_padding = 2 * n_det;
  const int offset_pad = num_ray / 2;
  const int iter = 0;
  int i, j, k;
  for (i = 0; i < 2 * num_ray_half_padding * n_ang; i++) sinogram[i] = 0.0f;
#include "shiftpad_ref.inc"
  (void)i;
}

// One translation of the brute-force search, as find_shift.cpp:1333-1351 runs it
// (template statistics as :902-973).
double ref_xcorr_score(double* templ, double* match, int width, int height, int x0, int x1, int y0,
                       int y1, double tx, double ty) {
  const int rw = x1 - x0 + 1, rh = y1 - y0 + 1;
  const long area = (long)rw * rh;
  double tavg = 0.0, trms = 0.0;
  for (long i = 0; i < area; ++i) tavg += templ[i];
  tavg /= area;
  for (long i = 0; i < area; ++i) trms += (templ[i] - tavg) * (templ[i] - tavg);
  trms = sqrt(trms);
  vector<double> roi(area);
  double mavg = 0.0, res = 0.0;
  data_interp(match, roi.data(), &mavg, tx, ty, x0, x1, y0, y1, width, height);
  cross_correlation(roi.data(), templ, tavg, mavg, &res, x0, x1, y0, y1, trms);
  return res;
}

}  // extern "C"
