// Test-infrastructure driver around the reference's own CPU GridRec class.
//
// This file is compiled together with the reference sources where they lie
// (gridrec/GPU/gridrec.cu as C++, recon_algorithm.cpp, fft_nr.cpp) by
// oracle/build_ref.sh; the result goes to oracle/_ref/ and is used only by the
// tests and by the CPU-baseline arm of bench.py, never by the product path.
//
// It drives the reference's public setter API exactly as the reference's own
// caller does (gridrec/GPU/tomo_recon.cpp:1701-1706 and :3846-3852):
//   setSinogramDimensions, setThetaList, setFilter, init,
//   setSinoAndReconBuffers(1,..), setSinoAndReconBuffers(2,..), reconstruct, destroy.
//
// REAL is float for the reference build and double for the FP64 build (the same
// source run through `sed s/float/double/` on temporary copies).
#include <chrono>
#include <cstring>

#include "gridrec.h"

#ifndef REAL
#define REAL float
#endif

// recon_algorithm.h:98 declares this global; the reference's driver defines it.
char msg[256];

namespace {
double now_s() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
}  // namespace

extern "C" {

// Reconstructs one slice pair with the reference GridRec (centre fixed to
// n_det/2 by GridRec::init, gridrec/GPU/gridrec.cu:227).  out1/out2 are
// n_det x n_det buffers (row stride n_det, gridrec.cu:196-197); the reference
// fills the leading M0 x M0 block.  Returns M0 (imgsiz).  *t_recon receives the
// wall time of reconstruct() alone; *t_total includes init and destroy.
int ref_gridrec_pair(int n_det, int n_ang, REAL* theta_deg, int filter,
                     REAL* sino1, REAL* sino2, REAL* out1, REAL* out2,
                     double* t_recon, double* t_total) {
  double t0 = now_s();
  GridRec g;
  g.setSinogramDimensions(n_det, n_ang);
  g.setThetaList(theta_deg, n_ang);
  g.setFilter(filter);
  g.init();
  g.setSinoAndReconBuffers(1, sino1, out1);
  g.setSinoAndReconBuffers(2, sino2, out2);
  double t1 = now_s();
  g.reconstruct();
  double t2 = now_s();
  g.destroy();
  double t3 = now_s();
  if (t_recon) *t_recon = t2 - t1;
  if (t_total) *t_total = t3 - t0;
  // M0 for the GridRec defaults (sampl=1): M = next_pow2(n_det), M0 = M - 1.
  long M = 1, itmp = n_det - 1;
  while (itmp) { M <<= 1; itmp >>= 1; }
  return (int)(M - 1);
}

// Reconstructs `n_pairs` consecutive pairs with one GridRec instance (init
// once, then setSinoAndReconBuffers + reconstruct per pair) -- the loop of
// GridRecSlices (gridrec/GPU/tomo_recon.cpp:3702-3852).  Sinogram pair k is
// sinos[(2k) * n_ang * n_det] and sinos[(2k+1) * n_ang * n_det]; outputs are
// n_det x n_det each.  Returns the wall time of the reconstruct() calls.
double ref_gridrec_pairs(int n_det, int n_ang, REAL* theta_deg, int filter,
                         int n_pairs, REAL* sinos, REAL* outs) {
  GridRec g;
  g.setSinogramDimensions(n_det, n_ang);
  g.setThetaList(theta_deg, n_ang);
  g.setFilter(filter);
  g.init();
  const size_t sino_sz = (size_t)n_ang * n_det;
  const size_t out_sz = (size_t)n_det * n_det;
  double t = 0.0;
  for (int k = 0; k < n_pairs; ++k) {
    g.setSinoAndReconBuffers(1, sinos + (2 * k) * sino_sz, outs + (2 * k) * out_sz);
    g.setSinoAndReconBuffers(2, sinos + (2 * k + 1) * sino_sz, outs + (2 * k + 1) * out_sz);
    double t0 = now_s();
    g.reconstruct();
    t += now_s() - t0;
  }
  g.destroy();
  return t;
}

}  // extern "C"
