// Test-infrastructure driver around the reference's own CPU OptimizedFBP class
// (gridrec/GPU/filteredbackprojection.cpp:190-330), compiled where the sources
// lie by oracle/build_ref.sh into oracle/_ref/libfbp_ref.so.  It drives the
// ReconAlgorithm setter API as the reference's callers do (setSinogramDimensions,
// setThetaList, init, setSinoAndReconBuffers(1, ..), reconstruct, destroy).
#include <cstring>
#include <vector>

#include "filteredbackprojection.h"

char msg[256];  // recon_algorithm.h:98 declares it; the reference's driver defines it

extern "C" {

// One slice: sino n_ang x n_det, recon n_det x n_det (row = y).  theta in
// degrees; copied, because OptimizedFBP::init converts the list in place.
void ref_optimized_fbp(int n_det, int n_ang, const float* theta_deg, float* sino, float* recon) {
  std::vector<float> th(theta_deg, theta_deg + n_ang);
  OptimizedFBP f;
  f.setSinogramDimensions(n_det, n_ang);
  f.setThetaList(th.data(), n_ang);
  f.init();
  f.setSinoAndReconBuffers(1, sino, recon);
  f.reconstruct();
  f.destroy();
}

}  // extern "C"
