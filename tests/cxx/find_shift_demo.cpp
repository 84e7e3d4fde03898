// Exercises include/gridrec_b200.hpp the way find_shift uses its GridRec
// (find_shift/src/main/find_shift.cpp:1661-1666, 1836-1841; setCenterShift before
// init, find_shift/src/main/gridrec.cu:229, 809-813) and the ReconAlgorithm
// getters (gridrec/GPU/recon_algorithm.h:59-72).  Reads two float32 sinograms
// (n_ang x n_det) from argv[1]; writes the two n_det x n_det reconstructions to
// argv[2].  Usage: find_shift_demo in.bin out.bin n_det n_ang filter shift
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gridrec_b200.hpp"

int main(int argc, char** argv) {
  if (argc < 7) {
    std::fprintf(stderr, "usage: %s in.bin out.bin n_det n_ang filter shift\n", argv[0]);
    return 2;
  }
  const int n_det = std::atoi(argv[3]), n_ang = std::atoi(argv[4]), filter = std::atoi(argv[5]);
  const float shift = (float)std::atof(argv[6]);
  std::vector<float> sino(2 * (size_t)n_ang * n_det), recon(2 * (size_t)n_det * n_det, 0.f);
  std::vector<float> theta(n_ang);
  for (int i = 0; i < n_ang; ++i) theta[i] = 180.f * i / n_ang;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f || std::fread(sino.data(), sizeof(float), sino.size(), f) != sino.size()) return 3;
  std::fclose(f);
  gridrec_b200::GridRec g;
  g.setSinogramDimensions(n_det, n_ang);
  g.setThetaList(theta.data(), n_ang);
  g.setFilter(filter);
  g.setGPUDeviceID(0);
  g.setCenterShift(shift);
  // the ReconAlgorithm getters report what was set
  if (g.numberOfSinogramsNeeded() != 2 || g.numberOfReconstructions() != 2 ||
      g.getSinogramXDimension() != n_det || g.getSinogramYDimension() != n_ang ||
      g.getThetaListSize() != n_ang || g.getThetaList() != theta.data() || g.getFilter() != filter ||
      g.getGPUDeviceID() != 0 || g.getCenter() != (float)(n_det / 2) + shift)
    return 7;
  g.init();
  if (g.lastStatus() != GR_OK) {
    std::fprintf(stderr, "init: %s\n", g.lastError());
    return 4;
  }
  g.setSinoAndReconBuffers(1, sino.data(), recon.data());
  g.setSinoAndReconBuffers(2, sino.data() + (size_t)n_ang * n_det, recon.data() + (size_t)n_det * n_det);
  g.reconstruct();
  if (g.lastStatus() != GR_OK) {
    std::fprintf(stderr, "reconstruct: %s\n", g.lastError());
    return 5;
  }
  g.destroy();
  f = std::fopen(argv[2], "wb");
  std::fwrite(recon.data(), sizeof(float), recon.size(), f);
  std::fclose(f);
  return 0;
}
