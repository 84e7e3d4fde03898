// Test-infrastructure driver around the reference's GridrecCPP 5.2 C API
// (gridrec/GridrecCPP/Gridrec5.2/grid.h:89-91: recon_init / do_recon /
// recon_free on the globals G1, G2, S1, S2).
//
// Compiled with the GridrecCPP sources where they lie (grid.cpp, fftgr.cpp,
// filters.cpp, pswf.cpp, grid_math.cpp; not grid_io.cpp, which needs netCDF)
// by oracle/build_ref.sh into oracle/_ref/.  Unlike the GridRec class, this API
// honours an explicit rotation centre, oversampling ratio and filter name, so it
// pins the centre phase ramp and the sampl > 1 sizing.  Test use only.
#include <cstring>
#include <vector>

#include "grid.h"

// Globals that GridrecCPP's own main/grid_io would define.
int verbose = 0;
FILE* fshift = nullptr;
int global_index = 0;

extern "C" {

// Reconstructs one slice pair.  sino1/sino2 are n_ang x n_det (row = angle).
// out1/out2 receive the M0 x M0 image with row stride out_stride (which must
// be >= M0; pass out_stride = 0 to query M0 only).  Returns M0.
int refb_gridrec_pair(int n_det, int n_ang, float* theta_deg, float center,
                      const char* filter_name, float C, float sampl, int ltbl,
                      float* sino1, float* sino2, float* out1, float* out2,
                      int out_stride, int geom, float roi_size, float pixel_size, float x0,
                      float y0) {
  pswf_struct* pswf = nullptr;
  get_pswf(C, &pswf);
  grid_struct gp;
  std::memset(&gp, 0, sizeof(gp));
  gp.pswf = pswf;
  gp.sampl = sampl;
  gp.MaxPixSiz = pixel_size;
  gp.R = roi_size;
  gp.X0 = x0;
  gp.Y0 = y0;
  std::strncpy(gp.fname, filter_name, sizeof(gp.fname) - 1);
  gp.filter = get_filter(gp.fname);
  gp.ltbl = ltbl;
  sg_struct sg;
  sg.n_ang = n_ang;
  sg.n_det = n_det;
  sg.geom = geom;  // 0: the angle list; 1 / 2: uniform over pi / 2 pi
  sg.angles = theta_deg;
  sg.center = center;
  long im = 0;
  recon_init(&gp, &sg, &im);
  if (out_stride <= 0) {
    recon_free();
    return (int)im;
  }
  std::vector<float*> g1(n_ang), g2(n_ang), s1(im), s2(im);
  for (int a = 0; a < n_ang; ++a) {
    g1[a] = sino1 + (size_t)a * n_det;
    g2[a] = sino2 + (size_t)a * n_det;
  }
  for (long r = 0; r < im; ++r) {
    s1[r] = out1 + (size_t)r * out_stride;
    s2[r] = out2 + (size_t)r * out_stride;
  }
  G1 = g1.data();
  G2 = g2.data();
  S1 = s1.data();
  S2 = s2.data();
  imgsiz = im;
  do_recon();
  recon_free();
  return (int)im;
}

}  // extern "C"
