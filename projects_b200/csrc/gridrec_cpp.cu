// The GridrecCPP 5.2 C calling sequence (include/gridrec_cpp_b200.h) on a gridrec
// plan: recon_init / do_recon / recon_free over the caller's row-pointer globals
// G1, G2, S1, S2 (gridrec/GridrecCPP/Gridrec5.2/grid.h:73-91, grid.cpp:54-434),
// with get_pswf and get_filter (Gridrec5.2/pswf.cpp:36-47, filters.cpp:10-48).
// Host code only; the reconstruction is gr_reconstruct_pair_host on the plan.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#include "gr_internal.h"
#include "gridrec_b200.h"
#include "gridrec_cpp_b200.h"

extern "C" {
float **G1 = nullptr, **G2 = nullptr;
float **S1 = nullptr, **S2 = nullptr;
long imgsiz = 0;
}

namespace gr {
namespace {

// get_pswf's table: the plan database rounded to the struct's floats; a pointer
// into it maps back to the database entry (no rounding in the plan's tables)
struct PswfTable {
  pswf_struct rec[5];
  PswfTable() {
    const double Cs[5] = {4.0, 4.2, 5.0, 6.0, 7.0};
    for (int i = 0; i < 5; ++i) {
      const Pswf* p = find_pswf(Cs[i]);
      std::memset(&rec[i], 0, sizeof(pswf_struct));
      rec[i].C = (float)p->C;
      rec[i].nt = p->nt;
      rec[i].lmbda = (float)p->lmbda;
      for (int k = 0; k <= p->nt / 2 && k < 11; ++k) rec[i].coefs[k] = (float)p->coefs[k];
    }
  }
};
PswfTable& pswf_table() {
  static PswfTable t;
  return t;
}

// get_filter's functions: the filter formulas of the plan, x = j / pdim
float cpp_shlo(float x) { return (float)filter_value(GR_FILTER_SHEPP_LOGAN, x); }
float cpp_hann(float x) { return (float)filter_value(GR_FILTER_HANN, x); }
float cpp_hamm(float x) { return (float)filter_value(GR_FILTER_HAMMING, x); }
float cpp_ramp(float x) { return (float)filter_value(GR_FILTER_RAMP, x); }

struct CppState {
  int device = 0;
  int status = GR_OK;
  gr_plan* plan = nullptr;
  int n_det = 0, n_ang = 0;
  long m0 = 0;
  float* h_in = nullptr;   // pinned: the pair's sinograms when G1/G2 rows are not contiguous
  float* h_out = nullptr;  // pinned: the pair's images when S1/S2 rows are not evenly strided
};
CppState g_cpp;

void release() {
  if (g_cpp.plan) gr_plan_destroy(g_cpp.plan);
  if (g_cpp.h_in) cudaFreeHost(g_cpp.h_in);
  if (g_cpp.h_out) cudaFreeHost(g_cpp.h_out);
  g_cpp.plan = nullptr;
  g_cpp.h_in = g_cpp.h_out = nullptr;
}

// Row stride (in floats) of rows[0..n) when they are evenly spaced, ascending, with
// stride >= min_stride; else 0.
long even_stride(float** rows, long n, long min_stride) {
  if (n == 1) return min_stride;
  const uintptr_t d = (uintptr_t)rows[1] - (uintptr_t)rows[0];
  if ((uintptr_t)rows[1] < (uintptr_t)rows[0] || d % sizeof(float)) return 0;
  const long s = (long)(d / sizeof(float));
  if (s < min_stride) return 0;
  for (long i = 2; i < n; ++i)
    if ((uintptr_t)rows[i] - (uintptr_t)rows[i - 1] != d) return 0;
  return s;
}

}  // namespace
}  // namespace gr

extern "C" {

void get_pswf(float C, pswf_struct** P) {
  using namespace gr;
  if (!P) {
    g_cpp.status = fail(GR_ERR_ARG, "get_pswf: null argument");
    return;
  }
  *P = nullptr;
  for (pswf_struct& r : pswf_table().rec)
    if (std::fabs(C - r.C) <= 0.01f) {
      *P = &r;
      g_cpp.status = GR_OK;
      return;
    }
  g_cpp.status = fail(GR_ERR_PSWF, "Prolate parameter, C = %f not in data base", C);
}

float (*get_filter(char* name))(float) {
  using namespace gr;
  struct Entry {
    const char* name;
    float (*fp)(float);
  };
  static const Entry table[] = {{"shlo", cpp_shlo}, {"shepp", cpp_shlo}, {"hann", cpp_hann},
                                {"hamm", cpp_hamm}, {"hamming", cpp_hamm}, {"ramp", cpp_ramp},
                                {"ramlak", cpp_ramp}};
  if (name)
    for (const Entry& e : table)
      if (!std::strcmp(name, e.name)) return e.fp;
  if (name) std::strcpy(name, "shlo");  // the default choice, name overwritten as there
  return cpp_shlo;
}

void recon_init(grid_struct* GP, sg_struct* SGP, long* im_size) {
  using namespace gr;
  release();
  if (!GP || !SGP || !GP->pswf || !GP->filter) {
    g_cpp.status = fail(GR_ERR_ARG, "recon_init: grid_struct with pswf and filter, and sg_struct required");
    return;
  }
  gr_params p;
  gr_params_default(&p, SGP->n_det, SGP->n_ang, SGP->angles);
  p.center = SGP->center;
  p.geom = SGP->geom;
  p.sampl = GP->sampl;
  p.pixel_size = GP->MaxPixSiz;
  p.roi_size = GP->R;
  p.roi_x0 = GP->X0;
  p.roi_y0 = GP->Y0;
  p.ltbl = (int)GP->ltbl;
  p.pswf_c = GP->pswf->C;
  p.device = g_cpp.device;
  p.max_pairs = 1;
  // a filter of get_filter's maps to its code; any other function is sampled
  float (*fn)(float) = nullptr;
  if (GP->filter == cpp_shlo) p.filter = GR_FILTER_SHEPP_LOGAN;
  else if (GP->filter == cpp_hann) p.filter = GR_FILTER_HANN;
  else if (GP->filter == cpp_hamm) p.filter = GR_FILTER_HAMMING;
  else if (GP->filter == cpp_ramp) p.filter = GR_FILTER_RAMP;
  else fn = GP->filter;
  // a PSWF record of get_pswf's maps to the database entry; any other is used as given
  Pswf own{};
  const Pswf* pw = nullptr;
  const pswf_struct* tb = pswf_table().rec;
  if (!(GP->pswf >= tb && GP->pswf < tb + 5)) {
    own.C = GP->pswf->C;
    own.lmbda = GP->pswf->lmbda;
    own.nt = GP->pswf->nt;
    for (int k = 0; k <= own.nt / 2 && k < 11; ++k) own.coefs[k] = GP->pswf->coefs[k];
    pw = &own;
  }
  gr_plan* plan = nullptr;
  int rc = plan_create_ex(&p, pw, fn, &plan);
  if (rc) {
    g_cpp.status = rc;
    return;
  }
  int M = 0, M0 = 0;
  gr_plan_sizes(plan, nullptr, &M, &M0, nullptr, nullptr);
  g_cpp.plan = plan;
  g_cpp.n_det = SGP->n_det;
  g_cpp.n_ang = SGP->n_ang;
  g_cpp.m0 = M0;
  GP->sampl = (float)M / M0;  // as recon_init adjusts it (grid.cpp:119)
  imgsiz = M0;
  if (im_size) *im_size = M0;
  g_cpp.status = GR_OK;
}

void do_recon(void) {
  using namespace gr;
  if (!g_cpp.plan) {
    g_cpp.status = fail(GR_ERR_ARG, "do_recon: recon_init has not succeeded");
    return;
  }
  if (!G1 || !S1) {
    g_cpp.status = fail(GR_ERR_ARG, "do_recon: G1 and S1 must point to the pair's rows");
    return;
  }
  DeviceGuard guard(g_cpp.device);
  const long n_det = g_cpp.n_det, n_ang = g_cpp.n_ang, m0 = g_cpp.m0;
  const size_t slice = (size_t)n_ang * n_det;
  // inputs: contiguous rows go to the GPU directly, others through a pinned buffer
  const float* in1 = G1[0];
  const float* in2 = G2 ? G2[0] : nullptr;
  const bool g1_flat = even_stride(G1, n_ang, n_det) == n_det;
  const bool g2_flat = !G2 || even_stride(G2, n_ang, n_det) == n_det;
  if ((!g1_flat || !g2_flat) && !g_cpp.h_in &&
      cudaMallocHost((void**)&g_cpp.h_in, 2 * slice * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    g_cpp.h_in = nullptr;
    g_cpp.status = fail(GR_ERR_NOMEM, "do_recon: pinned staging of %zu bytes", 2 * slice * 4);
    return;
  }
  if (!g1_flat) {
    for (long n = 0; n < n_ang; ++n) std::memcpy(g_cpp.h_in + n * n_det, G1[n], n_det * sizeof(float));
    in1 = g_cpp.h_in;
  }
  if (!g2_flat) {
    for (long n = 0; n < n_ang; ++n)
      std::memcpy(g_cpp.h_in + slice + n * n_det, G2[n], n_det * sizeof(float));
    in2 = g_cpp.h_in + slice;
  }
  // outputs: evenly strided rows (stride >= M0) are written in place, others staged
  const long s1 = even_stride(S1, m0, m0), s2 = S2 ? even_stride(S2, m0, m0) : 0;
  if (s1 && (!S2 || s2 == s1)) {
    g_cpp.status = gr_reconstruct_pair_host(g_cpp.plan, in1, in2, S1[0], S2 ? S2[0] : nullptr, s1,
                                            nullptr);
    return;
  }
  if (!g_cpp.h_out &&
      cudaMallocHost((void**)&g_cpp.h_out, 2 * (size_t)m0 * m0 * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    g_cpp.h_out = nullptr;
    g_cpp.status = fail(GR_ERR_NOMEM, "do_recon: pinned staging of the images");
    return;
  }
  float* o2 = g_cpp.h_out + (size_t)m0 * m0;
  g_cpp.status = gr_reconstruct_pair_host(g_cpp.plan, in1, in2, g_cpp.h_out, S2 ? o2 : nullptr, m0,
                                          nullptr);
  if (g_cpp.status != GR_OK) return;
  for (long j = 0; j < m0; ++j) {
    std::memcpy(S1[j], g_cpp.h_out + j * m0, m0 * sizeof(float));
    if (S2) std::memcpy(S2[j], o2 + j * m0, m0 * sizeof(float));
  }
}

void recon_free(void) {
  gr::release();
  gr::g_cpp.status = GR_OK;
}

int gr_gridrec_cpp_status(void) { return gr::g_cpp.status; }

void gr_gridrec_cpp_set_device(int device) { gr::g_cpp.device = device; }

}  // extern "C"
