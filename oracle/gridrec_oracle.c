/*
 * gridrec_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, float64 restatement of the reference's gridrec algorithm
 * (gridrec/GPU/gridrec.cu, class GridRec, CPU path with USE_GRIDREC_GPU
 * undefined; identical to GridrecCPP 5.2 grid.cpp at the same parameters).
 * It is the checker for the CUDA path: only tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py load it.  The product never calls it.
 *
 * Written from the mathematics of the reference, not from its code: the FFTs
 * here are this file's own radix-2 transforms with exactly computed twiddles
 * (the reference uses Numerical Recipes four1/fourn, gridrec/GPU/fft_nr.cpp,
 * which is not reproduced).  Each step cites the reference lines it restates.
 *
 * Conventions (all from the reference):
 *   pdim = next power of two >= n_det                    gridrec.cu:243-249
 *   M    = next power of two >= sampl*n_det              gridrec.cu:251-260
 *   M02  = floor(M/2/sampl - 0.5), M0 = 2*M02 + 1         gridrec.cu:262-263
 *   sampl <- M/M0, L = 2*C*sampl/pi, scale = sampl*n/pdim gridrec.cu:265-268
 *   1-D FFT of the packed pair with exp(+2 pi i jk/N)     gridrec.cu:521 (isign=+1)
 *   2-D DFT of H with exp(-2 pi i ...)                    gridrec.cu:641-646 (isign=-1)
 *   output S[j][k], j along the first (U, cos) grid axis  gridrec.cu:691-719
 *
 * Extension beyond the reference (documented): the two slices of a pair may
 * have different rotation centres.  With P_j = f_j (e1_j + e2_j)/2 and
 * Q_j = f_j (e1_j - e2_j)/2, where e_k,j = exp(-2 pi i j c_k / pdim) and f_j
 * the filter*normalisation, the filtered samples are
 *   C1_j = P_j F_j + Q_j conj(F_{pdim-j}),  C2_j = conj(P_j) F_{pdim-j} + conj(Q_j) conj(F_j)
 * which reduces to the reference's C1 = filphase F_j, C2 = conj(filphase) F_{pdim-j}
 * (gridrec.cu:527-538) when c1 == c2.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "gridrec_oracle.h"

#define ORC_PI 3.14159265358979323846

/* ---- PSWF database: the numerical table of gridrec/GPU/gridrec.cu:21-114
 * (== GridrecCPP pswf.cpp:5-34).  C, eigenvalue, Legendre degree, even-order
 * Legendre expansion coefficients. */
typedef struct {
  double C, lmbda;
  int nt;
  double coefs[11];
} orc_pswf;

static const orc_pswf ORC_PSWF_DB[5] = {
    {4.0, 0.99588549, 16,
     {0.5239891E+01, -0.5308499E+01, 0.1184591E+01, -0.1230763E-00, 0.7371623E-02,
      -0.2864074E-03, 0.7789983E-05, -0.1564700E-06, 0.2414647E-08, 0.0, 0.0}},
    {4.2, 0.99657887, 16,
     {0.6062942E+01, -0.6450252E+01, 0.1551875E+01, -0.1755960E-01, 0.1150712E-01,
      -0.4903653E-03, 0.1464986E-04, -0.3235110E-06, 0.5492141E-08, 0.0, 0.0}},
    {5.0, 0.99935241, 18,
     {0.1115509E+02, -0.1384861E+02, 0.4289811E+01, -0.6514303E-00, 0.5844993E-01,
      -0.3447736E-02, 0.1435066E-03, -0.4433680E-05, 0.1056040E-06, -0.1997173E-08,
      0.0}},
    {6.0, 0.9990188, 18,
     {0.2495593E+02, -0.3531124E+02, 0.1383722E+02, -0.2799028E+01, 0.3437217E-00,
      -0.2818024E-01, 0.1645842E-02, -0.7179160E-04, 0.2424510E-05, -0.6520875E-07,
      0.0}},
    {7.0, 0.99998546, 20,
     {0.5767616E+02, -0.8931343E+02, 0.4167596E+02, -0.1053599E+02, 0.1662374E+01,
      -0.1780527E-00, 0.1372983E-01, -0.7963169E-03, 0.3593372E-04, -0.1295941E-05,
      0.3817796E-07}},
};

/* get_pswf: first entry with |C - C_db| <= 0.01 (gridrec.cu:906-922). */
static const orc_pswf* orc_get_pswf(double C) {
  for (int i = 0; i < 5; ++i)
    if (fabs(C - ORC_PSWF_DB[i].C) <= 0.01) return &ORC_PSWF_DB[i];
  return NULL;
}

/* Sum_k coefs[k] P_{2k}(x) by the three-term Legendre recurrence
 * (gridrec.cu:861-902). */
static double orc_legendre(int n, const double* coefs, double x) {
  double y = coefs[0], penult = 1.0, last = x;
  int k = 1, even = 1;
  for (int j = 2; j <= n; ++j) {
    double nw = (x * (2 * j - 1) * last - (j - 1) * penult) / j;
    if (even) {
      y += nw * coefs[k];
      k++;
      even = 0;
    } else {
      even = 1;
    }
    penult = last;
    last = nw;
  }
  return y;
}

/* Filter::filterData (recon_algorithm.cpp:36-73): codes 1..4 are
 * Shepp-Logan, Hann, Hamming, ramp; any other code returns x unchanged. */
static double orc_filter(int code, double x) {
  switch (code) {
    case 1: return fabs(sin(ORC_PI * x) / ORC_PI);
    case 2: return fabs(x) * 0.5 * (1.0 + cos(2 * ORC_PI * x));
    case 3: return fabs(x) * (0.54 + 0.46 * cos(2 * ORC_PI * x));
    case 4: return fabs(x);
    default: return x;
  }
}

int orc_sizes(const orc_params* p, orc_sizes_t* s) {
  if (p->n_det < 1 || p->n_ang < 1 || p->ltbl < 1 || !(p->sampl > 0)) return -1;
  const orc_pswf* pw = orc_get_pswf(p->C);
  if (!pw) return -2;
  long pdim = 1, itmp = p->n_det - 1;
  while (itmp) { pdim <<= 1; itmp >>= 1; }              /* gridrec.cu:243-249 */
  const double R = p->roi_size > 0 ? p->roi_size : 1.0;
  const double pix = p->pixel_size > 0 ? p->pixel_size : 1.0;
  double D0 = R * p->n_det;                               /* grid.cpp:95-96 */
  double D1 = p->sampl * D0;
  long M = 1;
  itmp = (long)(D1 / pix - 1);                            /* grid.cpp:100-106 */
  while (itmp) { M <<= 1; itmp >>= 1; }                   /* gridrec.cu:254-260 */
  long M02 = (long)floor((double)(M / 2) / p->sampl - 0.5);  /* gridrec.cu:262 */
  if (M02 < 0) M02 = 0;
  s->pdim = pdim;
  s->M = M;
  s->M02 = M02;
  s->M0 = 2 * M02 + 1;
  s->sampl = (double)M / (double)s->M0;                   /* gridrec.cu:265 */
  s->L = 2 * pw->C * s->sampl / ORC_PI;                   /* gridrec.cu:267 */
  s->scale = s->sampl * D0 / pdim;                        /* gridrec.cu:268 */
  s->C = pw->C;
  s->lmbda = pw->lmbda;
  return 0;
}

/* pswf_su (gridrec.cu:807-857): wtbl[0..ltbl] and winv[0..M0-1]. */
int orc_tables(const orc_params* p, double* wtbl, double* winv) {
  orc_sizes_t s;
  int rc = orc_sizes(p, &s);
  if (rc) return rc;
  const orc_pswf* pw = orc_get_pswf(p->C);
  long ltbl = p->ltbl;
  double polyz = orc_legendre(pw->nt, pw->coefs, 0.0);
  wtbl[0] = 1.0;
  for (long i = 1; i <= ltbl; ++i)
    wtbl[i] = orc_legendre(pw->nt, pw->coefs, (double)i / ltbl) / polyz;
  if (winv) {
    long linv = s.M02;
    double fac = (double)ltbl / (linv + 0.5);
    double norm = sqrt(ORC_PI / 2 / pw->C / pw->lmbda) / s.sampl;
    winv[linv] = norm / wtbl[0];
    for (long i = 1; i <= linv; ++i) {
      norm = -norm;                                       /* checkerboard sign */
      winv[linv + i] = winv[linv - i] = norm / wtbl[(long)(i * fac + 0.5)];
    }
  }
  return 0;
}

/* In-place radix-2 complex FFT of length n (power of two), interleaved
 * (re, im) doubles, out[k] = sum_t in[t] exp(sign * 2 pi i k t / n), with
 * a stride between consecutive elements (in complex units). */
static void orc_fft(double* x, long n, long stride, int sign) {
  for (long i = 1, j = 0; i < n; ++i) {                   /* bit reversal */
    long bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double* a = x + 2 * i * stride;
      double* b = x + 2 * j * stride;
      double t0 = a[0], t1 = a[1];
      a[0] = b[0]; a[1] = b[1];
      b[0] = t0; b[1] = t1;
    }
  }
  for (long len = 2; len <= n; len <<= 1) {
    long h = len >> 1;
    for (long k = 0; k < h; ++k) {
      double ang = sign * 2.0 * ORC_PI * (double)k / (double)len;
      double wr = cos(ang), wi = sin(ang);
      for (long i = k; i < n; i += len) {
        double* a = x + 2 * i * stride;
        double* b = x + 2 * (i + h) * stride;
        double br = b[0] * wr - b[1] * wi;
        double bi = b[0] * wi + b[1] * wr;
        b[0] = a[0] - br; b[1] = a[1] - bi;
        a[0] += br; a[1] += bi;
      }
    }
  }
}

void orc_fft1d(double* x, long n, int sign) { orc_fft(x, n, 1, sign); }

/* Filtered spectra of one pair (phase 1 steps 1-3, gridrec.cu:500-538):
 * spec[(n*2 + h)*J + j] (complex, J = pdim/2) holds C1_j (h=0) and C2_j (h=1)
 * for j = 1..pdim/2-1; entry j = 0 is zero. */
int orc_spectra(const orc_params* p, const double* sino1, const double* sino2,
                double* spec) {
  orc_sizes_t s;
  int rc = orc_sizes(p, &s);
  if (rc) return rc;
  long pdim = s.pdim, J = pdim / 2;
  double* cp = (double*)calloc(2 * pdim, sizeof(double));
  double* P = (double*)malloc(2 * J * sizeof(double));
  double* Q = (double*)malloc(2 * J * sizeof(double));
  if (!cp || !P || !Q) { free(cp); free(P); free(Q); return -3; }
  /* filphase_su (gridrec.cu:774-803) generalised to two centres */
  double norm = ORC_PI / pdim / p->n_ang;
  for (long j = 0; j < J; ++j) {
    double f = orc_filter(p->filter, (double)j / pdim) * norm;
    double a1 = -2 * ORC_PI * j * p->center1 / pdim;
    double a2 = -2 * ORC_PI * j * p->center2 / pdim;
    P[2 * j] = f * 0.5 * (cos(a1) + cos(a2));
    P[2 * j + 1] = f * 0.5 * (sin(a1) + sin(a2));
    Q[2 * j] = f * 0.5 * (cos(a1) - cos(a2));
    Q[2 * j + 1] = f * 0.5 * (sin(a1) - sin(a2));
  }
  for (long n = 0; n < p->n_ang; ++n) {
    memset(cp, 0, 2 * pdim * sizeof(double));
    for (long k = 0; k < p->n_det; ++k) {                  /* gridrec.cu:507-519 */
      cp[2 * k] = sino1[n * p->n_det + k];
      cp[2 * k + 1] = sino2[n * p->n_det + k];
    }
    orc_fft(cp, pdim, 1, +1);                              /* gridrec.cu:521 */
    double* o1 = spec + 2 * ((n * 2 + 0) * J);
    double* o2 = spec + 2 * ((n * 2 + 1) * J);
    o1[0] = o1[1] = o2[0] = o2[1] = 0.0;
    for (long j = 1; j < J; ++j) {                         /* gridrec.cu:523-538 */
      double Fr = cp[2 * j], Fi = cp[2 * j + 1];
      double Gr = cp[2 * (pdim - j)], Gi = cp[2 * (pdim - j) + 1];
      double Pr = P[2 * j], Pi = P[2 * j + 1], Qr = Q[2 * j], Qi = Q[2 * j + 1];
      /* C1 = P F + Q conj(G) */
      o1[2 * j] = Pr * Fr - Pi * Fi + Qr * Gr + Qi * Gi;
      o1[2 * j + 1] = Pr * Fi + Pi * Fr - Qr * Gi + Qi * Gr;
      /* C2 = conj(P) G + conj(Q) conj(F) */
      o2[2 * j] = Pr * Gr + Pi * Gi + Qr * Fr - Qi * Fi;
      o2[2 * j + 1] = Pr * Gi - Pi * Gr - Qr * Fi - Qi * Fr;
    }
  }
  free(cp); free(P); free(Q);
  return 0;
}

/* Convolution gridding (phase 1 step 4, gridrec.cu:540-576) of the filtered
 * spectra onto H (M x M complex, natural order, H[iu*M + iv]). */
int orc_grid(const orc_params* p, const double* theta_deg, const double* spec,
             double* H) {
  orc_sizes_t s;
  int rc = orc_sizes(p, &s);
  if (rc) return rc;
  long M = s.M, J = s.pdim / 2, M2 = M / 2;
  double* wtbl = (double*)malloc((p->ltbl + 1) * sizeof(double));
  if (!wtbl) return -3;
  orc_tables(p, wtbl, NULL);
  double L2 = s.L / 2, tblspcg = 2 * p->ltbl / s.L;
  memset(H, 0, 2 * M * M * sizeof(double));
  double wv[64];
  for (long n = 0; n < p->n_ang; ++n) {
    double th = theta_deg[n] * (ORC_PI / 180.0);           /* trig_su, gridrec.cu:737-742 */
    double sn = sin(th), cs = cos(th);
    const double* c1 = spec + 2 * ((n * 2 + 0) * J);
    const double* c2 = spec + 2 * ((n * 2 + 1) * J);
    /* ROI offset (GridrecCPP grid.cpp:237, 258-268): C1 times exp(-i j off), C2 times
     * its conjugate, off = (X0 cos + Y0 sin) pi */
    const double off = (p->x0 * cs + p->y0 * sn) * ORC_PI;
    for (long j = 1; j < J; ++j) {
      const double pr = cos(j * off), pi = -sin(j * off);
      const double a1r = c1[2 * j] * pr - c1[2 * j + 1] * pi, a1i = c1[2 * j] * pi + c1[2 * j + 1] * pr;
      const double a2r = c2[2 * j] * pr + c2[2 * j + 1] * pi, a2i = -c2[2 * j] * pi + c2[2 * j + 1] * pr;
      double r = s.scale * j;
      double U = r * cs + M2, V = r * sn + M2;
      long iul = (long)ceil(U - L2), iuh = (long)floor(U + L2);
      long ivl = (long)ceil(V - L2), ivh = (long)floor(V + L2);
      if (iul < 1) iul = 1;
      if (iuh >= M) iuh = M - 1;
      if (ivl < 1) ivl = 1;
      if (ivh >= M) ivh = M - 1;
      for (long iv = ivl, k = 0; iv <= ivh; ++iv, ++k)
        wv[k] = wtbl[(long)(fabs(V - iv) * tblspcg + 0.5)];
      for (long iu = iul; iu <= iuh; ++iu) {
        double wu = wtbl[(long)(fabs(U - iu) * tblspcg + 0.5)];
        for (long iv = ivl, k = 0; iv <= ivh; ++iv, ++k) {
          double w = wu * wv[k];
          double* h1 = H + 2 * (iu * M + iv);
          double* h2 = H + 2 * ((M - iu) * M + (M - iv));
          h1[0] += w * a1r;
          h1[1] += w * a1i;
          h2[0] += w * a2r;
          h2[1] += w * a2i;
        }
      }
    }
  }
  free(wtbl);
  return 0;
}

/* Phase 2 (gridrec.cu:641-646): unnormalised 2-D DFT, exp(-2 pi i ...). */
void orc_fft2d(double* H, long M) {
  for (long r = 0; r < M; ++r) orc_fft(H + 2 * r * M, M, 1, -1);
  for (long c = 0; c < M; ++c) orc_fft(H + 2 * c, M, M, -1);
}

/* Phase 3 (gridrec.cu:691-719): S[j][k] = winv[j] winv[k] H[(j-M02) mod M][(k-M02) mod M]. */
int orc_deapod(const orc_params* p, const double* H, double* out1, double* out2,
               long out_stride) {
  orc_sizes_t s;
  int rc = orc_sizes(p, &s);
  if (rc) return rc;
  double* wtbl = (double*)malloc((p->ltbl + 1) * sizeof(double));
  double* winv = (double*)malloc(s.M0 * sizeof(double));
  if (!wtbl || !winv) { free(wtbl); free(winv); return -3; }
  orc_tables(p, wtbl, winv);
  long M = s.M;
  for (long j = 0; j < s.M0; ++j) {
    long iu = (j - s.M02 + M) % M;
    for (long k = 0; k < s.M0; ++k) {
      long iv = (k - s.M02 + M) % M;
      double c = winv[j] * winv[k];
      out1[j * out_stride + k] = c * H[2 * (iu * M + iv)];
      out2[j * out_stride + k] = c * H[2 * (iu * M + iv) + 1];
    }
  }
  free(wtbl); free(winv);
  return 0;
}

int orc_gridrec_pair(const orc_params* p, const double* theta_deg,
                     const double* sino1, const double* sino2, double* out1,
                     double* out2, long out_stride) {
  orc_sizes_t s;
  int rc = orc_sizes(p, &s);
  if (rc) return rc;
  if (out_stride < s.M0) return -4;
  long J = s.pdim / 2;
  double* spec = (double*)malloc(2 * (size_t)p->n_ang * 2 * J * sizeof(double));
  double* H = (double*)malloc(2 * (size_t)s.M * s.M * sizeof(double));
  if (!spec || !H) { free(spec); free(H); return -3; }
  rc = orc_spectra(p, sino1, sino2, spec);
  if (!rc) rc = orc_grid(p, theta_deg, spec, H);
  if (!rc) { orc_fft2d(H, s.M); rc = orc_deapod(p, H, out1, out2, out_stride); }
  free(spec); free(H);
  return rc;
}

/* ---------------------------------------------------------------- slice pipeline
 * Restatements of the steps around gridrec in the reference's drivers. */

/* RingCorrectionSinogram (gridrec/GPU/tomo_recon.cpp:3905-3965): `iterations`
 * rounds of (renormalise every projection to the global mean; column mean;
 * 3-tap low-pass; subtract ring_coeff * (mean - low-pass), clamped at 0). */
void orc_ring_removal(double* data, int n_det, int n_ang, double ring_coeff, int iterations) {
  double* mv = (double*)malloc(n_ang * sizeof(double));
  double* ms = (double*)malloc(n_det * sizeof(double));
  double* lp = (double*)malloc(n_det * sizeof(double));
  for (int m = 0; m < iterations; ++m) {
    double total = 0.0;
    for (int i = 0; i < n_ang; ++i) {
      double s = 0.0;
      for (int j = 0; j < n_det; ++j) s += data[(long)i * n_det + j];
      mv[i] = s / n_det;
      total += mv[i];
    }
    total /= n_ang;
    for (int i = 0; i < n_ang; ++i)
      if (mv[i] != 0.0)
        for (int j = 0; j < n_det; ++j) data[(long)i * n_det + j] *= total / mv[i];
    for (int j = 0; j < n_det; ++j) ms[j] = 0.0;
    for (int i = 0; i < n_ang; ++i)
      for (int j = 0; j < n_det; ++j) ms[j] += data[(long)i * n_det + j];
    for (int j = 0; j < n_det; ++j) ms[j] /= n_ang;
    for (int j = 1; j < n_det - 1; ++j) lp[j] = (ms[j - 1] + ms[j] + ms[j + 1]) / 3.0;
    lp[0] = ms[0];
    lp[n_det - 1] = ms[n_det - 1];
    for (int i = 0; i < n_ang; ++i)
      for (int j = 0; j < n_det; ++j) {
        const double tmp = ms[j] - lp[j];
        double* x = &data[(long)i * n_det + j];
        *x = (*x - tmp * ring_coeff > 0.0) ? *x - tmp * ring_coeff : 0.0;
      }
  }
  free(mv); free(ms); free(lp);
}

/* Sub-pixel shift by xoffset and half padding (GridRecSlices,
 * gridrec/GPU/tomo_recon.cpp:3708-3810; find_shift/src/main/find_shift.cpp:1729-1808),
 * in float like the reference: kk = k - xoffset, nkk = floor(kk), neighbours
 * clamped to the row, value = in[nkk] (nkk + 1 - kk) + in[nkk + 1] (kk - nkk) at
 * column k + n_det/2; the n_det/2 columns on each side repeat the edge value and
 * any column past them (odd n_det) stays zero. */
void orc_shift_pad(const float* in, float* out, int n_det, int n_ang, float xoffset,
                   int out_width) {
  const int pad = n_det / 2;
  for (int i = 0; i < n_ang; ++i) {
    const float* r = in + (long)i * n_det;
    float* o = out + (long)i * out_width;
    for (int k = 0; k < out_width; ++k) o[k] = 0.0f;
    for (int k = 0; k < n_det; ++k) {
      const float kk = (float)k - xoffset;
      const int nk = (int)floorf(kk);
      const int a = nk < 0 ? 0 : (nk >= n_det ? n_det - 1 : nk);
      const int b = nk + 1 < 0 ? 0 : (nk + 1 >= n_det ? n_det - 1 : nk + 1);
      float v = 0.0f;
      v += r[a] * ((float)(nk + 1) - kk);
      v += r[b] * (kk - (float)nk);
      o[k + pad] = v;
    }
    for (int k = 0; k < pad; ++k) o[k] = o[pad];
    for (int k = 0; k < pad && pad + n_det + k < out_width; ++k)
      o[pad + n_det + k] = o[pad + n_det - 1];
  }
}

/* Centre crop of GridRecSlices (tomo_recon.cpp:3855-3862) and the circular crop
 * of the output stage (tomo_recon.cpp:2150-2165): out[j][k] = rec[j + offset][k + offset],
 * and with radius > 0 pixels with (k - n/2)^2 + (j - n/2)^2 >= radius^2 are zero. */
void orc_crop(const float* rec, long rec_stride, float* out, int n, int offset, int radius) {
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) {
      const long dk = k - n / 2, dj = j - n / 2;
      float v = rec[(long)(j + offset) * rec_stride + k + offset];
      if (radius > 0 && dk * dk + dj * dj >= (long)radius * radius) v = 0.0f;
      out[(long)j * n + k] = v;
    }
}

/* Output thresholds of the reference's 8-bit (BMP/TIFF) slice writer
 * (gridrec/GPU/tomo_recon.cpp:2282-2311): lo / hi start at 1e10 / -1e10 and take the
 * min / max of every pixel of the slices written together (NaN compares false and
 * is skipped); hi is then capped by RECON_THRESHOLD_UPPER_VALUE and lo raised to
 * RECON_THRESHOLD_LOWER_VALUE. */
void orc_minmax(const float* img, long n, float lower_clamp, float upper_clamp, float* lo,
                float* hi) {
  float up = -1e10f, low = 1e10f;
  for (long i = 0; i < n; ++i) {
    if (up < img[i]) up = img[i];
    if (low > img[i]) low = img[i];
  }
  if (up > upper_clamp) up = upper_clamp;
  if (low < lower_clamp) low = lower_clamp;
  *lo = low;
  *hi = up;
}

/* Its 8-bit conversion (tomo_recon.cpp:2338-2361): 0 below lo, 255 above hi, else
 * (unsigned char)(255 * (p - lo) / (hi - lo)) in float, left to right; with
 * radius > 0 the cropped copy keeps pixels with (x - w/2)^2 + (y - h/2)^2 <= radius^2
 * (x the column, y the row, integer halves) and zeroes the rest.  A value the
 * reference would convert from NaN (a NaN pixel, or hi == lo) gives 0 here. */
void orc_to_u8(const float* img, int rows, int cols, long row_stride, float lo, float hi,
               int radius, unsigned char* out) {
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) {
      const float p = img[(long)y * row_stride + x];
      unsigned char v;
      if (p < lo) v = 0;
      else if (p > hi) v = 255;
      else {
        const float q = 255.0f * (p - lo) / (hi - lo);
        v = (q == q) ? (unsigned char)q : 0;
      }
      if (radius > 0) {
        const long dx = x - cols / 2, dy = y - rows / 2;
        if (dx * dx + dy * dy > (long)radius * radius) v = 0;
      }
      out[(long)y * cols + x] = v;
    }
}

/* Histogram entropy of find_shift (find_shift/src/main/find_shift.cpp:2078-2115):
 * num_hist_bin + 1 bins, bin = (int)((x - min) / inv) computed in float with
 * inv = (max - min) / num_hist_bin (truncation toward zero; bins outside
 * [0, num_hist_bin] and NaN ignored), entropy = -sum p log2 p with p = count / n,
 * accumulated in double. */
double orc_entropy(const float* data, long n, float vmin, float vmax, int num_hist_bin) {
  long* hist = (long*)calloc(num_hist_bin + 1, sizeof(long));
  const float inv = (vmax - vmin) / (float)num_hist_bin;
  for (long i = 0; i < n; ++i) {
    const float f = (data[i] - vmin) / inv;
    if (!(f == f) || f >= 2147483648.0f || f <= -2147483649.0f) continue;
    const int ind = (int)f;
    if (ind >= 0 && ind <= num_hist_bin) hist[ind]++;
  }
  double e = 0.0;
  for (int b = 0; b <= num_hist_bin; ++b)
    if (hist[b] > 0) {
      const double p = (double)hist[b] / n;
      e += -p * log(p) / log(2.0);
    }
  free(hist);
  return e;
}

/* Cross-correlation score of find_shift's brute-force search (data_interp +
 * cross_correlation, find_shift/src/main/find_shift.cpp:1975-2076), float64:
 * the match image is sampled at (nx - tx, ny - ty) for every ROI pixel by
 * bilinear interpolation over the in-image neighbours normalised by their
 * weight (0 when the weight is <= 1e-5); with M_avg the ROI mean of the samples,
 * score = sum (T - T_avg)(M - M_avg) / (T_rms sqrt(sum (M - M_avg)^2)), 0 when
 * |T_rms| or the sum is <= 1e-5; T_rms = sqrt(sum (T - T_avg)^2) over the ROI
 * template (roi_h x roi_w, row-major). */
double orc_xcorr_score(const double* templ, const double* match, int width, int height, int x0,
                       int x1, int y0, int y1, double tx, double ty) {
  const int rw = x1 - x0 + 1, rh = y1 - y0 + 1;
  const long area = (long)rw * rh;
  double tavg = 0.0, trms = 0.0;
  for (long i = 0; i < area; ++i) tavg += templ[i];
  tavg /= (double)area;
  for (long i = 0; i < area; ++i) trms += (templ[i] - tavg) * (templ[i] - tavg);
  trms = sqrt(trms);
  double* m = (double*)malloc(area * sizeof(double));
  double mavg = 0.0;
  for (int ny = y0; ny <= y1; ++ny)
    for (int nx = x0; nx <= x1; ++nx) {
      const double x = nx - tx, y = ny - ty;
      const int a = (int)floor(x), b = (int)floor(y);
      double pix = 0.0, w = 0.0;
      const double ax = a + 1 - x, bx = x - a, ay = b + 1 - y, by = y - b;
      const int xa = a >= 0 && a < width, xb = a + 1 >= 0 && a + 1 < width;
      const int ya = b >= 0 && b < height, yb = b + 1 >= 0 && b + 1 < height;
      if (xa && ya) { pix += match[(long)b * width + a] * ax * ay; w += ax * ay; }
      if (xb && ya) { pix += match[(long)b * width + a + 1] * bx * ay; w += bx * ay; }
      if (xa && yb) { pix += match[(long)(b + 1) * width + a] * ax * by; w += ax * by; }
      if (xb && yb) { pix += match[(long)(b + 1) * width + a + 1] * bx * by; w += bx * by; }
      pix = w > 1e-5 ? pix / w : 0.0;
      m[(long)(ny - y0) * rw + nx - x0] = pix;
      mavg += pix;
    }
  mavg /= (double)area;
  double cc = 0.0, msq = 0.0;
  for (long i = 0; i < area; ++i) {
    cc += (templ[i] - tavg) * (m[i] - mavg);
    msq += (m[i] - mavg) * (m[i] - mavg);
  }
  free(m);
  return (fabs(trms) > 1e-5 && fabs(msq) > 1e-5) ? cc / (trms * sqrt(msq)) : 0.0;
}

/* OptimizedFBP (gridrec/GPU/filteredbackprojection.cpp:190-330): every projection
 * row, gated to (-5, 5) (values outside become 0), is filtered by an FFT, a
 * multiplication of bin k by 1 - sqrt(|(k - n/2) / (n/2)|), and an unnormalised
 * inverse FFT (float64 here); pixel (x, y) of the n x n image (row y) then sums,
 * over the angles in order, filtered[a][(int)((r + 1) n/2)] for -1 <= r < 1, with
 * x = (col - n/2)/(n/2), y = (row - n/2)/(n/2), r = x cos + y sin -- all in float
 * as the reference, whose sines/cosines come from the degree list via
 * (theta * PI) / 180 stored as float.  n_det must be a power of two. */
int orc_optimized_fbp(int n_det, int n_ang, const float* theta_deg, const float* sino,
                      double* recon) {
  const int n = n_det;
  if (n < 2 || (n & (n - 1))) return -1;
  const double PI_REF = 3.1415926535897932385;  /* fft.h:5 */
  float* cs = (float*)malloc(n_ang * sizeof(float));
  float* sn = (float*)malloc(n_ang * sizeof(float));
  float* lut = (float*)malloc(n * sizeof(float));
  double* row = (double*)malloc(2 * (size_t)n * sizeof(double));
  double* filt = (double*)malloc((size_t)n_ang * n * sizeof(double));
  for (int a = 0; a < n_ang; ++a) {
    const float th = (float)((theta_deg[a] * PI_REF) / 180.0);
    sn[a] = (float)sin(th);
    cs[a] = (float)cos(th);
  }
  for (int k = 0; k < n; ++k) {
    const float t = (float)(k - (float)(n / 2)) / ((float)(n / 2));
    lut[k] = (float)(1 - sqrt(fabs(t)));
  }
  for (int a = 0; a < n_ang; ++a) {
    for (int k = 0; k < n; ++k) {
      const float v = sino[(long)a * n + k];
      row[2 * k] = (v > -5.0f && v < 5.0f) ? v : 0.0;
      row[2 * k + 1] = 0.0;
    }
    orc_fft1d(row, n, +1);
    for (int k = 0; k < n; ++k) {
      row[2 * k] *= lut[k];
      row[2 * k + 1] *= lut[k];
    }
    orc_fft1d(row, n, -1);
    for (int k = 0; k < n; ++k) filt[(long)a * n + k] = row[2 * k];
  }
  const float h = (float)n / 2.0f;
  for (int yi = 0; yi < n; ++yi) {
    const float y = ((float)(yi - h)) / h;
    for (int xi = 0; xi < n; ++xi) {
      const float x = ((float)(xi - h)) / h;
      double acc = 0.0;
      for (int a = 0; a < n_ang; ++a) {
        const float xc = x * cs[a];
        const float ys = y * sn[a];
        const float r = xc + ys;
        if (r >= -1 && r < 1) {
          int k = (int)((r + 1) * h);
          if (k > n - 1) k = n - 1; /* the reference reads outside the row there */
          acc += filt[(long)a * n + k];
        }
      }
      recon[(long)yi * n + xi] = acc;
    }
  }
  free(cs); free(sn); free(lut); free(row); free(filt);
  return 0;
}
