/* gridrec_oracle.h -- TEST INFRASTRUCTURE ONLY: float64 CPU restatement of the
 * reference gridrec (see gridrec_oracle.c).  Not part of the product. */
#ifndef GRIDREC_ORACLE_H
#define GRIDREC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int n_det, n_ang;
  double center1, center2; /* rotation centre of slice 1 / slice 2 (pixels) */
  int filter;              /* ReconAlgorithm codes: 0 none, 1 shlo, 2 hann, 3 hamm, 4 ramp */
  double C;                /* PSWF parameter: 4.0, 4.2, 5.0, 6.0 or 7.0 */
  double sampl;            /* oversampling request (1.0 = GridRec class default) */
  int ltbl;                /* convolvent table length (512) */
  /* GridrecCPP grid_struct extras (Gridrec5.2/grid.cpp:54-147, 225-275); 0 selects the
   * default of the first two (1.0) */
  double roi_size;         /* R: ROI size as a fraction of n_det */
  double pixel_size;       /* MaxPixSiz */
  double x0, y0;           /* ROI offset */
} orc_params;

typedef struct {
  long pdim, M, M02, M0;
  double sampl, L, scale, C, lmbda;
} orc_sizes_t;

int orc_sizes(const orc_params* p, orc_sizes_t* s);
int orc_tables(const orc_params* p, double* wtbl, double* winv);
void orc_fft1d(double* x, long n, int sign);
int orc_spectra(const orc_params* p, const double* sino1, const double* sino2, double* spec);
int orc_grid(const orc_params* p, const double* theta_deg, const double* spec, double* H);
void orc_fft2d(double* H, long M);
int orc_deapod(const orc_params* p, const double* H, double* out1, double* out2, long out_stride);
int orc_gridrec_pair(const orc_params* p, const double* theta_deg, const double* sino1,
                     const double* sino2, double* out1, double* out2, long out_stride);

/* Slice-pipeline steps around gridrec (see gridrec_oracle.c). */
void orc_ring_removal(double* data, int n_det, int n_ang, double ring_coeff, int iterations);
void orc_shift_pad(const float* in, float* out, int n_det, int n_ang, float xoffset, int out_width);
void orc_crop(const float* rec, long rec_stride, float* out, int n, int offset, int radius);
void orc_minmax(const float* img, long n, float lower_clamp, float upper_clamp, float* lo,
                float* hi);
void orc_to_u8(const float* img, int rows, int cols, long row_stride, float lo, float hi,
               int radius, unsigned char* out);
double orc_entropy(const float* data, long n, float vmin, float vmax, int num_hist_bin);
int orc_optimized_fbp(int n_det, int n_ang, const float* theta_deg, const float* sino,
                      double* recon);
double orc_xcorr_score(const double* templ, const double* match, int width, int height, int x0,
                       int x1, int y0, int y1, double tx, double ty);

#ifdef __cplusplus
}
#endif
#endif

