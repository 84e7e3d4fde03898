/* Exercises include/gridrec_cpp_b200.h the way a GridrecCPP 5.2 caller does
 * (gridrec/GridrecCPP/Gridrec5.2/grid_io.cpp:38-96 for the parameters, grid.h:89-91
 * for the row pointers): get_pswf, get_filter, recon_init, do_recon, recon_free.
 * Reads two float32 sinograms (n_ang x n_det) from argv[1]; writes imgsiz (as a
 * float) and the two imgsiz x imgsiz images to argv[2].
 * Usage: gridrec_cpp_demo in.bin out.bin n_det n_ang center filter C sampl layout
 *   filter: a GridrecCPP name, or "custom" (a caller's own Hann-shaped function);
 *   layout: "flat" (contiguous rows) or "rows" (every row its own allocation). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "gridrec_b200.h"
#include "gridrec_cpp_b200.h"

static float custom_hann(float x) { return fabsf(x) * 0.5f * (1.0f + cosf(6.2831853f * x)); }

static float** rows_of(float* base, long n, long stride, int own) {
  float** r = (float**)malloc(n * sizeof(float*));
  for (long i = 0; i < n; ++i) {
    if (own) {
      r[i] = (float*)malloc(stride * sizeof(float));
      memcpy(r[i], base + i * stride, stride * sizeof(float));
    } else {
      r[i] = base + i * stride;
    }
  }
  return r;
}

int main(int argc, char** argv) {
  if (argc < 10) {
    fprintf(stderr, "usage: %s in.bin out.bin n_det n_ang center filter C sampl layout\n", argv[0]);
    return 2;
  }
  const int n_det = atoi(argv[3]), n_ang = atoi(argv[4]);
  const int own = !strcmp(argv[9], "rows");
  float* sino = (float*)malloc(2 * (size_t)n_ang * n_det * sizeof(float));
  float* theta = (float*)malloc(n_ang * sizeof(float));
  FILE* f = fopen(argv[1], "rb");
  if (!f || fread(sino, sizeof(float), 2 * (size_t)n_ang * n_det, f) != 2 * (size_t)n_ang * n_det)
    return 3;
  fclose(f);
  for (int i = 0; i < n_ang; ++i) theta[i] = 180.0f * i / n_ang;

  sg_struct sg;
  grid_struct gp;
  sg.n_ang = n_ang;
  sg.n_det = n_det;
  sg.geom = 0;
  sg.angles = theta;
  sg.center = (float)atof(argv[5]);
  get_pswf((float)atof(argv[7]), &gp.pswf);
  if (gr_gridrec_cpp_status() != GR_OK) {
    fprintf(stderr, "get_pswf: %s\n", gr_last_error());
    return 4;
  }
  gp.sampl = (float)atof(argv[8]);
  gp.MaxPixSiz = 1.0f;
  gp.R = 1.0f;
  gp.X0 = gp.Y0 = 0.0f;
  strncpy(gp.fname, argv[6], sizeof(gp.fname) - 1);
  gp.fname[sizeof(gp.fname) - 1] = '\0';
  gp.filter = strcmp(gp.fname, "custom") ? get_filter(gp.fname) : custom_hann;
  gp.ltbl = 512;

  long size = 0;
  recon_init(&gp, &sg, &size);
  if (gr_gridrec_cpp_status() != GR_OK || size != imgsiz) {
    fprintf(stderr, "recon_init: %s\n", gr_last_error());
    return 5;
  }
  float* img = (float*)calloc(2 * (size_t)size * size, sizeof(float));
  G1 = rows_of(sino, n_ang, n_det, own);
  G2 = rows_of(sino + (size_t)n_ang * n_det, n_ang, n_det, own);
  S1 = rows_of(img, size, size, own);
  S2 = rows_of(img + (size_t)size * size, size, size, own);
  do_recon();
  if (gr_gridrec_cpp_status() != GR_OK) {
    fprintf(stderr, "do_recon: %s\n", gr_last_error());
    return 6;
  }
  if (own)  /* gather the separately allocated rows */
    for (long j = 0; j < size; ++j) {
      memcpy(img + j * size, S1[j], size * sizeof(float));
      memcpy(img + ((size_t)size + j) * size, S2[j], size * sizeof(float));
    }
  recon_free();
  f = fopen(argv[2], "wb");
  const float fs = (float)size;
  fwrite(&fs, sizeof(float), 1, f);
  fwrite(img, sizeof(float), 2 * (size_t)size * size, f);
  fclose(f);
  printf("imgsiz %ld sampl %.6f\n", size, gp.sampl);
  return 0;
}
