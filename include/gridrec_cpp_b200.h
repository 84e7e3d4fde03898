/*
 * gridrec_cpp_b200.h -- the GridrecCPP 5.2 C calling sequence on the B200 library.
 *
 * A GridrecCPP caller (gridrec/GridrecCPP/Gridrec5.2/grid.h:28-58, 73-91) fills a
 * grid_struct and an sg_struct, calls recon_init() once, then per slice pair sets
 * the row-pointer globals G1, G2 (n_ang rows of n_det floats each) and S1, S2
 * (imgsiz rows of at least imgsiz floats each) and calls do_recon(), and finally
 * recon_free().  Including this header instead of grid.h and linking
 * libgridrec_b200.so instead of grid.c, pswf.c, filters.c and fft.c keeps that
 * code unchanged; the reconstruction runs on the GPU through a gridrec plan.
 *
 * The structs below have grid.h's field order and types.  The functions keep
 * grid.h's names and signatures; where the reference exits (an unknown PSWF
 * parameter, grid.cpp's exit(2)) or prints, these record a status instead:
 * gr_gridrec_cpp_status() returns the last one (GR_OK = 0, or a gr_status of
 * gridrec_b200.h) and gr_last_error() its text.  Not thread-safe, like the
 * reference (its state is these globals).
 *
 * Differences: do_recon() takes no arguments and reads the globals, as
 * Gridrec5.2/grid.cpp:152-415 does (the older four-argument form that allocated
 * S1/S2 is not provided); the reference's internal tables (pdim, M, L, scale,
 * the work arrays) are not exported as globals -- recon_init reports the image
 * side in *imgsiz and in the global imgsiz.
 */
#ifndef GRIDREC_CPP_B200_H
#define GRIDREC_CPP_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Sinogram parameters <- sg_struct, Gridrec5.2/grid.h:28-37 */
typedef struct SG_STRUCT {
  int n_ang;     /* projection angles */
  int n_det;     /* detector elements per angle */
  int geom;      /* 0: angles[] (degrees) given; 1, 2: uniform over a half / full circle */
  float* angles; /* the angle list for geom 0 */
  float center;  /* rotation axis location (pixels) */
} sg_struct;

/* Prolate spheroidal wave function data <- pswf_struct, Gridrec5.2/grid.h:39-46 */
typedef struct PSWF_STRUCT {
  float C;         /* parameter of the 0th-order PSWF */
  int nt;          /* degree of the Legendre expansion */
  float lmbda;     /* eigenvalue */
  float coefs[15]; /* coefficients of the even Legendre polynomials */
} pswf_struct;

/* Gridding parameters <- grid_struct, Gridrec5.2/grid.h:48-58 */
typedef struct GRID_STRUCT {
  pswf_struct* pswf;       /* PSWF in use (get_pswf) */
  float sampl;             /* oversampling ratio; recon_init sets it to M / M0 */
  float MaxPixSiz;         /* maximum pixel size of the reconstruction */
  float R;                 /* region of interest, relative size */
  float X0;                /* ROI offset from the rotation axis, in units of */
  float Y0;                /*   the centre-to-edge distance */
  char fname[16];          /* filter name */
  float (*filter)(float);  /* filter function of x = j / pdim (get_filter) */
  long ltbl;               /* convolvent lookup-table length */
} grid_struct;

/* Row pointers of the current pair <- Gridrec5.2/grid.h:89-91 (set by the caller
 * before each do_recon): G1/G2[n][j] sinogram values, S1/S2[j][k] image values;
 * imgsiz: image side M0 after recon_init. */
extern float **G1, **G2;
extern float **S1, **S2;
extern long imgsiz;

/* get_pswf <- Gridrec5.2/pswf.cpp:36-47: *P = the database entry for C (4.0, 4.2,
 * 5.0, 6.0, 7.0; within 0.01); NULL and a GR_ERR_PSWF status when C is unknown. */
void get_pswf(float C, pswf_struct** P);

/* get_filter <- Gridrec5.2/filters.cpp:36-48: the filter function for "shlo",
 * "shepp", "hann", "hamm", "hamming", "ramp" or "ramlak"; an unknown name selects
 * Shepp-Logan and is overwritten with "shlo", as there. */
float (*get_filter(char* name))(float);

/* recon_init <- Gridrec5.2/grid.cpp:54-147: sizes (pdim, M, M0, L, scale), tables
 * and a gridrec plan on the selected GPU for this geometry; GP->sampl becomes
 * M / M0 and *im_size (and imgsiz) the image side M0.  Filters other than
 * get_filter's are sampled at (float)j / pdim, as filphase_su does
 * (grid.cpp:437-461); a PSWF record other than get_pswf's is used as given. */
void recon_init(grid_struct* GP, sg_struct* SGP, long* im_size);

/* do_recon <- Gridrec5.2/grid.cpp:152-415: reconstructs the pair G1, G2 into the
 * M0 x M0 blocks of S1, S2 (either of G2/S2 may be NULL: a zero second slice /
 * no second image).  Synchronous. */
void do_recon(void);

/* recon_free <- Gridrec5.2/grid.cpp:418-434: releases the plan. */
void recon_free(void);

/* Status of the last call above (no counterpart in the reference, which exits). */
int gr_gridrec_cpp_status(void);

/* GPU used by the next recon_init (default 0; no counterpart in the reference). */
void gr_gridrec_cpp_set_device(int device);

#ifdef __cplusplus
}
#endif
#endif /* GRIDREC_CPP_B200_H */
