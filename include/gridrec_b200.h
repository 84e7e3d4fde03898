/*
 * gridrec_b200.h -- C ABI of the B200 (sm_100a) gridrec reconstructor.
 *
 * Gridrec reconstructs parallel-beam tomography slices by Fourier gridding:
 * per projection a zero-padded 1-D FFT times filter and centre phase ramp,
 * PSWF convolution onto an oversampled Cartesian frequency grid, a 2-D FFT,
 * and deapodisation with a crop.  Two real slices are reconstructed per pass,
 * packed as the real and imaginary parts of one complex signal.
 *
 * Everything below is plain C: pointers, sizes and status codes.  Device
 * pointers are CUDA device addresses on the plan's device; `stream` is a
 * cudaStream_t (NULL = the legacy default stream).  Every call returns
 * GR_OK (0) or a negative gr_status; no call exits the process or prints.
 *
 * Interfaces replaced (reference, decarlof/projects):
 *   gr_plan_create       <- GridRec::init               gridrec/GPU/gridrec.cu:216-310
 *                           recon_init                 gridrec/GridrecCPP/Gridrec5.2/grid.cpp:54-147
 *   gr_reconstruct_pair  <- GridRec::setSinoAndReconBuffers + GridRec::reconstruct
 *                                                      gridrec/GPU/gridrec.cu:174-212, 314-369
 *                           do_recon                   gridrec/GridrecCPP/Gridrec5.2/grid.cpp:152-415
 *   gr_plan_destroy      <- GridRec::destroy           gridrec/GPU/gridrec.cu:373-422
 *                           recon_free                 gridrec/GridrecCPP/Gridrec5.2/grid.cpp:418-434
 *   gr_filter_code       <- get_filter (by name)       gridrec/GridrecCPP/Gridrec5.2/filters.cpp:26-48
 *   gr_reconstruct_batch <- the slice-pair loop of GridRecSlices
 *                                                      gridrec/GPU/tomo_recon.cpp:3702-3852
 *   gr_reconstruct_host  <- GridRec::reconstruct on host buffers (the reference keeps
 *                           sinograms and images in host memory, gridrec.cu:174-212)
 *   GR_DTYPE_U16_RAW     <- flat/dark normalisation and log of the slice pipeline
 *                                                      gridrec/GPU/tomo_recon.cpp:1533-1541
 *   GR_DTYPE_U16_LINEAR  <- 1 - (raw - dark)/(white - dark) of the HDF5 slice path
 *                                                      gridrec/GPU/tomo_recon.cpp:1871-1877, 2019
 */
#ifndef GRIDREC_B200_H
#define GRIDREC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  GR_OK = 0,
  GR_ERR_ARG = -1,      /* invalid argument (size, pointer, stride, dtype) */
  GR_ERR_PSWF = -2,     /* PSWF parameter C not in the database (gridrec.cu:906-922) */
  GR_ERR_CUDA = -3,     /* a CUDA runtime call failed; see gr_last_error() */
  GR_ERR_NOMEM = -4,    /* device or pinned host allocation failed */
  GR_ERR_UNSUPPORTED = -5, /* size outside what the kernels implement */
  GR_ERR_TIMEOUT = -6   /* a bounded device wait expired */
} gr_status;

/* Filter codes of ReconAlgorithm (gridrec/GPU/recon_algorithm.h:18-23).
 * Codes 0 and 5 (and any other value) leave |x| unfiltered, i.e. a ramp,
 * exactly like Filter::filterData (gridrec/GPU/recon_algorithm.cpp:36-48). */
enum {
  GR_FILTER_NONE = 0,
  GR_FILTER_SHEPP_LOGAN = 1,
  GR_FILTER_HANN = 2,
  GR_FILTER_HAMMING = 3,
  GR_FILTER_RAMP = 4,
  GR_FILTER_FBP = 5
};

/* Sinogram element types accepted by the batched entry points. */
typedef enum {
  GR_DTYPE_F32 = 0,
  GR_DTYPE_F16 = 1,
  GR_DTYPE_BF16 = 2,
  GR_DTYPE_U16_RAW = 3,   /* raw detector counts, log normalisation; needs flat/dark rows */
  GR_DTYPE_U16_LINEAR = 4 /* raw detector counts, 1 - (raw-dark)/(flat-dark); needs flat/dark */
} gr_dtype;

typedef struct {
  int n_det;               /* detector pixels per projection (sinogram row length) */
  int n_ang;               /* projections (sinogram rows) */
  const float* theta_deg;  /* n_ang projection angles in degrees, host memory;
                              copied at plan creation (the reference keeps the
                              pointer, gridrec/GPU/recon_algorithm.cpp:133-137) */
  float center;            /* rotation centre in pixels; < 0 selects n_det/2,
                              the GridRec class default (gridrec.cu:227) */
  int filter;              /* GR_FILTER_* */
  float pswf_c;            /* PSWF parameter C: 4.0, 4.2, 5.0, 6.0 (default) or 7.0 */
  float sampl;             /* oversampling request; 1.0 = GridRec class default,
                              1.2 = GridrecCPP CLI default (grid_io.cpp:47) */
  int ltbl;                /* convolvent table length (512) */
  int max_pairs;           /* slice pairs processed per launch (workspace size) */
  int device;              /* CUDA device ordinal (GridRec::setGPUDeviceID) */
  int geom;                /* angle geometry of GridrecCPP's sg_struct: 0 = the theta_deg
                              list; 1 / 2 = n_ang angles evenly over pi / 2 pi from its FP32
                              rotation recurrence (Gridrec5.2/grid.cpp:540-553), theta_deg
                              unused */
  /* GridrecCPP grid_struct extras (Gridrec5.2/grid.cpp:54-147, 225-275): */
  float roi_size;          /* R: the reconstructed region spans R * n_det pixels (0 = 1) */
  float pixel_size;        /* MaxPixSiz: M = next pow2 >= sampl * R * n_det / pixel_size
                              (0 = 1) */
  float roi_x0, roi_y0;    /* ROI offset X0, Y0: C1 times exp(-i j (X0 cos + Y0 sin) pi),
                              C2 times its conjugate */
  int wide_grid;           /* gridding kernel: 0 (default) = 32-pair kernel for chunks of
                              more than 16 pairs, 16-pair kernel for 7..16 pairs, else the
                              tile kernel; 1 = 16-pair kernel for every chunk, -1 = never
                              (2 pairs per warp over 32 x 32 tiles), 2 = tensor-core kernel
                              (tcgen05, 3xTF32) for every chunk, 3 = 32-pair kernel for
                              every chunk.  Same taps and weights; the sums differ only in
                              order (the 32- and 16-pair kernels agree bit for bit) and, for
                              2, in ~2^-22 relative rounding per term */
} gr_params;

typedef struct gr_plan gr_plan;

/* Fills *p with the GridRec class defaults for an n_det x n_ang sinogram. */
int gr_params_default(gr_params* p, int n_det, int n_ang, const float* theta_deg);

/* Filter code for a GridrecCPP filter name ("shlo", "shepp", "hann", "hamm",
 * "hamming", "ramp", "ramlak", plus "none"); unknown names map to Shepp-Logan,
 * the GridrecCPP default. */
int gr_filter_code(const char* name);

/* Creates a plan: sizes, FP64-built tables, the gridding work list and the
 * device workspaces for max_pairs pairs.  Allocates device memory. */
int gr_plan_create(const gr_params* p, gr_plan** plan);
int gr_plan_destroy(gr_plan* plan);

/* Sizes derived exactly as GridRec::init (gridrec.cu:243-268):
 * pdim = next pow2 >= n_det; M = next pow2 >= sampl*n_det;
 * M0 = 2*floor(M/2/sampl - 0.5) + 1 = side of the reconstructed image. */
int gr_plan_sizes(const gr_plan* plan, int* pdim, int* M, int* M0, float* L, float* scale);

/* Device bytes held by the plan (tables, work list, workspaces). */
int gr_plan_device_bytes(const gr_plan* plan, size_t* bytes);

/* One slice pair, device pointers.  sino1/sino2: n_ang x n_det float32, row
 * stride n_det.  out1/out2: M0 rows of out_stride floats (out_stride >= M0);
 * element [j*out_stride + k] is the reference's S[j][k] (j along the first,
 * cos-direction, frequency axis, gridrec.cu:691-719).  Both slices use the
 * plan's centre. */
int gr_reconstruct_pair(gr_plan* plan, const float* sino1, const float* sino2, float* out1,
                        float* out2, long out_stride, void* stream);

/* One slice pair from HOST buffers, synchronous: the GridRec::reconstruct call of
 * the reference's callers (gridrec/GPU/gridrec.cu:314-369 with the buffers of
 * setSinoAndReconBuffers, :174-212), which keep sinograms and images in host
 * memory.  sino1/sino2: n_ang x n_det float32 (pageable or pinned; sino2 may be
 * NULL = zeros); out1/out2: M0 rows of out_stride floats (out2 may be NULL);
 * only the M0 x M0 block is written.  Pinned (page-locked or registered) caller
 * buffers are copied straight to and from the plan's device buffers (allocated on
 * first use).  Pageable ones go through the plan's pinned staging (allocated on
 * first use: 8 (n_ang n_det + M0^2) bytes): up to 8 host threads copy 4 MiB chunks,
 * each chunk's DMA queued as soon as it is staged and each image chunk copied out
 * as soon as its DMA completes, so host copies overlap the transfers (2048 x 1500:
 * 2.8 ms per call against 4.4 ms through cudaMemcpy of pageable memory).  Returns
 * after the images are in place; a bounded-wait timeout is reported as by
 * gr_plan_device_status. */
int gr_reconstruct_pair_host(gr_plan* plan, const float* sino1, const float* sino2, float* out1,
                             float* out2, long out_stride, void* stream);

/* A batch of n_slices slices (n_slices even, or odd with the last slice
 * paired with zeros), device pointers:
 *   sinos      n_slices sinograms, each n_ang x n_det of `dtype`, contiguous
 *   centers    optional device array of n_slices float centres (NULL = plan centre);
 *              the two slices of a pair may have different centres
 *   flat, dark device rows of n_det floats (raw uint16 dtypes only), applied in
 *              the first kernel as the sinogram is loaded:
 *              GR_DTYPE_U16_RAW: v = raw - dark; r = (flat - dark)/v; value = log(r)
 *              when v > 0 and r > 0, else 0 (gridrec/GPU/tomo_recon.cpp:1533-1541);
 *              GR_DTYPE_U16_LINEAR: value = 1 - (raw - dark)/(flat - dark)
 *              (tomo_recon.cpp:1871-1877, where flat = 0.5 white1 + 0.5 white2)
 *   outs       n_slices images, each M0 rows of out_stride floats, contiguous
 *   flat_stride floats between consecutive slices' flat/dark rows: 0 = one row
 *              for all slices; n_det = one row per slice (each slice is a detector
 *              row with its own white and dark, tomo_recon.cpp:1533-1541)
 * Pairs are processed max_pairs at a time on `stream`. */
typedef struct {
  int n_slices;
  gr_dtype dtype;
  const void* sinos;
  const float* centers;
  const float* flat;
  const float* dark;
  float* outs;
  long out_stride;
  long flat_stride;
} gr_batch_desc;

int gr_reconstruct_batch(gr_plan* plan, const gr_batch_desc* batch, void* stream);

/* As gr_reconstruct_batch, with sinos, centers, flat, dark and outs in HOST
 * memory: the sinograms stream in double-buffered chunks of max_pairs pairs
 * through pinned staging buffers owned by the plan (host->device copies of
 * chunk i+1 overlap the kernels of chunk i; device->host copies of images
 * overlap likewise).  Synchronises `stream` before returning. */
int gr_reconstruct_host(gr_plan* plan, const gr_batch_desc* batch, void* stream);

/* One slice pair, device pointers, like gr_reconstruct_pair, but the call
 * allocates nothing: every intermediate of the pass (phase ramps, filtered
 * spectra, frequency grid, partial tiles of split tiles, work-queue head)
 * lives in a static 32 MiB device array that the library holds on each GPU it
 * runs on until the process exits, instead of in workspaces reached through
 * cudaMalloc.  It is for callers that cannot call cudaMalloc while they
 * reconstruct: an application whose own memory pool has already reserved the
 * GPU's memory, so that a further cudaMalloc fails, and loops in which the
 * device-wide synchronisation that cudaMalloc may imply is not acceptable.
 * The plan itself is created beforehand (that step allocates its tables).
 * Limits: the intermediates (about 8 (M^2 + n_ang pdim) bytes plus 16 KiB per
 * split tile) must fit in 32 MiB, else GR_ERR_UNSUPPORTED: M <= 1024 with up
 * to about 2500 angles fits (1024 x 1024 at sampl 1.0); 1024 x 1024 at
 * sampl 1.2 (M = 2048) and 2048 x 1500 do not.  It always grids with the tile kernel (the plan's
 * wide_grid choice does not apply), so its result equals gr_reconstruct_pair's
 * bit for bit on plans with the default wide_grid = 0 and agrees within the
 * usual tolerance otherwise.  A bounded-wait timeout of its column FFT is
 * reported by gr_plan_device_status(plan), like the plan's own calls.  The
 * first call on a device looks up the array's device address
 * (cudaGetSymbolAddress).  All calls on a device share the array and it keeps
 * the last call's contents, so calls that can overlap on the GPU (different
 * streams, or different host threads) race: serialise them.  No counterpart in
 * the reference: its GridRec allocates its grid in init()
 * (gridrec/GPU/gridrec.cu:281). */
int gr_reconstruct_pair_noalloc(gr_plan* plan, const float* sino1, const float* sino2, float* out1,
                                float* out2, long out_stride, void* stream);

/* Synchronises `stream`, then reports whether a kernel of this plan stopped
 * early because one of its bounded device waits (mbarrier polls on bulk
 * copies) ran out: GR_ERR_TIMEOUT, and the flag is cleared; GR_OK otherwise.
 * gr_reconstruct_host performs this check itself. */
int gr_plan_device_status(gr_plan* plan, void* stream);

/* Exercises the timeout path on `device`: a one-thread kernel polls an
 * mbarrier that nothing ever completes, a few thousand times, and records the
 * timeout.  Returns GR_ERR_TIMEOUT when the detection works. */
int gr_selftest_wait_timeout(int device);

/* Per-stage timing with CUDA events recorded on the launching stream around
 * each kernel of each chunk (stages: 0 phase ramps, 1 spectra, 2 gridding,
 * 3 first-axis FFT, 4 second-axis FFT + deapodisation).  Enabling resets
 * the record; gr_plan_stage_times synchronises on the last event and returns
 * the summed milliseconds per stage and the number of chunks recorded. */
int gr_plan_set_timing(gr_plan* plan, int enable);
int gr_plan_stage_times(gr_plan* plan, double* ms5, long* chunks);

/* Host-only export of the gridding work list a plan with these parameters
 * would use (no GPU needed).  With items/runs/splits NULL, only the counts
 * are returned.  Layouts: items = n_items x {tile, run_begin, run_end, slot};
 * runs = n_runs x {direction (2*angle + half), jlo, jhi, step spacing P}; splits = one
 * {counter, slot0, nsplit, 0} per tile (tile = tu * tiles_v + tv, 32 x 32 cells). */
int gr_worklist_export(const gr_params* p, int* n_items, int* n_runs, int* tiles_v, int* items,
                       int* runs, int* splits, int cap_items, int cap_runs);
/* The same for the 16-pair gridding kernel's list: tiles of 4 x 8 cells (tile index
 * tu * tiles_v + tv, 4 rows by 8 columns), runs of at most 16 samples, step spacing 1;
 * splits then holds 2 * tiles_v * tiles_v records (M/4 tile rows of M/8 tiles). */
int gr_worklist_export_wide(const gr_params* p, int* n_items, int* n_runs, int* tiles_v,
                            int* items, int* runs, int* splits, int cap_items, int cap_runs);
/* *wide = 0 (tile kernel), 1 (16-pair kernel), 2 (tensor-core kernel) or 3 (32-pair
 * kernel) for a chunk of `pairs` pairs. */
int gr_plan_grid_kernel(const gr_plan* plan, int pairs, int* wide);

/* Text of the last error recorded on this thread (never NULL). */
const char* gr_last_error(void);

/* Number of kernel launches the plan has issued since creation. */
int gr_plan_launch_count(const gr_plan* plan, long* launches);

/* Autotuner: on the plan's own workspaces, times
 *  - the gridding kernel of a full chunk (max_pairs pairs), in the default mode
 *    (wide_grid = 0) among every kernel the plan holds records for: the 32 x 32
 *    shared-memory tile kernel, and the 4 x 8 register sub-tile kernels at 16 and 32
 *    pairs per warp (each sub-tile shape and tile size has one compiled instance);
 *  - for each, the work-item cost cap (512..8192 sample slots per item on the tile
 *    list, 256..4096 on the 4 x 8 list: load balance against split-tile overhead);
 *  - the column-FFT group width (1..8 columns per CTA), each with one strip per
 *    CTA and with persistent CTAs that double-buffer their strips;
 * and keeps the fastest (gr_plan_grid_kernel then reports the kernel chosen for a
 * full chunk; smaller chunks keep the choice by chunk size).  The FFTs have one
 * radix sequence per length, so there is nothing to choose there.  Choices are
 * cached per shape in the process, so later plans of the same shape tune
 * instantly.  Synchronises `stream`; not for use inside stream capture.  Results
 * stay within the same tolerance; bitwise reproducibility holds per tuning (the
 * kernel and item cap set the gridding's summation order).  No reference
 * counterpart (the reference has fixed launch shapes). */
int gr_plan_autotune(gr_plan* plan, void* stream);  /* GR_ERR_ARG while a gr_graph holds the plan */
int gr_plan_tuning(const gr_plan* plan, int* item_cap, int* cols_group);
/* Pins a tuning instead of timing one: grid_kernel for full chunks (0 tiles, 1
 * 16-pair, 3 32-pair, as gr_plan_grid_kernel reports; -1: by chunk size; only in the
 * default mode and among the kernels the plan holds records for), item_cap of that
 * kernel's work list (0: keep), cols_group (1, 2, 4, 8; 0: keep) and cols_ring (1:
 * the persistent double-buffered column FFT where its two landing buffers fit in
 * shared memory, 0: one strip per CTA, -1: keep).  GR_ERR_ARG for an option the plan
 * cannot run, or while a gr_graph holds the plan. */
int gr_plan_set_tuning(gr_plan* plan, int grid_kernel, int item_cap, int cols_group,
                       int cols_ring);
/* The full tuning: gridding kernel of a full chunk, its item cap, column group width
 * and whether the column FFT runs persistent and double-buffered. */
int gr_plan_tuning_ex(const gr_plan* plan, int* grid_kernel, int* item_cap, int* cols_group,
                      int* cols_ring);

/* Shape of the gridding work list: work items (CTAs per pair), sample runs,
 * scratch slots of split tiles, and samples visited per pair (with halo). */
int gr_plan_work_stats(const gr_plan* plan, int* n_items, int* n_runs, int* n_slots,
                       long* total_samples);

/* ---- CUDA graphs: record once, replay with one launch.
 * gr_graph_create records gr_reconstruct_batch(item.plan, &item.batch) for every
 * item into one CUDA graph by stream capture.  Items of one plan run in order on
 * one branch (they share its workspaces); items of different plans (different
 * shapes: n_det, n_ang, dtype) run on parallel branches, so an uneven batch is
 * one launch.  The batch buffers are baked into the graph: gr_graph_launch
 * replays the same addresses on `stream`.  All plans must be on one device and
 * have stage timing off.  No reference counterpart: the reference launches per
 * slice pair (gridrec/GPU/tomo_recon.cpp:3846-3852). */
typedef struct gr_graph gr_graph;
typedef struct {
  gr_plan* plan;
  gr_batch_desc batch;
} gr_graph_item;
int gr_graph_create(const gr_graph_item* items, int n_items, gr_graph** graph);
int gr_graph_launch(gr_graph* graph, void* stream);  /* GR_ERR_ARG once a plan it holds is destroyed */
/* Kernel launches one replay performs. */
int gr_graph_launch_count(const gr_graph* graph, long* launches);
int gr_graph_destroy(gr_graph* graph);

/* ---- Slice pipeline around gridrec (the reference's tomo_recon and find_shift
 * drivers).  Sinograms are n_ang rows of n_det float32, slices contiguous, in
 * device memory; calls are asynchronous on `stream` unless stated. */

/* Ring suppression <- RingCorrectionSinogram   gridrec/GPU/tomo_recon.cpp:3905-3972
 * (the reference runs 20 rounds with RING_COEFF 1.0, tomo_recon.h:63).  In place on
 * n_slices sinograms; workspace: gr_ring_workspace_bytes() bytes of device memory. */
size_t gr_ring_workspace_bytes(int n_slices, int n_det, int n_ang);
int gr_ring_removal(float* sinos, int n_slices, int n_det, int n_ang, float ring_coeff,
                    int iterations, void* workspace, void* stream);

/* Sub-pixel shift and half padding <- GridRecSlices  gridrec/GPU/tomo_recon.cpp:3708-3807
 * (also find_shift/src/main/find_shift.cpp:1729-1808).  Slice s is shifted by
 * xoffsets[s] (device array) with linear interpolation (neighbours clamped to the
 * row), placed at column n_det/2 of rows of out_width floats, with the n_det/2
 * columns on each side repeating the edge values.  Equal to the reference's float
 * arithmetic bit for bit. */
int gr_shift_pad(const float* in, float* out, int n_slices, int n_det, int n_ang,
                 const float* xoffsets, int out_width, void* stream);

/* Centre crop <- GridRecSlices  tomo_recon.cpp:3855-3862: out[j][k] =
 * recon[j + offset][k + offset] for j, k < n; with radius > 0 also the circular
 * crop of tomo_recon.cpp:2150-2165 (pixels with (k-n/2)^2 + (j-n/2)^2 >= radius^2
 * set to 0).  Strides and per-slice sizes in floats. */
int gr_crop_center(const float* recon, long recon_stride, long recon_slice_elems, float* out,
                   long out_stride, long out_slice_elems, int n_slices, int n, int offset,
                   int radius, void* stream);

/* Output thresholds <- the 8-bit slice writer of tomo_recon.cpp:2282-2311: lohi[0] /
 * lohi[1] (device, 2 floats) = min / max over every pixel of the n_slices images
 * (rows x cols, strides in floats; NaN skipped), then hi capped at upper_clamp and
 * lo raised to lower_clamp (RECON_THRESHOLD_UPPER/LOWER_VALUE).  workspace: device,
 * gr_threshold_workspace_bytes() bytes. */
size_t gr_threshold_workspace_bytes(void);
int gr_threshold_range(const float* images, int n_slices, int rows, int cols, long row_stride,
                       long slice_stride, float lower_clamp, float upper_clamp, float* lohi,
                       void* workspace, void* stream);
/* 8-bit slices <- tomo_recon.cpp:2338-2361: 0 below lo, 255 above hi, else
 * (unsigned char)(255 * (p - lo) / (hi - lo)) in float; with radius > 0 the
 * writer's cropped copy: pixels with (x - cols/2)^2 + (y - rows/2)^2 > radius^2 set
 * to 0 (this writer keeps the boundary circle, gr_crop_center's float crop does
 * not).  lohi from gr_threshold_range (device).  Bit-exact with the reference's
 * float arithmetic; a NaN result gives 0. */
int gr_to_u8(const float* images, int n_slices, int rows, int cols, long row_stride,
             long slice_stride, const float* lohi, int radius, unsigned char* out,
             long out_row_stride, long out_slice_stride, void* stream);

/* Histogram entropy <- entropy()  find_shift/src/main/find_shift.cpp:2078-2115.
 * For each of n_groups groups of `group` image windows (rows x cols, row_stride;
 * images image_stride apart, groups group_stride apart, all in floats): nbins + 1
 * bins of width (vmax - vmin) / nbins, bin = (int)((x - vmin) / width) in float,
 * entropies[g] = -sum p log2 p (device array of n_groups floats).  Workspace:
 * gr_entropy_workspace_bytes() bytes.  nbins <= 50000. */
size_t gr_entropy_workspace_bytes(int n_groups, int nbins);
int gr_entropy(const float* images, int n_groups, int group, int rows, int cols, long row_stride,
               long image_stride, long group_stride, float vmin, float vmax, int nbins,
               float* entropies, void* workspace, void* stream);

/* Half-padded slice reconstruction <- GridRecSlices  tomo_recon.cpp:3679-3862:
 * every slice shifted by xoffset and half padded to the plan's width (the plan is
 * made for 2 n_det detector pixels and n_ang angles), reconstructed in pairs, and
 * cropped to n_det x n_det (rows of out_stride floats, slices n_det * out_stride
 * apart).  Allocates its intermediates (stream-ordered). */
int gr_reconstruct_padded(gr_plan* plan, const float* sinos, int n_slices, int n_det, int n_ang,
                          float xoffset, float* outs, long out_stride, void* stream);

/* Rotation-centre refinement by entropy <- find_shift  find_shift/src/main/find_shift.cpp:1653-1900.
 * For each of n_cand shifts (host array) the slice pair (sino1, sino2; device) is
 * shifted, half padded and reconstructed with `plan` (2 n_det wide, n_ang angles),
 * both n_det x n_det crops are scored together with the histogram entropy
 * [hist_lo, hist_hi] in nbins bins, and scores[c] (host) receives the score.
 * *best = first index of the minimum score.  best_images (optional, device,
 * 2 x n_det x n_det) receives the pair at the best shift.  Synchronises `stream`. */
int gr_center_search(gr_plan* plan, const float* sino1, const float* sino2, int n_det, int n_ang,
                     const float* shifts, int n_cand, float hist_lo, float hist_hi, int nbins,
                     float* scores, int* best, float* best_images, void* stream);

/* Rotation-axis search by cross-correlation <- find_shift's brute-force search
 * (data_interp + cross_correlation, find_shift/src/main/find_shift.cpp:1975-2076;
 * GPU twin cross_correlation.cu:19-413).  templ_roi: the (roi_y1-roi_y0+1) x
 * (roi_x1-roi_x0+1) template (device, float); match: height x width (device).
 * For every translation (tx0 + i dtx, ty0 + k dty), i < n_tx, k < n_ty, the match
 * image is sampled at (nx - tx, ny - ty) over the ROI by weight-normalised bilinear
 * interpolation and scored by normalised cross-correlation with the template
 * (double arithmetic, as the reference's CPU path; the reference's GPU path uses
 * 8-bit texture filtering weights instead).  scores: host, n_ty x n_tx doubles.
 * Synchronises `stream`. */
int gr_xcorr_scores(const float* templ_roi, const float* match, int width, int height, int roi_x0,
                    int roi_x1, int roi_y0, int roi_y1, double tx0, double ty0, double dtx,
                    double dty, int n_tx, int n_ty, double* scores, void* stream);

/* FBP comparator <- OptimizedFBP, the reference's ReconAlgorithm filtered
 * backprojection (gridrec/GPU/filteredbackprojection.cpp:190-330; tomo_recon's GPU
 * FBP, gridrec/GPU/fbp.cu:22-169, is the same pipeline with a floor() sampler).
 * Each projection row, gated to (-5, 5), is filtered by 1 - sqrt(|k - n/2|/(n/2))
 * in frequency (unnormalised FFT pair), and pixel (x, y) of the n x n image sums
 * filtered[a][(int)((r + 1) n/2)] over the angles, r = x cos + y sin with x, y in
 * [-1, 1).  n_det a power of two in [16, 8192].  sinos: n_slices x n_ang x n_det
 * (device); recons: n_slices x n_det x n_det (device, row = y).  One slice per
 * call of the reference; max_slices per launch here. */
typedef struct gr_fbp gr_fbp;
int gr_fbp_create(int n_det, int n_ang, const float* theta_deg, int max_slices, int device,
                  gr_fbp** fbp);
int gr_fbp_reconstruct(gr_fbp* fbp, const float* sinos, int n_slices, float* recons, void* stream);
int gr_fbp_destroy(gr_fbp* fbp);

/* ---- Learned correction of narrow-kernel gridrec (no reference counterpart; the
 * learned part of the project's specification).  A 3-layer, 16-channel, 3x3 residual
 * CNN y = x + conv3(relu(conv2(relu(conv1(x))))) on n_img images of h x w (device
 * float32).  params: gr_cnn_param_count() floats, layout w1[9][16], b1[16],
 * w2[9][16][16], b2[16], w3[9][16], b3.  conv2 runs on BF16 tensor cores with FP32
 * accumulation; hidden activations are stored as BF16.  The workspace
 * (gr_cnn_workspace_bytes) keeps the forward activations that gr_cnn_backward uses:
 * call backward after forward on the same images and workspace.  gr_cnn_backward
 * writes the mean-squared-loss gradient to grads and the loss to *loss (synchronises
 * when loss is non-NULL); gr_cnn_adam applies one Adam step (step counts from 1). */
int gr_cnn_param_count(void);
size_t gr_cnn_workspace_bytes(int n_img, int h, int w);          /* forward + backward */
size_t gr_cnn_forward_workspace_bytes(int n_img, int h, int w);  /* forward only */
int gr_cnn_forward(const float* params, const float* x, float* y, int n_img, int h, int w,
                   void* workspace, void* stream);
int gr_cnn_backward(const float* params, const float* x, const float* y, const float* target,
                    int n_img, int h, int w, float* grads, double* loss, void* workspace,
                    void* stream);
int gr_cnn_adam(float* params, const float* grads, float* m, float* v, int step, float lr,
                float beta1, float beta2, float eps, void* stream);
/* Fused inference: the same network in one kernel per call, for inference only.
 * conv1 (on a BF16 im2col of x), conv2 and conv3 (as a 1x1 product to its nine
 * per-tap partials, then a shifted FP32 sum) run as tcgen05 BF16 MMAs with FP32
 * accumulators in tensor memory; h1, h2 and the partials stay in shared memory, so
 * only x and y cross HBM.  Differs from gr_cnn_forward by conv1's input and conv1's
 * and conv3's weights rounded to BF16 and the tensor core's summation order.
 * scale (device, n_img floats, or NULL for 1): image i is corrected at unit scale,
 * y = s_i * net(x / s_i), the scaling fused into the x loads and y stores.
 * workspace: gr_cnn_infer_workspace_bytes() device bytes, zeroed once by the caller
 * (it holds the error word of the kernel's bounded waits); gr_cnn_infer_status
 * synchronises `stream`, reports GR_ERR_TIMEOUT if a wait ran out and clears the word. */
size_t gr_cnn_infer_workspace_bytes(void);
int gr_cnn_infer(const float* params, const float* x, float* y, const float* scale, int n_img,
                 int h, int w, void* workspace, void* stream);
int gr_cnn_infer_status(void* workspace, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GRIDREC_B200_H */
