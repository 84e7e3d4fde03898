// Internal definitions shared by the gridrec kernels and the plan code.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "gridrec_b200.h"

namespace gr {

// Gridding tile: T x T grid cells per work item.
constexpr int kTile = 32;
// Largest number of taps per dimension the gridding kernel handles
// (floor(L) + 1 with L = 2*C*sampl/pi < 6).
constexpr int kMaxTaps = 6;
// Longest run of samples the gridding kernel stages at once (longer runs
// are split on the host).
constexpr int kRunMax = 64;
// Work per gridding item before a tile is split over several items, in
// sample slots (steps x samples per step).
constexpr int kItemCap = 2048;

// The 16-pair gridding kernel (grid_wide_kernel): a warp's lanes carry the
// (re, im) components of 16 slice pairs and hold a kWideRows x kWideCols
// sub-tile of cells in registers (kWideCols = 8: four packed column pairs).
constexpr int kWideRows = 4;
constexpr int kWideCols = 8;
// precomputed weights per (run, sample) of the 16-pair list: 4 row + 8 column
constexpr int kWideRec = kWideRows + kWideCols;
constexpr int kWideNoReach = 16;  // column-pair range code of a run that reaches no column
constexpr int kWideMinBlocks = 5;
constexpr int kWidePairs = 16;
// Longest run it stages at once (longer runs are split on the host).
constexpr int kRunMaxW = 16;
// Work per item before a sub-tile is split (samples + per-run overhead).
constexpr int kItemCapW = 1024;
// Chunks of at least this many pairs use it when gr_params.wide_grid is 0: its
// cost per launch does not depend on the pairs (idle lanes), the tile kernel's
// grows with them (two pairs per warp): 6 pairs 538 against 563 us per launch,
// 7 pairs 681 against 571 at 2048 x 1500; the same step at 4096 x 3000.
constexpr int kWideMinPairs = 7;

// The 32-pair gridding kernel (grid_w32_kernel): the 16-pair kernel's work list
// (4 x 8 sub-tiles, runs of <= kRunMaxW samples), one complex value per lane for
// 32 slice pairs; per (run, sample) 12 table indices of 16 bits, each run's
// index block padded to 16 bytes.
constexpr int kW32Pairs = 32;
constexpr int kW32MinBlocks = 4;
// Index of a zero weight (a tap beyond L/2) in the kernel's table copy.
inline int w32_zero_index(int ltbl) { return ltbl + 1; }

// The tensor-core gridding kernel (grid_tc_kernel): a CTA accumulates a
// kTcRows x kTcCols sub-tile (128 cells, the MMA M) for 16 pairs x (re, im)
// (the MMA N) in tensor memory, 8 samples (the MMA K) per step.
constexpr int kTcRows = 16;
constexpr int kTcCols = 8;
constexpr int kItemCapT = 2048;
// Work-list kinds (gridrec_plan.cu).
constexpr int kListTiles = 0, kListWide = 1, kListTensor = 2;

// One run of samples: direction d (= 2*angle + half), samples j in [jlo, jhi],
// gridded in steps of samples P apart (footprints of one step disjoint).
struct Run {
  int dir;
  int jlo;
  int jhi;
  int P;
};

// One gridding work item: runs [run_begin, run_end) of `tile`; slot >= 0 when
// the tile is split over several items (partial tile written to scratch slot).
struct Item {
  int tile;
  int run_begin;
  int run_end;
  int slot;
};

// Per split tile: counter index, first scratch slot, number of items.
struct Split {
  int counter;
  int slot0;
  int nsplit;
  int pad;
};

struct SpectraArgs {
  const void* s1;        // slice 1 of pair 0
  const void* s2;        // slice 2 of pair 0
  long pair_stride;      // elements between consecutive pairs' sinograms
  int n_slices_valid;    // slices that exist (2*pairs or 2*pairs-1)
  int slice_base;        // global index of slice 1 of pair 0 (for centres)
  const float* flat;     // u16 raw only: row of slice s at flat + s * flat_stride
  const float* dark;
  long flat_stride;
  const float4* pq;      // [pair][J] (P.re, P.im, Q.re, Q.im)
  float2* spec;          // [pair][n_ang][2][J], or the wide layout below
  const float2* tw;      // two-level twiddle table for pdim (see gridrec_kernels.cu)
  int n_det, n_ang, pdim, J, pairs;
  const double* roi_off; // per angle (X0 cos + Y0 sin) pi of the ROI offset, or null
  // 0: plain [pair][dir][j]; 16 or 32: the 16- or 32-pair gridding kernel's
  // [pair / G][dir][j / 4][pair % G][j % 4] (G = wide), for G = 32 with the two
  // 16-byte halves of a pair's chunk swapped when (pair / 4) is odd
  int wide = 0;
  // device error word for the bounded wait of the staged input (null: the rows are
  // loaded element by element, with no wait)
  int* err = nullptr;
  // u16 raw only: per slice of the chunk, {dark, log(flat - dark) or NaN} per detector
  // (launch_dark_log), so that a sample costs one load and one logarithm; null: the
  // flat and dark rows above are read per sample
  const float2* dl = nullptr;
};

struct PhaseArgs {
  const float* centers;  // device, per slice (may be null)
  float center_default;
  int slice_base;
  int n_slices_valid;
  const float* filt;     // [J] filter * pi/(pdim*n_ang)
  float4* pq;
  int J, pdim, pairs;
};

struct GridArgs {
  const float2* spec;
  float2* H;             // [pair][M][M]
  float4* scratch;       // [pair group][n_slots][T*T] partial tiles of split tiles
  unsigned* queue;       // work-queue head (zeroed before each launch)
  const Item* items;
  const Run* runs;
  const int4* split_list;  // per split tile: (tile, slot0, nsplit, 0)
  int n_split_tiles;
  // Tap geometry is FP64, as the FP64 restatement forms it: sample j of
  // direction d sits at u = j * dir[d] + (M/2 - tile origin), and its tap in
  // cell c weighs wtbl[(int)(|u - c| * tblspcg + 0.5)] where |u - c| <= L2.
  const double2* dir;    // per direction (scale*dx, scale*dy)
  const float* wtbl;     // ltbl + 1
  int n_items, pairs, n_ang, J, M, tiles_v, n_slots, ltbl;
  double L2, tblspcg;    // L/2, 2 ltbl / L
  const unsigned* codes = nullptr;  // grid_tc_kernel: flat (direction << 13 | j) per sample
  int* err = nullptr;               // device error word for bounded-wait timeouts
  // grid_wide_kernel: weights per (run, sample), 4 row + 8 column, and per run
  // {first sample's record, column-pair range}, from launch_wide_weights
  const float* wts = nullptr;
  const int2* wmeta = nullptr;
  // grid_w32_kernel: per run {first quad (direction * J / 4 + jlo / 4), index
  // block (16-byte units), n | (jlo % 4) << 5 | column-pair range << 12, 0}, and
  // the 16-bit table indices (launch_w32_index)
  const int4* xmeta = nullptr;
  const unsigned short* xidx = nullptr;
};

struct ColArgs {
  float2* H;
  const float2* tw;      // two-level twiddle table for M
  int M, pairs;
  int* err;              // device error word for bounded-wait timeouts (null: plain loads)
  int G = 0;             // columns per CTA (0: cols_group(M))
  int ring = 0;          // 1: persistent CTAs with two landing buffers (cols_ring_kernel)
};

struct RowArgs {
  const float2* H;
  const float2* tw;
  const float* winv;     // M0
  float* out1;           // slice 1 of pair 0
  float* out2;
  long pair_stride;      // floats between consecutive pairs' images
  long out_stride;
  int n_slices_valid;
  int M, M0, M02, pairs;
};

// FBP comparator: OptimizedFBP's row filter on pairs of projection rows packed
// as one complex line (gridrec_kernels.cu); backprojection in gridrec_fbp.cu.
struct FbpFilterArgs {
  const float* sino;     // [slice][n_ang][n]
  float* filt;           // [slice][n_ang][n]
  const float* lut;      // n filter weights
  const float2* tw;      // two-level twiddle table for n
  int n, n_ang, slices;
};
cudaError_t launch_fbp_filter(const FbpFilterArgs& a, cudaStream_t s);

// Records a formatted message for gr_last_error() and returns code (gridrec_plan.cu).
int fail(int code, const char* fmt, ...);

// A prolate spheroidal wave function record: C, eigenvalue, Legendre degree and
// the even-order Legendre coefficients (the layout of gridrec/GPU/gridrec.h:60-68,
// in double).
struct Pswf {
  double C, lmbda;
  int nt;
  double coefs[11];
};
// The PSWF database entry within 0.01 of C, or null (gridrec_plan.cu).
const Pswf* find_pswf(double C);
// Filter value at x = j / pdim for a ReconAlgorithm filter code (gridrec_plan.cu).
double filter_value(int code, double x);
// Plan creation (gr_plan_create) with two GridrecCPP extras: the PSWF from a record
// instead of the database lookup by p->pswf_c (null: the lookup), and the filter as
// a caller's function of the frequency j / pdim (null: p->filter's formula).
int plan_create_ex(const gr_params* p, const Pswf* pswf, float (*filter_fn)(float),
                   gr_plan** plan);

// Shape of a plan, for the pre/post-processing entry points (gridrec_plan.cu).
int plan_shape(const gr_plan* p, int* n_det, int* n_ang, int* M0, int* max_pairs, int* device);
// Grow-only device scratch owned by the plan (the slice-pipeline entry points).
int plan_scratch(gr_plan* p, size_t bytes, void** out);

// Makes `dev` current for the scope and restores the caller's device after.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Kernel launchers (gridrec_kernels.cu).  Return cudaGetLastError().
cudaError_t init_kernel_attributes();
cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t s);
cudaError_t launch_spectra(const SpectraArgs& a, gr_dtype dt, cudaStream_t s);
// Gridding: grid_kernel over 32 x 32 tiles (two pairs per warp) or
// grid_wide_kernel over 8 x 8 sub-tiles (16 pairs per warp), each followed by
// its split-tile reduction when tiles are split.
cudaError_t launch_grid(const GridArgs& a, int ntaps, cudaStream_t s);
cudaError_t launch_grid_wide(const GridArgs& a, cudaStream_t s);
// Weights of the 16-pair work list (once per list): meta[r] = {record base,
// sub-tile index} on entry; .y becomes the run's column-pair range code.
cudaError_t launch_wide_weights(const GridArgs& a, int n_runs, float* wts, int2* meta,
                                cudaStream_t s);
cudaError_t launch_grid_tc(const GridArgs& a, cudaStream_t s);
// 32-pair gridding: the index records of the 16-pair work list (once per list;
// rinfo[r] = {index block in 16-byte units, sub-tile index}) and the kernel.
cudaError_t launch_w32_index(const GridArgs& a, int n_runs, const int2* rinfo,
                             unsigned short* idx, int4* xmeta, cudaStream_t s);
cudaError_t launch_dark_log(const float* flat, const float* dark, long flat_stride, int slice_base,
                            int n_valid, int n_det, float2* out, cudaStream_t s);
cudaError_t launch_grid_w32(const GridArgs& a, cudaStream_t s);
int cols_group(int M);
cudaError_t launch_cols(const ColArgs& a, cudaStream_t s);
cudaError_t launch_rows(const RowArgs& a, cudaStream_t s);
cudaError_t launch_wait_probe(int* err, int limit, cudaStream_t s);

}  // namespace gr
