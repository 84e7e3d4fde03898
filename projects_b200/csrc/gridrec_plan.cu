// Host side of the gridrec C ABI: plan creation (sizes, FP64 tables, the
// gridding work list, device workspaces), the per-chunk launch sequence, and
// the host-memory streaming entry point.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <condition_variable>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "gr_internal.h"

namespace gr {

thread_local std::string g_err = "no error";

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

namespace {

#define GR_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return fail(GR_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                  \
  } while (0)

// PSWF database: the numerical table of gridrec/GPU/gridrec.cu:21-114 (C,
// eigenvalue, Legendre degree, even-order Legendre coefficients).
const Pswf kPswfDb[5] = {
    {4.0, 0.99588549, 16,
     {0.5239891E+01, -0.5308499E+01, 0.1184591E+01, -0.1230763E-00, 0.7371623E-02,
      -0.2864074E-03, 0.7789983E-05, -0.1564700E-06, 0.2414647E-08, 0.0, 0.0}},
    {4.2, 0.99657887, 16,
     {0.6062942E+01, -0.6450252E+01, 0.1551875E+01, -0.1755960E-01, 0.1150712E-01,
      -0.4903653E-03, 0.1464986E-04, -0.3235110E-06, 0.5492141E-08, 0.0, 0.0}},
    {5.0, 0.99935241, 18,
     {0.1115509E+02, -0.1384861E+02, 0.4289811E+01, -0.6514303E-00, 0.5844993E-01,
      -0.3447736E-02, 0.1435066E-03, -0.4433680E-05, 0.1056040E-06, -0.1997173E-08, 0.0}},
    {6.0, 0.9990188, 18,
     {0.2495593E+02, -0.3531124E+02, 0.1383722E+02, -0.2799028E+01, 0.3437217E-00,
      -0.2818024E-01, 0.1645842E-02, -0.7179160E-04, 0.2424510E-05, -0.6520875E-07, 0.0}},
    {7.0, 0.99998546, 20,
     {0.5767616E+02, -0.8931343E+02, 0.4167596E+02, -0.1053599E+02, 0.1662374E+01,
      -0.1780527E-00, 0.1372983E-01, -0.7963169E-03, 0.3593372E-04, -0.1295941E-05,
      0.3817796E-07}},
};

}  // namespace

const Pswf* find_pswf(double C) {
  for (const Pswf& p : kPswfDb)
    if (std::fabs(C - p.C) <= 0.01) return &p;
  return nullptr;
}

// Sum_k coefs[k] P_2k(x) via the Legendre three-term recurrence.
double legendre_even(const Pswf& p, double x) {
  double y = p.coefs[0], penult = 1.0, last = x;
  int k = 1;
  for (int j = 2; j <= p.nt; ++j) {
    const double nw = (x * (2 * j - 1) * last - (j - 1) * penult) / j;
    if ((j & 1) == 0) y += nw * p.coefs[k++];
    penult = last;
    last = nw;
  }
  return y;
}

// Filter::filterData semantics (gridrec/GPU/recon_algorithm.cpp:36-73).
double filter_value(int code, double x) {
  switch (code) {
    case GR_FILTER_SHEPP_LOGAN: return std::fabs(std::sin(M_PI * x) / M_PI);
    case GR_FILTER_HANN: return std::fabs(x) * 0.5 * (1.0 + std::cos(2 * M_PI * x));
    case GR_FILTER_HAMMING: return std::fabs(x) * (0.54 + 0.46 * std::cos(2 * M_PI * x));
    case GR_FILTER_RAMP: return std::fabs(x);
    default: return x;
  }
}

// ------------------------------------------------------------------ the plan

struct Plan {
  int device = 0;
  int n_det = 0, n_ang = 0, pdim = 0, M = 0, M02 = 0, M0 = 0, J = 0, ltbl = 0, filter = 0;
  int ntaps = 0, max_pairs = 1;
  double sampl = 1, L = 0, scale = 0, C = 6, lmbda = 0;
  float center = 0;
  // device tables
  float* d_wtbl = nullptr;
  float* d_winv = nullptr;
  float* d_filt = nullptr;
  float2* d_tw_p = nullptr;
  float2* d_tw_m = nullptr;
  double2* d_dir = nullptr;         // per direction (scale*dx, scale*dy): tap positions
  double* d_roi_off = nullptr;  // per-angle ROI offset phase step, or null
  // gridding work list
  int tiles_u = 0, tiles_v = 0, n_items = 0, n_runs = 0, n_slots = 0, n_split = 0;
  long total_samples = 0;
  Item* d_items = nullptr;
  Run* d_runs = nullptr;
  Split* d_splits = nullptr;
  int4* d_split_list = nullptr;
  int n_split_tiles = 0;
  unsigned* d_queue = nullptr;
  int* d_err = nullptr;  // device error word: nonzero after a bounded wait ran out
  // workspaces (max_pairs pairs)
  float2* d_spec = nullptr;
  float2* d_H = nullptr;
  float4* d_scratch = nullptr;
  size_t scratch_cells = 0;         // float4 cells allocated in d_scratch
  std::vector<double> dxy;          // per-direction (du, dv) steps, kept for rebuilding
  int item_cap = kItemCap;          // gridding work-item cost cap (autotuned)
  // 16-pair gridding (grid_wide_kernel): its own work list over 8 x 8 sub-tiles,
  // present when chunks can be wide enough to use it (gr_params.wide_grid)
  int wide_mode = 0;                // gr_params.wide_grid: 0 auto, 1 always, -1 never
  int w_tiles_v = 0, w_items = 0, w_runs = 0, w_slots = 0, w_split_tiles = 0;
  int w_item_cap = kItemCapW;
  Item* d_w_items = nullptr;
  Run* d_w_runs = nullptr;
  int4* d_w_split_list = nullptr;
  float4* d_w_scratch = nullptr;    // [pair group of 16][slot][64 cells x 32 lanes] floats
  float* d_w_wts = nullptr;         // [sample of the list][4 row + 8 column weights]
  int2* d_w_meta = nullptr;         // per run: {first weight record, column-pair range}
  size_t w_scratch_cells = 0;
  int spec_pairs = 0;               // pairs the spectra workspace holds
  // tensor-core gridding (grid_tc_kernel, gr_params.wide_grid = 2): 16 x 8
  // sub-tiles, each item's samples as one flat code array padded to 8
  int t_tiles_v = 0, t_items = 0, t_slots = 0, t_split_tiles = 0, t_item_cap = kItemCapT;
  Item* d_t_items = nullptr;
  unsigned* d_t_codes = nullptr;
  int4* d_t_split_list = nullptr;
  float4* d_t_scratch = nullptr;    // [group of 16][slot][128 cells][32 values] floats
  size_t t_scratch_cells = 0;
  // 32-pair gridding (grid_w32_kernel): the 16-pair list's runs as index records
  unsigned short* d_x_idx = nullptr;  // per run: 12 16-bit table indices per sample, 16-byte blocks
  int4* d_x_meta = nullptr;           // per run: {first quad, index block, packed n/offset/quads/range}
  float4* d_x_scratch = nullptr;      // [pair group of 32][slot][32 cells x 32 pairs] complex
  size_t x_scratch_cells = 0;
  bool x_ready = false;
  int cols_G = 0;                   // column-FFT group width (0 = cols_group(M); autotuned)
  int cols_ring = 0;                // 1: persistent double-buffered column FFT (autotuned)
  // gridding kernel of full chunks (max_pairs pairs) in the default mode, chosen by the
  // autotuner or gr_plan_set_tuning: 0 tiles, 1 16-pair, 3 32-pair (-1: by chunk size)
  int tuned_kernel = -1;
  std::vector<gr_graph*> graphs;    // live CUDA graphs replaying this plan's buffers
  float4* d_pq = nullptr;
  float2* d_dl = nullptr;  // raw u16 chunks: {dark, log(flat - dark)} per slice and detector
  // pair slots of d_pq holding the ramps of the plan's own centre (no per-slice
  // centres): such calls skip the phase kernel.  Off for good once a call is
  // captured into a graph, whose replays may rewrite d_pq at any time.
  int pq_default = 0;
  bool pq_cache_off = false;
  // host streaming (gr_reconstruct_host)
  void* h_in[2] = {nullptr, nullptr};
  float* h_out[2] = {nullptr, nullptr};
  void* d_in[2] = {nullptr, nullptr};
  float* d_out[2] = {nullptr, nullptr};
  size_t in_bytes = 0, out_bytes = 0;  // per staging buffer
  long out_stride_staged = 0;
  float* d_pair_in = nullptr;          // gr_reconstruct_pair_host: one pair of sinograms
  float* d_pair_out = nullptr;         //   and its two M0 x M0 images
  float* h_pair_in = nullptr;          // pinned staging of the pair for pageable callers
  float* h_pair_out = nullptr;
  std::vector<cudaEvent_t> pair_events;  // one per staged image chunk
  cudaStream_t copy_stream = nullptr;   // host->device copies
  cudaStream_t d2h_stream = nullptr;    // device->host copies (runs beside the H2D ones)
  cudaEvent_t ev_h2d[2] = {}, ev_comp[2] = {}, ev_d2h[2] = {};
  size_t device_bytes = 0;
  long launches = 0;
  // scratch of the slice-pipeline entry points (grow-only, freed with the plan)
  void* d_prep = nullptr;
  size_t prep_bytes = 0;
  // optional per-stage timing: 6 events per chunk (before phase, after each stage)
  bool timing = false;
  std::vector<cudaEvent_t> events;
  size_t events_used = 0;
  std::vector<std::pair<void*, size_t>> allocs;  // device allocations and their bytes
  std::vector<double> h_winv, h_wtbl;
};

namespace {

template <typename T>
int dev_alloc(Plan* p, T** ptr, size_t count) {
  *ptr = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)ptr, count * sizeof(T));
  if (e != cudaSuccess) {
    *ptr = nullptr;
    cudaGetLastError();
    return fail(GR_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T),
                cudaGetErrorString(e));
  }
  p->allocs.emplace_back((void*)*ptr, count * sizeof(T));
  p->device_bytes += count * sizeof(T);
  return GR_OK;
}

template <typename T>
int upload(Plan* p, T** dptr, const std::vector<T>& h) {
  int rc = dev_alloc(p, dptr, h.size());
  if (rc) return rc;
  GR_CUDA(cudaMemcpy(*dptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  return GR_OK;
}

template <typename T>
void dev_free(Plan* p, T** ptr) {
  if (!*ptr) return;
  auto it = std::find_if(p->allocs.begin(), p->allocs.end(),
                         [&](const std::pair<void*, size_t>& x) { return x.first == (void*)*ptr; });
  if (it != p->allocs.end()) {
    p->device_bytes -= it->second;
    p->allocs.erase(it);
  }
  cudaFree(*ptr);
  *ptr = nullptr;
}

// The gridding work list: for each T x T tile, the runs of samples
// (direction, j range) whose L x L footprint can reach the tile; tiles whose
// runs exceed the item cap are split into several items.  T = kTile (32) for
// grid_kernel, kWideRows x kWideCols (4 x 8) for grid_wide_kernel.
struct WorkList {
  std::vector<Item> items;
  std::vector<Run> runs;
  std::vector<Split> splits;
  int tiles_u = 0, tiles_v = 0, n_slots = 0, n_split = 0;
  long total = 0;
};

// Step spacing P of a run (see grid_kernel): the smallest P with
// P * max(|du|,|dv|) >= NT (with the kernel's margin) and, above it, the P
// needing the fewest steps of spw samples; returns the step count in *steps.
int run_spacing(double du, double dv, int n, double L, int spw, int* steps) {
  // valid taps lie within L/2 of a sample, so samples more than L apart in
  // one coordinate never share a cell (margin above FP32 position error)
  const double step = std::max(std::fabs(du), std::fabs(dv));
  const int pmin = std::max(1, (int)((L + 2e-3) / step) + 1);
  auto count = [&](int P) {
    int st = 0;
    for (int b = 0; b < n; b += spw * P) st += std::min(P, n - b);
    return st;
  };
  int best = count(pmin), P = pmin;
  for (int q = pmin + 1; q <= pmin + spw; ++q) {
    const int c = count(q);
    if (c < best) {
      best = c;
      P = q;
    }
  }
  *steps = best;
  return P;
}

// kind: kListTiles (32 x 32, grid_kernel), kListWide (8 x 8, grid_wide_kernel) or
// kListTensor (16 x 8, grid_tc_kernel; its runs are flattened by build_tc_list).
void build_work_list(int M, int J, double L, int n_ang, const std::vector<double>& dxy,
                     WorkList* wl, int item_cap = kItemCap, int kind = kListTiles) {
  const bool wide = kind != kListTiles;
  const int Tu = kind == kListTiles ? kTile : (kind == kListWide ? kWideRows : kTcRows);
  const int Tv = kind == kListTiles ? kTile : (kind == kListWide ? kWideCols : kTcCols);
  const int run_max = kind == kListWide ? kRunMaxW : kRunMax;
  const double M2 = M / 2;
  const double L2 = L / 2 + 2e-3;  // box margin covers FP32 position rounding
  wl->tiles_u = (M + Tu - 1) / Tu;
  wl->tiles_v = (M + Tv - 1) / Tv;
  const int n_tiles = wl->tiles_u * wl->tiles_v;
  const int n_dir = 2 * n_ang;
  struct TRun { int tile, dir, jlo, jhi; };
  std::vector<TRun> all;
  auto slab = [](double o, double dd, double lo, double hi, double& tmin, double& tmax) {
    if (std::fabs(dd) < 1e-12) return o >= lo && o <= hi;
    double t1 = (lo - o) / dd, t2 = (hi - o) / dd;
    if (t1 > t2) std::swap(t1, t2);
    tmin = std::max(tmin, t1);
    tmax = std::min(tmax, t2);
    return tmin <= tmax;
  };
  // runs of directions [d0, d1) in (direction, tile row, tile column, j) order
  auto enumerate_dirs = [&](int d0, int d1, std::vector<TRun>& out) {
    for (int d = d0; d < d1; ++d) {
      const double dx = dxy[2 * d], dy = dxy[2 * d + 1];
      for (int tu = 0; tu < wl->tiles_u; ++tu) {
        const double x0 = tu * Tu - L2, x1 = std::min(tu * Tu + Tu, M) - 1 + L2;
        double ta = 1.0, tb = J - 1.0;
        if (!slab(M2, dx, x0, x1, ta, tb)) continue;
        // y extent of the samples in this x slab -> candidate tile columns
        const double ya = M2 + ta * dy, yb = M2 + tb * dy;
        const double ymin = std::min(ya, yb), ymax = std::max(ya, yb);
        int tv0 = (int)std::floor((ymin - L2) / Tv) - 1;
        int tv1 = (int)std::floor((ymax + L2) / Tv) + 1;
        tv0 = std::max(tv0, 0);
        tv1 = std::min(tv1, wl->tiles_v - 1);
        for (int tv = tv0; tv <= tv1; ++tv) {
          const double y0 = tv * Tv - L2, y1 = std::min(tv * Tv + Tv, M) - 1 + L2;
          double sa = ta, sb = tb;
          if (!slab(M2, dy, y0, y1, sa, sb)) continue;
          const int jlo = std::max(1, (int)std::ceil(sa - 1e-6));
          const int jhi = std::min(J - 1, (int)std::floor(sb + 1e-6));
          for (int j0 = jlo; j0 <= jhi; j0 += run_max)  // runs of at most run_max samples
            out.push_back({tu * wl->tiles_v + tv, d, j0, std::min(jhi, j0 + run_max - 1)});
        }
      }
    }
  };
  // directions split over host threads in contiguous blocks, concatenated in
  // direction order: the same list as one thread builds
  const long work = (long)n_dir * wl->tiles_u;
  const int n_thr = work < (1L << 16)
                        ? 1
                        : (int)std::min<long>(std::min<long>(16, n_dir),
                                              std::max(1u, std::thread::hardware_concurrency()));
  if (n_thr == 1) {
    all.reserve((size_t)n_dir * wl->tiles_u * 2);
    enumerate_dirs(0, n_dir, all);
  } else {
    std::vector<std::vector<TRun>> parts(n_thr);
    std::vector<std::thread> pool;
    bool threaded = true;
    try {
      for (int k = 0; k < n_thr; ++k)
        pool.emplace_back([&, k] {
          enumerate_dirs((int)((long)n_dir * k / n_thr), (int)((long)n_dir * (k + 1) / n_thr),
                         parts[k]);
        });
    } catch (...) {  // no thread to be had: the threads started finish, then one pass
      threaded = false;
    }
    for (auto& th : pool) th.join();
    if (threaded) {
      size_t total_runs = 0;
      for (const auto& part : parts) total_runs += part.size();
      all.reserve(total_runs);
      for (const auto& part : parts) all.insert(all.end(), part.begin(), part.end());
    } else {
      enumerate_dirs(0, n_dir, all);
    }
  }
  // stable counting sort by tile (runs of a tile keep their enumeration order)
  {
    std::vector<size_t> at(n_tiles + 1, 0);
    for (const TRun& r : all) at[r.tile + 1]++;
    for (int t = 0; t < n_tiles; ++t) at[t + 1] += at[t];
    std::vector<TRun> sorted(all.size());
    for (const TRun& r : all) sorted[at[r.tile]++] = r;
    all.swap(sorted);
  }
  wl->runs.resize(all.size());
  std::vector<long> run_cost(all.size());
  // the kernel's NT: footprint rows per sample (3 for L < 3, e.g. C = 4 at sampl = 1)
  const int taps = (int)std::floor(L) + 1;
  const int nt = taps <= 3 ? 3 : (taps <= 4 ? 4 : kMaxTaps);
  const int spw = 32 / nt;
  std::vector<int> first(n_tiles + 1, 0);
  for (size_t i = 0; i < all.size(); ++i) {
    const int n = all[i].jhi - all[i].jlo + 1;
    if (wide) {
      // one pass per sample over the register tile; the run's copies, restaging and dispatch
      wl->runs[i] = {all[i].dir, all[i].jlo, all[i].jhi, 1};
      run_cost[i] = n + 6;
    } else {
      int steps = 0;
      const int P = run_spacing(dxy[2 * all[i].dir], dxy[2 * all[i].dir + 1], n, L, spw, &steps);
      wl->runs[i] = {all[i].dir, all[i].jlo, all[i].jhi, P};
      run_cost[i] = (long)steps * spw + 4;  // sample slots + per-run overhead
    }
    first[all[i].tile + 1]++;
  }
  for (int t = 0; t < n_tiles; ++t) first[t + 1] += first[t];
  struct CItem { Item it; long cost; };
  std::vector<CItem> items;
  wl->splits.assign(n_tiles, Split{0, 0, 1, 0});
  int n_slots = 0, n_split = 0;
  long total = 0;
  for (int t = 0; t < n_tiles; ++t) {
    const int b = first[t], e = first[t + 1];
    long cost = 0;
    for (int r = b; r < e; ++r) {
      cost += run_cost[r];
      total += wl->runs[r].jhi - wl->runs[r].jlo + 1;
    }
    if (cost <= item_cap) {
      items.push_back({{t, b, e, -1}, cost});
      continue;
    }
    std::vector<std::pair<int, long>> cuts;  // (run_end, cost)
    long c = 0;
    for (int r = b; r < e; ++r) {
      const long rc = run_cost[r];
      if (c > 0 && c + rc > item_cap) {
        cuts.push_back({r, c});
        c = 0;
      }
      c += rc;
    }
    cuts.push_back({e, c});
    wl->splits[t] = Split{n_split++, n_slots, (int)cuts.size(), 0};
    int start = b;
    for (const auto& cut : cuts) {
      items.push_back({{t, start, cut.first, n_slots++}, cut.second});
      start = cut.first;
    }
  }
  if (kind == kListWide) {
    // 4 x 8 sub-tiles in Morton order of (tile row, tile column): the warps running at
    // once take neighbouring sub-tiles, which share the spectra quads of the rays that
    // cross them, so a quad is read from DRAM about once
    auto spread = [](unsigned x) {
      x &= 0xffffu;
      x = (x | (x << 8)) & 0x00ff00ffu;
      x = (x | (x << 4)) & 0x0f0f0f0fu;
      x = (x | (x << 2)) & 0x33333333u;
      x = (x | (x << 1)) & 0x55555555u;
      return x;
    };
    // in eight cost classes, heaviest first, so that no heavy item starts late and holds
    // up the launch's tail; Morton order within a class
    const int tv_n = wl->tiles_v;
    long cmax = 1;
    for (const CItem& c : items) cmax = std::max(cmax, c.cost);
    auto cls = [&](const CItem& c) { return (int)std::min<long>(7, c.cost * 8 / (cmax + 1)); };
    std::stable_sort(items.begin(), items.end(), [&](const CItem& a, const CItem& b) {
      const int ca = cls(a), cb = cls(b);
      if (ca != cb) return ca > cb;
      const unsigned ma = spread((unsigned)(a.it.tile / tv_n)) | spread((unsigned)(a.it.tile % tv_n)) << 1;
      const unsigned mb = spread((unsigned)(b.it.tile / tv_n)) | spread((unsigned)(b.it.tile % tv_n)) << 1;
      return ma < mb;
    });
  } else {
    // heaviest items first so that the long ones start early
    std::stable_sort(items.begin(), items.end(),
                     [](const CItem& a, const CItem& b) { return a.cost > b.cost; });
  }
  wl->items.resize(items.size());
  for (size_t i = 0; i < items.size(); ++i) wl->items[i] = items[i].it;
  wl->n_slots = n_slots;
  wl->n_split = n_split;
  wl->total = total;
}

// Builds the work list with the given item cap and (re)places it on the
// device; grows the split-tile scratch when needed.
int install_work_list(Plan* p, int item_cap) {
  WorkList wl;
  build_work_list(p->M, p->J, p->L, p->n_ang, p->dxy, &wl, item_cap);
  std::vector<int4> split_list;
  for (size_t t = 0; t < wl.splits.size(); ++t)
    if (wl.splits[t].nsplit > 1)
      split_list.push_back(make_int4((int)t, wl.splits[t].slot0, wl.splits[t].nsplit, 0));
  dev_free(p, &p->d_items);
  dev_free(p, &p->d_runs);
  dev_free(p, &p->d_splits);
  dev_free(p, &p->d_split_list);
  int rc;
  if ((rc = upload(p, &p->d_items, wl.items)) || (rc = upload(p, &p->d_runs, wl.runs)) ||
      (rc = upload(p, &p->d_splits, wl.splits)) || (rc = upload(p, &p->d_split_list, split_list)))
    return rc;
  const size_t cells =
      ((size_t)(p->max_pairs + 1) / 2) * (size_t)std::max(wl.n_slots, 1) * kTile * kTile;
  if (cells != p->scratch_cells) {  // exact: a reinstall with fewer splits gives memory back
    dev_free(p, &p->d_scratch);
    if ((rc = dev_alloc(p, &p->d_scratch, cells))) return rc;
    p->scratch_cells = cells;
  }
  p->tiles_u = wl.tiles_u;
  p->tiles_v = wl.tiles_v;
  p->n_items = (int)wl.items.size();
  p->n_runs = (int)wl.runs.size();
  p->n_slots = wl.n_slots;
  p->n_split = wl.n_split;
  p->total_samples = wl.total;
  p->n_split_tiles = (int)split_list.size();
  p->item_cap = item_cap;
  return GR_OK;
}

// Whether chunks of this plan can use the 16-pair kernel (its weights) or the
// 32-pair kernel (its index records); both run on the 4 x 8 work list.
bool wide16_possible(const Plan* p) {
  return p->wide_mode == 1 || (p->wide_mode == 0 && p->max_pairs >= kWideMinPairs);
}
bool w32_possible(const Plan* p) {
  return p->wide_mode == 3 || (p->wide_mode == 0 && p->max_pairs > kWidePairs);
}

// The 16- and 32-pair kernels' work list (4 x 8 sub-tiles), placed on the device
// with the records of whichever of the two kernels the plan can use.
int install_work_list_wide(Plan* p, int item_cap) {
  WorkList wl;
  build_work_list(p->M, p->J, p->L, p->n_ang, p->dxy, &wl, item_cap, kListWide);
  std::vector<int4> split_list;
  for (size_t t = 0; t < wl.splits.size(); ++t)
    if (wl.splits[t].nsplit > 1)
      split_list.push_back(make_int4((int)t, wl.splits[t].slot0, wl.splits[t].nsplit, 0));
  // per run: its first weight record (samples of the runs before it) and its
  // sub-tile, which the weights kernel replaces by the run's column-pair range
  std::vector<int2> meta(wl.runs.size(), make_int2(0, 0));
  for (const Item& it : wl.items)
    for (int r = it.run_begin; r < it.run_end; ++r) meta[r].y = it.tile;
  size_t n_rec = 0;
  for (size_t r = 0; r < wl.runs.size(); ++r) {
    meta[r].x = (int)n_rec;
    n_rec += (size_t)(wl.runs[r].jhi - wl.runs[r].jlo + 1);
  }
  if (n_rec > (size_t)INT_MAX) return fail(GR_ERR_UNSUPPORTED, "work list too large");
  // the 32-pair kernel's records: per run an index block of n * 12 16-bit indices,
  // padded to whole 16-byte units (its bulk copies move whole units)
  const bool need16 = wide16_possible(p), need32 = w32_possible(p);
  std::vector<int2> rinfo;
  size_t n_units = 0;
  if (need32) {
    rinfo.resize(wl.runs.size());
    for (size_t r = 0; r < wl.runs.size(); ++r) {
      rinfo[r] = make_int2((int)n_units, meta[r].y);
      n_units += ((size_t)(wl.runs[r].jhi - wl.runs[r].jlo + 1) * kWideRec * 2 + 15) / 16;
    }
    if (n_units > (size_t)INT_MAX) return fail(GR_ERR_UNSUPPORTED, "work list too large");
  }
  dev_free(p, &p->d_w_items);
  dev_free(p, &p->d_w_runs);
  dev_free(p, &p->d_w_split_list);
  dev_free(p, &p->d_w_meta);
  dev_free(p, &p->d_w_wts);
  dev_free(p, &p->d_x_idx);
  dev_free(p, &p->d_x_meta);
  p->x_ready = false;
  int rc;
  if ((rc = upload(p, &p->d_w_items, wl.items)) || (rc = upload(p, &p->d_w_runs, wl.runs)) ||
      (rc = upload(p, &p->d_w_split_list, split_list)) ||
      (need16 && ((rc = upload(p, &p->d_w_meta, meta)) ||
                  (rc = dev_alloc(p, &p->d_w_wts, std::max<size_t>(n_rec, 1) * kWideRec)))))
    return rc;
  GridArgs g{};
  g.runs = p->d_w_runs;
  g.dir = p->d_dir;
  g.wtbl = p->d_wtbl;
  g.M = p->M;
  g.J = p->J;
  g.tiles_v = wl.tiles_v;
  g.ltbl = p->ltbl;
  g.L2 = p->L / 2;
  g.tblspcg = 2.0 * p->ltbl / p->L;
  if (need16) GR_CUDA(launch_wide_weights(g, (int)wl.runs.size(), p->d_w_wts, p->d_w_meta, 0));
  if (need32) {
    int2* d_rinfo = nullptr;
    if ((rc = upload(p, &d_rinfo, rinfo)) ||
        (rc = dev_alloc(p, &p->d_x_idx, std::max<size_t>(n_units, 1) * 8)) ||
        (rc = dev_alloc(p, &p->d_x_meta, std::max<size_t>(wl.runs.size(), 1)))) {
      dev_free(p, &d_rinfo);
      return rc;
    }
    cudaError_t e = cudaMemsetAsync(p->d_x_idx, 0, std::max<size_t>(n_units, 1) * 16, 0);
    if (e == cudaSuccess)
      e = launch_w32_index(g, (int)wl.runs.size(), d_rinfo, p->d_x_idx, p->d_x_meta, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    dev_free(p, &d_rinfo);
    if (e != cudaSuccess) return fail(GR_ERR_CUDA, "32-pair index records: %s", cudaGetErrorString(e));
    // 32 cells x 32 pairs complex = 512 float4 per slot and group of 32 pairs
    const size_t groups32 = (size_t)(p->max_pairs + kW32Pairs - 1) / kW32Pairs;
    const size_t xcells = groups32 * (size_t)std::max(wl.n_slots, 1) * (kWideRows * kWideCols * 32 / 2);
    if (xcells != p->x_scratch_cells) {
      dev_free(p, &p->d_x_scratch);
      if ((rc = dev_alloc(p, &p->d_x_scratch, xcells))) return rc;
      p->x_scratch_cells = xcells;
    }
    p->x_ready = true;
  }
  GR_CUDA(cudaStreamSynchronize(0));
  // 64 cells x 32 lanes floats = 512 float4 per slot and group of 16 pairs
  const size_t groups = (size_t)(p->max_pairs + kWidePairs - 1) / kWidePairs;
  const size_t cells = groups * (size_t)std::max(wl.n_slots, 1) * (kWideRows * kWideCols * 32 / 4);
  if (need16 && cells != p->w_scratch_cells) {
    dev_free(p, &p->d_w_scratch);
    if ((rc = dev_alloc(p, &p->d_w_scratch, cells))) return rc;
    p->w_scratch_cells = cells;
  }
  p->w_tiles_v = wl.tiles_v;
  p->w_items = (int)wl.items.size();
  p->w_runs = (int)wl.runs.size();
  p->w_slots = wl.n_slots;
  p->w_split_tiles = (int)split_list.size();
  p->w_item_cap = item_cap;
  return GR_OK;
}

// The tensor-core kernel's work list: 16 x 8 sub-tiles; each item's runs
// flattened into (direction << 13 | j) codes, padded with j = 0 (a zero
// spectrum) to a whole number of 8-sample steps.
int install_work_list_tc(Plan* p, int item_cap) {
  WorkList wl;
  build_work_list(p->M, p->J, p->L, p->n_ang, p->dxy, &wl, item_cap, kListTensor);
  std::vector<unsigned> codes;
  codes.reserve((size_t)wl.total + 8 * wl.items.size());
  std::vector<Item> items(wl.items.size());
  for (size_t i = 0; i < wl.items.size(); ++i) {
    const Item& it = wl.items[i];
    const int begin = (int)codes.size();
    for (int r = it.run_begin; r < it.run_end; ++r)
      for (int j = wl.runs[r].jlo; j <= wl.runs[r].jhi; ++j)
        codes.push_back(((unsigned)wl.runs[r].dir << 13) | (unsigned)j);
    while ((codes.size() - begin) % 8) codes.push_back(0u);
    items[i] = {it.tile, begin, (int)codes.size(), it.slot};
  }
  std::vector<int4> split_list;
  for (size_t t = 0; t < wl.splits.size(); ++t)
    if (wl.splits[t].nsplit > 1)
      split_list.push_back(make_int4((int)t, wl.splits[t].slot0, wl.splits[t].nsplit, 0));
  dev_free(p, &p->d_t_items);
  dev_free(p, &p->d_t_codes);
  dev_free(p, &p->d_t_split_list);
  int rc;
  if ((rc = upload(p, &p->d_t_items, items)) || (rc = upload(p, &p->d_t_codes, codes)) ||
      (rc = upload(p, &p->d_t_split_list, split_list)))
    return rc;
  const size_t groups = (size_t)(p->max_pairs + kWidePairs - 1) / kWidePairs;
  const size_t cells = groups * (size_t)std::max(wl.n_slots, 1) * (kTcRows * kTcCols * 32 / 4);
  if (cells != p->t_scratch_cells) {
    dev_free(p, &p->d_t_scratch);
    if ((rc = dev_alloc(p, &p->d_t_scratch, cells))) return rc;
    p->t_scratch_cells = cells;
  }
  p->t_tiles_v = wl.tiles_v;
  p->t_items = (int)items.size();
  p->t_slots = wl.n_slots;
  p->t_split_tiles = (int)split_list.size();
  p->t_item_cap = item_cap;
  return GR_OK;
}

bool use_tc(const Plan* p, int pairs) {
  (void)pairs;
  return p->t_items > 0 && p->wide_mode == 2;
}

// Whether a chunk of `pairs` pairs grids with grid_w32_kernel: always in mode 3;
// by default for chunks of more than 16 pairs.  Its cost per launch does not
// depend on the live pairs (idle lanes): one launch for 17..32 pairs costs less
// than the 16-pair kernel's two groups (2048 x 1500: 32.1 against 2 x 39.3 us per
// group pair-slot), while up to 16 pairs the 16-pair kernel's launch is cheaper.
bool use_w32(const Plan* p, int pairs) {
  if (!p->x_ready || p->w_items == 0) return false;
  if (p->wide_mode == 0 && p->tuned_kernel >= 0 && pairs == p->max_pairs) return p->tuned_kernel == 3;
  return p->wide_mode == 3 || (p->wide_mode == 0 && pairs > kWidePairs);
}

// Whether a chunk of `pairs` pairs grids with grid_wide_kernel.
bool use_wide(const Plan* p, int pairs) {
  if (p->w_items == 0 || p->wide_mode < 0 || use_tc(p, pairs) || use_w32(p, pairs)) return false;
  if (p->wide_mode == 0 && p->tuned_kernel >= 0 && pairs == p->max_pairs) return p->tuned_kernel == 1;
  return p->wide_mode == 1 || pairs >= kWideMinPairs;
}

GridArgs grid_args_tc(const Plan* p, int pairs) {
  GridArgs g{p->d_spec, p->d_H, p->d_t_scratch, p->d_queue, p->d_t_items, nullptr,
             p->d_t_split_list, p->t_split_tiles, p->d_dir, p->d_wtbl, p->t_items, pairs,
             p->n_ang, p->J, p->M, p->t_tiles_v, p->t_slots, p->ltbl, p->L / 2,
             2.0 * p->ltbl / p->L, p->d_t_codes, p->d_err};
  return g;
}

GridArgs grid_args(const Plan* p, int pairs, bool wide) {
  GridArgs g =
      wide ? GridArgs{p->d_spec, p->d_H, p->d_w_scratch, p->d_queue, p->d_w_items, p->d_w_runs,
                      p->d_w_split_list, p->w_split_tiles, p->d_dir, p->d_wtbl, p->w_items, pairs,
                      p->n_ang, p->J, p->M, p->w_tiles_v, p->w_slots, p->ltbl, p->L / 2,
                      2.0 * p->ltbl / p->L}
           : GridArgs{p->d_spec, p->d_H, p->d_scratch, p->d_queue, p->d_items, p->d_runs,
                      p->d_split_list, p->n_split_tiles, p->d_dir, p->d_wtbl, p->n_items, pairs,
                      p->n_ang, p->J, p->M, p->tiles_v, p->n_slots, p->ltbl, p->L / 2,
                      2.0 * p->ltbl / p->L};
  if (wide) {
    g.wts = p->d_w_wts;
    g.wmeta = p->d_w_meta;
  }
  return g;
}

GridArgs grid_args_w32(const Plan* p, int pairs) {
  GridArgs g{p->d_spec, p->d_H, p->d_x_scratch, p->d_queue, p->d_w_items, p->d_w_runs,
             p->d_w_split_list, p->w_split_tiles, p->d_dir, p->d_wtbl, p->w_items, pairs,
             p->n_ang, p->J, p->M, p->w_tiles_v, p->w_slots, p->ltbl, p->L / 2,
             2.0 * p->ltbl / p->L};
  g.err = p->d_err;
  g.xmeta = p->d_x_meta;
  g.xidx = p->d_x_idx;
  return g;
}

// Sizes exactly as GridRec::init (gridrec/GPU/gridrec.cu:243-268), in FP64.
struct Geometry {
  long pdim, M, M02, M0;
  double sampl, L, scale;
  int ntaps;
};

int geometry(const gr_params* prm, const Pswf* pw, Geometry* g) {
  long pdim = 1, itmp = prm->n_det - 1;
  while (itmp) { pdim <<= 1; itmp >>= 1; }
  const double R = prm->roi_size > 0.f ? prm->roi_size : 1.0;
  const double pix = prm->pixel_size > 0.f ? prm->pixel_size : 1.0;
  const double D0 = R * prm->n_det;  // GridrecCPP grid.cpp:95-106 (R = MaxPixSiz = 1: GridRec)
  const double D1 = (double)prm->sampl * D0;
  long M = 1;
  itmp = (long)(D1 / pix - 1);
  while (itmp) { M <<= 1; itmp >>= 1; }
  long M02 = (long)std::floor((double)(M / 2) / (double)prm->sampl - 0.5);
  if (M02 < 0) M02 = 0;
  g->pdim = pdim;
  g->M = M;
  g->M02 = M02;
  g->M0 = 2 * M02 + 1;
  g->sampl = (double)M / g->M0;
  g->L = 2 * pw->C * g->sampl / M_PI;
  g->scale = g->sampl * D0 / pdim;
  g->ntaps = (int)std::floor(g->L) + 1;
  if (pdim > 8192 || M > 8192 || M < 16 || g->ntaps > kMaxTaps)
    return fail(GR_ERR_UNSUPPORTED, "sizes pdim=%ld M=%ld L=%.3f outside the kernels' range", pdim,
                M, g->L);
  return GR_OK;
}

int check_params(const gr_params* prm, const Pswf** pw, const Pswf* pswf_override = nullptr) {
  if (!prm) return fail(GR_ERR_ARG, "null argument");
  if (prm->geom < 0 || prm->geom > 2) return fail(GR_ERR_ARG, "geom must be 0, 1 or 2");
  if (prm->n_det < 9 || prm->n_ang < 1 || (prm->geom == 0 && !prm->theta_deg))
    return fail(GR_ERR_ARG, "need n_det >= 9, n_ang >= 1 and (geom 0) a theta list");
  if (prm->ltbl < 1 || prm->ltbl > 1024) return fail(GR_ERR_ARG, "ltbl must be in [1, 1024]");
  if (!(prm->sampl >= 1.0f) || prm->sampl > 4.0f)
    return fail(GR_ERR_ARG, "sampl must be in [1, 4]");
  if (prm->max_pairs < 1) return fail(GR_ERR_ARG, "max_pairs must be >= 1");
  if (prm->wide_grid < -1 || prm->wide_grid > 3)
    return fail(GR_ERR_ARG, "wide_grid must be -1, 0, 1, 2 or 3");
  if (prm->roi_size < 0.f || prm->roi_size > 4.f || prm->pixel_size < 0.f || prm->pixel_size > 16.f)
    return fail(GR_ERR_ARG, "roi_size in [0, 4] and pixel_size in [0, 16] (0 = 1)");
  if (pswf_override) {
    if (pswf_override->nt < 0 || pswf_override->nt > 20 || !(pswf_override->C > 0.0) ||
        !(pswf_override->lmbda > 0.0))
      return fail(GR_ERR_PSWF, "PSWF record: C > 0, eigenvalue > 0 and degree 0..20 required");
    *pw = pswf_override;
    return GR_OK;
  }
  *pw = find_pswf(prm->pswf_c);
  if (!*pw) return fail(GR_ERR_PSWF, "Prolate parameter C = %f not in data base", prm->pswf_c);
  return GR_OK;
}

// Direction vectors in grid units: half 0 = scale*(cos, sin), half 1 = mirrored.
// geom 0: FP64 sin/cos of the degree list (the GridRec class, gridrec.cu:724-770).
// geom 1 / 2: GridrecCPP's uniform angles over pi / 2 pi, generated by its FP32
// rotation recurrence from (sin, cos) = (0, 1) (Gridrec5.2/grid.cpp:540-553, pi =
// 3.14159265359), drift included, since that is what its gridding uses.
std::vector<double> directions(const gr_params* prm, double scale) {
  std::vector<double> dxy(4 * (size_t)prm->n_ang);
  std::vector<float> rs, rc;
  if (prm->geom != 0) {
    const float dtheta = (float)(prm->geom * 3.14159265359 / prm->n_ang);
    const float dcos = (float)std::cos((double)dtheta), dsin = (float)std::sin((double)dtheta);
    rs.assign(prm->n_ang, 0.f);
    rc.assign(prm->n_ang, 1.f);
    for (int j = 1; j < prm->n_ang; ++j) {
      const float a = dcos * rs[j - 1], b = dsin * rc[j - 1];
      const float c = dcos * rc[j - 1], d = dsin * rs[j - 1];
      rs[j] = a + b;
      rc[j] = c - d;
    }
  }
  for (int n = 0; n < prm->n_ang; ++n) {
    double cs, sn;
    if (prm->geom == 0) {
      const double th = (double)prm->theta_deg[n] * (M_PI / 180.0);
      cs = std::cos(th) * scale;
      sn = std::sin(th) * scale;
    } else {
      cs = (double)rc[n] * scale;
      sn = (double)rs[n] * scale;
    }
    dxy[4 * n + 0] = cs;
    dxy[4 * n + 1] = sn;
    dxy[4 * n + 2] = -cs;
    dxy[4 * n + 3] = -sn;
  }
  return dxy;
}

cudaEvent_t next_event(Plan* p) {
  if (p->events_used == p->events.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    p->events.push_back(e);
  }
  return p->events[p->events_used++];
}

#define GR_MARK()                                                  \
  do {                                                             \
    if (p->timing) {                                               \
      cudaEvent_t ev_ = next_event(p);                             \
      if (!ev_) return fail(GR_ERR_CUDA, "cudaEventCreate failed"); \
      GR_CUDA(cudaEventRecord(ev_, st));                           \
    }                                                              \
  } while (0)

int launch_chunk(Plan* p, int pairs, int n_valid, int slice_base, const void* s1,
                 const void* s2, long in_pair_stride, gr_dtype dt, const float* centers,
                 const float* flat, const float* dark, long flat_stride, float* o1, float* o2,
                 long out_pair_stride, long out_stride, cudaStream_t st) {
  GR_MARK();
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    p->pq_cache_off = true;
  }
  int launched = 0;
  if (centers || p->pq_cache_off || p->pq_default < pairs) {
    PhaseArgs ph{centers, p->center, slice_base, n_valid, p->d_filt, p->d_pq, p->J, p->pdim, pairs};
    GR_CUDA(launch_phase(ph, st));
    p->pq_default = (centers || p->pq_cache_off) ? 0 : pairs;
    ++launched;
  }
  // raw counts: the chunk's {dark, log(flat - dark)} rows once, not once per angle
  const bool dl = dt == GR_DTYPE_U16_RAW && flat && dark;
  if (dl) {
    GR_CUDA(launch_dark_log(flat, dark, flat_stride, slice_base, n_valid, p->n_det, p->d_dl, st));
    ++launched;
  }
  GR_MARK();
  const bool tc = use_tc(p, pairs);
  const bool w32 = use_w32(p, pairs);
  const bool wide = use_wide(p, pairs);
  SpectraArgs sa{s1, s2, in_pair_stride, n_valid, slice_base, flat, dark, flat_stride, p->d_pq,
                 p->d_spec,
                 p->d_tw_p, p->n_det, p->n_ang, p->pdim, p->J, pairs, p->d_roi_off,
                 w32 ? kW32Pairs : ((wide || tc) ? kWidePairs : 0), p->d_err};
  if (dl) sa.dl = p->d_dl;
  GR_CUDA(launch_spectra(sa, dt, st));
  GR_MARK();
  const GridArgs ga = tc ? grid_args_tc(p, pairs)
                         : (w32 ? grid_args_w32(p, pairs) : grid_args(p, pairs, wide));
  GR_CUDA(tc ? launch_grid_tc(ga, st)
             : (w32 ? launch_grid_w32(ga, st)
                    : (wide ? launch_grid_wide(ga, st) : launch_grid(ga, p->ntaps, st))));
  GR_MARK();
  ColArgs ca{p->d_H, p->d_tw_m, p->M, pairs, p->d_err, p->cols_G, p->cols_ring};
  GR_CUDA(launch_cols(ca, st));
  GR_MARK();
  RowArgs ra{p->d_H, p->d_tw_m, p->d_winv, o1, o2, out_pair_stride, out_stride, n_valid,
             p->M, p->M0, p->M02, pairs};
  GR_CUDA(launch_rows(ra, st));
  GR_MARK();
  // (phase unless its ramps are cached, dark/log for raw counts,) spectra, grid (+ split
  // reduction when tiles are split), cols, rows
  p->launches += launched + 4 + (ga.n_items > 0 && ga.n_split_tiles > 0 ? 1 : 0);
  return GR_OK;
}

size_t dtype_size(gr_dtype dt) {
  switch (dt) {
    case GR_DTYPE_F32: return 4;
    case GR_DTYPE_F16:
    case GR_DTYPE_BF16:
    case GR_DTYPE_U16_RAW: return 2;
    case GR_DTYPE_U16_LINEAR: return 2;
  }
  return 0;
}

int validate_batch(const Plan* p, const gr_batch_desc* b) {
  if (!b || b->n_slices < 1 || !b->sinos || !b->outs)
    return fail(GR_ERR_ARG, "batch: n_slices >= 1, sinos and outs are required");
  if (b->out_stride < p->M0)
    return fail(GR_ERR_ARG, "out_stride %ld < M0 %d", b->out_stride, p->M0);
  if (dtype_size(b->dtype) == 0) return fail(GR_ERR_ARG, "unknown dtype %d", (int)b->dtype);
  if ((b->dtype == GR_DTYPE_U16_RAW || b->dtype == GR_DTYPE_U16_LINEAR) && (!b->flat || !b->dark))
    return fail(GR_ERR_ARG, "raw uint16 dtypes need flat and dark rows");
  if (b->flat_stride != 0 && b->flat_stride < p->n_det)
    return fail(GR_ERR_ARG, "flat_stride %ld: 0 or >= n_det %d", b->flat_stride, p->n_det);
  return GR_OK;
}

// Whether [ptr, ptr + bytes) lies in page-locked (or registered) host memory: both ends
// are checked.
bool is_pinned(const void* ptr, size_t bytes) {
  for (const void* q : {ptr, (const void*)((const char*)ptr + (bytes ? bytes - 1 : 0))}) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, q) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    if (at.type != cudaMemoryTypeHost) return false;
  }
  return true;
}

// gr_reconstruct_pair_host on pageable caller buffers.  cudaMemcpy from pageable
// memory goes through the driver's small bounce buffers at a fraction of the link
// rate; here host threads copy the sinograms into the plan's pinned staging in
// chunks, each chunk's H2D copy queued as soon as it is staged (copies of later
// chunks overlap the DMA of earlier ones), and the images come back in row chunks
// whose host copies into the caller's rows (stride out_stride) start as each
// chunk's DMA completes (one event per chunk).  The calling thread is worker 0 and
// queues the reconstruction between the two phases.
int pair_host_staged(Plan* p, const float* sino1, const float* sino2, float* out1, float* out2,
                     long out_stride, cudaStream_t st, int n_valid) {
  const size_t slice = (size_t)p->n_ang * p->n_det, img = (size_t)p->M0 * p->M0;
  if (!p->h_pair_in) {
    if (cudaHostAlloc((void**)&p->h_pair_in, 2 * slice * sizeof(float), cudaHostAllocDefault) !=
        cudaSuccess) {
      cudaGetLastError();
      p->h_pair_in = nullptr;
      return fail(GR_ERR_NOMEM, "pinned staging of %zu bytes", 2 * slice * sizeof(float));
    }
  }
  if (!p->h_pair_out) {
    if (cudaHostAlloc((void**)&p->h_pair_out, 2 * img * sizeof(float), cudaHostAllocDefault) !=
        cudaSuccess) {
      cudaGetLastError();
      p->h_pair_out = nullptr;
      return fail(GR_ERR_NOMEM, "pinned staging of %zu bytes", 2 * img * sizeof(float));
    }
  }
  constexpr size_t kChunk = (size_t)4 << 20;  // bytes per staged copy
  struct InChunk {
    const char* src;
    char* pin;
    char* dev;
    size_t n;
  };
  std::vector<InChunk> in;
  auto add_in = [&](const float* src, size_t off) {
    const size_t bytes = slice * sizeof(float);
    for (size_t b = 0; b < bytes; b += kChunk)
      in.push_back({reinterpret_cast<const char*>(src) + b,
                    reinterpret_cast<char*>(p->h_pair_in + off) + b,
                    reinterpret_cast<char*>(p->d_pair_in + off) + b, std::min(kChunk, bytes - b)});
  };
  add_in(sino1, 0);
  if (sino2) add_in(sino2, slice);
  struct OutChunk {
    int image, r0, r1;
  };
  std::vector<OutChunk> out;
  const int rows_per = (int)std::max<size_t>(1, kChunk / ((size_t)p->M0 * sizeof(float)));
  for (int i = 0; i < n_valid; ++i)
    for (int r = 0; r < p->M0; r += rows_per) out.push_back({i, r, std::min(p->M0, r + rows_per)});
  while (p->pair_events.size() < out.size()) {
    cudaEvent_t e = nullptr;
    GR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    p->pair_events.push_back(e);
  }
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int T = std::max(1, std::min({8, hw / 2, (int)std::max(in.size(), out.size())}));
  std::mutex mu;
  std::condition_variable cv;
  int h2d_left = T, stage = 0;  // stage 1: images queued; -1: give up
  std::atomic<int> cuda_err{0};
  float* outs[2] = {out1, out2};
  auto h2d = [&](int t) {
    for (size_t k = (size_t)t; k < in.size(); k += (size_t)T) {
      std::memcpy(in[k].pin, in[k].src, in[k].n);
      if (cudaMemcpyAsync(in[k].dev, in[k].pin, in[k].n, cudaMemcpyHostToDevice, st) != cudaSuccess)
        cuda_err = 1;
    }
    std::lock_guard<std::mutex> lk(mu);
    if (--h2d_left == 0) cv.notify_all();
  };
  auto d2h = [&](int t) {
    for (size_t k = (size_t)t; k < out.size(); k += (size_t)T) {
      if (cudaEventSynchronize(p->pair_events[k]) != cudaSuccess) {
        cuda_err = 1;
        continue;
      }
      const OutChunk& c = out[k];
      const float* src = p->h_pair_out + (size_t)c.image * img;
      for (int r = c.r0; r < c.r1; ++r)
        std::memcpy(outs[c.image] + (size_t)r * out_stride, src + (size_t)r * p->M0,
                    (size_t)p->M0 * sizeof(float));
    }
  };
  std::vector<std::thread> pool;
  try {
    for (int t = 1; t < T; ++t)
      pool.emplace_back([&, t] {
        cudaSetDevice(p->device);
        h2d(t);
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stage != 0; });
        const bool go = stage > 0;
        lk.unlock();
        if (go) d2h(t);
      });
  } catch (...) {  // no thread to be had: the started ones stop after their copies in
    {               // (the caller synchronises the stream on the error)
      std::lock_guard<std::mutex> lk(mu);
      stage = -1;
    }
    cv.notify_all();
    for (auto& th : pool) th.join();
    return fail(GR_ERR_CUDA, "host threads for the pair's staged copies could not be started");
  }
  h2d(0);
  int rc = GR_OK;
  {
    std::unique_lock<std::mutex> lk(mu);
    cv.wait(lk, [&] { return h2d_left == 0; });
  }
  if (cuda_err) rc = fail(GR_ERR_CUDA, "staged host-to-device copy failed");
  if (rc == GR_OK)
    rc = launch_chunk(p, 1, n_valid, 0, p->d_pair_in, p->d_pair_in + slice, 0, GR_DTYPE_F32,
                      nullptr, nullptr, nullptr, 0, p->d_pair_out, p->d_pair_out + img, 0, p->M0, st);
  for (size_t k = 0; k < out.size() && rc == GR_OK; ++k) {
    const OutChunk& c = out[k];
    const size_t off = (size_t)c.image * img + (size_t)c.r0 * p->M0;
    const size_t n = (size_t)(c.r1 - c.r0) * p->M0 * sizeof(float);
    if (cudaMemcpyAsync(p->h_pair_out + off, p->d_pair_out + off, n, cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaEventRecord(p->pair_events[k], st) != cudaSuccess)
      rc = fail(GR_ERR_CUDA, "staged device-to-host copy: %s", cudaGetErrorString(cudaGetLastError()));
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    stage = rc == GR_OK ? 1 : -1;
  }
  cv.notify_all();
  if (rc == GR_OK) d2h(0);
  for (auto& th : pool) th.join();
  if (rc == GR_OK && cuda_err) rc = fail(GR_ERR_CUDA, "staged device-to-host copy failed");
  return rc;
}

}  // namespace
}  // namespace gr

using gr::Plan;
struct gr_plan : public Plan {};

struct gr_graph {
  int device = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long launches = 0;
  std::vector<gr_plan*> plans;  // the plans whose buffers the graph replays
  bool dead = false;            // a plan it replays was destroyed: launch refused
};

namespace gr {
int plan_shape(const gr_plan* p, int* n_det, int* n_ang, int* M0, int* max_pairs, int* device) {
  if (!p) return fail(GR_ERR_ARG, "null plan");
  *n_det = p->n_det;
  *n_ang = p->n_ang;
  *M0 = p->M0;
  *max_pairs = p->max_pairs;
  *device = p->device;
  return GR_OK;
}

int plan_scratch(gr_plan* p, size_t bytes, void** out) {
  if (bytes > p->prep_bytes) {
    if (p->d_prep) cudaFree(p->d_prep);  // synchronises with work still using it
    p->d_prep = nullptr;
    p->prep_bytes = 0;
    cudaError_t e = cudaMalloc(&p->d_prep, bytes);
    if (e != cudaSuccess) {
      p->d_prep = nullptr;
      return fail(GR_ERR_NOMEM, "cudaMalloc(%zu bytes) for pipeline scratch: %s", bytes,
                  cudaGetErrorString(e));
    }
    p->prep_bytes = bytes;
  }
  *out = p->d_prep;
  return GR_OK;
}
}  // namespace gr

extern "C" {

const char* gr_last_error(void) { return gr::g_err.c_str(); }

int gr_filter_code(const char* name) {
  if (!name) return GR_FILTER_SHEPP_LOGAN;
  struct { const char* n; int c; } tbl[] = {{"shlo", 1}, {"shepp", 1}, {"hann", 2}, {"hamm", 3},
                                            {"hamming", 3}, {"ramp", 4}, {"ramlak", 4},
                                            {"none", 0}};
  for (auto& e : tbl)
    if (!std::strcmp(name, e.n)) return e.c;
  return GR_FILTER_SHEPP_LOGAN;
}

int gr_params_default(gr_params* p, int n_det, int n_ang, const float* theta_deg) {
  if (!p) return gr::fail(GR_ERR_ARG, "null params");
  std::memset(p, 0, sizeof(*p));
  p->n_det = n_det;
  p->n_ang = n_ang;
  p->theta_deg = theta_deg;
  p->center = -1.0f;
  p->filter = GR_FILTER_SHEPP_LOGAN;
  p->pswf_c = 6.0f;
  p->sampl = 1.0f;
  p->ltbl = 512;
  p->max_pairs = 1;
  p->device = 0;
  p->roi_size = 1.0f;
  p->pixel_size = 1.0f;
  return GR_OK;
}

int gr_plan_destroy(gr_plan* plan) {
  if (!plan) return GR_OK;
  gr::DeviceGuard g(plan->device);
  // graphs that replay this plan can no longer run; they forget the plan so
  // that destroying them later touches nothing freed here
  for (gr_graph* gg : plan->graphs) {
    gg->dead = true;
    gg->plans.erase(std::find(gg->plans.begin(), gg->plans.end(), plan));
  }
  for (const auto& x : plan->allocs) cudaFree(x.first);
  for (int b = 0; b < 2; ++b) {
    if (plan->h_in[b]) cudaFreeHost(plan->h_in[b]);
    if (plan->h_out[b]) cudaFreeHost(plan->h_out[b]);
    if (plan->d_in[b]) cudaFree(plan->d_in[b]);
    if (plan->d_out[b]) cudaFree(plan->d_out[b]);
    if (plan->ev_h2d[b]) cudaEventDestroy(plan->ev_h2d[b]);
    if (plan->ev_comp[b]) cudaEventDestroy(plan->ev_comp[b]);
    if (plan->ev_d2h[b]) cudaEventDestroy(plan->ev_d2h[b]);
  }
  if (plan->h_pair_in) cudaFreeHost(plan->h_pair_in);
  if (plan->h_pair_out) cudaFreeHost(plan->h_pair_out);
  for (cudaEvent_t e : plan->pair_events) cudaEventDestroy(e);
  if (plan->copy_stream) cudaStreamDestroy(plan->copy_stream);
  if (plan->d2h_stream) cudaStreamDestroy(plan->d2h_stream);
  for (cudaEvent_t e : plan->events) cudaEventDestroy(e);
  if (plan->d_prep) cudaFree(plan->d_prep);
  delete plan;
  return GR_OK;
}

int gr_plan_create(const gr_params* prm, gr_plan** out) {
  return gr::plan_create_ex(prm, nullptr, nullptr, out);
}

}  // extern "C"

int gr::plan_create_ex(const gr_params* prm, const Pswf* pswf, float (*filter_fn)(float),
                       gr_plan** out) {
  using namespace gr;
  if (!out) return fail(GR_ERR_ARG, "null argument");
  *out = nullptr;
  const Pswf* pw = nullptr;
  int rc = check_params(prm, &pw, pswf);
  if (rc) return rc;
  Geometry geo;
  if ((rc = geometry(prm, pw, &geo))) return rc;
  int ndev = 0;
  GR_CUDA(cudaGetDeviceCount(&ndev));
  if (prm->device < 0 || prm->device >= ndev)
    return fail(GR_ERR_ARG, "device %d out of range (%d devices)", prm->device, ndev);
  DeviceGuard guard(prm->device);
  GR_CUDA(init_kernel_attributes());

  gr_plan* p = new gr_plan();
  p->device = prm->device;
  p->n_det = prm->n_det;
  p->n_ang = prm->n_ang;
  p->ltbl = prm->ltbl;
  p->filter = prm->filter;
  p->max_pairs = prm->max_pairs;
  p->wide_mode = prm->wide_grid;
  p->center = prm->center < 0 ? (float)(prm->n_det / 2) : prm->center;
  const long pdim = geo.pdim, M = geo.M, M02 = geo.M02;
  p->pdim = (int)pdim;
  p->J = (int)(pdim / 2);
  p->M = (int)M;
  p->M02 = (int)M02;
  p->M0 = (int)geo.M0;
  p->sampl = geo.sampl;
  p->C = pw->C;
  p->lmbda = pw->lmbda;
  p->L = geo.L;
  p->scale = geo.scale;
  p->ntaps = geo.ntaps;
  // PSWF tables (pswf_su, gridrec.cu:807-857), FP64 then rounded once
  std::vector<double> wtbl(p->ltbl + 1), winv(p->M0);
  const double polyz = legendre_even(*pw, 0.0);
  wtbl[0] = 1.0;
  for (int i = 1; i <= p->ltbl; ++i) wtbl[i] = legendre_even(*pw, (double)i / p->ltbl) / polyz;
  {
    const double fac = (double)p->ltbl / (M02 + 0.5);
    double norm = std::sqrt(M_PI / 2 / pw->C / pw->lmbda) / p->sampl;
    winv[M02] = norm / wtbl[0];
    for (long i = 1; i <= M02; ++i) {
      norm = -norm;
      winv[M02 + i] = winv[M02 - i] = norm / wtbl[(long)(i * fac + 0.5)];
    }
  }
  p->h_wtbl = wtbl;
  p->h_winv = winv;
  std::vector<float> fw(wtbl.begin(), wtbl.end()), fi(winv.begin(), winv.end());
  // filter x normalisation (filphase_su magnitude, gridrec.cu:789-797)
  std::vector<float> filt(p->J);
  const double norm = M_PI / pdim / prm->n_ang;
  for (int j = 0; j < p->J; ++j)
    filt[j] = filter_fn  // a caller's filter function, sampled as filphase_su does (grid.cpp:437-461)
                  ? (float)((double)filter_fn((float)j / (float)pdim) * norm)
                  : (float)(filter_value(prm->filter, (double)j / pdim) * norm);
  // two-level twiddle table of exp(+2 pi i e/N): lo[e] for e < 64, then
  // hi[f] = exp(+2 pi i 64 f/N) for f < max(1, N/64); FP64, rounded once
  auto twiddles = [](int N) {
    const int nhi = std::max(1, N / 64);
    std::vector<float2> t(64 + nhi);
    for (int e = 0; e < 64; ++e) {
      const double a = 2.0 * M_PI * e / N;
      t[e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    for (int f = 0; f < nhi; ++f) {
      const double a = 2.0 * M_PI * 64.0 * f / N;
      t[64 + f] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    return t;
  };
  const std::vector<double> dxy = directions(prm, p->scale);
  std::vector<double2> dirs(2 * (size_t)prm->n_ang);
  for (size_t d = 0; d < dirs.size(); ++d) dirs[d] = make_double2(dxy[2 * d], dxy[2 * d + 1]);
  p->dxy = dxy;
  if (prm->roi_x0 != 0.f || prm->roi_y0 != 0.f) {
    // (X0 cos + Y0 sin) pi per angle, from the unscaled direction (GridrecCPP grid.cpp:237)
    std::vector<double> off(prm->n_ang);
    for (int n = 0; n < prm->n_ang; ++n)
      off[n] = ((double)prm->roi_x0 * dxy[4 * n] + (double)prm->roi_y0 * dxy[4 * n + 1]) /
               p->scale * M_PI;
    if ((rc = upload(p, &p->d_roi_off, off))) {
      gr_plan_destroy(p);
      return rc;
    }
  }
  if ((rc = upload(p, &p->d_wtbl, fw)) || (rc = upload(p, &p->d_winv, fi)) ||
      (rc = upload(p, &p->d_filt, filt)) || (rc = upload(p, &p->d_tw_p, twiddles((int)pdim))) ||
      (rc = upload(p, &p->d_tw_m, twiddles((int)M))) || (rc = upload(p, &p->d_dir, dirs)) ||
      (rc = install_work_list(p, kItemCap)) ||
      (p->wide_mode == 2 && (rc = install_work_list_tc(p, kItemCapT))) ||
      ((wide16_possible(p) || w32_possible(p)) && (rc = install_work_list_wide(p, kItemCapW)))) {
    gr_plan_destroy(p);
    return rc;
  }
  const size_t P = (size_t)p->max_pairs;
  // the 16- and 32-pair kernels' spectra layouts hold whole groups of pairs
  const size_t G_spec = p->x_ready ? kW32Pairs : ((p->w_items || p->t_items) ? kWidePairs : 1);
  const size_t P_spec = (P + G_spec - 1) / G_spec * G_spec;
  p->spec_pairs = (int)P_spec;
  if ((rc = dev_alloc(p, &p->d_spec, P_spec * p->n_ang * 2 * p->J)) ||
      (rc = dev_alloc(p, &p->d_H, P * (size_t)M * M)) ||
      (rc = dev_alloc(p, &p->d_pq, P * p->J)) ||
      (rc = dev_alloc(p, &p->d_dl, 2 * P * (size_t)p->n_det)) ||
      (rc = dev_alloc(p, &p->d_queue, 1)) || (rc = dev_alloc(p, &p->d_err, 1))) {
    gr_plan_destroy(p);
    return rc;
  }
  cudaError_t e = cudaMemset(p->d_err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    gr_plan_destroy(p);
    return fail(GR_ERR_CUDA, "plan init: %s", cudaGetErrorString(e));
  }
  *out = p;
  return GR_OK;
}

extern "C" {

static int worklist_export(const gr_params* prm, bool wide, int* n_items, int* n_runs,
                           int* tiles_v, int* items, int* runs, int* splits, int cap_items,
                           int cap_runs) {
  using namespace gr;
  const Pswf* pw = nullptr;
  int rc = check_params(prm, &pw);
  if (rc) return rc;
  Geometry geo;
  if ((rc = geometry(prm, pw, &geo))) return rc;
  WorkList wl;
  build_work_list((int)geo.M, (int)(geo.pdim / 2), geo.L, prm->n_ang, directions(prm, geo.scale),
                  &wl, wide ? kItemCapW : kItemCap, wide ? kListWide : kListTiles);
  if (n_items) *n_items = (int)wl.items.size();
  if (n_runs) *n_runs = (int)wl.runs.size();
  if (tiles_v) *tiles_v = wl.tiles_v;
  if (!items || !runs || !splits) return GR_OK;
  if (cap_items < (int)wl.items.size() || cap_runs < (int)wl.runs.size())
    return fail(GR_ERR_ARG, "work list needs %zu items / %zu runs", wl.items.size(), wl.runs.size());
  std::memcpy(items, wl.items.data(), wl.items.size() * sizeof(Item));
  std::memcpy(runs, wl.runs.data(), wl.runs.size() * sizeof(Run));
  std::memcpy(splits, wl.splits.data(), wl.splits.size() * sizeof(Split));
  return GR_OK;
}

int gr_worklist_export(const gr_params* prm, int* n_items, int* n_runs, int* tiles_v,
                       int* items, int* runs, int* splits, int cap_items, int cap_runs) {
  return worklist_export(prm, false, n_items, n_runs, tiles_v, items, runs, splits, cap_items,
                         cap_runs);
}

int gr_worklist_export_wide(const gr_params* prm, int* n_items, int* n_runs, int* tiles_v,
                            int* items, int* runs, int* splits, int cap_items, int cap_runs) {
  return worklist_export(prm, true, n_items, n_runs, tiles_v, items, runs, splits, cap_items,
                         cap_runs);
}

int gr_plan_grid_kernel(const gr_plan* p, int pairs, int* wide) {
  if (!p || !wide) return gr::fail(GR_ERR_ARG, "null argument");
  const int pr = std::min(std::max(pairs, 1), p->max_pairs);
  *wide = gr::use_tc(p, pr) ? 2 : (gr::use_w32(p, pr) ? 3 : (gr::use_wide(p, pr) ? 1 : 0));
  return GR_OK;
}

int gr_plan_device_status(gr_plan* p, void* stream) {
  using namespace gr;
  if (!p) return fail(GR_ERR_ARG, "null plan");
  DeviceGuard g(p->device);
  GR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  int flag = 0;
  GR_CUDA(cudaMemcpy(&flag, p->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag) {
    GR_CUDA(cudaMemset(p->d_err, 0, sizeof(int)));
    return fail(GR_ERR_TIMEOUT, "a bounded device wait ran out (kernel stopped early)");
  }
  return GR_OK;
}

int gr_selftest_wait_timeout(int device) {
  using namespace gr;
  DeviceGuard g(device);
  int* d = nullptr;
  GR_CUDA(cudaMalloc(&d, sizeof(int)));
  int flag = 0;
  cudaError_t e = cudaMemset(d, 0, sizeof(int));
  if (e == cudaSuccess) e = launch_wait_probe(d, 1 << 12, nullptr);
  if (e == cudaSuccess) e = cudaMemcpy(&flag, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(GR_ERR_CUDA, "wait self-test: %s", cudaGetErrorString(e));
  return flag ? fail(GR_ERR_TIMEOUT, "mbarrier wait ran out as intended (self-test)") : GR_OK;
}

int gr_plan_set_timing(gr_plan* p, int enable) {
  if (!p) return gr::fail(GR_ERR_ARG, "null plan");
  p->timing = enable != 0;
  p->events_used = 0;
  return GR_OK;
}

int gr_plan_stage_times(gr_plan* p, double* ms, long* chunks) {
  using namespace gr;
  if (!p || !ms) return gr::fail(GR_ERR_ARG, "null argument");
  for (int k = 0; k < 5; ++k) ms[k] = 0.0;
  const size_t n = p->events_used / 6;
  if (chunks) *chunks = (long)n;
  if (n == 0) return GR_OK;
  gr::DeviceGuard g(p->device);
  GR_CUDA(cudaEventSynchronize(p->events[6 * n - 1]));
  for (size_t c = 0; c < n; ++c)
    for (int k = 0; k < 5; ++k) {
      float t = 0.f;
      GR_CUDA(cudaEventElapsedTime(&t, p->events[6 * c + k], p->events[6 * c + k + 1]));
      ms[k] += t;
    }
  return GR_OK;
}

int gr_plan_sizes(const gr_plan* p, int* pdim, int* M, int* M0, float* L, float* scale) {
  if (!p) return gr::fail(GR_ERR_ARG, "null plan");
  if (pdim) *pdim = p->pdim;
  if (M) *M = p->M;
  if (M0) *M0 = p->M0;
  if (L) *L = (float)p->L;
  if (scale) *scale = (float)p->scale;
  return GR_OK;
}

int gr_plan_device_bytes(const gr_plan* p, size_t* bytes) {
  if (!p || !bytes) return gr::fail(GR_ERR_ARG, "null argument");
  *bytes = p->device_bytes;
  return GR_OK;
}

int gr_plan_launch_count(const gr_plan* p, long* launches) {
  if (!p || !launches) return gr::fail(GR_ERR_ARG, "null argument");
  *launches = p->launches;
  return GR_OK;
}

int gr_plan_autotune(gr_plan* p, void* stream) {
  using namespace gr;
  if (!p) return fail(GR_ERR_ARG, "null plan");
  if (!p->graphs.empty())
    return fail(GR_ERR_ARG, "autotune replaces buffers that %d live graph(s) replay: tune before "
                "capture", (int)p->graphs.size());
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  // tuned choices depend on the work-list geometry and the chunk size: key on them
  unsigned long long h = 1469598103934665603ull;
  auto mix = [&](unsigned long long v) { h = (h ^ v) * 1099511628211ull; };
  mix((unsigned long long)p->device);
  mix((unsigned long long)p->M);
  mix((unsigned long long)p->J);
  mix((unsigned long long)p->n_ang);
  mix((unsigned long long)p->max_pairs);
  mix((unsigned long long)(p->wide_mode + 1));
  mix((unsigned long long)std::llround(p->L * 1e6));
  for (double d : p->dxy) mix((unsigned long long)std::llround(d * 1e9));
  static std::mutex mu;
  // kernel: gridding kernel of full chunks (-1: the mode's fixed choice); cap_t / cap_w:
  // item caps of the tile and 4 x 8 work lists
  struct Tuned { int kernel, cap_t, cap_w, G, ring; };
  static std::map<unsigned long long, Tuned> cache;
  const int pairs = p->max_pairs;
  // the gridding kernels a full chunk can run: in the default mode every kernel the
  // plan holds records for; in a forced mode the forced one
  std::vector<int> kernels;
  if (p->wide_mode == 0) {
    kernels.push_back(0);
    if (wide16_possible(p) && p->w_items) kernels.push_back(1);
    if (w32_possible(p) && p->x_ready && p->w_items) kernels.push_back(3);
  } else {
    kernels.push_back(use_tc(p, pairs) ? 2 : (use_w32(p, pairs) ? 3 : (use_wide(p, pairs) ? 1 : 0)));
  }
  auto install = [&](int kernel, int cap) -> int {
    if (kernel == 2) return GR_OK;  // the tensor-core list keeps its cap
    if (kernel == 1 || kernel == 3)
      return cap == p->w_item_cap ? GR_OK : install_work_list_wide(p, cap);
    return cap == p->item_cap ? GR_OK : install_work_list(p, cap);
  };
  auto apply = [&](const Tuned& t) -> int {
    int rc = install(0, t.cap_t);
    if (rc == GR_OK && p->w_items) rc = install(1, t.cap_w);
    if (rc == GR_OK) {
      p->cols_G = t.G;
      p->cols_ring = t.ring;
      p->tuned_kernel = p->wide_mode == 0 && kernels.size() > 1 ? t.kernel : -1;
    }
    return rc;
  };
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(h);
    if (it != cache.end()) return apply(it->second);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  GR_CUDA(cudaEventCreate(&e0));
  GR_CUDA(cudaEventCreate(&e1));
  auto time_ms = [&](auto&& launch) -> float {
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
      cudaEventRecord(e0, st);
      launch();
      cudaEventRecord(e1, st);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) best = std::min(best, ms);  // first run warms up
    }
    return best;
  };
  cudaMemsetAsync(p->d_spec, 0, (size_t)p->spec_pairs * p->n_ang * 2 * p->J * sizeof(float2), st);
  cudaMemsetAsync(p->d_H, 0, (size_t)pairs * p->M * p->M * sizeof(float2), st);
  Tuned best{kernels[0], p->item_cap, p->w_item_cap, 0, 0};
  float best_t = 1e30f;
  int best_cap_t = p->item_cap, best_cap_w = p->w_item_cap, rc = GR_OK;
  float best_tt = 1e30f, best_tw = 1e30f;
  const int saved = p->tuned_kernel;
  for (int kernel : kernels) {
    if (kernel == 2) {  // forced tensor-core mode: nothing to choose in the gridding
      best.kernel = 2;
      break;
    }
    const bool wl4x8 = kernel != 0;
    const std::vector<int> caps = wl4x8 ? std::vector<int>{256, 512, 1024, 2048, 4096}
                                        : std::vector<int>{512, 1024, 2048, 4096, 8192};
    for (int cap : caps) {
      if ((rc = install(kernel, cap))) break;
      const GridArgs ga =
          kernel == 3 ? grid_args_w32(p, pairs) : grid_args(p, pairs, kernel == 1);
      const float t = time_ms([&] {
        if (kernel == 3) launch_grid_w32(ga, st);
        else if (kernel == 1) launch_grid_wide(ga, st);
        else launch_grid(ga, p->ntaps, st);
      });
      if (wl4x8 && t < best_tw) {
        best_tw = t;
        best_cap_w = cap;
      }
      if (!wl4x8 && t < best_tt) {
        best_tt = t;
        best_cap_t = cap;
      }
      if (t < best_t) {
        best_t = t;
        best.kernel = kernel;
      }
    }
    if (rc) break;
  }
  p->tuned_kernel = saved;
  best.cap_t = best_cap_t;
  best.cap_w = best_cap_w;
  if (rc == GR_OK) rc = apply(best);
  int best_G = 0, best_ring = 0;
  float best_c = 1e30f;
  for (int G = 1; G <= 8 && rc == GR_OK; G *= 2) {
    const int threads = G * (p->M / 16);
    // up to 1024 threads (the TMA-fed kernel); the plain one stops at 512
    if (threads < 32 || threads > 1024 || p->M % G) continue;
    for (int ring = 0; ring < 2; ++ring) {
      ColArgs ca{p->d_H, p->d_tw_m, p->M, pairs, p->d_err, G, ring};
      const float t = time_ms([&] { launch_cols(ca, st); });
      if (t < best_c) {
        best_c = t;
        best_G = G;
        best_ring = ring;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaError_t e = cudaGetLastError();
  if (rc == GR_OK && e != cudaSuccess) rc = fail(GR_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
  if (rc == GR_OK) {
    best.G = best_G;
    best.ring = best_ring;
    p->cols_G = best_G;
    p->cols_ring = best_ring;
    std::lock_guard<std::mutex> lk(mu);
    cache[h] = best;
  }
  return rc;
}

int gr_plan_set_tuning(gr_plan* p, int grid_kernel, int item_cap, int cols_group, int cols_ring) {
  using namespace gr;
  if (!p) return fail(GR_ERR_ARG, "null plan");
  if (!p->graphs.empty())
    return fail(GR_ERR_ARG, "set_tuning replaces buffers that %d live graph(s) replay",
                (int)p->graphs.size());
  const bool ok_kernel =
      grid_kernel < 0 ||
      (p->wide_mode == 0 &&
       (grid_kernel == 0 || (grid_kernel == 1 && wide16_possible(p) && p->w_items) ||
        (grid_kernel == 3 && w32_possible(p) && p->x_ready && p->w_items)));
  if (!ok_kernel)
    return fail(GR_ERR_ARG, "grid kernel %d is not available on this plan (wide_grid %d, "
                "max_pairs %d)", grid_kernel, p->wide_mode, p->max_pairs);
  if (item_cap != 0 && (item_cap < 64 || item_cap > (1 << 20)))
    return fail(GR_ERR_ARG, "item cap %d outside 64 .. 2^20 (0: keep)", item_cap);
  if (cols_group != 0) {
    const int threads = cols_group * (p->M / 16);
    if (cols_group < 1 || (cols_group & (cols_group - 1)) || cols_group > 8 || threads < 32 ||
        threads > 1024 || p->M % cols_group)
      return fail(GR_ERR_ARG, "column group %d not valid for M = %d", cols_group, p->M);
  }
  DeviceGuard g(p->device);
  p->tuned_kernel = grid_kernel;
  const int k = grid_kernel >= 0 ? grid_kernel : (use_w32(p, p->max_pairs) ? 3 : (use_wide(p, p->max_pairs) ? 1 : 0));
  int rc = GR_OK;
  if (item_cap > 0) {
    if (k == 0 && item_cap != p->item_cap) rc = install_work_list(p, item_cap);
    if ((k == 1 || k == 3) && item_cap != p->w_item_cap) rc = install_work_list_wide(p, item_cap);
  }
  if (rc == GR_OK && cols_group > 0) p->cols_G = cols_group;
  if (rc == GR_OK && cols_ring >= 0) p->cols_ring = cols_ring ? 1 : 0;
  return rc;
}

int gr_plan_tuning_ex(const gr_plan* p, int* grid_kernel, int* item_cap, int* cols_group,
                      int* cols_ring) {
  if (!p) return gr::fail(GR_ERR_ARG, "null plan");
  if (grid_kernel) {
    const int pr = p->max_pairs;
    *grid_kernel = gr::use_tc(p, pr) ? 2 : (gr::use_w32(p, pr) ? 3 : (gr::use_wide(p, pr) ? 1 : 0));
  }
  if (cols_ring) *cols_ring = p->cols_ring;
  return gr_plan_tuning(p, item_cap, cols_group);
}

int gr_plan_tuning(const gr_plan* p, int* item_cap, int* cols_group_width) {
  if (!p) return gr::fail(GR_ERR_ARG, "null plan");
  // the item cap of the work list a full chunk grids with
  const bool wl4x8 = gr::use_wide(p, p->max_pairs) || gr::use_w32(p, p->max_pairs);
  if (item_cap) *item_cap = wl4x8 ? p->w_item_cap : p->item_cap;
  if (cols_group_width) *cols_group_width = p->cols_G > 0 ? p->cols_G : gr::cols_group(p->M);
  return GR_OK;
}

int gr_plan_work_stats(const gr_plan* p, int* n_items, int* n_runs, int* n_slots,
                       long* total_samples) {
  if (!p) return gr::fail(GR_ERR_ARG, "null plan");
  if (n_items) *n_items = p->n_items;
  if (n_runs) *n_runs = p->n_runs;
  if (n_slots) *n_slots = p->n_slots;
  if (total_samples) *total_samples = p->total_samples;
  return GR_OK;
}

int gr_reconstruct_pair(gr_plan* p, const float* sino1, const float* sino2, float* out1,
                        float* out2, long out_stride, void* stream) {
  using namespace gr;
  if (!p || !sino1 || !out1) return fail(GR_ERR_ARG, "null argument");
  if (out_stride < p->M0) return fail(GR_ERR_ARG, "out_stride %ld < M0 %d", out_stride, p->M0);
  DeviceGuard g(p->device);
  const int n_valid = (sino2 && out2) ? 2 : 1;
  return launch_chunk(p, 1, n_valid, 0, sino1, sino2 ? sino2 : sino1, 0, GR_DTYPE_F32, nullptr,
                      nullptr, nullptr, 0, out1, out2 ? out2 : out1, 0, out_stride,
                      (cudaStream_t)stream);
}

int gr_reconstruct_pair_host(gr_plan* p, const float* sino1, const float* sino2, float* out1,
                             float* out2, long out_stride, void* stream) {
  using namespace gr;
  if (!p || !sino1 || !out1) return fail(GR_ERR_ARG, "null argument");
  if (out_stride < p->M0) return fail(GR_ERR_ARG, "out_stride %ld < M0 %d", out_stride, p->M0);
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t slice = (size_t)p->n_ang * p->n_det, img = (size_t)p->M0 * p->M0;
  int rc;
  if (!p->d_pair_in && ((rc = dev_alloc(p, &p->d_pair_in, 2 * slice)) ||
                        (rc = dev_alloc(p, &p->d_pair_out, 2 * img))))
    return rc;
  const int n_valid = (sino2 && out2) ? 2 : 1;
  const size_t out_span = ((size_t)(p->M0 - 1) * out_stride + p->M0) * sizeof(float);
  if (is_pinned(sino1, slice * sizeof(float)) && (!sino2 || is_pinned(sino2, slice * sizeof(float))) &&
      is_pinned(out1, out_span) && (!out2 || is_pinned(out2, out_span))) {
    // pinned caller buffers: straight to and from the device, the images with the
    // caller's row stride
    GR_CUDA(cudaMemcpyAsync(p->d_pair_in, sino1, slice * sizeof(float), cudaMemcpyHostToDevice, st));
    if (sino2)
      GR_CUDA(cudaMemcpyAsync(p->d_pair_in + slice, sino2, slice * sizeof(float),
                              cudaMemcpyHostToDevice, st));
    rc = launch_chunk(p, 1, n_valid, 0, p->d_pair_in, p->d_pair_in + slice, 0, GR_DTYPE_F32, nullptr,
                      nullptr, nullptr, 0, p->d_pair_out, p->d_pair_out + img, 0, p->M0, st);
    if (rc) return rc;
    const size_t row = (size_t)p->M0 * sizeof(float);
    GR_CUDA(cudaMemcpy2DAsync(out1, (size_t)out_stride * sizeof(float), p->d_pair_out, row, row,
                              p->M0, cudaMemcpyDeviceToHost, st));
    if (out2 && n_valid == 2)
      GR_CUDA(cudaMemcpy2DAsync(out2, (size_t)out_stride * sizeof(float), p->d_pair_out + img, row,
                                row, p->M0, cudaMemcpyDeviceToHost, st));
    return gr_plan_device_status(p, stream);  // synchronises the stream
  }
  rc = pair_host_staged(p, sino1, sino2, out1, out2, out_stride, st, n_valid);
  if (rc) {
    cudaStreamSynchronize(st);
    return rc;
  }
  return gr_plan_device_status(p, stream);
}

int gr_reconstruct_batch(gr_plan* p, const gr_batch_desc* b, void* stream) {
  using namespace gr;
  if (!p) return fail(GR_ERR_ARG, "null plan");
  int rc = validate_batch(p, b);
  if (rc) return rc;
  DeviceGuard g(p->device);
  const size_t es = dtype_size(b->dtype);
  const long slice_in = (long)p->n_ang * p->n_det;
  const long slice_out = (long)p->M0 * b->out_stride;
  const int n_pairs = (b->n_slices + 1) / 2;
  for (int c0 = 0; c0 < n_pairs; c0 += p->max_pairs) {
    const int pairs = std::min(p->max_pairs, n_pairs - c0);
    const int s0 = 2 * c0;
    const int n_valid = std::min(2 * pairs, b->n_slices - s0);
    const char* base = static_cast<const char*>(b->sinos) + (size_t)s0 * slice_in * es;
    float* ob = b->outs + (size_t)s0 * slice_out;
    rc = launch_chunk(p, pairs, n_valid, s0, base, base + slice_in * es, 2 * slice_in,
                      b->dtype, b->centers, b->flat, b->dark, b->flat_stride, ob, ob + slice_out,
                      2 * slice_out,
                      b->out_stride, (cudaStream_t)stream);
    if (rc) return rc;
  }
  return GR_OK;
}

int gr_reconstruct_host(gr_plan* p, const gr_batch_desc* b, void* stream) {
  using namespace gr;
  if (!p) return fail(GR_ERR_ARG, "null plan");
  int rc = validate_batch(p, b);
  if (rc) return rc;
  DeviceGuard g(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t es = dtype_size(b->dtype);
  const size_t slice_in = (size_t)p->n_ang * p->n_det * es;
  const size_t slice_out = (size_t)p->M0 * b->out_stride * sizeof(float);
  const size_t in_bytes = 2 * (size_t)p->max_pairs * slice_in;
  const size_t out_bytes = 2 * (size_t)p->max_pairs * slice_out;
  // pinned user buffers are copied directly; pageable ones go through staging
  auto is_pinned = [](const void* ptr) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return at.type == cudaMemoryTypeHost;
  };
  const bool in_pinned = is_pinned(b->sinos);
  const bool out_pinned = is_pinned(b->outs);
  if (!p->copy_stream) {
    GR_CUDA(cudaStreamCreateWithFlags(&p->copy_stream, cudaStreamNonBlocking));
    GR_CUDA(cudaStreamCreateWithFlags(&p->d2h_stream, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) {
      GR_CUDA(cudaEventCreateWithFlags(&p->ev_h2d[k], cudaEventDisableTiming));
      GR_CUDA(cudaEventCreateWithFlags(&p->ev_comp[k], cudaEventDisableTiming));
      GR_CUDA(cudaEventCreateWithFlags(&p->ev_d2h[k], cudaEventDisableTiming));
    }
  }
  if (p->in_bytes < in_bytes || p->out_bytes < out_bytes) {
    for (int k = 0; k < 2; ++k) {
      if (p->h_in[k]) cudaFreeHost(p->h_in[k]);
      if (p->h_out[k]) cudaFreeHost(p->h_out[k]);
      if (p->d_in[k]) cudaFree(p->d_in[k]);
      if (p->d_out[k]) cudaFree(p->d_out[k]);
      p->h_in[k] = p->h_out[k] = nullptr;
      p->d_in[k] = p->d_out[k] = nullptr;
    }
    for (int k = 0; k < 2; ++k) {
      if (cudaMallocHost(&p->h_in[k], in_bytes) != cudaSuccess ||
          cudaMallocHost((void**)&p->h_out[k], out_bytes) != cudaSuccess ||
          cudaMalloc(&p->d_in[k], in_bytes) != cudaSuccess ||
          cudaMalloc((void**)&p->d_out[k], out_bytes) != cudaSuccess) {
        cudaGetLastError();
        p->in_bytes = p->out_bytes = 0;
        return fail(GR_ERR_NOMEM, "staging buffers (%zu + %zu bytes x 2)", in_bytes, out_bytes);
      }
    }
    p->in_bytes = in_bytes;
    p->out_bytes = out_bytes;
  }
  // per-slice centres are small: upload once to the device
  float* d_centers = nullptr;
  float* d_flat = nullptr;
  float* d_dark = nullptr;
  auto cleanup = [&]() {
    if (d_centers) cudaFree(d_centers);
    if (d_flat) cudaFree(d_flat);
    if (d_dark) cudaFree(d_dark);
  };
  if (b->centers) {
    GR_CUDA(cudaMalloc(&d_centers, b->n_slices * sizeof(float)));
    GR_CUDA(cudaMemcpy(d_centers, b->centers, b->n_slices * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (b->dtype == GR_DTYPE_U16_RAW || b->dtype == GR_DTYPE_U16_LINEAR) {
    const size_t nf = (size_t)(b->n_slices - 1) * b->flat_stride + p->n_det;
    GR_CUDA(cudaMalloc(&d_flat, nf * sizeof(float)));
    GR_CUDA(cudaMalloc(&d_dark, nf * sizeof(float)));
    GR_CUDA(cudaMemcpy(d_flat, b->flat, nf * sizeof(float), cudaMemcpyHostToDevice));
    GR_CUDA(cudaMemcpy(d_dark, b->dark, nf * sizeof(float), cudaMemcpyHostToDevice));
  }
  const int n_pairs = (b->n_slices + 1) / 2;
  const int n_chunks = (n_pairs + p->max_pairs - 1) / p->max_pairs;
  struct Pending { int chunk = -1; size_t bytes = 0; size_t off = 0; };
  Pending pend[2];
  auto finish = [&](int k) -> int {  // copy a finished chunk's images to the user
    if (pend[k].chunk < 0) return GR_OK;
    GR_CUDA(cudaEventSynchronize(p->ev_d2h[k]));
    if (!out_pinned)
      std::memcpy(reinterpret_cast<char*>(b->outs) + pend[k].off, p->h_out[k], pend[k].bytes);
    pend[k].chunk = -1;
    return GR_OK;
  };
  for (int c = 0; c < n_chunks; ++c) {
    const int k = c & 1;
    const int c0 = c * p->max_pairs;
    const int pairs = std::min(p->max_pairs, n_pairs - c0);
    const int s0 = 2 * c0;
    const int n_valid = std::min(2 * pairs, b->n_slices - s0);
    const size_t ib = (size_t)n_valid * slice_in, ob = (size_t)n_valid * slice_out;
    const char* src = static_cast<const char*>(b->sinos) + (size_t)s0 * slice_in;
    if ((rc = finish(k))) { cleanup(); return rc; }
    // the staging input k was last read by the H2D of chunk c-2 (finished:
    // its D2H completed above); the device input k by the kernels of chunk c-2
    GR_CUDA(cudaStreamWaitEvent(p->copy_stream, p->ev_comp[k], 0));
    if (in_pinned) {
      GR_CUDA(cudaMemcpyAsync(p->d_in[k], src, ib, cudaMemcpyHostToDevice, p->copy_stream));
    } else {
      std::memcpy(p->h_in[k], src, ib);
      GR_CUDA(cudaMemcpyAsync(p->d_in[k], p->h_in[k], ib, cudaMemcpyHostToDevice, p->copy_stream));
    }
    GR_CUDA(cudaEventRecord(p->ev_h2d[k], p->copy_stream));
    GR_CUDA(cudaStreamWaitEvent(st, p->ev_h2d[k], 0));
    // the device output k was last read by the D2H of chunk c-2 (complete)
    const char* dbase = static_cast<const char*>(p->d_in[k]);
    const long slice_in_el = (long)p->n_ang * p->n_det;
    const long slice_out_el = (long)p->M0 * b->out_stride;
    rc = launch_chunk(p, pairs, n_valid, s0, dbase, dbase + slice_in, 2 * slice_in_el, b->dtype,
                      d_centers, d_flat, d_dark, b->flat_stride, p->d_out[k],
                      p->d_out[k] + slice_out_el,
                      2 * slice_out_el, b->out_stride, st);
    if (rc) { cleanup(); return rc; }
    GR_CUDA(cudaEventRecord(p->ev_comp[k], st));
    GR_CUDA(cudaStreamWaitEvent(p->d2h_stream, p->ev_comp[k], 0));
    char* dst = out_pinned ? reinterpret_cast<char*>(b->outs) + (size_t)s0 * slice_out
                           : reinterpret_cast<char*>(p->h_out[k]);
    GR_CUDA(cudaMemcpyAsync(dst, p->d_out[k], ob, cudaMemcpyDeviceToHost, p->d2h_stream));
    GR_CUDA(cudaEventRecord(p->ev_d2h[k], p->d2h_stream));
    pend[k].chunk = c;
    pend[k].bytes = ob;
    pend[k].off = (size_t)s0 * slice_out;
  }
  for (int k = 0; k < 2; ++k)
    if ((rc = finish(k))) { cleanup(); return rc; }
  GR_CUDA(cudaStreamSynchronize(st));
  cleanup();
  return gr_plan_device_status(p, stream);
}

}  // extern "C"

// ------------------------------------------------------------------ allocation-free pair entry
// gr_reconstruct_pair_noalloc keeps every per-call intermediate (phase
// ramps, filtered spectra, frequency grid, partial tiles of split tiles,
// work-queue head) in one file-scope device array instead of the plan's
// cudaMalloc'd workspaces.  Every GPU that loads the library holds the array
// until the process exits; all calls on a device share it.

namespace gr {
namespace {

constexpr size_t kNoallocBytes = size_t(32) << 20;  // 32 MiB per device
constexpr int kNoallocMaxDevices = 64;

}  // namespace
}  // namespace gr

static __device__ __align__(256) unsigned char g_noalloc_scratch[gr::kNoallocBytes];

namespace gr {
namespace {

std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoallocMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (the array's
// name in host code is only a stand-in).  Looked up once per device.
int noalloc_scratch(int dev, unsigned char** ptr) {
  if (dev < 0 || dev >= kNoallocMaxDevices)
    return fail(GR_ERR_UNSUPPORTED, "device %d: static scratch covers devices 0..%d", dev,
                kNoallocMaxDevices - 1);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* a = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
    if (e != cudaSuccess)
      return fail(GR_ERR_CUDA, "cudaGetSymbolAddress(static scratch) failed: %s",
                  cudaGetErrorString(e));
    g_noalloc_addr[dev] = a;
  }
  *ptr = static_cast<unsigned char*>(g_noalloc_addr[dev]);
  return GR_OK;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace gr

extern "C" int gr_reconstruct_pair_noalloc(gr_plan* p, const float* sino1, const float* sino2,
                                           float* out1, float* out2, long out_stride,
                                           void* stream) {
  using namespace gr;
  if (!p || !sino1 || !out1) return fail(GR_ERR_ARG, "null argument");
  if (out_stride < p->M0) return fail(GR_ERR_ARG, "out_stride %ld < M0 %d", out_stride, p->M0);
  // carve the static array: ramps | spectra | grid | partial tiles | queue head
  const size_t off_pq = 0;
  const size_t off_spec = align256(off_pq + (size_t)p->J * sizeof(float4));
  const size_t off_H = align256(off_spec + (size_t)p->n_ang * 2 * p->J * sizeof(float2));
  const size_t off_part = align256(off_H + (size_t)p->M * p->M * sizeof(float2));
  const size_t off_queue =
      align256(off_part + (size_t)std::max(p->n_slots, 1) * kTile * kTile * sizeof(float4));
  const size_t need = off_queue + sizeof(unsigned);
  if (need > kNoallocBytes)
    return fail(GR_ERR_UNSUPPORTED,
                "gr_reconstruct_pair_noalloc: %d x %d needs %zu bytes of scratch, the static "
                "array holds %zu; use gr_reconstruct_pair",
                p->n_det, p->n_ang, need, kNoallocBytes);
  DeviceGuard g(p->device);
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(p->device, &base);
  if (rc) return rc;
  float4* pq = reinterpret_cast<float4*>(base + off_pq);
  float2* spec = reinterpret_cast<float2*>(base + off_spec);
  float2* H = reinterpret_cast<float2*>(base + off_H);
  float4* part = reinterpret_cast<float4*>(base + off_part);
  unsigned* queue = reinterpret_cast<unsigned*>(base + off_queue);
  cudaStream_t st = (cudaStream_t)stream;
  const int n_valid = (sino2 && out2) ? 2 : 1;
  const void* s2 = sino2 ? sino2 : sino1;
  float* o2 = out2 ? out2 : out1;
  // the same five kernels as gr_reconstruct_pair, one pair, workspaces above;
  // launch_grid zeroes the queue head in-stream before the gridding kernel
  PhaseArgs ph{nullptr, p->center, 0, n_valid, p->d_filt, pq, p->J, p->pdim, 1};
  GR_CUDA(launch_phase(ph, st));
  SpectraArgs sa{sino1, s2, 0, n_valid, 0, nullptr, nullptr, 0, pq, spec, p->d_tw_p, p->n_det,
                 p->n_ang, p->pdim, p->J, 1, p->d_roi_off};
  GR_CUDA(launch_spectra(sa, GR_DTYPE_F32, st));
  GridArgs ga{spec, H, part, queue, p->d_items, p->d_runs, p->d_split_list, p->n_split_tiles,
              p->d_dir, p->d_wtbl, p->n_items, 1, p->n_ang, p->J, p->M, p->tiles_v, p->n_slots,
              p->ltbl, p->L / 2, 2.0 * p->ltbl / p->L};
  GR_CUDA(launch_grid(ga, p->ntaps, st));
  // the plan's own error word (allocated with the plan): a bounded-wait timeout of
  // the column FFT is reported by gr_plan_device_status, as for the plan's other calls
  ColArgs ca{H, p->d_tw_m, p->M, 1, p->d_err, p->cols_G, p->cols_ring};
  GR_CUDA(launch_cols(ca, st));
  RowArgs ra{H, p->d_tw_m, p->d_winv, out1, o2, 0, out_stride, n_valid, p->M, p->M0, p->M02, 1};
  GR_CUDA(launch_rows(ra, st));
  // phase, spectra, grid (+ split reduction when tiles are split), cols, rows
  p->launches += 5 + (ga.n_items > 0 && ga.n_split_tiles > 0 ? 1 : 0);
  return GR_OK;
}

// ------------------------------------------------------------------ CUDA graphs
// A graph holds the launches of one or more batches, recorded once by stream
// capture and replayed with one cudaGraphLaunch.  Batches of one plan run in
// order on one branch (they share its workspaces); different plans get their
// own branches, forked from and joined to the capture stream, so batches of
// different shapes can overlap on the GPU.


extern "C" {

int gr_graph_create(const gr_graph_item* items, int n_items, gr_graph** out) {
  using namespace gr;
  if (!items || n_items < 1 || !out) return fail(GR_ERR_ARG, "graph: items and out required");
  *out = nullptr;
  const int dev = items[0].plan ? items[0].plan->device : -1;
  std::vector<gr_plan*> plans;
  for (int i = 0; i < n_items; ++i) {
    gr_plan* p = items[i].plan;
    if (!p) return fail(GR_ERR_ARG, "graph: item %d has no plan", i);
    if (p->device != dev) return fail(GR_ERR_ARG, "graph: all plans must be on one device");
    if (p->timing) return fail(GR_ERR_ARG, "graph: disable stage timing before capture");
    int rc = validate_batch(p, &items[i].batch);
    if (rc) return rc;
    if (std::find(plans.begin(), plans.end(), p) == plans.end()) plans.push_back(p);
  }
  DeviceGuard g(dev);
  const size_t np = plans.size();
  cudaStream_t s0 = nullptr;
  std::vector<cudaStream_t> br(np, nullptr);
  std::vector<cudaEvent_t> join(np, nullptr);
  cudaEvent_t fork = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  auto cleanup = [&]() {
    for (auto s : br)
      if (s) cudaStreamDestroy(s);
    for (auto e : join)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (s0) cudaStreamDestroy(s0);
  };
  cudaError_t e = cudaStreamCreateWithFlags(&s0, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  for (size_t k = 0; k < np && e == cudaSuccess; ++k) {
    e = cudaStreamCreateWithFlags(&br[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[k], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    cleanup();
    return fail(GR_ERR_CUDA, "graph set-up: %s", cudaGetErrorString(e));
  }
  long launches0 = 0;
  for (auto p : plans) launches0 += p->launches;
  e = cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    cleanup();
    return fail(GR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  }
  int rc = GR_OK;
  e = cudaEventRecord(fork, s0);
  for (size_t k = 0; k < np && e == cudaSuccess && rc == GR_OK; ++k) {
    e = cudaStreamWaitEvent(br[k], fork, 0);
    for (int i = 0; i < n_items && e == cudaSuccess && rc == GR_OK; ++i)
      if (items[i].plan == plans[k]) rc = gr_reconstruct_batch(plans[k], &items[i].batch, br[k]);
    if (e == cudaSuccess && rc == GR_OK) e = cudaEventRecord(join[k], br[k]);
    if (e == cudaSuccess && rc == GR_OK) e = cudaStreamWaitEvent(s0, join[k], 0);
  }
  const std::string err_rc = rc ? g_err : std::string();
  cudaError_t ee = cudaStreamEndCapture(s0, &graph);
  if (e == cudaSuccess) e = ee;
  if (rc == GR_OK && e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  cleanup();
  long launches1 = 0;
  for (auto p : plans) launches1 += p->launches;
  if (rc != GR_OK || e != cudaSuccess) {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (rc != GR_OK) return fail(rc, "graph capture: %s", err_rc.c_str());
    return fail(GR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  }
  gr_graph* gg = new gr_graph;
  gg->device = dev;
  gg->graph = graph;
  gg->exec = exec;
  gg->launches = launches1 - launches0;
  gg->plans = plans;
  for (auto p : plans) p->graphs.push_back(gg);
  *out = gg;
  return GR_OK;
}

int gr_graph_launch(gr_graph* g, void* stream) {
  using namespace gr;
  if (!g) return fail(GR_ERR_ARG, "null graph");
  if (g->dead) return fail(GR_ERR_ARG, "graph replays a destroyed plan's buffers");
  DeviceGuard guard(g->device);
  GR_CUDA(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return GR_OK;
}

int gr_graph_launch_count(const gr_graph* g, long* launches) {
  if (!g || !launches) return gr::fail(GR_ERR_ARG, "null argument");
  *launches = g->launches;
  return GR_OK;
}

int gr_graph_destroy(gr_graph* g) {
  if (!g) return GR_OK;
  gr::DeviceGuard guard(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (auto p : g->plans) p->graphs.erase(std::find(p->graphs.begin(), p->graphs.end(), g));
  delete g;
  return GR_OK;
}

}  // extern "C"
