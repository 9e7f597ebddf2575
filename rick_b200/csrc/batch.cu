// Batched imaging: many independent jobs of uneven sizes in one launch per
// stage, the launch sequence captured once in a CUDA graph.
//
// Every job is a full imaging call (rick_plan_image: w-stacking gridding,
// per-plane inverse FFT, w-correction and plane sum, i.e. the reference's
// wstack + fftw_data + phase_correction for one dataset, w-stacking.cu:211-543,
// fourier_transform.c:13-93, phase_correction.cu:97-328).  The batch numbers
// the work units of all jobs consecutively -- 32-row binning units, (plane,
// tile) bins and their work items, touched rows, column groups -- so that one
// persistent kernel per stage serves every job; the FFT stages launch once per
// FFT length present.  A project-written autotuner picks the gridder's work-item
// size (records per item), its blocks per SM and the planes in flight of the
// column pass by timing the batch itself.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "rick_internal.h"

using namespace rick;

namespace {

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DevGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int ilog2_exact(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return (1 << l) == n ? l : -1;
}

uint64_t align256(uint64_t b) { return (b + 255) & ~255ull; }

// Layout of one batch in HBM: offsets (bytes) into one arena.
struct Layout {
  std::vector<uint64_t> cube, blocked, lm, table;  // per job
  std::vector<int> tw_log;                          // FFT lengths with twiddles
  std::map<int, uint64_t> tw;                       // log -> offset
  uint64_t jobs = 0, row_units = 0, bin_base = 0, mask_base = 0, fft_tabs = 0, sc_tabs = 0;
  uint64_t rowmask = 0, tilemask = 0, rowlist = 0, counts = 0;
  uint64_t bin_count = 0, bin_cursor = 0, item_off = 0, scan_tmp = 0, counters = 0, records = 0;
  uint64_t total = 0;
  // sizes
  uint64_t total_rows = 0, total_row_units = 0, max_records = 0;
  uint32_t total_bins = 0, total_count_words = 0;
  uint64_t total_mask_words = 0, total_tile_words = 0, total_list = 0;
};

int validate_job(const rick_job_desc &d, int i) {
  auto bad = [&](const char *what) {
    return set_error(RICK_ERR_INVALID_ARG, "batch job %d: %s", i, what);
  };
  const int lx = ilog2_exact(d.grid_size_x), ly = ilog2_exact(d.grid_size_y);
  if (lx < 6 || ly < 6 || d.grid_size_x > RICK_BATCH_MAX_GRID || d.grid_size_y > RICK_BATCH_MAX_GRID)
    return bad("grid sizes must be powers of two in [64, 4096]");
  if (d.num_w_planes <= 0) return bad("num_w_planes must be positive");
  if (d.w_support < 1 || d.w_support > kMaxSupport || d.w_support % 2 == 0)
    return bad("w_support must be odd in [1, 15]");
  if (d.kernel < RICK_KERNEL_GAUSS || d.kernel > RICK_KERNEL_KAISER_BESSEL) return bad("unknown kernel");
  if (d.freq_per_chan == 0 || d.polarizations == 0) return bad("freq_per_chan and polarizations must be positive");
  if (d.num_rows && (!d.uu || !d.vv || !d.ww || !d.weight || !d.vis_real || !d.vis_img))
    return bad("null row pointer");
  if (!d.image_real || !d.image_imag) return bad("null image pointer");
  if (!(d.wmax > d.wmin) && d.num_w_planes > 1) return bad("wmax must exceed wmin");
  return RICK_OK;
}

int plan_layout(const std::vector<rick_job_desc> &jobs, int precision, Layout &L) {
  const int n = (int)jobs.size();
  const uint64_t vb = precision == RICK_PREC_FP64 ? 8 : 4;
  uint64_t off = 0;
  auto take = [&](uint64_t bytes) {
    const uint64_t o = off;
    off += align256(std::max<uint64_t>(bytes, 16));
    return o;
  };
  L.cube.resize(n);
  L.blocked.resize(n);
  L.lm.resize(n);
  L.table.resize(n);
  uint64_t bins = 0;
  for (int j = 0; j < n; j++) {
    const rick_job_desc &d = jobs[j];
    const uint64_t nx = d.grid_size_x, ny = d.grid_size_y, nw = d.num_w_planes;
    const uint64_t ntx = (nx + kTile - 1) / kTile, nty = (ny + kTile - 1) / kTile;
    const uint64_t cube = 2 * nw * nx * ny * vb;
    L.cube[j] = take(cube);
    L.blocked[j] = take(cube);
    L.lm[j] = take((nx + ny) * 8);
    L.table[j] = take(kIncreasePrecision * kMaxSupport * 8);
    bins += nw * ntx * nty;
    L.total_rows += d.num_rows;
    L.total_row_units += (d.num_rows + 31) / 32;
    L.total_mask_words += nw * nty;
    L.total_tile_words += nw * nty * ((ntx + 31) / 32);
    L.total_list += nw * ny;
    L.total_count_words += (uint32_t)(1 + nw);
    for (int l : {ilog2_exact((int)nx), ilog2_exact((int)ny)})
      if (!L.tw.count(l)) L.tw[l] = 0;
  }
  if (bins >= 0xffffffffull) return set_error(RICK_ERR_INVALID_ARG, "batch has too many tiles");
  if (4 * L.total_rows >= 0xffffffffull)
    return set_error(RICK_ERR_INVALID_ARG, "batch has too many rows (records are 32-bit indexed)");
  L.total_bins = (uint32_t)bins;
  L.max_records = 4 * L.total_rows;
  for (auto &kv : L.tw) kv.second = take((uint64_t)(1 << kv.first) * 2 * vb);
  L.jobs = take(sizeof(BatchJob) * n);
  L.row_units = take(8ull * (n + 1));
  L.bin_base = take(4ull * (n + 1));
  L.mask_base = take(8ull * (n + 1));
  L.fft_tabs = take(4ull * (3 * n + 2));  // fft_units [n+1], col_jobs [n], col_units [n+1]
  L.sc_tabs = take(8ull * (n + 1) + 4ull * n);  // sc_units [n+1] (u64), sc_jobs [n] (u32)
  L.rowmask = take(4 * L.total_mask_words);
  L.tilemask = take(4 * L.total_tile_words);
  L.rowlist = take(4 * L.total_list);
  L.counts = take(4ull * L.total_count_words);
  L.bin_count = take(4ull * (bins + 1));
  L.bin_cursor = take(4ull * (bins + 1));
  L.item_off = take(4ull * (bins + 1));
  L.scan_tmp = take(4ull * scan_tmp_words(bins + 1));
  L.counters = take(8ull * kNumCounters);
  L.records = take(sizeof(RecF64) * std::max<uint64_t>(L.max_records, 1));
  L.total = off;
  return RICK_OK;
}

struct TuneKey {
  int precision;
  std::vector<uint64_t> sig;
  bool operator<(const TuneKey &o) const {
    return precision != o.precision ? precision < o.precision : sig < o.sig;
  }
};
std::mutex g_tune_mu;
std::map<TuneKey, rick_batch_tuning> g_tune_cache;

}  // namespace

struct rick_batch {
  int device = 0;
  int precision = RICK_PREC_MIXED;
  std::vector<rick_job_desc> jobs;  // sorted by grid_size_x (internal order)
  Layout L;
  char *arena = nullptr;
  bool own_arena = true;
  BatchLaunch bl{};
  FftJobs fj{};
  Scratch s{};
  rick_batch_tuning tune{};
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  uint32_t kernels_per_run = 0;  // kernel nodes of the captured graph
  // Batches launched side by side on several streams (the server): the column
  // pass waits for this event and records it, so that the column passes of two
  // batches never run at once.  Their blocks allocate tensor memory, and blocks
  // of two such kernels may share an SM by shared memory and registers yet ask
  // for more than its 512 TMEM columns together; a block that cannot allocate
  // waits, holding its SM.  Null: no gate.
  cudaEvent_t cols_gate = nullptr;
};

namespace {

// The launch sequence of one batch run (stream-ordered; captured in the graph).
int batch_launch(rick_batch *b, cudaStream_t st) {
  b->bl.grid_blocks_per_sm = b->tune.grid_blocks_per_sm;
  b->fj.cols_pp = b->tune.planes_in_flight;
  RICK_CUDA(cudaMemsetAsync(b->s.counters, 0, kNumCounters * sizeof(uint64_t), st));
  RICK_CUDA(cudaMemsetAsync(b->bl.rowmask, 0, 4 * b->L.total_mask_words, st));
  RICK_CUDA(cudaMemsetAsync(b->bl.tilemask, 0, 4 * b->L.total_tile_words, st));
  RICK_TRY(bin_rows_batch(b->bl, b->s, b->tune.max_chunk, st));
  RICK_TRY(grid_tiles_batch(b->bl, b->precision, b->s, b->tune.max_chunk, st));
  RICK_TRY(sparse_fft_lists(b->fj, st));
  RICK_TRY(sparse_fft_rows(b->fj, b->precision, st));
  if (b->cols_gate) RICK_CUDA(cudaStreamWaitEvent(st, b->cols_gate, 0));
  RICK_TRY(sparse_fft_cols(b->fj, b->precision, st));
  if (b->cols_gate) RICK_CUDA(cudaEventRecord(b->cols_gate, st));
  return RICK_OK;
}

// Device tables of the batch, copied on `st` (from pageable memory: each call
// returns once its source has been staged).
int build_tables(rick_batch *b, cudaStream_t st) {
  const int n = (int)b->jobs.size();
  const Layout &L = b->L;
  char *A = b->arena;
  const bool f64 = b->precision == RICK_PREC_FP64;
  // twiddles per FFT length
  std::map<int, const void *> tw;
  for (auto &kv : L.tw) {
    const int len = 1 << kv.first;
    std::vector<double2> t64(len);
    std::vector<float2> t32(len);
    make_twiddles(len, t64.data(), t32.data());
    const void *src = f64 ? (const void *)t64.data() : (const void *)t32.data();
    RICK_CUDA(cudaMemcpyAsync(A + kv.second, src, (size_t)len * (f64 ? 16 : 8),
                              cudaMemcpyHostToDevice, st));
    tw[kv.first] = A + kv.second;
  }
  std::vector<BatchJob> hj(n);
  std::vector<uint64_t> row_units(n + 1), mask_base(n + 1);
  std::vector<uint32_t> bin_base(n + 1);
  uint64_t ru = 0, mb = 0, tb = 0, lb = 0;
  uint32_t bb = 0, cb = 0;
  std::vector<double> lm, tab(kIncreasePrecision * kMaxSupport);
  for (int j = 0; j < n; j++) {
    const rick_job_desc &d = b->jobs[j];
    BatchJob &J = hj[j];
    Geometry &g = J.g;
    g.nx = d.grid_size_x;
    g.ny = d.grid_size_y;
    g.nw = d.num_w_planes;
    g.support = d.w_support;
    g.half = (d.w_support - 1) / 2;
    g.ntx = (g.nx + kTile - 1) / kTile;
    g.nty = (g.ny + kTile - 1) / kTile;
    g.dx = 1.0 / g.nx;  // init.c:11-12
    g.dw = 1.0 / g.nw;
    g.w_supporth = (double)g.half * (1.0 / (double)g.nx);  // init.c:13
    g.select_sector0 = d.row_selection == RICK_ROWS_SECTOR0;
    J.kernel = d.kernel;
    J.logx = ilog2_exact(g.nx);
    J.logy = ilog2_exact(g.ny);
    J.nrows = d.num_rows;
    J.nchan = d.freq_per_chan;
    J.npol = d.polarizations;
    {
      const uint32_t nv = d.freq_per_chan * d.polarizations;
      const bool aligned = ((uintptr_t)d.vis_real % 16 == 0) && ((uintptr_t)d.vis_img % 16 == 0);
      J.scatter_v4 = aligned && nv % 4 == 0 &&
                     (d.polarizations == 1 || d.polarizations == 2 || d.polarizations == 4);
      J.scatter_lanes = lanes_per_row(J.scatter_v4 ? nv / 4 : nv);
    }
    J.bin_base = bb;
    J.counts_base = cb;
    J.mask_base = mb;
    J.tile_base = tb;
    J.list_base = lb;
    J.uu = d.uu;
    J.vv = d.vv;
    J.ww = d.ww;
    J.weight = d.weight;
    J.vis_re = d.vis_real;
    J.vis_im = d.vis_img;
    J.cube = A + L.cube[j];
    J.blocked = A + L.blocked[j];
    J.table = (const double *)(A + L.table[j]);
    J.tw_x = tw[J.logx];
    J.tw_y = tw[J.logy];
    J.ltab = (const double *)(A + L.lm[j]);
    J.mtab = J.ltab + g.nx;
    J.wmin = d.wmin;
    J.dw_phase = (d.wmax - d.wmin) / (double)g.nw;  // phase_correction.cu:100-102
    J.dwnorm = J.dw_phase / (d.wmax - d.wmin);
    J.norm = 1.0 / (double)((long long)g.nx * g.ny);  // fourier_transform.c:24
    J.phase_on = d.phase_on;
    J.img_re = d.image_real;
    J.img_im = d.image_imag;
    row_units[j] = ru;
    bin_base[j] = bb;
    mask_base[j] = mb;
    ru += (d.num_rows + 31) / 32;
    bb += (uint32_t)g.nbins();
    cb += 1 + g.nw;
    mb += (uint64_t)g.nw * g.nty;
    tb += (uint64_t)g.nw * g.nty * ((g.ntx + 31) / 32);
    lb += (uint64_t)g.nw * g.ny;
    lm.assign(g.nx + g.ny, 0.0);
    phase_tables(g.nx, g.ny, g.nx, g.ny, d.resolution, lm.data(), lm.data() + g.nx);
    RICK_CUDA(cudaMemcpyAsync(A + L.lm[j], lm.data(), lm.size() * 8, cudaMemcpyHostToDevice, st));
    make_table(d.kernel, d.w_support, tab.data());
    RICK_CUDA(cudaMemcpyAsync(A + L.table[j], tab.data(), tab.size() * 8, cudaMemcpyHostToDevice,
                              st));
  }
  row_units[n] = ru;
  bin_base[n] = bb;
  mask_base[n] = mb;
  std::vector<uint32_t> tabs(3 * n + 2, 0);
  FftJobs &f = b->fj;
  fft_classes(hj.data(), n, f, tabs.data() + (n + 1), tabs.data() + (2 * n + 1));
  RICK_CUDA(cudaMemcpyAsync(A + L.jobs, hj.data(), sizeof(BatchJob) * n, cudaMemcpyHostToDevice, st));
  RICK_CUDA(cudaMemcpyAsync(A + L.row_units, row_units.data(), 8 * (n + 1), cudaMemcpyHostToDevice,
                            st));
  RICK_CUDA(cudaMemcpyAsync(A + L.bin_base, bin_base.data(), 4 * (n + 1), cudaMemcpyHostToDevice, st));
  RICK_CUDA(cudaMemcpyAsync(A + L.mask_base, mask_base.data(), 8 * (n + 1), cudaMemcpyHostToDevice,
                            st));
  RICK_CUDA(cudaMemcpyAsync(A + L.fft_tabs, tabs.data(), 4 * tabs.size(), cudaMemcpyHostToDevice, st));
  // sample-pass schedules: the jobs grouped by (lanes per row, 16-byte loads)
  BatchLaunch &bl = b->bl;
  {
    std::vector<uint64_t> sc_units(n + 1, 0);
    std::vector<uint32_t> sc_jobs(n, 0);
    int k = 0;
    uint64_t acc = 0;
    bl.n_sc = 0;
    for (int v4 = 1; v4 >= 0; v4--)
      for (int lanes = 1; lanes <= 32; lanes *= 2) {
        const int lo = k;
        uint64_t units = 0;
        for (int j = 0; j < n; j++) {
          if (hj[j].scatter_v4 != v4 || hj[j].scatter_lanes != lanes) continue;
          sc_jobs[k] = (uint32_t)j;
          sc_units[k] = acc;
          const uint64_t u = (hj[j].nrows + 31) / 32;
          acc += u;
          units += u;
          k++;
        }
        if (k > lo && units > 0) bl.sc[bl.n_sc++] = ScatterClass{lanes, v4 != 0, lo, k, units};
      }
    sc_units[n] = acc;
    RICK_CUDA(cudaMemcpyAsync(A + L.sc_tabs, sc_units.data(), 8 * (n + 1), cudaMemcpyHostToDevice,
                              st));
    RICK_CUDA(cudaMemcpyAsync(A + L.sc_tabs + 8 * (n + 1), sc_jobs.data(), 4 * n,
                              cudaMemcpyHostToDevice, st));
    bl.sc_units = (const uint64_t *)(A + L.sc_tabs);
    bl.sc_jobs = (const uint32_t *)(A + L.sc_tabs + 8 * (n + 1));
  }

  bl.jobs = (const BatchJob *)(A + L.jobs);
  bl.njobs = n;
  bl.u.row_units = (const uint64_t *)(A + L.row_units);
  bl.u.bin_base = (const uint32_t *)(A + L.bin_base);
  bl.total_row_units = L.total_row_units;
  bl.total_bins = L.total_bins;
  bl.max_support = 1;
  bl.min_support = 1 << 30;
  for (const rick_job_desc &d : b->jobs) {
    bl.max_support = std::max(bl.max_support, d.w_support);
    bl.min_support = std::min(bl.min_support, d.w_support);
  }
  bl.rowmask = (uint32_t *)(A + L.rowmask);
  bl.tilemask = (uint32_t *)(A + L.tilemask);

  f.jobs = bl.jobs;
  f.njobs = n;
  f.fft_units = (uint32_t *)(A + L.fft_tabs);
  f.col_jobs = f.fft_units + (n + 1);
  f.col_units = f.fft_units + (2 * n + 1);
  f.mask_base = (const uint64_t *)(A + L.mask_base);
  f.total_mask_words = L.total_mask_words;
  f.total_count_words = L.total_count_words;
  f.rowmask = bl.rowmask;
  f.tilemask = bl.tilemask;
  f.rowlist = (uint32_t *)(A + L.rowlist);
  f.counts = (uint32_t *)(A + L.counts);

  Scratch &s = b->s;
  s.bin_count = (uint32_t *)(A + L.bin_count);
  s.bin_cursor = (uint32_t *)(A + L.bin_cursor);
  s.item_off = (uint32_t *)(A + L.item_off);
  s.scan_tmp = (uint32_t *)(A + L.scan_tmp);
  s.counters = (uint64_t *)(A + L.counters);
  s.records = (RecF64 *)(A + L.records);
  s.max_records = L.max_records;
  return RICK_OK;
}

// Mean milliseconds of `reps` eager runs of the batch (after one warm-up).
int time_runs(rick_batch *b, int reps, float *ms) {
  cudaEvent_t e0, e1;
  RICK_CUDA(cudaEventCreate(&e0));
  RICK_CUDA(cudaEventCreate(&e1));
  int st = batch_launch(b, b->cap);
  if (st == RICK_OK && cudaEventRecord(e0, b->cap) != cudaSuccess) st = RICK_ERR_CUDA;
  for (int r = 0; r < reps && st == RICK_OK; r++) st = batch_launch(b, b->cap);
  if (st == RICK_OK && cudaEventRecord(e1, b->cap) != cudaSuccess) st = RICK_ERR_CUDA;
  if (st == RICK_OK && cudaEventSynchronize(e1) != cudaSuccess) st = RICK_ERR_CUDA;
  float t = 0.f;
  if (st == RICK_OK) cudaEventElapsedTime(&t, e0, e1);
  *ms = t / std::max(reps, 1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st == RICK_ERR_CUDA) return cuda_status(cudaGetLastError(), "autotune run", __FILE__, __LINE__);
  return st;
}

// Coordinate descent over the gridder's records per work item, its blocks per
// SM and the column pass's form (state in tensor memory, or planes in flight),
// timing the batch.
int autotune(rick_batch *b) {
  TuneKey key;
  key.precision = b->precision;
  for (const rick_job_desc &d : b->jobs) {
    key.sig.push_back(((uint64_t)d.grid_size_x << 40) | ((uint64_t)d.grid_size_y << 20) |
                      (uint64_t)d.num_w_planes);
    key.sig.push_back(d.num_rows * 1000003ull + d.freq_per_chan * 31ull + d.polarizations);
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      b->tune = it->second;
      return RICK_OK;
    }
  }
  rick_batch_tuning best{2048, 6, 0};
  b->tune = best;
  float best_ms = 0.f;
  RICK_TRY(time_runs(b, 2, &best_ms));
  auto trial = [&](rick_batch_tuning t) -> int {
    b->tune = t;
    float ms = 0.f;
    RICK_TRY(time_runs(b, 2, &ms));
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
    return RICK_OK;
  };
  for (uint32_t c : {1024u, 4096u, 8192u}) {
    rick_batch_tuning t = best;
    t.max_chunk = c;
    RICK_TRY(trial(t));
  }
  for (int bps : {4, 8}) {
    rick_batch_tuning t = best;
    t.grid_blocks_per_sm = bps;
    RICK_TRY(trial(t));
  }
  // the column pass: state in tensor memory (0), or in registers with one or
  // (mixed form) two planes per iteration
  for (int pif : {1, 2}) {
    if (pif == 2 && b->precision != RICK_PREC_MIXED) continue;
    rick_batch_tuning t = best;
    t.planes_in_flight = pif;
    RICK_TRY(trial(t));
  }
  b->tune = best;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = best;
  return RICK_OK;
}

int capture(rick_batch *b) {
  RICK_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  const unsigned long long l0 = g_launches.load();
  const int st = batch_launch(b, b->cap);
  b->kernels_per_run = (uint32_t)(g_launches.load() - l0);
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
  if (st != RICK_OK) {
    if (g) cudaGraphDestroy(g);
    return st;
  }
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture", __FILE__, __LINE__);
  b->graph = g;
  RICK_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
  return RICK_OK;
}

void batch_free(rick_batch *b) {
  if (!b) return;
  DevGuard guard(b->device);
  if (b->cap) cudaStreamSynchronize(b->cap);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->arena && b->own_arena) cudaFree(b->arena);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
}

// st: the stream of the table copies (and of every run: the server's path);
// nullptr gives the batch its own stream (the graph path).
int batch_prepare(rick_batch **out, const rick_job_desc *jobs, int njobs, int precision,
                  int device, void *arena, uint64_t arena_bytes, cudaStream_t stream) {
  if (!out) return set_error(RICK_ERR_INVALID_ARG, "null batch pointer");
  *out = nullptr;
  if (njobs <= 0 || !jobs) return set_error(RICK_ERR_INVALID_ARG, "a batch needs at least one job");
  if (precision != RICK_PREC_FP64 && precision != RICK_PREC_MIXED)
    return set_error(RICK_ERR_INVALID_ARG, "unknown precision %d", precision);
  for (int i = 0; i < njobs; i++) RICK_TRY(validate_job(jobs[i], i));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(RICK_ERR_NO_ACCELERATORS_FOUND, "No accelerators found");
  }
  rick_batch *b = new rick_batch();
  b->device = device >= 0 ? device % ndev : 0;
  if (device < 0) cudaGetDevice(&b->device);
  b->precision = precision;
  b->jobs.assign(jobs, jobs + njobs);
  // the row pass launches once per x length: jobs of one length contiguous
  std::stable_sort(b->jobs.begin(), b->jobs.end(), [](const rick_job_desc &x, const rick_job_desc &y) {
    return x.grid_size_x < y.grid_size_x;
  });
  DevGuard guard(b->device);
  int st = plan_layout(b->jobs, precision, b->L);
  if (st == RICK_OK) {
    if (arena) {
      if (arena_bytes < b->L.total) {
        st = set_error(RICK_ERR_BUDGET, "batch needs %llu bytes, the arena holds %llu",
                       (unsigned long long)b->L.total, (unsigned long long)arena_bytes);
      } else {
        b->arena = (char *)arena;
        b->own_arena = false;
      }
    } else {
      const cudaError_t e = cudaMalloc((void **)&b->arena, b->L.total);
      if (e != cudaSuccess) {
        cudaGetLastError();
        st = set_error(RICK_ERR_NOT_ENOUGH_MEM, "cudaMalloc of %llu bytes for the batch failed",
                       (unsigned long long)b->L.total);
      }
    }
  }
  if (st == RICK_OK && !stream) {
    const cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) st = cuda_status(e, "cudaStreamCreate", __FILE__, __LINE__);
  }
  if (st == RICK_OK) st = build_tables(b, stream ? stream : b->cap);
  if (st != RICK_OK) {
    batch_free(b);
    return st;
  }
  *out = b;
  return RICK_OK;
}

}  // namespace

extern "C" {

int rick_batch_footprint(const rick_job_desc *jobs, int njobs, int precision, uint64_t *bytes) {
  if (!jobs || njobs <= 0 || !bytes) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  for (int i = 0; i < njobs; i++) RICK_TRY(validate_job(jobs[i], i));
  std::vector<rick_job_desc> v(jobs, jobs + njobs);
  std::stable_sort(v.begin(), v.end(), [](const rick_job_desc &x, const rick_job_desc &y) {
    return x.grid_size_x < y.grid_size_x;
  });
  Layout L;
  RICK_TRY(plan_layout(v, precision, L));
  *bytes = L.total;
  return RICK_OK;
}

int rick_batch_create(rick_batch **out, const rick_job_desc *jobs, int njobs, int precision,
                      int device, const rick_batch_tuning *tuning) {
  RICK_TRY(batch_prepare(out, jobs, njobs, precision, device, nullptr, 0, nullptr));
  rick_batch *b = *out;
  DevGuard guard(b->device);
  int st = RICK_OK;
  if (tuning) {
    b->tune = *tuning;
    if (b->tune.max_chunk < 64) b->tune.max_chunk = 64;
    if (b->tune.grid_blocks_per_sm < 1) b->tune.grid_blocks_per_sm = 1;
    if (b->tune.planes_in_flight < 0 || b->tune.planes_in_flight > 2) b->tune.planes_in_flight = 0;
  } else {
    st = autotune(b);
  }
  if (st == RICK_OK) st = capture(b);
  // the tables were copied on the batch's own stream; runs go on the caller's
  if (st == RICK_OK && cudaStreamSynchronize(b->cap) != cudaSuccess)
    st = cuda_status(cudaGetLastError(), "cudaStreamSynchronize", __FILE__, __LINE__);
  if (st != RICK_OK) {
    batch_free(b);
    *out = nullptr;
  }
  return st;
}

int rick_batch_run(rick_batch *b, void *stream) {
  if (!b) return set_error(RICK_ERR_INVALID_ARG, "null batch");
  DevGuard guard(b->device);
  RICK_CUDA(cudaGraphLaunch(b->exec, (cudaStream_t)stream));
  return RICK_OK;
}

int rick_batch_get_tuning(rick_batch *b, rick_batch_tuning *t) {
  if (!b || !t) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  *t = b->tune;
  return RICK_OK;
}

int rick_batch_kernels_per_run(rick_batch *b, uint32_t *kernels) {
  if (!b || !kernels) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  *kernels = b->kernels_per_run;
  return RICK_OK;
}

int rick_batch_get_stats(rick_batch *b, rick_plan_stats *out) {
  if (!b || !out) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  DevGuard guard(b->device);
  uint64_t c[kNumCounters];
  RICK_CUDA(cudaDeviceSynchronize());
  RICK_CUDA(cudaMemcpy(c, b->s.counters, sizeof(c), cudaMemcpyDeviceToHost));
  memset(out, 0, sizeof(*out));
  out->rows_in = b->L.total_rows;
  out->rows_gridded = c[kCntGridded];
  out->rows_dropped = c[kCntDropped];
  out->records = c[kCntRecords];
  uint32_t items = 0;
  RICK_CUDA(cudaMemcpy(&items, b->s.item_off + b->L.total_bins, 4, cudaMemcpyDeviceToHost));
  out->work_items = items;
  out->device_bytes = b->L.total;
  uint32_t rows = 0;
  std::vector<uint32_t> counts(b->L.total_count_words);
  RICK_CUDA(cudaMemcpy(counts.data(), b->fj.counts, 4 * counts.size(), cudaMemcpyDeviceToHost));
  uint32_t cb = 0;
  for (const rick_job_desc &d : b->jobs) {
    rows += counts[cb];
    cb += 1 + d.num_w_planes;
  }
  out->fft_rows = rows;
  return RICK_OK;
}

int rick_batch_destroy(rick_batch *b) {
  batch_free(b);
  return RICK_OK;
}

}  // extern "C"

// ---- used by the serving loop (serve.cu) ----------------------------------
namespace rick {

int batch_create_in(rick_batch **out, const rick_job_desc *jobs, int njobs, int precision,
                    int device, void *arena, uint64_t arena_bytes, const rick_batch_tuning &t,
                    cudaStream_t st, cudaEvent_t cols_gate) {
  RICK_TRY(batch_prepare(out, jobs, njobs, precision, device, arena, arena_bytes, st));
  (*out)->tune = t;
  (*out)->use_graph = false;
  (*out)->cols_gate = cols_gate;
  return RICK_OK;
}

int batch_launch_eager(rick_batch *b, cudaStream_t st) { return batch_launch(b, st); }

void batch_destroy(rick_batch *b) { batch_free(b); }

uint64_t batch_bytes(const rick_job_desc *jobs, int njobs, int precision) {
  uint64_t bytes = 0;
  if (rick_batch_footprint(jobs, njobs, precision, &bytes) != RICK_OK) return 0;
  return bytes;
}

bool batch_cached_tuning(int precision, rick_batch_tuning *t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  for (auto &kv : g_tune_cache)
    if (kv.first.precision == precision) {
      *t = kv.second;
      return true;
    }
  return false;
}

}  // namespace rick
