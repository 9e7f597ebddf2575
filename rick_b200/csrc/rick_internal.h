// Internal declarations shared by the librick_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <atomic>

#include "rick_b200.h"

namespace rick {

// Truncated pi of the reference (allvars.h:47, w-stacking.h:6); the w-phase and
// the Gaussian norm use it, and 1e-12 parity needs the same constant.
constexpr double kPi = 3.14159265359;
// Oversampling of the 1-D kernel tables (w-stacking.cu:253).
constexpr int kIncreasePrecision = 5;
// Gaussian width 1/(2 std^2) with std = 1 (w-stacking.cu:254-255).
constexpr double kStd22 = 0.5;
// Edge of a grid tile owned by one gridder work item.
constexpr int kTile = 32;
// Largest supported w_support (odd): footprints fit inside one tile border.
constexpr int kMaxSupport = 15;
// Threads per gridder block.
constexpr int kGridThreads = 256;

// Status plumbing: every internal call returns an int status and records a
// message in thread-local storage.
int set_error(int status, const char *fmt, ...);
int cuda_status(cudaError_t e, const char *what, const char *file, int line);
int cufft_status(cufftResult r, const char *what, const char *file, int line);

#define RICK_CUDA(call)                                                              \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return ::rick::cuda_status(e_, #call, __FILE__, __LINE__); \
  } while (0)
#define RICK_CUFFT(call)                                                               \
  do {                                                                                 \
    cufftResult r_ = (call);                                                           \
    if (r_ != CUFFT_SUCCESS) return ::rick::cufft_status(r_, #call, __FILE__, __LINE__); \
  } while (0)
#define RICK_TRY(call)            \
  do {                            \
    int s_ = (call);              \
    if (s_ != RICK_OK) return s_; \
  } while (0)

// Geometry of one imaging job, as the kernels see it.
struct Geometry {
  int nx, ny, nw;       // grid_size_x, grid_size_y, num_w_planes
  int support;          // w_support (odd)
  int half;             // KernelLen = (w_support-1)/2
  int ntx, nty;         // tiles per row / column
  double dx, dw;        // 1/Nx, 1/Nw (init.c:11-12) or as passed to wstack
  double w_supporth;    // (double)half*dx (init.c:13)
  int select_sector0;   // apply gridding.c:149-188 membership
  int w_first;          // first plane of a w-plane shard (nw planes from here)
  int nw_total;         // planes of the whole cube (0: nw)
  uint64_t nbins() const { return (uint64_t)nw * ntx * nty; }
};

// Binned row record (32 bytes: one DRAM sector, two 16-byte loads).  pu, pv
// are the FP64 pixel positions u/dx, v/dx of w-stacking.cu:143-144; the
// gridder re-derives the cell (int)pos and the fraction pos - (int)pos, exact
// in FP64, so (d + 0.5) - f rounds to the reference's (j + 0.5) - pos exactly.
struct __align__(16) RecF64 {
  double sre, sim;   // sum over channels and polarisations of weight*vis
  double pu, pv;     // pixel position
};

// Device scratch owned by a plan.
struct Scratch {
  uint32_t *bin_count = nullptr;   // [nbins+1] counts, then exclusive offsets
  uint32_t *bin_cursor = nullptr;  // [nbins]
  uint32_t *item_off = nullptr;    // [nbins+1] work-item offsets
  uint32_t *scan_tmp = nullptr;    // block sums for the scans
  uint64_t *counters = nullptr;    // [8] device counters (see Counter)
  RecF64 *records = nullptr;       // [max_records]
  uint64_t max_records = 0;
  double *table = nullptr;         // 1-D kernel table, 5*support doubles
};

// Scratch of the sparse-aware FFT (fft.cu).
struct FftScratch {
  uint32_t *rowmask = nullptr;  // [nw * nty] bit k%32 of word (w, k/32): row k touched
  uint32_t *rowlist = nullptr;  // [nw * ny] touched (plane, row) ids
  uint32_t *counts = nullptr;   // [1 + nw] touched rows, then touched rows per plane
  uint32_t *tilemask = nullptr; // [nw * nty * ceil(ntx/32)] bit tx: tile (w, ty, tx) holds records
  double2 *tw_x64 = nullptr, *tw_y64 = nullptr;  // per-pass twiddles of the two axes
  float2 *tw_x32 = nullptr, *tw_y32 = nullptr;
  void *blocked = nullptr;      // row-transformed planes, column-blocked (cube-sized)
};

// One job of a batch (batch.cu), as the batch kernels see it: the job's
// geometry, its inputs and outputs, and where its slices of the batch-wide
// arrays start.  Work units of every stage are numbered across all jobs; a
// kernel finds the job of a unit by binary search over the unit bases.
struct BatchJob {
  Geometry g;
  int kernel;                      // RICK_KERNEL_*
  int logx, logy;                  // log2 of the axes (sparse FFT sizes)
  uint64_t nrows;                  // rows of the job
  uint32_t nchan, npol;
  int scatter_lanes;               // lanes per row of the sample pass (1, 2, 4, ..., 32)
  int scatter_v4;                  // 16-byte sample loads (aligned rows, nchan*npol % 4 == 0)
  uint32_t bin_base;               // first global bin (nw*nty*ntx bins per job)
  uint32_t counts_base;            // first word of the job's [1 + nw] row counts
  uint64_t mask_base;              // first word of the job's row mask [nw * nty]
  uint64_t tile_base;              // first word of the job's tile bitmap [nw * nty * tmw]
  uint64_t list_base;              // first entry of the job's row list [nw * ny]
  const double *uu, *vv, *ww;      // rows (device)
  const float *weight, *vis_re, *vis_im;
  void *cube;                      // [nw][ny][nx] complex (T)
  void *blocked;                   // column-blocked row transforms (cube-sized)
  const double *table;             // 1-D kernel table (5*support)
  const void *tw_x, *tw_y;         // per-pass twiddles of the two axes (T)
  const double *ltab, *mtab;       // phase tables (nx, ny)
  double wmin, dw_phase, dwnorm, norm;
  int phase_on;
  double *img_re, *img_im;         // image (device, [ny][nx])
};

// Batch-wide unit bases of the binning and gridding stages (device arrays of
// njobs + 1 entries, exclusive prefix sums).
struct BatchUnits {
  const uint64_t *row_units;   // 32-row binning units per job
  const uint32_t *bin_base;    // bins per job (== BatchJob::bin_base, plus the total)
};

// FFT stages of a set of jobs (a plan is a set of one): jobs sorted by logx, so
// that the jobs of one row-FFT length are contiguous; the column pass lists them
// grouped by logy.  One launch per FFT length present.
struct FftClass {
  int log;         // log2 of the FFT length
  int lo, hi;      // jobs[lo..hi) (row pass) or col_jobs[lo..hi) (column pass)
  uint32_t units;  // column groups of the class (column pass)
};
struct FftJobs {
  const BatchJob *jobs = nullptr;    // device [njobs]
  int njobs = 0;
  uint32_t *fft_units = nullptr;     // device [njobs + 1], row-pass units (filled on the device)
  const uint32_t *col_jobs = nullptr;   // device [njobs]
  const uint32_t *col_units = nullptr;  // device [njobs + 1], in col_jobs order
  const uint64_t *mask_base = nullptr;  // device [njobs + 1], row-mask words per job
  uint64_t total_mask_words = 0;
  uint32_t total_count_words = 0;
  uint32_t *rowmask = nullptr, *tilemask = nullptr, *rowlist = nullptr, *counts = nullptr;
  int n_row_cls = 0, n_col_cls = 0;
  FftClass row_cls[8], col_cls[8];
  int cols_pp = 2;                   // planes per column-pass iteration allowed (1 or 2)
  // a set of one job (a plan): its host copy; the FFT kernels then take the
  // job as kernel parameters instead of reading the device table
  const BatchJob *one = nullptr;
};

// Rows (columns) one block of the row (column) pass transforms at length 2^logn:
// a row takes 2^logn / 8 threads, a block max(256, 2^logn / 8).
__host__ __device__ inline int fft_rows_per_block(int logn) {
  const int g = (1 << logn) / 8;
  return (g > 256 ? g : 256) / g;
}

enum Counter : int {
  kCntDropped = 0,    // rows outside the cube / sector
  kCntGridded = 1,    // rows that produced records
  kCntRecords = 2,    // records written
  kCntItemNext = 3,   // persistent gridder work counter
  kCntOtherShard = 6, // rows of planes outside the shard
  kNumCounters = 8
};

// Kernel-table construction on the host (w-stacking.cu:35-89).
void make_table(int kernel, int support, double *tab);

// Pipeline stages (bin.cu, grid.cu, phase.cu).
int bin_rows(const Geometry &g, int kernel, int precision, uint64_t nrows, const double *uu,
             const double *vv, const double *ww, const float *weight, const float *vis_re,
             const float *vis_im, uint32_t nchan, uint32_t npol, Scratch &s,
             uint32_t max_chunk, cudaStream_t st, cudaEvent_t mid = nullptr);
// The two passes of bin_rows, for callers that stream the samples in slices.
int bin_count_rows(const Geometry &g, uint64_t nrows, const double *uu, const double *vv,
                   const double *ww, Scratch &s, uint32_t max_chunk, cudaStream_t st);
int bin_scatter_rows(const Geometry &g, uint64_t nrows, const double *uu, const double *vv,
                     const double *ww, const float *weight, const float *vis_re,
                     const float *vis_im, uint32_t nchan, uint32_t npol, Scratch &s,
                     cudaStream_t st);
int grid_tiles(const Geometry &g, int kernel, int precision, Scratch &s, void *cube,
               int accumulate, uint32_t max_chunk, cudaStream_t st,
               uint32_t *rowmask = nullptr, uint32_t *tilemask = nullptr);
// Zeroes the tiles that several work items add into (the sparse path does not
// clear the cube).
int zero_split_tiles(const Geometry &g, int precision, Scratch &s, void *cube, cudaStream_t st);
// Sparse-aware FFT (fft.cu).
bool sparse_fft_supported(int nx, int ny);
void make_twiddles(int n, double2 *t64, float2 *t32);
void phase_tables(int xaxis, int yaxis, int xaxistot, int yaxistot, double resolution,
                  double *l, double *m);
// Planes w_first .. w_first+nw-1 of an nw_total-plane cube (phase_correction
// with the global plane index; nw_total = nw, w_first = 0 for a whole cube).
int phase_sum(int precision, const void *cube, int xaxis, int yaxis, int nw, int w_first,
              int nw_total, const double *ltab, const double *mtab, double wmin, double wmax,
              double norm, int phase_on, int accumulate, double *img_re, double *img_im,
              cudaStream_t st);
// gridding.c:21-83 on device rows (uvw.cu); scratch: RICK_NORMALIZE_SCRATCH bytes.
int normalize_uvw(uint64_t n, double *uu, double *vv, double *ww, void *scratch,
                  cudaStream_t st);
int exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *tmp,
                       cudaStream_t st);
uint64_t scan_tmp_words(uint64_t n);

#ifdef __CUDACC__
// Index j of the job that owns unit x: the last j with base[j] <= x, for an
// exclusive prefix base[0..njobs] with x < base[njobs].
template <typename U>
__device__ __forceinline__ int batch_job_of(const U *__restrict__ base, int njobs, U x) {
  int lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (base[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}
#endif

// Batch stages: every job of the batch in one launch per kernel.
// Jobs of one sample-pass schedule (lanes per row, 16-byte loads): entries
// lo..hi-1 of the schedule-ordered job list.
struct ScatterClass {
  int lanes;
  bool v4;
  int lo, hi;
  uint64_t units;  // 32-row units of the class
};

struct BatchLaunch {
  const BatchJob *jobs;    // device [njobs]
  int njobs;
  BatchUnits u;
  const uint32_t *sc_jobs;   // device [njobs]: jobs grouped by sample-pass schedule
  const uint64_t *sc_units;  // device [njobs + 1]: 32-row unit prefix in that order
  int n_sc;
  ScatterClass sc[12];
  uint64_t total_row_units;
  uint32_t total_bins;
  int max_support;
  int min_support;
  uint32_t *rowmask, *tilemask;  // batch-wide arrays
  int grid_blocks_per_sm;  // gridder occupancy (tuned)
};
int bin_rows_batch(const BatchLaunch &b, Scratch &s, uint32_t max_chunk, cudaStream_t st);
int grid_tiles_batch(const BatchLaunch &b, int precision, Scratch &s, uint32_t max_chunk,
                     cudaStream_t st);

// The sparse-aware FFT stages (fft.cu) of a set of jobs.  fft_classes fills the
// classes and the host copies of col_jobs / col_units (njobs and njobs + 1
// entries) from the host copy of the jobs (sorted by logx).
void fft_classes(const BatchJob *host_jobs, int njobs, FftJobs &f, uint32_t *col_jobs,
                 uint32_t *col_units);
int sparse_fft_lists(const FftJobs &f, cudaStream_t st);  // row lists and row-pass units
int sparse_fft_rows(const FftJobs &f, int precision, cudaStream_t st);
int sparse_fft_cols(const FftJobs &f, int precision, cudaStream_t st);

// The batch internals the serving loop (serve.cu) builds on (batch.cu).
// cols_gate: an event the batch's column pass waits for and records (batches
// launched side by side on several streams), or null.
int batch_create_in(rick_batch **out, const rick_job_desc *jobs, int njobs, int precision,
                    int device, void *arena, uint64_t arena_bytes, const rick_batch_tuning &t,
                    cudaStream_t st, cudaEvent_t cols_gate);
int batch_launch_eager(rick_batch *b, cudaStream_t st);
void batch_destroy(rick_batch *b);
uint64_t batch_bytes(const rick_job_desc *jobs, int njobs, int precision);
bool batch_cached_tuning(int precision, rick_batch_tuning *t);

// Lanes per row of the sample pass for rows of `per_row` loads (bin.cu).
int lanes_per_row(uint64_t per_row);

int num_sms();

// Synchronous copies between host memory (pageable or pinned) and device
// memory; pageable memory goes through a ring of pinned buffers filled and
// drained by a pool of host threads while the copy engine runs (hostcopy.cu).
int copy_to_device(void *dst, const void *src, uint64_t bytes, cudaStream_t st);
int copy_to_host(void *dst, const void *src, uint64_t bytes, cudaStream_t st);

// Kernels launched by this library (reported by rick_launch_count).
extern std::atomic<unsigned long long> g_launches;
#define RICK_LAUNCHED() (::rick::g_launches++)

}  // namespace rick
