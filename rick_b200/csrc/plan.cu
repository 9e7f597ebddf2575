// Plan object: device-resident imaging pipeline (binning -> gridding -> FFT ->
// w-correction) with all scratch, the w-plane cube and the cuFFT plan held
// across calls.  Every call is stream-ordered; none synchronises the host
// except rick_plan_image_host and rick_plan_get_stats.
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>

#include "rick_internal.h"

namespace rick {

static thread_local char g_msg[1024];
std::atomic<unsigned long long> g_launches{0};

int set_error(int status, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return status;
}

int cuda_status(cudaError_t e, const char *what, const char *file, int line) {
  const int st = (e == cudaErrorMemoryAllocation) ? RICK_ERR_NOT_ENOUGH_MEM
                 : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
                     ? RICK_ERR_NO_ACCELERATORS_FOUND
                     : RICK_ERR_CUDA;
  cudaGetLastError();  // clear a non-sticky error so the context stays usable
  return set_error(st, "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
}

int cufft_status(cufftResult r, const char *what, const char *file, int line) {
  const int st = (r == CUFFT_ALLOC_FAILED) ? RICK_ERR_NOT_ENOUGH_MEM : RICK_ERR_CUFFT;
  return set_error(st, "%s failed at %s:%d: cufftResult %d", what, file, line, (int)r);
}

int num_sms() {
  static thread_local int cached_dev = -1, cached_sms = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev != cached_dev) {
    cudaDeviceGetAttribute(&cached_sms, cudaDevAttrMultiProcessorCount, dev);
    if (cached_sms <= 0) cached_sms = 148;
    cached_dev = dev;
  }
  return cached_sms;
}

// w-stacking.cu:35-51 (Gaussian) and :54-89 (Kaiser-Bessel, alpha 8.6,
// oversampling 1, no sinc); the same expressions, so the tables match the
// reference's to the bit.
static double bessel0(double x, double precision) {
  double d = 0.0, ds = 1.0, sum = 1.0;
  do {
    d += 2.0;
    ds *= x * x / (d * d);
    sum += ds;
  } while (ds > sum * precision);
  return sum;
}

void make_table(int kernel, int support, double *tab) {
  const int n = kIncreasePrecision * support, mid = n / 2;
  if (kernel == RICK_KERNEL_GAUSS) {
    const double norm = kStd22 / kPi;
    for (int i = 0; i <= mid; i++) {
      const double term = (double)i / (double)kIncreasePrecision;
      tab[mid + i] = sqrt(norm) * exp(-(term * term) * kStd22);
    }
  } else if (kernel == RICK_KERNEL_KAISER_BESSEL) {
    const double alpha = 8.6, oversampling = 1.0, filter_ratio = 1.0 / oversampling;
    const double norm_factor = oversampling / bessel0(alpha, 1e-8);
    for (int i = 0; i <= mid; i++) {
      const double term = (double)i / mid;
      tab[mid + i] = filter_ratio * bessel0(alpha * sqrt(1.0 - (term * term)), 1e-8) * norm_factor;
    }
  } else {
    for (int i = 0; i < n; i++) tab[i] = 0.0;  // high-precision Gaussian evaluates exp per cell
    return;
  }
  for (int i = 0; i < mid; i++) tab[i] = tab[n - 1 - i];
}

namespace {

template <typename T>
__global__ void k_export_cube(const T *__restrict__ src, double *__restrict__ dst, uint64_t n,
                              double scale, int accumulate) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * (uint64_t)blockDim.x) {
    const double v = scale == 1.0 ? (double)src[i] : scale * (double)src[i];
    dst[i] = accumulate ? dst[i] + v : v;
  }
}

__global__ void k_import_cube(const double *__restrict__ src, float *__restrict__ dst,
                              uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * (uint64_t)blockDim.x)
    dst[i] = (float)src[i];
}

}  // namespace

}  // namespace rick

using namespace rick;

// kCubeSparse: after the fused imaging call the cube holds row-transformed
// touched rows only; it is not a valid input to export, FFT or phase.
enum CubeState { kCubeRaw = 0, kCubeTransformed = 1, kCubeNormalised = 2, kCubeSparse = 3 };

struct rick_plan {
  rick_plan_desc d{};
  int device = 0;
  Geometry g{};
  Scratch s{};
  void *cube = nullptr;
  uint64_t cube_vals = 0;     // real values in the cube (2*Nw*Ny*Nx)
  size_t val_bytes = 8;       // 8 (FP64) or 4 (mixed)
  int cube_state = kCubeRaw;
  cufftHandle fft = 0;
  int fft_batch = 0;
  void *fft_work = nullptr;
  size_t fft_work_bytes = 0;
  double *d_lm = nullptr;     // l table [Nx] then m table [Ny]
  double *h_lm = nullptr;     // pinned staging
  double lm_resolution = NAN;
  int lm_xtot = -1, lm_ytot = -1;
  // rows staged by the host entry point
  double *h_rows_d = nullptr;  // device copies of uu,vv,ww,weights,vis (one block)
  double *d_img = nullptr;     // [2*Ny*Nx] image staging for host calls
  double *d_stage = nullptr;   // conversion staging for mixed import/export
  void *d_norm = nullptr;      // NORMALIZE_UVW scratch (extrema)
  uint32_t chunk = 1024;       // gridder records per work item of the current gridding
  // streaming ingest (rick_plan_ingest_*): rows staged in h_rows_d, samples by slices
  bool ingest = false;
  uint64_t ing_rows = 0, ing_next = 0;
  int ing_select = 0;
  cudaStream_t ing_comp = nullptr, ing_copy = nullptr;
  cudaEvent_t ing_ev[2] = {nullptr, nullptr};
  int ing_k = 0;
  size_t stage_bytes = 0;
  uint64_t last_rows = 0;
  size_t device_bytes = 0;
  // stage timers: ev[k] marks the start of stage k, ev[k+1] its end
  bool timing = false;
  cudaEvent_t ev[RICK_NUM_STAGES + 1] = {};
  bool ran[RICK_NUM_STAGES] = {};
  cudaEvent_t ev_fft0 = nullptr, ev_phase0 = nullptr;
  // sparse-aware FFT (power-of-two axes): the plan is a set of one job
  bool sparse = false;
  FftScratch f{};
  FftJobs fj{};
  BatchJob *d_job = nullptr;      // [1]
  uint32_t *d_fft_tabs = nullptr; // fft_units [2], col_jobs [1], col_units [2]
  uint64_t *d_mask_base = nullptr;  // [2]
};

namespace {

constexpr size_t kStageBytes = 64ull << 20;

int dev_alloc(rick_plan *p, void **ptr, size_t bytes) {
  *ptr = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(ptr, bytes);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    cudaGetLastError();
    return set_error(RICK_ERR_NOT_ENOUGH_MEM, "cudaMalloc of %zu bytes failed: %s", bytes,
                     cudaGetErrorString(e));
  }
  p->device_bytes += bytes;
  return RICK_OK;
}

// Planes the plan holds: its w-plane shard, or the whole cube.
int plan_planes(const rick_plan_desc *d) { return d->w_count > 0 ? d->w_count : d->num_w_planes; }

int validate_desc(const rick_plan_desc *d) {
  if (!d) return set_error(RICK_ERR_INVALID_ARG, "null plan description");
  if (d->grid_size_x <= 0 || d->grid_size_y <= 0 || d->num_w_planes <= 0)
    return set_error(RICK_ERR_INVALID_ARG, "grid sizes must be positive (got %d x %d x %d)",
                     d->grid_size_x, d->grid_size_y, d->num_w_planes);
  if (d->w_support < 1 || d->w_support > kMaxSupport || d->w_support % 2 == 0)
    return set_error(RICK_ERR_INVALID_ARG, "w_support must be odd in [1,%d] (got %d)", kMaxSupport,
                     d->w_support);
  if (d->kernel < RICK_KERNEL_GAUSS || d->kernel > RICK_KERNEL_KAISER_BESSEL)
    return set_error(RICK_ERR_INVALID_ARG, "unknown kernel %d", d->kernel);
  if (d->precision != RICK_PREC_FP64 && d->precision != RICK_PREC_MIXED)
    return set_error(RICK_ERR_INVALID_ARG, "unknown precision %d", d->precision);
  if (d->freq_per_chan == 0 || d->polarizations == 0)
    return set_error(RICK_ERR_INVALID_ARG, "freq_per_chan and polarizations must be positive");
  if (d->w_count < 0 || d->w_first < 0 ||
      (d->w_count > 0 && d->w_first + d->w_count > d->num_w_planes) ||
      (d->w_count == 0 && d->w_first != 0))
    return set_error(RICK_ERR_INVALID_ARG, "w-plane shard %d+%d outside the %d planes", d->w_first,
                     d->w_count, d->num_w_planes);
  const uint64_t nbins = (uint64_t)plan_planes(d) * ((d->grid_size_x + kTile - 1) / kTile) *
                         ((d->grid_size_y + kTile - 1) / kTile);
  if (nbins >= 0xffffffffull) return set_error(RICK_ERR_INVALID_ARG, "grid too large");
  if (4 * d->max_rows >= 0xffffffffull)
    return set_error(RICK_ERR_INVALID_ARG, "max_rows too large (records are 32-bit indexed)");
  return RICK_OK;
}

void fill_geometry(rick_plan *p, double dx, double dw, int select) {
  Geometry &g = p->g;
  g.nx = p->d.grid_size_x;
  g.ny = p->d.grid_size_y;
  g.nw = plan_planes(&p->d);
  g.w_first = p->d.w_count > 0 ? p->d.w_first : 0;
  g.nw_total = p->d.num_w_planes;
  g.support = p->d.w_support;
  g.half = (p->d.w_support - 1) / 2;
  g.ntx = (g.nx + kTile - 1) / kTile;
  g.nty = (g.ny + kTile - 1) / kTile;
  g.dx = dx;
  g.dw = dw;
  g.w_supporth = (double)g.half * (1.0 / (double)g.nx);  // init.c:13 uses the global dx
  g.select_sector0 = select;
}


int choose_fft(rick_plan *p) {
  const int nx = p->d.grid_size_x, ny = p->d.grid_size_y, nw = plan_planes(&p->d);
  int n[2] = {ny, nx};
  const cufftType type = p->d.precision == RICK_PREC_FP64 ? CUFFT_Z2Z : CUFFT_C2C;
  const long long plane = (long long)nx * ny;
  const size_t cube_bytes = (size_t)p->cube_vals * p->val_bytes;
  const size_t budget = std::max(cube_bytes / 4, (size_t)(512ull << 20));
  int batch = nw;
  for (int b = nw; b >= 1; b--) {
    if (nw % b) continue;
    size_t ws = 0;
    if (cufftEstimateMany(2, n, nullptr, 1, (int)plane, nullptr, 1, (int)plane, type, b, &ws) !=
        CUFFT_SUCCESS)
      continue;
    batch = b;
    if (ws <= budget) break;
  }
  RICK_CUFFT(cufftCreate(&p->fft));
  RICK_CUFFT(cufftSetAutoAllocation(p->fft, 0));
  size_t ws = 0;
  RICK_CUFFT(cufftMakePlanMany(p->fft, 2, n, nullptr, 1, (int)plane, nullptr, 1, (int)plane, type,
                               batch, &ws));
  RICK_TRY(dev_alloc(p, &p->fft_work, ws));
  p->fft_work_bytes = ws;
  RICK_CUFFT(cufftSetWorkArea(p->fft, p->fft_work));
  p->fft_batch = batch;
  return RICK_OK;
}

uint32_t choose_chunk(uint64_t nrows) {
  const uint64_t per = nrows / ((uint64_t)num_sms() * 4 + 1);
  return (uint32_t)std::min<uint64_t>(8192, std::max<uint64_t>(1024, per));
}

int ensure_lm(rick_plan *p, int xaxis, int yaxis, int xtot, int ytot, double resolution,
              cudaStream_t st) {
  if (p->lm_resolution == resolution && p->lm_xtot == xtot && p->lm_ytot == ytot) return RICK_OK;
  // the staging buffer may still feed an earlier copy
  RICK_CUDA(cudaStreamSynchronize(st));
  phase_tables(xaxis, yaxis, xtot, ytot, resolution, p->h_lm, p->h_lm + xaxis);
  RICK_CUDA(cudaMemcpyAsync(p->d_lm, p->h_lm, sizeof(double) * (xaxis + yaxis),
                            cudaMemcpyHostToDevice, st));
  p->lm_resolution = resolution;
  p->lm_xtot = xtot;
  p->lm_ytot = ytot;
  return RICK_OK;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int mark(rick_plan *p, cudaEvent_t e, cudaStream_t st) {
  if (p->timing && e) RICK_CUDA(cudaEventRecord(e, st));
  return RICK_OK;
}

// The plan as the one job of its FFT stages (fft.cu): geometry, cube, buffers
// and twiddles; the image fields are filled per call.
BatchJob plan_job(const rick_plan *p) {
  BatchJob j{};
  j.g = p->g;
  j.kernel = p->d.kernel;
  int lx = 0, ly = 0;
  while ((1 << lx) < p->d.grid_size_x) lx++;
  while ((1 << ly) < p->d.grid_size_y) ly++;
  j.logx = lx;
  j.logy = ly;
  j.nchan = p->d.freq_per_chan;
  j.npol = p->d.polarizations;
  j.cube = p->cube;
  j.blocked = p->f.blocked;
  j.table = p->s.table;
  const bool f64 = p->d.precision == RICK_PREC_FP64;
  j.tw_x = f64 ? (const void *)p->f.tw_x64 : (const void *)p->f.tw_x32;
  j.tw_y = f64 ? (const void *)p->f.tw_y64 : (const void *)p->f.tw_y32;
  j.ltab = p->d_lm;
  j.mtab = p->d_lm + p->d.grid_size_x;
  return j;
}

// Gridding in three steps, so that the samples may arrive in slices between the
// first and the last (rick_plan_ingest_*): the row positions of all rows
// (normalised if asked, histogram, offsets), the samples of a slice of rows,
// then the tiles.
int grid_begin(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
               const double *ww, int select, double dx, double dw, cudaStream_t st) {
  if (nrows > p->d.max_rows)
    return set_error(RICK_ERR_INVALID_ARG, "nrows %llu exceeds the plan capacity %llu",
                     (unsigned long long)nrows, (unsigned long long)p->d.max_rows);
  if (nrows && (!uu || !vv || !ww)) return set_error(RICK_ERR_INVALID_ARG, "null row pointer");
  fill_geometry(p, dx, dw, select);
  for (int k = 0; k < RICK_NUM_STAGES; k++) p->ran[k] = false;
  RICK_TRY(mark(p, p->ev[0], st));
  if (p->d.normalize_uvw && nrows)  // gridding.c:21-83, in place
    RICK_TRY(normalize_uvw(nrows, const_cast<double *>(uu), const_cast<double *>(vv),
                           const_cast<double *>(ww), p->d_norm, st));
  RICK_CUDA(cudaMemsetAsync(p->s.counters, 0, kNumCounters * sizeof(uint64_t), st));
  p->chunk = choose_chunk(nrows);
  RICK_TRY(bin_count_rows(p->g, nrows, uu, vv, ww, p->s, p->chunk, st));
  return mark(p, p->ev[1], st);
}

int grid_samples(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                 const double *ww, const float *weight, const float *vis_re, const float *vis_im,
                 cudaStream_t st) {
  return bin_scatter_rows(p->g, nrows, uu, vv, ww, weight, vis_re, vis_im, p->d.freq_per_chan,
                          p->d.polarizations, p->s, st);
}

int grid_finish(rick_plan *p, uint64_t nrows, int accumulate, bool sparse, cudaStream_t st) {
  RICK_TRY(mark(p, p->ev[2], st));
  if (sparse) {
    // only the tiles several work items add into are cleared; the row mask
    // records which grid rows the footprints reach
    RICK_CUDA(cudaMemsetAsync(p->f.rowmask, 0, (size_t)p->g.nw * p->g.nty * 4, st));
    RICK_CUDA(cudaMemsetAsync(p->f.tilemask, 0,
                              (size_t)p->g.nw * p->g.nty * ((p->g.ntx + 31) / 32) * 4, st));
    RICK_TRY(zero_split_tiles(p->g, p->d.precision, p->s, p->cube, st));
  } else if (!accumulate) {
    RICK_CUDA(cudaMemsetAsync(p->cube, 0, p->cube_vals * p->val_bytes, st));
  }
  RICK_TRY(mark(p, p->ev[3], st));
  RICK_TRY(grid_tiles(p->g, p->d.kernel, p->d.precision, p->s, p->cube, accumulate, p->chunk,
                      st, sparse ? p->f.rowmask : nullptr, sparse ? p->f.tilemask : nullptr));
  RICK_TRY(mark(p, p->ev[4], st));
  p->ran[0] = p->ran[1] = p->ran[3] = true;
  p->ran[2] = !accumulate;
  p->cube_state = sparse ? kCubeSparse : kCubeRaw;
  p->last_rows = nrows;
  return RICK_OK;
}

int plan_grid_impl(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                   const double *ww, const float *weight, const float *vis_re, const float *vis_im,
                   int select, int accumulate, double dx, double dw, cudaStream_t st,
                   bool sparse = false) {
  if (nrows && (!weight || !vis_re || !vis_im))
    return set_error(RICK_ERR_INVALID_ARG, "null row pointer");
  RICK_TRY(grid_begin(p, nrows, uu, vv, ww, select, dx, dw, st));
  RICK_TRY(grid_samples(p, nrows, uu, vv, ww, weight, vis_re, vis_im, st));
  return grid_finish(p, nrows, accumulate, sparse, st);
}

// grid -> touched-row FFT -> column FFT fused with the w-correction.
// The sparse-aware FFT passes and the fused w-correction after a sparse gridding.
int image_sparse_after_grid(rick_plan *p, uint64_t nrows, double resolution, double wmin,
                            double wmax, double *img_re, double *img_im, cudaStream_t st) {
  RICK_TRY(mark(p, p->ev_fft0, st));
  const int nx = p->d.grid_size_x, ny = p->d.grid_size_y;
  BatchJob j = plan_job(p);
  j.nrows = nrows;
  j.wmin = wmin;
  j.dw_phase = (wmax - wmin) / (double)p->d.num_w_planes;  // phase_correction.cu:100-102
  j.dwnorm = j.dw_phase / (wmax - wmin);
  j.norm = 1.0 / (double)((long long)nx * ny);  // fourier_transform.c:24
  j.phase_on = p->d.phase_on;
  j.img_re = img_re;
  j.img_im = img_im;
  // from pageable memory: the call returns once `j` has been staged
  RICK_CUDA(cudaMemcpyAsync(p->d_job, &j, sizeof(j), cudaMemcpyHostToDevice, st));
  p->fj.one = &j;
  RICK_TRY(sparse_fft_lists(p->fj, st));
  RICK_TRY(sparse_fft_rows(p->fj, p->d.precision, st));
  RICK_TRY(mark(p, p->ev[5], st));
  RICK_TRY(ensure_lm(p, nx, ny, nx, ny, resolution, st));
  RICK_TRY(mark(p, p->ev_phase0, st));
  RICK_TRY(sparse_fft_cols(p->fj, p->d.precision, st));
  p->fj.one = nullptr;
  RICK_TRY(mark(p, p->ev[6], st));
  p->ran[4] = p->ran[5] = true;
  p->cube_state = kCubeSparse;
  return RICK_OK;
}

int plan_image_sparse(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                      const double *ww, const float *weight, const float *vis_re,
                      const float *vis_im, int select, double resolution, double wmin,
                      double wmax, double *img_re, double *img_im, cudaStream_t st) {
  RICK_TRY(plan_grid_impl(p, nrows, uu, vv, ww, weight, vis_re, vis_im, select, 0,
                          1.0 / p->d.grid_size_x, 1.0 / p->d.num_w_planes, st, true));
  return image_sparse_after_grid(p, nrows, resolution, wmin, wmax, img_re, img_im, st);
}

int plan_fft_impl(rick_plan *p, cudaStream_t st) {
  if (p->cube_state != kCubeRaw)
    return set_error(RICK_ERR_INVALID_ARG, "the cube is not a gridded (untransformed) cube");
  if (!p->fft) RICK_TRY(choose_fft(p));
  RICK_CUFFT(cufftSetStream(p->fft, st));
  RICK_TRY(mark(p, p->ev_fft0, st));
  const uint64_t plane = (uint64_t)p->d.grid_size_x * p->d.grid_size_y;
  for (int b0 = 0; b0 < plan_planes(&p->d); b0 += p->fft_batch) {
    if (p->d.precision == RICK_PREC_FP64) {
      cufftDoubleComplex *ptr = (cufftDoubleComplex *)p->cube + (uint64_t)b0 * plane;
      RICK_CUFFT(cufftExecZ2Z(p->fft, ptr, ptr, CUFFT_INVERSE));
    } else {
      cufftComplex *ptr = (cufftComplex *)p->cube + (uint64_t)b0 * plane;
      RICK_CUFFT(cufftExecC2C(p->fft, ptr, ptr, CUFFT_INVERSE));
    }
  }
  RICK_TRY(mark(p, p->ev[5], st));
  p->ran[4] = true;
  p->cube_state = kCubeTransformed;
  return RICK_OK;
}

double cube_scale(const rick_plan *p) {
  // fourier_transform.c:24: 1/(grid_size_x*grid_size_y)
  return p->cube_state == kCubeTransformed
             ? 1.0 / (double)((long long)p->d.grid_size_x * p->d.grid_size_y)
             : 1.0;
}

int plan_phase_impl(rick_plan *p, int xtot, int ytot, double resolution, double wmin,
                    double wmax, double *img_re, double *img_im, int accumulate,
                    cudaStream_t st) {
  if (p->cube_state == kCubeRaw || p->cube_state == kCubeSparse)
    return set_error(RICK_ERR_INVALID_ARG, "phase correction needs a transformed cube");
  const int nx = p->d.grid_size_x, ny = p->d.grid_size_y;
  RICK_TRY(ensure_lm(p, nx, ny, xtot, ytot, resolution, st));
  RICK_TRY(mark(p, p->ev_phase0, st));
  RICK_TRY(phase_sum(p->d.precision, p->cube, nx, ny, plan_planes(&p->d), p->g.w_first,
                     p->d.num_w_planes, p->d_lm, p->d_lm + nx,
                     wmin, wmax, cube_scale(p), p->d.phase_on, accumulate, img_re, img_im, st));
  g_launches++;
  RICK_TRY(mark(p, p->ev[6], st));
  p->ran[5] = true;
  return RICK_OK;
}

}  // namespace

extern "C" {

int rick_plan_footprint(const rick_plan_desc *desc, uint64_t *bytes) {
  RICK_TRY(validate_desc(desc));
  const uint64_t nx = desc->grid_size_x, ny = desc->grid_size_y, nw = plan_planes(desc);
  const uint64_t nbins = nw * ((nx + kTile - 1) / kTile) * ((ny + kTile - 1) / kTile);
  const uint64_t vb = desc->precision == RICK_PREC_FP64 ? 8 : 4;
  uint64_t b = 2 * nw * nx * ny * vb;                      // cube
  if (sparse_fft_supported((int)nx, (int)ny))
    b *= 2;                                                // + column-blocked planes
  else
    b += std::max<uint64_t>(b / 4, 512ull << 20);          // cuFFT work (upper bound)
  b += 4 * (nbins + 1) * 4 + 4 * scan_tmp_words(nbins + 1);  // bins, items, cursor, scan
  b += 4 * desc->max_rows * sizeof(RecF64);                // records
  b += (nx + ny) * 8 + 64;
  *bytes = b;
  return RICK_OK;
}

int rick_plan_create(rick_plan **out, const rick_plan_desc *desc) {
  if (!out) return set_error(RICK_ERR_INVALID_ARG, "null plan pointer");
  *out = nullptr;
  RICK_TRY(validate_desc(desc));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(RICK_ERR_NO_ACCELERATORS_FOUND, "No accelerators found");
  }
  rick_plan *p = new rick_plan();
  p->d = *desc;
  if (desc->device >= 0) p->device = desc->device % ndev;
  else cudaGetDevice(&p->device);
  DeviceGuard guard(p->device);
  fill_geometry(p, 1.0 / desc->grid_size_x, 1.0 / desc->num_w_planes, 0);
  const uint64_t nbins = p->g.nbins();
  p->val_bytes = desc->precision == RICK_PREC_FP64 ? 8 : 4;
  const int nwl = plan_planes(desc);
  p->cube_vals = 2ull * nwl * desc->grid_size_x * desc->grid_size_y;
  int st = RICK_OK;
  auto A = [&](void **ptr, size_t bytes) {
    if (st == RICK_OK) st = dev_alloc(p, ptr, bytes);
  };
  A(&p->cube, p->cube_vals * p->val_bytes);
  if (desc->normalize_uvw) A(&p->d_norm, RICK_NORMALIZE_SCRATCH);
  A((void **)&p->s.bin_count, (nbins + 1) * 4);
  A((void **)&p->s.bin_cursor, nbins * 4);
  A((void **)&p->s.item_off, (nbins + 1) * 4);
  A((void **)&p->s.scan_tmp, scan_tmp_words(nbins + 1) * 4);
  A((void **)&p->s.counters, kNumCounters * 8);
  p->s.max_records = 4 * std::max<uint64_t>(desc->max_rows, 1);
  A((void **)&p->s.records, p->s.max_records * sizeof(RecF64));
  A((void **)&p->s.table, kIncreasePrecision * kMaxSupport * 8);
  A((void **)&p->d_lm, (size_t)(desc->grid_size_x + desc->grid_size_y) * 8);
  if (st == RICK_OK) {
    cudaError_t e = cudaMallocHost(&p->h_lm, (size_t)(desc->grid_size_x + desc->grid_size_y) * 8);
    if (e != cudaSuccess) st = cuda_status(e, "cudaMallocHost", __FILE__, __LINE__);
  }
  if (st == RICK_OK) {
    double tab[kIncreasePrecision * kMaxSupport];
    make_table(desc->kernel, desc->w_support, tab);
    cudaError_t e = cudaMemcpy(p->s.table, tab, sizeof(double) * kIncreasePrecision * desc->w_support,
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_status(e, "cudaMemcpy(table)", __FILE__, __LINE__);
  }
  p->sparse = sparse_fft_supported(desc->grid_size_x, desc->grid_size_y) &&
              getenv("RICK_DENSE_FFT") == nullptr;
  if (st == RICK_OK && p->sparse) {
    const int nx = desc->grid_size_x, ny = desc->grid_size_y;
    A((void **)&p->f.rowmask, (size_t)nwl * p->g.nty * 4);
    A((void **)&p->f.rowlist, (size_t)nwl * ny * 4);
    A((void **)&p->f.counts, (size_t)(1 + nwl) * 4);
    A((void **)&p->f.tilemask, (size_t)nwl * p->g.nty * ((p->g.ntx + 31) / 32) * 4);
    A((void **)&p->f.tw_x64, (size_t)nx * sizeof(double2));
    A((void **)&p->f.tw_y64, (size_t)ny * sizeof(double2));
    A((void **)&p->f.tw_x32, (size_t)nx * sizeof(float2));
    A((void **)&p->f.tw_y32, (size_t)ny * sizeof(float2));
    A(&p->f.blocked, p->cube_vals * p->val_bytes);
    if (st == RICK_OK) {
      const int nmax = std::max(nx, ny);
      double2 *t64 = (double2 *)malloc(sizeof(double2) * nmax);
      float2 *t32 = (float2 *)malloc(sizeof(float2) * nmax);
      if (!t64 || !t32) st = set_error(RICK_ERR_NOT_ENOUGH_MEM, "host twiddle tables");
      for (int axis = 0; axis < 2 && st == RICK_OK; axis++) {
        const int n = axis == 0 ? nx : ny;
        make_twiddles(n, t64, t32);
        cudaError_t e = cudaMemcpy(axis == 0 ? p->f.tw_x64 : p->f.tw_y64, t64, sizeof(double2) * n,
                                   cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
          e = cudaMemcpy(axis == 0 ? p->f.tw_x32 : p->f.tw_y32, t32, sizeof(float2) * n,
                         cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = cuda_status(e, "cudaMemcpy(twiddles)", __FILE__, __LINE__);
      }
      free(t64);
      free(t32);
    }
    A((void **)&p->d_job, sizeof(BatchJob));
    A((void **)&p->d_fft_tabs, 8 * sizeof(uint32_t));
    A((void **)&p->d_mask_base, 2 * sizeof(uint64_t));
    if (st == RICK_OK) {
      FftJobs &fj = p->fj;
      BatchJob hj = plan_job(p);
      uint32_t tabs[8] = {};
      fft_classes(&hj, 1, fj, tabs + 2, tabs + 3);
      const uint64_t mb[2] = {0, (uint64_t)nwl * p->g.nty};
      fj.jobs = p->d_job;
      fj.njobs = 1;
      fj.fft_units = p->d_fft_tabs;
      fj.col_jobs = p->d_fft_tabs + 2;
      fj.col_units = p->d_fft_tabs + 3;
      fj.mask_base = p->d_mask_base;
      fj.total_mask_words = mb[1];
      fj.total_count_words = 1 + nwl;
      fj.rowmask = p->f.rowmask;
      fj.tilemask = p->f.tilemask;
      fj.rowlist = p->f.rowlist;
      fj.counts = p->f.counts;
      cudaError_t e = cudaMemcpy(p->d_fft_tabs, tabs, sizeof(tabs), cudaMemcpyHostToDevice);
      if (e == cudaSuccess) e = cudaMemcpy(p->d_mask_base, mb, sizeof(mb), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) st = cuda_status(e, "cudaMemcpy(fft tables)", __FILE__, __LINE__);
    }
  }
  // the sparse-aware path needs no cuFFT plan: the stage API creates it (and its
  // work area) on first use
  if (st == RICK_OK && !p->sparse) st = choose_fft(p);
  if (st != RICK_OK) {
    rick_plan_destroy(p);
    return st;
  }
  *out = p;
  return RICK_OK;
}

int rick_plan_destroy(rick_plan *p) {
  if (!p) return RICK_OK;
  DeviceGuard guard(p->device);
  cudaDeviceSynchronize();
  if (p->fft) cufftDestroy(p->fft);
  if (p->ing_comp) cudaStreamDestroy(p->ing_comp);
  if (p->ing_copy) cudaStreamDestroy(p->ing_copy);
  for (cudaEvent_t e : p->ing_ev)
    if (e) cudaEventDestroy(e);
  void *ptrs[] = {p->cube, p->s.bin_count, p->s.bin_cursor, p->s.item_off, p->s.scan_tmp,
                  p->s.counters, p->s.records, p->s.table, p->d_lm, p->fft_work, p->h_rows_d,
                  p->d_img, p->d_stage, p->d_norm, p->f.rowmask, p->f.rowlist, p->f.counts,
                  p->f.tw_x64, p->f.tw_y64, p->f.tw_x32, p->f.tw_y32, p->f.blocked,
                  p->f.tilemask, p->d_job, p->d_fft_tabs, p->d_mask_base};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (p->h_lm) cudaFreeHost(p->h_lm);
  for (cudaEvent_t e : p->ev)
    if (e) cudaEventDestroy(e);
  if (p->ev_fft0) cudaEventDestroy(p->ev_fft0);
  if (p->ev_phase0) cudaEventDestroy(p->ev_phase0);
  delete p;
  return RICK_OK;
}

int rick_plan_grid(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                   const double *ww, const float *weight, const float *vis_real,
                   const float *vis_img, int row_selection, void *stream) {
  if (!p) return set_error(RICK_ERR_INVALID_ARG, "null plan");
  DeviceGuard guard(p->device);
  return plan_grid_impl(p, nrows, uu, vv, ww, weight, vis_real, vis_img,
                        row_selection == RICK_ROWS_SECTOR0, 0, 1.0 / p->d.grid_size_x,
                        1.0 / p->d.num_w_planes, (cudaStream_t)stream);
}

int rick_plan_fft(rick_plan *p, void *stream) {
  if (!p) return set_error(RICK_ERR_INVALID_ARG, "null plan");
  DeviceGuard guard(p->device);
  return plan_fft_impl(p, (cudaStream_t)stream);
}

int rick_plan_phase(rick_plan *p, double resolution, double wmin, double wmax,
                    double *image_real, double *image_imag, int accumulate, void *stream) {
  if (!p || !image_real || !image_imag) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(p->device);
  return plan_phase_impl(p, p->d.grid_size_x, p->d.grid_size_y, resolution, wmin, wmax,
                         image_real, image_imag, accumulate, (cudaStream_t)stream);
}

int rick_plan_image(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                    const double *ww, const float *weight, const float *vis_real,
                    const float *vis_img, int row_selection, double resolution, double wmin,
                    double wmax, double *image_real, double *image_imag, void *stream) {
  if (!p || !image_real || !image_imag) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (p->sparse)
    return plan_image_sparse(p, nrows, uu, vv, ww, weight, vis_real, vis_img,
                             row_selection == RICK_ROWS_SECTOR0, resolution, wmin, wmax,
                             image_real, image_imag, st);
  RICK_TRY(plan_grid_impl(p, nrows, uu, vv, ww, weight, vis_real, vis_img,
                          row_selection == RICK_ROWS_SECTOR0, 0, 1.0 / p->d.grid_size_x,
                          1.0 / p->d.num_w_planes, st));
  RICK_TRY(plan_fft_impl(p, st));
  return plan_phase_impl(p, p->d.grid_size_x, p->d.grid_size_y, resolution, wmin, wmax,
                         image_real, image_imag, 0, st);
}

namespace {

// Device copies of one dataset's rows, in the plan's staging block: uu, vv, ww
// (doubles) then weights, vis_re, vis_im (floats), each 256-byte aligned.
struct RowsDev {
  double *uu, *vv, *ww;
  float *wt, *vr, *vi;
};

int stage_rows(rick_plan *p, uint64_t nrows, RowsDev *r) {
  const uint64_t npol = p->d.polarizations, nv = (uint64_t)p->d.freq_per_chan * npol;
  auto up = [](uint64_t b) { return (b + 255) & ~255ull; };
  if (!p->h_rows_d) {
    const uint64_t cap = p->d.max_rows;
    const uint64_t cap_bytes = 3 * up(cap * 8) + up(cap * npol * 4) + 2 * up(cap * nv * 4);
    RICK_TRY(dev_alloc(p, (void **)&p->h_rows_d, cap_bytes));
  }
  if (!p->d_img) RICK_TRY(dev_alloc(p, (void **)&p->d_img, 16ull * p->d.grid_size_x * p->d.grid_size_y));
  const uint64_t o_vv = up(nrows * 8), o_ww = o_vv + up(nrows * 8), o_wt = o_ww + up(nrows * 8);
  const uint64_t o_vr = o_wt + up(nrows * npol * 4), o_vi = o_vr + up(nrows * nv * 4);
  char *base = (char *)p->h_rows_d;
  r->uu = (double *)base;
  r->vv = (double *)(base + o_vv);
  r->ww = (double *)(base + o_ww);
  r->wt = (float *)(base + o_wt);
  r->vr = (float *)(base + o_vr);
  r->vi = (float *)(base + o_vi);
  return RICK_OK;
}

int h2d(void *dst, const void *src, size_t bytes, cudaStream_t st) {
  if (bytes) RICK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
  return RICK_OK;
}

// The gridded plan's image into host arrays (after the gridding on st).
int image_to_host(rick_plan *p, uint64_t nrows, double resolution, double wmin, double wmax,
                  double *image_real, double *image_imag, cudaStream_t st) {
  const uint64_t plane = (uint64_t)p->d.grid_size_x * p->d.grid_size_y;
  if (p->sparse) {
    RICK_TRY(image_sparse_after_grid(p, nrows, resolution, wmin, wmax, p->d_img, p->d_img + plane,
                                     st));
  } else {
    RICK_TRY(plan_fft_impl(p, st));
    RICK_TRY(plan_phase_impl(p, p->d.grid_size_x, p->d.grid_size_y, resolution, wmin, wmax,
                             p->d_img, p->d_img + plane, 0, st));
  }
  RICK_CUDA(cudaMemcpyAsync(image_real, p->d_img, plane * 8, cudaMemcpyDeviceToHost, st));
  RICK_CUDA(cudaMemcpyAsync(image_imag, p->d_img + plane, plane * 8, cudaMemcpyDeviceToHost, st));
  RICK_CUDA(cudaStreamSynchronize(st));
  return RICK_OK;
}

}  // namespace

int rick_plan_image_host(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                         const double *ww, const float *weight, const float *vis_real,
                         const float *vis_img, int row_selection, double resolution,
                         double wmin, double wmax, double *image_real, double *image_imag) {
  if (!p || !image_real || !image_imag) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  if (nrows > p->d.max_rows)
    return set_error(RICK_ERR_INVALID_ARG, "nrows exceeds the plan capacity");
  if (nrows && (!uu || !vv || !ww || !weight || !vis_real || !vis_img))
    return set_error(RICK_ERR_INVALID_ARG, "null row pointer");
  DeviceGuard guard(p->device);
  const uint64_t npol = p->d.polarizations, nv = (uint64_t)p->d.freq_per_chan * npol;
  RowsDev r;
  RICK_TRY(stage_rows(p, nrows, &r));
  cudaStream_t st = 0;
  RICK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int status = RICK_OK;
  auto run = [&]() -> int {
    RICK_TRY(h2d(r.uu, uu, nrows * 8, st));
    RICK_TRY(h2d(r.vv, vv, nrows * 8, st));
    RICK_TRY(h2d(r.ww, ww, nrows * 8, st));
    RICK_TRY(h2d(r.wt, weight, nrows * npol * 4, st));
    RICK_TRY(h2d(r.vr, vis_real, nrows * nv * 4, st));
    RICK_TRY(h2d(r.vi, vis_img, nrows * nv * 4, st));
    RICK_TRY(plan_grid_impl(p, nrows, r.uu, r.vv, r.ww, r.wt, r.vr, r.vi,
                            row_selection == RICK_ROWS_SECTOR0, 0, 1.0 / p->d.grid_size_x,
                            1.0 / p->d.num_w_planes, st, p->sparse));
    return image_to_host(p, nrows, resolution, wmin, wmax, image_real, image_imag, st);
  };
  status = run();
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return status;
}

// ---- streaming ingest ------------------------------------------------------
int rick_plan_ingest_begin(rick_plan *p, uint64_t nrows, const double *uu, const double *vv,
                           const double *ww, const float *weight, int row_selection) {
  if (!p) return set_error(RICK_ERR_INVALID_ARG, "null plan");
  if (nrows > p->d.max_rows)
    return set_error(RICK_ERR_INVALID_ARG, "nrows exceeds the plan capacity");
  if (nrows && (!uu || !vv || !ww || !weight))
    return set_error(RICK_ERR_INVALID_ARG, "null row pointer");
  DeviceGuard guard(p->device);
  if (!p->ing_comp) {
    RICK_CUDA(cudaStreamCreateWithFlags(&p->ing_comp, cudaStreamNonBlocking));
    RICK_CUDA(cudaStreamCreateWithFlags(&p->ing_copy, cudaStreamNonBlocking));
    for (auto &e : p->ing_ev) RICK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  // a dataset left unfinished is abandoned
  RICK_CUDA(cudaStreamSynchronize(p->ing_copy));
  RICK_CUDA(cudaStreamSynchronize(p->ing_comp));
  p->ingest = false;
  RowsDev r;
  RICK_TRY(stage_rows(p, nrows, &r));
  const uint64_t npol = p->d.polarizations;
  RICK_TRY(h2d(r.uu, uu, nrows * 8, p->ing_comp));
  RICK_TRY(h2d(r.vv, vv, nrows * 8, p->ing_comp));
  RICK_TRY(h2d(r.ww, ww, nrows * 8, p->ing_comp));
  RICK_TRY(h2d(r.wt, weight, nrows * npol * 4, p->ing_comp));
  RICK_TRY(grid_begin(p, nrows, r.uu, r.vv, r.ww, row_selection == RICK_ROWS_SECTOR0,
                      1.0 / p->d.grid_size_x, 1.0 / p->d.num_w_planes, p->ing_comp));
  p->ingest = true;
  p->ing_rows = nrows;
  p->ing_next = 0;
  p->ing_k = 0;
  return RICK_OK;
}

int rick_plan_ingest_samples(rick_plan *p, uint64_t row0, uint64_t nrows, const float *vis_real,
                             const float *vis_img) {
  if (!p) return set_error(RICK_ERR_INVALID_ARG, "null plan");
  if (!p->ingest) return set_error(RICK_ERR_INVALID_ARG, "no ingest in progress");
  if (row0 != p->ing_next || row0 + nrows > p->ing_rows)
    return set_error(RICK_ERR_INVALID_ARG, "samples of rows %llu..%llu: expected the rows from %llu",
                     (unsigned long long)row0, (unsigned long long)(row0 + nrows),
                     (unsigned long long)p->ing_next);
  if (nrows && (!vis_real || !vis_img)) return set_error(RICK_ERR_INVALID_ARG, "null sample pointer");
  DeviceGuard guard(p->device);
  RowsDev r;
  RICK_TRY(stage_rows(p, p->ing_rows, &r));
  const uint64_t npol = p->d.polarizations, nv = (uint64_t)p->d.freq_per_chan * npol;
  const int k = p->ing_k & 1;
  RICK_TRY(h2d(r.vr + row0 * nv, vis_real, nrows * nv * 4, p->ing_copy));
  RICK_TRY(h2d(r.vi + row0 * nv, vis_img, nrows * nv * 4, p->ing_copy));
  RICK_CUDA(cudaEventRecord(p->ing_ev[k], p->ing_copy));
  RICK_CUDA(cudaStreamWaitEvent(p->ing_comp, p->ing_ev[k], 0));
  RICK_TRY(grid_samples(p, nrows, r.uu + row0, r.vv + row0, r.ww + row0, r.wt + row0 * npol,
                        r.vr + row0 * nv, r.vi + row0 * nv, p->ing_comp));
  // the previous slice's host buffers are free once its copy has completed
  if (p->ing_k > 0) RICK_CUDA(cudaEventSynchronize(p->ing_ev[k ^ 1]));
  p->ing_next += nrows;
  p->ing_k++;
  return RICK_OK;
}

int rick_plan_ingest_end(rick_plan *p, double resolution, double wmin, double wmax,
                         double *image_real, double *image_imag) {
  if (!p || !image_real || !image_imag) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  if (!p->ingest) return set_error(RICK_ERR_INVALID_ARG, "no ingest in progress");
  if (p->ing_next != p->ing_rows)
    return set_error(RICK_ERR_INVALID_ARG, "only %llu of %llu rows have their samples",
                     (unsigned long long)p->ing_next, (unsigned long long)p->ing_rows);
  DeviceGuard guard(p->device);
  p->ingest = false;
  RICK_TRY(grid_finish(p, p->ing_rows, 0, p->sparse, p->ing_comp));
  return image_to_host(p, p->ing_rows, resolution, wmin, wmax, image_real, image_imag,
                       p->ing_comp);
}

int rick_plan_export_cube(rick_plan *p, double *dst, int dst_is_host, void *stream) {
  if (!p || !dst) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  if (p->cube_state == kCubeSparse)
    return set_error(RICK_ERR_INVALID_ARG,
                     "rick_plan_image keeps no full cube; grid with rick_plan_grid to export it");
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const double scale = cube_scale(p);
  const uint64_t n = p->cube_vals;
  const int sms = num_sms();
  if (!dst_is_host) {
    if (p->d.precision == RICK_PREC_FP64)
      k_export_cube<double><<<sms * 8, 256, 0, st>>>((const double *)p->cube, dst, n, scale, 0);
    else
      k_export_cube<float><<<sms * 8, 256, 0, st>>>((const float *)p->cube, dst, n, scale, 0);
    RICK_CUDA(cudaGetLastError());
    g_launches++;
    return RICK_OK;
  }
  if (p->d.precision == RICK_PREC_FP64 && scale == 1.0) return copy_to_host(dst, p->cube, n * 8, st);
  if (!p->d_stage) {
    RICK_TRY(dev_alloc(p, (void **)&p->d_stage, kStageBytes));
    p->stage_bytes = kStageBytes;
  }
  const uint64_t per = p->stage_bytes / 8;
  for (uint64_t o = 0; o < n; o += per) {
    const uint64_t m = std::min(per, n - o);
    if (p->d.precision == RICK_PREC_FP64)
      k_export_cube<double><<<sms * 8, 256, 0, st>>>((const double *)p->cube + o, p->d_stage, m,
                                                     scale, 0);
    else
      k_export_cube<float><<<sms * 8, 256, 0, st>>>((const float *)p->cube + o, p->d_stage, m,
                                                    scale, 0);
    RICK_CUDA(cudaGetLastError());
    g_launches++;
    RICK_CUDA(cudaMemcpyAsync(dst + o, p->d_stage, m * 8, cudaMemcpyDeviceToHost, st));
    RICK_CUDA(cudaStreamSynchronize(st));
  }
  return RICK_OK;
}

int rick_plan_import_cube(rick_plan *p, const double *src, int src_is_host, void *stream) {
  if (!p || !src) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  const uint64_t n = p->cube_vals;
  if (p->d.precision == RICK_PREC_FP64) {
    if (src_is_host)
      RICK_TRY(copy_to_device(p->cube, src, n * 8, st));
    else
      RICK_CUDA(cudaMemcpyAsync(p->cube, src, n * 8, cudaMemcpyDeviceToDevice, st));
  } else {
    const int sms = num_sms();
    if (!src_is_host) {
      k_import_cube<<<sms * 8, 256, 0, st>>>(src, (float *)p->cube, n);
      RICK_CUDA(cudaGetLastError());
      g_launches++;
    } else {
      if (!p->d_stage) {
        RICK_TRY(dev_alloc(p, (void **)&p->d_stage, kStageBytes));
        p->stage_bytes = kStageBytes;
      }
      const uint64_t per = p->stage_bytes / 8;
      for (uint64_t o = 0; o < n; o += per) {
        const uint64_t m = std::min(per, n - o);
        RICK_CUDA(cudaMemcpyAsync(p->d_stage, src + o, m * 8, cudaMemcpyHostToDevice, st));
        k_import_cube<<<sms * 8, 256, 0, st>>>(p->d_stage, (float *)p->cube + o, m);
        RICK_CUDA(cudaGetLastError());
        g_launches++;
        RICK_CUDA(cudaStreamSynchronize(st));
      }
    }
  }
  p->cube_state = kCubeNormalised;
  return RICK_OK;
}

int rick_plan_get_stats(rick_plan *p, rick_plan_stats *out) {
  if (!p || !out) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(p->device);
  uint64_t c[kNumCounters];
  RICK_CUDA(cudaDeviceSynchronize());
  RICK_CUDA(cudaMemcpy(c, p->s.counters, sizeof(c), cudaMemcpyDeviceToHost));
  memset(out, 0, sizeof(*out));
  out->rows_in = p->last_rows;
  out->rows_gridded = c[kCntGridded];
  out->rows_dropped = c[kCntDropped];
  out->records = c[kCntRecords];
  uint32_t items = 0;
  RICK_CUDA(cudaMemcpy(&items, p->s.item_off + p->g.nbins(), 4, cudaMemcpyDeviceToHost));
  out->work_items = items;
  out->device_bytes = p->device_bytes;
  out->rows_other_shard = c[kCntOtherShard];
  if (p->cube_state == kCubeSparse) {
    uint32_t rows = 0;
    RICK_CUDA(cudaMemcpy(&rows, p->f.counts, 4, cudaMemcpyDeviceToHost));
    out->fft_rows = rows;
  }
  return RICK_OK;
}

// ---- internal hooks used by the drop-in entry points (dropin.cu) ----------
int rick_internal_plan_grid_accumulate(rick_plan *p, uint64_t nrows, const double *uu,
                                       const double *vv, const double *ww, const float *weight,
                                       const float *vis_re, const float *vis_im, double dx,
                                       double dw, void *stream) {
  DeviceGuard guard(p->device);
  return plan_grid_impl(p, nrows, uu, vv, ww, weight, vis_re, vis_im, 0, 1, dx, dw,
                        (cudaStream_t)stream);
}

int rick_internal_plan_mark_raw(rick_plan *p) {
  p->cube_state = kCubeRaw;
  return RICK_OK;
}

int rick_internal_plan_phase_full(rick_plan *p, int xtot, int ytot, double resolution,
                                  double wmin, double wmax, double *img_re, double *img_im,
                                  int accumulate, void *stream) {
  DeviceGuard guard(p->device);
  return plan_phase_impl(p, xtot, ytot, resolution, wmin, wmax, img_re, img_im, accumulate,
                         (cudaStream_t)stream);
}

const rick_plan_desc *rick_internal_plan_desc(const rick_plan *p) { return &p->d; }

int rick_plan_set_timing(rick_plan *p, int on) {
  if (!p) return set_error(RICK_ERR_INVALID_ARG, "null plan");
  DeviceGuard guard(p->device);
  if (on && !p->ev[0]) {
    for (cudaEvent_t &e : p->ev) RICK_CUDA(cudaEventCreate(&e));
    RICK_CUDA(cudaEventCreate(&p->ev_fft0));
    RICK_CUDA(cudaEventCreate(&p->ev_phase0));
  }
  p->timing = on != 0;
  return RICK_OK;
}

int rick_plan_stage_ms(rick_plan *p, float *ms, int n) {
  if (!p || !ms) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  DeviceGuard guard(p->device);
  if (!p->ev[0]) return set_error(RICK_ERR_INVALID_ARG, "stage timing was never enabled");
  RICK_CUDA(cudaDeviceSynchronize());
  const cudaEvent_t start[RICK_NUM_STAGES] = {p->ev[0], p->ev[1], p->ev[2], p->ev[3], p->ev_fft0, p->ev_phase0};
  const cudaEvent_t stop[RICK_NUM_STAGES] = {p->ev[1], p->ev[2], p->ev[3], p->ev[4], p->ev[5], p->ev[6]};
  for (int k = 0; k < n && k < RICK_NUM_STAGES; k++) {
    ms[k] = -1.0f;
    if (p->ran[k]) RICK_CUDA(cudaEventElapsedTime(&ms[k], start[k], stop[k]));
  }
  return RICK_OK;
}

const char *rick_last_error_message(void) { return g_msg; }

unsigned long long rick_launch_count(void) { return g_launches.load(); }

}  // extern "C"
