// Drop-in entry points with the reference's C prototypes (w-stacking.h:39-83)
// and the FFT step of fourier_transform.c:13-93 on explicit buffers.
//
// They keep one cached plan per device (grown when a call needs more capacity)
// so repeated calls do not re-allocate.  Host buffers cross PCIe on every call,
// as in the reference's CUDA wstack (w-stacking.cu:338-348, :414) and
// phase_correction (phase_correction.cu:137-138, :171-173) -- through pinned
// staging buffers filled by a pool of host threads when the caller's memory is
// pageable (hostcopy.cu); device-resident callers use the plan API instead.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>

#include "rick_internal.h"

using namespace rick;

extern "C" {
int rick_internal_plan_grid_accumulate(rick_plan *p, uint64_t nrows, const double *uu,
                                       const double *vv, const double *ww, const float *weight,
                                       const float *vis_re, const float *vis_im, double dx,
                                       double dw, void *stream);
int rick_internal_plan_mark_raw(rick_plan *p);
int rick_internal_plan_phase_full(rick_plan *p, int xtot, int ytot, double resolution,
                                  double wmin, double wmax, double *img_re, double *img_im,
                                  int accumulate, void *stream);
const rick_plan_desc *rick_internal_plan_desc(const rick_plan *p);
}

namespace {

std::mutex g_mu;
int g_kernel = -1;     // -1: read RICK_KERNEL on first use
int g_phase_on = -1;   // -1: read RICK_PHASE_ON on first use
int g_device = -1;     // -1: rank % device_count
thread_local int g_last_status = RICK_OK;
constexpr int kMaxDevices = 64;
rick_plan *g_plans[kMaxDevices] = {};
uint64_t g_plans_created = 0;   // plans the drop-ins have created in this process
uint64_t g_row_allocs = 0;      // device allocations of their row buffers
double *g_dimg[kMaxDevices] = {};
uint64_t g_dimg_vals[kMaxDevices] = {};

int kernel_setting() {
  if (g_kernel < 0) {
    g_kernel = RICK_KERNEL_KAISER_BESSEL;  // Makefile:70 default
    const char *e = getenv("RICK_KERNEL");
    if (e) {
      if (!strcmp(e, "gauss") || !strcmp(e, "GAUSS")) g_kernel = RICK_KERNEL_GAUSS;
      else if (!strcmp(e, "gauss_hi") || !strcmp(e, "GAUSS_HI_PRECISION"))
        g_kernel = RICK_KERNEL_GAUSS_HI_PRECISION;
      else if (!strcmp(e, "kaiser_bessel") || !strcmp(e, "KAISERBESSEL"))
        g_kernel = RICK_KERNEL_KAISER_BESSEL;
    }
  }
  return g_kernel;
}

int phase_setting() {
  if (g_phase_on < 0) {
    const char *e = getenv("RICK_PHASE_ON");
    g_phase_on = (e && (!strcmp(e, "0") || !strcmp(e, "off"))) ? 0 : 1;  // Makefile:56 default on
  }
  return g_phase_on;
}

int pick_device(int rank, int *dev) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return set_error(RICK_ERR_NO_ACCELERATORS_FOUND, "No accelerators found");
  }
  *dev = g_device >= 0 ? g_device % n : (rank < 0 ? 0 : rank % n);  // w-stacking.cu:279-281
  if (*dev >= kMaxDevices) return set_error(RICK_ERR_UNSUPPORTED, "device ordinal too large");
  RICK_CUDA(cudaSetDevice(*dev));
  return RICK_OK;
}

// The cached plan of a device serves every drop-in call on the same cube:
// wstack needs its gridding settings (support, kernel, channels,
// polarisations, row capacity) as well; rick_fft_planes and phase_correction
// need only the cube's geometry and the PHASE_ON setting, so the reference's
// call sequence wstack -> fft -> phase_correction, repeated, reuses one plan
// (and its HBM) throughout.  A plan is re-created only when a call needs
// something the cached one lacks.
enum class Need { kGrid, kCube };

int get_plan(int dev, Need need, int nx, int ny, int nw, int support, int kernel, uint64_t rows,
             uint32_t nchan, uint32_t npol, rick_plan **out) {
  rick_plan *p = g_plans[dev];
  if (p) {
    const rick_plan_desc *d = rick_internal_plan_desc(p);
    bool ok = d->grid_size_x == nx && d->grid_size_y == ny && d->num_w_planes == nw &&
              d->phase_on == phase_setting();
    if (need == Need::kGrid)
      ok = ok && d->w_support == support && d->kernel == kernel && d->max_rows >= rows &&
           d->freq_per_chan == nchan && d->polarizations == npol;
    if (!ok) {
      rick_plan_destroy(p);
      g_plans[dev] = p = nullptr;
    }
  }
  if (!p) {
    rick_plan_desc d{};
    d.grid_size_x = nx;
    d.grid_size_y = ny;
    d.num_w_planes = nw;
    d.w_support = support;
    d.kernel = kernel;
    d.precision = RICK_PREC_FP64;
    d.phase_on = phase_setting();
    d.device = dev;
    d.max_rows = rows + rows / 2 + 1;
    d.freq_per_chan = nchan;
    d.polarizations = npol;
    RICK_TRY(rick_plan_create(&p, &d));
    g_plans[dev] = p;
    g_plans_created++;
  }
  *out = p;
  return RICK_OK;
}

// Device copies of wstack's row arrays, kept per device across calls and grown
// (with headroom) when a call brings more rows or samples.
struct RowBufs {
  double *uvw = nullptr;
  float *wt = nullptr, *vr = nullptr, *vi = nullptr;
  uint64_t cap_uvw = 0, cap_wt = 0, cap_vr = 0, cap_vi = 0;
};
RowBufs g_rows[kMaxDevices];

template <typename T>
int grow(T **ptr, uint64_t *cap, uint64_t n) {
  if (*cap >= n && *ptr) return RICK_OK;
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  *cap = 0;
  const uint64_t want = n + n / 4 + 16;
  const cudaError_t e = cudaMalloc((void **)ptr, want * sizeof(T));
  if (e != cudaSuccess) {
    *ptr = nullptr;
    return cuda_status(e, "cudaMalloc", __FILE__, __LINE__);
  }
  g_row_allocs++;
  *cap = want;
  return RICK_OK;
}

int do_wstack(int nw, unsigned int npts, unsigned int nchan, unsigned int npol, const double *uu,
              const double *vv, const double *ww, const float *vr, const float *vi,
              const float *wt, double dx, double dw, int support, int nx, int ny, double *grid,
              int rank) {
  if (!grid || (npts && (!uu || !vv || !ww || !vr || !vi || !wt)))
    return set_error(RICK_ERR_INVALID_ARG, "wstack: null pointer");
  if (nw <= 0 || nx <= 0 || ny <= 0 || nchan == 0 || npol == 0)
    return set_error(RICK_ERR_INVALID_ARG, "wstack: non-positive size");
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  RICK_TRY(pick_device(rank, &dev));
  rick_plan *p = nullptr;
  RICK_TRY(get_plan(dev, Need::kGrid, nx, ny, nw, support, kernel_setting(), npts, nchan, npol,
                    &p));
  const uint64_t nv = (uint64_t)npts * nchan * npol;
  RowBufs &b = g_rows[dev];
  RICK_TRY(grow(&b.uvw, &b.cap_uvw, 3ull * npts));
  RICK_TRY(grow(&b.wt, &b.cap_wt, (uint64_t)npts * npol));
  RICK_TRY(grow(&b.vr, &b.cap_vr, nv));
  RICK_TRY(grow(&b.vi, &b.cap_vi, nv));
  struct { double *ptr; } duvw{b.uvw};
  struct { float *ptr; } dwt{b.wt}, dvr{b.vr}, dvi{b.vi};
  cudaStream_t st = 0;
  RICK_TRY(copy_to_device(duvw.ptr, uu, npts * 8ull, st));
  RICK_TRY(copy_to_device(duvw.ptr + npts, vv, npts * 8ull, st));
  RICK_TRY(copy_to_device(duvw.ptr + 2ull * npts, ww, npts * 8ull, st));
  RICK_TRY(copy_to_device(dwt.ptr, wt, (uint64_t)npts * npol * 4, st));
  RICK_TRY(copy_to_device(dvr.ptr, vr, nv * 4, st));
  RICK_TRY(copy_to_device(dvi.ptr, vi, nv * 4, st));
  // accumulate semantics (w-stacking.cu:530-532): start from the caller's grid
  RICK_TRY(rick_plan_import_cube(p, grid, 1, st));
  RICK_TRY(rick_internal_plan_mark_raw(p));
  RICK_TRY(rick_internal_plan_grid_accumulate(p, npts, duvw.ptr, duvw.ptr + npts,
                                              duvw.ptr + 2ull * npts, dwt.ptr, dvr.ptr, dvi.ptr,
                                              dx, dw, st));
  RICK_TRY(rick_plan_export_cube(p, grid, 1, st));
  RICK_CUDA(cudaStreamSynchronize(st));
  return RICK_OK;
}

int do_phase(double *gridss, double *img_re, double *img_im, int xaxis, int yaxis, int nw,
             int xtot, int ytot, double resolution, double wmin, double wmax, int rank) {
  if (!gridss || !img_re || !img_im) return set_error(RICK_ERR_INVALID_ARG, "phase_correction: null pointer");
  if (xaxis <= 0 || yaxis <= 0 || nw <= 0)
    return set_error(RICK_ERR_INVALID_ARG, "phase_correction: non-positive size");
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  RICK_TRY(pick_device(rank, &dev));
  rick_plan *p = nullptr;
  RICK_TRY(get_plan(dev, Need::kCube, xaxis, yaxis, nw, 7, kernel_setting(), 1, 1, 1, &p));
  const uint64_t plane = (uint64_t)xaxis * yaxis;
  if (g_dimg_vals[dev] < 2 * plane) {
    if (g_dimg[dev]) cudaFree(g_dimg[dev]);
    g_dimg[dev] = nullptr;
    RICK_CUDA(cudaMalloc(&g_dimg[dev], 16 * plane));
    g_dimg_vals[dev] = 2 * plane;
  }
  double *dimg = g_dimg[dev];
  cudaStream_t st = 0;
  RICK_TRY(rick_plan_import_cube(p, gridss, 1, st));
  // the CPU path accumulates into the caller's image (phase_correction.cu:233-235)
  RICK_CUDA(cudaMemcpyAsync(dimg, img_re, plane * 8, cudaMemcpyHostToDevice, st));
  RICK_CUDA(cudaMemcpyAsync(dimg + plane, img_im, plane * 8, cudaMemcpyHostToDevice, st));
  RICK_TRY(rick_internal_plan_phase_full(p, xtot, ytot, resolution, wmin, wmax, dimg,
                                         dimg + plane, 1, st));
  RICK_CUDA(cudaMemcpyAsync(img_re, dimg, plane * 8, cudaMemcpyDeviceToHost, st));
  RICK_CUDA(cudaMemcpyAsync(img_im, dimg + plane, plane * 8, cudaMemcpyDeviceToHost, st));
  RICK_CUDA(cudaStreamSynchronize(st));
  return RICK_OK;
}

int do_fft(const double *grid, double *gridss, int nw, int nx, int ny) {
  if (!grid || !gridss) return set_error(RICK_ERR_INVALID_ARG, "rick_fft_planes: null pointer");
  if (nw <= 0 || nx <= 0 || ny <= 0)
    return set_error(RICK_ERR_INVALID_ARG, "rick_fft_planes: non-positive size");
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  RICK_TRY(pick_device(0, &dev));
  rick_plan *p = nullptr;
  RICK_TRY(get_plan(dev, Need::kCube, nx, ny, nw, 7, kernel_setting(), 1, 1, 1, &p));
  cudaStream_t st = 0;
  RICK_TRY(rick_plan_import_cube(p, grid, 1, st));
  RICK_TRY(rick_internal_plan_mark_raw(p));
  RICK_TRY(rick_plan_fft(p, st));
  RICK_TRY(rick_plan_export_cube(p, gridss, 1, st));
  RICK_CUDA(cudaStreamSynchronize(st));
  return RICK_OK;
}

void report(const char *fn, int st) {
  g_last_status = st;
  if (st != RICK_OK)
    fprintf(stderr, "%s: error %d (%s): %s\n", fn, st, rick_status_string(st),
            rick_last_error_message());
}

}  // namespace

extern "C" {

void wstack(int num_w_planes, unsigned int num_points, unsigned int freq_per_chan,
            unsigned int polarizations, double *uu, double *vv, double *ww, float *vis_real,
            float *vis_img, float *weight, double dx, double dw, int w_support, int grid_size_x,
            int grid_size_y, double *grid, int num_threads, int rank) {
  (void)num_threads;
  report("wstack", do_wstack(num_w_planes, num_points, freq_per_chan, polarizations, uu, vv, ww,
                             vis_real, vis_img, weight, dx, dw, w_support, grid_size_x,
                             grid_size_y, grid, rank));
}

void phase_correction(double *gridss, double *image_real, double *image_imag, int xaxis,
                      int yaxis, int num_w_planes, int xaxistot, int yaxistot, double resolution,
                      double wmin, double wmax, int num_threads, int rank) {
  (void)num_threads;
  report("phase_correction", do_phase(gridss, image_real, image_imag, xaxis, yaxis, num_w_planes,
                                      xaxistot, yaxistot, resolution, wmin, wmax, rank));
}

int rick_fft_planes(const double *grid, double *gridss, int num_w_planes, int grid_size_x,
                    int grid_size_y) {
  const int st = do_fft(grid, gridss, num_w_planes, grid_size_x, grid_size_y);
  report("rick_fft_planes", st);
  return st;
}

int rick_set_kernel(int kernel) {
  if (kernel < RICK_KERNEL_GAUSS || kernel > RICK_KERNEL_KAISER_BESSEL)
    return set_error(RICK_ERR_INVALID_ARG, "unknown kernel %d", kernel);
  std::lock_guard<std::mutex> lock(g_mu);
  g_kernel = kernel;
  return RICK_OK;
}

int rick_set_phase_on(int on) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_phase_on = on ? 1 : 0;
  return RICK_OK;
}

int rick_set_device(int device) {
  std::lock_guard<std::mutex> lock(g_mu);
  g_device = device;
  return RICK_OK;
}

int rick_last_status(void) { return g_last_status; }

int rick_dropin_release(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  int prev = 0;
  cudaGetDevice(&prev);
  for (int dev = 0; dev < kMaxDevices; dev++) {
    RowBufs &b = g_rows[dev];
    if (!g_plans[dev] && !g_dimg[dev] && !b.uvw && !b.wt && !b.vr && !b.vi) continue;
    RICK_CUDA(cudaSetDevice(dev));
    if (g_plans[dev]) rick_plan_destroy(g_plans[dev]);
    g_plans[dev] = nullptr;
    if (g_dimg[dev]) cudaFree(g_dimg[dev]);
    g_dimg[dev] = nullptr;
    g_dimg_vals[dev] = 0;
    for (void *p : {(void *)b.uvw, (void *)b.wt, (void *)b.vr, (void *)b.vi})
      if (p) cudaFree(p);
    b = RowBufs{};
  }
  cudaSetDevice(prev);
  return RICK_OK;
}

int rick_dropin_counters(uint64_t *plans_created, uint64_t *row_allocations) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (plans_created) *plans_created = g_plans_created;
  if (row_allocations) *row_allocations = g_row_allocs;
  return RICK_OK;
}

const char *rick_status_string(int status) {
  switch (status) {
    case RICK_OK: return "ok";
    case RICK_ERR_NO_THREADS_SUPPORT: return "no threads support";
    case RICK_ERR_IN_PARAMFILE: return "error in paramfile";
    case RICK_ERR_NOT_ENOUGH_MEM: return "not enough memory";
    case RICK_ERR_REDUCE: return "reduce error";
    case RICK_ERR_INVALID_ARG: return "invalid argument";
    case RICK_ERR_CUDA: return "CUDA error";
    case RICK_ERR_CUFFT: return "cuFFT error";
    case RICK_ERR_IO: return "I/O error";
    case RICK_ERR_UNSUPPORTED: return "unsupported";
    case RICK_ERR_BUDGET: return "HBM budget exceeded";
    case RICK_ERR_CANCELLED: return "cancelled";
    case RICK_ERR_NO_ACCELERATORS_FOUND: return "no accelerators found";
    default: return "unknown status";
  }
}

int rick_host_alloc(void **ptr, uint64_t bytes) {
  if (!ptr) return set_error(RICK_ERR_INVALID_ARG, "null pointer");
  *ptr = nullptr;
  const cudaError_t e = cudaMallocHost(ptr, bytes ? bytes : 1);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver
                         ? RICK_ERR_NO_ACCELERATORS_FOUND
                         : RICK_ERR_NOT_ENOUGH_MEM,
                     "cudaMallocHost of %llu bytes: %s", (unsigned long long)bytes,
                     cudaGetErrorString(e));
  }
  return RICK_OK;
}

int rick_host_free(void *ptr) {
  if (ptr) cudaFreeHost(ptr);
  return RICK_OK;
}

int rick_kernel_names(const char **names, int max_names) {
  static const char *k[] = {"k_bin_count",        "k_item_count",       "k_bin_scatter",
                            "k_scan_block",       "k_scan_add",         "k_grid_tiles",
                            "k_zero_split_tiles", "k_row_list",         "k_fft_units",
                            "k_fft_rows",         "k_fft_cols_image",   "k_fft_cols_tm",      "k_fft_cols_tm_multi", "k_fft_cols_pair", "k_fft_cols_pair_multi", "k_fft_cols_split", "k_phase_sum",
                            "k_export_cube",      "k_import_cube",      "k_bin_count_batch",
                            "k_bin_scatter_batch", "k_grid_tiles_batch", "k_zero_split_tiles_batch",
                            "k_fft_rows_multi",   "k_fft_cols_multi",   "k_uvw_init",
                            "k_uvw_extrema",      "k_uvw_normalize"};
  const int n = (int)(sizeof(k) / sizeof(k[0]));
  for (int i = 0; i < n && i < max_names; i++) names[i] = k[i];
  return n;
}

}  // extern "C"
