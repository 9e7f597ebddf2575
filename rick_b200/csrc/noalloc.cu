// rick_wstack_noalloc: gridding of device-resident rows into a caller-owned
// device cube without any device allocation.
//
// The plan API allocates its scratch (bin histogram and offsets, binned row
// records, counters, the kernel table) with cudaMalloc when a plan is created.
// Some callers cannot allocate at run time: real-time pipelines that reserve all
// device memory at start-up and may not grow it inside the streaming loop
// (cudaMalloc can synchronise the device and stall concurrent streams), and host
// frameworks that own the GPU's memory pool and forbid libraries from calling
// the CUDA allocator.  This entry point serves them: the same binning and tiled
// gridding kernels run with their scratch carved out of one statically sized
// __device__ array that lives as long as the library stays loaded.
//
// Limits and rules (also stated in include/rick_b200.h):
//  * the scratch holds kNoAllocScratchBytes (32 MiB) on every device that loads
//    the library; a job whose scratch would not fit is rejected with
//    RICK_ERR_INVALID_ARG before anything runs (rick_wstack_noalloc_capacity
//    reports the limit for a geometry);
//  * every call shares the array and it keeps the last call's contents: each
//    call clears the parts that must start at zero, and calls whose GPU work
//    overlaps (different streams, or host threads) race on it;
//  * the first call on a device sets that device up: it looks the arrays'
//    device addresses up with cudaGetSymbolAddress (host code only holds a
//    stand-in for each symbol) and fills the kernel tables of every kernel and
//    support with one synchronous copy, so make that first call before any
//    stream capture (a first call on a capturing stream is refused); later
//    calls copy nothing from the host.
#include <string.h>

#include <mutex>

#include "rick_internal.h"

namespace rick {
namespace {

constexpr size_t kNoAllocScratchBytes = 32ull << 20;
constexpr int kMaxDev = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Kernel tables of the three kernels at every odd support 1..kMaxSupport
// (w-stacking.cu:35-89), filled once per device when the device is set up.
constexpr int kTabLen = kIncreasePrecision * kMaxSupport;
constexpr int kSupports = (kMaxSupport + 1) / 2;
static __device__ __align__(256) double g_noalloc_tables[3][kSupports][kTabLen];

std::mutex g_mu;
struct DevArrays {
  void *scratch;
  double *tables;
};
DevArrays g_dev[kMaxDev] = {};

// Device addresses of the static arrays on the current device; the first call
// on a device looks them up and fills the tables (synchronously).
int device_arrays(cudaStream_t st, DevArrays *out) {
  int dev = 0;
  RICK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDev) return set_error(RICK_ERR_UNSUPPORTED, "device ordinal %d", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_dev[dev].scratch) {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    RICK_CUDA(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone)
      return set_error(RICK_ERR_INVALID_ARG,
                       "rick_wstack_noalloc: the first call on a device sets it up and must come "
                       "before any stream capture");
    DevArrays a{};
    cudaError_t e = cudaGetSymbolAddress(&a.scratch, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(scratch)", __FILE__, __LINE__);
    void *t = nullptr;
    e = cudaGetSymbolAddress(&t, g_noalloc_tables);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(tables)", __FILE__, __LINE__);
    a.tables = (double *)t;
    static double host[3][kSupports][kTabLen];
    for (int k = 0; k < 3; k++)
      for (int i = 0; i < kSupports; i++) make_table(k, 2 * i + 1, host[k][i]);
    RICK_CUDA(cudaMemcpy(a.tables, host, sizeof(host), cudaMemcpyHostToDevice));
    g_dev[dev] = a;
  }
  *out = g_dev[dev];
  return RICK_OK;
}

struct Layout {
  size_t counters, bin_count, bin_cursor, item_off, scan_tmp, records, total;
};

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

Layout layout_for(uint64_t nbins, uint64_t nrows) {
  Layout L;
  size_t o = 0;
  L.counters = o;   o += up256(kNumCounters * sizeof(uint64_t));
  L.bin_count = o;  o += up256((nbins + 1) * 4);
  L.bin_cursor = o; o += up256(nbins * 4);
  L.item_off = o;   o += up256((nbins + 1) * 4);
  L.scan_tmp = o;   o += up256(scan_tmp_words(nbins + 1) * 4);
  L.records = o;    o += up256(4 * nrows * sizeof(RecF64));
  L.total = o;
  return L;
}

}  // namespace
}  // namespace rick

using namespace rick;

extern "C" {

int rick_wstack_noalloc_capacity(int num_w_planes, int grid_size_x, int grid_size_y,
                                 uint64_t *max_rows) {
  if (!max_rows || num_w_planes <= 0 || grid_size_x <= 0 || grid_size_y <= 0)
    return set_error(RICK_ERR_INVALID_ARG, "rick_wstack_noalloc_capacity: bad argument");
  const uint64_t tiles = (uint64_t)((grid_size_x + kTile - 1) / kTile) *
                        (uint64_t)((grid_size_y + kTile - 1) / kTile);
  if (tiles >= (1ull << 32) || tiles * (uint64_t)num_w_planes >= (1ull << 32)) {  // < 2^63: no wrap
    *max_rows = 0;
    return RICK_OK;
  }
  const uint64_t nbins = tiles * (uint64_t)num_w_planes;
  // total(n) = base + up256(4*n*sizeof(RecF64)): the largest n whose padded
  // record block still fits (n + 1 rows do not fit)
  const Layout L = layout_for(nbins, 0);
  const size_t avail = L.total >= kNoAllocScratchBytes
                           ? 0
                           : (kNoAllocScratchBytes - L.total) & ~(size_t)255;
  *max_rows = avail / (4 * sizeof(RecF64));
  return RICK_OK;
}

int rick_wstack_noalloc(int num_w_planes, uint64_t num_points, uint32_t freq_per_chan,
                        uint32_t polarizations, const double *uu, const double *vv,
                        const double *ww, const float *vis_real, const float *vis_img,
                        const float *weight, double dx, double dw, int w_support, int kernel,
                        int grid_size_x, int grid_size_y, double *grid, void *stream) {
  if (!grid || (num_points && (!uu || !vv || !ww || !vis_real || !vis_img || !weight)))
    return set_error(RICK_ERR_INVALID_ARG, "rick_wstack_noalloc: null pointer");
  if (num_w_planes <= 0 || grid_size_x <= 0 || grid_size_y <= 0 || freq_per_chan == 0 ||
      polarizations == 0)
    return set_error(RICK_ERR_INVALID_ARG, "rick_wstack_noalloc: non-positive size");
  if (w_support < 1 || w_support > kMaxSupport || w_support % 2 == 0)
    return set_error(RICK_ERR_INVALID_ARG, "rick_wstack_noalloc: w_support must be odd in [1,%d]",
                     kMaxSupport);
  if (kernel < RICK_KERNEL_GAUSS || kernel > RICK_KERNEL_KAISER_BESSEL)
    return set_error(RICK_ERR_INVALID_ARG, "rick_wstack_noalloc: unknown kernel %d", kernel);
  Geometry g{};
  g.nx = grid_size_x;
  g.ny = grid_size_y;
  g.nw = num_w_planes;
  g.support = w_support;
  g.half = (w_support - 1) / 2;
  g.ntx = (g.nx + kTile - 1) / kTile;
  g.nty = (g.ny + kTile - 1) / kTile;
  g.dx = dx;
  g.dw = dw;
  g.w_supporth = (double)g.half * (1.0 / (double)g.nx);
  g.select_sector0 = 0;
  const uint64_t tiles = (uint64_t)g.ntx * (uint64_t)g.nty;  // < 2^52
  const uint64_t nbins = tiles < (1ull << 32) ? g.nbins() : ~0ull;
  // bounds that keep the layout arithmetic below from wrapping: no job with
  // more rows than the scratch holds records for, bin indices in 32 bits
  if (num_points > kNoAllocScratchBytes / (4 * sizeof(RecF64)) || nbins >= (1ull << 32))
    return set_error(RICK_ERR_INVALID_ARG,
                     "rick_wstack_noalloc: %llu rows / %llu bins exceed the static scratch "
                     "(%llu bytes)", (unsigned long long)num_points, (unsigned long long)nbins,
                     (unsigned long long)kNoAllocScratchBytes);
  const Layout L = layout_for(nbins, num_points);
  if (L.total > kNoAllocScratchBytes)
    return set_error(RICK_ERR_INVALID_ARG,
                     "rick_wstack_noalloc: the job needs %llu bytes of scratch but the static "
                     "scratch holds %llu (fewer rows or a smaller grid)",
                     (unsigned long long)L.total, (unsigned long long)kNoAllocScratchBytes);
  cudaStream_t st = (cudaStream_t)stream;
  DevArrays arr{};
  RICK_TRY(device_arrays(st, &arr));
  char *b = (char *)arr.scratch;
  Scratch s{};
  s.counters = (uint64_t *)(b + L.counters);
  s.table = arr.tables + ((size_t)kernel * kSupports + (w_support - 1) / 2) * kTabLen;
  s.bin_count = (uint32_t *)(b + L.bin_count);
  s.bin_cursor = (uint32_t *)(b + L.bin_cursor);
  s.item_off = (uint32_t *)(b + L.item_off);
  s.scan_tmp = (uint32_t *)(b + L.scan_tmp);
  s.records = (RecF64 *)(b + L.records);
  s.max_records = 4 * num_points;
  // what must start at zero: the counters (bin counts and cursors are cleared
  // by bin_rows itself), and the caller's cube (overwrite semantics)
  RICK_CUDA(cudaMemsetAsync(s.counters, 0, kNumCounters * sizeof(uint64_t), st));
  const uint64_t per = num_points / ((uint64_t)num_sms() * 4 + 1);
  const uint32_t chunk = (uint32_t)(per < 1024 ? 1024 : (per > 8192 ? 8192 : per));
  RICK_TRY(bin_rows(g, kernel, RICK_PREC_FP64, num_points, uu, vv, ww, weight, vis_real, vis_img,
                    freq_per_chan, polarizations, s, chunk, st));
  RICK_CUDA(cudaMemsetAsync(grid, 0, 2ull * num_w_planes * grid_size_x * grid_size_y * 8, st));
  RICK_TRY(grid_tiles(g, kernel, RICK_PREC_FP64, s, grid, 0, chunk, st));
  return RICK_OK;
}

}  // extern "C"
