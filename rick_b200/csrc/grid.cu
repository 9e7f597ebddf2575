// Tiled convolutional gridding onto the w-stacked cube.
//
// Replaces convolve_g (w-stacking.cu:104-206), which scatters every footprint
// cell of every row with two FP64 atomics straight into HBM.  Here a persistent
// kernel takes work items (a bounded chunk of the binned records of one
// 32x32 tile of one w-plane), accumulates their footprints in shared memory as
// exact 64-bit fixed-point sums (weights and products formed in FP64; each
// item scales its contributions by a power of two chosen from a bound on its
// records, so that no sum can overflow), and writes the tile once: with
// plain coalesced stores when the tile is
// a single item, or with one atomic per non-zero cell when a dense tile was
// split over several items.  The kernel weights follow w-stacking.cu:162-180:
//   u_dist = j + 0.5 - pos_u, table index (int)(5*|u_dist + KernelLen|),
//   weight tab[jKer]*tab[kKer] (Gaussian / Kaiser-Bessel tables), or
//   norm*exp(-(u_dist^2+v_dist^2)*std22) (high-precision Gaussian, evaluated
//   as norm*exp(-u^2*std22)*exp(-v^2*std22)).
// Table indices are computed with round-to-nearest intrinsics in FP64 from the
// exact fractional position, so they equal the reference's indices bit for bit.
#include <algorithm>

#include "rick_internal.h"

namespace rick {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kPitch = kTile + 1;  // shared-memory row pitch (avoids bank conflicts)

template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// The shared tile: per cell and component a two's-complement fixed-point sum,
// because 32-bit integer atomics are the fast shared-memory atomics (about 3x
// the FP32 and 6x the FP64 add rate on B200).  The plain form keeps 64-bit
// sums as two 32-bit words: an add puts the low word in with an atomic that
// returns the old value, and the carry out of the low word goes into the high
// word with the high part.  The mixed form, whose tiles are FP32, keeps one
// 32-bit word (resolution 2^-30 of the item's bound, finer than FP32 rounding
// of the cells that matter).  Integer sums do not depend on the order of the
// adds, so a tile's sum is reproducible.
struct FixTile {
  uint32_t lo_re[kTile * kPitch], hi_re[kTile * kPitch];
  uint32_t lo_im[kTile * kPitch], hi_im[kTile * kPitch];
};
template <typename OutT> __host__ __device__ constexpr int fix_bits() { return sizeof(OutT) == 8 ? 61 : 30; }

// The arithmetic type of a footprint cell's contribution: FP64 for the plain
// form; FP32 for the mixed form, whose tiles are FP32 -- its weights, products
// and float-to-integer conversions then run on the FP32 pipes (the FP64
// conversion to integer is a slow instruction), rounding each contribution at
// about 6e-8 of itself against the 2^-30 of the item's bound the 32-bit sums
// resolve.
template <typename OutT> struct Contrib { using type = double; };
template <> struct Contrib<float> { using type = float; };

__device__ __forceinline__ void fix_put_v(uint32_t *lo, uint32_t *hi, double v) {
  const long long x = __double2ll_rn(v);
  const uint32_t l = (uint32_t)(unsigned long long)x;
  const uint32_t h = (uint32_t)((unsigned long long)x >> 32);
  const uint32_t old = atomicAdd(lo, l);
  atomicAdd(hi, h + ((old + l) < old ? 1u : 0u));
}
__device__ __forceinline__ void fix_put_v(uint32_t *lo, uint32_t *, float v) {
  atomicAdd(lo, (uint32_t)__float2int_rn(v));
}
template <typename OutT>
__device__ __forceinline__ void fix_put(uint32_t *lo, uint32_t *hi,
                                        typename Contrib<OutT>::type v) {
  fix_put_v(lo, hi, v);
}

template <typename OutT>
__device__ __forceinline__ double fix_value(const uint32_t *lo, const uint32_t *hi, int c) {
  if constexpr (sizeof(OutT) == 8)
    return (double)(long long)(((unsigned long long)hi[c] << 32) | (unsigned long long)lo[c]);
  else
    return (double)(int)lo[c];
}

__device__ __forceinline__ void fix_zero(FixTile *t) {
  for (int c = threadIdx.x; c < kTile * kPitch; c += blockDim.x) {
    t->lo_re[c] = 0u;
    t->hi_re[c] = 0u;
    t->lo_im[c] = 0u;
    t->hi_im[c] = 0u;
  }
}

// Largest |weight product| of a footprint cell: the high-precision Gaussian's
// u factor carries norm (w-stacking.cu:256), the tables' entries are at most
// their maximum.
__device__ __forceinline__ double weight_bound(bool hi, const double *s_tab, int ntab) {
  if (hi) return kStd22 / kPi;
  double m = 0.0;
  for (int t = 0; t < ntab; t++) m = fmax(m, fabs(s_tab[t]));
  return m * m;
}

// Scale 2^k of an item's fixed-point sums: every |cell sum| is at most
// bound = sum over the records of (|sre| + |sim|) * wmax < 2^e, and sums are
// kept below 2^bits (k = bits - e, clamped to the double exponent range).  All
// threads take part; returns the scale, *inv = 2^-k.
__device__ __forceinline__ double item_scale(const RecF64 *__restrict__ rec, uint32_t r0,
                                             uint32_t r1, double wmax, int bits, double *s_red,
                                             double *inv) {
  double part = 0.0;
  for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x)
    part += fabs(rec[r].sre) + fabs(rec[r].sim);
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = part;
  __syncthreads();
  double bound = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); i++) bound += s_red[i];
  bound = bound * wmax * (1.0 + 1e-9);
  int e = 0;
  frexp(bound, &e);  // bound < 2^e
  const int k = bound > 0.0 ? max(-1000, min(1000, bits - e)) : 0;
  __syncthreads();  // s_red is reused by the next item
  *inv = scalbn(1.0, -k);
  return scalbn(1.0, k);
}

// Records r0..r1 of tile (tx, ty) of plane w: footprints accumulated in the
// shared tile (s_re, s_im, zeroed by the caller), then the tile written to the
// cube and the rows/tile it touched marked.  LPR lanes per record (>= w_support:
// 8 or 16, or the support itself when it is a compile-time constant that does
// not divide 32 well -- 9 lanes give three records a warp step where 16 gave
// two); 32/LPR records per warp step, lanes past RPW*LPR idle.
template <typename OutT, int LPR, int SUP = 0>
__device__ __forceinline__ void grid_item(const RecF64 *__restrict__ rec, uint32_t r0, uint32_t r1,
                                          const Geometry &g, bool hi, const double *s_tab,
                                          int ntab, double wmax, int tx, int ty, int w,
                                          bool single, int accumulate,
                                          typename Vec2<OutT>::type *__restrict__ cube,
                                          uint32_t *__restrict__ rowmask,
                                          uint32_t *__restrict__ tilemask, FixTile *tile,
                                          double *s_red, uint32_t *s_rows) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const unsigned d = lane % LPR;                 // footprint column / row handled
  const unsigned grp_base = lane - d;            // first lane of this record's group
  constexpr int RPW = 32 / LPR;                  // records per warp step
  constexpr int kWarps = kGridThreads / 32;
  const double gnorm = kStd22 / kPi;             // w-stacking.cu:256
  const int x0 = tx * kTile, y0 = ty * kTile;
  const int sup = SUP > 0 ? SUP : g.support, ghalf = SUP > 0 ? (SUP - 1) / 2 : g.half;
  double inv_scale;
  const double scale = item_scale(rec, r0, r1, wmax, fix_bits<OutT>(), s_red, &inv_scale);

  // Footprints of the chunk's records into the shared tile.
  for (uint32_t rb = r0 + (warp * RPW); rb < r1; rb += kWarps * RPW) {
    const uint32_t r = rb + lane / LPR;
    const bool valid = lane < (unsigned)(RPW * LPR) && r < r1;
    RecF64 q;
    if (valid) q = rec[r];
    else q.sre = q.sim = q.pu = q.pv = 0.0;
    // the cell and the exact fraction (Sterbenz) of the record's position
    const int qgu = valid ? (int)q.pu : -1000000, qgv = valid ? (int)q.pv : -1000000;
    const double qfu = __dsub_rn(q.pu, (double)(int)q.pu), qfv = __dsub_rn(q.pv, (double)(int)q.pv);
    double wu = 0.0, wv = 0.0;
    if (valid && (int)d < sup) {
      const double off = __dadd_rn((double)((int)d - ghalf), 0.5);
      const double ud = __dsub_rn(off, qfu);  // == (j + 0.5) - pos_u exactly
      const double vd = __dsub_rn(off, qfv);
      if (hi) {
        wu = exp(-__dmul_rn(ud, ud) * kStd22);
        wv = exp(-__dmul_rn(vd, vd) * kStd22);
      } else {
        const int jk = (int)__dmul_rn((double)kIncreasePrecision, fabs(__dadd_rn(ud, (double)ghalf)));
        const int kk = (int)__dmul_rn((double)kIncreasePrecision, fabs(__dadd_rn(vd, (double)ghalf)));
        // In range for positions >= 0; rows with u or v in (-dx, 0) would index
        // past the table (the reference reads out of bounds there): clamp.
        wu = s_tab[min(jk, ntab - 1)];
        wv = s_tab[min(kk, ntab - 1)];
      }
    }
    const int j = qgu - ghalf + (int)d;
    const bool col_ok = valid && (int)d < sup && j >= 0 && j < g.nx && j >= x0 && j < x0 + kTile;
    if (rowmask && valid && d == 0) {
      // grid rows of this tile the record's footprint reaches
      const int lo = max(max(qgv - ghalf, 0), y0);
      const int hi_r = min(min(qgv + ghalf, g.ny - 1), y0 + kTile - 1);
      if (lo <= hi_r) {
        const uint32_t span = (uint32_t)(hi_r - lo + 1);
        const uint32_t bits = (span >= 32u ? 0xffffffffu : ((1u << span) - 1u)) << (lo - y0);
        atomicOr(s_rows, bits);
      }
    }
    using W = typename Contrib<OutT>::type;
    const W su = (W)(hi ? gnorm * wu : wu);
    const W wvw = (W)wv;
    // the scale is a power of two: (s * cw) * scale == (s * scale) * cw exactly
    const W sre_s = (W)(q.sre * scale), sim_s = (W)(q.sim * scale);
    // footprint rows e with 0 <= k < ny and y0 <= k < y0 + kTile, k = kb + e
    const int kb = qgv - ghalf;
    const int e_lo = max(max(-kb, y0 - kb), 0);
    const int e_hi = min(min(g.ny - kb, y0 + kTile - kb), sup);
    const int cell0 = (kb - y0) * kPitch + (j - x0);
#pragma unroll
    for (int e = 0; e < (SUP > 0 ? SUP : g.support); e++) {
      const W wve = __shfl_sync(kFull, wvw, grp_base + e);
      if (col_ok && e >= e_lo && e < e_hi) {
        const W cw = su * wve;
        const int cell = cell0 + e * kPitch;
        fix_put<OutT>(&tile->lo_re[cell], &tile->hi_re[cell], sre_s * cw);
        fix_put<OutT>(&tile->lo_im[cell], &tile->hi_im[cell], sim_s * cw);
      }
    }
  }
  __syncthreads();

  // Flush the tile (and the rows it touched).
  if (rowmask && threadIdx.x == 0 && *s_rows) {
    atomicOr(&rowmask[(uint64_t)w * g.nty + ty], *s_rows);
    const int tmw = (g.ntx + 31) / 32;
    atomicOr(&tilemask[((uint64_t)w * g.nty + ty) * tmw + (tx >> 5)], 1u << (tx & 31));
  }
  const uint64_t plane = (uint64_t)g.nx * g.ny;
  for (int c = threadIdx.x; c < kTile * kTile; c += blockDim.x) {
    const int y = c / kTile, x = c % kTile;
    const int gy = y0 + y, gx = x0 + x;
    if (gy >= g.ny || gx >= g.nx) continue;
    const uint64_t idx = (uint64_t)w * plane + (uint64_t)gy * g.nx + gx;
    const int cs = y * kPitch + x;
    const OutT vr = (OutT)(fix_value<OutT>(tile->lo_re, tile->hi_re, cs) * inv_scale);
    const OutT vi = (OutT)(fix_value<OutT>(tile->lo_im, tile->hi_im, cs) * inv_scale);
    if (single) {
      if (accumulate) {
        auto o = cube[idx];
        o.x += vr;
        o.y += vi;
        cube[idx] = o;
      } else {
        typename Vec2<OutT>::type o;
        o.x = vr;
        o.y = vi;
        cube[idx] = o;
      }
    } else if (vr != (OutT)0 || vi != (OutT)0) {
      atomicAdd(&cube[idx].x, vr);
      atomicAdd(&cube[idx].y, vi);
    }
  }
}

// last bin b with item_off[b] <= item
__device__ __forceinline__ uint32_t bin_of_item(const uint32_t *__restrict__ item_off,
                                                uint32_t nbins, uint32_t item) {
  uint32_t lo = 0, hi_b = nbins;
  while (hi_b - lo > 1) {
    const uint32_t mid = (lo + hi_b) >> 1;
    if (item_off[mid] <= item) lo = mid; else hi_b = mid;
  }
  return lo;
}

// Six blocks per SM (the launch's grid): registers bounded to 40 a thread
// (c2 FP64 gridder 1.00 -> 0.955 ms against the compiler's own choice, five).
template <typename OutT, int LPR, int SUP = 0>
__global__ void __launch_bounds__(kGridThreads, 6)
    k_grid_tiles(const RecF64 *__restrict__ rec, const uint32_t *__restrict__ bin_off,
                 const uint32_t *__restrict__ item_off, uint32_t nbins, uint32_t max_chunk,
                 Geometry g, int kernel, const double *__restrict__ table, int accumulate,
                 uint64_t *__restrict__ counters,
                 typename Vec2<OutT>::type *__restrict__ cube, uint32_t *__restrict__ rowmask,
                 uint32_t *__restrict__ tilemask) {
  __shared__ FixTile tile;
  __shared__ double s_tab[kIncreasePrecision * kMaxSupport];
  __shared__ double s_red[kGridThreads / 32];
  __shared__ uint32_t s_item, s_bin, s_first, s_nitems, s_rows;

  const int ntab = kIncreasePrecision * g.support;
  for (int t = threadIdx.x; t < ntab; t += blockDim.x) s_tab[t] = table[t];
  const uint32_t total_items = item_off[nbins];
  const bool hi = (kernel == RICK_KERNEL_GAUSS_HI_PRECISION);
  __syncthreads();
  const double wmax = weight_bound(hi, s_tab, ntab);

  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t item = (uint32_t)atomicAdd((unsigned long long *)&counters[kCntItemNext], 1ull);
      uint32_t bin = 0;
      if (item < total_items) {
        bin = bin_of_item(item_off, nbins, item);
        s_first = item_off[bin];
        s_nitems = item_off[bin + 1] - item_off[bin];
      }
      s_item = item;
      s_bin = bin;
      s_rows = 0;
    }
    fix_zero(&tile);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= total_items) break;
    const uint32_t bin = s_bin;
    const uint32_t chunk = item - s_first;
    const int tx = (int)(bin % (uint32_t)g.ntx);
    const int ty = (int)((bin / (uint32_t)g.ntx) % (uint32_t)g.nty);
    const int w = (int)(bin / ((uint32_t)g.ntx * (uint32_t)g.nty));
    const uint32_t r0 = bin_off[bin] + chunk * max_chunk;
    const uint32_t r1 = min(bin_off[bin + 1], r0 + max_chunk);
    grid_item<OutT, LPR, SUP>(rec, r0, r1, g, hi, s_tab, ntab, wmax, tx, ty, w, s_nitems == 1,
                         accumulate, cube, rowmask, tilemask, &tile, s_red, &s_rows);
    __syncthreads();
  }
}

// The same over every job of a batch: the bins of all jobs are numbered
// consecutively, so the work items are too; a block reloads the kernel table
// when its next item belongs to another job.
template <typename OutT, int LPR, int SUP = 0>
__global__ void __launch_bounds__(kGridThreads)
    k_grid_tiles_batch(const BatchJob *__restrict__ jobs, int njobs,
                       const uint32_t *__restrict__ bin_base, const RecF64 *__restrict__ rec,
                       const uint32_t *__restrict__ bin_off, const uint32_t *__restrict__ item_off,
                       uint32_t nbins, uint32_t max_chunk, uint64_t *__restrict__ counters,
                       uint32_t *__restrict__ rowmask, uint32_t *__restrict__ tilemask) {
  __shared__ FixTile tile;
  __shared__ double s_tab[kIncreasePrecision * kMaxSupport];
  __shared__ double s_red[kGridThreads / 32];
  __shared__ uint32_t s_item, s_bin, s_first, s_nitems, s_rows;
  __shared__ int s_job;

  const uint32_t total_items = item_off[nbins];
  int cur_job = -1;
  double wmax = 0.0;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t item = (uint32_t)atomicAdd((unsigned long long *)&counters[kCntItemNext], 1ull);
      uint32_t bin = 0;
      int job = 0;
      if (item < total_items) {
        bin = bin_of_item(item_off, nbins, item);
        s_first = item_off[bin];
        s_nitems = item_off[bin + 1] - item_off[bin];
        job = batch_job_of(bin_base, njobs, bin);
      }
      s_item = item;
      s_bin = bin;
      s_job = job;
      s_rows = 0;
    }
    fix_zero(&tile);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= total_items) break;
    const int j = s_job;
    const BatchJob &J = jobs[j];
    const Geometry g = J.g;
    const int ntab = kIncreasePrecision * g.support;
    const bool hi = J.kernel == RICK_KERNEL_GAUSS_HI_PRECISION;
    if (j != cur_job) {  // block-uniform
      for (int t = threadIdx.x; t < ntab; t += blockDim.x) s_tab[t] = J.table[t];
      cur_job = j;
      __syncthreads();
      wmax = weight_bound(hi, s_tab, ntab);
    }
    const uint32_t bin = s_bin;
    const uint32_t lbin = bin - J.bin_base;
    const uint32_t chunk = item - s_first;
    const int tx = (int)(lbin % (uint32_t)g.ntx);
    const int ty = (int)((lbin / (uint32_t)g.ntx) % (uint32_t)g.nty);
    const int w = (int)(lbin / ((uint32_t)g.ntx * (uint32_t)g.nty));
    const uint32_t r0 = bin_off[bin] + chunk * max_chunk;
    const uint32_t r1 = min(bin_off[bin + 1], r0 + max_chunk);
    grid_item<OutT, LPR, SUP>(rec, r0, r1, g, hi, s_tab, ntab, wmax, tx, ty, w, s_nitems == 1, 0,
                         (typename Vec2<OutT>::type *)J.cube, rowmask + J.mask_base,
                         tilemask + J.tile_base, &tile, s_red, &s_rows);
    __syncthreads();
  }
}

// Tiles split over several work items receive their parts with atomics, so
// they must start at zero when the cube is not cleared as a whole.
template <typename OutT>
__device__ __forceinline__ void zero_tile(const Geometry &g, uint64_t b,
                                          typename Vec2<OutT>::type *__restrict__ cube) {
  const unsigned lane = threadIdx.x & 31u;
  const uint64_t plane = (uint64_t)g.nx * g.ny;
  const int tx = (int)(b % (uint32_t)g.ntx);
  const int ty = (int)((b / (uint32_t)g.ntx) % (uint32_t)g.nty);
  const int w = (int)(b / ((uint64_t)g.ntx * g.nty));
  const int gx = tx * kTile + (int)lane;
  if (gx >= g.nx) return;
  typename Vec2<OutT>::type z;
  z.x = 0;
  z.y = 0;
  for (int y = 0; y < kTile; y++) {
    const int gy = ty * kTile + y;
    if (gy < g.ny) cube[(uint64_t)w * plane + (uint64_t)gy * g.nx + gx] = z;
  }
}

template <typename OutT>
__global__ void k_zero_split_tiles(const uint32_t *__restrict__ item_off, uint32_t nbins, Geometry g,
                                   typename Vec2<OutT>::type *__restrict__ cube) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  for (uint64_t b = warp; b < nbins; b += nwarps) {
    if (item_off[b + 1] - item_off[b] <= 1) continue;
    zero_tile<OutT>(g, b, cube);
  }
}

template <typename OutT>
__global__ void k_zero_split_tiles_batch(const BatchJob *__restrict__ jobs, int njobs,
                                         const uint32_t *__restrict__ bin_base,
                                         const uint32_t *__restrict__ item_off, uint32_t nbins) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  for (uint64_t b = warp; b < nbins; b += nwarps) {
    if (item_off[b + 1] - item_off[b] <= 1) continue;
    const int j = batch_job_of(bin_base, njobs, (uint32_t)b);
    const Geometry g = jobs[j].g;
    zero_tile<OutT>(g, b - jobs[j].bin_base, (typename Vec2<OutT>::type *)jobs[j].cube);
  }
}

template <typename OutT>
int launch_grid(const Geometry &g, int kernel, Scratch &s, void *cube, int accumulate,
                uint32_t max_chunk, cudaStream_t st, uint32_t *rowmask, uint32_t *tilemask) {
  const int sms = num_sms();
  using V = typename Vec2<OutT>::type;
  const uint32_t nbins = (uint32_t)g.nbins();
  // 16 KB + 16 KB of tile: several blocks per SM
  const int blocks = sms * 6;
  RICK_LAUNCHED();
#define RICK_GRID(LPR, SUP)                                                                    \
  k_grid_tiles<OutT, LPR, SUP><<<blocks, kGridThreads, 0, st>>>(                               \
      s.records, s.bin_count, s.item_off, nbins, max_chunk, g, kernel, s.table, accumulate,    \
      s.counters, (V *)cube, rowmask, tilemask)
  // the common supports unrolled (7: 1.16 -> 1.00 ms FP64 at 4096^2 x 32; 9
  // with 9 lanes a record: 1.73 -> 1.20 ms at 8192^2 x 64)
  if (g.support == 7)
    RICK_GRID(8, 7);
  else if (g.support == 9)
    RICK_GRID(9, 9);
  else if (g.support <= 8)
    RICK_GRID(8, 0);
  else
    RICK_GRID(16, 0);
#undef RICK_GRID
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

}  // namespace

int grid_tiles(const Geometry &g, int kernel, int precision, Scratch &s, void *cube,
               int accumulate, uint32_t max_chunk, cudaStream_t st, uint32_t *rowmask,
               uint32_t *tilemask) {
  if (precision == RICK_PREC_FP64)
    return launch_grid<double>(g, kernel, s, cube, accumulate, max_chunk, st, rowmask, tilemask);
  return launch_grid<float>(g, kernel, s, cube, accumulate, max_chunk, st, rowmask, tilemask);
}

int zero_split_tiles(const Geometry &g, int precision, Scratch &s, void *cube, cudaStream_t st) {
  const uint32_t nbins = (uint32_t)g.nbins();
  const int blocks = (int)std::min<uint64_t>(((uint64_t)nbins * 32 + 255) / 256,
                                             (uint64_t)num_sms() * 16);
  RICK_LAUNCHED();
  if (precision == RICK_PREC_FP64)
    k_zero_split_tiles<double><<<std::max(blocks, 1), 256, 0, st>>>(s.item_off, nbins, g,
                                                                    (double2 *)cube);
  else
    k_zero_split_tiles<float><<<std::max(blocks, 1), 256, 0, st>>>(s.item_off, nbins, g,
                                                                   (float2 *)cube);
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

namespace {

template <typename OutT>
int launch_grid_batch(const BatchLaunch &b, Scratch &s, uint32_t max_chunk, cudaStream_t st) {
  const int sms = num_sms();
  const uint32_t nbins = b.total_bins;
  const int zblocks = (int)std::min<uint64_t>(((uint64_t)nbins * 32 + 255) / 256, (uint64_t)sms * 16);
  RICK_LAUNCHED();
  k_zero_split_tiles_batch<OutT><<<std::max(zblocks, 1), 256, 0, st>>>(b.jobs, b.njobs,
                                                                      b.u.bin_base, s.item_off,
                                                                      nbins);
  RICK_CUDA(cudaGetLastError());
  const int blocks = sms * std::max(1, b.grid_blocks_per_sm);
  RICK_LAUNCHED();
#define RICK_GRID(LPR, SUP)                                                                   \
  k_grid_tiles_batch<OutT, LPR, SUP><<<blocks, kGridThreads, 0, st>>>(                        \
      b.jobs, b.njobs, b.u.bin_base, s.records, s.bin_count, s.item_off, nbins, max_chunk,    \
      s.counters, b.rowmask, b.tilemask)
  // one support over the whole batch: unrolled as for one job
  if (b.min_support == 7 && b.max_support == 7)
    RICK_GRID(8, 7);
  else if (b.min_support == 9 && b.max_support == 9)
    RICK_GRID(9, 9);
  else if (b.max_support <= 8)
    RICK_GRID(8, 0);
  else
    RICK_GRID(16, 0);
#undef RICK_GRID
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

}  // namespace

int grid_tiles_batch(const BatchLaunch &b, int precision, Scratch &s, uint32_t max_chunk,
                     cudaStream_t st) {
  if (precision == RICK_PREC_FP64) return launch_grid_batch<double>(b, s, max_chunk, st);
  return launch_grid_batch<float>(b, s, max_chunk, st);
}

}  // namespace rick
