// Device binning of visibility rows by (w-plane, grid tile).
//
// The reference grids every row with one thread that re-reads the row's
// nchan*npol samples for each of the (2K+1)^2 footprint cells
// (w-stacking.cu:104-206).  The per-cell sum
//     sum_{f,p} weight[p] * vis[f][p] * conv_weight
// factors as conv_weight * S with S = sum_{f,p} weight[p]*vis[f][p], so this
// pass reads each row's samples once, forms S in FP64 (each weight*vis product
// is the FP32 product the reference forms, w-stacking.cu:194-195; a sample whose
// real part is NaN is skipped, :191-192), and emits one compact record per grid
// tile the row's footprint touches.  Records are placed with an integer counting
// sort by (plane, tile), so the gridder reads only the rows of the tile it owns.
//
// Cell assignment is bit-exact with w-stacking.cu:143-149: FP64 IEEE division
// by dx / dw and truncation toward zero, written with explicit round-to-nearest
// intrinsics so that no multiply-add contraction can change a rounding.
#include <algorithm>

#include "rick_internal.h"

namespace rick {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kNoBin = 0xffffffffu;

struct RowPos {
  double pu, pv;  // pos_u, pos_v
  int gu, gv, gw;  // gw: plane within the shard
  bool keep;       // gridded here
  bool other;      // a valid row of a plane outside the shard
};

// gridding.c:149-188 with nsectors = 1 and yaxis = grid_size_y: the rows one
// rank grids are those of sector 0 plus the halo rows its neighbours share.
__device__ __forceinline__ bool in_sector0(double v, const Geometry &g) {
  const int binphi = (int)v;  // (int)(vvh*nsectors), nsectors = 1
  const double updist = __dsub_rn(__dmul_rn((double)((binphi + 1) * g.ny), g.dx), v);
  const double downdist = __dsub_rn(v, __dmul_rn((double)(binphi * g.ny), g.dx));
  bool in0 = (binphi == 0);
  if (binphi + 1 == 0 && updist < g.w_supporth && updist >= 0.0) in0 = true;
  if (binphi - 1 == 0 && downdist < g.w_supporth && binphi > 0 && downdist >= 0.0) in0 = true;
  return in0;
}

// w-stacking.cu:143-149.  Rows whose plane index falls outside the cube, or
// whose footprint bounds would wrap as unsigned in the reference
// (grid_u < -KernelLen), are dropped and counted.  With a w-plane shard, valid
// rows of the other shards' planes are skipped (counted apart).
__device__ __forceinline__ RowPos row_position(double u, double v, double w, const Geometry &g) {
  RowPos p;
  p.pu = __ddiv_rn(u, g.dx);
  p.pv = __ddiv_rn(v, g.dx);
  const double wi = __ddiv_rn(w, g.dw);
  p.gw = (int)wi;
  p.gu = (int)p.pu;
  p.gv = (int)p.pv;
  const int ntot = g.nw_total > 0 ? g.nw_total : g.nw;
  bool keep = p.gw >= 0 && p.gw < ntot && p.gu >= -g.half && p.gv >= -g.half;
  if (g.select_sector0) keep = keep && in_sector0(v, g);
  p.other = keep && (p.gw < g.w_first || p.gw >= g.w_first + g.nw);
  p.keep = keep && !p.other;
  p.gw -= g.w_first;
  return p;
}

// Bins of the (up to 2x2) tiles a footprint touches, kNoBin for unused slots.
__device__ __forceinline__ void footprint_bins(const RowPos &p, const Geometry &g,
                                               uint32_t bins[4]) {
  bins[0] = bins[1] = bins[2] = bins[3] = kNoBin;
  if (!p.keep) return;
  const int jmin = max(p.gu - g.half, 0), jmax = min(p.gu + g.half, g.nx - 1);
  const int kmin = max(p.gv - g.half, 0), kmax = min(p.gv + g.half, g.ny - 1);
  if (jmin > jmax || kmin > kmax) return;  // footprint entirely off the grid
  const int tx0 = jmin / kTile, tx1 = jmax / kTile;
  const int ty0 = kmin / kTile, ty1 = kmax / kTile;
  int n = 0;
  for (int ty = ty0; ty <= ty1; ty++)
    for (int tx = tx0; tx <= tx1; tx++)
      bins[n++] = (uint32_t)(((uint64_t)p.gw * g.nty + ty) * g.ntx + tx);
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void offset_bins(uint32_t bins[4], uint32_t bin_base) {
#pragma unroll
  for (int s = 0; s < 4; s++) bins[s] = bins[s] == kNoBin ? kNoBin : bins[s] + bin_base;
}

// Per-block cache of record counts: the warps of a block add into a
// direct-mapped shared table and the block adds the table into the global
// histogram once at its end, so the bins the uv centre shares across time
// steps take shared- instead of global-memory atomics.  A slot taken by
// another bin sends the count straight to the global histogram (counts stay
// exact either way).
constexpr int kCountCache = 2048;
struct CountCache {
  uint32_t key[kCountCache];
  uint32_t cnt[kCountCache];
};
__device__ __forceinline__ void cache_init(CountCache *c) {
  for (int i = threadIdx.x; i < kCountCache; i += blockDim.x) {
    c->key[i] = kNoBin;
    c->cnt[i] = 0;
  }
  __syncthreads();
}
__device__ __forceinline__ void cache_add(CountCache *c, uint32_t bin, uint32_t n,
                                          uint32_t *__restrict__ bin_count) {
  const uint32_t h = (bin * 2654435761u) >> (32 - 11);  // multiplicative hash, 11 bits
  const uint32_t k = atomicCAS(&c->key[h], kNoBin, bin);
  if (k == kNoBin || k == bin) atomicAdd(&c->cnt[h], n);
  else atomicAdd(&bin_count[bin], n);
}
__device__ __forceinline__ void cache_flush(CountCache *c, uint32_t *__restrict__ bin_count) {
  __syncthreads();
  for (int i = threadIdx.x; i < kCountCache; i += blockDim.x)
    if (c->cnt[i]) atomicAdd(&bin_count[c->key[i]], c->cnt[i]);
}

// Pass 1 over rows base..base+31 (one per lane): histogram of records per bin.
// Every lane adds its row's bins into the block's cache (the uv centre is
// dense: hot bins are counted in shared memory, not by global atomics; a
// warp-level match before the cache measured slower).  Returns 1 on a lane
// whose row was dropped; `other` counts rows of other shards.
__device__ __forceinline__ uint32_t count_rows(const double *__restrict__ uu,
                                               const double *__restrict__ vv,
                                               const double *__restrict__ ww, uint64_t nrows,
                                               const Geometry &g, uint64_t base,
                                               uint32_t bin_base, uint32_t *__restrict__ bin_count,
                                               uint32_t &other, CountCache *cache) {
  const unsigned lane = lane_id();
  const uint64_t i = base + lane;
  RowPos p;
  p.keep = false;
  uint32_t dropped = 0;
  if (i < nrows) {
    p = row_position(uu[i], vv[i], ww[i], g);
    dropped = (p.keep || p.other) ? 0u : 1u;
    other += p.other ? 1u : 0u;
  }
  uint32_t bins[4];
  footprint_bins(p, g, bins);
  offset_bins(bins, bin_base);
#pragma unroll
  for (int s = 0; s < 4; s++)
    if (bins[s] != kNoBin) cache_add(cache, bins[s], 1u, bin_count);
  return dropped;
}

__device__ __forceinline__ void add_dropped(uint32_t dropped, uint32_t other, uint64_t *counters) {
  for (int o = 16; o; o >>= 1) {
    dropped += __shfl_xor_sync(kFull, dropped, o);
    other += __shfl_xor_sync(kFull, other, o);
  }
  if (lane_id() == 0 && dropped) atomicAdd((unsigned long long *)&counters[kCntDropped], dropped);
  if (lane_id() == 0 && other) atomicAdd((unsigned long long *)&counters[kCntOtherShard], other);
}

__global__ void k_bin_count(const double *__restrict__ uu, const double *__restrict__ vv,
                            const double *__restrict__ ww, uint64_t nrows, Geometry g,
                            uint32_t *__restrict__ bin_count, uint64_t *__restrict__ counters) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  __shared__ CountCache cache;
  cache_init(&cache);
  uint32_t dropped = 0, other = 0;
  for (uint64_t base = warp * 32; base < nrows; base += nwarps * 32)
    dropped += count_rows(uu, vv, ww, nrows, g, base, 0, bin_count, other, &cache);
  cache_flush(&cache, bin_count);
  add_dropped(dropped, other, counters);
}

// The same over every job of a batch: one warp per 32-row unit of one job.
__global__ void k_bin_count_batch(const BatchJob *__restrict__ jobs, int njobs,
                                  const uint64_t *__restrict__ row_units, uint64_t total_units,
                                  uint32_t *__restrict__ bin_count,
                                  uint64_t *__restrict__ counters) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  __shared__ CountCache cache;
  cache_init(&cache);
  uint32_t dropped = 0, other = 0;
  for (uint64_t u = warp; u < total_units; u += nwarps) {
    const int j = batch_job_of(row_units, njobs, u);
    const BatchJob &J = jobs[j];
    const Geometry g = J.g;
    dropped += count_rows(J.uu, J.vv, J.ww, J.nrows, g, (u - row_units[j]) * 32, J.bin_base,
                          bin_count, other, &cache);
  }
  cache_flush(&cache, bin_count);
  add_dropped(dropped, other, counters);
}

// Work items of the gridder: a bin with c records is split into ceil(c/max_chunk)
// chunks (0 for an empty bin) so that no item is much larger than another.
__global__ void k_item_count(const uint32_t *__restrict__ bin_off, uint64_t nbins,
                             uint32_t max_chunk, uint32_t *__restrict__ item_count) {
  for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b <= nbins;
       b += gridDim.x * (uint64_t)blockDim.x) {
    uint32_t c = b < nbins ? bin_off[b + 1] - bin_off[b] : 0;
    item_count[b] = (c + max_chunk - 1) / max_chunk;
  }
}

// Pass 2 over rows base..base+31: row sums and record scatter.  Each group of
// G lanes reduces one row's samples with 16-byte loads (V4) or scalar loads;
// after G rounds every lane holds the sum of "its" row, and the records are
// scattered one row per lane with warp-combined cursor increments.
template <int G, bool V4, bool SHARD>
__device__ __forceinline__ void scatter_rows(
    const double *__restrict__ uu, const double *__restrict__ vv, const double *__restrict__ ww,
    const float *__restrict__ weight, const float *__restrict__ vis_re,
    const float *__restrict__ vis_im, uint64_t nrows, uint32_t nchan, uint32_t npol,
    const Geometry &g, uint64_t base, uint32_t bin_base, const uint32_t *__restrict__ bin_off,
    uint32_t *__restrict__ bin_cursor, RecF64 *__restrict__ rec, uint32_t &gridded,
    uint32_t &nrec) {
  constexpr int R = 32 / G;  // rows per round
  const unsigned lane = lane_id();
  const unsigned sub = lane % G, grp = lane / G;
  const uint64_t nv = (uint64_t)nchan * npol;
  // A w-plane shard (SHARD) holds a fraction of the rows: its rows of other
  // planes (and rows that reach no tile) are found before any sample is read,
  // so they never stream their samples.  A whole-cube plan keeps nearly every
  // row and compiles without the check.
  bool need = true;
  if (SHARD) {
    const uint64_t i_own = base + lane;
    RowPos q;
    q.keep = false;
    if (i_own < nrows) q = row_position(uu[i_own], vv[i_own], ww[i_own], g);
    uint32_t qb[4];
    footprint_bins(q, g, qb);
    need = qb[0] != kNoBin;
  }
  double my_re = 0.0, my_im = 0.0;
#pragma unroll 1
  for (int round = 0; round < G; round++) {
    const uint64_t i = base + (uint64_t)round * R + grp;
    double sre = 0.0, sim = 0.0;
    const bool need_i = __shfl_sync(kFull, need, round * R + grp);
    if (i < nrows && need_i) {
      const float *wrow = weight + i * npol;
      if (V4) {
        // npol divides 4, so component c of every float4 is polarisation c % npol
        float wc[4];
#pragma unroll
        for (int c = 0; c < 4; c++) wc[c] = __ldg(wrow + (c % npol));
        const float4 *r4 = reinterpret_cast<const float4 *>(vis_re + i * nv);
        const float4 *i4 = reinterpret_cast<const float4 *>(vis_im + i * nv);
        const uint64_t nq = nv / 4;
#pragma unroll 2
        for (uint64_t q = sub; q < nq; q += G) {
          const float4 a = __ldcs(r4 + q);
          const float4 b = __ldcs(i4 + q);
          const float ar[4] = {a.x, a.y, a.z, a.w}, bi[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
          for (int c = 0; c < 4; c++) {
            if (!isnan(ar[c])) {
              sre += (double)__fmul_rn(wc[c], ar[c]);
              sim += (double)__fmul_rn(wc[c], bi[c]);
            }
          }
        }
      } else {
        for (uint64_t q = sub; q < nv; q += G) {
          const float a = __ldcs(vis_re + i * nv + q);
          if (!isnan(a)) {
            const float wq = __ldg(wrow + (q % npol));
            sre += (double)__fmul_rn(wq, a);
            sim += (double)__fmul_rn(wq, __ldcs(vis_im + i * nv + q));
          }
        }
      }
    }
#pragma unroll
    for (int o = G / 2; o; o >>= 1) {
      sre += __shfl_xor_sync(kFull, sre, o);
      sim += __shfl_xor_sync(kFull, sim, o);
    }
    // lane (round*R + grp') receives the sum of group grp' (its sub-lane 0)
    const int src = (int)(lane - round * R) * G;
    const double t_re = __shfl_sync(kFull, sre, src & 31);
    const double t_im = __shfl_sync(kFull, sim, src & 31);
    if (lane / R == (unsigned)round) {
      my_re = t_re;
      my_im = t_im;
    }
  }

  const uint64_t i = base + lane;
  RowPos p;
  p.keep = false;
  if (i < nrows) p = row_position(uu[i], vv[i], ww[i], g);
  uint32_t bins[4];
  footprint_bins(p, g, bins);
  offset_bins(bins, bin_base);
  gridded += p.keep ? 1u : 0u;
  RecF64 r;
  r.sre = my_re;
  r.sim = my_im;
  r.pu = p.pu;
  r.pv = p.pv;
#pragma unroll
  for (int s = 0; s < 4; s++) {
    const unsigned peers = __match_any_sync(kFull, bins[s]);
    const unsigned leader = __ffs(peers) - 1;
    uint32_t slot = 0;
    if (bins[s] != kNoBin && lane == leader) slot = atomicAdd(&bin_cursor[bins[s]], __popc(peers));
    slot = __shfl_sync(kFull, slot, leader);
    if (bins[s] != kNoBin) {
      slot += __popc(peers & ((1u << lane) - 1u));
      rec[(uint64_t)bin_off[bins[s]] + slot] = r;
      nrec++;
    }
  }
}

__device__ __forceinline__ void add_scatter_counts(uint32_t gridded, uint32_t nrec,
                                                   uint64_t *counters) {
  for (int o = 16; o; o >>= 1) {
    gridded += __shfl_xor_sync(kFull, gridded, o);
    nrec += __shfl_xor_sync(kFull, nrec, o);
  }
  if (lane_id() == 0) {
    if (gridded) atomicAdd((unsigned long long *)&counters[kCntGridded], gridded);
    if (nrec) atomicAdd((unsigned long long *)&counters[kCntRecords], nrec);
  }
}

template <int G, bool V4, bool SHARD>
__global__ void __launch_bounds__(256)
    k_bin_scatter(const double *__restrict__ uu, const double *__restrict__ vv,
                  const double *__restrict__ ww, const float *__restrict__ weight,
                  const float *__restrict__ vis_re, const float *__restrict__ vis_im,
                  uint64_t nrows, uint32_t nchan, uint32_t npol, Geometry g,
                  const uint32_t *__restrict__ bin_off, uint32_t *__restrict__ bin_cursor,
                  RecF64 *__restrict__ rec, uint64_t *__restrict__ counters) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  uint32_t gridded = 0, nrec = 0;
  for (uint64_t base = warp * 32; base < nrows; base += nwarps * 32)
    scatter_rows<G, V4, SHARD>(uu, vv, ww, weight, vis_re, vis_im, nrows, nchan, npol, g, base,
                               0, bin_off, bin_cursor, rec, gridded, nrec);
  add_scatter_counts(gridded, nrec, counters);
}

// The same over the jobs of one sample-pass schedule of a batch (lanes per row
// G, load width V4): the k-th listed job's rows are units sc_units[k] ..
// sc_units[k+1]-1 (a unit is 32 rows of one job).  Bounded to three blocks
// per SM: the job lookup and the per-job geometry add registers to the
// single-job kernel's set.
template <int G, bool V4>
__global__ void __launch_bounds__(256, 3)
    k_bin_scatter_batch(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ sc_jobs,
                        const uint64_t *__restrict__ sc_units, int lo, int hi,
                        const uint32_t *__restrict__ bin_off, uint32_t *__restrict__ bin_cursor,
                        RecF64 *__restrict__ rec, uint64_t *__restrict__ counters) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = (gridDim.x * (uint64_t)blockDim.x) >> 5;
  uint32_t gridded = 0, nrec = 0;
  const uint64_t u1 = sc_units[hi];
  for (uint64_t u = sc_units[lo] + warp; u < u1; u += nwarps) {
    const int k = lo + batch_job_of(sc_units + lo, hi - lo, u);
    const BatchJob &J = jobs[sc_jobs[k]];
    const Geometry g = J.g;
    scatter_rows<G, V4, false>(J.uu, J.vv, J.ww, J.weight, J.vis_re, J.vis_im, J.nrows, J.nchan, J.npol,
                        g, (u - sc_units[k]) * 32, J.bin_base, bin_off, bin_cursor, rec, gridded,
                        nrec);
  }
  add_scatter_counts(gridded, nrec, counters);
}

template <int G, bool V4>
void launch_scatter(int blocks, cudaStream_t st, const double *uu, const double *vv,
                    const double *ww, const float *weight, const float *vis_re,
                    const float *vis_im, uint64_t nrows, uint32_t nchan, uint32_t npol,
                    const Geometry &g, Scratch &s) {
  RICK_LAUNCHED();
  if (g.nw_total > 0 && g.nw_total != g.nw)
    k_bin_scatter<G, V4, true><<<blocks, 256, 0, st>>>(uu, vv, ww, weight, vis_re, vis_im, nrows,
                                                       nchan, npol, g, s.bin_count, s.bin_cursor,
                                                       s.records, s.counters);
  else
    k_bin_scatter<G, V4, false><<<blocks, 256, 0, st>>>(uu, vv, ww, weight, vis_re, vis_im, nrows,
                                                        nchan, npol, g, s.bin_count, s.bin_cursor,
                                                        s.records, s.counters);
}

}  // namespace

int lanes_per_row(uint64_t per_row);

// Pass 1 and the offsets: histogram of records per bin over all rows, bin
// offsets and work-item offsets (records are not written yet).
int bin_count_rows(const Geometry &g, uint64_t nrows, const double *uu, const double *vv,
                   const double *ww, Scratch &s, uint32_t max_chunk, cudaStream_t st) {
  const uint64_t nbins = g.nbins();
  RICK_CUDA(cudaMemsetAsync(s.bin_count, 0, (nbins + 1) * sizeof(uint32_t), st));
  RICK_CUDA(cudaMemsetAsync(s.bin_cursor, 0, nbins * sizeof(uint32_t), st));
  if (nrows == 0) {
    RICK_CUDA(cudaMemsetAsync(s.item_off, 0, (nbins + 1) * sizeof(uint32_t), st));
    return RICK_OK;
  }
  const int sms = num_sms();
  const uint64_t warps_needed = (nrows + 31) / 32;
  const int blocks_cnt = (int)std::min<uint64_t>((warps_needed + 7) / 8, (uint64_t)sms * 16);
  RICK_LAUNCHED();
  k_bin_count<<<blocks_cnt, 256, 0, st>>>(uu, vv, ww, nrows, g, s.bin_count, s.counters);
  RICK_CUDA(cudaGetLastError());
  // counts -> exclusive offsets, in place (bin_count[nbins] becomes the total)
  RICK_TRY(exclusive_scan_u32(s.bin_count, s.bin_count, nbins + 1, s.scan_tmp, st));
  // work items
  const int blocks_items = (int)std::min<uint64_t>((nbins + 256) / 256, (uint64_t)sms * 32);
  RICK_LAUNCHED();
  k_item_count<<<blocks_items, 256, 0, st>>>(s.bin_count, nbins, max_chunk, s.item_off);
  RICK_CUDA(cudaGetLastError());
  RICK_TRY(exclusive_scan_u32(s.item_off, s.item_off, nbins + 1, s.scan_tmp, st));
  return RICK_OK;
}

// Pass 2 over rows [0, nrows) of the arrays given (a contiguous slice of the
// rows pass 1 counted: records are placed through the shared bin cursors, so
// slices may follow one another in any order).
int bin_scatter_rows(const Geometry &g, uint64_t nrows, const double *uu, const double *vv,
                     const double *ww, const float *weight, const float *vis_re,
                     const float *vis_im, uint32_t nchan, uint32_t npol, Scratch &s,
                     cudaStream_t st) {
  if (nrows == 0) return RICK_OK;
  const int sms = num_sms();
  const uint64_t warps_needed = (nrows + 31) / 32;
  const uint64_t nv = (uint64_t)nchan * npol;
  const bool aligned = ((uintptr_t)vis_re % 16 == 0) && ((uintptr_t)vis_im % 16 == 0);
  const bool v4 = aligned && nv % 4 == 0 && (npol == 1 || npol == 2 || npol == 4);
  const uint64_t per_row = v4 ? nv / 4 : nv;
  // lanes per row: enough to cover a row's 16-byte chunks in one or two sweeps
  const int G = lanes_per_row(per_row);
  const int blocks = (int)std::min<uint64_t>((warps_needed + 7) / 8, (uint64_t)sms * 8);
#define RICK_SCATTER(GG)                                                                    \
  case GG:                                                                                  \
    if (v4)                                                                                 \
      launch_scatter<GG, true>(blocks, st, uu, vv, ww, weight, vis_re, vis_im, nrows, nchan, \
                               npol, g, s);                                                 \
    else                                                                                    \
      launch_scatter<GG, false>(blocks, st, uu, vv, ww, weight, vis_re, vis_im, nrows,      \
                                nchan, npol, g, s);                                         \
    break;
  switch (G) {
    RICK_SCATTER(1)
    RICK_SCATTER(2)
    RICK_SCATTER(4)
    RICK_SCATTER(8)
    RICK_SCATTER(16)
    RICK_SCATTER(32)
  }
#undef RICK_SCATTER
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

int bin_rows(const Geometry &g, int kernel, int precision, uint64_t nrows, const double *uu,
             const double *vv, const double *ww, const float *weight, const float *vis_re,
             const float *vis_im, uint32_t nchan, uint32_t npol, Scratch &s,
             uint32_t max_chunk, cudaStream_t st, cudaEvent_t mid) {
  (void)kernel;
  (void)precision;
  RICK_TRY(bin_count_rows(g, nrows, uu, vv, ww, s, max_chunk, st));
  if (mid) RICK_CUDA(cudaEventRecord(mid, st));
  return bin_scatter_rows(g, nrows, uu, vv, ww, weight, vis_re, vis_im, nchan, npol, s, st);
}

// Lanes that share one row's samples: enough to cover the row's loads in one
// or two sweeps; rows of at most 8 loads are read by one lane each (a row
// spread over lanes would leave each lane one load and the warp waiting).
int lanes_per_row(uint64_t per_row) {
  if (per_row <= 8) return 1;
  int G = 1;
  while (G < 32 && (uint64_t)G * 2 <= per_row) G *= 2;
  return G;
}

int bin_rows_batch(const BatchLaunch &b, Scratch &s, uint32_t max_chunk, cudaStream_t st) {
  const uint64_t nbins = b.total_bins;
  RICK_CUDA(cudaMemsetAsync(s.bin_count, 0, (nbins + 1) * sizeof(uint32_t), st));
  RICK_CUDA(cudaMemsetAsync(s.bin_cursor, 0, std::max<uint64_t>(nbins, 1) * sizeof(uint32_t), st));
  const int sms = num_sms();
  const uint64_t units = b.total_row_units;
  const int blocks_cnt = (int)std::max<uint64_t>(1, std::min<uint64_t>((units + 7) / 8, (uint64_t)sms * 16));
  RICK_LAUNCHED();
  k_bin_count_batch<<<blocks_cnt, 256, 0, st>>>(b.jobs, b.njobs, b.u.row_units, units,
                                                s.bin_count, s.counters);
  RICK_CUDA(cudaGetLastError());
  RICK_TRY(exclusive_scan_u32(s.bin_count, s.bin_count, nbins + 1, s.scan_tmp, st));
  const int blocks_items = (int)std::min<uint64_t>((nbins + 256) / 256, (uint64_t)sms * 32);
  RICK_LAUNCHED();
  k_item_count<<<blocks_items, 256, 0, st>>>(s.bin_count, nbins, max_chunk, s.item_off);
  RICK_CUDA(cudaGetLastError());
  RICK_TRY(exclusive_scan_u32(s.item_off, s.item_off, nbins + 1, s.scan_tmp, st));
  for (int c = 0; c < b.n_sc; c++) {
    const ScatterClass &k = b.sc[c];
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((k.units + 7) / 8,
                                                                      (uint64_t)sms * 8));
#define RICK_SC(GG)                                                                            \
  case GG:                                                                                     \
    RICK_LAUNCHED();                                                                           \
    if (k.v4)                                                                                  \
      k_bin_scatter_batch<GG, true><<<blocks, 256, 0, st>>>(b.jobs, b.sc_jobs, b.sc_units, k.lo, \
                                                            k.hi, s.bin_count, s.bin_cursor,    \
                                                            s.records, s.counters);             \
    else                                                                                       \
      k_bin_scatter_batch<GG, false><<<blocks, 256, 0, st>>>(b.jobs, b.sc_jobs, b.sc_units,     \
                                                             k.lo, k.hi, s.bin_count,           \
                                                             s.bin_cursor, s.records,           \
                                                             s.counters);                       \
    break;
    switch (k.lanes) {
      RICK_SC(1)
      RICK_SC(2)
      RICK_SC(4)
      RICK_SC(8)
      RICK_SC(16)
      RICK_SC(32)
    }
#undef RICK_SC
    RICK_CUDA(cudaGetLastError());
  }
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

}  // namespace rick
