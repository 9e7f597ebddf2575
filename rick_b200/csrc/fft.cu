// Sparse-aware 2-D inverse FFT of the w-stacked cube, fused with the w-term
// correction and the sum over planes.
//
// fourier_transform.c:34-76 transforms every w-plane with FFTW_BACKWARD and
// scales by 1/(Nx*Ny); phase_correction.cu:191-250 then multiplies each plane by
// its w-phase screen and adds the planes into the image.  A w-plane of a real
// observation holds data on a minority of its rows (the uv tracks of one w
// slice), so here:
//   * the row pass transforms only the rows any footprint touched (a per-tile
//     row mask written by the gridder), reading only the tiles that received
//     records and treating the others as zeros -- so the cube is never cleared;
//   * the column pass loads, for each column, only the touched rows of every
//     plane, transforms the column, and multiplies the result by the plane's
//     phase screen straight into per-pixel FP64 accumulators: the transformed
//     cube is never written back, and the image is written once.
// Each 1-D transform runs in shared memory as an in-place mixed-radix Stockham
// FFT (radix-8 passes and one radix-2 or -4 pass), eight values per thread,
// with FP64 twiddles computed on the host in long double.  Power-of-two sizes
// from 64 to 8192; other sizes use the cuFFT plan.
#include <math.h>

#include <algorithm>

#include "rick_internal.h"

namespace rick {

namespace {

template <typename T> struct V2;
template <> struct V2<double> { using t = double2; };
template <> struct V2<float> { using t = float2; };

template <typename T> struct Cx {
  T re, im;
};
template <typename T>
__device__ __forceinline__ Cx<T> cadd(Cx<T> a, Cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
__device__ __forceinline__ Cx<T> csub(Cx<T> a, Cx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, T br, T bi) {
  return {a.re * br - a.im * bi, a.re * bi + a.im * br};
}

// exp(+2 pi i j / 16) applied to a, j = 0..7 known at compile time after unrolling.
template <typename T>
__device__ __forceinline__ Cx<T> w16(Cx<T> a, int j) {
  constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173;
  constexpr double h = 0.70710678118654752440;
  switch (j) {
    case 0: return a;
    case 1: return cmul<T>(a, (T)c1, (T)s1);
    case 2: return {(a.re - a.im) * (T)h, (a.re + a.im) * (T)h};
    case 3: return cmul<T>(a, (T)s1, (T)c1);
    case 4: return {-a.im, a.re};
    case 5: return cmul<T>(a, (T)-s1, (T)c1);
    case 6: return {(-a.re - a.im) * (T)h, (a.re - a.im) * (T)h};
    default: return cmul<T>(a, (T)-c1, (T)s1);
  }
}

// In-register inverse DFT (exp(+i)) of R points, natural order in and out.
template <typename T, int R> struct Dft {
  __device__ __forceinline__ static void run(Cx<T> *v) {
    Cx<T> e[R / 2], o[R / 2];
#pragma unroll
    for (int i = 0; i < R / 2; i++) {
      e[i] = v[2 * i];
      o[i] = v[2 * i + 1];
    }
    Dft<T, R / 2>::run(e);
    Dft<T, R / 2>::run(o);
#pragma unroll
    for (int k = 0; k < R / 2; k++) {
      const Cx<T> t = w16<T>(o[k], k * (16 / R));
      v[k] = cadd(e[k], t);
      v[k + R / 2] = csub(e[k], t);
    }
  }
};
template <typename T> struct Dft<T, 1> {
  __device__ __forceinline__ static void run(Cx<T> *) {}
};

// Shared-memory index with one pad element every 16: the stride-R stores of
// the first pass then spread over the banks.
__device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

template <typename T>
__device__ __forceinline__ Cx<T> lds(const typename V2<T>::t *s, int i) {
  const typename V2<T>::t v = s[pad(i)];
  return {v.x, v.y};
}
template <typename T>
__device__ __forceinline__ void sts(typename V2<T>::t *s, int i, Cx<T> c) {
  typename V2<T>::t v;
  v.x = c.re;
  v.y = c.im;
  s[pad(i)] = v;
}

// Asynchronous global->shared copy of one complex value; zero-filled when
// `valid` is false (no byte of the source is read then).
template <typename T>
__device__ __forceinline__ void cp_async_zfill(typename V2<T>::t *dst, const typename V2<T>::t *src,
                                               bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  if (sizeof(typename V2<T>::t) == 16) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n)
                 : "memory");
  } else {
    const int n = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(n)
                 : "memory");
  }
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}

constexpr int kVpt = 8;  // values per thread

// Column-blocked layout of the row-transformed planes: 128-byte blocks of
// columns, each block holding every row: element (w, k, n) sits at
//   ((w * (nx / CB) + n / CB) * ny + k) * CB + n % CB,   CB = 128 / sizeof(complex).
// Row-pass writes are whole 128-byte lines; the column pass of the CB columns
// of a block streams one contiguous region per plane.
template <typename T> __host__ __device__ constexpr int col_block() { return 128 / (int)sizeof(typename V2<T>::t); }
template <typename T>
__device__ __forceinline__ uint64_t blocked_index(uint32_t w, uint32_t k, uint32_t n, int nx, int ny) {
  constexpr int CB = col_block<T>();
  return (((uint64_t)w * (nx / CB) + n / CB) * ny + k) * CB + (n % CB);
}

// One Stockham pass of radix R over N points held in shared memory by the N/8
// threads of a row group (every value is read into registers before any is
// written back, so the pass works in place).
template <typename T, int N, int R>
__device__ __forceinline__ void stockham_pass(typename V2<T>::t *s, int t, int Ns,
                                              const typename V2<T>::t *__restrict__ tw) {
  constexpr int G = N / kVpt, B = kVpt / R;
  Cx<T> v[B][R];
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * G;
#pragma unroll
    for (int r = 0; r < R; r++) v[b][r] = lds<T>(s, j + r * (N / R));
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * G;
    const int jm = j & (Ns - 1);
    if (Ns > 1) {
      // per-pass table: entry (Ns-1) + (r-1)*Ns + jm = exp(+2 pi i jm r / (Ns R)),
      // so consecutive lanes read consecutive entries.  Radix 8 loads the powers
      // 1, 2, 4 and forms 3, 5, 6, 7 as products (a few ulp, far inside 1e-12).
      const typename V2<T>::t *twp = tw + (Ns - 1) + jm;
      if (R == 8) {
        const typename V2<T>::t a = __ldg(twp), b2 = __ldg(twp + Ns), b4 = __ldg(twp + 3 * Ns);
        const Cx<T> w1 = {a.x, a.y}, w2 = {b2.x, b2.y}, w4 = {b4.x, b4.y};
        const Cx<T> w3 = cmul<T>(w1, w2.re, w2.im);
        const Cx<T> w5 = cmul<T>(w1, w4.re, w4.im);
        const Cx<T> w6 = cmul<T>(w2, w4.re, w4.im);
        const Cx<T> w7 = cmul<T>(w3, w4.re, w4.im);
        const Cx<T> w[8] = {{(T)1, (T)0}, w1, w2, w3, w4, w5, w6, w7};
#pragma unroll
        for (int r = 1; r < R; r++) v[b][r] = cmul<T>(v[b][r], w[r].re, w[r].im);
      } else {
#pragma unroll
        for (int r = 1; r < R; r++) {
          const typename V2<T>::t w = __ldg(twp + (r - 1) * Ns);
          v[b][r] = cmul<T>(v[b][r], w.x, w.y);
        }
      }
    }
    Dft<T, R>::run(v[b]);
    const int idx = (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; r++) sts<T>(s, idx + r * Ns, v[b][r]);
  }
  __syncthreads();
}

// Whole inverse FFT of N = 2^LOGN points (unnormalised), in place.
template <typename T, int LOGN>
__device__ __forceinline__ void fft_inplace(typename V2<T>::t *s, int t,
                                            const typename V2<T>::t *__restrict__ tw) {
  constexpr int N = 1 << LOGN;
  constexpr int P8 = LOGN / 3, REM = LOGN % 3;
  int Ns = 1;
#pragma unroll
  for (int p = 0; p < P8; p++) {
    stockham_pass<T, N, 8>(s, t, Ns, tw);
    Ns *= 8;
  }
  if (REM == 1) stockham_pass<T, N, 2>(s, t, Ns, tw);
  if (REM == 2) stockham_pass<T, N, 4>(s, t, Ns, tw);
}

template <int LOGN> constexpr int group_threads() { return (1 << LOGN) / kVpt; }
template <int LOGN> constexpr int block_threads() {
  return group_threads<LOGN>() > 256 ? group_threads<LOGN>() : 256;
}

// Row pass: inverse FFT along x of the listed (plane, row) pairs, from the
// gridded cube (tiles without records read as zeros) into the column-blocked
// buffer.
template <typename T, int LOGN>
__global__ void __launch_bounds__(block_threads<LOGN>())
    k_fft_rows(const typename V2<T>::t *__restrict__ cube, typename V2<T>::t *__restrict__ out,
               int nx, int ny, int nty, int ntx, const uint32_t *__restrict__ rowlist,
               const uint32_t *__restrict__ counts, const uint32_t *__restrict__ bin_off,
               const typename V2<T>::t *__restrict__ tw) {
  constexpr int N = 1 << LOGN, G = N / kVpt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  typename V2<T>::t *s = reinterpret_cast<typename V2<T>::t *>(smem_raw);
  const int rpc = blockDim.x / G;
  const int grp = threadIdx.x / G, t = threadIdx.x % G;
  typename V2<T>::t *srow = s + grp * (N + N / 16);
  const uint32_t nrows = counts[0];
  for (uint32_t base = blockIdx.x * rpc; base < nrows; base += gridDim.x * rpc) {
    const uint32_t li = base + grp;
    const bool active = li < nrows;
    uint32_t w = 0, k = 0;
    if (active) {
      const uint32_t rid = rowlist[li];
      w = rid / (uint32_t)ny;
      k = rid % (uint32_t)ny;
    }
    const uint64_t rowbase = ((uint64_t)w * ny + k) * nx;
    const uint32_t binbase = (w * (uint32_t)nty + (k >> 5)) * (uint32_t)ntx;
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      const int x = t + q * G;
      typename V2<T>::t v;
      v.x = 0;
      v.y = 0;
      if (active) {
        const uint32_t b = binbase + (x >> 5);
        if (bin_off[b + 1] != bin_off[b]) v = cube[rowbase + x];  // tile holds records
      }
      srow[pad(x)] = v;
    }
    __syncthreads();
    fft_inplace<T, LOGN>(srow, t, tw);
    if (active) {
#pragma unroll
      for (int q = 0; q < kVpt; q++) {
        const int x = t + q * G;
        out[blocked_index<T>(w, k, x, nx, ny)] = srow[pad(x)];
      }
    }
    __syncthreads();
  }
}

// Column pass fused with the w-correction and the plane sum: each row group
// owns one image column and walks the planes in increasing w.  With DB the
// next plane's column is copied into a second shared buffer (cp.async,
// untouched rows zero-filled) while the current one is transformed.
// sqrt(1 - l^2 - m^2) of the column's pixels is formed once per column
// (shared memory).  The plain form evaluates every plane's phase with sincos
// of the reference's argument; with RECUR (mixed form) the phase advances from
// plane to plane by a per-pixel step exp(i 2 pi dw (root - 1)) kept in shared
// memory, re-anchored with an exact sincos every kAnchor planes.
constexpr int kAnchor = 8;

template <typename T, int LOGN, bool DB, bool RECUR>
__global__ void __launch_bounds__(block_threads<LOGN>())
    k_fft_cols_image(const typename V2<T>::t *__restrict__ cube, int nx, int ny, int nw, int nty,
                     const uint32_t *__restrict__ rowmask, const uint32_t *__restrict__ counts,
                     const typename V2<T>::t *__restrict__ tw, const double *__restrict__ ltab,
                     const double *__restrict__ mtab, double wmin, double dw, double dwnorm,
                     double norm, int phase_on, double *__restrict__ img_re,
                     double *__restrict__ img_im) {
  constexpr int N = 1 << LOGN, G = N / kVpt, LEN = N + N / 16;
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *s = reinterpret_cast<V *>(smem_raw);
  const int rpc = blockDim.x / G;
  const int grp = threadIdx.x / G, t = threadIdx.x % G;
  V *buf[2] = {s + grp * LEN, s + (DB ? rpc + grp : grp) * LEN};
  double *sroot = reinterpret_cast<double *>(s + (DB ? 2 : 1) * rpc * LEN) + grp * N;
  double2 *sstep = reinterpret_cast<double2 *>(reinterpret_cast<double *>(s + (DB ? 2 : 1) * rpc * LEN) + rpc * N) + grp * N;
  const bool phase = phase_on && nw > 1;
  const double twopi = 2.0 * kPi;  // exact doubling of the reference's pi
  auto next_plane = [&](int iw) {
    do { iw++; } while (iw < nw && counts[1 + iw] == 0);  // planes without data add exact zeros
    return iw;
  };
  auto load_column = [&](V *dst, int iw, uint32_t n, bool active) {
    const uint32_t *mask = rowmask + (uint64_t)iw * nty;
    constexpr int CB = col_block<T>();
    const uint32_t nn = active ? n : 0;
    const V *col = cube + blocked_index<T>(iw, 0, nn, nx, ny);  // row k at col + k * CB
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      const int k = t + q * G;
      const bool touched = active && ((mask[k >> 5] >> (k & 31)) & 1u);
      if (DB) {
        cp_async_zfill<T>(dst + pad(k), touched ? col + (uint64_t)k * CB : col, touched);
      } else {
        V v;
        v.x = 0;
        v.y = 0;
        if (touched) v = col[(uint64_t)k * CB];
        dst[pad(k)] = v;
      }
    }
  };
  const double dwstep = __dmul_rn(twopi, dw);
  for (uint32_t base = blockIdx.x * rpc; base < (uint32_t)nx; base += gridDim.x * rpc) {
    const uint32_t n = base + grp;
    const bool active = n < (uint32_t)nx;
    double acc_re[kVpt], acc_im[kVpt], ph_re[kVpt], ph_im[kVpt];
#pragma unroll
    for (int q = 0; q < kVpt; q++) acc_re[q] = acc_im[q] = ph_re[q] = ph_im[q] = 0.0;
    int iw = next_plane(-1);
    int cur = 0;
    if (DB && iw < nw) {
      load_column(buf[0], iw, n, active);
      cp_async_commit();
    }
    if (phase) {
      // phase_correction.cu:56-64 per pixel of this column, once
      const double l = active ? ltab[n] : 0.0;
#pragma unroll
      for (int q = 0; q < kVpt; q++) {
        const int m = t + q * G;
        const double mm = mtab[m];
        const double radius2 = __dadd_rn(__dmul_rn(l, l), __dmul_rn(mm, mm));
        const double root = __dsqrt_rn(__dsub_rn(1.0, radius2));
        sroot[m] = root;
        if (RECUR) {
          double sn, cs;
          sincos(__dmul_rn(dwstep, __dsub_rn(root, 1.0)), &sn, &cs);
          sstep[m] = make_double2(cs, sn);
        }
      }
    }
    int last_anchor = -kAnchor, prev_iw = -1;
    while (iw < nw) {
      const int nxt = next_plane(iw);
      if (DB) {
        if (nxt < nw) load_column(buf[cur ^ 1], nxt, n, active);
        cp_async_commit();
        cp_async_wait<1>();
      } else {
        load_column(buf[0], iw, n, active);
      }
      __syncthreads();
      V *scol = buf[cur];
      fft_inplace<T, LOGN>(scol, t, tw);
      // phase_correction.cu:51-80 for pixel (m, n) of plane iw
      const double wterm = __dadd_rn(wmin, __dmul_rn((double)iw, dw));
      const double cw = __dmul_rn(twopi, wterm);
      const bool anchor = !RECUR || iw - last_anchor >= kAnchor;
      const int gap = iw - prev_iw;  // planes since the previous phase (empty planes are skipped)
      if (anchor) last_anchor = iw;
      prev_iw = iw;
#pragma unroll
      for (int q = 0; q < kVpt; q++) {
        const int m = t + q * G;
        const Cx<T> x = lds<T>(scol, m);
        const double p = __dmul_rn(norm, (double)x.re), qq = __dmul_rn(norm, (double)x.im);
        if (phase) {
          const double root = sroot[m];
          double sn, cs;
          if (anchor) {
            sincos(__dmul_rn(cw, __dsub_rn(root, 1.0)), &sn, &cs);
          } else {
            // advance by `gap` planes: exp(i gap B), gap >= 1 (empty planes skipped)
            const double2 st = sstep[m];
            double sr = st.x, si = st.y;
            for (int g2 = 1; g2 < gap; g2++) {
              const double tr = sr * st.x - si * st.y;
              si = sr * st.y + si * st.x;
              sr = tr;
            }
            cs = ph_re[q] * sr - ph_im[q] * si;
            sn = ph_re[q] * si + ph_im[q] * sr;
          }
          if (RECUR) {
            ph_re[q] = cs;
            ph_im[q] = sn;
          }
          acc_re[q] += (p * cs - qq * sn) * dwnorm * root;
          acc_im[q] += (p * sn + qq * cs) * dwnorm * root;
        } else {
          acc_re[q] += p;
          acc_im[q] += qq;
        }
      }
      __syncthreads();
      if (DB) cur ^= 1;
      iw = nxt;
    }
    if (DB) cp_async_wait<0>();
    if (active) {
#pragma unroll
      for (int q = 0; q < kVpt; q++) {
        const int m = t + q * G;
        img_re[(uint64_t)m * nx + n] = acc_re[q];
        img_im[(uint64_t)m * nx + n] = acc_im[q];
      }
    }
    __syncthreads();  // sroot / sstep are rewritten for the next column
  }
}

// Compacts the row mask into a list of (plane, row) ids and per-plane counts.
// counts[0] = total rows, counts[1 + w] = rows of plane w.
__global__ void k_row_list(const uint32_t *__restrict__ rowmask, int nw, int ny, int nty,
                           uint32_t *__restrict__ rowlist, uint32_t *__restrict__ counts) {
  const uint64_t nwords = (uint64_t)nw * nty;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nwords;
       i += gridDim.x * (uint64_t)blockDim.x) {
    uint32_t bits = rowmask[i];
    if (!bits) continue;
    const uint32_t w = (uint32_t)(i / nty), band = (uint32_t)(i % nty);
    const uint32_t c = __popc(bits);
    uint32_t slot = atomicAdd(&counts[0], c);
    atomicAdd(&counts[1 + w], c);
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t k = band * 32 + b;
      if (k < (uint32_t)ny) rowlist[slot] = w * (uint32_t)ny + k;
      slot++;
    }
  }
}

template <typename T, int LOGN>
size_t fft_smem(int rpc) {
  constexpr int N = 1 << LOGN;
  return (size_t)rpc * (N + N / 16) * sizeof(typename V2<T>::t);
}

template <typename T, int LOGN>
int launch_rows(FftScratch &f, void *cube, const Geometry &g, const uint32_t *bin_off,
                cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  const int rpc = BT / G;
  const size_t sm = fft_smem<T, LOGN>(rpc);
  RICK_CUDA(cudaFuncSetAttribute(k_fft_rows<T, LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sm));
  int per_sm = 0;
  RICK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fft_rows<T, LOGN>, BT, sm));
  const int blocks = num_sms() * std::max(per_sm, 1);
  RICK_LAUNCHED();
  k_fft_rows<T, LOGN><<<blocks, BT, sm, st>>>(
      (const typename V2<T>::t *)cube, (typename V2<T>::t *)f.blocked, g.nx, g.ny, g.nty, g.ntx,
      f.rowlist, f.counts, bin_off,
      (const typename V2<T>::t *)(sizeof(T) == 8 ? (void *)f.tw_x64 : (void *)f.tw_x32));
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

template <typename T, int LOGN, bool DB, bool RECUR>
size_t cols_smem(int rpc) {
  constexpr int N = 1 << LOGN;
  return fft_smem<T, LOGN>(rpc) * (DB ? 2 : 1) + (size_t)rpc * N * 8 +
         (RECUR ? (size_t)rpc * N * 16 : 0);
}

template <typename T, int LOGN, bool DB, bool RECUR>
int launch_cols_impl(FftScratch &f, const void *cube, const Geometry &g, const double *ltab,
                     const double *mtab, double wmin, double wmax, double norm, int phase_on,
                     double *img_re, double *img_im, cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  const int rpc = BT / G;
  const size_t sm = cols_smem<T, LOGN, DB, RECUR>(rpc);
  RICK_CUDA(cudaFuncSetAttribute(k_fft_cols_image<T, LOGN, DB, RECUR>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  int per_sm = 0;
  RICK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, k_fft_cols_image<T, LOGN, DB, RECUR>, BT, sm));
  const int want = (g.nx + rpc - 1) / rpc;
  const int blocks = std::min(want, num_sms() * std::max(per_sm, 1));
  // phase_correction.cu:100-102
  const double dw = (wmax - wmin) / (double)g.nw;
  const double dwnorm = dw / (wmax - wmin);
  RICK_LAUNCHED();
  k_fft_cols_image<T, LOGN, DB, RECUR><<<blocks, BT, sm, st>>>(
      (const typename V2<T>::t *)f.blocked, g.nx, g.ny, g.nw, g.nty, f.rowmask, f.counts,
      (const typename V2<T>::t *)(sizeof(T) == 8 ? (void *)f.tw_y64 : (void *)f.tw_y32), ltab,
      mtab, wmin, dw, dwnorm, norm, phase_on, img_re, img_im);
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

template <typename T, int LOGN>
int launch_cols(FftScratch &f, const void *cube, const Geometry &g, const double *ltab,
                const double *mtab, double wmin, double wmax, double norm, int phase_on,
                double *img_re, double *img_im, cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  constexpr bool RECUR = sizeof(T) == 4;  // mixed form
  constexpr size_t kMax = 220 * 1024;
  // double-buffer when two column buffers and the per-pixel tables fit
  if (cols_smem<T, LOGN, true, RECUR>(BT / G) <= kMax)
    return launch_cols_impl<T, LOGN, true, RECUR>(f, cube, g, ltab, mtab, wmin, wmax, norm,
                                                  phase_on, img_re, img_im, st);
  if (cols_smem<T, LOGN, false, RECUR>(BT / G) <= kMax)
    return launch_cols_impl<T, LOGN, false, RECUR>(f, cube, g, ltab, mtab, wmin, wmax, norm,
                                                   phase_on, img_re, img_im, st);
  return launch_cols_impl<T, LOGN, false, false>(f, cube, g, ltab, mtab, wmin, wmax, norm,
                                                 phase_on, img_re, img_im, st);
}

int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) l++;
  return l;
}

}  // namespace

bool sparse_fft_supported(int nx, int ny) {
  // power-of-two axes; nx >= 64 also makes nx a multiple of the column block
  auto ok = [](int n) { return n >= 64 && n <= 8192 && (n & (n - 1)) == 0; };
  return ok(nx) && ok(ny);
}

// Per-pass twiddles of the in-place Stockham FFT of N = 2^L points (radix-8
// passes, then one radix-2 or -4 pass): the pass of stride Ns and radix R uses
// entries (Ns-1) + (r-1)*Ns + jm = exp(+2 pi i jm r / (Ns R)), jm < Ns, 1 <= r < R.
// The passes tile [0, N-1) exactly.  Long double, rounded once.
void make_twiddles(int n, double2 *t64, float2 *t32) {
  const long double two_pi = 6.283185307179586476925286766559005768L;
  int L = 0;
  while ((1 << L) < n) L++;
  const int p8 = L / 3, rem = L % 3;
  int Ns = 1;
  for (int p = 0; p < p8 + (rem ? 1 : 0); p++) {
    const int R = p < p8 ? 8 : (1 << rem);
    for (int r = 1; r < R && Ns > 1; r++)
      for (int jm = 0; jm < Ns; jm++) {
        const long double a = two_pi * (long double)(jm * r) / (long double)(Ns * R);
        const int e = (Ns - 1) + (r - 1) * Ns + jm;
        t64[e] = make_double2((double)cosl(a), (double)sinl(a));
        t32[e] = make_float2((float)cosl(a), (float)sinl(a));
      }
    Ns *= R;
  }
  t64[n - 1] = make_double2(1.0, 0.0);  // unused pad entry
  t32[n - 1] = make_float2(1.0f, 0.0f);
}

int sparse_row_list(FftScratch &f, const Geometry &g, cudaStream_t st) {
  RICK_CUDA(cudaMemsetAsync(f.counts, 0, sizeof(uint32_t) * (1 + g.nw), st));
  const uint64_t nwords = (uint64_t)g.nw * g.nty;
  const int blocks = (int)std::min<uint64_t>((nwords + 255) / 256, (uint64_t)num_sms() * 8);
  RICK_LAUNCHED();
  k_row_list<<<std::max(blocks, 1), 256, 0, st>>>(f.rowmask, g.nw, g.ny, g.nty, f.rowlist,
                                                  f.counts);
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

#define RICK_FFT_SIZES(X) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13)

int sparse_fft_rows(int precision, FftScratch &f, void *cube, const Geometry &g,
                    const uint32_t *bin_off, cudaStream_t st) {
  const int lx = ilog2(g.nx);
  if (precision == RICK_PREC_FP64) {
    switch (lx) {
#define X(L) case L: return launch_rows<double, L>(f, cube, g, bin_off, st);
      RICK_FFT_SIZES(X)
#undef X
    }
  } else {
    switch (lx) {
#define X(L) case L: return launch_rows<float, L>(f, cube, g, bin_off, st);
      RICK_FFT_SIZES(X)
#undef X
    }
  }
  return set_error(RICK_ERR_UNSUPPORTED, "sparse FFT: unsupported row length %d", g.nx);
}

int sparse_fft_cols_image(int precision, FftScratch &f, const void *cube, const Geometry &g,
                          const double *ltab, const double *mtab, double wmin, double wmax,
                          double norm, int phase_on, double *img_re, double *img_im,
                          cudaStream_t st) {
  const int ly = ilog2(g.ny);
  if (precision == RICK_PREC_FP64) {
    switch (ly) {
#define X(L)                                                                                   \
  case L:                                                                                      \
    return launch_cols<double, L>(f, cube, g, ltab, mtab, wmin, wmax, norm, phase_on, img_re, \
                                  img_im, st);
      RICK_FFT_SIZES(X)
#undef X
    }
  } else {
    switch (ly) {
#define X(L)                                                                                  \
  case L:                                                                                     \
    return launch_cols<float, L>(f, cube, g, ltab, mtab, wmin, wmax, norm, phase_on, img_re, \
                                 img_im, st);
      RICK_FFT_SIZES(X)
#undef X
    }
  }
  return set_error(RICK_ERR_UNSUPPORTED, "sparse FFT: unsupported column length %d", g.ny);
}

}  // namespace rick
