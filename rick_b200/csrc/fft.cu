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
#include <stdlib.h>

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
// a * (br + i bi) with two fused multiply-adds: the library is built without
// FP contraction (the cell assignment and the phase arguments must round as
// the reference does), so the transforms ask for their FMAs explicitly.
template <typename T>
__device__ __forceinline__ Cx<T> cmul(Cx<T> a, T br, T bi) {
  return {fma(a.re, br, -(a.im * bi)), fma(a.re, bi, a.im * br)};
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

// Shared-memory position of element i of a transform: an XOR swizzle of the
// low bits (no padding), chosen so that every access pattern of the passes is
// free of bank conflicts -- the runs of consecutive elements, the stride-8
// stores of the first pass and the pairs of 8-element runs 64 apart of the
// second (checked by counting wavefronts for every pass of every length).  A
// 16-byte element (FP64 complex) spans 4 banks and 8 lanes share a wavefront:
// bits 3..5 are folded into bits 0..2.  An 8-byte element (FP32) spans 2 banks
// and 16 lanes share a wavefront: bits 4..6 into bits 0..3.  (A pad element
// every 16, the layout this replaces, left 11-20 % more wavefronts.)  The
// swizzle keeps i within its aligned 8- or 16-element block, so the lower half
// of a column stays the lower half.
template <typename T> __host__ __device__ constexpr int padded(int n) { return n; }
template <typename T> __device__ __forceinline__ int pad(int i) {
  if (sizeof(typename V2<T>::t) == 16) return i ^ ((i >> 3) & 7);
  return i ^ (((i >> 4) & 7) | (((i >> 6) & 1) << 3));
}

template <typename T>
__device__ __forceinline__ Cx<T> lds(const typename V2<T>::t *s, int i) {
  const typename V2<T>::t v = s[pad<T>(i)];
  return {v.x, v.y};
}
template <typename T>
__device__ __forceinline__ void sts(typename V2<T>::t *s, int i, Cx<T> c) {
  typename V2<T>::t v;
  v.x = c.re;
  v.y = c.im;
  s[pad<T>(i)] = v;
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

// A global address's line into L2 (no register is written).
__device__ __forceinline__ void prefetch_l2(const void *p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

constexpr int kVpt = 8;  // values per thread

// Row-transformed planes are stored column-blocked: 128-byte blocks of
// columns, each block holding every row -- element (w, k, n) sits at
//   ((w * (nx / CB) + n / CB) * ny + k) * CB + n % CB,   CB = 128 / sizeof(complex).
// Row-pass writes are whole 128-byte lines; the CB CTAs that transform the
// columns of one block stream one contiguous region per plane and share its
// lines in L2.
template <typename T> __host__ __device__ constexpr int col_block() {
  return 128 / (int)sizeof(typename V2<T>::t);
}
template <typename T>
__device__ __forceinline__ uint64_t blocked_index(uint32_t w, uint32_t k, uint32_t n, int nx,
                                                  int ny) {
  constexpr int CB = col_block<T>();
  return (((uint64_t)w * (nx / CB) + n / CB) * ny + k) * CB + (n % CB);
}

// One Stockham pass of radix R over N points held in shared memory by the N/8
// threads of a row group (every value is read into registers before any is
// written back, so the pass works in place).
// The R twiddles of butterfly jm of the pass of stride Ns: w[r] =
// exp(+2 pi i jm r / (Ns R)).  Only w[1] is read (entry (Ns-1) + jm of the
// per-pass table, consecutive lanes reading consecutive entries; the entries a
// column FFT reads total N/7 complex values, which stay in L1); the other
// powers are products of it (w2 = w1^2, w4 = w2^2, w3 = w1 w2, w5 = w1 w4,
// w6 = w2 w4, w7 = w3 w4: a few ulp, far inside the tolerances).
template <typename T, int R>
__device__ __forceinline__ void pass_twiddles(const typename V2<T>::t *__restrict__ twp,
                                              Cx<T> w[R]) {
  w[0] = {(T)1, (T)0};
  if (R == 1) return;
  const typename V2<T>::t a = __ldg(twp);
  w[1] = {a.x, a.y};
  if (R >= 4) {
    w[2] = cmul<T>(w[1], w[1].re, w[1].im);
    w[3] = cmul<T>(w[1], w[2].re, w[2].im);
  }
  if (R == 8) {
    w[4] = cmul<T>(w[2], w[2].re, w[2].im);
    w[5] = cmul<T>(w[1], w[4].re, w[4].im);
    w[6] = cmul<T>(w[2], w[4].re, w[4].im);
    w[7] = cmul<T>(w[3], w[4].re, w[4].im);
  }
}

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
      Cx<T> w[R];
      pass_twiddles<T, R>(tw + (Ns - 1) + jm, w);
#pragma unroll
      for (int r = 1; r < R; r++) v[b][r] = cmul<T>(v[b][r], w[r].re, w[r].im);
    }
    Dft<T, R>::run(v[b]);
    const int idx = (j - jm) * R + jm;
#pragma unroll
    for (int r = 0; r < R; r++) sts<T>(s, idx + r * Ns, v[b][r]);
  }
  __syncthreads();
}

// The last Stockham pass (Ns * R == N) with its outputs kept in registers:
// thread t's butterflies write positions t + q*G, q = b + B*r, so out[q] is the
// transform's value at index t + q*G -- exactly the points the thread owns next.
template <typename T, int N, int R>
__device__ __forceinline__ void stockham_last_pass(const typename V2<T>::t *s, int t,
                                                   const typename V2<T>::t *__restrict__ tw,
                                                   Cx<T> out[kVpt]) {
  constexpr int G = N / kVpt, B = kVpt / R, Ns = N / R;
  Cx<T> v[B][R];
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * G;
#pragma unroll
    for (int r = 0; r < R; r++) v[b][r] = lds<T>(s, j + r * (N / R));
  }
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * G;  // j < Ns, so jm = j and the output index is j + r*Ns
    if (Ns > 1) {
      Cx<T> w[R];
      pass_twiddles<T, R>(tw + (Ns - 1) + j, w);
#pragma unroll
      for (int r = 1; r < R; r++) v[b][r] = cmul<T>(v[b][r], w[r].re, w[r].im);
    }
    Dft<T, R>::run(v[b]);
#pragma unroll
    for (int r = 0; r < R; r++) out[b + B * r] = v[b][r];
  }
}

// Inverse FFT of N = 2^LOGN points held in shared memory; the result of the
// last pass stays in registers (out[q] = value at t + q*G).  The buffer may be
// overwritten after the caller's next barrier.
template <typename T, int LOGN>
__device__ __forceinline__ void fft_to_regs(typename V2<T>::t *s, int t,
                                            const typename V2<T>::t *__restrict__ tw,
                                            Cx<T> out[kVpt]) {
  constexpr int N = 1 << LOGN;
  constexpr int P8 = LOGN / 3, REM = LOGN % 3;
  constexpr int LASTR = REM == 0 ? 8 : (1 << REM);
  constexpr int NPASS = P8 + (REM ? 1 : 0);
  int Ns = 1;
#pragma unroll
  for (int p = 0; p < NPASS - 1; p++) {
    stockham_pass<T, N, 8>(s, t, Ns, tw);
    Ns *= 8;
  }
  stockham_last_pass<T, N, LASTR>(s, t, tw, out);
}

// The passes of an N = 2^LOGN transform after its first (stride-1, radix-8)
// pass, whose outputs are in shared memory; the last pass leaves its results
// in registers (out[q] = value at t + q*G).
template <typename T, int LOGN>
__device__ __forceinline__ void fft_tail_to_regs(typename V2<T>::t *s, int t,
                                                 const typename V2<T>::t *__restrict__ tw,
                                                 Cx<T> out[kVpt]) {
  constexpr int N = 1 << LOGN;
  constexpr int P8 = LOGN / 3, REM = LOGN % 3;
  constexpr int LASTR = REM == 0 ? 8 : (1 << REM);
  constexpr int NPASS = P8 + (REM ? 1 : 0);
  static_assert(NPASS >= 2, "the first pass is a radix-8 pass before the last one");
  int Ns = 8;
#pragma unroll
  for (int p = 1; p < NPASS - 1; p++) {
    stockham_pass<T, N, 8>(s, t, Ns, tw);
    Ns *= 8;
  }
  stockham_last_pass<T, N, LASTR>(s, t, tw, out);
}

// The first pass (stride 1, radix 8) from registers: v[r] is thread t's input
// at t + r*N/8 (its first butterfly's inputs); its outputs go to t*8 + r.  The
// buffer must be free (no thread still reading it) when this is called.
template <typename T>
__device__ __forceinline__ void first_pass_from_regs(typename V2<T>::t *s, int t, Cx<T> v[8]) {
  Dft<T, 8>::run(v);
#pragma unroll
  for (int r = 0; r < 8; r++) sts<T>(s, t * 8 + r, v[r]);
  __syncthreads();
}

// fft_to_regs with the first pass fed from registers (as first_pass_from_regs).
template <typename T, int LOGN>
__device__ __forceinline__ void fft_to_regs_r(typename V2<T>::t *s, int t,
                                              const typename V2<T>::t *__restrict__ tw,
                                              Cx<T> v[8], Cx<T> out[kVpt]) {
  first_pass_from_regs<T>(s, t, v);
  fft_tail_to_regs<T, LOGN>(s, t, tw, out);
}

// PP transforms at once, one per shared buffer, sharing every barrier (twice
// the independent work between barriers for PP = 2).
template <typename T, int N, int R, int PP>
__device__ __forceinline__ void stockham_pass_pp(typename V2<T>::t *const *s, int t, int Ns,
                                                 const typename V2<T>::t *__restrict__ tw) {
  constexpr int G = N / kVpt, B = kVpt / R;
  Cx<T> v[PP][B][R];
#pragma unroll
  for (int pp = 0; pp < PP; pp++)
#pragma unroll
    for (int b = 0; b < B; b++) {
      const int j = t + b * G;
#pragma unroll
      for (int r = 0; r < R; r++) v[pp][b][r] = lds<T>(s[pp], j + r * (N / R));
    }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * G;
    const int jm = j & (Ns - 1);
    Cx<T> w[R];
    w[0] = {(T)1, (T)0};
    if (Ns > 1) pass_twiddles<T, R>(tw + (Ns - 1) + jm, w);
    const int idx = (j - jm) * R + jm;
#pragma unroll
    for (int pp = 0; pp < PP; pp++) {
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) v[pp][b][r] = cmul<T>(v[pp][b][r], w[r].re, w[r].im);
      }
      Dft<T, R>::run(v[pp][b]);
#pragma unroll
      for (int r = 0; r < R; r++) sts<T>(s[pp], idx + r * Ns, v[pp][b][r]);
    }
  }
  __syncthreads();
}

template <typename T, int N, int R, int PP>
__device__ __forceinline__ void stockham_last_pass_pp(typename V2<T>::t *const *s, int t,
                                                      const typename V2<T>::t *__restrict__ tw,
                                                      Cx<T> out[PP][kVpt]) {
  constexpr int G = N / kVpt, B = kVpt / R, Ns = N / R;
#pragma unroll
  for (int b = 0; b < B; b++) {
    const int j = t + b * G;  // j < Ns: the output index is j + r*Ns
    Cx<T> w[R];
    w[0] = {(T)1, (T)0};
    if (Ns > 1) pass_twiddles<T, R>(tw + (Ns - 1) + j, w);
#pragma unroll
    for (int pp = 0; pp < PP; pp++) {
      Cx<T> v[R];
#pragma unroll
      for (int r = 0; r < R; r++) v[r] = lds<T>(s[pp], j + r * (N / R));
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = cmul<T>(v[r], w[r].re, w[r].im);
      }
      Dft<T, R>::run(v);
#pragma unroll
      for (int r = 0; r < R; r++) out[pp][b + B * r] = v[r];
    }
  }
}

// Passes of the FFT of N = 2^LOGN points: radix-8 passes, the last one of
// radix 2, 4 or 8.
template <int LOGN> __host__ __device__ constexpr int fft_passes() { return LOGN / 3 + (LOGN % 3 ? 1 : 0); }

// after(p) runs between the passes (p = 0 .. passes - 2), behind each pass's
// closing barrier.
template <typename T, int LOGN, int PP, typename After>
__device__ __forceinline__ void fft_to_regs_pp(typename V2<T>::t *const *s, int t,
                                               const typename V2<T>::t *__restrict__ tw,
                                               Cx<T> out[PP][kVpt], After after) {
  constexpr int N = 1 << LOGN;
  constexpr int REM = LOGN % 3;
  constexpr int LASTR = REM == 0 ? 8 : (1 << REM);
  constexpr int NPASS = fft_passes<LOGN>();
  int Ns = 1;
#pragma unroll
  for (int p = 0; p < NPASS - 1; p++) {
    stockham_pass_pp<T, N, 8, PP>(s, t, Ns, tw);
    after(p);
    Ns *= 8;
  }
  stockham_last_pass_pp<T, N, LASTR, PP>(s, t, tw, out);
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

template <int LOGN> __host__ __device__ constexpr int group_threads() { return (1 << LOGN) / kVpt; }
template <int LOGN> __host__ __device__ constexpr int block_threads() {
  return group_threads<LOGN>() > 256 ? group_threads<LOGN>() : 256;
}
// Blocks of 256 threads (lengths up to 2048) are bounded to 128 registers so
// that two share an SM.
template <int LOGN> constexpr int min_blocks() { return block_threads<LOGN>() <= 256 ? 2 : 1; }
// FP32 column passes of one plane in flight fit 80 registers without spills:
// three 256-thread blocks share an SM (24 warps against 16 to hide latency).
template <typename T, int LOGN, int PP> constexpr int col_min_blocks() {
  return sizeof(T) == 4 && PP == 1 && block_threads<LOGN>() <= 256 ? 3 : min_blocks<LOGN>();
}
// The row pass holds no per-pixel state: 64 registers a thread, so that 1024
// threads (4, 2 or 1 blocks) share an SM.
template <int LOGN> constexpr int row_min_blocks() { return 1024 / block_threads<LOGN>(); }

// Row pass: inverse FFT along x of the listed touched rows, from the gridded
// cube into the column-blocked buffer.  Tiles that received no record (bit
// clear in the band's tile bitmap) were never written and read as zeros.  The
// last FFT pass leaves each thread's outputs in registers, stored as whole
// 128-byte lines.  One call transforms one row per row group (blockDim / G rows
// per block); every thread of the block takes part.
template <typename T, int LOGN>
__device__ __forceinline__ void fft_row_unit(typename V2<T>::t *s, bool active, uint32_t w,
                                             uint32_t k, const typename V2<T>::t *__restrict__ cube,
                                             typename V2<T>::t *__restrict__ out, int nx, int ny,
                                             int nty, int tmw,
                                             const uint32_t *__restrict__ tilemask,
                                             const typename V2<T>::t *__restrict__ tw) {
  constexpr int N = 1 << LOGN, G = N / kVpt, LEN = padded<T>(N);
  using V = typename V2<T>::t;
  const int grp = threadIdx.x / G, t = threadIdx.x % G;
  V *srow = s + grp * LEN;
  if (!active) w = k = 0;
  const uint32_t *tm = tilemask + ((uint64_t)w * nty + (k >> 5)) * tmw;
  const uint64_t rowbase = ((uint64_t)w * ny + k) * nx;
  // thread t's inputs x = t + q*G are its first butterfly's: straight to registers
  Cx<T> in[kVpt];
#pragma unroll
  for (int q = 0; q < kVpt; q++) {
    const int x = t + q * G;
    V v;
    v.x = 0;
    v.y = 0;
    if (active && ((tm[x >> 10] >> ((x >> 5) & 31)) & 1u)) v = cube[rowbase + x];
    in[q] = {v.x, v.y};
  }
  Cx<T> res[kVpt];
  fft_to_regs_r<T, LOGN>(srow, t, tw, in, res);
  if (active) {
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      V v;
      v.x = res[q].re;
      v.y = res[q].im;
      out[blocked_index<T>(w, k, t + q * G, nx, ny)] = v;
    }
  }
  __syncthreads();
}

// One job's row pass (the plan): the job's arrays as kernel parameters.
template <typename T, int LOGN>
__global__ void __launch_bounds__(block_threads<LOGN>(), row_min_blocks<LOGN>())
    k_fft_rows(const typename V2<T>::t *__restrict__ cube, typename V2<T>::t *__restrict__ out,
               int nx, int ny, int nty, int tmw, const uint32_t *__restrict__ tilemask,
               const uint32_t *__restrict__ rowlist, const uint32_t *__restrict__ counts,
               const typename V2<T>::t *__restrict__ tw) {
  constexpr int G = (1 << LOGN) / kVpt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto *s = reinterpret_cast<typename V2<T>::t *>(smem_raw);
  const int rpc = blockDim.x / G;  // rows per CTA
  const int grp = threadIdx.x / G;
  const uint32_t nrows = counts[0];
  for (uint32_t base = blockIdx.x * rpc; base < nrows; base += gridDim.x * rpc) {
    const uint32_t li = base + grp;
    const bool active = li < nrows;
    const uint32_t rid = active ? rowlist[li] : 0;
    if constexpr (LOGN >= 13) {
      // 8192-point rows: one block (one row) per SM, so the next row's touched
      // tiles are prefetched into L2 while this one is transformed (c3 row pass
      // 5.51 -> 5.14 ms FP64; at 4096 points, two blocks per SM, it slowed it)
      const uint32_t ln = li + gridDim.x * rpc;
      if (ln < nrows) {
        const uint32_t rn = rowlist[ln];
        const uint32_t wn = rn / (uint32_t)ny, kn = rn % (uint32_t)ny;
        const uint32_t *tmn = tilemask + ((uint64_t)wn * nty + (kn >> 5)) * tmw;
        const typename V2<T>::t *pn = cube + ((uint64_t)wn * ny + kn) * nx;
        const int t = threadIdx.x % G;
#pragma unroll
        for (int q = 0; q < kVpt; q++) {
          const int x = t + q * G;
          if ((tmn[x >> 10] >> ((x >> 5) & 31)) & 1u) prefetch_l2(pn + x);
        }
      }
    }
    fft_row_unit<T, LOGN>(s, active, rid / (uint32_t)ny, rid % (uint32_t)ny, cube, out, nx, ny,
                          nty, tmw, tilemask, tw);
  }
}

// Row pass over the jobs lo..hi-1 of a batch (all of FFT length 2^LOGN along x): the
// row-pass units of job j (groups of rows_per_block touched rows) are
// fft_units[j] .. fft_units[j+1]-1.
template <typename T, int LOGN>
__global__ void __launch_bounds__(block_threads<LOGN>(), row_min_blocks<LOGN>())
    k_fft_rows_multi(const BatchJob *__restrict__ jobs, int lo, int hi,
               const uint32_t *__restrict__ fft_units, const uint32_t *__restrict__ tilemask,
               const uint32_t *__restrict__ rowlist, const uint32_t *__restrict__ counts) {
  constexpr int G = (1 << LOGN) / kVpt;
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto *s = reinterpret_cast<V *>(smem_raw);
  const int rpc = blockDim.x / G;  // rows per CTA
  const int grp = threadIdx.x / G;
  const uint32_t u1 = fft_units[hi];
  for (uint32_t u = fft_units[lo] + blockIdx.x; u < u1; u += gridDim.x) {
    const int j = lo + batch_job_of(fft_units + lo, hi - lo, u);
    const BatchJob &J = jobs[j];
    const uint32_t li = (u - fft_units[j]) * rpc + grp;
    const bool active = li < counts[J.counts_base];
    const uint32_t rid = active ? rowlist[J.list_base + li] : 0;
    const uint32_t ny = (uint32_t)J.g.ny;
    fft_row_unit<T, LOGN>(s, active, rid / ny, rid % ny, (const V *)J.cube, (V *)J.blocked,
                          J.g.nx, J.g.ny, J.g.nty, (J.g.ntx + 31) / 32, tilemask + J.tile_base,
                          (const V *)J.tw_x);
  }
}

// Column pass fused with the w-correction and the plane sum: each row group
// owns one image column and walks the planes in increasing w.  With DB the
// next plane's column is copied into a second shared buffer (cp.async,
// untouched rows zero-filled) while the current one is transformed; the last
// FFT pass leaves the column's values in the registers of the threads that
// accumulate those pixels.  PP planes share one pass through the FFT's
// barriers.
//
// Phase (phase_correction.cu:51-80): every kAnchor planes (and at the first
// plane; at every plane without RECUR, when the step table does not fit) the
// factor exp(i*(2 pi wterm)*(root-1)) is evaluated with sincos of the
// reference's FP64 argument and scaled by dwnorm*root; between anchors it
// advances by the per-pixel step exp(i*(2 pi dw)*(root-1)) (shared memory).
// Over 8 planes the advanced factor differs from a long-double evaluation by
// < 1e-13 per pixel at the w range of a 4096^2 x 32-plane LOFAR-like image --
// less than the rounding of the reference's own argument (~3e-13).
constexpr int kAnchor = 8;

// The per-job inputs of the column pass.
template <typename T> struct ColJob {
  const typename V2<T>::t *cube;  // column-blocked row transforms
  int nx, ny, nw, nty;
  int w_first, nw_total;          // w-plane shard: global index of local plane 0, cube planes
  const uint32_t *rowmask;        // [nw * nty]
  const uint32_t *counts;         // [1 + nw]
  const typename V2<T>::t *tw;    // twiddles of the y axis
  const double *ltab, *mtab;
  double wmin, dw, dwnorm, norm;
  int phase_on;
  double *img_re, *img_im;
};

// Shared memory of one block of the column pass: NB column buffers per row
// group, the per-pixel phase steps (RECUR; complex in the accumulation type T)
// and the row masks of 2*PP planes.
template <typename T, int LOGN, bool DB, bool RECUR, int PP>
__host__ __device__ constexpr size_t cols_smem_bytes(int rpc) {
  return (size_t)rpc * padded<T>(1 << LOGN) * sizeof(typename V2<T>::t) *
             (DB ? 2 : 1) * PP +
         (RECUR ? (size_t)rpc * (1 << LOGN) * sizeof(typename V2<T>::t) : 0) +
         2 * PP * (size_t)((1 << LOGN) / 32) * 4;
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }

// Columns base..base+rpc-1 (one per row group) of one job.  The pixel sums,
// the phase factors and the per-pixel steps are kept in the FFT's type: FP64
// for the plain form; FP32 for the mixed form, whose phase arguments (and
// their sincos) stay FP64 -- only the unit-modulus factors are rounded.
template <typename T, int LOGN, bool DB, bool RECUR, int PP>
__device__ __forceinline__ void fft_col_unit(typename V2<T>::t *s, uint32_t base,
                                             const ColJob<T> &J) {
  constexpr int N = 1 << LOGN, G = N / kVpt, LEN = padded<T>(N);
  constexpr int NB = (DB ? 2 : 1) * PP;  // column buffers per row group
  using V = typename V2<T>::t;
  const int rpc = blockDim.x / G;
  const int grp = threadIdx.x / G, t = threadIdx.x % G;
  const int nx = J.nx, ny = J.ny, nw = J.nw, nty = J.nty;
  const uint32_t *__restrict__ rowmask = J.rowmask;
  const uint32_t *__restrict__ counts = J.counts;
  const double *__restrict__ mtab = J.mtab;
  V *sbase = s + grp * NB * LEN;  // buffers [set][pp]: set = cur (DB), pp < PP
  V *tables = s + rpc * NB * LEN;
  V *sstep = tables + grp * N;  // RECUR only
  // row masks of the planes of the next two sets (2 * PP slots)
  uint32_t *smask = reinterpret_cast<uint32_t *>(tables + (RECUR ? rpc * N : 0));
  const bool phase = J.phase_on && J.nw_total > 1;
  const double twopi = 2.0 * kPi;  // exact doubling of the reference's pi
  auto next_plane = [&](int iw) {
    do { iw++; } while (iw < nw && counts[1 + iw] == 0);  // planes without data add exact zeros
    return iw;
  };
  // the next PP planes with data after plane `after` (nw = none)
  auto next_set = [&](int after, int set[PP]) {
#pragma unroll
    for (int pp = 0; pp < PP; pp++) {
      after = next_plane(after);
      set[pp] = after;
      if (after >= nw) after = nw;
    }
  };
  auto stage_masks = [&](int slot, const int set[PP]) {
    for (int i = threadIdx.x; i < PP * nty; i += blockDim.x) {
      const int pp = i / nty, word = i % nty;
      if (set[pp] < nw) smask[(slot * PP + pp) * nty + word] = rowmask[(uint64_t)set[pp] * nty + word];
    }
  };
  const uint32_t n = base + grp;
  const bool active = n < (uint32_t)nx;
  // rows t + q*G, q in [Q0, Q1), of the planes `set` into buffer set `bset`
  // (q0, q1 are constants once the pass loop is unrolled)
  auto load_rows = [&](int q0, int q1, int bset, const int set[PP], int slot) {
#pragma unroll
    for (int pp = 0; pp < PP; pp++) {
      if (set[pp] >= nw) continue;
      V *dst = sbase + (bset * PP + pp) * LEN;
      const uint32_t *mask = smask + (slot * PP + pp) * nty;
      constexpr int CB = col_block<T>();
      const V *col = J.cube + blocked_index<T>(set[pp], 0, active ? n : 0, nx, ny);
#pragma unroll
      for (int q = 0; q < kVpt; q++) {
        if (q < q0 || q >= q1) continue;
        const int k = t + q * G;
        const bool touched = active && ((mask[k >> 5] >> (k & 31)) & 1u);
        if (DB) {
          cp_async_zfill<T>(dst + pad<T>(k), touched ? col + (uint64_t)k * CB : col, touched);
        } else {
          V v;
          v.x = 0;
          v.y = 0;
          if (touched) v = col[(uint64_t)k * CB];
          dst[pad<T>(k)] = v;
        }
      }
    }
  };
  // sqrt(1 - l^2 - m^2), phase_correction.cu:56-64, always the same bits
  auto root_of = [&](double l, int m) {
    const double mm = mtab[m];
    return __dsqrt_rn(__dsub_rn(1.0, __dadd_rn(__dmul_rn(l, l), __dmul_rn(mm, mm))));
  };
  const double dwstep = __dmul_rn(twopi, J.dw);
  const double l = active ? J.ltab[n] : 0.0;
  T acc_re[kVpt], acc_im[kVpt], ph_re[kVpt], ph_im[kVpt];
#pragma unroll
  for (int q = 0; q < kVpt; q++) acc_re[q] = acc_im[q] = ph_re[q] = ph_im[q] = (T)0;
  // 1/(Nx*Ny), a power of two (exact in FP32): every rounding commutes with
  // it (away from underflow), so scaling the sums once at the end gives the
  // bits of scaling each plane's transform, as the reference does
  const T norm = (T)J.norm;
  int cur[PP], nxt[PP];
  next_set(-1, cur);
  next_set(cur[PP - 1], nxt);
  stage_masks(0, cur);
  stage_masks(1, nxt);
  if (phase && RECUR) {
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      const int m = t + q * G;
      double sn, cs;
      sincos(__dmul_rn(dwstep, __dsub_rn(root_of(l, m), 1.0)), &sn, &cs);
      V st;
      st.x = (T)cs;
      st.y = (T)sn;
      sstep[m] = st;
    }
  }
  __syncthreads();
  if (DB && cur[0] < nw) {
    load_rows(0, kVpt, 0, cur, 0);
    cp_async_commit();
  }
  // With DB the next set's copies are spread over this set's FFT passes (a
  // share of the rows before each of the first NS passes): issued all at
  // once, behind the barrier where every warp stands, they fill the
  // global-load queue while no warp has arithmetic to issue.  Measured at
  // 4096 points: FP64 (one plane an iteration) is fastest with the copies in
  // flight by the second pass, FP32 (two planes) with a share before every pass.
  constexpr int NS = sizeof(T) == 8 ? 2 : fft_passes<LOGN>();
  int bset = 0, it = 0;
  int last_anchor = -kAnchor, prev_iw = -1;
  while (cur[0] < nw) {
    int nn[PP];
    next_set(nxt[PP - 1], nn);  // the set after the next one
    if (DB) {
      cp_async_wait<0>();  // this set's copies
    } else {
      load_rows(0, kVpt, 0, cur, it & 1);
    }
    // every copy of this set has landed; every thread is done with the
    // previous set's buffers and mask slot
    __syncthreads();
    // this set's mask slot is free now: stage the set after next
    stage_masks(it & 1, nn);
    V *bufs[PP];
#pragma unroll
    for (int pp = 0; pp < PP; pp++) bufs[pp] = sbase + ((DB ? bset : 0) * PP + pp) * LEN;
    const bool more = DB && nxt[0] < nw;
    auto load_share = [&](int c) {  // share c of NS of the next set's rows
      if (more && c < NS) load_rows(c * kVpt / NS, (c + 1) * kVpt / NS, bset ^ 1, nxt, (it + 1) & 1);
    };
    load_share(0);
    Cx<T> x[PP][kVpt];
    fft_to_regs_pp<T, LOGN, PP>(bufs, t, J.tw, x, [&](int p) { load_share(p + 1); });
    if (DB) cp_async_commit();
#pragma unroll
    for (int pp = 0; pp < PP; pp++) {
      const int iw = cur[pp];
      if (iw >= nw) break;
      const bool anchor = !RECUR || iw - last_anchor >= kAnchor;
      const int gap = iw - prev_iw;  // planes since the previous factor (empty planes skipped)
      double cw = 0.0;
      if (anchor) {
        last_anchor = iw;
        cw = __dmul_rn(twopi, __dadd_rn(J.wmin, __dmul_rn((double)(J.w_first + iw), J.dw)));  // 2 pi wterm
      }
      prev_iw = iw;
#pragma unroll
      for (int q = 0; q < kVpt; q++) {
        const int m = t + q * G;
        const T p = x[pp][q].re, qq = x[pp][q].im;
        if (phase) {
          if (anchor) {
            const double root = root_of(l, m);
            double sn, cs;
            sincos(__dmul_rn(cw, __dsub_rn(root, 1.0)), &sn, &cs);
            const double amp = J.dwnorm * root;
            ph_re[q] = (T)(cs * amp);
            ph_im[q] = (T)(sn * amp);
          } else {
            const V st = sstep[m];
            T sr = st.x, si = st.y;
            for (int g2 = 1; g2 < gap; g2++) {
              const T tr = sr * st.x - si * st.y;
              si = sr * st.y + si * st.x;
              sr = tr;
            }
            const T tr = ph_re[q] * sr - ph_im[q] * si;
            ph_im[q] = ph_re[q] * si + ph_im[q] * sr;
            ph_re[q] = tr;
          }
          acc_re[q] += p * ph_re[q] - qq * ph_im[q];
          acc_im[q] += p * ph_im[q] + qq * ph_re[q];
        } else {
          acc_re[q] += p;
          acc_im[q] += qq;
        }
      }
    }
    // single buffer: the next set is copied at the top of the next iteration
    // (with DB the barrier there, before any copy into this buffer, suffices)
    if (!DB) __syncthreads();
    if (DB) bset ^= 1;
#pragma unroll
    for (int pp = 0; pp < PP; pp++) {
      cur[pp] = nxt[pp];
      nxt[pp] = nn[pp];
    }
    it++;
  }
  if (DB) cp_async_wait<0>();
  if (active) {
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      const int m = t + q * G;
      J.img_re[(uint64_t)m * nx + n] = (double)mul_rn(norm, acc_re[q]);
      J.img_im[(uint64_t)m * nx + n] = (double)mul_rn(norm, acc_im[q]);
    }
  }
  __syncthreads();  // sstep / smask are rewritten for the next column
}

// ---- Column pass with the per-pixel state in tensor memory ---------------
//
// The w-correction as a Horner recurrence over the planes, walked in
// decreasing w: with s = exp(i 2 pi dw (root - 1)) the per-pixel factor
// between consecutive planes and P = dwnorm root exp(i 2 pi wterm_lo (root-1))
// the factor of the lowest plane with data,
//     image = P * (((x_hi s^g + ...) s^g' + x_lo)
// so each pixel carries two complex values across planes -- its running sum
// and its step s -- and the phase needs one sincos per pixel for s and one
// for P per column, none per plane.  The reference evaluates every plane's
// factor with its own sincos (phase_correction.cu:205-226); the recurrence's
// products move each factor by a few ulp per plane.  Modelled in long double
// for the worst pixels: 8.4e-14 at 4096^2 x 32 planes (w from -7.5e3 to 7.8e3
// wavelengths) and 2.6e-13 at 8192^2 x 64 planes (w to 1.1e5), below the
// rounding of the reference's own per-plane phase argument there (1.3e-13 and
// 3.3e-13 at the image corner).
//
// The two complex values of the thread's 8 pixels (64 32-bit words) live in
// tensor memory (TMEM, 512 columns x 128 lanes of 32 bits per SM), not in
// registers: the thread's FFT then runs in 64 registers, so 1024 threads
// share an SM (two 4096-point columns, four blocks of shorter ones) where the
// register-resident form held one.  Warp w of a block reaches lanes
// 32 (w % 4) .. +31 (its lane quarter); the warps of one quarter split its
// columns, 64 each, so a block allocates (warps / 4) * 64 columns and two,
// one or four blocks fill an SM's 512.  Column loads are single-buffered: the
// next plane's copies are issued as soon as the FFT's last pass has read the
// buffer and land during the recurrence, and the other blocks of the SM
// overlap the rest.
namespace tm {

__device__ __forceinline__ void alloc(uint32_t *smem_dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                   (uint32_t)__cvta_generic_to_shared(smem_dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// 8 consecutive columns of the thread's lane; the registers are ready after
// wait_ld8, which names them so that no use moves above the wait.
__device__ __forceinline__ void ld8(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void wait_ld8(uint32_t (&a)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]),
                 "+r"(a[6]), "+r"(a[7])
               :
               : "memory");
}

// 4 consecutive columns; the registers are ready after wait_ld4.
__device__ __forceinline__ void ld4(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void wait_ld4(uint32_t (&a)[4]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3])
               :
               : "memory");
}
__device__ __forceinline__ void st4(uint32_t taddr, const uint32_t (&r)[4]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(taddr),
               "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3])
               : "memory");
}
// The stored registers stay untouched until the store has completed.
__device__ __forceinline__ void wait_st4(uint32_t (&r)[4]) {
  asm volatile("tcgen05.wait::st.sync.aligned;\n"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3])
               :
               : "memory");
}

// 16 consecutive columns (two pixels' sums and steps); ready after wait_ld16.
__device__ __forceinline__ void ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
}
__device__ __forceinline__ void wait_ld16(uint32_t (&a)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]),
                 "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]),
                 "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15])
               :
               : "memory");
}
__device__ __forceinline__ void st2(uint32_t taddr, const uint32_t (&r)[2]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};\n" ::"r"(taddr), "r"(r[0]),
               "r"(r[1])
               : "memory");
}
__device__ __forceinline__ void wait_st2(uint32_t (&r)[2]) {
  asm volatile("tcgen05.wait::st.sync.aligned;\n" : "+r"(r[0]), "+r"(r[1]) : : "memory");
}
__device__ __forceinline__ void ld2(uint32_t taddr, uint32_t (&r)[2]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n"
               : "=r"(r[0]), "=r"(r[1])
               : "r"(taddr)
               : "memory");
}
__device__ __forceinline__ void wait_ld2(uint32_t (&a)[2]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" : "+r"(a[0]), "+r"(a[1]) : : "memory");
}
__device__ __forceinline__ void st16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16};\n" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void wait_st16(uint32_t (&a)[16]) {
  asm volatile("tcgen05.wait::st.sync.aligned;\n"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]),
                 "+r"(a[6]), "+r"(a[7]), "+r"(a[8]), "+r"(a[9]), "+r"(a[10]), "+r"(a[11]),
                 "+r"(a[12]), "+r"(a[13]), "+r"(a[14]), "+r"(a[15])
               :
               : "memory");
}
// Two 4-column stores in flight: both register sets stay untouched until done.
__device__ __forceinline__ void wait_st4x2(uint32_t (&a)[4], uint32_t (&b)[4]) {
  asm volatile("tcgen05.wait::st.sync.aligned;\n"
               : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(b[0]), "+r"(b[1]),
                 "+r"(b[2]), "+r"(b[3])
               :
               : "memory");
}

__device__ __forceinline__ double join(uint32_t lo, uint32_t hi) {
  return __hiloint2double((int)hi, (int)lo);
}
__device__ __forceinline__ void split(double v, uint32_t &lo, uint32_t &hi) {
  lo = (uint32_t)__double2loint(v);
  hi = (uint32_t)__double2hiint(v);
}

}  // namespace tm

// TMEM columns a block of `threads` allocates: 64 per warp of a lane quarter.
__host__ __device__ constexpr uint32_t tm_cols(int threads) {
  return (uint32_t)(threads / 32 / 4) * 64u;
}

// Shared memory of the TMEM column pass: a column buffer per row group and 16
// bytes for the TMEM address.
template <typename T, int LOGN>
__host__ __device__ constexpr size_t cols_tm_smem_bytes(int rpc) {
  return (size_t)rpc * padded<T>(1 << LOGN) * sizeof(typename V2<T>::t) + 16;
}

// Columns base..base+rpc-1 of one job (one per row group).  The FFT runs in
// T (FP64 for the plain form, FP32 for the mixed one); the recurrence, its
// steps and the anchor factor are FP64 in both, so the mixed form adds no
// phase error to its FP32 transform's.  Only the touched rows of a plane are
// copied in: thread t copies rows t + q*G (q = 0..7), exactly the inputs of
// its first-pass butterfly, and reads zero for the untouched ones (bit q of
// its row mask clear).  The next plane's row bits are read before this plane's
// transform (3.78 -> 3.60 ms FP64, 3.14 -> 2.85 ms FP32 at 4096^2 x 32 against
// reading them after it); its rows are copied once the transform has read the
// buffer, during the recurrence, and the SM's other blocks cover the rest of
// the copies' latency (copying between the last pass's loads and its
// arithmetic measured slower at 4096 points: 3.78 against 3.60 ms).  (A half buffer for the lower rows, copied as soon as
// the first pass had read them, and a second full buffer where it fits, were
// both measured slower: 3.86 and 3.14 ms against 3.73 and 3.02 ms for the FP64
// and FP32 passes at 4096^2 x 32.)  `taddr` is the thread's TMEM address: its
// lane quarter and its warp's 64 columns, 8 per pixel q at 8q -- the running
// sum (re lo/hi, im lo/hi) then the step -- so one 8-column load brings both.
template <typename T, int LOGN>
__device__ __forceinline__ void fft_col_unit_tm(typename V2<T>::t *s, uint32_t base,
                                                const ColJob<T> &J, uint32_t taddr) {
  constexpr int N = 1 << LOGN, G = N / kVpt, LEN = padded<T>(N);
  constexpr int CB = col_block<T>();
  using V = typename V2<T>::t;
  const int grp = threadIdx.x / G, t = threadIdx.x % G;
  const int nx = J.nx, ny = J.ny, nw = J.nw, nty = J.nty;
  const uint32_t *__restrict__ counts = J.counts;
  V *buf = s + grp * LEN;
  const uint32_t n = base + grp;
  const bool active = n < (uint32_t)nx;
  const bool phase = J.phase_on && J.nw_total > 1;
  const double twopi = 2.0 * kPi;  // exact doubling of the reference's pi
  auto prev_plane = [&](int iw) {   // planes without data add exact zeros
    do { iw--; } while (iw >= 0 && counts[1 + iw] == 0);
    return iw;
  };
  // bit q: whether row t + q*G of plane iw was touched (read before the
  // transform of the plane before it, so that these loads fly during it)
  auto row_bits = [&](int iw) {
    const uint32_t *__restrict__ mask = J.rowmask + (uint64_t)iw * nty;
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      const int k = t + q * G;
      const bool touched = active && ((__ldg(mask + (k >> 5)) >> (k & 31)) & 1u);
      bits |= (touched ? 1u : 0u) << q;
    }
    return bits;
  };
  // the touched rows t + q*G of plane iw into the buffer
  auto copy_rows = [&](int iw, uint32_t bits) {
    const V *col = J.cube + blocked_index<T>(iw, 0, active ? n : 0, nx, ny);
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      const int k = t + q * G;
      if ((bits >> q) & 1u) cp_async_zfill<T>(buf + pad<T>(k), col + (uint64_t)k * CB, true);
    }
    cp_async_commit();
  };
  auto load_rows = [&](int iw) {
    const uint32_t b = row_bits(iw);
    copy_rows(iw, b);
    return b;
  };
  // sqrt(1 - l^2 - m^2), phase_correction.cu:56-64, always the same bits (l
  // is read where it is needed rather than held across the transforms)
  auto root_of = [&](int m) {
    const double l = active ? J.ltab[n] : 0.0;
    const double mm = J.mtab[m];
    return __dsqrt_rn(__dsub_rn(1.0, __dadd_rn(__dmul_rn(l, l), __dmul_rn(mm, mm))));
  };
  int iw = prev_plane(nw);
  uint32_t rows8 = iw >= 0 ? load_rows(iw) : 0u;
  // the per-pixel steps into TMEM
  const double dwstep = __dmul_rn(twopi, J.dw);
#pragma unroll
  for (int q = 0; q < kVpt; q++) {
    const int m = t + q * G;
    double sn = 0.0, cs = 1.0;
    if (phase) sincos(__dmul_rn(dwstep, __dsub_rn(root_of(m), 1.0)), &sn, &cs);
    uint32_t w4[4];
    tm::split(cs, w4[0], w4[1]);
    tm::split(sn, w4[2], w4[3]);
    tm::st4(taddr + 8 * q + 4, w4);
    tm::wait_st4(w4);
  }
  bool first = true;
  int prev = iw;
  while (iw >= 0) {
    cp_async_wait<0>();  // this thread's rows of plane iw have landed
    const int nxt = prev_plane(iw);
    const uint32_t next8 = nxt >= 0 ? row_bits(nxt) : 0u;
    // first pass: the thread's own rows (zero where not copied)
    Cx<T> v[8];
#pragma unroll
    for (int r = 0; r < 8; r++)
      v[r] = ((rows8 >> r) & 1u) ? lds<T>(buf, t + r * G) : Cx<T>{(T)0, (T)0};
    __syncthreads();  // every row is read: the buffer is writable
    first_pass_from_regs<T>(buf, t, v);
    Cx<T> x[kVpt];
    fft_tail_to_regs<T, LOGN>(buf, t, J.tw, x);
    __syncthreads();  // every thread has read the buffer
    if (nxt >= 0) copy_rows(nxt, next8);
    rows8 = next8;
    const int gap = prev - iw;
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      uint32_t a4[4];
      if (first) {
        tm::split((double)x[q].re, a4[0], a4[1]);
        tm::split((double)x[q].im, a4[2], a4[3]);
      } else {
        uint32_t r8[8];
        tm::ld8(taddr + 8 * q, r8);
        tm::wait_ld8(r8);
        double ar = tm::join(r8[0], r8[1]);
        double ai = tm::join(r8[2], r8[3]);
        const double sr = tm::join(r8[4], r8[5]);
        const double si = tm::join(r8[6], r8[7]);
        for (int g2 = 1; g2 < gap; g2++) {  // planes without data in between
          const double tr = fma(ar, sr, -ai * si);
          ai = fma(ar, si, ai * sr);
          ar = tr;
        }
        const double nr = fma(ar, sr, fma(-ai, si, (double)x[q].re));
        const double ni = fma(ar, si, fma(ai, sr, (double)x[q].im));
        tm::split(nr, a4[0], a4[1]);
        tm::split(ni, a4[2], a4[3]);
      }
      tm::st4(taddr + 8 * q, a4);
      tm::wait_st4(a4);
    }
    first = false;
    prev = iw;
    iw = nxt;
  }
  // image = norm * P * sum, P the factor of the lowest plane with data
  const double cw = __dmul_rn(twopi, __dadd_rn(J.wmin, __dmul_rn((double)(J.w_first + prev), J.dw)));
#pragma unroll
  for (int q = 0; q < kVpt; q++) {
    const int m = t + q * G;
    double re = 0.0, im = 0.0;
    if (!first) {
      uint32_t a4[4];
      tm::ld4(taddr + 8 * q, a4);
      tm::wait_ld4(a4);
      const double ar = tm::join(a4[0], a4[1]);
      const double ai = tm::join(a4[2], a4[3]);
      double pr = 1.0, pi = 0.0;
      if (phase) {
        const double root = root_of(m);
        double sn, cs;
        sincos(__dmul_rn(cw, __dsub_rn(root, 1.0)), &sn, &cs);
        const double amp = J.dwnorm * root;
        pr = cs * amp;
        pi = sn * amp;
      }
      re = J.norm * fma(ar, pr, -ai * pi);
      im = J.norm * fma(ar, pi, ai * pr);
    }
    if (active) {
      J.img_re[(uint64_t)m * nx + n] = re;
      J.img_im[(uint64_t)m * nx + n] = im;
    }
  }
}

template <int LOGN> constexpr int tm_min_blocks() { return 1024 / block_threads<LOGN>(); }

template <typename T, int LOGN>
__global__ void __launch_bounds__(block_threads<LOGN>(), tm_min_blocks<LOGN>())
    k_fft_cols_tm(ColJob<T> J) {
  constexpr int G = (1 << LOGN) / kVpt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto *s = reinterpret_cast<typename V2<T>::t *>(smem_raw);
  const int rpc = blockDim.x / G;
  // the TMEM address slot sits after the column buffers
  uint32_t *slot =
      reinterpret_cast<uint32_t *>(smem_raw + cols_tm_smem_bytes<T, LOGN>(rpc) - 16);
  constexpr uint32_t ncols = tm_cols(block_threads<LOGN>());
  const int warp = threadIdx.x / 32;
  if (warp == 0) {
    tm::alloc(slot, ncols);
    tm::relinquish();
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tbase = *slot;
  const uint32_t taddr = tbase + ((uint32_t)(32 * (warp % 4)) << 16) + (uint32_t)(warp / 4) * 64u;
  for (uint32_t base = blockIdx.x * rpc; base < (uint32_t)J.nx; base += gridDim.x * rpc) {
    fft_col_unit_tm<T, LOGN>(s, base, J, taddr);
    __syncthreads();  // the column buffers are rewritten for the next columns
  }
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    tm::dealloc(tbase, ncols);
  }
}

// The TMEM column pass over the jobs col_jobs[lo..hi-1] of a batch (all of FFT
// length 2^LOGN along y): the column groups of the k-th listed job are
// col_units[k] .. col_units[k+1]-1.
template <typename T, int LOGN>
__global__ void __launch_bounds__(block_threads<LOGN>(), tm_min_blocks<LOGN>())
    k_fft_cols_tm_multi(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ col_jobs,
                        int lo, int hi, const uint32_t *__restrict__ col_units,
                        const uint32_t *__restrict__ rowmask, const uint32_t *__restrict__ counts) {
  constexpr int G = (1 << LOGN) / kVpt;
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto *s = reinterpret_cast<V *>(smem_raw);
  const int rpc = blockDim.x / G;
  uint32_t *slot =
      reinterpret_cast<uint32_t *>(smem_raw + cols_tm_smem_bytes<T, LOGN>(rpc) - 16);
  constexpr uint32_t ncols = tm_cols(block_threads<LOGN>());
  const int warp = threadIdx.x / 32;
  if (warp == 0) {
    tm::alloc(slot, ncols);
    tm::relinquish();
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tbase = *slot;
  const uint32_t taddr = tbase + ((uint32_t)(32 * (warp % 4)) << 16) + (uint32_t)(warp / 4) * 64u;
  const uint32_t u1 = col_units[hi];
  for (uint32_t u = col_units[lo] + blockIdx.x; u < u1; u += gridDim.x) {
    const int k = lo + batch_job_of(col_units + lo, hi - lo, u);
    const BatchJob &B = jobs[col_jobs[k]];
    ColJob<T> J;
    J.cube = (const V *)B.blocked;
    J.nx = B.g.nx;
    J.ny = B.g.ny;
    J.nw = B.g.nw;
    J.nty = B.g.nty;
    J.w_first = B.g.w_first;
    J.nw_total = B.g.nw_total > 0 ? B.g.nw_total : B.g.nw;
    J.rowmask = rowmask + B.mask_base;
    J.counts = counts + B.counts_base;
    J.tw = (const V *)B.tw_y;
    J.ltab = B.ltab;
    J.mtab = B.mtab;
    J.wmin = B.wmin;
    J.dw = B.dw_phase;
    J.dwnorm = B.dwnorm;
    J.norm = B.norm;
    J.phase_on = B.phase_on;
    J.img_re = B.img_re;
    J.img_im = B.img_im;
    fft_col_unit_tm<T, LOGN>(s, (u - col_units[k]) * (uint32_t)rpc, J, taddr);
    __syncthreads();
  }
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    tm::dealloc(tbase, ncols);
  }
}

// ---- The column pass, two columns per block ---------------------------------
//
// A block that transforms one column alternates between the shared-memory pipe
// (a pass's loads and stores) and the FP64 pipe (its butterflies), and the
// barriers between the passes keep its warps in step, so the two pipes mostly
// take turns.  Here one block of N/8 threads holds two columns, A and B, one
// pass apart: in each barrier interval it computes one pass of one column on
// values already in registers while it loads the inputs of the other column's
// next pass, so both pipes are busy at once.  Per plane (N = 1024..4096: a
// first pass, two radix-8 middle passes, a last pass of radix N/512 to
// registers; N = 8192, FP32 only: three middle passes and a radix-2 last
// pass) the intervals are
//   A: read rows | first pass | read | pass 2 | read | pass 3 | read | last + w-step
//   B: last + w-step (previous plane) | read rows | first pass | read | ... | read
// with a barrier after each interval from the second to the last but one (the
// first two and the last touch no shared memory the other threads use next).
// The first pass's inputs (the plane's touched rows) come from the cube
// straight into registers; the next plane's rows are prefetched into L2 a
// plane ahead.  Each thread holds 16 pixels' running sums and w-steps in TMEM
// (8 of each column): a block of N/8 threads allocates N/8 TMEM columns with
// FP64 state (all 512 of its SM at N = 4096), N/16 with FP32 state.

// v[r] *= w1^r (r = 1..7), the powers formed from w1 as in pass_twiddles.
template <typename T>
__device__ __forceinline__ void twiddle8(Cx<T> (&v)[8], typename V2<T>::t a) {
  const Cx<T> w1 = {a.x, a.y};
  const Cx<T> w2 = cmul<T>(w1, w1.re, w1.im);
  const Cx<T> w3 = cmul<T>(w1, w2.re, w2.im);
  const Cx<T> w4 = cmul<T>(w2, w2.re, w2.im);
  v[1] = cmul<T>(v[1], w1.re, w1.im);
  v[2] = cmul<T>(v[2], w2.re, w2.im);
  v[3] = cmul<T>(v[3], w3.re, w3.im);
  v[4] = cmul<T>(v[4], w4.re, w4.im);
  const Cx<T> w5 = cmul<T>(w1, w4.re, w4.im);
  v[5] = cmul<T>(v[5], w5.re, w5.im);
  const Cx<T> w6 = cmul<T>(w2, w4.re, w4.im);
  v[6] = cmul<T>(v[6], w6.re, w6.im);
  const Cx<T> w7 = cmul<T>(w3, w4.re, w4.im);
  v[7] = cmul<T>(v[7], w7.re, w7.im);
}

// the inputs of a pass after the first: values t + r*G
template <typename T, int N>
__device__ __forceinline__ void pair_read(const typename V2<T>::t *s, int t, Cx<T> (&v)[8]) {
#pragma unroll
  for (int r = 0; r < 8; r++) v[r] = lds<T>(s, t + r * (N / 8));
}
// the first pass (stride 1): outputs to t*8 + r
template <typename T>
__device__ __forceinline__ void pair_first(typename V2<T>::t *s, int t, Cx<T> (&v)[8]) {
  Dft<T, 8>::run(v);
#pragma unroll
  for (int r = 0; r < 8; r++) sts<T>(s, t * 8 + r, v[r]);
}
// a middle pass of stride Ns (butterfly t, twiddle w1 = a)
template <typename T>
__device__ __forceinline__ void pair_mid(typename V2<T>::t *s, int t, int Ns,
                                         typename V2<T>::t a, Cx<T> (&v)[8]) {
  twiddle8<T>(v, a);
  Dft<T, 8>::run(v);
  const int jm = t & (Ns - 1);
  const int idx = (t - jm) * 8 + jm;
#pragma unroll
  for (int r = 0; r < 8; r++) sts<T>(s, idx + r * Ns, v[r]);
}
// The last pass, of radix R and stride N/R: the thread's B = 8/R butterflies
// j = t + b*G take v[b + B*r] (the values t + (b + B*r)*G that pair_read
// brought in) and leave there the transform's value at t + (b + B*r)*G.
// twl = the thread's first twiddle entry, tw + (N/R - 1) + t.
template <typename T, int R>
__device__ __forceinline__ void pair_last(const typename V2<T>::t *__restrict__ twl, int G,
                                          Cx<T> (&v)[8]) {
  if constexpr (R == 8) {
    twiddle8<T>(v, __ldg(twl));
    Dft<T, 8>::run(v);
  } else {
    constexpr int B = 8 / R;
#pragma unroll
    for (int b = 0; b < B; b++) {
      Cx<T> u[R], w[R];
#pragma unroll
      for (int r = 0; r < R; r++) u[r] = v[b + B * r];
      pass_twiddles<T, R>(twl + b * G, w);
#pragma unroll
      for (int r = 1; r < R; r++) u[r] = cmul<T>(u[r], w[r].re, w[r].im);
      Dft<T, R>::run(u);
#pragma unroll
      for (int r = 0; r < R; r++) v[b + B * r] = u[r];
    }
  }
}

// TMEM words a pixel's running sum and w-step take in the two-column pass: FP64
// complex pairs (8) for the FP64 transform, FP32 pairs (4) for the FP32 one.
// The FP32 recurrence adds ~4e-7 relative error over 32 planes (modelled at
// 4096^2 x 32, w from -7.5e3 to 7.8e3 wavelengths), within the FP32
// transform's own; with half the TMEM, two 4096-point blocks share an SM.
template <typename T> __host__ __device__ constexpr uint32_t pair_pixel_words() {
  return sizeof(T) == 8 ? 8u : 4u;
}

// One w-plane's transform x into the running sums of one column's 8 pixels
// (TMEM at tcol: pixel q at tcol + W*q, W = pair_pixel_words, sum then step):
// sum = sum*step^gap + x, or sum = x for the first plane.  FP64 state: two
// pixels per TMEM access; FP32 state: four.
template <typename T>
__device__ __forceinline__ void pair_horner(uint32_t tcol, const Cx<T> (&x)[8], bool first,
                                            int gap) {
  if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int q = 0; q < kVpt; q += 4) {
      uint32_t r[16];
      if (first) {
#pragma unroll
        for (int h = 0; h < 4; h++) {
          r[4 * h + 0] = __float_as_uint(x[q + h].re);
          r[4 * h + 1] = __float_as_uint(x[q + h].im);
        }
        // the steps are kept: write the sums only
#pragma unroll
        for (int h = 0; h < 4; h++) {
          uint32_t a2[2] = {r[4 * h + 0], r[4 * h + 1]};
          tm::st2(tcol + 4 * (q + h), a2);
          tm::wait_st2(a2);
        }
      } else {
        tm::ld16(tcol + 4 * q, r);
        tm::wait_ld16(r);
#pragma unroll
        for (int h = 0; h < 4; h++) {
          float ar = __uint_as_float(r[4 * h + 0]);
          float ai = __uint_as_float(r[4 * h + 1]);
          const float sr = __uint_as_float(r[4 * h + 2]);
          const float si = __uint_as_float(r[4 * h + 3]);
          for (int g2 = 1; g2 < gap; g2++) {  // planes without data in between
            const float tr = fmaf(ar, sr, -ai * si);
            ai = fmaf(ar, si, ai * sr);
            ar = tr;
          }
          r[4 * h + 0] = __float_as_uint(fmaf(ar, sr, fmaf(-ai, si, (float)x[q + h].re)));
          r[4 * h + 1] = __float_as_uint(fmaf(ar, si, fmaf(ai, sr, (float)x[q + h].im)));
        }
        tm::st16(tcol + 4 * q, r);
        tm::wait_st16(r);
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < kVpt; q += 2) {
      uint32_t a4[2][4];
      if (first) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
          tm::split((double)x[q + h].re, a4[h][0], a4[h][1]);
          tm::split((double)x[q + h].im, a4[h][2], a4[h][3]);
        }
      } else {
        uint32_t r[16];
        tm::ld16(tcol + 8 * q, r);
        tm::wait_ld16(r);
#pragma unroll
        for (int h = 0; h < 2; h++) {
          double ar = tm::join(r[8 * h + 0], r[8 * h + 1]);
          double ai = tm::join(r[8 * h + 2], r[8 * h + 3]);
          const double sr = tm::join(r[8 * h + 4], r[8 * h + 5]);
          const double si = tm::join(r[8 * h + 6], r[8 * h + 7]);
          for (int g2 = 1; g2 < gap; g2++) {  // planes without data in between
            const double tr = fma(ar, sr, -ai * si);
            ai = fma(ar, si, ai * sr);
            ar = tr;
          }
          const double nr = fma(ar, sr, fma(-ai, si, (double)x[q + h].re));
          const double ni = fma(ar, si, fma(ai, sr, (double)x[q + h].im));
          tm::split(nr, a4[h][0], a4[h][1]);
          tm::split(ni, a4[h][2], a4[h][3]);
        }
      }
      tm::st4(tcol + 8 * q, a4[0]);
      tm::st4(tcol + 8 * q + 8, a4[1]);
      tm::wait_st4x2(a4[0], a4[1]);
    }
  }
}

// Columns nA and nA + 1 (nA even) of one job; taddr is the thread's TMEM base
// (A's pixels at +0, B's at +8W, W = pair_pixel_words).  The w1 twiddles of the
// thread's butterflies are read where they are used (L1 hits).
// SPLIT: one column nA of length 2N (8192), as two transforms of length N:
// with x_lo = x[j], x_hi = x[j + N] (j < N), A transforms x_lo + x_hi (its
// outputs are the column's even rows 2k) and B transforms
// (x_lo - x_hi)·exp(+2 pi i j / 2N) (the odd rows 2k + 1) -- the first pass
// of a decimation-in-frequency radix-2 step, done as the rows are read.
template <typename T, int LOGN, bool SPLIT = false>
__device__ __forceinline__ void fft_col_pair_tm(typename V2<T>::t *sA, typename V2<T>::t *sB,
                                                uint32_t nA, const ColJob<T> &J, uint32_t taddr) {
  constexpr int LF = SPLIT ? LOGN - 1 : LOGN;           // length of the transforms run
  static_assert(LF >= 10 && LF <= 13, "the pair schedule has two or three middle passes");
  static_assert(!SPLIT || LOGN == 13, "the split form is for 8192-point columns");
  constexpr int N = 1 << LF, G = N / kVpt;
  constexpr int NMID = LF <= 12 ? 2 : 3;                // radix-8 passes after the first
  constexpr int NSL = NMID == 2 ? 512 : 4096;           // stride of the last pass
  constexpr int LASTR = N / NSL;                        // its radix (2, 4 or 8)
  constexpr int CB = col_block<T>();
  using V = typename V2<T>::t;
  const int t = threadIdx.x;
  const int nx = J.nx, ny = J.ny, nw = J.nw, nty = J.nty;
  const uint32_t *__restrict__ counts = J.counts;
  const bool phase = J.phase_on && J.nw_total > 1;
  const double twopi = 2.0 * kPi;  // exact doubling of the reference's pi
  auto prev_plane = [&](int iw) {   // planes without data add exact zeros
    do { iw--; } while (iw >= 0 && counts[1 + iw] == 0);
    return iw;
  };
  // bit q: whether row t + q*G of plane iw was touched (the same for A and B);
  // SPLIT: bit 8 + q for row t + q*G + N
  auto row_bits = [&](int iw) {
    const uint32_t *__restrict__ mask = J.rowmask + (uint64_t)iw * nty;
    uint32_t bits = 0;
#pragma unroll
    for (int q = 0; q < (SPLIT ? 2 * kVpt : kVpt); q++) {
      const int k = t + q * G;
      bits |= ((__ldg(mask + (k >> 5)) >> (k & 31)) & 1u) << q;
    }
    return bits;
  };
  // the touched rows t + q*G of plane iw of column n (zero elsewhere)
  auto read_rows = [&](int iw, uint32_t bits, uint32_t n, Cx<T>(&v)[8]) {
    const V *col = J.cube + blocked_index<T>(iw, 0, n, nx, ny);
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      v[q] = {(T)0, (T)0};
      if ((bits >> q) & 1u) {
        const V x = __ldg(col + (uint64_t)(t + q * G) * CB);
        v[q] = {x.x, x.y};
      }
    }
  };
  // SPLIT: transform c's inputs (A: c = 0, B: c = 1) from the rows t + q*G
  // and t + q*G + N of plane iw (read twice, once for each: the second read
  // hits the caches)
  auto read_half = [&](int iw, uint32_t bits, int c, Cx<T>(&v)[8]) {
    const V *col = J.cube + blocked_index<T>(iw, 0, nA, nx, ny);
    typename V2<T>::t wt;
    if (c) wt = __ldg(J.tw + (N - 1) + t);  // exp(+2 pi i t / 2N), the 2N-point table's last pass
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      Cx<T> lo = {(T)0, (T)0}, hi = {(T)0, (T)0};
      if ((bits >> q) & 1u) {
        const V x = __ldg(col + (uint64_t)(t + q * G) * CB);
        lo = {x.x, x.y};
      }
      if ((bits >> (kVpt + q)) & 1u) {
        const V x = __ldg(col + (uint64_t)(t + q * G + N) * CB);
        hi = {x.x, x.y};
      }
      if (c == 0) {
        v[q] = cadd(lo, hi);
      } else {
        // exp(+2 pi i (t + q*G) / 2N) = exp(+2 pi i q / 16) * exp(+2 pi i t / 2N)
        const Cx<T> d = w16<T>(csub(lo, hi), q);
        v[q] = cmul<T>(d, wt.x, wt.y);
      }
    }
  };
  // the same rows into L2 (pairs: one 32-byte sector holds both columns'
  // values; SPLIT: both halves of the column)
  auto prefetch_rows = [&](int iw, uint32_t bits) {
    const V *col = J.cube + blocked_index<T>(iw, 0, nA, nx, ny);
#pragma unroll
    for (int q = 0; q < (SPLIT ? 2 * kVpt : kVpt); q++)
      if ((bits >> q) & 1u) prefetch_l2(col + (uint64_t)(t + q * G) * CB);
  };
  // the pixel of transform c's value q: (column, row)
  auto pix_col = [&](int c) { return SPLIT ? nA : nA + (uint32_t)c; };
  auto pix_row = [&](int c, int q) { return SPLIT ? 2 * (t + q * G) + c : t + q * G; };
  // sqrt(1 - l^2 - m^2), phase_correction.cu:56-64
  auto root_of = [&](uint32_t n, int m) {
    const double l = J.ltab[n];
    const double mm = J.mtab[m];
    return __dsqrt_rn(__dsub_rn(1.0, __dadd_rn(__dmul_rn(l, l), __dmul_rn(mm, mm))));
  };
  int iw = prev_plane(nw);
  uint32_t bits = iw >= 0 ? row_bits(iw) : 0u;
  // the per-pixel steps into TMEM
  const double dwstep = __dmul_rn(twopi, J.dw);
  // the thread's twiddle entries, formed where used (fewer live registers)
  auto tw_mid = [&](int Ns) { return J.tw + (Ns - 1) + (t & (Ns - 1)); };
  auto twl = [&] { return J.tw + (NSL - 1) + t; };
  constexpr uint32_t PW = pair_pixel_words<T>(), tB = 8 * PW;  // column B's TMEM offset
#pragma unroll
  for (int c = 0; c < 2; c++) {
#pragma unroll
    for (int q = 0; q < kVpt; q++) {
      double sn = 0.0, cs = 1.0;
      if (phase)
        sincos(__dmul_rn(dwstep, __dsub_rn(root_of(pix_col(c), pix_row(c, q)), 1.0)), &sn, &cs);
      if constexpr (PW == 8) {
        uint32_t w4[4];
        tm::split(cs, w4[0], w4[1]);
        tm::split(sn, w4[2], w4[3]);
        tm::st4(taddr + tB * c + PW * q + 4, w4);
        tm::wait_st4(w4);
      } else {
        uint32_t w2[2] = {__float_as_uint((float)cs), __float_as_uint((float)sn)};
        tm::st2(taddr + tB * c + PW * q + 2, w2);
        tm::wait_st2(w2);
      }
    }
  }
  Cx<T> vA[8], vB[8];
  bool first = true, b_pending = false, b_first = true;
  int prev = iw, b_gap = 0;
  while (iw >= 0) {
    // A: the plane's rows | B: last pass and w-step of the previous plane
    if constexpr (SPLIT)
      read_half(iw, bits, 0, vA);
    else
      read_rows(iw, bits, nA, vA);
    const int nxt = prev_plane(iw);
    const uint32_t nbits = nxt >= 0 ? row_bits(nxt) : 0u;
    if (b_pending) {
      pair_last<T, LASTR>(twl(), G, vB);
      pair_horner<T>(taddr + tB, vB, b_first, b_gap);
    }
    // A: first pass | B: the plane's rows
    if constexpr (SPLIT)
      read_half(iw, bits, 1, vB);
    else
      read_rows(iw, bits, nA + 1, vB);
    pair_first<T>(sA, t, vA);
    if (nxt >= 0) prefetch_rows(nxt, nbits);
    __syncthreads();
    // A: read | B: first pass
    pair_read<T, N>(sA, t, vA);
    pair_first<T>(sB, t, vB);
    __syncthreads();
    // the middle passes, of strides 8, 64 (, 512): A computes while B reads,
    // then A reads while B computes
#pragma unroll
    for (int mp = 0, Ns = 8; mp < NMID; mp++, Ns *= 8) {
      pair_read<T, N>(sB, t, vB);
      pair_mid<T>(sA, t, Ns, __ldg(tw_mid(Ns)), vA);
      __syncthreads();
      pair_read<T, N>(sA, t, vA);
      pair_mid<T>(sB, t, Ns, __ldg(tw_mid(Ns)), vB);
      __syncthreads();
    }
    // A: last pass and w-step | B: read (its last pass runs with the next plane's rows)
    pair_read<T, N>(sB, t, vB);
    pair_last<T, LASTR>(twl(), G, vA);
    const int gap = prev - iw;
    pair_horner<T>(taddr, vA, first, gap);
    b_pending = true;
    b_first = first;
    b_gap = gap;
    first = false;
    prev = iw;
    iw = nxt;
    bits = nbits;
  }
  if (b_pending) {
    pair_last<T, LASTR>(twl(), G, vB);
    pair_horner<T>(taddr + tB, vB, b_first, b_gap);
  }
  // image = norm * P * sum, P the factor of the lowest plane with data
  const double cw = __dmul_rn(twopi, __dadd_rn(J.wmin, __dmul_rn((double)(J.w_first + prev), J.dw)));
  const bool vec = ((reinterpret_cast<uintptr_t>(J.img_re) | reinterpret_cast<uintptr_t>(J.img_im)) &
                    15u) == 0;
#pragma unroll
  for (int q = 0; q < kVpt; q++) {
    double re[2] = {0.0, 0.0}, im[2] = {0.0, 0.0};
    if (!first) {
#pragma unroll
      for (int c = 0; c < 2; c++) {
        double ar, ai;
        if constexpr (PW == 8) {
          uint32_t a4[4];
          tm::ld4(taddr + tB * c + PW * q, a4);
          tm::wait_ld4(a4);
          ar = tm::join(a4[0], a4[1]);
          ai = tm::join(a4[2], a4[3]);
        } else {
          uint32_t a2[2];
          tm::ld2(taddr + tB * c + PW * q, a2);
          tm::wait_ld2(a2);
          ar = (double)__uint_as_float(a2[0]);
          ai = (double)__uint_as_float(a2[1]);
        }
        double pr = 1.0, pi = 0.0;
        if (phase) {
          const double root = root_of(pix_col(c), pix_row(c, q));
          double sn, cs;
          sincos(__dmul_rn(cw, __dsub_rn(root, 1.0)), &sn, &cs);
          const double amp = J.dwnorm * root;
          pr = cs * amp;
          pi = sn * amp;
        }
        re[c] = J.norm * fma(ar, pr, -ai * pi);
        im[c] = J.norm * fma(ar, pi, ai * pr);
      }
    }
    if constexpr (SPLIT) {  // rows 2k and 2k + 1 of one column
#pragma unroll
      for (int c = 0; c < 2; c++) {
        const uint64_t o = (uint64_t)pix_row(c, q) * nx + nA;
        J.img_re[o] = re[c];
        J.img_im[o] = im[c];
      }
      continue;
    }
    const uint64_t o = (uint64_t)(t + q * G) * nx + nA;
    if (vec) {
      *reinterpret_cast<double2 *>(J.img_re + o) = make_double2(re[0], re[1]);
      *reinterpret_cast<double2 *>(J.img_im + o) = make_double2(im[0], im[1]);
    } else {
      J.img_re[o] = re[0];
      J.img_re[o + 1] = re[1];
      J.img_im[o] = im[0];
      J.img_im[o + 1] = im[1];
    }
  }
}

template <typename T, int LOGN>
__host__ __device__ constexpr size_t cols_pair_smem_bytes() {
  return 2 * (size_t)(1 << LOGN) * sizeof(typename V2<T>::t) + 16;
}

// TMEM columns a pair block of `threads` threads allocates: 16 pixels x W
// words per warp of a lane quarter.
template <typename T> __host__ __device__ constexpr uint32_t pair_tm_cols(int threads) {
  return (uint32_t)(threads / 32 / 4) * 16u * pair_pixel_words<T>();
}

// One job's column pass, column pairs (nx / 2 of them) over a persistent grid.
// Blocks of G threads, as many per SM as their TMEM allows (512 / the columns
// a block allocates): 128 registers a thread for the FP64 pass, 64 for the
// FP32 pass (twice the blocks).
template <typename T, int LOGN> constexpr int pair_min_blocks() {
  return (int)(512u / pair_tm_cols<T>(group_threads<LOGN>()));
}

template <typename T, int LOGN>
__global__ void __launch_bounds__(group_threads<LOGN>(), pair_min_blocks<T, LOGN>())
    k_fft_cols_pair(ColJob<T> J) {
  constexpr int N = 1 << LOGN;
  constexpr uint32_t ncols = pair_tm_cols<T>(group_threads<LOGN>());
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *sA = reinterpret_cast<V *>(smem_raw);
  V *sB = sA + N;
  uint32_t *slot = reinterpret_cast<uint32_t *>(smem_raw + cols_pair_smem_bytes<T, LOGN>() - 16);
  const int warp = threadIdx.x / 32;
  if (warp == 0) {
    tm::alloc(slot, ncols);
    tm::relinquish();
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tbase = *slot;
  const uint32_t taddr = tbase + ((uint32_t)(32 * (warp % 4)) << 16) +
                         (uint32_t)(warp / 4) * 16u * pair_pixel_words<T>();
  const uint32_t pairs = (uint32_t)J.nx / 2u;
  for (uint32_t p = blockIdx.x; p < pairs; p += gridDim.x) {
    fft_col_pair_tm<T, LOGN>(sA, sB, 2u * p, J, taddr);
    __syncthreads();  // the column buffers are rewritten for the next pair
  }
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    tm::dealloc(tbase, ncols);
  }
}

// One job's column pass at 8192 points with FP64 state: each column split into
// two 4096-point transforms (even and odd rows) run one pass apart, columns
// over a persistent grid of one block per SM.
template <typename T, int LOGN>
__global__ void __launch_bounds__(group_threads<LOGN - 1>(), 1) k_fft_cols_split(ColJob<T> J) {
  constexpr int NH = 1 << (LOGN - 1);
  constexpr uint32_t ncols = pair_tm_cols<T>(group_threads<LOGN - 1>());
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *sA = reinterpret_cast<V *>(smem_raw);
  V *sB = sA + NH;
  uint32_t *slot =
      reinterpret_cast<uint32_t *>(smem_raw + cols_pair_smem_bytes<T, LOGN - 1>() - 16);
  const int warp = threadIdx.x / 32;
  if (warp == 0) {
    tm::alloc(slot, ncols);
    tm::relinquish();
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tbase = *slot;
  const uint32_t taddr = tbase + ((uint32_t)(32 * (warp % 4)) << 16) +
                         (uint32_t)(warp / 4) * 16u * pair_pixel_words<T>();
  for (uint32_t n = blockIdx.x; n < (uint32_t)J.nx; n += gridDim.x) {
    fft_col_pair_tm<T, LOGN, true>(sA, sB, n, J, taddr);
    __syncthreads();  // the buffers are rewritten for the next column
  }
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    tm::dealloc(tbase, ncols);
  }
}

// The pair pass over the jobs col_jobs[lo..hi-1] of a batch (all of FFT length
// 2^LOGN along y): the k-th listed job's columns are the global columns
// col_units[k]*rpc .. col_units[k+1]*rpc - 1 (each job's count even), taken
// two at a time.
template <typename T, int LOGN>
__global__ void __launch_bounds__(group_threads<LOGN>(), pair_min_blocks<T, LOGN>())
    k_fft_cols_pair_multi(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ col_jobs,
                          int lo, int hi, const uint32_t *__restrict__ col_units, int rpc,
                          const uint32_t *__restrict__ rowmask, const uint32_t *__restrict__ counts) {
  constexpr int N = 1 << LOGN;
  constexpr uint32_t ncols = pair_tm_cols<T>(group_threads<LOGN>());
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  V *sA = reinterpret_cast<V *>(smem_raw);
  V *sB = sA + N;
  uint32_t *slot = reinterpret_cast<uint32_t *>(smem_raw + cols_pair_smem_bytes<T, LOGN>() - 16);
  const int warp = threadIdx.x / 32;
  if (warp == 0) {
    tm::alloc(slot, ncols);
    tm::relinquish();
  }
  tm::fence_before();
  __syncthreads();
  tm::fence_after();
  const uint32_t tbase = *slot;
  const uint32_t taddr = tbase + ((uint32_t)(32 * (warp % 4)) << 16) +
                         (uint32_t)(warp / 4) * 16u * pair_pixel_words<T>();
  const uint32_t p0 = col_units[lo] * (uint32_t)rpc / 2u, p1 = col_units[hi] * (uint32_t)rpc / 2u;
  // the pair's job, in shared memory (its fields are read where used, not held
  // in registers across the transform)
  __shared__ ColJob<T> sJ;
  __shared__ uint32_t sA0;
  for (uint32_t p = p0 + blockIdx.x; p < p1; p += gridDim.x) {
    if (threadIdx.x == 0) {
      const int k = lo + batch_job_of(col_units + lo, hi - lo, 2u * p / (uint32_t)rpc);
      const BatchJob &B = jobs[col_jobs[k]];
      ColJob<T> &J = sJ;
      sA0 = 2u * p - col_units[k] * (uint32_t)rpc;
      J.cube = (const V *)B.blocked;
      J.nx = B.g.nx;
      J.ny = B.g.ny;
      J.nw = B.g.nw;
      J.nty = B.g.nty;
      J.w_first = B.g.w_first;
      J.nw_total = B.g.nw_total > 0 ? B.g.nw_total : B.g.nw;
      J.rowmask = rowmask + B.mask_base;
      J.counts = counts + B.counts_base;
      J.tw = (const V *)B.tw_y;
      J.ltab = B.ltab;
      J.mtab = B.mtab;
      J.wmin = B.wmin;
      J.dw = B.dw_phase;
      J.dwnorm = B.dwnorm;
      J.norm = B.norm;
      J.phase_on = B.phase_on;
      J.img_re = B.img_re;
      J.img_im = B.img_im;
    }
    __syncthreads();
    fft_col_pair_tm<T, LOGN>(sA, sB, sA0, sJ, taddr);
    __syncthreads();  // the buffers and the job are rewritten for the next pair
  }
  tm::fence_before();
  __syncthreads();
  if (warp == 0) {
    tm::fence_after();
    tm::dealloc(tbase, ncols);
  }
}

// One job's column pass (the plan): the job as a kernel parameter.
template <typename T, int LOGN, bool DB, bool RECUR, int PP>
__global__ void __launch_bounds__(block_threads<LOGN>(), col_min_blocks<T, LOGN, PP>())
    k_fft_cols_image(ColJob<T> J) {
  constexpr int G = (1 << LOGN) / kVpt;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto *s = reinterpret_cast<typename V2<T>::t *>(smem_raw);
  const int rpc = blockDim.x / G;
  for (uint32_t base = blockIdx.x * rpc; base < (uint32_t)J.nx; base += gridDim.x * rpc)
    fft_col_unit<T, LOGN, DB, RECUR, PP>(s, base, J);
}

// Column pass over the jobs col_jobs[lo..hi-1] of a batch (all of FFT length 2^LOGN
// along y): the column groups of the k-th listed job are col_units[k] ..
// col_units[k+1]-1.
template <typename T, int LOGN, bool DB, bool RECUR, int PP>
__global__ void __launch_bounds__(block_threads<LOGN>(), col_min_blocks<T, LOGN, PP>())
    k_fft_cols_multi(const BatchJob *__restrict__ jobs, const uint32_t *__restrict__ col_jobs,
                     int lo, int hi, const uint32_t *__restrict__ col_units,
                     const uint32_t *__restrict__ rowmask, const uint32_t *__restrict__ counts) {
  constexpr int G = (1 << LOGN) / kVpt;
  using V = typename V2<T>::t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  auto *s = reinterpret_cast<V *>(smem_raw);
  const int rpc = blockDim.x / G;
  const uint32_t u1 = col_units[hi];
  for (uint32_t u = col_units[lo] + blockIdx.x; u < u1; u += gridDim.x) {
    const int k = lo + batch_job_of(col_units + lo, hi - lo, u);
    const BatchJob &B = jobs[col_jobs[k]];
    ColJob<T> J;
    J.cube = (const V *)B.blocked;
    J.nx = B.g.nx;
    J.ny = B.g.ny;
    J.nw = B.g.nw;
    J.nty = B.g.nty;
    J.w_first = B.g.w_first;
    J.nw_total = B.g.nw_total > 0 ? B.g.nw_total : B.g.nw;
    J.rowmask = rowmask + B.mask_base;
    J.counts = counts + B.counts_base;
    J.tw = (const V *)B.tw_y;
    J.ltab = B.ltab;
    J.mtab = B.mtab;
    J.wmin = B.wmin;
    J.dw = B.dw_phase;
    J.dwnorm = B.dwnorm;
    J.norm = B.norm;
    J.phase_on = B.phase_on;
    J.img_re = B.img_re;
    J.img_im = B.img_im;
    fft_col_unit<T, LOGN, DB, RECUR, PP>(s, (u - col_units[k]) * (uint32_t)rpc, J);
  }
}

// Compacts the row masks of every job into its list of touched (plane, row)
// ids and per-plane counts: counts[0] = rows, counts[1 + w] = touched rows of
// plane w (at the job's counts_base).
__global__ void k_row_list(const BatchJob *__restrict__ jobs, int njobs,
                           const uint64_t *__restrict__ mask_base, uint64_t nwords,
                           const uint32_t *__restrict__ rowmask, uint32_t *__restrict__ rowlist,
                           uint32_t *__restrict__ counts) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nwords;
       i += gridDim.x * (uint64_t)blockDim.x) {
    uint32_t bits = rowmask[i];
    if (!bits) continue;
    const int j = batch_job_of(mask_base, njobs, i);
    const BatchJob &J = jobs[j];
    const uint64_t li = i - J.mask_base;
    const uint32_t nty = (uint32_t)J.g.nty, ny = (uint32_t)J.g.ny;
    const uint32_t w = (uint32_t)(li / nty), band = (uint32_t)(li % nty);
    const uint32_t c = __popc(bits);
    uint32_t slot = atomicAdd(&counts[J.counts_base], c);
    atomicAdd(&counts[J.counts_base + 1 + w], c);
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const uint32_t k = band * 32 + b;
      if (k < ny) rowlist[J.list_base + slot] = w * ny + k;
      slot++;
    }
  }
}

// Row-pass units per job (groups of rows_per_block(logx) touched rows),
// exclusive prefix over the jobs; one thread (a few hundred jobs at most).
__global__ void k_fft_units(const BatchJob *__restrict__ jobs, int njobs,
                            const uint32_t *__restrict__ counts, uint32_t *__restrict__ fft_units) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t acc = 0;
  for (int j = 0; j < njobs; j++) {
    fft_units[j] = acc;
    const uint32_t rpc = (uint32_t)fft_rows_per_block(jobs[j].logx);
    acc += (counts[jobs[j].counts_base] + rpc - 1) / rpc;
  }
  fft_units[njobs] = acc;
}

template <typename T, int LOGN>
size_t fft_smem(int rpc) {
  constexpr int N = 1 << LOGN;
  return (size_t)rpc * padded<T>(N) * sizeof(typename V2<T>::t);
}

// Longest transform of the multi-job (batch) kernels: 4096.
constexpr int kMultiMaxLog = 12;

template <typename T> ColJob<T> col_job(const BatchJob &B, const FftJobs &f) {
  using V = typename V2<T>::t;
  ColJob<T> J;
  J.cube = (const V *)B.blocked;
  J.nx = B.g.nx;
  J.ny = B.g.ny;
  J.nw = B.g.nw;
  J.nty = B.g.nty;
  J.w_first = B.g.w_first;
  J.nw_total = B.g.nw_total > 0 ? B.g.nw_total : B.g.nw;
  J.rowmask = f.rowmask + B.mask_base;
  J.counts = f.counts + B.counts_base;
  J.tw = (const V *)B.tw_y;
  J.ltab = B.ltab;
  J.mtab = B.mtab;
  J.wmin = B.wmin;
  J.dw = B.dw_phase;
  J.dwnorm = B.dwnorm;
  J.norm = B.norm;
  J.phase_on = B.phase_on;
  J.img_re = B.img_re;
  J.img_im = B.img_im;
  return J;
}

template <typename T, int LOGN>
int launch_rows(const FftJobs &f, const FftClass &c, cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  const int rpc = BT / G;
  const size_t sm = fft_smem<T, LOGN>(rpc);
  using V = typename V2<T>::t;
  if (f.one) {
    const BatchJob &B = *f.one;
    RICK_CUDA(cudaFuncSetAttribute(k_fft_rows<T, LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)sm));
    int per_sm = 0;
    RICK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fft_rows<T, LOGN>, BT, sm));
    RICK_LAUNCHED();
    k_fft_rows<T, LOGN><<<num_sms() * std::max(per_sm, 1), BT, sm, st>>>(
        (const V *)B.cube, (V *)B.blocked, B.g.nx, B.g.ny, B.g.nty, (B.g.ntx + 31) / 32,
        f.tilemask + B.tile_base, f.rowlist + B.list_base, f.counts + B.counts_base,
        (const V *)B.tw_x);
  } else {
    if constexpr (LOGN > kMultiMaxLog) {
      return set_error(RICK_ERR_INVALID_ARG, "batch FFT length above %d", 1 << kMultiMaxLog);
    } else {
      RICK_CUDA(cudaFuncSetAttribute(k_fft_rows_multi<T, LOGN>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      int per_sm = 0;
      RICK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fft_rows_multi<T, LOGN>,
                                                              BT, sm));
      RICK_LAUNCHED();
      k_fft_rows_multi<T, LOGN><<<num_sms() * std::max(per_sm, 1), BT, sm, st>>>(
          f.jobs, c.lo, c.hi, f.fft_units, f.tilemask, f.rowlist, f.counts);
    }
  }
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

template <typename T, int LOGN, bool DB, bool RECUR, int PP>
size_t cols_smem(int rpc) {
  return cols_smem_bytes<T, LOGN, DB, RECUR, PP>(rpc);
}

template <typename T, int LOGN, bool DB, bool RECUR, int PP>
int launch_cols_impl(const FftJobs &f, const FftClass &c, cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  const int rpc = BT / G;
  const size_t sm = cols_smem<T, LOGN, DB, RECUR, PP>(rpc);
  int per_sm = 0;
  if (f.one) {
    RICK_CUDA(cudaFuncSetAttribute(k_fft_cols_image<T, LOGN, DB, RECUR, PP>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    RICK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_fft_cols_image<T, LOGN, DB, RECUR, PP>, BT, sm));
    const int blocks = (int)std::min<uint64_t>(std::max<uint32_t>(c.units, 1),
                                               (uint64_t)num_sms() * std::max(per_sm, 1));
    RICK_LAUNCHED();
    k_fft_cols_image<T, LOGN, DB, RECUR, PP><<<blocks, BT, sm, st>>>(col_job<T>(*f.one, f));
  } else {
    // batch sizes (<= 4096) always fit double-buffered loads and the phase steps
    if constexpr (LOGN > kMultiMaxLog || !DB || !RECUR) {
      return set_error(RICK_ERR_INVALID_ARG, "batch FFT length above %d", 1 << kMultiMaxLog);
    } else {
      RICK_CUDA(cudaFuncSetAttribute(k_fft_cols_multi<T, LOGN, DB, RECUR, PP>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
      RICK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, k_fft_cols_multi<T, LOGN, DB, RECUR, PP>, BT, sm));
      const int blocks = (int)std::min<uint64_t>(std::max<uint32_t>(c.units, 1),
                                                 (uint64_t)num_sms() * std::max(per_sm, 1));
      RICK_LAUNCHED();
      k_fft_cols_multi<T, LOGN, DB, RECUR, PP><<<blocks, BT, sm, st>>>(
          f.jobs, f.col_jobs, c.lo, c.hi, f.col_units, f.rowmask, f.counts);
    }
  }
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

// Implementation choice of the column pass, for measurements: RICK_COLS_TMEM=0
// selects the register-resident kernels.
bool cols_tm_enabled() {
  static const bool on = [] {
    const char *e = getenv("RICK_COLS_TMEM");
    return !(e && e[0] == '0');
  }();
  return on;
}

// The column pass with the per-pixel state in TMEM (one job, or the jobs of a
// batch class).  The dynamic shared memory is padded so that shared memory,
// not the TMEM allocation, bounds the blocks per SM at 512 / (columns a block
// allocates): a further block could not allocate and would wait for one of
// the others to finish.
template <typename T, int LOGN>
int launch_cols_tm(const FftJobs &f, const FftClass &c, cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  const int rpc = BT / G;
  const int max_blocks = (int)(512u / tm_cols(BT));
  int dev = 0, smem_sm = 0, reserved = 0;
  RICK_CUDA(cudaGetDevice(&dev));
  RICK_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  RICK_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  size_t sm = cols_tm_smem_bytes<T, LOGN>(rpc);
  const size_t floor_b = (size_t)smem_sm / (size_t)(max_blocks + 1) + 1;
  if (sm + (size_t)reserved < floor_b) sm = floor_b - (size_t)reserved;
  sm = (sm + 15) & ~(size_t)15;
  const void *fn = f.one ? (const void *)k_fft_cols_tm<T, LOGN>
                         : (const void *)k_fft_cols_tm_multi<T, LOGN>;
  RICK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  // blocks per SM from the kernel's own needs: registers, shared memory, threads
  cudaFuncAttributes fa{};
  RICK_CUDA(cudaFuncGetAttributes(&fa, fn));
  const int regs_per_warp = ((std::max(fa.numRegs, 1) * 32 + 255) / 256) * 256;
  const int by_regs = 65536 / (regs_per_warp * (BT / 32));
  const int by_smem = (int)((size_t)smem_sm / (sm + (size_t)reserved));
  const int by_threads = 2048 / BT;
  const int per_sm = std::max(1, std::min({max_blocks, by_regs, by_smem, by_threads}));
  // a shared-memory carveout just large enough for those blocks: the rest of
  // the SM's 256 KB stays L1, which holds the FFT's twiddles (with the whole
  // carveout as shared memory, the mixed form's 8-byte column copies, cached
  // in L1, evicted them: its column pass ran 3.47 ms at 4096^2 x 32, 3.04 ms
  // with this carveout)
  const int pct = (int)std::min<size_t>(
      100, ((size_t)per_sm * (sm + (size_t)reserved) * 100 + (size_t)smem_sm - 1) / (size_t)smem_sm);
  RICK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  const int blocks = (int)std::min<uint64_t>(std::max<uint32_t>(c.units, 1),
                                             (uint64_t)num_sms() * per_sm);
  RICK_LAUNCHED();
  if (f.one) {
    k_fft_cols_tm<T, LOGN><<<blocks, BT, sm, st>>>(col_job<T>(*f.one, f));
  } else {
    k_fft_cols_tm_multi<T, LOGN><<<blocks, BT, sm, st>>>(f.jobs, f.col_jobs, c.lo, c.hi,
                                                         f.col_units, f.rowmask, f.counts);
  }
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

// Implementation choice of the 1024- to 4096-point column passes, for
// measurements: RICK_COLS_PAIR=0 selects the one-column TMEM kernel.
bool cols_pair_enabled() {
  static const bool on = [] {
    const char *e = getenv("RICK_COLS_PAIR");
    return !(e && e[0] == '0');
  }();
  return on;
}

// The two-column pass (one job, or the jobs of a batch class), for column
// lengths 1024..4096 (and 8192 for one FP32 job).  A block of G threads allocates G TMEM columns; its
// dynamic shared memory is padded so that shared memory, not the TMEM
// allocation, bounds the blocks per SM (a further block could not allocate).
template <typename T, int LOGN>
int launch_cols_pair(const FftJobs &f, const FftClass &c, cudaStream_t st) {
  constexpr int BT = group_threads<LOGN>();
  const int max_blocks = (int)(512u / pair_tm_cols<T>(BT));
  int dev = 0, smem_sm = 0, reserved = 0;
  RICK_CUDA(cudaGetDevice(&dev));
  RICK_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  RICK_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  size_t sm = cols_pair_smem_bytes<T, LOGN>();
  const size_t floor_b = (size_t)smem_sm / (size_t)(max_blocks + 1) + 1;
  if (sm + (size_t)reserved < floor_b) sm = floor_b - (size_t)reserved;
  sm = (sm + 15) & ~(size_t)15;
  // batches carry column lengths up to 2^kMultiMaxLog: no multi-job kernel beyond
  const void *fn = (const void *)k_fft_cols_pair<T, LOGN>;
  if constexpr (LOGN <= kMultiMaxLog) {
    if (!f.one) fn = (const void *)k_fft_cols_pair_multi<T, LOGN>;
  } else {
    if (!f.one) return set_error(RICK_ERR_INVALID_ARG, "batch FFT length above %d", 1 << kMultiMaxLog);
  }
  RICK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  cudaFuncAttributes fa{};
  RICK_CUDA(cudaFuncGetAttributes(&fa, fn));
  const int regs_per_warp = ((std::max(fa.numRegs, 1) * 32 + 255) / 256) * 256;
  const int by_regs = 65536 / (regs_per_warp * (BT / 32));
  const int by_smem = (int)((size_t)smem_sm / (sm + (size_t)reserved));
  const int by_threads = 2048 / BT;
  const int per_sm = std::max(1, std::min({max_blocks, by_regs, by_smem, by_threads}));
  const int pct = (int)std::min<size_t>(
      100, ((size_t)per_sm * (sm + (size_t)reserved) * 100 + (size_t)smem_sm - 1) / (size_t)smem_sm);
  RICK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  const uint64_t slots = (uint64_t)num_sms() * per_sm;
  RICK_LAUNCHED();
  if (f.one) {
    const BatchJob &B = *f.one;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)B.g.nx / 2, slots));
    k_fft_cols_pair<T, LOGN><<<blocks, BT, sm, st>>>(col_job<T>(B, f));
  } else if constexpr (LOGN <= kMultiMaxLog) {
    const int rpc = fft_rows_per_block(LOGN);
    const uint64_t pairs = (uint64_t)c.units * (uint64_t)rpc / 2u;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>(pairs, slots));
    k_fft_cols_pair_multi<T, LOGN><<<blocks, BT, sm, st>>>(f.jobs, f.col_jobs, c.lo, c.hi,
                                                           f.col_units, rpc, f.rowmask, f.counts);
  }
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

// The split pass (one FP64 job, 8192-point columns): one block per SM, which
// allocates all 512 TMEM columns; shared memory padded above half the SM's.
template <typename T, int LOGN>
int launch_cols_split(const BatchJob &B, const FftJobs &f, cudaStream_t st) {
  constexpr int BT = group_threads<LOGN - 1>();
  int dev = 0, smem_sm = 0, reserved = 0;
  RICK_CUDA(cudaGetDevice(&dev));
  RICK_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
  RICK_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
  size_t sm = cols_pair_smem_bytes<T, LOGN - 1>();
  const size_t floor_b = (size_t)smem_sm / 2 + 1;
  if (sm + (size_t)reserved < floor_b) sm = floor_b - (size_t)reserved;
  sm = (sm + 15) & ~(size_t)15;
  const void *fn = (const void *)k_fft_cols_split<T, LOGN>;
  RICK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int pct = (int)std::min<size_t>(
      100, ((sm + (size_t)reserved) * 100 + (size_t)smem_sm - 1) / (size_t)smem_sm);
  RICK_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
  const int blocks = std::max(1, std::min(B.g.nx, num_sms()));
  RICK_LAUNCHED();
  k_fft_cols_split<T, LOGN><<<blocks, BT, sm, st>>>(col_job<T>(B, f));
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

template <typename T, int LOGN>
int launch_cols(const FftJobs &f, const FftClass &c, cudaStream_t st) {
  constexpr int G = group_threads<LOGN>(), BT = block_threads<LOGN>();
  constexpr int rpc = BT / G;
  // in order of preference, the first that fits: two planes per iteration
  // (FP32), double-buffered loads, the per-pixel phase steps
  constexpr size_t kMax = 220 * 1024;
  // the TMEM-state passes: always for one job; for a batch when its schedule
  // asks for them (planes in flight 0).  Two columns per block from 1024 to
  // 4096 points, and at 8192 for FP32 (both columns' buffers in shared
  // memory); at 8192 for FP64 one column split into two 4096-point halves;
  // one column per block otherwise.
  const bool tm_one = cols_tm_enabled() && f.one;
  const bool tm_batch = cols_tm_enabled() && !f.one && f.cols_pp == 0 && LOGN <= kMultiMaxLog;
  if constexpr ((LOGN >= 10 && LOGN <= 12) || (LOGN == 13 && sizeof(T) == 4)) {
    if ((tm_one || tm_batch) && cols_pair_enabled()) return launch_cols_pair<T, LOGN>(f, c, st);
  }
  if constexpr (LOGN == 13 && sizeof(T) == 8) {
    if (tm_one && cols_pair_enabled()) return launch_cols_split<T, LOGN>(*f.one, f, st);
  }
  if (tm_one) return launch_cols_tm<T, LOGN>(f, c, st);
  if constexpr (LOGN <= kMultiMaxLog) {
    if (tm_batch) return launch_cols_tm<T, LOGN>(f, c, st);
  }
#define RICK_TRY_COLS(DB, RC, PP)                            \
  if (cols_smem<T, LOGN, DB, RC, PP>(rpc) <= kMax)           \
    return launch_cols_impl<T, LOGN, DB, RC, PP>(f, c, st);
  if constexpr (sizeof(T) == 4) {
    if (f.cols_pp >= 2) {
      RICK_TRY_COLS(true, true, 2)
    }
  }
  RICK_TRY_COLS(true, true, 1)
  RICK_TRY_COLS(false, true, 1)
#undef RICK_TRY_COLS
  return launch_cols_impl<T, LOGN, false, false, 1>(f, c, st);
}

}  // namespace

bool sparse_fft_supported(int nx, int ny) {
  // power-of-two axes from 64 to 8192 (nx >= 64 makes it a multiple of the tile)
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

void fft_classes(const BatchJob *jobs, int njobs, FftJobs &f, uint32_t *col_jobs,
                 uint32_t *col_units) {
  f.n_row_cls = 0;
  for (int j = 0; j < njobs; j++) {
    if (f.n_row_cls == 0 || f.row_cls[f.n_row_cls - 1].log != jobs[j].logx)
      f.row_cls[f.n_row_cls++] = FftClass{jobs[j].logx, j, j + 1, 0};
    else
      f.row_cls[f.n_row_cls - 1].hi = j + 1;
  }
  // column pass: the jobs grouped by logy (stable), units = column groups
  int n = 0;
  f.n_col_cls = 0;
  uint32_t acc = 0;
  for (int l = 6; l <= 13; l++) {
    const int lo = n;
    uint32_t units = 0;
    for (int j = 0; j < njobs; j++) {
      if (jobs[j].logy != l) continue;
      col_jobs[n] = (uint32_t)j;
      col_units[n] = acc;
      const uint32_t rpc = (uint32_t)fft_rows_per_block(l);
      const uint32_t u = ((uint32_t)jobs[j].g.nx + rpc - 1) / rpc;
      acc += u;
      units += u;
      n++;
    }
    if (n > lo) f.col_cls[f.n_col_cls++] = FftClass{l, lo, n, units};
  }
  col_units[n] = acc;
}

int sparse_fft_lists(const FftJobs &f, cudaStream_t st) {
  RICK_CUDA(cudaMemsetAsync(f.counts, 0, sizeof(uint32_t) * f.total_count_words, st));
  const uint64_t nwords = f.total_mask_words;
  const int blocks = (int)std::min<uint64_t>((nwords + 255) / 256, (uint64_t)num_sms() * 8);
  RICK_LAUNCHED();
  k_row_list<<<std::max(blocks, 1), 256, 0, st>>>(f.jobs, f.njobs, f.mask_base, nwords,
                                                  f.rowmask, f.rowlist, f.counts);
  RICK_CUDA(cudaGetLastError());
  if (!f.one) {  // one job's row pass reads its row count directly
    RICK_LAUNCHED();
    k_fft_units<<<1, 32, 0, st>>>(f.jobs, f.njobs, f.counts, f.fft_units);
    RICK_CUDA(cudaGetLastError());
  }
  return RICK_OK;
}

#define RICK_FFT_SIZES(X) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13)

int sparse_fft_rows(const FftJobs &f, int precision, cudaStream_t st) {
  for (int i = 0; i < f.n_row_cls; i++) {
    const FftClass &c = f.row_cls[i];
    int r = RICK_ERR_INVALID_ARG;
    if (precision == RICK_PREC_FP64) {
      switch (c.log) {
#define X(L) case L: r = launch_rows<double, L>(f, c, st); break;
        RICK_FFT_SIZES(X)
#undef X
      }
    } else {
      switch (c.log) {
#define X(L) case L: r = launch_rows<float, L>(f, c, st); break;
        RICK_FFT_SIZES(X)
#undef X
      }
    }
    RICK_TRY(r);
  }
  return RICK_OK;
}

int sparse_fft_cols(const FftJobs &f, int precision, cudaStream_t st) {
  for (int i = 0; i < f.n_col_cls; i++) {
    const FftClass &c = f.col_cls[i];
    int r = RICK_ERR_INVALID_ARG;
    if (precision == RICK_PREC_FP64) {
      switch (c.log) {
#define X(L) case L: r = launch_cols<double, L>(f, c, st); break;
        RICK_FFT_SIZES(X)
#undef X
      }
    } else {
      switch (c.log) {
#define X(L) case L: r = launch_cols<float, L>(f, c, st); break;
        RICK_FFT_SIZES(X)
#undef X
      }
    }
    RICK_TRY(r);
  }
  return RICK_OK;
}

}  // namespace rick
