// NORMALIZE_UVW on the device (gridding.c:21-83 for one rank).
//
// The reference scans the rows for the extrema of u, v and w (minima start at
// 1e20, maxima at 0), sets maxg = 1.001 * the largest |extremum| of u and v,
// and rewrites the rows in place: u, v -> (x + maxg) / (2 maxg),
// w -> (w - wmin) / (wmax - wmin).  Here one kernel reduces the extrema (block
// reductions, then one atomic per block on order-preserving integer keys of
// the doubles: minima and maxima are exact, so any order gives the
// reference's values) and a second rewrites the rows with round-to-nearest
// intrinsics in the reference's expression order, reading the extrema from
// device memory: no host round trip between the passes.
#include <algorithm>

#include "rick_internal.h"

namespace rick {

namespace {

// Order-preserving map of (non-NaN) doubles to unsigned keys.
__device__ __forceinline__ unsigned long long dkey(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dval(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

constexpr int kKeys = 8;  // keys start 64 bytes into the scratch

__global__ void k_uvw_init(unsigned long long *keys) {
  if (threadIdx.x < 3) keys[threadIdx.x] = dkey(1e20);      // minima of u, v, w
  else if (threadIdx.x < 6) keys[threadIdx.x] = dkey(0.0);  // maxima
}

__global__ void __launch_bounds__(256)
    k_uvw_extrema(const double *__restrict__ uu, const double *__restrict__ vv,
                  const double *__restrict__ ww, uint64_t n, unsigned long long *keys) {
  double m[6] = {1e20, 1e20, 1e20, 0.0, 0.0, 0.0};
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * (uint64_t)blockDim.x) {
    const double u = uu[i], v = vv[i], w = ww[i];
    m[0] = u < m[0] ? u : m[0];
    m[1] = v < m[1] ? v : m[1];
    m[2] = w < m[2] ? w : m[2];
    m[3] = u > m[3] ? u : m[3];
    m[4] = v > m[4] ? v : m[4];
    m[5] = w > m[5] ? w : m[5];
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const double t = __shfl_xor_sync(0xffffffffu, m[k], o);
      m[k] = k < 3 ? (t < m[k] ? t : m[k]) : (t > m[k] ? t : m[k]);
    }
  }
  __shared__ double s[8][6];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int k = 0; k < 6; k++) s[warp][k] = m[k];
  __syncthreads();
  if (threadIdx.x < 6) {
    const int k = threadIdx.x;
    double r = s[0][k];
    for (int w = 1; w < (int)(blockDim.x >> 5); w++)
      r = k < 3 ? (s[w][k] < r ? s[w][k] : r) : (s[w][k] > r ? s[w][k] : r);
    if (k < 3) atomicMin(&keys[k], dkey(r));
    else atomicMax(&keys[k], dkey(r));
  }
}

__global__ void __launch_bounds__(256)
    k_uvw_normalize(double *__restrict__ uu, double *__restrict__ vv, double *__restrict__ ww,
                    uint64_t n, const unsigned long long *__restrict__ keys,
                    double *__restrict__ extrema) {
  const double mnu = dval(keys[0]), mnv = dval(keys[1]), mnw = dval(keys[2]);
  const double mxu = dval(keys[3]), mxv = dval(keys[4]), mxw = dval(keys[5]);
  // gridding.c:68-72
  const double ming = fmax(fabs(mnu), fabs(mnv));
  double maxg = fmax(fabs(mxu), fabs(mxv));
  maxg = maxg > ming ? maxg : ming;
  maxg = __dadd_rn(maxg, __dmul_rn(0.001, maxg));
  const double two_maxg = __dmul_rn(2.0, maxg);
  const double wrange = __dsub_rn(mxw, mnw);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    extrema[0] = mnu;
    extrema[1] = mnv;
    extrema[2] = mnw;
    extrema[3] = mxu;
    extrema[4] = mxv;
    extrema[5] = mxw;
    extrema[6] = maxg;
  }
  // gridding.c:77-79
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * (uint64_t)blockDim.x) {
    uu[i] = __ddiv_rn(__dadd_rn(uu[i], maxg), two_maxg);
    vv[i] = __ddiv_rn(__dadd_rn(vv[i], maxg), two_maxg);
    ww[i] = __ddiv_rn(__dsub_rn(ww[i], mnw), wrange);
  }
}

}  // namespace

int normalize_uvw(uint64_t n, double *uu, double *vv, double *ww, void *scratch,
                  cudaStream_t st) {
  double *extrema = (double *)scratch;
  unsigned long long *keys = (unsigned long long *)scratch + kKeys;
  RICK_LAUNCHED();
  k_uvw_init<<<1, 32, 0, st>>>(keys);
  RICK_CUDA(cudaGetLastError());
  const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((n + 255) / 256,
                                                                    (uint64_t)num_sms() * 4));
  RICK_LAUNCHED();
  k_uvw_extrema<<<blocks, 256, 0, st>>>(uu, vv, ww, n, keys);
  RICK_CUDA(cudaGetLastError());
  RICK_LAUNCHED();
  k_uvw_normalize<<<blocks, 256, 0, st>>>(uu, vv, ww, n, keys, extrema);
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

}  // namespace rick

extern "C" int rick_normalize_uvw(uint64_t nrows, double *uu, double *vv, double *ww,
                                  void *scratch, void *stream) {
  using namespace rick;
  if (!scratch || (nrows && (!uu || !vv || !ww)))
    return set_error(RICK_ERR_INVALID_ARG, "null argument");
  if ((uintptr_t)scratch % 8 != 0) return set_error(RICK_ERR_INVALID_ARG, "scratch must be 8-byte aligned");
  return normalize_uvw(nrows, uu, vv, ww, scratch, (cudaStream_t)stream);
}
