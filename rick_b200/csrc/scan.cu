// Exclusive prefix sum of 32-bit counts (bin offsets, work-item offsets).
// Reduce-then-scan: each block scans 4096 entries and writes its total; the
// totals are scanned recursively and added back.  In-place use is allowed.
#include "rick_internal.h"

namespace rick {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 4;
constexpr int kScanBlock = kScanThreads * kScanPerThread;

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
  const unsigned lane = threadIdx.x & 31u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= (unsigned)o) v += t;
  }
  return v;
}

// Scans one block of kScanBlock entries of `in` into `out` (exclusive) and
// stores the block total in sums[blockIdx.x] (if sums != nullptr).
__global__ void __launch_bounds__(kScanThreads)
    k_scan_block(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *sums) {
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const uint64_t base = (uint64_t)blockIdx.x * kScanBlock + (uint64_t)threadIdx.x * kScanPerThread;
  uint32_t v[kScanPerThread];
  uint32_t local = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; k++) {
    v[k] = (base + k < n) ? in[base + k] : 0u;
    local += v[k];
  }
  const uint32_t incl = warp_inclusive(local);
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t t = warp_tot[lane];
    const uint32_t ti = warp_inclusive(t);
    warp_tot[lane] = ti - t;  // exclusive over warps
  }
  __syncthreads();
  uint32_t run = warp_tot[warp] + incl - local;
#pragma unroll
  for (int k = 0; k < kScanPerThread; k++) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (sums && threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = run;
}

__global__ void k_scan_add(uint32_t *out, uint64_t n, const uint32_t *sums) {
  const uint32_t add = sums[blockIdx.x];
  const uint64_t base = (uint64_t)blockIdx.x * kScanBlock;
  for (int k = threadIdx.x; k < kScanBlock; k += blockDim.x)
    if (base + k < n) out[base + k] += add;
}

}  // namespace

uint64_t scan_tmp_words(uint64_t n) {
  uint64_t words = 0;
  while (n > (uint64_t)kScanBlock) {
    n = (n + kScanBlock - 1) / kScanBlock;
    words += n;
  }
  return words + 64;
}

int exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *tmp,
                       cudaStream_t st) {
  if (n == 0) return RICK_OK;
  if (n <= (uint64_t)kScanBlock) {
    RICK_LAUNCHED();
    k_scan_block<<<1, kScanThreads, 0, st>>>(in, out, n, nullptr);
    RICK_CUDA(cudaGetLastError());
    return RICK_OK;
  }
  const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
  RICK_LAUNCHED();
  k_scan_block<<<(unsigned)nb, kScanThreads, 0, st>>>(in, out, n, tmp);
  RICK_CUDA(cudaGetLastError());
  RICK_TRY(exclusive_scan_u32(tmp, tmp, nb, tmp + nb, st));
  RICK_LAUNCHED();
  k_scan_add<<<(unsigned)nb, 256, 0, st>>>(out, n, tmp);
  RICK_CUDA(cudaGetLastError());
  return RICK_OK;
}

}  // namespace rick
