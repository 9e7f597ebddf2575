// Copies between pageable host memory and device memory at link speed.
//
// cudaMemcpy from pageable memory is staged by the driver through its own
// pinned buffers with one host thread doing the page copy; for the drop-ins,
// whose contract moves whole cubes between the caller's malloc'd arrays and the
// device on every call (wstack: rows in, cube in and out; rick_fft_planes: cube
// in and out; phase_correction: cube in), that host copy is the bound.  Here the
// copy goes through a ring of pinned buffers: a pool of host threads copies
// chunk c + 1 between the caller's memory and a pinned buffer while the copy
// engine moves chunk c, so the host copies overlap the PCIe transfer.  Pinned
// (page-locked or registered) caller memory is copied directly.
#include <string.h>

#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "rick_internal.h"

namespace rick {
namespace {

constexpr uint64_t kChunk = 64ull << 20;  // bytes per pinned buffer
constexpr int kSlots = 4;

// A fixed pool of host threads running one parallel-for at a time; the
// calling thread takes part.
class Pool {
 public:
  Pool() {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int n = (int)std::min(16u, hw) - 1;
    for (int i = 0; i < n; i++) th_.emplace_back([this, i] { worker(i + 1); });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto &t : th_) t.join();
  }
  int size() const { return (int)th_.size() + 1; }
  // fn(part) for part = 0 .. size()-1
  void run(const std::function<void(int)> &fn) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      pending_ = (int)th_.size();
      gen_++;
    }
    cv_.notify_all();
    fn(0);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [this] { return pending_ == 0; });
    fn_ = nullptr;
  }

 private:
  void worker(int part) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int)> *fn;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        fn = fn_;
      }
      (*fn)(part);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)> *fn_ = nullptr;
  uint64_t gen_ = 0;
  int pending_ = 0;
  bool stop_ = false;
};

struct Stager {
  std::mutex mu;  // one staged copy at a time per process
  Pool *pool = nullptr;
  void *slot[kSlots] = {};
  cudaEvent_t ev[kSlots] = {};
  int dev = -1;  // device the events belong to
};
Stager g_st;

// memcpy of n bytes split over the pool's threads (64-byte aligned parts)
void par_copy(void *dst, const void *src, uint64_t n) {
  const int parts = g_st.pool->size();
  const uint64_t per = ((n + parts - 1) / parts + 63) & ~63ull;
  g_st.pool->run([&](int p) {
    const uint64_t lo = std::min(n, (uint64_t)p * per), hi = std::min(n, lo + per);
    if (hi > lo) memcpy((char *)dst + lo, (const char *)src + lo, hi - lo);
  });
}

bool is_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int setup(int dev) {
  if (!g_st.pool) g_st.pool = new Pool();
  if (!g_st.slot[0]) {
    for (int i = 0; i < kSlots; i++) {
      // portable: the drop-ins pick the device per call
      const cudaError_t e = cudaHostAlloc(&g_st.slot[i], kChunk, cudaHostAllocPortable);
      if (e != cudaSuccess) {
        g_st.slot[i] = nullptr;
        return cuda_status(e, "cudaHostAlloc (copy staging)", __FILE__, __LINE__);
      }
    }
  }
  if (g_st.dev != dev) {  // events are recorded on this device's streams
    for (int i = 0; i < kSlots; i++) {
      if (g_st.ev[i]) cudaEventDestroy(g_st.ev[i]);
      RICK_CUDA(cudaEventCreateWithFlags(&g_st.ev[i], cudaEventDisableTiming));
    }
    g_st.dev = dev;
  }
  return RICK_OK;
}

}  // namespace

int copy_to_device(void *dst, const void *src, uint64_t bytes, cudaStream_t st) {
  if (!bytes) return RICK_OK;
  if (bytes < kChunk || is_pinned(src)) {
    RICK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    RICK_CUDA(cudaStreamSynchronize(st));
    return RICK_OK;
  }
  std::lock_guard<std::mutex> lk(g_st.mu);
  int dev = 0;
  RICK_CUDA(cudaGetDevice(&dev));
  RICK_TRY(setup(dev));
  bool used[kSlots] = {};
  for (uint64_t o = 0, c = 0; o < bytes; o += kChunk, c++) {
    const int s = (int)(c % kSlots);
    const uint64_t n = std::min(kChunk, bytes - o);
    if (used[s]) RICK_CUDA(cudaEventSynchronize(g_st.ev[s]));  // its last transfer is done
    par_copy(g_st.slot[s], (const char *)src + o, n);
    RICK_CUDA(cudaMemcpyAsync((char *)dst + o, g_st.slot[s], n, cudaMemcpyHostToDevice, st));
    RICK_CUDA(cudaEventRecord(g_st.ev[s], st));
    used[s] = true;
  }
  RICK_CUDA(cudaStreamSynchronize(st));
  return RICK_OK;
}

int copy_to_host(void *dst, const void *src, uint64_t bytes, cudaStream_t st) {
  if (!bytes) return RICK_OK;
  if (bytes < kChunk || is_pinned(dst)) {
    RICK_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st));
    RICK_CUDA(cudaStreamSynchronize(st));
    return RICK_OK;
  }
  std::lock_guard<std::mutex> lk(g_st.mu);
  int dev = 0;
  RICK_CUDA(cudaGetDevice(&dev));
  RICK_TRY(setup(dev));
  const uint64_t nchunks = (bytes + kChunk - 1) / kChunk;
  auto issue = [&](uint64_t c) -> int {
    const int s = (int)(c % kSlots);
    const uint64_t o = c * kChunk, n = std::min(kChunk, bytes - o);
    RICK_CUDA(cudaMemcpyAsync(g_st.slot[s], (const char *)src + o, n, cudaMemcpyDeviceToHost, st));
    RICK_CUDA(cudaEventRecord(g_st.ev[s], st));
    return RICK_OK;
  };
  for (uint64_t c = 0; c < std::min<uint64_t>(nchunks, kSlots); c++) RICK_TRY(issue(c));
  for (uint64_t c = 0; c < nchunks; c++) {
    const int s = (int)(c % kSlots);
    const uint64_t o = c * kChunk, n = std::min(kChunk, bytes - o);
    RICK_CUDA(cudaEventSynchronize(g_st.ev[s]));
    par_copy((char *)dst + o, g_st.slot[s], n);
    if (c + kSlots < nchunks) RICK_TRY(issue(c + kSlots));
  }
  return RICK_OK;
}

}  // namespace rick
