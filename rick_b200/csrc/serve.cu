// Served imaging: a request loop with continuous batching.
//
// Jobs (rick_job_desc: device-resident rows, device images) are submitted from
// any thread as they arrive.  A scheduler thread admits waiting jobs, oldest
// first, while their HBM footprint fits the server's budget, launches the
// admitted ones as one batch (batch.cu: one launch per stage over all its
// jobs) on one of several streams, and keeps admitting while earlier batches
// run: batches overlap on the device, and memory freed by a finished batch is
// reused by the next.  Working memory comes from a stream-ordered pool
// (cudaMallocAsync / cudaFreeAsync), so admission never synchronises the
// device.  Completion is signalled by a host function enqueued after the batch
// (cudaLaunchHostFunc), which only records the time and wakes the scheduler.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "rick_internal.h"

using namespace rick;

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct ServedJob {
  rick_job_desc d{};
  uint64_t bytes = 0;       // footprint alone (admission bound)
  double t_submit = 0, t_launch = 0, t_done = 0;
  int status = RICK_OK;
  bool done = false;
  uint64_t batch = 0;
  uint32_t batch_jobs = 0;
};

struct InFlight {
  rick_batch *b = nullptr;
  uint64_t bytes = 0;
  uint64_t id = 0;
  std::vector<uint64_t> tickets;
  int stream = 0;
  bool done = false;
  double t_done = 0;
  struct rick_server *srv = nullptr;
};

}  // namespace

struct rick_server {
  rick_server_desc d{};
  std::mutex mu;
  std::condition_variable cv;       // scheduler wake-ups
  std::condition_variable done_cv;  // waiters
  std::deque<uint64_t> pending;
  std::unordered_map<uint64_t, ServedJob> jobs;
  std::list<InFlight *> inflight;
  std::vector<cudaStream_t> streams;
  std::vector<int> stream_busy;
  cudaMemPool_t pool = nullptr;
  uint64_t next_ticket = 1, next_batch = 1;
  uint64_t used = 0;
  bool stop = false;
  std::thread th;
  // the column passes of batches on different streams run one at a time (their
  // blocks allocate tensor memory; see rick_batch::cols_gate); batches are
  // launched by the scheduler thread alone, in order
  cudaEvent_t cols_gate = nullptr;
  rick_batch_tuning tune{2048, 6, 1};
  rick_server_stats stats{};
};

namespace {

void CUDART_CB on_batch_done(void *arg) {
  InFlight *f = static_cast<InFlight *>(arg);
  rick_server *s = f->srv;
  std::lock_guard<std::mutex> lk(s->mu);
  f->done = true;
  f->t_done = now_ms();
  s->cv.notify_all();
}

void fail_jobs(rick_server *s, const std::vector<uint64_t> &tickets, int status) {
  for (uint64_t t : tickets) {
    ServedJob &j = s->jobs[t];
    j.status = status;
    j.done = true;
    j.t_done = now_ms();
  }
  s->done_cv.notify_all();
}

// Launches `tickets` as one batch on a free stream (mu is not held).
int launch_batch(rick_server *s, InFlight *f, const std::vector<rick_job_desc> &descs) {
  cudaStream_t st = s->streams[f->stream];
  void *arena = nullptr;
  RICK_CUDA(cudaMallocFromPoolAsync(&arena, f->bytes, s->pool, st));
  rick_batch *b = nullptr;
  int r = batch_create_in(&b, descs.data(), (int)descs.size(), s->d.precision, s->d.device, arena,
                          f->bytes, s->tune, st, s->cols_gate);
  if (r == RICK_OK) r = batch_launch_eager(b, st);
  // stream-ordered: the arena returns to the pool once the batch has run
  const cudaError_t e = cudaFreeAsync(arena, st);
  if (r == RICK_OK && e != cudaSuccess) r = cuda_status(e, "cudaFreeAsync", __FILE__, __LINE__);
  f->b = b;
  if (r == RICK_OK) {
    const cudaError_t e2 = cudaLaunchHostFunc(st, on_batch_done, f);
    if (e2 != cudaSuccess) r = cuda_status(e2, "cudaLaunchHostFunc", __FILE__, __LINE__);
  }
  return r;
}

void scheduler(rick_server *s) {
  cudaSetDevice(s->d.device);
  std::unique_lock<std::mutex> lk(s->mu);
  std::vector<InFlight *> running;
  std::vector<cudaError_t> state;
  for (;;) {
    // A stream that reports an error will never run its completion function,
    // so its jobs fail here.  The streams are queried without holding the
    // lock: the completion function (run by CUDA's callback thread) takes it,
    // and a CUDA call made while holding it could wait on that function.  Only
    // this thread removes batches, so the pointers stay valid meanwhile.
    running.clear();
    for (InFlight *f : s->inflight)
      if (!f->done) running.push_back(f);
    state.assign(running.size(), cudaSuccess);
    if (!running.empty()) {
      lk.unlock();
      for (size_t i = 0; i < running.size(); i++)
        state[i] = cudaStreamQuery(s->streams[running[i]->stream]);
      lk.lock();
    }
    // retire finished batches and those whose stream failed
    for (auto it = s->inflight.begin(); it != s->inflight.end();) {
      InFlight *f = *it;
      if (!f->done) {
        cudaError_t q = cudaSuccess;
        for (size_t i = 0; i < running.size(); i++)
          if (running[i] == f) q = state[i];
        if (q == cudaSuccess || q == cudaErrorNotReady) {
          ++it;
          continue;
        }
        const int r = cuda_status(q, "served batch", __FILE__, __LINE__);
        fail_jobs(s, f->tickets, r);
        s->used -= f->bytes;
        it = s->inflight.erase(it);  // the batch's host state is left to the failed context
        continue;
      }
      for (uint64_t t : f->tickets) {
        ServedJob &j = s->jobs[t];
        j.done = true;
        j.t_done = f->t_done;
        s->stats.jobs_done++;
        s->stats.vis_done += j.d.num_rows * j.d.freq_per_chan * j.d.polarizations;
      }
      s->used -= f->bytes;
      s->stream_busy[f->stream] = 0;
      lk.unlock();
      batch_destroy(f->b);  // host side only: the device work has finished
      lk.lock();
      delete f;
      it = s->inflight.erase(it);
      s->done_cv.notify_all();
    }
    if (s->stop && s->pending.empty() && s->inflight.empty()) break;
    // admit: oldest first, every waiting job that fits the free budget
    int free_stream = -1;
    for (int k = 0; k < (int)s->streams.size(); k++)
      if (!s->stream_busy[k]) {
        free_stream = k;
        break;
      }
    if (!s->pending.empty() && free_stream >= 0) {
      std::vector<uint64_t> pick;
      std::vector<rick_job_desc> descs;
      uint64_t bytes = 0;
      const uint64_t solo = s->d.solo_vis ? s->d.solo_vis : 50000000ull;
      for (auto it = s->pending.begin(); it != s->pending.end();) {
        if ((int)pick.size() >= s->d.max_batch_jobs) break;
        const ServedJob &j = s->jobs[*it];
        const bool big = j.d.num_rows * j.d.freq_per_chan * j.d.polarizations >= solo;
        if (big && !pick.empty()) {  // a large job runs alone; the small ones go on without it
          ++it;
          continue;
        }
        descs.push_back(j.d);
        const uint64_t need = batch_bytes(descs.data(), (int)descs.size(), s->d.precision);
        if (need && s->used + need <= s->d.hbm_budget) {
          pick.push_back(*it);
          bytes = need;
          it = s->pending.erase(it);
          if (big) break;
        } else {
          descs.pop_back();
          ++it;
        }
      }
      if (!pick.empty()) {
        InFlight *f = new InFlight();
        f->srv = s;
        f->bytes = bytes;
        f->id = s->next_batch++;
        f->tickets = pick;
        f->stream = free_stream;
        s->stream_busy[free_stream] = 1;
        s->used += bytes;
        s->stats.batches++;
        s->stats.peak_bytes = std::max(s->stats.peak_bytes, s->used);
        const double t = now_ms();
        for (uint64_t tk : pick) {
          ServedJob &j = s->jobs[tk];
          j.t_launch = t;
          j.batch = f->id;
          j.batch_jobs = (uint32_t)pick.size();
        }
        s->inflight.push_back(f);
        lk.unlock();
        const int r = launch_batch(s, f, descs);
        lk.lock();
        if (r != RICK_OK) {
          // nothing of this batch will signal: retire it here
          s->inflight.remove(f);
          s->used -= f->bytes;
          s->stream_busy[f->stream] = 0;
          fail_jobs(s, f->tickets, r);
          if (f->b) {
            lk.unlock();
            cudaStreamSynchronize(s->streams[f->stream]);
            batch_destroy(f->b);
            lk.lock();
          }
          delete f;
        }
        continue;
      }
    }
    s->cv.wait_for(lk, std::chrono::milliseconds(5));
  }
}

}  // namespace

extern "C" {

int rick_server_create(rick_server **out, const rick_server_desc *d) {
  if (!out || !d) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  if (d->precision != RICK_PREC_FP64 && d->precision != RICK_PREC_MIXED)
    return set_error(RICK_ERR_INVALID_ARG, "unknown precision %d", d->precision);
  if (d->hbm_budget == 0 || d->max_batch_jobs <= 0 || d->streams <= 0)
    return set_error(RICK_ERR_INVALID_ARG, "budget, max_batch_jobs and streams must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_error(RICK_ERR_NO_ACCELERATORS_FOUND, "No accelerators found");
  }
  rick_server *s = new rick_server();
  s->d = *d;
  s->d.device = d->device >= 0 ? d->device % ndev : 0;
  cudaSetDevice(s->d.device);
  rick_batch_tuning t;
  if (batch_cached_tuning(d->precision, &t)) s->tune = t;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s->d.device;
  cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
  if (e == cudaSuccess) {
    uint64_t keep = d->hbm_budget;  // keep freed blocks for the next batches
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->cols_gate, cudaEventDisableTiming);
  for (int k = 0; k < d->streams && e == cudaSuccess; k++) {
    cudaStream_t st = nullptr;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
      s->streams.push_back(st);
      s->stream_busy.push_back(0);
    }
  }
  if (e == cudaSuccess) {
    // map the whole budget now, so that no admission waits for the pool to grow
    void *all = nullptr;
    e = cudaMallocFromPoolAsync(&all, d->hbm_budget, s->pool, s->streams[0]);
    if (e == cudaSuccess) e = cudaFreeAsync(all, s->streams[0]);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->streams[0]);
    if (e == cudaErrorMemoryAllocation) {
      cudaGetLastError();
      for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
      if (s->cols_gate) cudaEventDestroy(s->cols_gate);
      cudaMemPoolDestroy(s->pool);
      delete s;
      return set_error(RICK_ERR_NOT_ENOUGH_MEM, "the device cannot hold a budget of %llu bytes",
                       (unsigned long long)d->hbm_budget);
    }
  }
  if (e != cudaSuccess) {
    const int r = cuda_status(e, "rick_server_create", __FILE__, __LINE__);
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    if (s->cols_gate) cudaEventDestroy(s->cols_gate);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return r;
  }
  s->th = std::thread(scheduler, s);
  *out = s;
  return RICK_OK;
}

int rick_server_submit(rick_server *s, const rick_job_desc *job, uint64_t *ticket) {
  if (!s || !job || !ticket) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  uint64_t bytes = 0;
  RICK_TRY(rick_batch_footprint(job, 1, s->d.precision, &bytes));
  if (bytes > s->d.hbm_budget)
    return set_error(RICK_ERR_BUDGET, "job needs %llu bytes, the budget is %llu",
                     (unsigned long long)bytes, (unsigned long long)s->d.hbm_budget);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return set_error(RICK_ERR_CANCELLED, "server is shutting down");
  const uint64_t t = s->next_ticket++;
  ServedJob &j = s->jobs[t];
  j.d = *job;
  j.bytes = bytes;
  j.t_submit = now_ms();
  s->pending.push_back(t);
  s->stats.jobs_submitted++;
  *ticket = t;
  s->cv.notify_all();
  return RICK_OK;
}

int rick_server_wait(rick_server *s, uint64_t ticket, double timeout_ms, rick_job_result *res) {
  if (!s) return set_error(RICK_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) return set_error(RICK_ERR_INVALID_ARG, "unknown ticket %llu",
                                            (unsigned long long)ticket);
  auto ready = [&] { return s->jobs[ticket].done; };
  if (timeout_ms < 0) {
    s->done_cv.wait(lk, ready);
  } else if (!s->done_cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                                  ready)) {
    return set_error(RICK_ERR_CANCELLED, "timed out waiting for ticket %llu",
                     (unsigned long long)ticket);
  }
  const ServedJob j = s->jobs[ticket];
  s->jobs.erase(ticket);
  if (res) {
    memset(res, 0, sizeof(*res));
    res->status = j.status;
    res->queue_ms = j.t_launch - j.t_submit;
    res->latency_ms = j.t_done - j.t_submit;
    res->batch_id = j.batch;
    res->batch_jobs = j.batch_jobs;
  }
  if (j.status == RICK_ERR_CANCELLED)
    return set_error(j.status, "job %llu was cancelled before it was launched",
                     (unsigned long long)ticket);
  return j.status == RICK_OK ? RICK_OK
                             : set_error(j.status, "job %llu failed", (unsigned long long)ticket);
}

int rick_server_cancel(rick_server *s, uint64_t ticket) {
  if (!s) return set_error(RICK_ERR_INVALID_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it) {
    if (*it != ticket) continue;
    s->pending.erase(it);
    fail_jobs(s, {ticket}, RICK_ERR_CANCELLED);
    return RICK_OK;
  }
  return set_error(RICK_ERR_INVALID_ARG, "ticket %llu is not waiting (unknown, launched or done)",
                   (unsigned long long)ticket);
}

int rick_server_shutdown(rick_server *s, int drain) {
  if (!s) return set_error(RICK_ERR_INVALID_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->stop = true;
  if (!drain) {
    std::vector<uint64_t> waiting(s->pending.begin(), s->pending.end());
    s->pending.clear();
    fail_jobs(s, waiting, RICK_ERR_CANCELLED);
  }
  s->cv.notify_all();
  return RICK_OK;
}

int rick_server_get_stats(rick_server *s, rick_server_stats *out) {
  if (!s || !out) return set_error(RICK_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  out->bytes_in_use = s->used;
  out->jobs_waiting = s->pending.size();
  return RICK_OK;
}

int rick_server_destroy(rick_server *s) {
  if (!s) return RICK_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->th.joinable()) s->th.join();  // drains: every submitted job finishes
  cudaSetDevice(s->d.device);
  for (cudaStream_t st : s->streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  if (s->cols_gate) cudaEventDestroy(s->cols_gate);
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
  return RICK_OK;
}

}  // extern "C"
