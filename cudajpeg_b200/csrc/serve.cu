// serve.cu -- continuous-batching decode server over the batch decoder.
//
// Requests (one JPEG each) are queued by any host thread.  A worker thread
// keeps up to `engines` batches in flight, each on its own CUDA stream:
// whenever an engine is free it admits the oldest waiting requests whose
// projected HBM footprint fits the budget left by the batches still in
// flight, stages them (host parse + one H2D copy), launches the batch kernel
// and moves on.  Requests that arrive while earlier batches run join the next
// one, so a batch's host parse and copies overlap another batch's kernel.
// Results stay on the device (the engine's output buffer) until the caller
// releases them; an engine is reused only when all of its results are
// released.
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/cj_dlpack.h"
#include "../../include/cudajpeg.h"
#include "cj_internal.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t ticket = 0;
  std::vector<unsigned char> owned;  // copy of the file (cjServerSubmit)
  const unsigned char* data = nullptr;
  size_t size = 0;
  int64_t footprint = 0;
  Clock::time_point t0, done_at;     // arrival (submit or scheduled) and batch end
  int engine = -1, slot = -1;
  bool done = false;
  int error = 0;
  const unsigned char* device_pixels = nullptr;
};

struct Engine {
  CJBatch* batch = nullptr;
  cudaEvent_t done = nullptr;
  CJHostBuf blob;
  std::vector<int64_t> offsets, sizes, tickets;
  std::vector<const unsigned char*> srcs;
  int64_t footprint = 0;
  int held = 0;  // finished results not yet released
  enum { FREE, RUNNING, HELD } state = FREE;
};

}  // namespace

struct CJServer {
  int device = 0;
  int64_t budget = 0;
  int max_batch = 256;
  std::vector<Engine> engines;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<int64_t> pending;
  std::unordered_map<int64_t, Request> reqs;
  int64_t next_ticket = 0, inflight_bytes = 0;
  int64_t batches = 0, images = 0, max_running = 0, max_batch_seen = 0;
  bool stop = false;
  int fatal = 0;
  // applied to each engine before it stages; serving batches are small at low
  // load, where short subsequences give the lowest latency
  int tune_sub = 512, tune_ctas = 0, tune_cap = 0;
  std::thread worker;
};

// Projected device bytes of one request from its file size and SOF geometry:
// compressed + destuffed bytes (2 x file), decoder records (~1 x file),
// int16 coefficients (at most 2 bytes per pixel per component, 4:4:4) and
// the output (1 byte per pixel per channel), plus a fixed 64 KiB.
static int64_t cj_footprint(const unsigned char* p, size_t n) {
  int64_t w = 0, h = 0, nch = 3;
  for (size_t i = 2; i + 4 <= n;) {
    if (p[i] != 0xFF) break;
    unsigned m = p[i + 1];
    if (m == 0xFF) {  // fill byte
      i++;
      continue;
    }
    unsigned len = (p[i + 2] << 8) | p[i + 3];
    if ((m == 0xC0 || m == 0xC1) && i + 10 <= n) {
      h = (p[i + 5] << 8) | p[i + 6];
      w = (p[i + 7] << 8) | p[i + 8];
      nch = p[i + 9] == 1 ? 1 : 3;
      break;
    }
    if (m == 0xDA || m == 0xD9) break;
    i += 2 + len;
  }
  const int64_t px = w * h;
  return 3 * (int64_t)n + px * 2 * nch + px * nch + (1 << 16);
}

static int64_t cj_server_enqueue(CJServer* s, const unsigned char* jpeg, size_t size, bool copy,
                                 Clock::time_point t0) {
  std::lock_guard<std::mutex> g(s->mu);
  if (s->fatal) return s->fatal > 0 ? -s->fatal : s->fatal;
  int64_t t = s->next_ticket++;
  Request& r = s->reqs[t];
  r.ticket = t;
  if (copy) {
    r.owned.assign(jpeg, jpeg + size);
    r.data = r.owned.data();
  } else {
    r.data = jpeg;
  }
  r.size = size;
  r.footprint = cj_footprint(jpeg, size);
  r.t0 = t0;
  s->pending.push_back(t);
  s->cv_work.notify_one();
  return t;
}

static void cj_server_loop(CJServer* s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    bool progressed = false;
    // completions
    for (size_t e = 0; e < s->engines.size(); e++) {
      Engine& en = s->engines[e];
      if (en.state == Engine::RUNNING && cudaEventQuery(en.done) == cudaSuccess) {
        std::vector<int> errs(en.tickets.size(), 0);
        int berr = cjBatchWait(en.batch, errs.data());
        Clock::time_point now = Clock::now();
        for (size_t k = 0; k < en.tickets.size(); k++) {
          Request& r = s->reqs[en.tickets[k]];
          r.error = berr ? berr : errs[k];
          r.device_pixels = cjBatchDeviceImage(en.batch, (int)k);
          r.done = true;
          r.done_at = now;
        }
        en.state = Engine::HELD;
        en.held = (int)en.tickets.size();
        progressed = true;
        s->cv_done.notify_all();
      }
      if (en.state == Engine::HELD && en.held == 0) {
        en.state = Engine::FREE;
        s->inflight_bytes -= en.footprint;
        en.footprint = 0;
        progressed = true;
      }
    }
    // admission: a free engine takes the oldest waiting requests that fit
    for (size_t e = 0; e < s->engines.size() && !s->pending.empty() && !s->fatal; e++) {
      Engine& en = s->engines[e];
      if (en.state != Engine::FREE) continue;
      en.tickets.clear();
      en.offsets.clear();
      en.sizes.clear();
      en.srcs.clear();
      int64_t bytes = 0, fp = 0;
      while (!s->pending.empty() && (int)en.tickets.size() < s->max_batch) {
        Request& r = s->reqs[s->pending.front()];
        bool fits = s->inflight_bytes + fp + r.footprint <= s->budget;
        bool lone = en.tickets.empty() && s->inflight_bytes == 0;  // always runs
        if (!fits && !lone) break;
        r.engine = (int)e;
        r.slot = (int)en.tickets.size();
        en.tickets.push_back(r.ticket);
        en.offsets.push_back(bytes);
        en.sizes.push_back((int64_t)r.size);
        en.srcs.push_back(r.data);
        bytes += ((int64_t)r.size + 15) & ~(int64_t)15;
        fp += r.footprint;
        s->pending.pop_front();
      }
      if (en.tickets.empty()) break;  // the budget is full: wait for a completion
      en.footprint = fp;
      s->inflight_bytes += fp;
      cjBatchSetTuning(en.batch, s->tune_sub, s->tune_ctas, s->tune_cap);
      const int n = (int)en.tickets.size();
      // packing, host parse, H2D and launch happen outside the lock
      lk.unlock();
      int err = cj_host_ensure(en.blob, (size_t)bytes + 64) ? OOM_ERROR : 0;
      if (!err)
        for (int k = 0; k < n; k++)
          memcpy((unsigned char*)en.blob.p + en.offsets[k], en.srcs[k], (size_t)en.sizes[k]);
      if (!err) err = cjBatchStage(en.batch, n, (const unsigned char*)en.blob.p, en.offsets.data(), en.sizes.data());
      if (!err) err = cjBatchRun(en.batch);
      if (!err && cudaEventRecord(en.done, (cudaStream_t)cjBatchStream(en.batch)) != cudaSuccess)
        err = CUDA_KERNEL_LAUNCH_ERROR;
      lk.lock();
      if (err) {
        Clock::time_point now = Clock::now();
        for (int64_t t : en.tickets) {
          Request& r = s->reqs[t];
          r.error = err;
          r.done = true;
          r.done_at = now;
        }
        en.state = Engine::HELD;
        en.held = n;
        if (err == OOM_ERROR || err == CUDA_MEM_ERROR || err == CUDA_KERNEL_LAUNCH_ERROR) s->fatal = err;
        s->cv_done.notify_all();
      } else {
        en.state = Engine::RUNNING;
      }
      s->batches++;
      s->images += n;
      if (n > s->max_batch_seen) s->max_batch_seen = n;
      int64_t running = 0;
      for (const Engine& x : s->engines) running += x.state == Engine::RUNNING;
      if (running > s->max_running) s->max_running = running;
      progressed = true;
    }
    if (!progressed) s->cv_work.wait_for(lk, std::chrono::microseconds(20));
  }
}

extern "C" {

CJServer* cjServerCreate(int engines, long long hbm_budget_bytes, int max_batch_images) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    fprintf(stderr, "libcudajpeg: no CUDA device available; the decoder has no CPU path\n");
    return NULL;
  }
  CJServer* s = new (std::nothrow) CJServer();
  if (!s) return NULL;
  cudaGetDevice(&s->device);
  s->budget = hbm_budget_bytes > 0 ? hbm_budget_bytes : (8ll << 30);
  s->max_batch = max_batch_images > 0 ? max_batch_images : 256;
  s->engines.resize(engines > 0 ? engines : 2);
  for (Engine& e : s->engines) {
    e.batch = cjBatchCreate();
    if (!e.batch || cudaEventCreateWithFlags(&e.done, cudaEventDisableTiming) != cudaSuccess) {
      cjServerDestroy(s);
      return NULL;
    }
  }
  s->worker = std::thread(cj_server_loop, s);
  return s;
}

void cjServerDestroy(CJServer* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (Engine& e : s->engines) {
    if (e.batch) cjBatchDestroy(e.batch);  // waits for its stream
    if (e.done) cudaEventDestroy(e.done);
    if (e.blob.p) cudaFreeHost(e.blob.p);
  }
  delete s;
}

long long cjServerSubmit(CJServer* s, const unsigned char* jpeg, size_t size) {
  if (!s || !jpeg) return PROGRAMMER_ERROR;
  return cj_server_enqueue(s, jpeg, size, true, Clock::now());
}

int cjServerWait(CJServer* s, long long ticket, double timeout_s, CJServerResult* out) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return PROGRAMMER_ERROR;
  auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                     std::chrono::duration<double>(timeout_s));
  while (!it->second.done) {
    bool timed_out = s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout;
    it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return PROGRAMMER_ERROR;  // released by another thread
    if (timed_out && !it->second.done) return 1;
  }
  Request& r = it->second;
  if (out) {
    out->error = r.error;
    out->width = out->height = out->channels = 0;
    out->device_pixels = r.error ? NULL : r.device_pixels;
    out->latency_ms = std::chrono::duration<double, std::milli>(r.done_at - r.t0).count();
    if (r.engine >= 0)
      cjBatchImageGeometry(s->engines[r.engine].batch, r.slot, &out->width, &out->height, &out->channels);
  }
  return 0;
}

int cjServerCopyOut(CJServer* s, long long ticket, unsigned char* host_dst, size_t capacity) {
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end() || !it->second.done || it->second.error || !it->second.device_pixels)
    return PROGRAMMER_ERROR;
  Request& r = it->second;
  int w = 0, h = 0, c = 0;
  cjBatchImageGeometry(s->engines[r.engine].batch, r.slot, &w, &h, &c);
  size_t n = (size_t)w * h * c;
  if (capacity < n) return PROGRAMMER_ERROR;
  const unsigned char* src = r.device_pixels;
  lk.unlock();  // the engine is HELD until this ticket is released
  CJ_CUDA_TRY(cudaMemcpy(host_dst, src, n, cudaMemcpyDeviceToHost), CUDA_MEM_ERROR);
  return 0;
}

DLManagedTensor* cjServerDLPack(CJServer* s, long long ticket) {
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end() || !it->second.done || it->second.error || !it->second.device_pixels) return NULL;
  return cjBatchDLPack(s->engines[it->second.engine].batch, it->second.slot);
}

void cjServerRelease(CJServer* s, long long ticket) {
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end() || !it->second.done) return;
  int e = it->second.engine;
  if (e >= 0) s->engines[e].held--;
  s->reqs.erase(it);
  s->cv_work.notify_one();
}

int cjServerSetTuning(CJServer* s, int sub_bits, int decode_ctas_per_sm, int pixel_tile_cap) {
  if (!s) return PROGRAMMER_ERROR;
  // validate on a scratch batch object (no device work)
  CJBatch* probe = cjBatchCreate();
  if (!probe) return OOM_ERROR;
  int e = cjBatchSetTuning(probe, sub_bits, decode_ctas_per_sm, pixel_tile_cap);
  cjBatchDestroy(probe);
  if (e) return e;
  std::lock_guard<std::mutex> g(s->mu);
  s->tune_sub = sub_bits;
  s->tune_ctas = decode_ctas_per_sm;
  s->tune_cap = pixel_tile_cap;
  return 0;
}

void cjServerStats(CJServer* s, long long* st) {
  std::lock_guard<std::mutex> g(s->mu);
  st[0] = s->batches;
  st[1] = s->images;
  st[2] = s->max_running;
  st[3] = s->max_batch_seen;
  st[4] = (long long)s->pending.size();
  st[5] = s->inflight_bytes;
}

int cjServerReplay(CJServer* s, const unsigned char* blob, const int64_t* offsets, const int64_t* sizes,
                   int nfiles, const double* arrival_s, int nreq, double* latency_ms, int* errors,
                   double* wall_s) {
  if (!s || !blob || nfiles <= 0 || nreq < 0 || !latency_ms) return PROGRAMMER_ERROR;
  std::vector<int64_t> tickets(nreq, -1);
  std::atomic<int> submitted{0};
  std::atomic<int> fatal{0};
  const Clock::time_point start = Clock::now() + std::chrono::milliseconds(1);
  auto at = [&](int k) {
    return start + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[k]));
  };
  Clock::time_point last_done = start;
  std::thread collector([&] {
    for (int k = 0; k < nreq; k++) {
      while (submitted.load(std::memory_order_acquire) <= k) std::this_thread::yield();
      if (tickets[k] < 0) {
        latency_ms[k] = -1.0;
        if (errors) errors[k] = fatal.load();
        continue;
      }
      std::unique_lock<std::mutex> lk(s->mu);
      auto it = s->reqs.find(tickets[k]);
      while (it != s->reqs.end() && !it->second.done) {
        s->cv_done.wait_for(lk, std::chrono::milliseconds(100));
        it = s->reqs.find(tickets[k]);
      }
      if (it == s->reqs.end()) {
        latency_ms[k] = -1.0;
        if (errors) errors[k] = PROGRAMMER_ERROR;
        continue;
      }
      Request& r = it->second;
      latency_ms[k] = std::chrono::duration<double, std::milli>(r.done_at - at(k)).count();
      if (errors) errors[k] = r.error;
      if (r.done_at > last_done) last_done = r.done_at;
      if (r.engine >= 0) s->engines[r.engine].held--;
      s->reqs.erase(it);
      s->cv_work.notify_one();
    }
  });
  for (int k = 0; k < nreq; k++) {
    const Clock::time_point t = at(k);
    while (Clock::now() < t) {
    }
    const int f = k % nfiles;
    int64_t tk = cj_server_enqueue(s, blob + offsets[f], (size_t)sizes[f], false, t);
    if (tk < 0) fatal.store((int)tk);
    tickets[k] = tk < 0 ? -1 : tk;
    submitted.store(k + 1, std::memory_order_release);
  }
  collector.join();
  if (wall_s) *wall_s = std::chrono::duration<double>(last_done - start).count();
  return fatal.load();
}

}  // extern "C"
