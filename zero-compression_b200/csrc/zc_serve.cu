// zc_serve.cu -- the serving loop of include/zero_cuda.h: jobs admitted by free device memory, their
// blocks batched across jobs tick by tick, each batch one replayed CUDA graph, two batches in flight (the
// next one runs on the GPU while the host hands out the last one's results).  Host code only; the work
// goes through the device entry points (zc_compress_device / zc_decompress_device) of one context.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/zero_cuda.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// first-fit allocation of 256-byte aligned ranges of one device allocation
struct Arena {
  uint8_t* base = nullptr;
  uint64_t size = 0, used = 0;
  std::map<uint64_t, uint64_t> free_;  // offset -> length
  static uint64_t round(uint64_t n) { return (n + 255) & ~(uint64_t)255; }
  bool alloc(uint64_t n, uint64_t& off) {
    n = round(std::max<uint64_t>(n, 1));
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      off = it->first;
      const uint64_t rest = it->second - n;
      free_.erase(it);
      if (rest) free_[off + n] = rest;
      used += n;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t n) {
    n = round(std::max<uint64_t>(n, 1));
    used -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
    }
  }
};

struct Job {
  uint64_t id = 0;
  zc_job j{};
  double t_submit = 0, t_done = 0;
  int status = ZC_OK;
  bool done = false, admitted = false;
  uint64_t footprint = 0, in_off = 0, out_off = 0;  // arena placement
  uint32_t nb = 0, next = 0, finished = 0;          // blocks; handed to batches; completed
  std::vector<uint64_t> bin, bout;                  // per block: input offset, output offset (in the job)
  std::vector<uint32_t> blen, rlen;                 // per block: input length, raw length
  uint64_t pay_at = 0;                              // compress: next free byte of the job's payload buffer
  uint64_t raw_total = 0;
  cudaEvent_t up = nullptr;                         // recorded after the job's upload
  bool uploaded = false;                            // its upload is queued and `up` recorded
  bool out_pinned = false;                          // extract: `out` is page-locked (copied into directly)
};

// a batch's class: the kind of kernels, block size and level it shares
struct Cls {
  bool compress;
  uint32_t bl;
  int level;
  bool operator==(const Cls& o) const { return compress == o.compress && bl == o.bl && level == o.level; }
};
Cls cls_of(const Job* J) {
  const bool c = J->j.kind == ZC_JOB_COMPRESS;
  return Cls{c, J->j.block_log, c ? J->j.level : 0};
}

constexpr uint32_t kCap = 4096;  // blocks per batch at most (padded to a fixed count per block size)
constexpr uint64_t kFreeMargin = 1ull << 30;  // device memory the arena leaves free

}  // namespace

// one batch in flight: its descriptors and results (device, and pinned host), its payload / raw-byte
// staging, and the event recorded after its small results are copied down
struct Slot {
  uint64_t *d_a64 = nullptr, *d_b64 = nullptr, *d_total = nullptr;
  uint32_t *d_a32 = nullptr, *d_b32 = nullptr, *d_c32 = nullptr, *d_err = nullptr;
  uint8_t *d_meth = nullptr, *d_stage = nullptr;
  uint8_t* h = nullptr;        // pinned: descriptors up, results down
  uint8_t* h_stage = nullptr;  // pinned: payloads (compress) or raw bytes (extract) down
  cudaEvent_t ev = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;  // timing: around the batch's graph
  bool busy = false;
  Cls k{};
  std::vector<std::pair<Job*, uint32_t>> take;
  std::vector<std::pair<uint64_t, uint64_t>> runs;  // extract: per run of a job's blocks, stage offset, length
  int rc = ZC_OK;
};

struct zc_server {
  int device = 0;
  zc_ctx* ctx = nullptr;
  cudaStream_t st = nullptr;   // kernels and small result copies, in order
  cudaStream_t ust = nullptr;  // job uploads (the kernel stream waits on each job's upload event)
  cudaStream_t cst = nullptr;  // payload copies of a finished batch, beside the next batch's kernels
  Arena arena;
  uint64_t max_batch = 256ull << 20;
  std::mutex mu, tmu;  // (tmu: the timing totals)
  std::condition_variable cv_work, cv_done;
  std::deque<Job*> pending;
  std::vector<Job*> active;
  std::map<uint64_t, Job*> jobs;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  std::thread uploader;              // uploads admitted jobs' bytes (pageable copies block their caller)
  std::deque<Job*> upq;
  std::condition_variable cv_up;
  bool worker_done = false;          // the uploader outlives the worker (its jobs may still need uploads)
  bool admit_blocked = false;        // the oldest pending job does not fit until some job finishes
  uint64_t jobs_done = 0, raw_bytes = 0, ticks = 0;
  double gpu_s = 0, wait_s = 0, handout_s = 0, upload_s = 0;  // accumulated (zc_serve_times)
  Slot slot[2];
  int failed = 0;  // a device failure ends the server: every job gets ZC_E_DEVICE
};

namespace {

uint32_t batch_cap(const zc_server* S, uint32_t bl) {
  return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(kCap, S->max_batch >> bl));
}

// places a job in the arena and hands it to the uploader; false when it does not fit now
bool admit(zc_server* S, Job* J) {
  uint64_t off;
  if (!S->arena.alloc(J->footprint, off)) return false;
  J->in_off = off;
  J->out_off = off + Arena::round(J->j.in_len + 64);
  J->admitted = true;
  S->upq.push_back(J);
  S->cv_up.notify_one();
  return true;
}

// the uploader thread: each admitted job's bytes to its arena range on the upload stream, then the event
// the kernel stream waits on; the job becomes batchable once the event is recorded
void uploader(zc_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    S->cv_up.wait(lk, [&] { return S->worker_done || !S->upq.empty(); });
    if (S->upq.empty()) return;  // (the worker has ended)
    Job* J = S->upq.front();
    S->upq.pop_front();
    lk.unlock();
    const double u0 = now_s();
    if (J->j.in_len) cudaMemcpyAsync(S->arena.base + J->in_off, J->j.in, J->j.in_len, cudaMemcpyHostToDevice, S->ust);
    cudaMemsetAsync(S->arena.base + J->in_off + J->j.in_len, 0, 64, S->ust);
    cudaEvent_t ev = nullptr;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess) cudaEventRecord(ev, S->ust);
    {
      std::lock_guard<std::mutex> g(S->tmu);
      S->upload_s += now_s() - u0;
    }
    lk.lock();
    J->up = ev;
    J->uploaded = true;
    S->cv_work.notify_all();
  }
}

void finish(zc_server* S, Job* J, int status) {
  if (J->done) return;
  if (status && !J->status) J->status = status;
  J->done = true;
  J->t_done = now_s();
  if (J->admitted) {
    S->arena.release(J->in_off, J->footprint);
    S->admit_blocked = false;
  }
  if (J->up) { cudaEventDestroy(J->up); J->up = nullptr; }
  S->jobs_done += 1;
  S->raw_bytes += J->raw_total;
}

// host views of a slot's pinned descriptor / result area
struct Views {
  uint64_t *ha, *hb;
  uint32_t *h1, *h2;
  uint8_t* hm;
  uint64_t* r_off;
  uint32_t *r_len, *r_crc, *r_err;
  uint8_t* r_meth;
  uint64_t* r_total;
};
Views views(Slot& L) {
  Views v;
  v.ha = reinterpret_cast<uint64_t*>(L.h);
  v.hb = v.ha + kCap;
  v.h1 = reinterpret_cast<uint32_t*>(v.hb + kCap);
  v.h2 = v.h1 + kCap;
  v.hm = reinterpret_cast<uint8_t*>(v.h2 + kCap);
  v.r_off = reinterpret_cast<uint64_t*>(v.hm + kCap);
  v.r_len = reinterpret_cast<uint32_t*>(v.r_off + kCap);
  v.r_crc = v.r_len + kCap;
  v.r_err = v.r_crc + kCap;
  v.r_meth = reinterpret_cast<uint8_t*>(v.r_err + kCap);
  v.r_total = reinterpret_cast<uint64_t*>(v.r_meth + kCap + 8);
  return v;
}

// queues a tick's batch (blocks of one class, from the admitted jobs in arrival order) on the stream:
// descriptors up, the batch's graph, small results down, the raw bytes of extract jobs to the stage;
// returns without waiting
void enqueue_batch(zc_server* S, Slot& L) {
  const Cls& k = L.k;
  Views v = views(L);
  const uint32_t n = (uint32_t)L.take.size();
  // padded to the next power of two (at least 16, at most the class's capacity): one graph per class and
  // size bucket, and a small tick does not launch the CTAs of a full one
  uint32_t cap = 16;
  while (cap < n) cap <<= 1;
  cap = std::min(cap, batch_cap(S, k.bl));
  for (uint32_t i = 0; i < cap; ++i) {
    if (i < n) {
      Job* J = L.take[i].first;
      const uint32_t b = L.take[i].second;
      v.ha[i] = J->in_off + J->bin[b];
      v.hb[i] = J->out_off + J->bout[b];
      v.h1[i] = J->blen[b];
      v.h2[i] = J->rlen[b];
      v.hm[i] = k.compress ? 0 : J->j.methods[b];
    } else {  // padding: an empty block
      v.ha[i] = 0; v.hb[i] = 0; v.h1[i] = 0; v.h2[i] = 0; v.hm[i] = 0;
    }
  }
  cudaStream_t st = S->st;
  L.rc = ZC_OK;
  L.runs.clear();
  for (uint32_t i = 0; i < n; ++i)
    if (L.take[i].first->up && (i == 0 || L.take[i - 1].first != L.take[i].first))
      cudaStreamWaitEvent(st, L.take[i].first->up, 0);
  cudaMemcpyAsync(L.d_a64, v.ha, cap * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(L.d_b64, v.hb, cap * 8, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(L.d_a32, v.h1, cap * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(L.d_b32, v.h2, cap * 4, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(L.d_meth, v.hm, cap, cudaMemcpyHostToDevice, st);
  cudaEventRecord(L.t0, st);
  if (k.compress) {
    L.rc = zc_compress_device(S->ctx, S->arena.base, L.d_a64, L.d_a32, cap, k.bl, k.level, L.d_meth, L.d_c32,
                              L.d_err, L.d_stage, S->max_batch + 64, L.d_b64, L.d_total, st);
    cudaEventRecord(L.t1, st);
    if (!L.rc) {
      cudaMemcpyAsync(v.r_off, L.d_b64, cap * 8, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(v.r_len, L.d_c32, cap * 4, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(v.r_crc, L.d_err, cap * 4, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(v.r_meth, L.d_meth, cap, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(v.r_total, L.d_total, 8, cudaMemcpyDeviceToHost, st);
    }
  } else {
    L.rc = zc_decompress_device(S->ctx, S->arena.base, L.d_a64, L.d_a32, L.d_meth, L.d_b32, cap, k.bl,
                                S->arena.base, L.d_b64, L.d_c32, L.d_err, st);
    cudaEventRecord(L.t1, st);
    if (!L.rc) {
      cudaMemcpyAsync(v.r_crc, L.d_c32, cap * 4, cudaMemcpyDeviceToHost, st);
      cudaMemcpyAsync(v.r_err, L.d_err, cap * 4, cudaMemcpyDeviceToHost, st);
      // the raw bytes of extract jobs to the stage, one copy per run of a job's blocks
      uint64_t at = 0;
      for (uint32_t i = 0; i < n;) {
        Job* J = L.take[i].first;
        uint32_t e = i;
        while (e < n && L.take[e].first == J) ++e;
        uint64_t len = 0;
        if (J->j.kind == ZC_JOB_EXTRACT) {
          const uint32_t b0 = L.take[i].second, b1 = L.take[e - 1].second;
          const uint64_t o0 = J->bout[b0], o1 = J->bout[b1] + J->rlen[b1];
          len = o1 > o0 ? o1 - o0 : 0;
          if (len && J->out_pinned) {  // straight into the caller's page-locked buffer: nothing to hand out
            cudaMemcpyAsync(J->j.out + o0, S->arena.base + J->out_off + o0, len, cudaMemcpyDeviceToHost, st);
            len = 0;
          } else if (len) {
            cudaMemcpyAsync(L.h_stage + at, S->arena.base + J->out_off + o0, len, cudaMemcpyDeviceToHost, st);
          }
        }
        L.runs.emplace_back(at, len);
        at += len;
        i = e;
      }
    }
  }
  if (cudaEventRecord(L.ev, st) != cudaSuccess && !L.rc) L.rc = ZC_E_DEVICE;
  L.busy = true;
}

// waits for a queued batch and hands its results to its jobs (payloads copied down on the second stream
// while the next batch's kernels run)
void complete_batch(zc_server* S, Slot& L) {
  const Cls& k = L.k;
  Views v = views(L);
  const uint32_t n = (uint32_t)L.take.size();
  int rc = L.rc;
  const double w0 = now_s();
  if (!rc && cudaEventSynchronize(L.ev) != cudaSuccess) rc = ZC_E_DEVICE;
  const double w1 = now_s();
  float gms = 0;
  if (!rc) cudaEventElapsedTime(&gms, L.t0, L.t1);
  if (k.compress) {
    if (!rc && *v.r_total) {
      cudaMemcpyAsync(L.h_stage, L.d_stage, *v.r_total, cudaMemcpyDeviceToHost, S->cst);
      if (cudaStreamSynchronize(S->cst) != cudaSuccess) rc = ZC_E_DEVICE;
    }
    for (uint32_t i = 0; i < n && !rc; ++i) {
      Job* J = L.take[i].first;
      const uint32_t b = L.take[i].second;
      J->j.out_methods[b] = v.r_meth[i];
      J->j.out_lens[b] = v.r_len[i];
      if (J->j.out_crcs) J->j.out_crcs[b] = v.r_crc[i];
      if (v.r_meth[i]) {
        if (J->pay_at + v.r_len[i] > J->j.out_cap) { J->status = ZC_E_ARG; continue; }
        memcpy(J->j.out + J->pay_at, L.h_stage + v.r_off[i], v.r_len[i]);
        J->j.out_offs[b] = J->pay_at;
        J->pay_at += v.r_len[i];
      } else {
        J->j.out_offs[b] = 0;
      }
    }
  } else if (!rc) {
    size_t run = 0;
    for (uint32_t i = 0; i < n; ++run) {
      Job* J = L.take[i].first;
      uint32_t e = i;
      while (e < n && L.take[e].first == J) ++e;
      if (L.runs[run].second) memcpy(J->j.out + J->bout[L.take[i].second], L.h_stage + L.runs[run].first, L.runs[run].second);
      i = e;
    }
    for (uint32_t i = 0; i < n; ++i) {
      Job* J = L.take[i].first;
      const uint32_t b = L.take[i].second;
      if (J->j.out_crcs) J->j.out_crcs[b] = v.r_crc[i];
      if (v.r_err[i]) J->status = ZC_E_DATA;
      else if (J->j.kind == ZC_JOB_TEST && J->j.crcs_expected && J->j.crcs_expected[b] != v.r_crc[i]) J->status = ZC_E_DATA;
    }
  }
  if (rc) S->failed = rc;
  for (uint32_t i = 0; i < n; ++i) L.take[i].first->finished += 1;
  L.busy = false;
  L.take.clear();
  const double w2 = now_s();
  std::lock_guard<std::mutex> g(S->tmu);
  S->gpu_s += gms * 1e-3;
  S->wait_s += w1 - w0;
  S->handout_s += w2 - w1;
}

void finish_done(zc_server* S) {
  for (auto it = S->active.begin(); it != S->active.end();) {
    Job* J = *it;
    if (J->uploaded && J->finished == J->nb && J->next == J->nb) { finish(S, J, ZC_OK); it = S->active.erase(it); }
    else ++it;
  }
  S->cv_done.notify_all();
}

// Each pass queues the next batch in one slot, then finishes the batch queued in the other slot on the
// pass before: the GPU runs batch k + 1 while the host hands out batch k's results.
void worker_loop(zc_server* S, std::unique_lock<std::mutex>& lk);

void worker(zc_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  worker_loop(S, lk);
  S->worker_done = true;
  S->cv_up.notify_all();
}

void worker_loop(zc_server* S, std::unique_lock<std::mutex>& lk) {
  int cur = 0;  // the slot the next batch goes to
  for (;;) {
    const bool inflight = S->slot[0].busy || S->slot[1].busy;
    S->cv_work.wait(lk, [&] {
      if (inflight || (!S->pending.empty() && !S->admit_blocked) || S->failed) return true;
      for (Job* J : S->active) if (J->uploaded && (J->next < J->nb || J->finished == J->nb)) return true;
      return S->stop && S->active.empty();
    });
    if (S->stop && S->pending.empty() && S->active.empty() && !inflight) return;
    if (S->failed) {  // the GPU failed: batches in flight end, then everything left ends with the error
      for (Slot& L : S->slot) if (L.busy) { lk.unlock(); complete_batch(S, L); lk.lock(); }
      for (Job* J : S->active) finish(S, J, S->failed);
      for (Job* J : S->pending) finish(S, J, S->failed);
      S->upq.clear();
      S->active.clear();
      S->pending.clear();
      S->cv_done.notify_all();
      if (S->stop) return;
      S->cv_work.wait(lk, [&] { return S->stop || !S->pending.empty(); });
      continue;
    }
    // admission in arrival order, while the arena has room
    while (!S->pending.empty() && !S->admit_blocked) {
      if (!admit(S, S->pending.front())) { S->admit_blocked = true; break; }
      S->active.push_back(S->pending.front());
      S->pending.pop_front();
    }
    // the next batch: the class of the oldest job with blocks left; its blocks, then later jobs' of the class
    bool queued = false;
    Slot& L = S->slot[cur];
    Job* first = nullptr;
    for (Job* J : S->active) if (J->uploaded && J->next < J->nb) { first = J; break; }
    if (first && !L.busy) {
      const Cls k = cls_of(first);
      const uint32_t cap = batch_cap(S, k.bl);
      L.k = k;
      L.take.clear();
      uint64_t bytes = 0;
      for (Job* J : S->active) {
        if (!J->uploaded || !(cls_of(J) == k)) continue;
        while (J->next < J->nb && L.take.size() < cap) {
          const uint64_t nbytes = (uint64_t)(k.compress ? J->blen[J->next] : J->rlen[J->next]);
          if (!L.take.empty() && bytes + nbytes > S->max_batch) break;
          L.take.emplace_back(J, J->next++);
          bytes += nbytes;
        }
        if (L.take.size() >= cap || bytes >= S->max_batch) break;
      }
      lk.unlock();
      enqueue_batch(S, L);
      lk.lock();
      S->ticks += 1;
      queued = true;
    }
    Slot& P = S->slot[cur ^ 1];
    if (P.busy) {
      lk.unlock();
      complete_batch(S, P);
      lk.lock();
    }
    if (queued) cur ^= 1;
    finish_done(S);
  }
}

}  // namespace

extern "C" {

int zc_serve_open(zc_server** out, int device, uint64_t budget_bytes, uint64_t max_batch_bytes) {
  if (!out) return ZC_E_ARG;
  *out = nullptr;
  zc_server* S = new zc_server;
  S->device = device;
  if (max_batch_bytes) S->max_batch = std::max<uint64_t>(max_batch_bytes, 1u << 20);
  int rc = zc_open(&S->ctx, device);
  if (rc) { zc_close(S->ctx); delete S; return rc; }
  cudaError_t e = cudaSetDevice(device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->ust, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->cst, cudaStreamNonBlocking);
  for (Slot& L : S->slot) {
    if (e == cudaSuccess) e = cudaMalloc(&L.d_a64, kCap * 8 * 3);
    if (e == cudaSuccess) { L.d_b64 = L.d_a64 + kCap; L.d_total = L.d_b64 + kCap; }
    if (e == cudaSuccess) e = cudaMalloc(&L.d_a32, kCap * 4 * 4 + kCap);
    if (e == cudaSuccess) {
      L.d_b32 = L.d_a32 + kCap; L.d_c32 = L.d_b32 + kCap; L.d_err = L.d_c32 + kCap;
      L.d_meth = reinterpret_cast<uint8_t*>(L.d_err + kCap);
    }
    if (e == cudaSuccess) e = cudaMalloc(&L.d_stage, S->max_batch + 64);
    if (e == cudaSuccess) e = cudaMallocHost(&L.h, kCap * 64 + 64);
    if (e == cudaSuccess) e = cudaMallocHost(&L.h_stage, S->max_batch + 64);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L.ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&L.t0);
    if (e == cudaSuccess) e = cudaEventCreate(&L.t1);
  }
  if (e == cudaSuccess) rc = zc_set_graphs(S->ctx, 1);
  // the codec's scratch for the largest batch of every block size, once: ticks then never reallocate it
  for (uint32_t bl = 16; bl <= 20 && e == cudaSuccess && !rc; ++bl) rc = zc_reserve(S->ctx, bl, batch_cap(S, bl));
  // the jobs' arena, last: the budget, but no more than the device has free now beside everything above
  // (less kFreeMargin for the runtime and other users), so that admission against it is admission by the
  // device's free memory
  if (e == cudaSuccess && !rc) {
    size_t free_b = 0, total_b = 0;
    e = cudaMemGetInfo(&free_b, &total_b);
    const uint64_t room = free_b > kFreeMargin ? free_b - kFreeMargin : 0;
    const uint64_t size = std::min<uint64_t>(std::max<uint64_t>(budget_bytes, 1u << 20), room);
    if (e == cudaSuccess && size < (1u << 20)) e = cudaErrorMemoryAllocation;
    if (e == cudaSuccess) e = cudaMalloc(&S->arena.base, size);
    if (e == cudaSuccess) {
      S->arena.size = size;
      S->arena.free_[0] = size;
    }
  }
  if (e != cudaSuccess || rc) {
    zc_serve_close(S);
    return e == cudaErrorMemoryAllocation ? ZC_E_NOMEM : (rc ? rc : ZC_E_DEVICE);
  }
  S->worker = std::thread(worker, S);
  S->uploader = std::thread(uploader, S);
  *out = S;
  return ZC_OK;
}

void zc_serve_close(zc_server* S) {
  if (!S) return;
  if (S->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->stop = true;
    }
    S->cv_work.notify_all();
    S->cv_up.notify_all();
    S->worker.join();
  }
  if (S->uploader.joinable()) {
    S->cv_up.notify_all();
    S->uploader.join();
  }
  cudaSetDevice(S->device);
  for (cudaStream_t x : {S->st, S->ust, S->cst})
    if (x) cudaStreamSynchronize(x);
  for (auto& kv : S->jobs) {
    if (kv.second->up) cudaEventDestroy(kv.second->up);
    delete kv.second;
  }
  if (S->arena.base) cudaFree(S->arena.base);
  for (Slot& L : S->slot) {
    if (L.d_a64) cudaFree(L.d_a64);
    if (L.d_a32) cudaFree(L.d_a32);
    if (L.d_stage) cudaFree(L.d_stage);
    if (L.h) cudaFreeHost(L.h);
    if (L.h_stage) cudaFreeHost(L.h_stage);
    if (L.ev) cudaEventDestroy(L.ev);
    if (L.t0) cudaEventDestroy(L.t0);
    if (L.t1) cudaEventDestroy(L.t1);
  }
  for (cudaStream_t x : {S->st, S->ust, S->cst})
    if (x) cudaStreamDestroy(x);
  zc_close(S->ctx);
  delete S;
}

int zc_serve_submit(zc_server* S, const zc_job* job, uint64_t* id) {
  if (!S || !job || !id) return ZC_E_ARG;
  const zc_job& j = *job;
  if (j.block_log < 16 || j.block_log > 20 || (j.in_len && !j.in)) return ZC_E_ARG;
  Job* J = new Job;
  J->j = j;
  const uint64_t B = 1ull << j.block_log;
  if (j.kind == ZC_JOB_COMPRESS) {
    if (!j.out_methods || !j.out_lens || !j.out_offs || (j.in_len && (!j.out || j.out_cap < j.in_len))) {
      delete J;
      return ZC_E_ARG;
    }
    J->nb = (uint32_t)((j.in_len + B - 1) / B);
    for (uint32_t b = 0; b < J->nb; ++b) {
      J->bin.push_back((uint64_t)b * B);
      J->bout.push_back(0);
      J->blen.push_back((uint32_t)std::min<uint64_t>(B, j.in_len - (uint64_t)b * B));
      J->rlen.push_back(J->blen.back());
    }
    J->raw_total = j.in_len;
    J->footprint = Arena::round(j.in_len + 64);
  } else if (j.kind == ZC_JOB_EXTRACT || j.kind == ZC_JOB_TEST) {
    if (j.nb && (!j.comp_lens || !j.methods || !j.raw_lens)) { delete J; return ZC_E_ARG; }
    J->nb = j.nb;
    uint64_t ci = 0, ro = 0;
    for (uint32_t b = 0; b < j.nb; ++b) {
      if (j.raw_lens[b] > B) { delete J; return ZC_E_ARG; }
      J->bin.push_back(ci);
      J->bout.push_back(ro);
      J->blen.push_back(j.comp_lens[b]);
      J->rlen.push_back(j.raw_lens[b]);
      ci += j.comp_lens[b];
      ro += j.raw_lens[b];
    }
    if (ci > j.in_len || (j.kind == ZC_JOB_EXTRACT && ro && (!j.out || j.out_cap < ro))) { delete J; return ZC_E_ARG; }
    J->raw_total = ro;
    J->footprint = Arena::round(j.in_len + 64) + Arena::round(ro + 64);
    if (j.kind == ZC_JOB_EXTRACT && j.out) {
      cudaPointerAttributes pa;
      if (cudaPointerGetAttributes(&pa, j.out) == cudaSuccess) J->out_pinned = pa.type == cudaMemoryTypeHost;
      else cudaGetLastError();
    }
  } else {
    delete J;
    return ZC_E_ARG;
  }
  if (J->footprint > S->arena.size) { delete J; return ZC_E_ARG; }
  {
    std::lock_guard<std::mutex> lk(S->mu);
    J->id = S->next_id++;
    J->t_submit = now_s();
    S->jobs[J->id] = J;
    S->pending.push_back(J);
    *id = J->id;
  }
  S->cv_work.notify_all();
  return ZC_OK;
}

int zc_serve_wait(zc_server* S, uint64_t id, double* latency_s) {
  if (!S) return ZC_E_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return ZC_E_ARG;
  Job* J = it->second;
  S->cv_done.wait(lk, [&] { return J->done; });
  const int st = J->status;
  if (latency_s) *latency_s = J->t_done - J->t_submit;
  S->jobs.erase(it);
  delete J;
  return st;
}

int zc_serve_stats(zc_server* S, uint64_t* jobs_done, uint64_t* raw_bytes, uint64_t* ticks, uint64_t* arena_used) {
  if (!S) return ZC_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  if (jobs_done) *jobs_done = S->jobs_done;
  if (raw_bytes) *raw_bytes = S->raw_bytes;
  if (ticks) *ticks = S->ticks;
  if (arena_used) *arena_used = S->arena.used;
  return ZC_OK;
}

int zc_serve_times(zc_server* S, double* gpu_s, double* wait_s, double* handout_s, double* upload_s) {
  if (!S) return ZC_E_ARG;
  std::lock_guard<std::mutex> g(S->tmu);
  if (gpu_s) *gpu_s = S->gpu_s;
  if (wait_s) *wait_s = S->wait_s;
  if (handout_s) *handout_s = S->handout_s;
  if (upload_s) *upload_s = S->upload_s;
  return ZC_OK;
}

}  // extern "C"
