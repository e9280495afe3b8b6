// fsm_server.cu -- continuous-batching request server (no counterpart in the
// reference, which computes one event per call).
//
// Requests (one event each, host buffers copied in at submit) wait in a FIFO.
// A scheduler thread forms launch waves from the head of the queue whenever one
// of the server's streams is idle and the device / pinned-host budgets have
// room, so requests that arrive while others run join the next wave; waves on
// different streams overlap on the device (one wave's copies with another's
// kernels).  Each wave is an ordinary batch (fsm_runtime) whose memory comes
// from the server's pools: one device allocation of hbm_budget_bytes and one
// pinned host allocation of host_budget_bytes, carved by a first-fit
// allocator, so admitting a wave calls no allocator of the CUDA runtime.  A
// host callback at the end of each wave's stream work timestamps its
// completion; latency is submit -> outputs in host memory.
//
// Every cell's result depends only on its own event, so a request's outputs
// are the same alone and in any mix of requests (tests/test_server.py).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fsm_runtime.h"

using namespace fsm;
using namespace fsm::rt;

namespace {

using Clock = std::chrono::steady_clock;

// First-fit allocator over one region, 256-byte granules, coalescing frees.
class Pool {
 public:
  void reset(char* base, size_t size) {
    base_ = base;
    size_ = size;
    free_.clear();
    if (size) free_[0] = size;
  }
  char* alloc(size_t n) {
    n = align_up(std::max<size_t>(n, 1));
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        const size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[off + n] = len - n;
        used_ += n;
        return base_ + off;
      }
    }
    return nullptr;
  }
  void release(char* p, size_t n) {
    if (!p) return;
    n = align_up(std::max<size_t>(n, 1));
    size_t off = (size_t)(p - base_);
    used_ -= n;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + n == next->first) {
      n += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += n;
        return;
      }
    }
    free_[off] = n;
  }
  size_t used() const { return used_; }

 private:
  char* base_ = nullptr;
  size_t size_ = 0, used_ = 0;
  std::map<size_t, size_t> free_;
};

// Pinned output slab of a retired wave, shared by its requests until each has
// been polled (the poller copies straight from it).
struct OutBlock {
  char* p = nullptr;
  size_t bytes = 0;
  int refs = 0;
};

struct Request {
  long long id = 0;
  fsm_params p{};
  Clock::time_point t_wave;  // when a wave took it from the queue
  std::vector<float> e, nB;
  Clock::time_point t_submit, t_done;
  bool done = false;
  fsm_status status = FSM_OK;
  std::string msg;  // error message of a failed request
  OutBlock* ob = nullptr;  // holds the event's outputs once done
  const float* grp[kOutGroups] = {};  // its component groups in the block (nullptr: not kept)
  fsm_run_info info{};
  size_t dim = 0;
  bool baryon = false;
};

struct Wave {
  std::vector<Request*> reqs;
  fsm_batch* b = nullptr;
  int slot = 0;
  // pool regions: the batch's own device and staging blocks, plus the host
  // input and output slabs (+ 16 bytes of kernel error words after the outputs)
  char *d = nullptr, *hs = nullptr, *hin = nullptr, *hout = nullptr;
  size_t dbytes = 0, hsbytes = 0, hinbytes = 0, houtbytes = 0;
  size_t hgrp[kOutGroups];  // element offset of each kept output group in hout, or -1
  bool done = false;
  Clock::time_point t_done;
  // breakdown: host time to plan (batch_build) and to stage the inputs into
  // the pinned slab; CUDA events before the H2D copy, before the kernels,
  // after the kernels and after the D2H copies (on the wave's stream)
  Clock::time_point t_start;
  double plan_ms = 0, stage_ms = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
};

}  // namespace

struct fsm_server {
  fsm_server_opts opts{};
  fsm_ctx* ctx = nullptr;
  char* d_pool = nullptr;
  char* h_pool = nullptr;
  Pool dpool, hpool;
  std::vector<cudaStream_t> streams;
  std::vector<Wave*> slot_wave;  // wave in flight per stream, or nullptr
  int slot_2d = -1;              // the stream reserved for boost-invariant waves, or -1
  std::mutex mu;
  std::condition_variable cv;       // scheduler wake-ups
  std::condition_variable cv_done;  // pollers
  std::deque<Request*> queue;
  std::unordered_map<long long, Request*> reqs;
  long long next_id = 1;
  bool stopping = false;
  bool mem_wait = false;  // admission waits for pool memory (a wave or a poll frees it)
  // Bumped under mu by every event the scheduler waits for (a wave done, a
  // submit, freed output memory, stop).  The scheduler releases mu while it
  // plans a wave, and a notify in that window finds nobody waiting; comparing
  // the count before it sleeps catches such events.
  unsigned long long wake_gen = 0;
  std::thread th;
  // statistics
  long long submitted = 0, completed = 0, failed = 0, waves = 0;
  std::vector<double> lat_ms;
  Clock::time_point t_first{}, t_last{};
  bool have_first = false;
  // per-wave breakdown sums (fsm_server_breakdown_get)
  double sum_plan = 0, sum_stage = 0, sum_h2d = 0, sum_kernels = 0, sum_d2h = 0, sum_queue = 0;
  long long sum_events = 0, timed_waves = 0, queued_reqs = 0;
  std::vector<cudaEvent_t> event_pool;
};

namespace {

char* pool_dev(void* u, size_t n) {
  auto* W = static_cast<std::pair<fsm_server*, Wave*>*>(u);
  std::lock_guard<std::mutex> g(W->first->mu);
  char* p = W->first->dpool.alloc(n);
  if (p) {
    W->second->d = p;
    W->second->dbytes = n;
  }
  return p;
}
char* pool_host(void* u, size_t n) {
  auto* W = static_cast<std::pair<fsm_server*, Wave*>*>(u);
  std::lock_guard<std::mutex> g(W->first->mu);
  char* p = W->first->hpool.alloc(n);
  if (p) {
    W->second->hs = p;
    W->second->hsbytes = n;
  }
  return p;
}

void CUDART_CB wave_done_cb(void* user) {
  auto* W = static_cast<std::pair<fsm_server*, Wave*>*>(user);
  fsm_server* S = W->first;
  {
    std::lock_guard<std::mutex> g(S->mu);
    W->second->t_done = Clock::now();
    W->second->done = true;
    ++S->wake_gen;
  }
  S->cv.notify_all();
  delete W;
}

cudaEvent_t take_event(fsm_server* S) {
  if (!S->event_pool.empty()) {
    cudaEvent_t e = S->event_pool.back();
    S->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return e;
}

// Releases a wave's pool regions and batch (mu held); the output slab only
// when keep_out is false.
void wave_release(fsm_server* S, Wave* w, bool keep_out = false) {
  for (auto& e : w->ev)
    if (e) {
      S->event_pool.push_back(e);
      e = nullptr;
    }
  if (w->b) batch_free(w->b);
  S->dpool.release(w->d, w->dbytes);
  S->hpool.release(w->hs, w->hsbytes);
  S->hpool.release(w->hin, w->hinbytes);
  if (!keep_out) S->hpool.release(w->hout, w->houtbytes);
  w->b = nullptr;
  w->d = w->hs = w->hin = w->hout = nullptr;
}

void drop_output(fsm_server* S, Request* r) {
  if (r->ob && --r->ob->refs == 0) {
    S->hpool.release(r->ob->p, r->ob->bytes);
    delete r->ob;
    S->mem_wait = false;  // pinned memory came back: admission may proceed
    ++S->wake_gen;
    S->cv.notify_all();
  }
  r->ob = nullptr;
  for (auto& g : r->grp) g = nullptr;
}

void finish_request(fsm_server* S, Request* r, fsm_status st, Clock::time_point t) {
  r->status = st;
  r->done = true;
  r->t_done = t;
  if (st == FSM_OK) {
    ++S->completed;
    S->lat_ms.push_back(std::chrono::duration<double, std::milli>(t - r->t_submit).count());
    S->t_last = std::max(S->t_last, t);
  } else {
    ++S->failed;
    r->msg = fsm_last_error();
  }
}

// Outputs of a completed wave into its requests (mu held).
void wave_retire(fsm_server* S, Wave* w) {
  {
    float t[3] = {0, 0, 0};
    bool ok = true;
    for (int k = 0; k < 3 && ok; ++k) {
      ok = w->ev[k] && w->ev[k + 1] && cudaEventElapsedTime(&t[k], w->ev[k], w->ev[k + 1]) == cudaSuccess;
    }
    if (ok) {
      S->sum_h2d += t[0];
      S->sum_kernels += t[1];
      S->sum_d2h += t[2];
      S->sum_plan += w->plan_ms;
      S->sum_stage += w->stage_ms;
      S->sum_events += (long long)w->reqs.size();
      ++S->timed_waves;
    } else {
      cudaGetLastError();
    }
    for (Request* r : w->reqs) {
      S->sum_queue += std::chrono::duration<double, std::milli>(r->t_wave - r->t_submit).count();
      ++S->queued_reqs;
    }
  }
  const int* err = reinterpret_cast<const int*>(w->hout + w->houtbytes - 16);
  fsm_status st = FSM_OK;
  if (err[1] != 0) st = FSM_ERR_TIMEOUT;
  else if (err[0] != 0) st = FSM_ERR_CUDA;
  if (st != FSM_OK) set_last_error("server wave: kernel error words set");
  const float* out = reinterpret_cast<const float*>(w->hout);
  auto* ob = new OutBlock{w->hout, w->houtbytes, (int)w->reqs.size()};
  for (size_t i = 0; i < w->reqs.size(); ++i) {
    Request* r = w->reqs[i];
    const EventPlan& P = w->b->plans[i];
    r->dim = (size_t)P.DIM;
    r->baryon = P.baryon;
    r->ob = ob;
    for (int g = 0; g < kOutGroups; ++g) {
      const bool have = w->hgrp[g] != (size_t)-1 && (g < 6 || P.baryon);
      r->grp[g] = have ? out + w->hgrp[g] + (w->b->out_goff[i][g] - w->b->group_off[g]) : nullptr;
    }
    fill_info(P, &r->info);
    finish_request(S, r, st, w->t_done);
  }
  wave_release(S, w, /*keep_out=*/true);
  S->cv_done.notify_all();
}

// Builds and enqueues one wave from the head of the queue on stream `slot`
// (mu held on entry and exit; released while planning).  Returns false when
// nothing could be admitted for lack of memory.
constexpr int kBacklogMix = 8;  // queued requests above which waves mix event kinds
// 3D events per wave at most: one 131^2 x 51 event already fills the GPU, so
// batching more of them gains no kernel efficiency, while every one added
// delays the results of the others by its kernels and its output copy
constexpr int kMax3DPerWave = 2;

bool queue_has_2d(const fsm_server* S) {
  for (const Request* r : S->queue)
    if (r->p.DIM_ETA == 1) return true;
  return false;
}

bool wave_launch(fsm_server* S, std::unique_lock<std::mutex>& lk, int slot) {
  const int cap = S->opts.max_wave_events;
  std::vector<Request*> take;
  // With a short queue a wave holds requests of one kind, that of the oldest
  // one (boost-invariant or 3D), in arrival order: a 2D request then does not
  // wait for the milliseconds of a 3D event sharing its wave.  Under a backlog
  // waves take the queue in order, mixed, for throughput.  The stream reserved
  // for boost-invariant waves takes 2D requests only.
  const bool only2d = slot == S->slot_2d;
  const bool kind3d = !only2d && S->queue.front()->p.DIM_ETA > 1;
  const bool mixed = !only2d && (int)S->queue.size() > kBacklogMix;
  int n3d = 0;
  for (auto it = S->queue.begin(); it != S->queue.end() && (int)take.size() < cap;) {
    const bool is3d = (*it)->p.DIM_ETA > 1;
    if ((mixed || is3d == kind3d) && !(is3d && n3d >= kMax3DPerWave)) {
      n3d += is3d ? 1 : 0;
      take.push_back(*it);
      it = S->queue.erase(it);
    } else {
      ++it;
    }
  }
  cudaStream_t s = S->streams[slot];
  const Clock::time_point t_take = Clock::now();
  for (Request* r : take) r->t_wave = t_take;
  while (!take.empty()) {
    auto* w = new Wave();
    w->slot = slot;
    w->reqs = take;
    w->t_start = Clock::now();
    std::vector<fsm_params> ps(take.size());
    std::vector<const float*> he(take.size());
    for (size_t i = 0; i < take.size(); ++i) {
      ps[i] = take[i]->p;
      he[i] = take[i]->e.data();
    }
    auto* user = new std::pair<fsm_server*, Wave*>(S, w);
    BatchMem mem;
    mem.user = user;
    mem.dev = pool_dev;
    mem.host = pool_host;
    mem.stream = s;
    mem.grouped_out = true;
    fsm_batch* b = nullptr;
    // planning runs without the lock; the pools are only touched by this thread
    lk.unlock();
    fsm_status st = batch_build(S->ctx, (int)take.size(), ps.data(), he.data(), nullptr, nullptr,
                                nullptr, &b, &mem);
    const Clock::time_point t_planned = Clock::now();
    w->plan_ms = std::chrono::duration<double, std::milli>(t_planned - w->t_start).count();
    lk.lock();
    if (st == FSM_OK) {
      w->b = b;
      w->hinbytes = b->in_slab_bytes;
      size_t kept = 0;
      for (int g = 0; g < kOutGroups; ++g) {
        const bool keep = (S->opts.output_mask & (1u << g)) && b->group_elems[g] > 0;
        w->hgrp[g] = keep ? kept : (size_t)-1;
        if (keep) kept += b->group_elems[g];
      }
      w->houtbytes = kept * 4 + 16;
      w->hin = S->hpool.alloc(w->hinbytes);
      w->hout = w->hin ? S->hpool.alloc(w->houtbytes) : nullptr;
      if (!w->hin || !w->hout) st = FSM_ERR_OUT_OF_MEMORY;
    }
    if (st == FSM_OK) {
      // inputs into the pinned slab, without the lock (the slab is this
      // wave's, the requests' inputs are read-only after submit), large ones
      // on several threads; then the stream work of the wave
      lk.unlock();
      {
        // all inputs of the wave in 1 MiB pieces, spread over the worker
        // pool in one job once the wave holds 2 MiB or more
        struct Piece {
          char* dst;
          const char* src;
          size_t bytes;
        };
        constexpr size_t kPiece = (size_t)1 << 20;
        std::vector<Piece> pieces;
        size_t total = 0;
        auto add = [&](float* dst, const float* src, size_t n) {
          for (size_t o = 0; o < n * 4; o += kPiece)
            pieces.push_back(Piece{reinterpret_cast<char*>(dst) + o, reinterpret_cast<const char*>(src) + o,
                                   std::min(kPiece, n * 4 - o)});
          total += n * 4;
        };
        for (size_t i = 0; i < take.size(); ++i) {
          float* dst = reinterpret_cast<float*>(w->hin) + b->in_off[i];
          const size_t n = take[i]->e.size();
          add(dst, take[i]->e.data(), n);
          if (b->plans[i].baryon) add(dst + n, take[i]->nB.data(), n);
        }
        parallel_for((int)pieces.size(), total >= 2 * kPiece ? host_threads() : 1, [&](int k) {
          std::memcpy(pieces[k].dst, pieces[k].src, pieces[k].bytes);
        });
      }
      w->stage_ms = std::chrono::duration<double, std::milli>(Clock::now() - t_planned).count();
      lk.lock();
      for (auto& e : w->ev) e = take_event(S);
      if (w->ev[0]) cudaEventRecord(w->ev[0], s);
      cudaError_t ce = cudaMemcpyAsync(b->d_mem + b->in_slab_off, w->hin, b->in_slab_bytes,
                                       cudaMemcpyHostToDevice, s);
      if (w->ev[1]) cudaEventRecord(w->ev[1], s);
      if (ce == cudaSuccess) st = enqueue(b, s, false);
      else st = FSM_ERR_CUDA;
      if (w->ev[2]) cudaEventRecord(w->ev[2], s);
      if (st == FSM_OK) {
        // only the output groups the server keeps: one copy per run of kept
        // groups that lie back to back in the slab and in the pinned buffer
        ce = cudaSuccess;
        for (int g = 0; g < kOutGroups && ce == cudaSuccess;) {
          if (w->hgrp[g] == (size_t)-1) {
            ++g;
            continue;
          }
          size_t elems = b->group_elems[g];
          int h = g + 1;
          while (h < kOutGroups && w->hgrp[h] == w->hgrp[g] + elems &&
                 b->group_off[h] == b->group_off[g] + elems) {
            elems += b->group_elems[h];
            ++h;
          }
          ce = cudaMemcpyAsync(w->hout + w->hgrp[g] * 4, b->d_mem + b->out_slab_off + b->group_off[g] * 4,
                               elems * 4, cudaMemcpyDeviceToHost, s);
          g = h;
        }
        if (ce == cudaSuccess)
          ce = cudaMemcpyAsync(w->hout + w->houtbytes - 16, b->d_err, 16, cudaMemcpyDeviceToHost, s);
        if (ce == cudaSuccess && w->ev[3]) ce = cudaEventRecord(w->ev[3], s);
        if (ce == cudaSuccess) ce = cudaLaunchHostFunc(s, wave_done_cb, user);
        if (ce != cudaSuccess) {
          set_last_error(std::string("server wave: ") + cudaGetErrorString(ce));
          st = FSM_ERR_CUDA;
        }
      }
      if (st != FSM_OK) {
        // the stream may still be using the regions: wait before releasing them
        lk.unlock();
        cudaStreamSynchronize(s);
        lk.lock();
        wave_release(S, w);
        for (Request* r : take) finish_request(S, r, st, Clock::now());
        delete w;
        delete user;
        S->cv_done.notify_all();
        return true;
      }
      ++S->waves;
      S->slot_wave[slot] = w;
      return true;
    }
    // planning error of some event, or the pools are full
    wave_release(S, w);
    delete w;
    delete user;
    if (st == FSM_ERR_OUT_OF_MEMORY) {
      if (take.size() > 1) {  // retry with the first half, requeue the rest in order
        const size_t h = take.size() / 2;
        for (size_t i = take.size(); i-- > h;) S->queue.push_front(take[i]);
        take.resize(h);
        continue;
      }
      if (S->dpool.used() != 0 || S->hpool.used() != 0) {
        // memory is held by waves in flight or by outputs not yet polled: wait
        S->queue.push_front(take[0]);
        return false;
      }
      set_last_error("request does not fit the server's memory budgets");
      finish_request(S, take[0], FSM_ERR_TOO_LARGE, Clock::now());
      S->cv_done.notify_all();
      return true;
    }
    // invalid parameters: fail the requests one by one so that one bad event
    // does not fail its neighbours
    if (take.size() > 1) {
      for (size_t i = take.size(); i-- > 1;) S->queue.push_front(take[i]);
      take.resize(1);
      continue;
    }
    finish_request(S, take[0], st, Clock::now());
    S->cv_done.notify_all();
    return true;
  }
  return true;
}

void scheduler(fsm_server* S) {
  cudaSetDevice(S->ctx->device);
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    const unsigned long long gen = S->wake_gen;
    // retire completed waves
    for (size_t k = 0; k < S->slot_wave.size(); ++k) {
      Wave* w = S->slot_wave[k];
      if (w && w->done) {
        wave_retire(S, w);
        delete w;
        S->slot_wave[k] = nullptr;
        S->mem_wait = false;
      }
    }
    bool inflight = false;
    for (Wave* x : S->slot_wave) inflight = inflight || (x != nullptr);
    if (S->stopping && S->queue.empty() && !inflight) break;
    // admit
    bool launched = false;
    if (!S->mem_wait) {
      for (size_t k = 0; k < S->slot_wave.size() && !S->queue.empty(); ++k) {
        if (S->slot_wave[k]) continue;
        if ((int)k == S->slot_2d && !queue_has_2d(S)) continue;
        const unsigned long long g0 = S->wake_gen;
        if (!wave_launch(S, lk, (int)k)) {
          // wait for memory only if none was freed while the wave was planned
          if (S->wake_gen == g0) S->mem_wait = true;
          break;
        }
        launched = true;
      }
    }
    if (launched) continue;
    if (S->wake_gen != gen) continue;  // something happened while mu was released
    S->cv.wait(lk);
  }
}

}  // namespace

extern "C" fsm_status fsm_server_start(fsm_server** out, const fsm_server_opts* opts) {
  if (!out) return FSM_ERR_INVALID_ARG;
  *out = nullptr;
  std::unique_ptr<fsm_server> S(new fsm_server());
  if (opts) S->opts = *opts;
  if (S->opts.hbm_budget_bytes == 0) S->opts.hbm_budget_bytes = (size_t)8 << 30;
  if (S->opts.host_budget_bytes == 0) S->opts.host_budget_bytes = (size_t)2 << 30;
  if (S->opts.max_wave_events <= 0) S->opts.max_wave_events = 512;
  if (S->opts.streams <= 0) S->opts.streams = 4;
  if (S->opts.output_mask == 0) S->opts.output_mask = FSM_OUT_ALL;
  fsm_ctx_opts co{S->opts.device, 0};
  fsm_status st = fsm_ctx_create(&S->ctx, &co);
  if (st != FSM_OK) return st;
  cudaError_t ce = cudaMalloc(&S->d_pool, S->opts.hbm_budget_bytes);
  if (ce == cudaSuccess) ce = cudaHostAlloc(&S->h_pool, S->opts.host_budget_bytes, cudaHostAllocDefault);
  if (ce != cudaSuccess) {
    cudaGetLastError();
    set_last_error(std::string("server pools: ") + cudaGetErrorString(ce));
    if (S->d_pool) cudaFree(S->d_pool);
    fsm_ctx_destroy(S->ctx);
    return FSM_ERR_OUT_OF_MEMORY;
  }
  S->dpool.reset(S->d_pool, S->opts.hbm_budget_bytes);
  S->hpool.reset(S->h_pool, S->opts.host_budget_bytes);
  S->streams.resize(S->opts.streams + (S->opts.stream_2d ? 1 : 0));
  if (S->opts.stream_2d) S->slot_2d = S->opts.streams;
  for (auto& s : S->streams) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  S->slot_wave.assign(S->streams.size(), nullptr);
  fsm_server* raw = S.get();
  S->th = std::thread(scheduler, raw);
  *out = S.release();
  return FSM_OK;
}

extern "C" fsm_status fsm_server_submit(fsm_server* S, const fsm_params* p, const float* e_gev,
                                        const float* nB, long long* id) {
  if (!S || !p || !e_gev || !id) return FSM_ERR_INVALID_ARG;
  const long long dim = (long long)p->DIM_X * p->DIM_Y * p->DIM_ETA;
  if (p->DIM_X < 1 || p->DIM_Y < 1 || p->DIM_ETA < 1 || dim > (1ll << 30)) {
    set_last_error("fsm_server_submit: invalid grid");
    return FSM_ERR_INVALID_ARG;
  }
  if (p->BARYON && !nB) {
    set_last_error("fsm_server_submit: BARYON = 1 needs the baryon density");
    return FSM_ERR_INVALID_ARG;
  }
  auto* r = new Request();
  r->p = *p;
  fsm_params_derive(&r->p);
  r->e.assign(e_gev, e_gev + dim);
  if (p->BARYON) r->nB.assign(nB, nB + dim);
  {
    std::lock_guard<std::mutex> g(S->mu);
    if (S->stopping) {
      delete r;
      set_last_error("fsm_server_submit: server is stopping");
      return FSM_ERR_CANCELLED;
    }
    r->id = S->next_id++;
    r->t_submit = Clock::now();
    if (!S->have_first) {
      S->t_first = r->t_submit;
      S->have_first = true;
    }
    ++S->submitted;
    S->reqs[r->id] = r;
    S->queue.push_back(r);
    *id = r->id;
    ++S->wake_gen;
  }
  S->cv.notify_all();
  return FSM_OK;
}

extern "C" fsm_status fsm_server_poll(fsm_server* S, long long id, const fsm_outputs* host_out,
                                      fsm_run_info* info, double timeout_ms, int* done) {
  if (!S || !done) return FSM_ERR_INVALID_ARG;
  *done = 0;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) {
    set_last_error("fsm_server_poll: unknown request id");
    return FSM_ERR_INVALID_ARG;
  }
  Request* r = it->second;
  if (!r->done && timeout_ms != 0.0) {
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0) S->cv_done.wait(lk, pred);
    else S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred);
  }
  if (!r->done) return FSM_OK;
  *done = 1;
  const fsm_status st = r->status;
  if (st == FSM_OK && host_out) {
    const size_t n = r->dim;
    float* dst[kOutGroups] = {host_out->T, host_out->e,  host_out->P, host_out->Pi, host_out->u,
                              host_out->pi, host_out->J, host_out->nB, host_out->V};
    for (int g = 0; g < kOutGroups; ++g)
      if (dst[g] && r->grp[g]) std::memcpy(dst[g], r->grp[g], (size_t)kOutGroupComps[g] * n * 4);
  }
  if (info) *info = r->info;
  if (st != FSM_OK) set_last_error(r->msg);
  drop_output(S, r);
  S->reqs.erase(it);
  delete r;
  return st;
}

extern "C" fsm_status fsm_server_poll_view(fsm_server* S, long long id, fsm_outputs* views,
                                           fsm_run_info* info, double timeout_ms, int* done) {
  if (!S || !done || !views) return FSM_ERR_INVALID_ARG;
  *done = 0;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) {
    set_last_error("fsm_server_poll_view: unknown request id");
    return FSM_ERR_INVALID_ARG;
  }
  Request* r = it->second;
  if (!r->done && timeout_ms != 0.0) {
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0) S->cv_done.wait(lk, pred);
    else S->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), pred);
  }
  if (!r->done) return FSM_OK;
  *done = 1;
  float** dst[kOutGroups] = {&views->T, &views->e,  &views->P,  &views->Pi, &views->u,
                             &views->pi, &views->J, &views->nB, &views->V};
  for (int g = 0; g < kOutGroups; ++g) *dst[g] = const_cast<float*>(r->grp[g]);
  if (info) *info = r->info;
  if (r->status != FSM_OK) set_last_error(r->msg);
  return r->status;
}

extern "C" fsm_status fsm_server_release(fsm_server* S, long long id) {
  if (!S) return FSM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end() || !it->second->done) {
    set_last_error("fsm_server_release: unknown or unfinished request id");
    return FSM_ERR_INVALID_ARG;
  }
  drop_output(S, it->second);
  delete it->second;
  S->reqs.erase(it);
  return FSM_OK;
}

extern "C" fsm_status fsm_server_stats_get(fsm_server* S, fsm_server_stats* st) {
  if (!S || !st) return FSM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(S->mu);
  *st = fsm_server_stats{};
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->failed = S->failed;
  st->waves = S->waves;
  if (!S->lat_ms.empty()) {
    std::vector<double> v = S->lat_ms;
    std::sort(v.begin(), v.end());
    auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)(f * (double)v.size()))]; };
    st->p50_ms = q(0.50);
    st->p99_ms = q(0.99);
    st->max_ms = v.back();
    const double span = std::chrono::duration<double>(S->t_last - S->t_first).count();
    st->events_per_s = span > 0 ? (double)S->completed / span : 0.0;
  }
  return FSM_OK;
}

extern "C" fsm_status fsm_server_breakdown_get(fsm_server* S, fsm_server_breakdown* bd) {
  if (!S || !bd) return FSM_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(S->mu);
  *bd = fsm_server_breakdown{};
  const double n = (double)std::max<long long>(S->timed_waves, 1);
  bd->waves = S->timed_waves;
  bd->events_per_wave = (double)S->sum_events / n;
  bd->plan_ms = S->sum_plan / n;
  bd->stage_ms = S->sum_stage / n;
  bd->h2d_ms = S->sum_h2d / n;
  bd->kernels_ms = S->sum_kernels / n;
  bd->d2h_ms = S->sum_d2h / n;
  bd->queue_ms = S->queued_reqs ? S->sum_queue / (double)S->queued_reqs : 0.0;
  const double span = std::chrono::duration<double, std::milli>(S->t_last - S->t_first).count();
  bd->device_busy = span > 0 ? (S->sum_h2d + S->sum_kernels + S->sum_d2h) / span : 0.0;
  bd->kernel_busy = span > 0 ? S->sum_kernels / span : 0.0;
  return FSM_OK;
}

extern "C" fsm_status fsm_server_stop(fsm_server* S) {
  if (!S) return FSM_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stopping = true;
    // queued requests are cancelled; waves in flight finish
    for (Request* r : S->queue) finish_request(S, r, FSM_ERR_CANCELLED, Clock::now());
    S->queue.clear();
    ++S->wake_gen;
  }
  S->cv.notify_all();
  S->cv_done.notify_all();
  if (S->th.joinable()) S->th.join();
  for (auto& kv : S->reqs) {
    drop_output(S, kv.second);
    delete kv.second;
  }
  for (auto& s : S->streams) cudaStreamDestroy(s);
  for (auto e : S->event_pool) cudaEventDestroy(e);
  cudaFreeHost(S->h_pool);
  cudaFree(S->d_pool);
  fsm_ctx_destroy(S->ctx);
  delete S;
  return FSM_OK;
}
