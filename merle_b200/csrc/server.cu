// server.cu - the serving loop: a dispatcher thread that batches queued
// queries into launches on one resident engine, with admission by the
// device bytes each request's group table and intermediate bitmaps need.
//
// No counterpart in the reference, whose drivers run a fixed query list once
// (ssb/ssbdemo.cu); the launches it issues are the engine's own batched scan
// (mb_engine_enqueue_batch) and plain path (run_lowered), so every answer is
// the one the engine gives the query alone.
//
// A batched-mode launch runs its queries either through the persistent
// batched scan or one after another on the plain path: a launch of few
// queries pays the scan's per-tile cost (one warp per query and tile) for
// little shared reading.  An online cost model of both kinds (device times of
// completed launches) picks the cheaper for each launch's size.
//
// Life of a request: submit (queued, t_submit) -> admitted into a launch by
// the dispatcher (reservation taken, group table carved from the arena,
// t_launch) -> the launch's completion event fires, its group tables come
// back through a pinned mirror of the arena, the request's values go to the
// caller's buffer (t_done) -> wait() hands out its record.  Launches run in
// order on the engine stream, so the arena is a ring: space is taken at the
// head and given back at the tail as launches complete.
#include <string.h>
#include <math.h>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>
#include "engine.h"

namespace mb {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  mb_query q{};
  int64_t *out_host = nullptr;
  uint32_t ngroups = 1;
  uint64_t foot = 0;  // admission bytes
  mb_plan plan{};     // plain mode: the plan it runs with
  bool planned = false, planning = false;
  bool done = false;
  mb_request_info info{};
};

// a batched-mode plain launch plans its query and up to this many queued
// ones in one learned-planner call
constexpr size_t PLAN_AHEAD = 15;

struct Launch {
  std::vector<Request *> reqs;
  bool scan = false;  // the batched scan (else the plain path, query by query)
  uint64_t off = 0, bytes = 0;  // arena bytes [off, off + bytes)
  uint64_t reserved = 0;
  uint32_t index = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  mb_status st = MB_OK;
  uint32_t *err = nullptr;  // pinned copy of the device error word
};

// Online cost model of the batched server's two launch kinds, from the
// device times of completed launches: the plain path as a time per query
// (decayed mean over about the last 128 queries), the batched scan as
// a + b * queries (a least-squares fit with exponentially decaying weights),
// and the arrival rate (decayed mean gap between submits).
//
// While the plain path alone keeps up with the arrivals (plain time per query
// below OVERLOAD of the mean gap) the queue stays short and what matters is
// latency: n queued queries take the batched scan only when that lowers the
// sum of their completion times, a + b * n < plain * (n + 1) / 2 (one after
// another they complete at plain, 2 plain, ..., n plain).  Past that load
// the queue grows and throughput decides: the scan when a + b * n < n * plain,
// or when n is beyond the batch sizes the fit has seen.
struct CostModel {
  // plain: ms per query, a decayed mean over the recent plain queries (the
  // load is the mean service time over the mean gap, not the latest query's)
  double p_ms = 0, p_sum = 0, p_w = 0;
  uint32_t p_cnt = 0;
  double w = 0, wn = 0, wt = 0, wnn = 0, wnt = 0;  // weighted sums over scan launches
  uint32_t b_cnt = 0, b_nmax = 0;                  // scan launches seen, their largest size
  // mean gap between arrivals: decayed sums of gaps and of weights, so that
  // the first few gaps give their plain mean rather than the first alone
  double g_sum = 0, g_w = 0, last_us = -1;
  static constexpr double DECAY = 0.97, GAP_DECAY = 1 - 1.0 / 128, OVERLOAD = 1.0;
  void add_arrival(double t_us) {
    if (last_us >= 0) {
      g_sum = GAP_DECAY * g_sum + (t_us - last_us) * 1e-3;
      g_w = GAP_DECAY * g_w + 1;
    }
    last_us = t_us;
  }
  bool overloaded() const { return p_cnt && g_w >= 8 && p_ms * g_w >= OVERLOAD * g_sum; }
  void add_plain(uint32_t n, float ms) {
    const double k = (double)(n ? n : 1), d = pow(GAP_DECAY, k);
    p_sum = d * p_sum + ms;
    p_w = d * p_w + k;
    p_ms = p_sum / p_w;
    ++p_cnt;
  }
  void add_scan(uint32_t n, float ms) {
    w = DECAY * w + 1, wn = DECAY * wn + n, wt = DECAY * wt + ms;
    wnn = DECAY * wnn + (double)n * n, wnt = DECAY * wnt + (double)n * ms;
    ++b_cnt;
    if (n > b_nmax) b_nmax = n;
  }
  bool ready() const { return p_cnt >= 3 && b_cnt >= 3; }
  bool scan_better(uint32_t n) const {
    const bool over = overloaded();
    // under overload, beyond the largest batch the fit has seen (and at
    // least 8 queries) the scan is tried: a line fitted on small batches
    // says little about large
    if (over && n > b_nmax && n >= 8) return true;
    const double var = w * wnn - wn * wn;
    double a = wt / w, b = 0;
    if (var > 1e-9 * w * w) {  // two or more distinct batch sizes seen
      b = (w * wnt - wn * wt) / var;
      a = (wt - b * wn) / w;
      if (b < 0) b = 0, a = wt / w;
    }
    return over ? a + b * n < n * p_ms : a + b * n < 0.5 * (n + 1) * p_ms;
  }
};

uint64_t splitmix(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace
}  // namespace mb

using namespace mb;

struct mb_server {
  mb_engine *eng = nullptr;
  mb_server_opts o{};
  // arena: device group tables and their pinned mirror
  char *arena = nullptr, *mirror = nullptr;
  uint64_t cap = 0, head = 0, tail = 0, used = 0;
  uint64_t reserved = 0;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request *> pending;
  std::unordered_map<uint64_t, Request *> reqs;
  std::deque<Launch *> inflight;
  std::vector<Launch *> free_launches;
  uint64_t next_id = 1;
  uint32_t next_launch = 0;
  bool stop = false;
  std::thread th;
  mb_server_stats stats{};
  CostModel cost;
  // injected faults (host side)
  uint32_t f_alloc = 0, f_launch = 0, f_slow = 0, f_slow_us = 0;

  double now_us() const { return std::chrono::duration<double, std::micro>(Clock::now() - t0).count(); }
  void run();
  bool launch_some(std::unique_lock<std::mutex> &lk);
  void complete(Launch *L);
  void finish(Request *r, int32_t status);
  uint64_t footprint(const mb_query &q, uint32_t *plan_idx, mb_plan *plan);
  uint64_t inter_bytes(const mb_query &q, const mb_plan &plan);
};

// Bytes a request reserves: its group table and row count in the arena, and
// the intermediate bitmaps its plan writes (materialised predicates: a
// (certain, uncertain) pair each; a materialised plan: its result pair and
// the row list).
uint64_t mb_server::footprint(const mb_query &q, uint32_t *plan_idx, mb_plan *plan) {
  Engine &E = eng->E;
  const uint64_t table = 8ull * (query_ngroups(q) + 1);
  memset(plan, 0, sizeof(*plan));
  plan->kind = MB_PLAN_FUSED;
  plan->launch.grp_strategy = MB_GRP_AUTO;
  *plan_idx = 0;
  if (o.mode == MB_SERVE_PLAIN && o.use_planner && E.planner) {
    if (mb_engine_plan_learned(eng, &q, 1, plan, plan_idx) != MB_OK) {
      mb_engine_plan_rule(eng, &q, plan);
      *plan_idx = 0;
    }
  }
  return table + inter_bytes(q, *plan);
}

// Intermediate bitmap bytes a plan writes: a (certain, uncertain) pair per
// materialised predicate; the materialised plan's result pair and row list.
uint64_t mb_server::inter_bytes(const mb_query &q, const mb_plan &plan) {
  Engine &E = eng->E;
  const uint64_t W = E.stride * 4;
  uint64_t inter = 0;
  if (plan.kind == MB_PLAN_MATERIALISED) inter = 2 * W + (E.nrows + 1) * 4;
  if (plan.materialise && plan.kind == MB_PLAN_FUSED) {
    Lowered L;
    if (lower_query(E, q, plan, L) == MB_OK) {
      uint32_t nmat = 0;
      for (uint32_t c = 0; c < L.prg.ncols; ++c)
        if (plan.materialise & (1u << L.col_pred[c])) ++nmat;
      inter = 2ull * nmat * W;
    }
  }
  return inter;
}

void mb_server::finish(Request *r, int32_t status) {
  r->info.status = status;
  r->info.t_done_us = now_us();
  r->done = true;
  if (status == MB_OK) ++stats.completed;
  else if (status == MB_ERR_REJECTED) ++stats.rejected;
  else if (status == MB_ERR_CANCELLED) ++stats.cancelled;
  else ++stats.failed;
}

// Takes queued requests into one launch and enqueues it (called with the
// lock held; the lock is released around the engine calls).  Returns false
// if nothing could launch.
bool mb_server::launch_some(std::unique_lock<std::mutex> &lk) {
  NvtxRange nvtx_("mb_server launch");
  const uint32_t maxb = o.mode == MB_SERVE_PLAIN ? 1 : o.max_batch;
  if (o.mode == MB_SERVE_PLAIN && !pending.front()->planned) {
    // a plain-mode request is planned when it reaches the front: its plan
    // decides the intermediate bytes it reserves.  Cancel leaves a request
    // alone while it is being planned, and only this thread pops the queue.
    Request *r = pending.front();
    r->planning = true;
    lk.unlock();
    mb_plan pl;
    uint32_t pi = 0;
    const uint64_t f = footprint(r->q, &pi, &pl);
    lk.lock();
    r->plan = pl;
    r->info.plan = pi;
    r->foot = f;
    r->planned = true;
    r->planning = false;
  }
  std::vector<Request *> take;
  uint64_t res = 0, bytes = 0;
  while (!pending.empty() && take.size() < maxb) {
    Request *r = pending.front();
    if (o.mode == MB_SERVE_PLAIN && !r->planned) break;
    const uint64_t tb = 8ull * (r->ngroups + 1);
    if (r->foot > o.mem_budget || tb > cap) {  // can never fit
      pending.pop_front();
      finish(r, MB_ERR_REJECTED);
      cv_done.notify_all();
      continue;
    }
    if (reserved + res + r->foot > o.mem_budget) break;  // waits for launches in flight
    take.push_back(r);
    pending.pop_front();
    res += r->foot;
    bytes += tb;
  }
  if (take.empty()) return false;
  // batched mode: the batched scan takes the whole lot (a fixed min_batch,
  // or the cost model once it has seen both kinds; until then 6 queries
  // when the plain path falls behind the arrivals);
  // otherwise the plain path runs one query per launch and the rest stay
  // queued for the next launches, so each answer returns when its own query
  // is done rather than when the last of the lot is
  const uint32_t nt = (uint32_t)take.size();
  bool scan;
  if (o.mode == MB_SERVE_PLAIN) scan = false;
  else if (o.min_batch) scan = nt >= o.min_batch;
  else scan = cost.ready() ? nt >= 2 && cost.scan_better(nt) : nt >= 6 && cost.overloaded();
  if (!scan && nt > 1) {
    for (size_t i = take.size(); i-- > 1;) {
      pending.push_front(take[i]);
      res -= take[i]->foot;
      bytes -= 8ull * (take[i]->ngroups + 1);
    }
    take.resize(1);
  }
  // Arena space, contiguous.  Launches complete in stream order, so the live
  // tables are [tail, head) or, once the head wrapped, [tail, end) + [0, head).
  uint64_t off = 0;
  bool fits;
  if (inflight.empty()) {
    head = tail = 0;
    fits = bytes <= cap;
  } else if (head > tail) {
    if (head + bytes <= cap) off = head, fits = true;
    else fits = bytes <= tail;  // wrap to 0
  } else {
    off = head;
    fits = head + bytes <= tail;
  }
  if (!fits) {  // put them back and wait for the oldest launch
    for (auto it = take.rbegin(); it != take.rend(); ++it) pending.push_front(*it);
    return false;
  }
  Launch *L;
  if (!free_launches.empty()) {
    L = free_launches.back();
    free_launches.pop_back();
  } else {
    L = new Launch();
    if (cudaEventCreate(&L->ev0) != cudaSuccess || cudaEventCreate(&L->ev1) != cudaSuccess ||
        cudaMallocHost(&L->err, 16) != cudaSuccess) {
      delete L;
      for (auto it = take.rbegin(); it != take.rend(); ++it) pending.push_front(*it);
      return false;
    }
  }
  L->reqs = take;
  L->scan = scan;
  L->off = off;
  L->bytes = bytes;
  L->reserved = res;
  L->index = next_launch++;
  L->st = MB_OK;
  memset(L->err, 0, 16);
  reserved += res;
  if (reserved > stats.peak_reserved) stats.peak_reserved = reserved;
  head = off + bytes;
  used += bytes;
  uint32_t slow = 0;
  bool f_a = false, f_l = false;
  if (f_slow) --f_slow, slow = f_slow_us;
  if (f_alloc) --f_alloc, f_a = true;
  else if (f_launch) --f_launch, f_l = true;
  // a batched-mode launch on the plain path plans with the learned planner
  // when it is on: its query together with up to PLAN_AHEAD queued ones not
  // yet planned, so that one sample wait and one network pass serve several
  // launches (cancel leaves a request alone while it is being planned)
  std::vector<Request *> ahead;
  const bool learn = o.mode == MB_SERVE_BATCHED && !scan && o.use_planner && eng->E.planner && !f_a && !f_l;
  if (learn && !take[0]->planned) {
    ahead.push_back(take[0]);
    for (Request *r : pending) {
      if (ahead.size() > PLAN_AHEAD) break;
      if (!r->planned && !r->planning) ahead.push_back(r);
    }
    for (Request *r : ahead) r->planning = true;
  }
  inflight.push_back(L);
  ++stats.launches;
  stats.launched_queries += take.size();
  const double tl = now_us();
  for (Request *r : take) {
    r->info.launch = L->index;
    r->info.batch_size = (uint32_t)take.size();
    r->info.t_launch_us = tl;
  }
  lk.unlock();
  if (slow) std::this_thread::sleep_for(std::chrono::microseconds(slow));
  Engine &E = eng->E;
  cudaStream_t st = E.stream;
  const uint32_t n = (uint32_t)take.size();
  std::vector<mb_query> qs(n);
  uint64_t total = 0;
  for (uint32_t i = 0; i < n; ++i) qs[i] = take[i]->q, total += take[i]->ngroups;
  int64_t *out_dev = reinterpret_cast<int64_t *>(arena + off);
  uint64_t *nq_dev = reinterpret_cast<uint64_t *>(out_dev + total);
  // planning comes before the launch's first event (it waits for its sample
  // pass, on the planner's own stream)
  std::vector<mb_plan> ahead_plans(ahead.size());
  std::vector<uint32_t> ahead_pick(ahead.size(), 0);
  bool ahead_ok = false;
  if (!ahead.empty()) {
    std::vector<mb_query> aq(ahead.size());
    for (size_t i = 0; i < ahead.size(); ++i) aq[i] = ahead[i]->q;
    ahead_ok = mb_engine_plan_learned(eng, aq.data(), (uint32_t)aq.size(), ahead_plans.data(), ahead_pick.data()) ==
               MB_OK;
  }
  const bool learned = learn && (take[0]->planned || ahead_ok);
  const mb_plan *lplan = take[0]->planned ? &take[0]->plan : ahead_ok ? &ahead_plans[0] : nullptr;
  // intermediate bytes of the plans just made (take[0]'s, if planned here, is
  // extra[0]; one planned ahead earlier already carries its own in its foot)
  std::vector<uint64_t> extra(std::max<size_t>(1, ahead.size()), 0);
  if (ahead_ok)
    for (size_t i = 0; i < ahead.size(); ++i) extra[i] = inter_bytes(ahead[i]->q, ahead_plans[i]);
  if (learn) take[0]->info.plan = take[0]->planned ? take[0]->info.plan : ahead_ok ? ahead_pick[0] : 0;
  mb_status s = MB_OK;
  if (f_a) s = fail(MB_ERR_OOM, "serving: injected arena allocation failure");
  if (s == MB_OK && cudaEventRecord(L->ev0, st) != cudaSuccess) s = fail(MB_ERR_CUDA, "serving: event record");
  if (s == MB_OK && f_l) s = fail(MB_ERR_CUDA, "serving: injected launch failure");
  if (s == MB_OK) {
    if (o.mode == MB_SERVE_PLAIN) s = mb_engine_enqueue(eng, qs.data(), 1, &take[0]->plan, out_dev, nq_dev, 0);
    else if (!L->scan) s = mb_engine_enqueue(eng, qs.data(), n, learned ? lplan : nullptr, out_dev, nq_dev, 0);
    else {
      // the server's batch options, or, left all zero with a batch planner on
      // the engine, the learned batch plan of this launch's queries
      static const mb_batch_opts zero = {};
      const bool learned_batch = eng->E.batch_planner && memcmp(&o.batch, &zero, sizeof(zero)) == 0;
      s = mb_engine_enqueue_batch(eng, qs.data(), n, learned_batch ? nullptr : &o.batch, out_dev, nq_dev);
    }
  }
  if (s == MB_OK && cudaMemcpyAsync(mirror + off, arena + off, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    s = fail(MB_ERR_CUDA, "serving: result copy");
  if (s == MB_OK && cudaMemcpyAsync(L->err, device_error_word(), 16, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    s = fail(MB_ERR_CUDA, "serving: error word copy");
  cudaEventRecord(L->ev1, st);
  lk.lock();
  // a learned plan may write intermediate bitmaps: the queued requests
  // planned ahead reserve them when they are admitted; the launched one adds
  // them to its launch's reservation now
  for (size_t i = 0; i < ahead.size(); ++i) {
    Request *r = ahead[i];
    r->planning = false;
    if (ahead_ok) {
      r->plan = ahead_plans[i], r->info.plan = ahead_pick[i], r->planned = true;
      if (i > 0) r->foot += extra[i];
    }
  }
  if (learned && extra[0]) {
    L->reserved += extra[0];
    reserved += extra[0];
    if (reserved > stats.peak_reserved) stats.peak_reserved = reserved;
  }
  L->st = s;
  return true;
}

void mb_server::complete(Launch *L) {
  // lock held
  float ms = 0;
  cudaEventElapsedTime(&ms, L->ev0, L->ev1);
  mb_status s = L->st;
  if (s == MB_OK && L->err && L->err[0]) {
    s = MB_ERR_TIMEOUT;  // a bounded device wait ran out in this launch
    cudaMemsetAsync(device_error_word(), 0, 16, eng->E.stream);
  }
  const int64_t *base = reinterpret_cast<const int64_t *>(mirror + L->off);
  uint64_t total = 0;
  for (Request *r : L->reqs) total += r->ngroups;
  uint64_t o_ = 0;
  for (uint32_t i = 0; i < L->reqs.size(); ++i) {
    Request *r = L->reqs[i];
    if (s == MB_OK) {
      memcpy(r->out_host, base + o_, (size_t)r->ngroups * 8);
      r->info.nqual = (uint64_t)base[total + i];
    }
    o_ += r->ngroups;
    r->info.gpu_ms = s == MB_OK ? ms : 0.f;
    finish(r, s);
  }
  stats.gpu_ms += s == MB_OK ? ms : 0.0;
  if (L->scan) ++stats.scan_launches;
  if (s == MB_OK && o.mode == MB_SERVE_BATCHED) {
    if (L->scan) cost.add_scan((uint32_t)L->reqs.size(), ms);
    else cost.add_plain((uint32_t)L->reqs.size(), ms);
  }
  reserved -= L->reserved;
  used -= L->bytes;
  // the caller popped L: the oldest live tables now start at the next launch
  tail = inflight.empty() ? head : inflight.front()->off;
  L->reqs.clear();
  free_launches.push_back(L);
  cv_done.notify_all();
}

void mb_server::run() {
  cudaSetDevice(eng->E.device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    // completions, oldest first (launches finish in stream order)
    while (!inflight.empty()) {
      Launch *L = inflight.front();
      const cudaError_t q = cudaEventQuery(L->ev1);
      if (q == cudaErrorNotReady) break;
      inflight.pop_front();
      if (q != cudaSuccess && L->st == MB_OK) L->st = cuda_fail(q, "serving: launch");
      complete(L);
    }
    bool launched = false;
    if (!stop && inflight.size() < o.max_inflight && !pending.empty()) launched = launch_some(lk);
    if (stop && inflight.empty()) break;
    if (launched) continue;
    if (!inflight.empty()) {
      // the GPU is busy: poll its completion finely (latency matters more
      // than this thread's core)
      lk.unlock();
      std::this_thread::sleep_for(std::chrono::microseconds(5));
      lk.lock();
    } else {
      cv_work.wait_for(lk, std::chrono::milliseconds(2), [&] { return stop || !pending.empty(); });
    }
  }
  // requests still queued when the server stops
  while (!pending.empty()) {
    finish(pending.front(), MB_ERR_CANCELLED);
    pending.pop_front();
  }
  cv_done.notify_all();
}

extern "C" mb_status mb_server_create(mb_engine *e, const mb_server_opts *opts, mb_server **out) {
  if (!e || !out) return fail(MB_ERR_INVALID, "mb_server_create: NULL argument");
  *out = nullptr;
  mb_server_opts o;
  if (opts) o = *opts;
  else memset(&o, 0, sizeof(o));
  if (o.mem_budget == 0) o.mem_budget = 256ull << 20;
  if (o.max_batch == 0) o.max_batch = 64;
  if (o.max_inflight == 0) o.max_inflight = 2;
  if (o.mode > MB_SERVE_PLAIN || o.max_batch > MB_BATCH_MAX || o.max_inflight > 8 || o.mem_budget < 4096)
    return fail(MB_ERR_INVALID, "mb_server_create: options out of range");
  if (!e->E.indexed) return fail(MB_ERR_INVALID, "mb_server_create: the engine has no index");
  MB_CUDA(cudaSetDevice(e->E.device));
  mb_server *s = new (std::nothrow) mb_server();
  if (!s) return fail(MB_ERR_OOM, "mb_server_create: host allocation");
  s->eng = e;
  s->o = o;
  s->cap = round_up(o.mem_budget, 256);
  cudaError_t r = cudaMalloc(&s->arena, s->cap);
  if (r == cudaSuccess) r = cudaMallocHost(&s->mirror, s->cap);
  if (r != cudaSuccess) {
    cudaFree(s->arena);
    if (s->mirror) cudaFreeHost(s->mirror);
    delete s;
    return cuda_fail(r, "mb_server_create: arena");
  }
  if (!device_error_word()) {
    cudaFree(s->arena);
    cudaFreeHost(s->mirror);
    delete s;
    return fail(MB_ERR_OOM, "mb_server_create: device error word");
  }
  s->t0 = Clock::now();
  s->th = std::thread([s] { s->run(); });
  *out = s;
  return MB_OK;
}

extern "C" mb_status mb_server_destroy(mb_server *s) {
  if (!s) return MB_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->th.joinable()) s->th.join();
  cudaSetDevice(s->eng->E.device);
  cudaStreamSynchronize(s->eng->E.stream);
  for (Launch *L : s->free_launches) {
    cudaEventDestroy(L->ev0);
    cudaEventDestroy(L->ev1);
    cudaFreeHost(L->err);
    delete L;
  }
  for (auto &kv : s->reqs) delete kv.second;
  cudaFree(s->arena);
  cudaFreeHost(s->mirror);
  delete s;
  return MB_OK;
}

extern "C" mb_status mb_server_submit(mb_server *s, const mb_query *q, int64_t *out_host, uint64_t *id) {
  if (!s || !q || !out_host) return fail(MB_ERR_INVALID, "mb_server_submit: NULL argument");
  if (q->tmpl < 1 || q->tmpl > 4) return fail(MB_ERR_INVALID, "mb_server_submit: template %u", q->tmpl);
  Request *r = new (std::nothrow) Request();
  if (!r) return fail(MB_ERR_OOM, "mb_server_submit: host allocation");
  r->q = *q;
  r->out_host = out_host;
  r->ngroups = query_ngroups(*q);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      delete r;
      return fail(MB_ERR_INVALID, "mb_server_submit: the server is stopping");
    }
    // the batched scan writes no intermediate bitmaps: a request reserves
    // its group table (plain-mode requests add their plan's bitmaps when
    // they are planned)
    r->foot = 8ull * (r->ngroups + 1);
    r->id = s->next_id++;
    r->info.t_submit_us = s->now_us();
    s->cost.add_arrival(r->info.t_submit_us);
    s->reqs[r->id] = r;
    s->pending.push_back(r);
    ++s->stats.submitted;
    if (id) *id = r->id;
  }
  s->cv_work.notify_one();
  return MB_OK;
}

extern "C" mb_status mb_server_cancel(mb_server *s, uint64_t id) {
  if (!s) return fail(MB_ERR_INVALID, "mb_server_cancel: NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  for (auto it = s->pending.begin(); it != s->pending.end(); ++it)
    if ((*it)->id == id && !(*it)->planning) {
      Request *r = *it;
      s->pending.erase(it);
      s->finish(r, MB_ERR_CANCELLED);
      s->cv_done.notify_all();
      return MB_OK;
    }
  return fail(MB_ERR_INVALID, "mb_server_cancel: request %llu is not queued", (unsigned long long)id);
}

extern "C" mb_status mb_server_wait(mb_server *s, uint64_t id, int64_t timeout_ms, mb_request_info *info) {
  if (!s) return fail(MB_ERR_INVALID, "mb_server_wait: NULL server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return fail(MB_ERR_INVALID, "mb_server_wait: unknown request %llu", (unsigned long long)id);
  Request *r = it->second;
  if (timeout_ms < 0) s->cv_done.wait(lk, [&] { return r->done; });
  else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->done; }))
    return fail(MB_ERR_TIMEOUT, "mb_server_wait: request %llu not done", (unsigned long long)id);
  if (info) *info = r->info;
  s->reqs.erase(it);
  delete r;
  return MB_OK;
}

extern "C" mb_status mb_server_get_stats(mb_server *s, mb_server_stats *out) {
  if (!s || !out) return fail(MB_ERR_INVALID, "mb_server_get_stats: NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return MB_OK;
}

extern "C" mb_status mb_server_inject(mb_server *s, uint32_t fault, uint32_t count, uint32_t arg_us) {
  if (!s || fault > MB_FAULT_SLOW) return fail(MB_ERR_INVALID, "mb_server_inject: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (fault == MB_FAULT_ALLOC) s->f_alloc = count;
  if (fault == MB_FAULT_LAUNCH) s->f_launch = count;
  if (fault == MB_FAULT_SLOW) s->f_slow = count, s->f_slow_us = arg_us;
  return MB_OK;
}

extern "C" mb_status mb_poisson_arrivals(uint64_t seed, double rate_qps, uint32_t n, double *t_us) {
  if ((!t_us && n) || !(rate_qps > 0)) return fail(MB_ERR_INVALID, "mb_poisson_arrivals: bad argument");
  double t = 0;
  const uint64_t key = splitmix(seed ^ 0x5e7f1a2b3c4d5e6full);
  for (uint32_t i = 0; i < n; ++i) {
    const double u = ((splitmix(key + i) >> 11) + 0.5) / 9007199254740992.0;  // (0, 1)
    t += -log(u) / rate_qps * 1e6;
    t_us[i] = t;
  }
  return MB_OK;
}

extern "C" mb_status mb_server_run_load(mb_server *s, const mb_query *qs, uint32_t n, double rate_qps, uint64_t seed,
                                        int64_t *out_host, mb_request_info *info) {
  if (!s || (n && (!qs || !out_host || !info))) return fail(MB_ERR_INVALID, "mb_server_run_load: NULL argument");
  std::vector<double> at(n);
  MB_CHECK(mb_poisson_arrivals(seed, rate_qps, n, at.data()));
  std::vector<uint64_t> offs(n), ids(n);
  mb_queries_layout(qs, n, offs.data());
  const auto start = Clock::now();
  for (uint32_t i = 0; i < n; ++i) {
    const auto due = start + std::chrono::nanoseconds((int64_t)(at[i] * 1e3));
    // sleep to within 50 us of the arrival, then spin: arrivals land within
    // a few microseconds of their schedule
    const auto early = due - std::chrono::microseconds(50);
    if (Clock::now() < early) std::this_thread::sleep_until(early);
    while (Clock::now() < due) {
    }
    MB_CHECK(mb_server_submit(s, &qs[i], out_host + offs[i], &ids[i]));
  }
  for (uint32_t i = 0; i < n; ++i) MB_CHECK(mb_server_wait(s, ids[i], -1, &info[i]));
  return MB_OK;
}
