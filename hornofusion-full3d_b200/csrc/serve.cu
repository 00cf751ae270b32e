// Serving loop for concurrent simulated furnace runs (no reference
// counterpart; the reference runs one simulation per mpirun).
//
// A run is one furnace's SIMPLE loop: a sequence of pressure solves on one
// mesh, each with new coefficients and right-hand side, each warm-started
// from the run's previous solution. The server keeps every admitted run's
// state on the device between solves (compact coefficients, Krylov
// workspace, and phi in the reference halo layout as the warm start),
// admits runs against an HBM budget, and solves their requests in batched
// persistent launches (batch.cu kernels):
//
//   * continuous batching, by size: requests that arrive while batches are
//     on the GPU wait in a FIFO; the next batch takes the oldest request's
//     mesh size and the queued requests of that size, as soon as a stream
//     slot and enough blocks are free; up to two batches are in flight on
//     separate streams, so uploads, downloads and compute of different
//     batches overlap;
//   * the persistent kernels of in-flight batches together never hold more
//     blocks than the device can keep resident, so no cooperative launch
//     waits on blocks that another one occupies;
//   * a run's lane width depends only on its mesh size, so each result is
//     bit-identical whether the run is served alone or in any mix;
//   * large runs (at least kSoloCells cells, FP64) take no lane: when the
//     oldest pending request is one, the server lets the device drain, then
//     solves that request and the queued requests of its mesh one after
//     another, each over the whole GPU with the single-system launch of its
//     mesh (as the batch does with its large systems), while nothing else
//     runs; their results are again the same alone and in any mix.
//
// Threading: any host thread may call the eaf_srv_* functions; one server
// thread owns the launches and never holds the server lock while it enqueues
// device work. A submitted request reads the caller's input arrays until its
// ticket completes, and writes phi_out (if given) before completing it.
// Page-locked inputs and outputs are transferred asynchronously; pageable
// inputs are staged by the driver during the enqueue, and a pageable phi_out
// is filled from a page-locked buffer of the run when the batch completes.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "cg_kernels.h"
#include "eafcg.h"
#include "eafcg_internal.h"
#include "tune_table.h"

using eaf::BatchSys;
using eaf::HaloInputs;
using eaf::SolveResult;
using Clock = std::chrono::steady_clock;

namespace {

constexpr int kSlots = 2;
constexpr long long kSoloCells = 300000;

struct SrvRun {
  int nr, nth, nz;
  long long n, nh;
  size_t bytes;
  BatchSys sys;
  double* stage[9];  // aW..Su inputs and phi (the device-resident warm start)
  double* h_phi;     // pinned download buffer for pageable phi_out
  bool busy;
};

struct SrvTicket {
  int run;
  const double* in[8];
  double* phi_out;
  bool out_pinned;  // phi_out is page-locked: downloaded into directly
  Clock::time_point t_submit, t_done;
  SolveResult res;
  bool done;
};

// What the launcher needs of one picked request (copied under the lock).
struct Pick {
  long long id;
  SrvRun* run;
  const double* in[8];
  double* phi_out;
  bool out_pinned;
};

bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

struct SrvSlot {
  cudaStream_t st;
  cudaEvent_t ev;
  int* d_tab;
  unsigned long long* d_counters;
  double* d_parts;
  int* d_err;
  BatchSys* d_sys;
  SolveResult* d_res;
  int* h_tab;          // pinned
  BatchSys* h_sys;     // pinned
  SolveResult* h_res;  // pinned
  std::vector<long long> tickets;
  int blocks;
  bool busy;
};

size_t run_bytes(long long n, long long nh, bool mixed) {
  size_t b = (size_t)n * sizeof(double) * 14 + (size_t)nh * sizeof(double) * 9 + 256;
  if (mixed) b += (size_t)n * sizeof(float) * 13;
  return b;
}

}  // namespace

struct eaf_srv {
  int device;
  double budget;
  size_t used;
  int mixed, max_iter, max_outer, max_batch;
  double tol, inner_tol;
  uint64_t timeout_ns;
  int capacity, blocks_in_use;
  int sms;
  std::mutex m;
  std::condition_variable cv, cv_done;
  std::thread th;
  bool stop, fault;
  std::map<int, SrvRun*> runs;
  int next_run;
  std::map<long long, SrvTicket> tickets;
  long long next_ticket;
  std::deque<long long> pending;
  SrvSlot slots[kSlots];
  // statistics
  std::vector<double> lat_ms;
  long long solves, batches, batched_systems, refused, admitted;
  Clock::time_point t_first, t_last;
  bool any;
};

namespace {

void free_run(SrvRun* r) {
  for (double* p : r->stage) cudaFree(p);
  if (r->h_phi) cudaFreeHost(r->h_phi);
  double* f64[] = {r->sys.s.aP, r->sys.s.aE, r->sys.s.aN, r->sys.s.aT, r->sys.s.aW,
                   r->sys.s.aS, r->sys.s.aB, r->sys.s.b,  r->sys.s.x,  r->sys.s.r,
                   r->sys.s.q,  r->sys.s.p,  r->sys.s.p2, r->sys.s.z};
  for (double* p : f64) cudaFree(p);
  cudaFree(r->sys.s.asym);
  float* f32[] = {r->sys.f.aP, r->sys.f.aE, r->sys.f.aN, r->sys.f.aT, r->sys.f.aW,
                  r->sys.f.aS, r->sys.f.aB, r->sys.f.r,  r->sys.f.z,  r->sys.f.q,
                  r->sys.f.e,  r->sys.f.p,  r->sys.f.p2};
  for (float* p : f32) cudaFree(p);
  delete r;
}

// Completes the tickets of finished batches (caller holds the lock).
void reap(eaf_srv* s) {
  for (SrvSlot& sl : s->slots) {
    if (!sl.busy) continue;
    const cudaError_t q = cudaEventQuery(sl.ev);
    if (q == cudaErrorNotReady) continue;
    for (size_t i = 0; i < sl.tickets.size(); ++i) {  // pageable outputs
      SrvTicket& t = s->tickets[sl.tickets[i]];
      if (q == cudaSuccess && t.phi_out && !t.out_pinned) {
        const SrvRun* r = s->runs[t.run];
        memcpy(t.phi_out, r->h_phi, (size_t)r->nh * sizeof(double));
      }
    }
    const Clock::time_point now = Clock::now();
    for (size_t i = 0; i < sl.tickets.size(); ++i) {
      SrvTicket& t = s->tickets[sl.tickets[i]];
      t.res = sl.h_res[i];
      if (q != cudaSuccess || s->fault) {
        t.res.status = EAF_ECUDA;
        if (q != cudaSuccess) eaf::set_error("eaf_srv: batch", q);
      }
      t.done = true;
      t.t_done = now;
      s->lat_ms.push_back(std::chrono::duration<double, std::milli>(now - t.t_submit).count());
      auto it = s->runs.find(t.run);
      if (it != s->runs.end()) it->second->busy = false;
      ++s->solves;
    }
    s->t_last = now;
    s->blocks_in_use -= sl.blocks;
    sl.busy = false;
    sl.tickets.clear();
    s->cv_done.notify_all();
  }
}

// Forms and launches one batch on a free slot. Called with the lock held;
// releases it while enqueueing device work (only the server thread touches
// slots and the device state of busy runs). Returns true if launched.
bool launch(eaf_srv* s, std::unique_lock<std::mutex>& lk) {
  if (s->pending.empty() || s->fault) return false;
  SrvSlot* sl = nullptr;
  for (SrvSlot& c : s->slots)
    if (!c.busy) { sl = &c; break; }
  if (!sl) return false;
  const int free_blocks = s->capacity - s->blocks_in_use;
  // Batches by size: the oldest pending request fixes the batch's mesh (lane
  // width class); requests of that mesh join in FIFO order while their
  // lanes fit. A batch's persistent launch ends when its slowest solve
  // does, so a batch of one mesh size keeps short solves from waiting on
  // long ones; the second stream slot runs another size meanwhile. A large
  // mesh waits for the whole device instead (see the file comment).
  const SrvRun* oldest = s->runs[s->tickets[s->pending.front()].run];
  const bool solo = !s->mixed && oldest->n >= kSoloCells;
  if (solo && s->blocks_in_use != 0) return false;  // let the device drain
  std::vector<Pick> pick;
  std::vector<int> widths;
  std::vector<long long> cells;
  int used = 0, cls_nr = -1, cls_nth = -1, cls_nz = -1;
  for (auto it = s->pending.begin(); it != s->pending.end();) {
    if ((int)pick.size() >= s->max_batch) break;
    const SrvTicket& t = s->tickets[*it];
    SrvRun* r = s->runs[t.run];
    if (cls_nr < 0) {
      cls_nr = r->nr;
      cls_nth = r->nth;
      cls_nz = r->nz;
    }
    if (r->nr != cls_nr || r->nth != cls_nth || r->nz != cls_nz) {
      ++it;
      continue;
    }
    const int w = eaf::tuned_lane_width(r->nr, r->nth, r->nz);
    if (!solo && used + w > free_blocks) break;
    used += w;
    Pick p;
    p.id = *it;
    p.run = r;
    for (int k = 0; k < 8; ++k) p.in[k] = t.in[k];
    p.phi_out = t.phi_out;
    p.out_pinned = t.out_pinned;
    pick.push_back(p);
    widths.push_back(w);
    cells.push_back(r->n);
    it = s->pending.erase(it);
  }
  if (pick.empty()) return false;
  // Blocks for this batch: no more than one lane per system needs, so the
  // rest stay free for the next batch to run beside this one; a batch of
  // large runs holds the whole device.
  int want = 0;
  for (int w : widths) want += w;
  const int G = solo ? s->capacity : std::min(free_blocks, want);
  eaf::LanePlan lp;
  if (!solo && eaf::plan_lanes(widths, cells, G, &lp) != EAF_OK) {
    for (auto it = pick.rbegin(); it != pick.rend(); ++it) s->pending.push_front(it->id);
    return false;
  }
  // Reserve the slot and the blocks, then enqueue without the lock.
  sl->busy = true;
  sl->blocks = G;
  s->blocks_in_use += G;
  sl->tickets.clear();
  for (const Pick& p : pick) sl->tickets.push_back(p.id);
  lk.unlock();
  const std::vector<int> tab = lp.packed();
  const int nb = (int)pick.size();
  cudaError_t e = cudaSuccess;
  if (!solo) {
    memcpy(sl->h_tab, tab.data(), sizeof(int) * tab.size());
    for (int i = 0; i < nb; ++i) {
      sl->h_sys[i] = pick[i].run->sys;
      sl->h_sys[i].result = sl->d_res + i;
    }
    e = cudaMemcpyAsync(sl->d_tab, sl->h_tab, sizeof(int) * tab.size(), cudaMemcpyHostToDevice,
                        sl->st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(sl->d_sys, sl->h_sys, sizeof(BatchSys) * nb, cudaMemcpyHostToDevice,
                          sl->st);
  }
  for (int i = 0; i < nb && e == cudaSuccess; ++i) {
    const SrvRun* r = pick[i].run;
    for (int k = 0; k < 8 && e == cudaSuccess; ++k)
      e = cudaMemcpyAsync(r->stage[k], pick[i].in[k], (size_t)r->nh * sizeof(double),
                          cudaMemcpyHostToDevice, sl->st);
    const HaloInputs in = {r->stage[0], r->stage[1], r->stage[2], r->stage[3], r->stage[4],
                           r->stage[5], r->stage[6], r->stage[7], r->stage[8]};
    if (e == cudaSuccess) e = eaf::launch_pack_f64(r->sys.d, in, r->sys.s, sl->st);
  }
  const int nlanes = (int)lp.lane_first.size();
  if (solo) {
    // one after another over the whole device, the single-system launch
    for (int i = 0; i < nb && e == cudaSuccess; ++i) {
      const SrvRun* r = pick[i].run;
      eaf::SolverLaunch L = eaf::choose_launch(r->nr, r->nth, r->nz, s->sms, 0, 0, 0,
                                               EAF_CG_FORM_REFERENCE, true);
      L.stream = 0;  // a run's compact arrays carry no padding cell
      const eaf::GroupWs ws = {sl->d_parts, sl->d_counters, sl->d_err, sl->d_res + i};
      e = eaf::launch_f64_solver(L, 1, r->sys.d, r->sys.s, ws, (size_t)8 * s->capacity,
                                 s->max_iter, s->tol, s->timeout_ns, sl->st);
    }
  }
  if (e == cudaSuccess && !solo)
    e = cudaMemsetAsync(sl->d_counters, 0,
                        sizeof(unsigned long long) * eaf::kCounterStride * nlanes, sl->st);
  if (e == cudaSuccess && !solo) e = cudaMemsetAsync(sl->d_err, 0, sizeof(int), sl->st);
  if (e == cudaSuccess && !solo) {
    const eaf::BatchTables tt = eaf::tables_from(sl->d_tab, G, nlanes, sl->d_sys,
                                                 sl->d_counters, sl->d_parts, sl->d_err);
    e = s->mixed ? eaf::launch_batch_mixed(tt, G, eaf::kBatchBlock, s->max_outer,
                                           s->max_iter, s->tol, s->inner_tol,
                                           s->timeout_ns, sl->st)
                 : eaf::launch_batch_f64(tt, G, eaf::kBatchBlock, s->max_iter, s->tol,
                                         s->timeout_ns, sl->st);
  }
  for (int i = 0; i < nb && e == cudaSuccess; ++i) {
    const SrvRun* r = pick[i].run;
    e = eaf::launch_unpack_f64(r->sys.d, r->sys.s.x, r->stage[8], sl->st);
    if (e == cudaSuccess && pick[i].phi_out)
      e = cudaMemcpyAsync(pick[i].out_pinned ? pick[i].phi_out : r->h_phi, r->stage[8],
                          (size_t)r->nh * sizeof(double), cudaMemcpyDeviceToHost, sl->st);
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(sl->h_res, sl->d_res, sizeof(SolveResult) * nb,
                        cudaMemcpyDeviceToHost, sl->st);
  if (e == cudaSuccess) e = cudaEventRecord(sl->ev, sl->st);
  lk.lock();
  if (e != cudaSuccess) {
    // Nothing of this batch can be trusted: fail its tickets once the
    // stream has drained, and give the slot back.
    eaf::set_error("eaf_srv: launch", e);
    lk.unlock();
    cudaStreamSynchronize(sl->st);
    lk.lock();
    const Clock::time_point now = Clock::now();
    for (const Pick& p : pick) {
      SrvTicket& t = s->tickets[p.id];
      t.res.status = EAF_ECUDA;
      t.done = true;
      t.t_done = now;
      p.run->busy = false;
    }
    s->blocks_in_use -= G;
    sl->busy = false;
    sl->tickets.clear();
    s->cv_done.notify_all();
    return false;
  }
  ++s->batches;
  s->batched_systems += nb;
  return true;
}

void server_main(eaf_srv* s) {
  eaf::DeviceGuard guard(s->device);
  std::unique_lock<std::mutex> lk(s->m);
  for (;;) {
    reap(s);
    if (s->fault) {  // simulated device loss: fail everything queued
      const Clock::time_point now = Clock::now();
      for (long long id : s->pending) {
        SrvTicket& t = s->tickets[id];
        t.res.status = EAF_ECUDA;
        t.done = true;
        t.t_done = now;
        s->runs[t.run]->busy = false;
      }
      s->pending.clear();
      s->cv_done.notify_all();
    }
    bool launched = false;
    while (launch(s, lk)) launched = true;
    bool in_flight = false;
    for (const SrvSlot& sl : s->slots) in_flight = in_flight || sl.busy;
    if (s->stop && !in_flight && (s->pending.empty() || s->fault)) break;
    if (launched) continue;
    if (in_flight)
      s->cv.wait_for(lk, std::chrono::microseconds(50));
    else
      s->cv.wait_for(lk, std::chrono::milliseconds(50));
  }
}

}  // namespace

extern "C" {

int eaf_srv_create(eaf_srv_t* out, int device, double hbm_budget_bytes, int mixed,
                   int max_iter, double tol, int max_outer, double inner_tol,
                   int max_batch) {
  if (!out || !(hbm_budget_bytes > 0.0) || max_iter < 0 || max_batch < 1 ||
      (mixed && !(inner_tol > 0.0 && inner_tol < 1.0)))
    return EAF_EINVAL;
  *out = nullptr;
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) return EAF_ECUDA;
  eaf_srv* s = new (std::nothrow) eaf_srv();
  if (!s) return EAF_ENOMEM;
  s->device = device;
  s->budget = hbm_budget_bytes;
  s->mixed = mixed ? 1 : 0;
  s->max_iter = max_iter;
  s->tol = tol;
  s->max_outer = max_outer;
  s->inner_tol = inner_tol;
  s->max_batch = max_batch;
  s->timeout_ns = 2000ull * 1000ull * 1000ull;
  s->next_run = 1;
  s->next_ticket = 1;
  int rc = eaf::batch_capacity(device, &s->capacity);
  cudaError_t e = cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, device);
  const size_t tab_ints = (size_t)s->capacity * 4 + 2 + max_batch;
  for (SrvSlot& sl : s->slots) {
    if (e != cudaSuccess || rc != EAF_OK) break;
    e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_tab, sizeof(int) * tab_ints);
    if (e == cudaSuccess)
      e = cudaMalloc((void**)&sl.d_counters,
                     sizeof(unsigned long long) * eaf::kCounterStride * s->capacity);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_parts, sizeof(double) * 8 * s->capacity);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_sys, sizeof(BatchSys) * max_batch);
    if (e == cudaSuccess) e = cudaMalloc((void**)&sl.d_res, sizeof(SolveResult) * max_batch);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&sl.h_tab, sizeof(int) * tab_ints, 0);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&sl.h_sys, sizeof(BatchSys) * max_batch, 0);
    if (e == cudaSuccess)
      e = cudaHostAlloc((void**)&sl.h_res, sizeof(SolveResult) * max_batch, 0);
  }
  if (rc != EAF_OK || e != cudaSuccess) {
    if (e != cudaSuccess) eaf::set_error("eaf_srv_create", e);
    for (SrvSlot& sl : s->slots) {
      if (sl.st) cudaStreamDestroy(sl.st);
      if (sl.ev) cudaEventDestroy(sl.ev);
      cudaFree(sl.d_tab);
      cudaFree(sl.d_counters);
      cudaFree(sl.d_parts);
      cudaFree(sl.d_err);
      cudaFree(sl.d_sys);
      cudaFree(sl.d_res);
      if (sl.h_tab) cudaFreeHost(sl.h_tab);
      if (sl.h_sys) cudaFreeHost(sl.h_sys);
      if (sl.h_res) cudaFreeHost(sl.h_res);
    }
    delete s;
    return rc != EAF_OK ? rc : EAF_ECUDA;
  }
  s->th = std::thread(server_main, s);
  *out = s;
  return EAF_OK;
}

int eaf_srv_destroy(eaf_srv_t s) {
  if (!s) return EAF_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->stop = true;
  }
  s->cv.notify_all();
  s->th.join();
  eaf::DeviceGuard guard(s->device);
  for (SrvSlot& sl : s->slots) {
    cudaStreamSynchronize(sl.st);
    cudaStreamDestroy(sl.st);
    cudaEventDestroy(sl.ev);
    cudaFree(sl.d_tab);
    cudaFree(sl.d_counters);
    cudaFree(sl.d_parts);
    cudaFree(sl.d_err);
    cudaFree(sl.d_sys);
    cudaFree(sl.d_res);
    cudaFreeHost(sl.h_tab);
    cudaFreeHost(sl.h_sys);
    cudaFreeHost(sl.h_res);
  }
  for (auto& kv : s->runs) free_run(kv.second);
  delete s;
  return EAF_OK;
}

int eaf_srv_open_run(eaf_srv_t s, int nr, int nth, int nz, int* run_id) {
  if (!s || !run_id || nr < 1 || nth < 1 || nz < 1) return EAF_EINVAL;
  const long long n = (long long)nr * nth * nz;
  const long long nh = (long long)(nr + 4) * (nth + 4) * (nz + 4);
  if (nh >= (1ll << 31)) return EAF_EINVAL;
  const size_t bytes = run_bytes(n, nh, s->mixed != 0);
  {
    std::lock_guard<std::mutex> lk(s->m);
    if (s->stop || s->fault) return EAF_ECLOSED;
    if ((double)(s->used + bytes) > s->budget) {
      ++s->refused;
      return EAF_EADMIT;
    }
    s->used += bytes;  // reserved before allocating
  }
  eaf::DeviceGuard guard(s->device);
  SrvRun* r = new (std::nothrow) SrvRun();
  cudaError_t e = r ? cudaSuccess : cudaErrorMemoryAllocation;
  if (r) {
    memset(r, 0, sizeof(*r));
    r->nr = nr;
    r->nth = nth;
    r->nz = nz;
    r->n = n;
    r->nh = nh;
    r->bytes = bytes;
    r->sys.d = eaf::make_dims(nr, nth, nz);
    double** f64[] = {&r->sys.s.aP, &r->sys.s.aE, &r->sys.s.aN, &r->sys.s.aT,
                      &r->sys.s.aW, &r->sys.s.aS, &r->sys.s.aB, &r->sys.s.b,
                      &r->sys.s.x,  &r->sys.s.r,  &r->sys.s.q,  &r->sys.s.p,
                      &r->sys.s.p2, &r->sys.s.z};
    for (double** p : f64)
      if (e == cudaSuccess) e = cudaMalloc((void**)p, (size_t)n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&r->sys.s.asym, sizeof(int));
    if (s->mixed) {
      float** f32[] = {&r->sys.f.aP, &r->sys.f.aE, &r->sys.f.aN, &r->sys.f.aT,
                       &r->sys.f.aW, &r->sys.f.aS, &r->sys.f.aB, &r->sys.f.r,
                       &r->sys.f.z,  &r->sys.f.q,  &r->sys.f.e,  &r->sys.f.p,
                       &r->sys.f.p2};
      for (float** p : f32)
        if (e == cudaSuccess) e = cudaMalloc((void**)p, (size_t)n * sizeof(float));
    }
    for (int k = 0; k < 9 && e == cudaSuccess; ++k)
      e = cudaMalloc((void**)&r->stage[k], (size_t)nh * sizeof(double));
    if (e == cudaSuccess) e = cudaMemset(r->stage[8], 0, (size_t)nh * sizeof(double));
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&r->h_phi, (size_t)nh * sizeof(double), 0);
  }
  std::lock_guard<std::mutex> lk(s->m);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_srv_open_run", e);
    s->used -= bytes;
    if (r) free_run(r);
    return EAF_ENOMEM;
  }
  const int id = s->next_run++;
  s->runs[id] = r;
  ++s->admitted;
  *run_id = id;
  return EAF_OK;
}

int eaf_srv_close_run(eaf_srv_t s, int run_id) {
  if (!s) return EAF_EINVAL;
  SrvRun* r = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->m);
    auto it = s->runs.find(run_id);
    if (it == s->runs.end()) return EAF_EINVAL;
    if (it->second->busy) return EAF_EBUSY;
    r = it->second;
    s->runs.erase(it);
    s->used -= r->bytes;
  }
  eaf::DeviceGuard guard(s->device);
  free_run(r);
  return EAF_OK;
}

int eaf_srv_submit(eaf_srv_t s, int run_id, const double* aW, const double* aE,
                   const double* aS, const double* aN, const double* aB, const double* aT,
                   const double* aP, const double* Su, double* phi_out, long long* ticket) {
  if (!s || !ticket) return EAF_EINVAL;
  const double* in[8] = {aW, aE, aS, aN, aB, aT, aP, Su};
  for (const double* p : in)
    if (!p) return EAF_EINVAL;
  const bool out_pinned = phi_out != nullptr && is_pinned(phi_out);
  {
    std::lock_guard<std::mutex> lk(s->m);
    if (s->stop || s->fault) return EAF_ECLOSED;
    auto it = s->runs.find(run_id);
    if (it == s->runs.end()) return EAF_EINVAL;
    if (it->second->busy) return EAF_EBUSY;  // one outstanding solve per run
    it->second->busy = true;
    SrvTicket t;
    memset(&t.res, 0, sizeof(t.res));
    t.run = run_id;
    for (int k = 0; k < 8; ++k) t.in[k] = in[k];
    t.phi_out = phi_out;
    t.out_pinned = out_pinned;
    t.t_submit = Clock::now();
    t.done = false;
    const long long id = s->next_ticket++;
    s->tickets[id] = t;
    s->pending.push_back(id);
    if (!s->any) {
      s->any = true;
      s->t_first = t.t_submit;
    }
    *ticket = id;
  }
  s->cv.notify_all();
  return EAF_OK;
}

static int take(eaf_srv* s, long long ticket, double* residual, int* n_iter, int* n_outer,
                int* status) {
  auto it = s->tickets.find(ticket);
  const SrvTicket& t = it->second;
  if (residual) *residual = t.res.residual;
  if (n_iter) *n_iter = t.res.n_iter;
  if (n_outer) *n_outer = t.res.n_outer;
  if (status) *status = t.res.status;
  s->tickets.erase(it);
  return EAF_OK;
}

int eaf_srv_poll(eaf_srv_t s, long long ticket, double* residual, int* n_iter, int* n_outer,
                 int* status) {
  if (!s) return EAF_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return EAF_EINVAL;
  if (!it->second.done) return EAF_EBUSY;
  return take(s, ticket, residual, n_iter, n_outer, status);
}

int eaf_srv_wait(eaf_srv_t s, long long ticket, double timeout_ms, double* residual,
                 int* n_iter, int* n_outer, int* status) {
  if (!s || !(timeout_ms >= 0.0)) return EAF_EINVAL;
  std::unique_lock<std::mutex> lk(s->m);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return EAF_EINVAL;
  const auto deadline = Clock::now() + std::chrono::microseconds((long long)(timeout_ms * 1e3));
  while (!s->tickets[ticket].done) {
    if (s->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
        !s->tickets[ticket].done)
      return EAF_ETIMEOUT;
  }
  return take(s, ticket, residual, n_iter, n_outer, status);
}

int eaf_srv_stats(eaf_srv_t s, eaf_srv_stats_t* st) {
  if (!s || !st) return EAF_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  memset(st, 0, sizeof(*st));
  st->solves = s->solves;
  st->batches = s->batches;
  st->mean_batch = s->batches ? (double)s->batched_systems / s->batches : 0.0;
  st->admitted_runs = s->admitted;
  st->refused_runs = s->refused;
  st->active_runs = (long long)s->runs.size();
  st->used_bytes = (double)s->used;
  st->budget_bytes = s->budget;
  if (!s->lat_ms.empty()) {
    std::vector<double> v = s->lat_ms;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      const size_t i = (size_t)std::min<double>(v.size() - 1, floor(p * (v.size() - 1) + 0.5));
      return v[i];
    };
    st->p50_ms = pct(0.50);
    st->p99_ms = pct(0.99);
    st->max_ms = v.back();
    double sum = 0.0;
    for (double x : v) sum += x;
    st->mean_ms = sum / v.size();
    const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
    st->solves_per_s = span > 0.0 ? s->solves / span : 0.0;
  }
  return EAF_OK;
}

int eaf_srv_reset_stats(eaf_srv_t s) {
  if (!s) return EAF_EINVAL;
  std::lock_guard<std::mutex> lk(s->m);
  s->lat_ms.clear();
  s->solves = s->batches = s->batched_systems = s->refused = 0;
  s->any = false;
  return EAF_OK;
}

int eaf_srv_inject_fault(eaf_srv_t s, int kind) {
  if (!s || kind != EAF_FAULT_DEVICE_LOST) return EAF_EINVAL;
  {
    std::lock_guard<std::mutex> lk(s->m);
    s->fault = true;
  }
  s->cv.notify_all();
  return EAF_OK;
}

}  // extern "C"
