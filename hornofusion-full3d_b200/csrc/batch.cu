// Batched pressure solves: many independent systems of uneven size in one
// persistent cooperative launch, replayed from a CUDA graph.
//
// Plan. Every system gets a lane width (blocks) that depends only on its
// mesh size -- from the committed tuning table, or eaf_batch_set_width --
// so that its reduction order, and hence its result, is the same in any
// batch. Lanes of equal width form a class; the planner gives each class
// lanes in proportion to its modelled work (longest-processing-time queue
// assignment inside a class) until the co-resident blocks are used up.
//
// Large systems. A system of at least kSoloCells cells (and no explicit
// width) does not take a lane: after the batched launch, the large systems
// run one after another, each over the whole GPU with the launch the
// single-system solver uses for its mesh (tuned table), in the same graph.
// A lane narrow enough to share the GPU with the small systems runs a
// system whose working set fills the L2 many times slower than the whole
// GPU does, and several such lanes side by side no longer fit in L2 at all;
// one at a time at full width each stays L2-resident. The association of a
// large system's dot products is that of its single-system launch, so its
// result is again the same alone and in any mix (eaf_batch_system_plan).
//
// Model of one system's solve on w blocks of 512 threads (B200 figures):
//   iterations   ~ 8 sqrt(cells)              (Jacobi-PCG on these meshes)
//   per iteration = 2 phases + 2 group reductions
//   phase        = max(2.5 us, cells/w x 64 B / 22 GB/s)   (latency floor;
//                  a block's share of HBM bandwidth when all stream)
//   reduction    = 0.3 us (w = 1) or 1.7 us + 7.5 ns x w  (measured,
//                  eaf_diag_allreduce_us)
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "cg_kernels.h"
#include "eafcg.h"
#include "eafcg_internal.h"
#include "tune_table.h"

using eaf::BatchSys;
using eaf::BatchTables;
using eaf::HaloInputs;
using eaf::SolveResult;

namespace {

constexpr long long kSoloCells = 300000;
constexpr int kSoloPartSlots = 8;

double model_iter_us(long long cells, int w) {
  const double cpb = (double)cells / w;
  const double phase = std::max(2.5, cpb * 64.0 / 22.0e3);
  const double red = w == 1 ? 0.3 : 1.7 + 0.0075 * w;
  return 2.0 * phase + 2.0 * red;
}

}  // namespace

namespace eaf {

double model_solve_us(long long cells, int w) {
  return 8.0 * sqrt((double)cells) * model_iter_us(cells, w);
}

int batch_capacity(int device, int* blocks) {
  int per_sm64 = 0, per_sm32 = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm64, batch_f64_kernel_ptr(),
                                                    eaf::kBatchBlock, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm32, batch_mixed_kernel_ptr(),
                                                    eaf::kBatchBlock, 0) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    set_error("batch: occupancy query", cudaErrorUnknown);
    return EAF_ECUDA;
  }
  *blocks = std::min(std::min(per_sm64, per_sm32) * sms, kMaxGroupBlocks);
  return EAF_OK;
}

std::vector<int> LanePlan::packed() const {
  std::vector<int> host;
  host.insert(host.end(), lane_of_block.begin(), lane_of_block.end());
  host.insert(host.end(), lane_first.begin(), lane_first.end());
  host.insert(host.end(), lane_width.begin(), lane_width.end());
  host.insert(host.end(), q_begin.begin(), q_begin.end());
  host.insert(host.end(), queue.begin(), queue.end());
  return host;
}

BatchTables tables_from(const int* d_tab, int grid, int nlanes, const BatchSys* d_sys,
                        unsigned long long* counters, double* parts, int* err) {
  BatchTables t;
  const int* p = d_tab;
  t.sys = d_sys;
  t.lane_of_block = p;
  p += grid;
  t.lane_first_block = p;
  p += nlanes;
  t.lane_width = p;
  p += nlanes;
  t.lane_q_begin = p;
  p += nlanes + 1;
  t.queue = p;
  t.counters = counters;
  t.parts = parts;
  t.err = err;
  return t;
}

int plan_lanes(const std::vector<int>& widths, const std::vector<long long>& cells, int G,
               LanePlan* out) {
  const int nsys = (int)widths.size();
  std::vector<int> cls = widths;
  std::sort(cls.begin(), cls.end());
  cls.erase(std::unique(cls.begin(), cls.end()), cls.end());
  long long need = 0;
  for (int w : cls) need += w;
  if (need > G) {
    set_error_text("batch: lane widths of the distinct mesh sizes exceed the blocks available");
    return EAF_EUNSUPPORTED;
  }
  const int C = (int)cls.size();
  std::vector<std::vector<int>> members(C);
  for (int s = 0; s < nsys; ++s)
    members[std::lower_bound(cls.begin(), cls.end(), widths[s]) - cls.begin()].push_back(s);
  std::vector<double> dur(nsys);
  for (int s = 0; s < nsys; ++s) dur[s] = model_solve_us(cells[s], widths[s]);
  for (auto& m : members)
    std::sort(m.begin(), m.end(), [&](int x, int y) {
      return dur[x] != dur[y] ? dur[x] > dur[y] : x < y;
    });
  auto lpt = [&](int c, int lanes, std::vector<std::vector<int>>* q) {
    std::vector<double> load(lanes, 0.0);
    if (q) q->assign(lanes, {});
    for (int s : members[c]) {
      int best = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      load[best] += dur[s];
      if (q) (*q)[best].push_back(s);
    }
    return *std::max_element(load.begin(), load.end());
  };
  std::vector<int> lanes(C, 1);
  int used = (int)need;
  for (;;) {  // add a lane to the class that finishes last, while blocks remain
    int worst = -1;
    double worst_t = -1.0;
    for (int c = 0; c < C; ++c) {
      if ((int)members[c].size() <= lanes[c]) continue;  // one system per lane already
      const double t = lpt(c, lanes[c], nullptr);
      if (t > worst_t) { worst_t = t; worst = c; }
    }
    if (worst < 0 || used + cls[worst] > G) break;
    lanes[worst] += 1;
    used += cls[worst];
  }
  LanePlan& lp = *out;
  lp.lane_of_block.assign(G, 0);
  lp.lane_first.clear();
  lp.lane_width.clear();
  lp.q_begin.assign(1, 0);
  lp.queue.clear();
  int blk = 0;
  for (int c = 0; c < C; ++c) {
    std::vector<std::vector<int>> qs;
    lpt(c, lanes[c], &qs);
    for (auto& q : qs) {
      const int L = (int)lp.lane_first.size();
      lp.lane_first.push_back(blk);
      lp.lane_width.push_back(cls[c]);
      for (int k = 0; k < cls[c]; ++k) lp.lane_of_block[blk + k] = L;
      blk += cls[c];
      lp.queue.insert(lp.queue.end(), q.begin(), q.end());
      lp.q_begin.push_back((int)lp.queue.size());
    }
  }
  // leftover blocks: single-block lanes with empty queues
  while (blk < G) {
    const int L = (int)lp.lane_first.size();
    lp.lane_first.push_back(blk);
    lp.lane_width.push_back(1);
    lp.lane_of_block[blk] = L;
    lp.q_begin.push_back((int)lp.queue.size());
    ++blk;
  }
  return EAF_OK;
}

}  // namespace eaf

struct eaf_batch {
  int device, nsys;
  cudaStream_t st;
  std::vector<int> nr, nth, nz, width;
  std::vector<long long> n, nh;
  std::vector<double*> stage;      // 9 per system (host path), halo layout
  std::vector<HaloInputs> in;      // what pack reads per system
  std::vector<double*> phi_out;    // where unpack writes per system
  std::vector<BatchSys> sys;       // host copy of the device table
  BatchSys* d_sys;
  SolveResult* d_res;
  SolveResult* h_res;  // pinned
  bool have_f32;
  // plan
  bool planned;
  int grid, nlanes;
  std::vector<int> lane_of_block, lane_first, lane_width, q_begin, queue;
  int* d_tab;  // all int tables, packed
  unsigned long long* d_counters;
  double* d_parts;
  int* d_err;
  // large systems solved one after another at full width
  std::vector<char> solo;
  std::vector<eaf::SolverLaunch> solo_f64;
  double* d_solo_part;
  unsigned long long* d_solo_counter;
  int* d_solo_err;
  int sms;
  // graph
  cudaGraphExec_t exec;
  bool graph_valid;
  int g_mixed, g_max_iter, g_max_outer;
  double g_tol, g_inner_tol;
  cudaEvent_t ev0, ev1;
  double last_ms;
  uint64_t timeout_ns;
};

namespace {

int width_for(const eaf_batch* b, int s) {
  if (b->width[s] > 0) return b->width[s];
  return eaf::tuned_lane_width(b->nr[s], b->nth[s], b->nz[s]);
}

bool is_solo(const eaf_batch* b, int s) { return b->width[s] == 0 && b->n[s] >= kSoloCells; }

void free_batch(eaf_batch* b) {
  if (b->graph_valid) cudaGraphExecDestroy(b->exec);
  for (double* p : b->stage) cudaFree(p);
  for (auto& s : b->sys) {
    double* f64[] = {s.s.aP, s.s.aE, s.s.aN, s.s.aT, s.s.aW, s.s.aS, s.s.aB,
                     s.s.b,  s.s.x,  s.s.r,  s.s.q,  s.s.p,  s.s.p2, s.s.z};
    for (double* p : f64) cudaFree(p);
    cudaFree(s.s.asym);
    float* f32[] = {s.f.aP, s.f.aE, s.f.aN, s.f.aT, s.f.aW, s.f.aS, s.f.aB,
                    s.f.r,  s.f.z,  s.f.q,  s.f.e,  s.f.p,  s.f.p2};
    for (float* p : f32) cudaFree(p);
  }
  cudaFree(b->d_sys);
  cudaFree(b->d_res);
  cudaFree(b->d_tab);
  cudaFree(b->d_counters);
  cudaFree(b->d_parts);
  cudaFree(b->d_err);
  cudaFree(b->d_solo_part);
  cudaFree(b->d_solo_counter);
  cudaFree(b->d_solo_err);
  if (b->h_res) cudaFreeHost(b->h_res);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->st) cudaStreamDestroy(b->st);
}

int alloc_f32(eaf_batch* b) {
  if (b->have_f32) return EAF_OK;
  for (int i = 0; i < b->nsys; ++i) {
    auto& f = b->sys[i].f;
    float** f32[] = {&f.aP, &f.aE, &f.aN, &f.aT, &f.aW, &f.aS, &f.aB,
                     &f.r,  &f.z,  &f.q,  &f.e,  &f.p,  &f.p2};
    for (float** p : f32) {
      cudaError_t e = cudaMalloc((void**)p, (size_t)b->n[i] * sizeof(float));
      if (e != cudaSuccess) {
        eaf::set_error("eaf_batch: cudaMalloc(f32)", e);
        return EAF_ENOMEM;
      }
    }
  }
  cudaError_t e = cudaMemcpy(b->d_sys, b->sys.data(), sizeof(BatchSys) * b->nsys,
                             cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_batch: table upload", e);
    return EAF_ECUDA;
  }
  b->have_f32 = true;
  return EAF_OK;
}

// Lanes and queues (see the file comment).
int plan(eaf_batch* b) {
  if (b->planned) return EAF_OK;
  int G = 0;
  int rc = eaf::batch_capacity(b->device, &G);
  if (rc != EAF_OK) return rc;
  std::vector<int> widths, ids;
  std::vector<long long> cells;
  b->solo.assign(b->nsys, 0);
  b->solo_f64.assign(b->nsys, eaf::SolverLaunch{0, 0, 1});
  for (int s = 0; s < b->nsys; ++s) {
    if (is_solo(b, s)) {
      b->solo[s] = 1;
      b->solo_f64[s] = eaf::choose_launch(b->nr[s], b->nth[s], b->nz[s], b->sms, 0, 0, 0,
                                          EAF_CG_FORM_REFERENCE, true);
      b->solo_f64[s].stream = 0;  // compact arrays here carry no padding cell
      continue;
    }
    ids.push_back(s);
    widths.push_back(width_for(b, s));
    cells.push_back(b->n[s]);
  }
  eaf::LanePlan lp;
  if (!ids.empty()) {
    rc = eaf::plan_lanes(widths, cells, G, &lp);
    if (rc != EAF_OK) return rc;
    for (int& q : lp.queue) q = ids[q];  // lane-system index -> system id
  } else {
    G = 0;
    lp.q_begin.assign(1, 0);
  }
  b->lane_of_block = lp.lane_of_block;
  b->lane_first = lp.lane_first;
  b->lane_width = lp.lane_width;
  b->q_begin = lp.q_begin;
  b->queue = lp.queue;
  b->grid = G;
  b->nlanes = (int)b->lane_first.size();
  // device tables
  const std::vector<int> host = lp.packed();
  cudaFree(b->d_tab);
  cudaFree(b->d_counters);
  cudaFree(b->d_parts);
  b->d_tab = nullptr;
  b->d_counters = nullptr;
  b->d_parts = nullptr;
  cudaError_t e = cudaMalloc((void**)&b->d_tab, sizeof(int) * host.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_tab, host.data(), sizeof(int) * host.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&b->d_counters,
                   sizeof(unsigned long long) * eaf::kCounterStride *
                       (b->nlanes > 0 ? b->nlanes : 1));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_parts, sizeof(double) * 8 * (G > 0 ? G : 1));
  if (e != cudaSuccess) {
    eaf::set_error("eaf_batch: plan tables", e);
    return EAF_ENOMEM;
  }
  b->planned = true;
  b->graph_valid = false;
  return EAF_OK;
}

BatchTables tables(const eaf_batch* b) {
  return eaf::tables_from(b->d_tab, b->grid, b->nlanes, b->d_sys, b->d_counters,
                          b->d_parts, b->d_err);
}

// Everything one batched solve does on the device, in stream order.
cudaError_t enqueue(eaf_batch* b) {
  cudaError_t e = cudaSuccess;
  for (int s = 0; s < b->nsys && e == cudaSuccess; ++s)
    e = eaf::launch_pack_f64(b->sys[s].d, b->in[s], b->sys[s].s, b->st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(b->d_counters, 0,
                        sizeof(unsigned long long) * eaf::kCounterStride * b->nlanes, b->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->d_err, 0, sizeof(int), b->st);
  // external event-record nodes: the graph's launches can be timed
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->ev0, b->st, cudaEventRecordExternal);
  if (e == cudaSuccess && b->grid > 0) {
    const BatchTables t = tables(b);
    if (b->g_mixed)
      e = eaf::launch_batch_mixed(t, b->grid, eaf::kBatchBlock, b->g_max_outer, b->g_max_iter,
                                  b->g_tol, b->g_inner_tol, b->timeout_ns, b->st);
    else
      e = eaf::launch_batch_f64(t, b->grid, eaf::kBatchBlock, b->g_max_iter, b->g_tol,
                                b->timeout_ns, b->st);
  }
  // the large systems, one after another over the whole GPU
  for (int s = 0; s < b->nsys && e == cudaSuccess; ++s) {
    if (!b->solo[s]) continue;
    const eaf::GroupWs ws = {b->d_solo_part, b->d_solo_counter, b->d_solo_err, b->d_res + s};
    if (b->g_mixed) {
      const eaf::SolverLaunch L = eaf::choose_launch(b->nr[s], b->nth[s], b->nz[s], b->sms, 0,
                                                     0, 0, EAF_CG_FORM_REFERENCE, false);
      e = eaf::launch_cg_mixed(b->sys[s].d, b->sys[s].s, b->sys[s].f, ws, b->g_max_outer,
                               b->g_max_iter, b->g_tol, b->g_inner_tol, b->timeout_ns,
                               L.grid, L.block, b->st);
    } else {
      e = eaf::launch_f64_solver(b->solo_f64[s], 1, b->sys[s].d, b->sys[s].s, ws,
                                 (size_t)kSoloPartSlots * b->sms * 8, b->g_max_iter,
                                 b->g_tol, b->timeout_ns, b->st);
    }
  }
  if (e == cudaSuccess) e = cudaEventRecordWithFlags(b->ev1, b->st, cudaEventRecordExternal);
  for (int s = 0; s < b->nsys && e == cudaSuccess; ++s)
    e = eaf::launch_unpack_f64(b->sys[s].d, b->sys[s].s.x, b->phi_out[s], b->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->h_res, b->d_res, sizeof(SolveResult) * b->nsys,
                        cudaMemcpyDeviceToHost, b->st);
  return e;
}

int capture(eaf_batch* b) {
  if (b->graph_valid) {
    cudaGraphExecDestroy(b->exec);
    b->graph_valid = false;
  }
  cudaGraph_t graph = nullptr;
  (void)cudaGetLastError();  // do not attribute an older failure to the capture
  cudaError_t e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t e2 = enqueue(b);
    e = cudaStreamEndCapture(b->st, &graph);
    if (e2 != cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_batch: graph capture", e);
    return EAF_ECUDA;
  }
  b->graph_valid = true;
  return EAF_OK;
}

}  // namespace

extern "C" {

int eaf_batch_create(eaf_batch_t* out, int nsys, const int* dims, int device) {
  if (!out || nsys < 1 || !dims) return EAF_EINVAL;
  *out = nullptr;
  for (int s = 0; s < nsys; ++s) {
    if (dims[3 * s] < 1 || dims[3 * s + 1] < 1 || dims[3 * s + 2] < 1) return EAF_EINVAL;
    if ((long long)(dims[3 * s] + 4) * (dims[3 * s + 1] + 4) * (dims[3 * s + 2] + 4) >=
        (1ll << 31))
      return EAF_EINVAL;
  }
  eaf::DeviceGuard guard(device);
  if (!guard.ok()) return EAF_ECUDA;
  eaf_batch* b = new (std::nothrow) eaf_batch();
  if (!b) return EAF_ENOMEM;
  b->device = device;
  b->nsys = nsys;
  b->timeout_ns = 2000ull * 1000ull * 1000ull;
  cudaError_t e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
  b->sys.resize(nsys);
  b->in.resize(nsys);
  b->phi_out.resize(nsys);
  b->width.assign(nsys, 0);
  for (int s = 0; s < nsys && e == cudaSuccess; ++s) {
    b->nr.push_back(dims[3 * s]);
    b->nth.push_back(dims[3 * s + 1]);
    b->nz.push_back(dims[3 * s + 2]);
    b->n.push_back((long long)dims[3 * s] * dims[3 * s + 1] * dims[3 * s + 2]);
    b->nh.push_back((long long)(dims[3 * s] + 4) * (dims[3 * s + 1] + 4) *
                    (dims[3 * s + 2] + 4));
    BatchSys& bs = b->sys[s];
    memset(&bs, 0, sizeof(bs));
    bs.d = eaf::make_dims(dims[3 * s], dims[3 * s + 1], dims[3 * s + 2]);
    double** f64[] = {&bs.s.aP, &bs.s.aE, &bs.s.aN, &bs.s.aT, &bs.s.aW,
                      &bs.s.aS, &bs.s.aB, &bs.s.b,  &bs.s.x,  &bs.s.r,
                      &bs.s.q,  &bs.s.p,  &bs.s.p2, &bs.s.z};
    for (double** p : f64)
      if (e == cudaSuccess) e = cudaMalloc((void**)p, (size_t)b->n[s] * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void**)&bs.s.asym, sizeof(int));
    for (int k = 0; k < 9 && e == cudaSuccess; ++k) {
      double* p = nullptr;
      e = cudaMalloc((void**)&p, (size_t)b->nh[s] * sizeof(double));
      b->stage.push_back(p);
    }
    const double* const* st9 = b->stage.data() + 9 * s;
    b->in[s] = {st9[0], st9[1], st9[2], st9[3], st9[4], st9[5], st9[6], st9[7], st9[8]};
    b->phi_out[s] = b->stage[9 * s + 8];
  }
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_sys, sizeof(BatchSys) * nsys);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_res, sizeof(SolveResult) * nsys);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_err, sizeof(int));
  if (e == cudaSuccess)
    e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess)
    e = cudaMalloc((void**)&b->d_solo_part, sizeof(double) * kSoloPartSlots * b->sms * 8);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_solo_counter, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->d_solo_err, sizeof(int));
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&b->h_res, sizeof(SolveResult) * nsys, 0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&b->ev1);
  for (int s = 0; s < nsys && e == cudaSuccess; ++s) b->sys[s].result = b->d_res + s;
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_sys, b->sys.data(), sizeof(BatchSys) * nsys, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_batch_create", e);
    free_batch(b);
    delete b;
    return e == cudaErrorMemoryAllocation ? EAF_ENOMEM : EAF_ECUDA;
  }
  *out = b;
  return EAF_OK;
}

int eaf_batch_destroy(eaf_batch_t b) {
  if (!b) return EAF_EINVAL;
  eaf::DeviceGuard guard(b->device);
  cudaStreamSynchronize(b->st);
  free_batch(b);
  delete b;
  return EAF_OK;
}

int eaf_batch_set_width(eaf_batch_t b, int sys, int width) {
  if (!b || sys < 0 || sys >= b->nsys || width < 0 || width > eaf::kMaxGroupBlocks)
    return EAF_EINVAL;
  b->width[sys] = width;
  b->planned = false;
  b->graph_valid = false;
  return EAF_OK;
}

int eaf_batch_lane_width(eaf_batch_t b, int sys, int* width) {
  if (!b || !width || sys < 0 || sys >= b->nsys) return EAF_EINVAL;
  *width = width_for(b, sys);
  return EAF_OK;
}

int eaf_batch_system_plan(eaf_batch_t b, int sys, int* grid, int* block, int* cluster) {
  if (!b || !grid || !block || !cluster || sys < 0 || sys >= b->nsys) return EAF_EINVAL;
  eaf::DeviceGuard guard(b->device);
  const int rc = plan(b);
  if (rc != EAF_OK) return rc;
  if (b->solo[sys]) {
    *grid = b->solo_f64[sys].grid;
    *block = b->solo_f64[sys].block;
    *cluster = b->solo_f64[sys].cluster;
  } else {
    *grid = width_for(b, sys);
    *block = eaf::kBatchBlock;
    *cluster = 1;
  }
  return EAF_OK;
}

int eaf_batch_plan(eaf_batch_t b, int* grid, int* block, int* nlanes) {
  if (!b || !grid || !block || !nlanes) return EAF_EINVAL;
  eaf::DeviceGuard guard(b->device);
  const int rc = plan(b);
  if (rc != EAF_OK) return rc;
  *grid = b->grid;
  *block = eaf::kBatchBlock;
  *nlanes = b->nlanes;
  return EAF_OK;
}

int eaf_batch_set_system(eaf_batch_t b, int sys, const double* aW, const double* aE,
                         const double* aS, const double* aN, const double* aB,
                         const double* aT, const double* aP, const double* Su,
                         const double* phi) {
  if (!b || sys < 0 || sys >= b->nsys) return EAF_EINVAL;
  const double* src[9] = {aW, aE, aS, aN, aB, aT, aP, Su, phi};
  for (const double* p : src)
    if (!p) return EAF_EINVAL;
  eaf::DeviceGuard guard(b->device);
  const size_t bytes = (size_t)b->nh[sys] * sizeof(double);
  for (int k = 0; k < 9; ++k) {
    cudaError_t e = cudaMemcpyAsync(b->stage[9 * sys + k], src[k], bytes,
                                    cudaMemcpyHostToDevice, b->st);
    if (e != cudaSuccess) {
      eaf::set_error("eaf_batch_set_system", e);
      return EAF_ECUDA;
    }
  }
  const double* const* st9 = b->stage.data() + 9 * sys;
  const HaloInputs hin = {st9[0], st9[1], st9[2], st9[3], st9[4],
                          st9[5], st9[6], st9[7], st9[8]};
  if (memcmp(&hin, &b->in[sys], sizeof(hin)) != 0 || b->phi_out[sys] != st9[8]) {
    b->in[sys] = hin;
    b->phi_out[sys] = b->stage[9 * sys + 8];
    b->graph_valid = false;
  }
  return EAF_OK;
}

int eaf_batch_set_system_device(eaf_batch_t b, int sys, const double* aW,
                                const double* aE, const double* aS, const double* aN,
                                const double* aB, const double* aT, const double* aP,
                                const double* Su, double* phi) {
  if (!b || sys < 0 || sys >= b->nsys) return EAF_EINVAL;
  const double* src[9] = {aW, aE, aS, aN, aB, aT, aP, Su, phi};
  for (const double* p : src)
    if (!p) return EAF_EINVAL;
  const HaloInputs hin = {aW, aE, aS, aN, aB, aT, aP, Su, phi};
  if (memcmp(&hin, &b->in[sys], sizeof(hin)) != 0 || b->phi_out[sys] != phi) {
    b->in[sys] = hin;
    b->phi_out[sys] = phi;
    b->graph_valid = false;
  }
  return EAF_OK;
}

int eaf_batch_solve(eaf_batch_t b, int mixed, int max_iter, double tol, int max_outer,
                    double inner_tol) {
  if (!b) return EAF_EINVAL;
  if (mixed && (!(inner_tol > 0.0 && inner_tol < 1.0) || max_iter < 1)) return EAF_EINVAL;
  eaf::DeviceGuard guard(b->device);
  int rc = plan(b);
  if (rc != EAF_OK) return rc;
  if (mixed && (rc = alloc_f32(b)) != EAF_OK) return rc;
  if (!b->graph_valid || b->g_mixed != mixed || b->g_max_iter != max_iter ||
      b->g_tol != tol || b->g_max_outer != max_outer || b->g_inner_tol != inner_tol) {
    b->g_mixed = mixed;
    b->g_max_iter = max_iter;
    b->g_tol = tol;
    b->g_max_outer = max_outer;
    b->g_inner_tol = inner_tol;
    if ((rc = capture(b)) != EAF_OK) return rc;
  }
  cudaError_t e = cudaGraphLaunch(b->exec, b->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->ev0, b->ev1);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_batch_solve", e);
    return EAF_ECUDA;
  }
  b->last_ms = ms;
  int worst = EAF_OK;
  for (int s = 0; s < b->nsys; ++s) {
    const int st = b->h_res[s].status;
    if (st == EAF_ETIMEOUT) worst = EAF_ETIMEOUT;
    else if (st != EAF_OK && worst == EAF_OK) worst = st;
  }
  return worst;
}

int eaf_batch_result(eaf_batch_t b, int sys, double* residual, int* n_iter, int* n_outer,
                     int* status) {
  if (!b || sys < 0 || sys >= b->nsys) return EAF_EINVAL;
  const SolveResult& r = b->h_res[sys];
  if (residual) *residual = r.residual;
  if (n_iter) *n_iter = r.n_iter;
  if (n_outer) *n_outer = r.n_outer;
  if (status) *status = r.status;
  return EAF_OK;
}

int eaf_batch_get_phi(eaf_batch_t b, int sys, double* phi) {
  if (!b || !phi || sys < 0 || sys >= b->nsys) return EAF_EINVAL;
  eaf::DeviceGuard guard(b->device);
  cudaError_t e = cudaMemcpyAsync(phi, b->phi_out[sys], (size_t)b->nh[sys] * sizeof(double),
                                  cudaMemcpyDeviceToHost, b->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
  if (e != cudaSuccess) {
    eaf::set_error("eaf_batch_get_phi", e);
    return EAF_ECUDA;
  }
  return EAF_OK;
}

double eaf_batch_last_ms(eaf_batch_t b) { return b ? b->last_ms : 0.0; }

void* eaf_batch_stream(eaf_batch_t b) { return b ? (void*)b->st : nullptr; }

}  // extern "C"
