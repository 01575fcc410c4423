// vh_batch.cu -- many independent events advanced together.
//
// Every event keeps its own context (grid, fields, clock); a batch replays
// one CUDA graph per driver-loop iteration that holds every event's steps as
// an independent branch (events spread round-robin, largest first, over a
// set of capture streams), so that small grids run side by side and the
// host issues one launch per iteration instead of ~30 per event.  The step
// kernels read tau and dt from each context's device clock and the graph
// advances those clocks itself, so a captured iteration stays valid; it is
// captured again only when its shape changes: an event's substep count
// (src/main.cpp:405-419), the parity of its double-buffered fill fractions,
// a grid resize (src/main.cpp:423-427), or the launch configuration.
//
// The stage-batched form captures instead, per substep index, one launch
// per stage of the step over a work table of every event's blocks (events
// with fewer substeps drop out of the later tables), with the events'
// clock operations batched too: a few dozen launches per iteration
// whatever the number of events.
//
// The launch configuration (capture streams, block size of the step
// kernels, or the stage-batched form) is picked by an online autotuner:
// with tuning on, successive iterations run under each candidate and are
// timed with CUDA events, and the fastest is kept.  Every configuration runs
// the same per-cell operations on the same data in the same per-event
// order, so results do not depend on it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/vhlle_b200.h"
#include "vh_ctx.cuh"
#include "vh_mlp.cuh"
#include "vh_step.cuh"

namespace {

struct Config {
  int nstreams, block;  // nstreams 0: the stage-batched form
};
const Config kConfigs[] = {{1, 128}, {4, 128}, {8, 128}, {16, 128}, {32, 128},
                           {8, 64},  {16, 64}, {32, 64},  {0, 128}};
constexpr int kDefaultConfig = 2;  // {8, 128}
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);
constexpr int kStageConfig = kNumConfigs - 1;
constexpr int kTuneReps = 2;  // iterations timed per candidate

thread_local std::string g_batch_error;

vh_status bfail(vh_status st, const std::string& m) {
  g_batch_error = m;
  return st;
}

}  // namespace

struct vh_batch {
  int device = 0;
  std::vector<vh_ctx*> ev;
  std::vector<int> order;  // events, largest first
  // driver parameters per event (src/main.cpp:70-81 globals)
  std::vector<double> dtau, etamin, etamax, tau_resize;
  std::vector<int> nz;
  std::vector<char> resized;
  std::vector<double*> bufA;  // each event's first fill-fraction buffer (parity 0)
  cudaStream_t origin = nullptr;
  std::vector<cudaStream_t> streams;
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr, ts = nullptr, te = nullptr;
  std::vector<cudaEvent_t> join;
  std::map<std::vector<int>, cudaGraphExec_t> graphs;
  // the device work tables a stage-batched graph reads, per graph key
  std::map<std::vector<int>, std::vector<void*>> tables;
  int captures = 0;
  int config = kDefaultConfig;  // index into kConfigs
  // the stage-batched form: the events' common EoS class (-1: unavailable)
  // and viscosity
  int stage_ek = -1;
  bool stage_viscous = false;
  std::vector<int> cands;  // the tuner's candidates (indices into kConfigs)
  // online tuning state
  bool tuning = false;
  int tune_cand = 0, tune_rep = 0;
  std::vector<float> tune_ms;
  double last_ms = 0.;

  void drop_graph(const std::vector<int>& key) {
    auto t = tables.find(key);
    if (t != tables.end()) {
      for (void* p : t->second) cudaFree(p);
      tables.erase(t);
    }
  }
  void clear_graphs() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    graphs.clear();
    for (auto& kv : tables)
      for (void* p : kv.second) cudaFree(p);
    tables.clear();
  }
};

namespace {

int substeps(const vh_batch* b, int e) {
  // src/main.cpp:405-409 with the event's parameters
  const vh_ctx* c = b->ev[e];
  int n = 1;
  while (b->dtau[e] / n > 1.0 * c->tau * (b->etamax[e] - b->etamin[e]) / (b->nz[e] - 1)) {
    if (n >= (1 << 20)) return -1;
    n *= 2;
  }
  return n;
}

vh_status ensure_streams(vh_batch* b, int n) {
  cudaError_t e;
  while ((int)b->streams.size() < n) {
    cudaStream_t s;
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess)
      return bfail(VH_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
    b->streams.push_back(s);
    cudaEvent_t j;
    if ((e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming)) != cudaSuccess)
      return bfail(VH_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(e));
    b->join.push_back(j);
  }
  return VH_OK;
}

// Captures one driver-loop iteration for every event with the given
// substep counts into an executable graph.
vh_status capture(vh_batch* b, const std::vector<int>& nsub, const Config& cfg,
                  cudaGraphExec_t* out) {
  vh_status st = ensure_streams(b, cfg.nstreams);
  if (st != VH_OK) return st;
  cudaError_t e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
  cudaEventRecord(b->fork, b->origin);
  for (int k = 0; k < cfg.nstreams; k++) cudaStreamWaitEvent(b->streams[k], b->fork, 0);
  for (size_t r = 0; r < b->order.size(); r++) {
    const int ei = b->order[r];
    vh_ctx* c = b->ev[ei];
    cudaStream_t s = b->streams[r % cfg.nstreams];
    vh::StepArgs a;
    a.g = c->g;
    a.eos = c->eos;
    a.eos.vguess = c->mlp ? c->vguess : nullptr;
    a.tr = c->tr;
    a.f = c->f;
    a.clk = c->clk;
    a.viscous = c->viscous;
    a.block = cfg.block;
    const int n = nsub[ei];
    if (n > 1) vh::launch_clock_op(c->clk, 1, n, s);  // dt / n
    for (int j = 0; j < n; j++) {
      if (c->mlp) vh::launch_mlp_guess(c->mlp->packed, a.f.Q, c->g.N, c->clk, c->vguess, s);
      vh::launch_step(a, s);
      vh::launch_clock_op(c->clk, 0, 0, s);  // tau += dt
      std::swap(a.f.m, a.f.m2);
    }
    if (n > 1) vh::launch_clock_op(c->clk, 2, n, s);  // dt * n
  }
  for (int k = 0; k < cfg.nstreams; k++) {
    cudaEventRecord(b->join[k], b->streams[k]);
    cudaStreamWaitEvent(b->origin, b->join[k], 0);
  }
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(b->origin, &graph);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  b->captures++;
  return VH_OK;
}

// The stage-batched form of one iteration: per substep index j a work
// table of every event with more than j substeps (its StepDev with the
// fill-fraction buffers of that substep's parity, and its blocks), the
// learned start points per event, the stage launches and the clocks'
// tau += dt over the table's events; dt / n before and dt * n after over all
// events (n = 1 leaves dt as it is).  The tables are device arrays written
// before the capture and kept with the graph.
vh_status capture_stages(vh_batch* b, const std::vector<int>& nsub, cudaGraphExec_t* out,
                         std::vector<void*>* keep) {
  const int n = (int)b->ev.size();
  int nmax = 1;
  for (int k = 0; k < n; k++) nmax = std::max(nmax, nsub[k]);
  std::vector<vh::StepDev> devs;
  std::vector<vh::BItem> items;
  std::vector<int> ns;
  struct Part {
    int dev0, nev, item0, nitems;
  };
  std::vector<Part> parts;
  for (int j = 0; j < nmax; j++) {
    Part pt{(int)devs.size(), 0, (int)items.size(), 0};
    for (int r = 0; r < n; r++) {
      const int ei = b->order[r];
      if (nsub[ei] <= j) continue;
      const vh_ctx* c = b->ev[ei];
      vh::StepDev d;
      d.g = c->g;
      d.eos = c->eos;
      d.eos.vguess = c->mlp ? c->vguess : nullptr;
      d.tr = c->tr;
      d.f = c->f;
      if (j & 1) std::swap(d.f.m, d.f.m2);
      d.clk = c->clk;
      d.viscous = c->viscous;
      const int idx = (int)devs.size() - pt.dev0;
      devs.push_back(d);
      if (j == 0) ns.push_back(nsub[ei]);
      const long long nb = (c->g.N + vh::kBatchBlock - 1) / vh::kBatchBlock;
      for (long long k = 0; k < nb; k++) items.push_back(vh::BItem{idx, (int)k});
      pt.nev++;
    }
    pt.nitems = (int)items.size() - pt.item0;
    parts.push_back(pt);
  }
  if (items.size() > (size_t)INT32_MAX)
    return bfail(VH_ERR_ARG, "vh_batch_advance: the stage-batched work table is too large");
  vh::StepDev* ddev = nullptr;
  vh::BItem* idev = nullptr;
  int* ndev = nullptr;
  cudaError_t e = cudaMalloc(&ddev, devs.size() * sizeof(vh::StepDev));
  if (e == cudaSuccess) e = cudaMalloc(&idev, items.size() * sizeof(vh::BItem));
  if (e == cudaSuccess) e = cudaMalloc(&ndev, ns.size() * sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(ddev, devs.data(), devs.size() * sizeof(vh::StepDev), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(idev, items.data(), items.size() * sizeof(vh::BItem), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(ndev, ns.data(), ns.size() * sizeof(int), cudaMemcpyHostToDevice);
  keep->push_back(ddev);
  keep->push_back(idev);
  keep->push_back(ndev);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("stage-batched tables: ") + cudaGetErrorString(e));
  e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
  vh::launch_clock_op_batched(ddev, parts[0].nev, 1, ndev, b->origin);  // dt / n
  for (int j = 0; j < nmax; j++) {
    const Part& pt = parts[j];
    for (int r = 0; r < n; r++) {
      const int ei = b->order[r];
      const vh_ctx* c = b->ev[ei];
      if (nsub[ei] > j && c->mlp)
        vh::launch_mlp_guess(c->mlp->packed, c->f.Q, c->g.N, c->clk, c->vguess, b->origin);
    }
    vh::launch_step_batched(b->stage_ek, b->stage_viscous, ddev + pt.dev0, pt.nev,
                            idev + pt.item0, pt.nitems, b->origin);
    vh::launch_clock_op_batched(ddev + pt.dev0, pt.nev, 0, nullptr, b->origin);  // tau += dt
  }
  vh::launch_clock_op_batched(ddev, parts[0].nev, 2, ndev, b->origin);  // dt * n
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(b->origin, &graph);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  b->captures++;
  return VH_OK;
}

}  // namespace

extern "C" {

const char* vh_batch_last_error(void) { return g_batch_error.c_str(); }

vh_status vh_batch_destroy(vh_batch* b) {
  if (!b) return VH_OK;
  cudaSetDevice(b->device);
  if (b->origin) cudaStreamSynchronize(b->origin);
  b->clear_graphs();
  for (cudaStream_t s : b->streams) cudaStreamDestroy(s);
  for (cudaEvent_t j : b->join) cudaEventDestroy(j);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->t0) cudaEventDestroy(b->t0);
  if (b->t1) cudaEventDestroy(b->t1);
  if (b->ts) cudaEventDestroy(b->ts);
  if (b->te) cudaEventDestroy(b->te);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
  return VH_OK;
}

vh_status vh_batch_create(vh_ctx* const* ctxs, int n, vh_batch** out) {
  if (!out) return bfail(VH_ERR_ARG, "vh_batch_create: out is NULL");
  *out = nullptr;
  if (!ctxs || n <= 0) return bfail(VH_ERR_ARG, "vh_batch_create: no events");
  const int dev = ctxs[0] ? ctxs[0]->device : -1;
  for (int k = 0; k < n; k++) {
    if (!ctxs[k]) return bfail(VH_ERR_ARG, "vh_batch_create: NULL context");
    if (ctxs[k]->device != dev)
      return bfail(VH_ERR_ARG, "vh_batch_create: all events must live on one device");
    if (!ctxs[k]->uploaded) return bfail(VH_ERR_STATE, "vh_batch_create: an event has no state");
    for (int j = 0; j < k; j++)
      if (ctxs[j] == ctxs[k]) return bfail(VH_ERR_ARG, "vh_batch_create: an event appears twice");
  }
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) return bfail(VH_ERR_CUDA, cudaGetErrorString(e));
  vh_batch* b = new vh_batch;
  b->device = dev;
  b->ev.assign(ctxs, ctxs + n);
  b->order.resize(n);
  std::iota(b->order.begin(), b->order.end(), 0);
  std::stable_sort(b->order.begin(), b->order.end(),
                   [&](int x, int y) { return b->ev[x]->g.N > b->ev[y]->g.N; });
  for (int k = 0; k < n; k++) {
    const vh_ctx* c = ctxs[k];
    b->dtau.push_back(c->dt);
    b->etamin.push_back(c->grid.etamin);
    b->etamax.push_back(c->grid.etamax);
    b->nz.push_back(c->grid.nz);
    b->tau_resize.push_back(HUGE_VAL);  // no resize unless asked for
    b->resized.push_back(0);
    b->bufA.push_back(c->f.m);
  }
  if ((e = cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreate(&b->t0)) != cudaSuccess || (e = cudaEventCreate(&b->t1)) != cudaSuccess ||
      (e = cudaEventCreate(&b->ts)) != cudaSuccess || (e = cudaEventCreate(&b->te)) != cudaSuccess) {
    vh_batch_destroy(b);
    return bfail(VH_ERR_CUDA, cudaGetErrorString(e));
  }
  // the stage-batched form: one EoS class and viscosity, no vorticity
  b->stage_ek = vh::step_ek(ctxs[0]->eos);
  b->stage_viscous = ctxs[0]->viscous;
  for (int k = 0; k < n; k++)
    if (vh::step_ek(ctxs[k]->eos) != b->stage_ek || ctxs[k]->viscous != b->stage_viscous ||
        ctxs[k]->vort_on)
      b->stage_ek = -1;
  for (int k = 0; k < kNumConfigs; k++)
    if (k != kStageConfig || b->stage_ek >= 0) b->cands.push_back(k);
  // the contexts' queued work comes first
  for (vh_ctx* c : b->ev) cudaStreamSynchronize(c->stream);
  *out = b;
  return VH_OK;
}

vh_status vh_batch_set_driver(vh_batch* b, int k, double dtau, double etamin, double etamax,
                              int nz, double tau_resize) {
  if (!b || k >= (int)b->ev.size() || nz < 1 || !(dtau > 0.))
    return bfail(VH_ERR_ARG, "vh_batch_set_driver: bad arguments");
  const int lo = k < 0 ? 0 : k, hi = k < 0 ? (int)b->ev.size() : k + 1;
  for (int e = lo; e < hi; e++) {
    b->dtau[e] = dtau;
    b->etamin[e] = etamin;
    b->etamax[e] = etamax;
    b->nz[e] = nz;
    b->tau_resize[e] = tau_resize;
  }
  return VH_OK;
}

vh_status vh_batch_tune(vh_batch* b, int enable) {
  if (!b) return VH_ERR_ARG;
  b->tuning = enable != 0;
  b->tune_cand = 0;
  b->tune_rep = 0;
  b->tune_ms.assign(b->cands.size(), 0.f);
  return VH_OK;
}

vh_status vh_batch_set_mode(vh_batch* b, int stage_batched) {
  if (!b) return VH_ERR_ARG;
  if (stage_batched) {
    if (b->stage_ek < 0)
      return bfail(VH_ERR_ARG,
                   "vh_batch_set_mode: the events differ in EoS class or viscosity, or one has "
                   "vorticity on");
    b->config = kStageConfig;
  } else if (b->config == kStageConfig) {
    b->config = kDefaultConfig;
  }
  b->tuning = false;
  return VH_OK;
}

vh_status vh_batch_advance(vh_batch* b, int* nsub_max) {
  if (!b) return VH_ERR_ARG;
  cudaError_t e = cudaSetDevice(b->device);
  if (e != cudaSuccess) return bfail(VH_ERR_CUDA, cudaGetErrorString(e));
  const int n = (int)b->ev.size();
  std::vector<int> nsub(n), key;
  int nmax = 1;
  for (int k = 0; k < n; k++) {
    nsub[k] = substeps(b, k);
    if (nsub[k] < 0) return bfail(VH_ERR_ARG, "vh_batch_advance: substep count overflow");
    nmax = std::max(nmax, nsub[k]);
  }
  // vorticity switched on after the batch was made rules the form out
  if (b->stage_ek >= 0)
    for (const vh_ctx* c : b->ev)
      if (c->vort_on)
        return bfail(VH_ERR_STATE,
                     "vh_batch_advance: an event turned vorticity on; make a new batch");
  const int cfg_idx = b->tuning ? b->cands[b->tune_cand] : b->config;
  const Config cfg = kConfigs[cfg_idx];
  key.reserve(3 * n + 1);
  key.push_back(cfg_idx);
  for (int k = 0; k < n; k++) {
    key.push_back(nsub[k]);
    key.push_back(b->ev[k]->f.m == b->bufA[k] ? 0 : 1);
    key.push_back(b->ev[k]->version);
  }
  cudaGraphExec_t exec = nullptr;
  auto it = b->graphs.find(key);
  if (it != b->graphs.end()) {
    exec = it->second;
  } else {
    vh_status st;
    if (cfg.nstreams == 0) {
      std::vector<void*> keep;
      st = capture_stages(b, nsub, &exec, &keep);
      if (st != VH_OK) {
        for (void* p : keep) cudaFree(p);
        return st;
      }
      b->tables[key] = keep;
    } else {
      st = capture(b, nsub, cfg, &exec);
      if (st != VH_OK) return st;
    }
    b->graphs[key] = exec;
  }
  cudaEventRecord(b->t0, b->origin);
  if ((e = cudaGraphLaunch(exec, b->origin)) != cudaSuccess)
    return bfail(VH_ERR_CUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
  cudaEventRecord(b->t1, b->origin);
  // host mirrors follow the device clocks' arithmetic exactly
  for (int k = 0; k < n; k++) {
    vh_ctx* c = b->ev[k];
    const int m = nsub[k];
    if (m > 1) c->dt = c->dt / m;
    for (int j = 0; j < m; j++) {
      c->tau += c->dt;
      std::swap(c->f.m, c->f.m2);
    }
    if (m > 1) c->dt = c->dt * m;
  }
  if (b->tuning) {
    float ms = 0.f;
    cudaEventSynchronize(b->t1);
    cudaEventElapsedTime(&ms, b->t0, b->t1);
    b->tune_ms[b->tune_cand] += ms;
    if (++b->tune_rep == kTuneReps) {
      b->tune_rep = 0;
      if (++b->tune_cand == (int)b->cands.size()) {
        b->tuning = false;
        b->config = b->cands[std::min_element(b->tune_ms.begin(), b->tune_ms.end()) -
                             b->tune_ms.begin()];
        // keep only the chosen configuration's graphs
        for (auto g = b->graphs.begin(); g != b->graphs.end();) {
          if (g->first[0] != b->config) {
            cudaGraphExecDestroy(g->second);
            b->drop_graph(g->first);
            g = b->graphs.erase(g);
          } else {
            ++g;
          }
        }
      }
    }
  }
  // the one-shot resize after the iteration (src/main.cpp:423-427)
  bool any = false;
  for (int k = 0; k < n; k++)
    if (!b->resized[k] && b->ev[k]->tau >= b->tau_resize[k]) any = true;
  if (any) {
    cudaStreamSynchronize(b->origin);
    for (int k = 0; k < n; k++) {
      vh_ctx* c = b->ev[k];
      if (b->resized[k] || c->tau < b->tau_resize[k]) continue;
      int done = 0;
      vh_status st = vh_resize2x(c, &done);
      if (st != VH_OK) return bfail(st, std::string("vh_batch_advance: ") + vh_last_error(c));
      b->resized[k] = 1;
      cudaStreamSynchronize(c->stream);
    }
    b->clear_graphs();  // grid spacings and steps are captured by value
  }
  if (nsub_max) *nsub_max = nmax;
  return VH_OK;
}

vh_status vh_batch_sync(vh_batch* b, unsigned* error_bits) {
  if (!b) return VH_ERR_ARG;
  cudaError_t e = cudaSetDevice(b->device);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->origin);
  if (e != cudaSuccess) return bfail(VH_ERR_CUDA, cudaGetErrorString(e));
  unsigned all = 0;
  for (vh_ctx* c : b->ev) {
    unsigned bits = 0;
    vh_status st = vh_error_bits(c, &bits);
    if (st != VH_OK) return bfail(st, vh_last_error(c));
    all |= bits;
  }
  if (error_bits) *error_bits = all;
  return all ? bfail(VH_ERR_NUMERIC, "vh_batch_sync: a step set the device error word") : VH_OK;
}

vh_status vh_batch_timer_start(vh_batch* b) {
  if (!b) return VH_ERR_ARG;
  cudaSetDevice(b->device);
  cudaError_t e = cudaEventRecord(b->ts, b->origin);
  return e == cudaSuccess ? VH_OK : bfail(VH_ERR_CUDA, cudaGetErrorString(e));
}

vh_status vh_batch_timer_stop(vh_batch* b, double* ms) {
  if (!b || !ms) return VH_ERR_ARG;
  cudaSetDevice(b->device);
  float f = 0.f;
  cudaError_t e;
  if ((e = cudaEventRecord(b->te, b->origin)) != cudaSuccess ||
      (e = cudaEventSynchronize(b->te)) != cudaSuccess ||
      (e = cudaEventElapsedTime(&f, b->ts, b->te)) != cudaSuccess)
    return bfail(VH_ERR_CUDA, cudaGetErrorString(e));
  *ms = f;
  return VH_OK;
}

vh_status vh_batch_info(vh_batch* b, int* captures, int* nstreams, int* block) {
  if (!b) return VH_ERR_ARG;
  if (captures) *captures = b->captures;
  if (nstreams) *nstreams = kConfigs[b->config].nstreams;
  if (block) *block = kConfigs[b->config].block;
  return VH_OK;
}

}  // extern "C"
