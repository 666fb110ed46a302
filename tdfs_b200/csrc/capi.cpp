// capi.cpp -- the extern "C" entry points of libtdfs_b200.so (include/tdfs.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <sstream>
#include <string>
#include <vector>

#include "csr.h"
#include "graph.h"
#include "match.cuh"
#include "plan.h"
#include "serve.h"

struct tdfs_plan {
  tdfs::HostPlan host;
  tdfs::DevPlan dev;
};

namespace tdfs {

namespace {

// Report a failed CUDA call and clear the runtime's last-error slot, so the
// error cannot resurface in a later launch check.
int cuda_err(cudaError_t e, const char *what) {
  (void)cudaGetLastError();
  return fail(TDFS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Choose the launch shape: a persistent grid of (resident CTAs per SM) x SMs.
}  // namespace

int launch_shape(const tdfs_graph *g, int kmax, bool labeled, const tdfs_options &o, LaunchShape *out) {
  // device properties are queried once per device (the query costs ~ms);
  // host threads that make their first calls at once fill the cache under
  // the lock, and readers copy the entry out under it
  static cudaDeviceProp props[64];
  static bool have[64] = {};
  static std::mutex mu;
  if (g->device < 0 || g->device >= 64) return fail(TDFS_ERR_ARG, "device index");
  cudaDeviceProp prop;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!have[g->device]) {
      cudaError_t e = cudaGetDeviceProperties(&props[g->device], g->device);
      if (e != cudaSuccess) return cuda_err(e, "cudaGetDeviceProperties");
      have[g->device] = true;
    }
    prop = props[g->device];
  }
  LaunchShape s;
  std::memset(&s, 0, sizeof s);
  s.warps_per_block = o.warps_per_block > 0 ? o.warps_per_block : 8;
  if (s.warps_per_block > 8) return fail(TDFS_ERR_ARG, "warps_per_block must be <= 8");
  // automatic depth per launch: small for patterns of at most 4 vertices
  // (their short DFS gains from more resident warps), large for 5, and 256
  // for the two extra stored levels of 6 and 7
  int cap = o.chunk_cap > 0 ? o.chunk_cap : (kmax >= 6 ? 256 : kmax == 5 ? 512 : 128);
  cap = (cap + 31) & ~31;
  if (cap < 64 || cap > 8192) return fail(TDFS_ERR_ARG, "chunk_cap must lie in [64, 8192]");
  int window = o.merge_window == 0 ? 128 : (o.merge_window < 0 ? 0 : o.merge_window);
  if (window % 128 != 0 || window > 256) return fail(TDFS_ERR_ARG, "merge_window must be 0, -1, 128 or 256");
  KernelCfg &c = s.cfg;
  c.cap = cap;
  c.window = window;
  c.fixed = o.fixed_stage < 0 ? 0 : 1;
  c.split_after_ns = o.split_after_us > 0 ? o.split_after_us * 1000 : (o.split_after_us < 0 ? 0 : 150000);
  c.warp_bytes = (int)((warp_smem_bytes(kmax, cap, window, c.fixed != 0) + 15) & ~(size_t)15);
  c.steal = o.steal < 0 ? 1 : (o.steal ? 1 : 0);
  if (o.wait_limit_ms < 0) return fail(TDFS_ERR_ARG, "wait_limit_ms must be >= 0");
  if (o.work_budget < 0) return fail(TDFS_ERR_ARG, "work_budget must be >= 0");
  c.idle_ms = o.wait_limit_ms > 0 ? o.wait_limit_ms : 30000;
  c.budgeted = o.work_budget > 0 ? 1 : 0;
  c.steal_min = o.steal_min > 0 ? o.steal_min : 2;
  c.steal_first = o.steal_first > 0 ? o.steal_first : 8;
  c.leaf_min = o.leaf_steal_min > 0 ? o.leaf_steal_min : (o.leaf_steal_min < 0 ? 2 : 64);
  c.hoist = o.level_hoist < 0 ? 0 : 1;
  c.segments = o.label_rows < 0 ? 0 : 1;
  c.tail = o.tail_count < 0 ? 0 : 1;
  c.prune = o.dead_prune < 0 ? 0 : 1;
  c.lane_list = o.lane_list > 0 ? o.lane_list : (o.lane_list < 0 ? 0 : 32);
  c.merge_ratio = o.merge_ratio > 0 ? o.merge_ratio : 4;
  if (c.steal_min < 2 || c.steal_min > 4096) return fail(TDFS_ERR_ARG, "steal_min must lie in [2, 4096]");
  if (c.steal_first < 2 || c.steal_first > 4096) return fail(TDFS_ERR_ARG, "steal_first must lie in [2, 4096]");
  if (c.lane_list > 4096) return fail(TDFS_ERR_ARG, "lane_list must be at most 4096");
  if (o.edge_chunk < 0 || o.edge_chunk > 32 || (o.edge_chunk & (o.edge_chunk - 1)) != 0)
    return fail(TDFS_ERR_ARG, "edge_chunk must be 0 or a power of two up to 32");
  const size_t smem = (size_t)c.warp_bytes * s.warps_per_block;
  if (smem > (size_t)prop.sharedMemPerBlockOptin)
    return fail(TDFS_ERR_CAPACITY, "per-CTA shared memory %zu exceeds %zu; lower chunk_cap or warps_per_block",
                smem, (size_t)prop.sharedMemPerBlockOptin);
  // occupancy of both register budgets, cached per (device, mode, CTA shape):
  // the queries set a kernel attribute and cost tens of microseconds, which
  // a small launch would otherwise pay on every call
  int fit = -1, fit_wide = -1;
  {
    static std::map<std::tuple<int, bool, int, size_t>, std::pair<int, int>> occ;
    static std::mutex occ_mu;
    const auto key = std::make_tuple(g->device, labeled, s.warps_per_block, smem);
    std::lock_guard<std::mutex> lk(occ_mu);
    auto it = occ.find(key);
    if (it == occ.end()) {
      fit = resident_blocks_per_sm(labeled, s.warps_per_block, smem, false);
      fit_wide = resident_blocks_per_sm(labeled, s.warps_per_block, smem, true);
      if (fit < 0 || fit_wide < 0)
        return fail(TDFS_ERR_CUDA, "occupancy query failed: %s", cudaGetErrorString(cudaGetLastError()));
      occ[key] = {fit, fit_wide};
    } else {
      fit = it->second.first;
      fit_wide = it->second.second;
    }
  }
  if (fit == 0) return fail(TDFS_ERR_CAPACITY, "the match kernel does not fit on an SM with this shape");
  // a persistent grid: every CTA resident at once (idle warps wait on busy ones);
  // the 80-register build whenever it holds as many CTAs per SM
  const int per_sm = o.blocks_per_sm > 0 ? std::min(o.blocks_per_sm, fit) : fit;
  c.wide_regs = per_sm <= fit_wide ? 1 : 0;
  s.blocks = prop.multiProcessorCount * per_sm;
  // the tail rush (opt-in): once a quarter of the grid is idle, split after
  // split_rush_us.  Off by default: on the labeled ER batch (config 3) it
  // turned 2.4 ms into 3.4 ms -- the extra splits of small subtrees cost more
  // than the idle time they recover.
  if (o.split_rush_us <= 0 || c.split_after_ns == 0) {
    c.rush_hungry = 0;
  } else {
    c.rush_hungry = std::max(1, s.blocks * s.warps_per_block / 4);
    c.rush_ns = o.split_rush_us * 1000;
    if (c.rush_ns > c.split_after_ns) c.rush_ns = c.split_after_ns;
  }
  *out = s;
  return TDFS_OK;
}

// The level-0 range of a slot: the edge ids [eb, ee), or -- for a labeled
// plan on a graph with a label index -- the positions of the index group of
// the plan's first two labels that hold those ids.
void level0_range(const tdfs_graph *g, const DevPlan &p, int64_t eb, int64_t ee, bool use_index, SlotInfo *in) {
  ee = std::max(eb, ee);
  in->perm = 0;
  if (use_index && p.labeled && g->lindex &&
      label_range(*g->lindex, p.label[0], p.label[1], eb, ee, &in->e_begin, &in->e_end)) {
    in->perm = 1;
    return;
  }
  in->e_begin = eb;
  in->e_end = ee;
}

namespace {

// Level-0 tickets of an edge range dealt round-robin: ticket t covers the
// chunk of `chunk` edges starting at e_begin + (t * stride + phase) * chunk.
int64_t ticket_count(int64_t b, int64_t e, int stride, int phase, int chunk) {
  const int64_t chunks = (e - b + chunk - 1) / chunk;
  if (chunks <= phase) return 0;
  return (chunks - phase + stride - 1) / stride;
}

// Captured launches: one CUDA graph per (batch size, mode, launch shape)
// holding the slot-table upload from the pinned staging copy, the control
// reset, the kernel and the read-back; replays read the staging copy as it is
// at replay time.
struct GraphEntry {
  int n;
  bool labeled;
  int blocks, warps;
  KernelCfg cfg;
  cudaGraphExec_t exec;
  cudaEvent_t k0, k1;  // recorded inside the graph around the match kernel
};

}  // namespace

void release_graphs(tdfs_graph *g) {
  if (!g->graphs) return;
  auto *v = static_cast<std::vector<GraphEntry> *>(g->graphs);
  for (auto &c : *v) {
    cudaGraphExecDestroy(c.exec);
    cudaEventDestroy(c.k0);
    cudaEventDestroy(c.k1);
  }
  delete v;
  g->graphs = nullptr;
}

namespace {

std::vector<GraphEntry> &graph_cache(tdfs_graph *g) {
  if (!g->graphs) g->graphs = new std::vector<GraphEntry>();
  return *static_cast<std::vector<GraphEntry> *>(g->graphs);
}

int enqueue_launch(tdfs_graph *g, const LaunchShape &s, bool labeled, int n, cudaStream_t st, cudaEvent_t k0,
                   cudaEvent_t k1) {
  SlotTable *h = g->htab, *d = g->tab;
  cudaError_t e = cudaMemcpyAsync(&d->ctl, &h->ctl, sizeof h->ctl, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->hot, h->hot, sizeof(SlotHot) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->info, h->info, sizeof(SlotInfo) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->plan, h->plan, sizeof(DevPlan) * n, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_err(e, "slot table upload");
  init_launch(g->ctl, queue_hdr(g), st);
  // external records: captured as event-record nodes, so they time the
  // kernel when the graph replays (a plain record is only a join point)
  e = cudaEventRecordWithFlags(k0, st, cudaEventRecordExternal);
  if (e != cudaSuccess) return cuda_err(e, "kernel start event");
  int rc = launch_match(labeled, graph_view(g), g->ctl, d, g->queue, queue_hdr(g), s.cfg, s.blocks,
                        s.warps_per_block, st);
  if (rc) return rc;
  e = cudaEventRecordWithFlags(k1, st, cudaEventRecordExternal);
  if (e != cudaSuccess) return cuda_err(e, "kernel end event");
  e = cudaMemcpyAsync(h->hot, d->hot, sizeof(SlotHot) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(g->hctl, g->ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_err(e, "read-back");
  return TDFS_OK;
}

// Counts of a finished launch from the read-back slot lines.  A slot that ran
// out of its work budget gets status TDFS_ERR_TIMEOUT and count 0; without a
// status array that fails the call.
int collect(const RunCtl &hc, const SlotHot *hot, int n, unsigned long long *raw, int *status) {
  if (hc.error == TDFS_ERR_TIMEOUT) return fail(TDFS_ERR_TIMEOUT, "a bounded device wait ran out");
  if (hc.error) return fail(hc.error, "device error %d", hc.error);
  int first_abort = -1;
  for (int i = 0; i < n; ++i) {
    if (hot[i].state != kSlotDone) return fail(TDFS_ERR_TIMEOUT, "slot %d did not complete", i);
    const bool ab = hot[i].aborted != 0;
    raw[i] = ab ? 0 : hot[i].count;
    if (status) status[i] = ab ? TDFS_ERR_TIMEOUT : TDFS_OK;
    if (ab && first_abort < 0) first_abort = i;
  }
  if (first_abort >= 0 && !status)
    return fail(TDFS_ERR_TIMEOUT, "pattern %d ran out of its work budget", first_abort);
  return TDFS_OK;
}

int run_captured(tdfs_graph *g, const LaunchShape &s, bool labeled, int n, float *ms, unsigned long long *raw,
                 int *status) {
  cudaError_t e;
  if (!g->ws->gstream) {
    cudaStream_t st;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_err(e, "capture stream");
    g->ws->gstream = st;
  }
  cudaStream_t st = static_cast<cudaStream_t>(g->ws->gstream);
  auto &cache = graph_cache(g);
  const GraphEntry *hit = nullptr;
  for (auto &c : cache)
    if (c.n == n && c.labeled == labeled && c.blocks == s.blocks && c.warps == s.warps_per_block &&
        !std::memcmp(&c.cfg, &s.cfg, sizeof c.cfg))
      hit = &c;
  if (!hit) {
    GraphEntry ent{n, labeled, s.blocks, s.warps_per_block, s.cfg, nullptr, nullptr, nullptr};
    e = cudaEventCreate(&ent.k0);
    if (e == cudaSuccess) e = cudaEventCreate(&ent.k1);
    if (e != cudaSuccess) return cuda_err(e, "cudaEventCreate");
    cudaGraph_t graph;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_err(e, "cudaStreamBeginCapture");
    int rc = enqueue_launch(g, s, labeled, n, st, ent.k0, ent.k1);
    e = cudaStreamEndCapture(st, &graph);
    if (!rc && e == cudaSuccess) {
      e = cudaGraphInstantiate(&ent.exec, graph, 0);
      cudaGraphDestroy(graph);
    }
    if (rc || e != cudaSuccess) {
      cudaEventDestroy(ent.k0);
      cudaEventDestroy(ent.k1);
      return rc ? rc : cuda_err(e, "capturing the launch");
    }
    cache.push_back(ent);
    hit = &cache.back();
  }
  e = cudaGraphLaunch(hit->exec, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  // the match kernel's own time, from the event nodes around it in the graph
  if (e == cudaSuccess && ms) e = cudaEventElapsedTime(ms, hit->k0, hit->k1);
  if (e != cudaSuccess) return cuda_err(e, "graph launch");
  return collect(*g->hctl, g->htab->hot, n, raw, status);
}

// One launch over n plans of the same mode: slot i counts plans[i] on the
// option's edge range; raw[i] receives the count before the |Aut| multiplier.
int run_batch(tdfs_graph *g, const DevPlan *const *plans, int n, const tdfs_options &o, unsigned long long *raw,
              int *status, float *ms) {
  if (n <= 0) return TDFS_OK;
  if (n > kMaxSlots) return fail(TDFS_ERR_CAPACITY, "at most %d plans per launch", kMaxSlots);
  const bool labeled = plans[0]->labeled != 0;
  int kmax = 3;
  for (int i = 0; i < n; ++i) {
    if ((plans[i]->labeled != 0) != labeled) return fail(TDFS_ERR_ARG, "a launch mixes labeled and unlabeled plans");
    kmax = std::max(kmax, (int)plans[i]->k);
  }
  if (labeled && !g->labeled) return fail(TDFS_ERR_ARG, "labeled pattern on a graph opened without labels");
  cudaError_t e = cudaSetDevice(g->device);
  if (e != cudaSuccess) return cuda_err(e, "cudaSetDevice");
  LaunchShape s;
  int rc = launch_shape(g, kmax, labeled, o, &s);
  if (rc) return rc;
  if ((rc = acquire_workspace(g))) return rc;
  const int64_t eb = std::max<int64_t>(0, o.edge_begin);
  const int64_t ee = (o.edge_end < 0 || o.edge_end > g->nedges) ? g->nedges : o.edge_end;
  const int stride = o.edge_stride > 0 ? o.edge_stride : 1;
  if (o.edge_phase < 0 || o.edge_phase >= stride) return fail(TDFS_ERR_ARG, "edge_phase must lie in [0, edge_stride)");
  SlotTable *h = g->htab;
  std::memset(&h->ctl, 0, sizeof h->ctl);
  h->ctl.admitted = (unsigned long long)n;
  h->ctl.shutdown = 1;
  const int warps = s.blocks * s.warps_per_block;
  for (int i = 0; i < n; ++i) {
    SlotInfo &in = h->info[i];
    level0_range(g, *plans[i], eb, ee, o.label_index >= 0, &in);
    in.stride = stride;
    in.phase = o.edge_phase;
    in.chunk = auto_chunk(in.e_end - in.e_begin, stride, warps, o.edge_chunk);
    in.ntickets = ticket_count(in.e_begin, in.e_end, stride, o.edge_phase, in.chunk);
    in.budget = o.work_budget;
    std::memset(&h->hot[i], 0, sizeof h->hot[i]);
    h->hot[i].state = in.ntickets > 0 ? kSlotActive : kSlotDone;  // an empty range is done at once
    if (in.ntickets == 0) ++h->ctl.completed;
    h->plan[i] = *plans[i];
  }
  g->last_warps = (int64_t)s.blocks * s.warps_per_block;
  if (o.graph_capture) return run_captured(g, s, labeled, n, ms, raw, status);
  cudaStream_t st = static_cast<cudaStream_t>(o.stream);
  SlotTable *d = g->tab;
  e = cudaMemcpyAsync(&d->ctl, &h->ctl, sizeof h->ctl, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->hot, h->hot, sizeof(SlotHot) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->info, h->info, sizeof(SlotInfo) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d->plan, h->plan, sizeof(DevPlan) * n, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_err(e, "slot table upload");
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  if (ms) {
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
  }
  init_launch(g->ctl, queue_hdr(g), st);
  if (ms) cudaEventRecord(ev0, st);
  rc = launch_match(labeled, graph_view(g), g->ctl, d, g->queue, queue_hdr(g), s.cfg, s.blocks, s.warps_per_block, st);
  if (ms) cudaEventRecord(ev1, st);
  if (!rc) {
    e = cudaMemcpyAsync(h->hot, d->hot, sizeof(SlotHot) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(g->hctl, g->ctl, sizeof(RunCtl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_err(e, "match kernel");
  }
  if (!rc && ms) {
    e = cudaEventElapsedTime(ms, ev0, ev1);
    if (e != cudaSuccess) rc = cuda_err(e, "cudaEventElapsedTime");
  }
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (rc) return rc;
  return collect(*g->hctl, h->hot, n, raw, status);
}

}  // namespace
}  // namespace tdfs

namespace tdfs {
const DevPlan &plan_device_table(const tdfs_plan *p) { return p->dev; }
}  // namespace tdfs

using namespace tdfs;

extern "C" {

int tdfs_version(void) { return 1; }

void tdfs_options_default(tdfs_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->steal = -1;
  o->edge_end = -1;
  o->edge_stride = 1;
}

int tdfs_graph_open(const char *prefix, int labeled, int device, tdfs_graph **out) {
  if (!prefix || !out) return fail(TDFS_ERR_ARG, "null argument");
  tdfs_csr *c = nullptr;
  int rc = tdfs_csr_read(prefix, labeled, &c);
  if (rc) return rc;
  rc = graph_upload(c->n, c->nedges, c->rowptr.data(), c->colidx.data(), labeled ? c->labels.data() : nullptr,
                    device, c->max_degree, out);
  delete c;
  return rc;
}

int tdfs_graph_from_csr(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx,
                        const int32_t *labels, int device, tdfs_graph **out) {
  if (!rowptr || (!colidx && nedges) || !out) return fail(TDFS_ERR_ARG, "null argument");
  int32_t md = 0;
  int rc = validate_csr(n, nedges, rowptr, colidx, &md);
  if (rc) return rc;
  return graph_upload(n, nedges, rowptr, colidx, labels, device, md, out);
}

int tdfs_graph_info(const tdfs_graph *g, int64_t *n, int64_t *nedges, int32_t *max_degree, int *labeled,
                    size_t *device_bytes) {
  if (!g) return fail(TDFS_ERR_ARG, "null graph");
  if (n) *n = g->n;
  if (nedges) *nedges = g->nedges;
  if (max_degree) *max_degree = g->max_degree;
  if (labeled) *labeled = g->labeled;
  if (device_bytes) *device_bytes = g->bytes;
  return TDFS_OK;
}

int tdfs_graph_free(tdfs_graph *g) {
  graph_release(g);
  return TDFS_OK;
}

int tdfs_plan_from_text(const char *text, int labeled, tdfs_plan **out) {
  if (!text || !out) return fail(TDFS_ERR_ARG, "null argument");
  auto p = std::make_unique<tdfs_plan>();
  int rc = compile_pattern(text, labeled != 0, &p->host);
  if (rc) return rc;
  p->dev = p->host.to_device();
  *out = p.release();
  return TDFS_OK;
}

int tdfs_plan_compile(const char *gpath, int labeled, tdfs_plan **out) {
  if (!gpath || !out) return fail(TDFS_ERR_ARG, "null argument");
  std::ifstream f(gpath);
  if (!f) return fail(TDFS_ERR_IO, "cannot open %s", gpath);
  std::stringstream ss;
  ss << f.rdbuf();
  return tdfs_plan_from_text(ss.str().c_str(), labeled, out);
}

int tdfs_plan_dump(const tdfs_plan *p, char *buf, size_t cap, size_t *len) {
  if (!p) return fail(TDFS_ERR_ARG, "null plan");
  const std::string s = p->host.dump_json();
  if (len) *len = s.size() + 1;
  if (buf && cap) {
    const size_t n = std::min(cap - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = 0;
    if (n < s.size()) return fail(TDFS_ERR_ARG, "buffer too small (%zu needed)", s.size() + 1);
  }
  return TDFS_OK;
}

int tdfs_plan_info(const tdfs_plan *p, int *k, int *labeled, int64_t *multiplicity) {
  if (!p) return fail(TDFS_ERR_ARG, "null plan");
  if (k) *k = p->host.k;
  if (labeled) *labeled = p->host.labeled;
  if (multiplicity) *multiplicity = p->host.multiplicity;
  return TDFS_OK;
}

int tdfs_plan_free(tdfs_plan *p) {
  delete p;
  return TDFS_OK;
}

int tdfs_count(tdfs_graph *g, const tdfs_plan *p, const tdfs_options *opt, uint64_t *count, float *kernel_ms) {
  if (!g || !p || !count) return fail(TDFS_ERR_ARG, "null argument");
  tdfs_options o;
  if (opt) o = *opt; else tdfs_options_default(&o);
  unsigned long long raw = 0;
  const DevPlan *dp = &p->dev;
  int rc = run_batch(g, &dp, 1, o, &raw, nullptr, kernel_ms);
  if (rc) return rc;
  // cu_test.cu:100-105: the unlabeled total is multiplied by |Aut|
  *count = (uint64_t)(raw * (unsigned long long)p->dev.multiplicity);
  return TDFS_OK;
}

int tdfs_count_batch(tdfs_graph *g, const tdfs_plan *const *plans, int nplans, const tdfs_options *opt,
                     uint64_t *counts, float *kernel_ms) {
  return tdfs_count_batch_status(g, plans, nplans, opt, counts, nullptr, kernel_ms);
}

int tdfs_count_batch_status(tdfs_graph *g, const tdfs_plan *const *plans, int nplans, const tdfs_options *opt,
                            uint64_t *counts, int *status, float *kernel_ms) {
  if (!g || (!plans && nplans) || (!counts && nplans) || nplans < 0) return fail(TDFS_ERR_ARG, "bad arguments");
  tdfs_options o;
  if (opt) o = *opt; else tdfs_options_default(&o);
  float total = 0.f;
  // one launch per mode (a launch runs either the labeled or the unlabeled kernel)
  for (int mode = 0; mode < 2; ++mode) {
    std::vector<const DevPlan *> dp;
    std::vector<int> idx;
    for (int i = 0; i < nplans; ++i) {
      if (!plans[i]) return fail(TDFS_ERR_ARG, "null plan %d", i);
      if ((plans[i]->dev.labeled != 0) == (mode == 1)) {
        dp.push_back(&plans[i]->dev);
        idx.push_back(i);
      }
    }
    for (size_t b = 0; b < dp.size(); b += kMaxSlots) {
      const int n = (int)std::min<size_t>(kMaxSlots, dp.size() - b);
      std::vector<unsigned long long> raw(n);
      std::vector<int> st(n, TDFS_OK);
      float ms = 0.f;
      int rc = run_batch(g, dp.data() + b, n, o, raw.data(), status ? st.data() : nullptr, kernel_ms ? &ms : nullptr);
      if (rc) return rc;
      total += ms;
      for (int j = 0; j < n; ++j) {
        counts[idx[b + j]] = (uint64_t)(raw[j] * (unsigned long long)dp[b + j]->multiplicity);
        if (status) status[idx[b + j]] = st[j];
      }
    }
  }
  if (kernel_ms) *kernel_ms = total;
  return TDFS_OK;
}

int tdfs_autotune(tdfs_graph *g, const tdfs_plan *const *plans, int nplans, const tdfs_options *base,
                  int sample_stride, tdfs_options *best, float *best_ms) {
  if (!g || !plans || nplans <= 0 || !best) return fail(TDFS_ERR_ARG, "bad arguments");
  tdfs_options b;
  if (base) b = *base; else tdfs_options_default(&b);
  if (sample_stride < 1) sample_stride = 1;
  // resolve the automatic values so every knob has a concrete start
  tdfs_options cur = b;
  if (cur.warps_per_block <= 0) cur.warps_per_block = 8;
  // chunk_cap stays automatic (0) unless a fixed depth wins: the automatic
  // depth is chosen per launch, so a batch that mixes modes gets each
  // launch's own
  cur.chunk_cap = std::max(0, cur.chunk_cap);
  if (cur.merge_window == 0) cur.merge_window = 128;
  if (cur.steal < 0) cur.steal = 1;
  if (cur.steal_min <= 0) cur.steal_min = 2;
  if (cur.merge_ratio <= 0) cur.merge_ratio = 4;
  if (cur.tail_count == 0) cur.tail_count = 1;
  if (cur.dead_prune == 0) cur.dead_prune = 1;
  cur.edge_stride = sample_stride;
  cur.edge_phase = 0;
  std::vector<uint64_t> counts(nplans);
  std::vector<int> status(nplans);
  // the score is the sample's kernel time per completed plan, scaled to the
  // batch: the plain time when every plan completes; under a work budget a
  // shape that completes more plans in the same time scores better (a plan
  // abandoned early is cheap, but it is not an answer)
  auto measure = [&](const tdfs_options &o, float *out) -> int {
    float bestt = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {
      float ms = 0.f;
      int rc = tdfs_count_batch_status(g, plans, nplans, &o, counts.data(), status.data(), &ms);
      if (rc) return rc;
      int done = 0;
      for (int i = 0; i < nplans; ++i) done += status[i] == TDFS_OK;
      bestt = std::min(bestt, ms * (float)nplans / (float)std::max(1, done));
    }
    *out = bestt;
    return TDFS_OK;
  };
  float cur_ms = 0.f;
  int rc = measure(cur, &cur_ms);
  if (rc) return rc;
  struct Knob {
    int tdfs_options::*field;
    std::vector<int> values;
  };
  const std::vector<Knob> knobs = {
      {&tdfs_options::warps_per_block, {4, 8}},
      {&tdfs_options::chunk_cap, {64, 128, 256, 512, 1024}},
      {&tdfs_options::merge_window, {-1, 128, 256}},
      {&tdfs_options::merge_ratio, {1, 4, 16}},
      // (stealing stays on: without it one warp keeps a hub's whole subtree,
      // minutes on a power-law slice, and a launch cannot be cut short)
      {&tdfs_options::steal_min, {2, 8, 32}},
      {&tdfs_options::steal_first, {2, 8, 32}},
      {&tdfs_options::lane_list, {-1, 16, 64}},
      {&tdfs_options::blocks_per_sm, {1, 2, 3}},
      {&tdfs_options::edge_chunk, {1, 4, 8, 32}},
      {&tdfs_options::fixed_stage, {-1, 1}},
      {&tdfs_options::split_after_us, {-1, 5, 50, 150, 500}},
      {&tdfs_options::split_rush_us, {0, 10, 40}},
      {&tdfs_options::leaf_steal_min, {-1, 16, 64, 256}},
      {&tdfs_options::level_hoist, {-1, 1}},
      {&tdfs_options::tail_count, {-1, 1}},
      {&tdfs_options::dead_prune, {-1, 1}},
  };
  for (const Knob &k : knobs) {
    for (int v : k.values) {
      if (cur.*(k.field) == v) continue;
      tdfs_options t = cur;
      t.*(k.field) = v;
      float ms = 0.f;
      if (measure(t, &ms)) continue;  // a shape that does not fit is skipped
      if (ms < cur_ms * 0.97f) {
        cur = t;
        cur_ms = ms;
      }
    }
  }
  cur.edge_stride = b.edge_stride;
  cur.edge_phase = b.edge_phase;
  *best = cur;
  if (best_ms) *best_ms = cur_ms;
  return TDFS_OK;
}

int tdfs_selftest_wait_limit(tdfs_graph *g, int wait_limit_ms, float *kernel_ms) {
  if (!g || wait_limit_ms <= 0 || wait_limit_ms > 60000) return fail(TDFS_ERR_ARG, "wait_limit_ms must lie in [1, 60000]");
  cudaError_t e = cudaSetDevice(g->device);
  if (e != cudaSuccess) return cuda_err(e, "cudaSetDevice");
  tdfs_options o;
  tdfs_options_default(&o);
  o.wait_limit_ms = wait_limit_ms;
  LaunchShape s;
  int rc = launch_shape(g, 3, false, o, &s);
  if (rc) return rc;
  if ((rc = acquire_workspace(g))) return rc;
  // one admitted slot that no warp can ever complete: active, no tickets,
  // no holds -- every warp finds no work and waits until its bound runs out
  SlotTable *h = g->htab, *d = g->tab;
  std::memset(&h->ctl, 0, sizeof h->ctl);
  h->ctl.admitted = 1;
  h->ctl.shutdown = 1;
  std::memset(&h->hot[0], 0, sizeof h->hot[0]);
  h->hot[0].state = kSlotActive;
  std::memset(&h->info[0], 0, sizeof h->info[0]);
  h->info[0].stride = 1;
  h->info[0].chunk = 1;
  DevPlan p;
  std::memset(&p, 0, sizeof p);
  p.k = 3;
  h->plan[0] = p;
  e = cudaMemcpy(&d->ctl, &h->ctl, sizeof h->ctl, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d->hot, h->hot, sizeof(SlotHot), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d->info, h->info, sizeof(SlotInfo), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d->plan, h->plan, sizeof(DevPlan), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_err(e, "slot upload");
  cudaEvent_t ev0, ev1;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  init_launch(g->ctl, queue_hdr(g), nullptr);
  cudaEventRecord(ev0, nullptr);
  rc = launch_match(false, graph_view(g), g->ctl, d, g->queue, queue_hdr(g), s.cfg, s.blocks, s.warps_per_block,
                    nullptr);
  cudaEventRecord(ev1, nullptr);
  RunCtl hc;
  if (!rc) {
    e = cudaMemcpy(&hc, g->ctl, sizeof hc, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && kernel_ms) e = cudaEventElapsedTime(kernel_ms, ev0, ev1);
    if (e != cudaSuccess) rc = cuda_err(e, "self-test launch");
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (rc) return rc;
  if (hc.error) return fail(hc.error, "the launch reported device status %d after its bounded waits", hc.error);
  return TDFS_OK;
}

int tdfs_last_launch(const tdfs_graph *g, tdfs_launch_stats *st) {
  if (!g || !st) return fail(TDFS_ERR_ARG, "null argument");
  std::memset(st, 0, sizeof *st);
  if (!g->hctl || !g->last_warps) return fail(TDFS_ERR_ARG, "no launch on this graph yet");
  const RunCtl &c = *g->hctl;
  st->steals = c.steals;
  st->splits = c.splits;
  st->warps = g->last_warps;
  st->idle_fraction = c.warp_ns ? (double)c.idle_ns / (double)c.warp_ns : 0.0;
  st->mean_warp_ms = (double)c.warp_ns / 1e6 / (double)g->last_warps;
  return TDFS_OK;
}

struct tdfs_server {
  tdfs::Server *impl;
};

void tdfs_server_options_default(tdfs_server_options *o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->max_inflight = 256;
  o->max_k = TDFS_MAX_PATTERN;
  o->idle_exit_ms = 50;
  tdfs_options_default(&o->launch);
}

int tdfs_server_create(tdfs_graph *g, const tdfs_server_options *opt, tdfs_server **out) {
  if (!g || !out) return fail(TDFS_ERR_ARG, "null argument");
  Server *s = nullptr;
  int rc = server_create(g, opt, &s);
  if (rc) return rc;
  *out = new tdfs_server{s};
  return TDFS_OK;
}

int tdfs_server_submit(tdfs_server *s, const tdfs_plan *p, uint64_t *ticket) {
  if (!s || !p || !ticket) return fail(TDFS_ERR_ARG, "null argument");
  return server_submit(s->impl, p->dev, ticket);
}

int tdfs_server_wait(tdfs_server *s, uint64_t ticket, uint64_t *count, double *latency_us) {
  if (!s) return fail(TDFS_ERR_ARG, "null server");
  return server_wait(s->impl, ticket, count, latency_us);
}

int tdfs_server_stats(tdfs_server *s, tdfs_serve_stats *st) {
  if (!s || !st) return fail(TDFS_ERR_ARG, "null argument");
  return server_stats(s->impl, st);
}

int tdfs_server_destroy(tdfs_server *s) {
  if (!s) return TDFS_OK;
  const int rc = server_destroy(s->impl);
  delete s;
  return rc;
}

}  // extern "C"
