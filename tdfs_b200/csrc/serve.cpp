// serve.cpp -- continuous-batching query server over a device-resident graph.
//
// No counterpart in the reference (it counts one pattern per process run).
// A persistent match kernel (match.cu) runs in serving mode: its slot table
// stays open (`shutdown` = 0) and a host scheduler thread admits queries into
// fresh slots while earlier ones are still on the device, so the work of
// queries that arrive at different times overlaps on the GPU.
//
//   admission   a query is admitted when an in-flight place is free and its
//               estimated device bytes fit the budget; a query that can never
//               fit (pattern larger than the server's stack layout, or larger
//               than the whole budget) is rejected at submit with
//               TDFS_ERR_ADMISSION.
//   slots       admitted queries take consecutive slots of the table; a slot
//               is never reused while the kernel runs.  When the table is
//               spent the scheduler closes it (shutdown = 1), waits for the
//               kernel to drain, and opens a fresh table ("epoch").
//   completion  the completing warp marks its slot done on the device; the
//               scheduler polls the in-flight slots' state lines and hands the
//               counts to waiting callers.  Latency = completion seen on the
//               host minus submit time.
//   idle        the kernel retires after `idle_exit_ms` without work (bounded
//               wait); the scheduler relaunches it on the next admission.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "graph.h"
#include "match.cuh"
#include "plan.h"
#include "serve.h"

namespace tdfs {

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  uint64_t ticket;
  DevPlan plan;
  size_t bytes;
  Clock::time_point submitted;
};

struct Result {
  bool done = false;
  int error = 0;
  uint64_t count = 0;
  double latency_us = 0;
};

}  // namespace

// Device bytes a query is charged at admission: its slot record plus the DFS
// stack of one CTA (warps_per_block warps x (k - 2) candidate levels of `cap`
// vertices) and its share of split units, which bound what it can hold on the
// device at once.
size_t query_bytes(int k, int cap, int warps_per_block) {
  const size_t record = sizeof(SlotHot) + sizeof(SlotInfo) + sizeof(DevPlan);
  const size_t stack = (size_t)warps_per_block * (size_t)std::max(1, k - 2) * (size_t)cap * 4;
  const size_t units = (size_t)4 * sizeof(SplitUnit);
  return record + stack + units;
}

struct Server {
  tdfs_graph *g = nullptr;
  tdfs_server_options opt{};
  bool labeled = false;
  int cap = 256;
  LaunchShape shape{};
  cudaStream_t kstream = nullptr, cstream = nullptr;
  SlotHot *mirror = nullptr;  // pinned: polled copies of the in-flight slots' lines

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> pending;
  std::unordered_map<uint64_t, Result> results;
  uint64_t next_ticket = 1;
  bool stopping = false;
  int fatal = 0;
  std::string fatal_msg;

  // scheduler-thread state
  int next_slot = 0;              // slots [0, next_slot) of this epoch are admitted
  int lo_slot = 0;                // first slot not yet seen done
  std::vector<uint64_t> slot_ticket;
  std::vector<size_t> slot_bytes;
  std::vector<Clock::time_point> slot_submit;
  std::vector<char> slot_done;
  size_t used_bytes = 0;
  int inflight = 0;
  bool kernel_live = false;
  std::vector<double> latencies;
  uint64_t completed = 0;
  uint64_t aborted = 0;
  Clock::time_point first_submit{}, last_done{};
  std::thread th;
};

namespace {

int cuda_err(cudaError_t e, const char *what) {
  (void)cudaGetLastError();  // a reported error must not resurface in a later launch check
  return fail(TDFS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// Open a fresh slot table (no kernel may be running on it).
int open_epoch(Server &S) {
  SlotTable *h = S.g->htab;
  std::memset(&h->ctl, 0, sizeof h->ctl);
  h->ctl.idle_exit_ms = S.opt.idle_exit_ms;
  cudaError_t e = cudaMemcpyAsync(&S.g->tab->ctl, &h->ctl, sizeof h->ctl, cudaMemcpyHostToDevice, S.cstream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S.cstream);
  if (e != cudaSuccess) return cuda_err(e, "server epoch");
  S.next_slot = S.lo_slot = 0;
  std::fill(S.slot_done.begin(), S.slot_done.end(), 0);
  return TDFS_OK;
}

int launch_kernel(Server &S) {
  init_launch(S.g->ctl, queue_hdr(S.g), S.kstream);
  int rc = launch_match(S.labeled, graph_view(S.g), S.g->ctl, S.g->tab, S.g->queue, queue_hdr(S.g), S.shape.cfg,
                        S.shape.blocks, S.shape.warps_per_block, S.kstream);
  if (!rc) S.kernel_live = true;
  return rc;
}

// Is the persistent kernel still running?  Reports a device error it ended with.
int kernel_state(Server &S, bool *running) {
  *running = false;
  if (!S.kernel_live) return TDFS_OK;
  cudaError_t e = cudaStreamQuery(S.kstream);
  if (e == cudaErrorNotReady) {
    *running = true;
    return TDFS_OK;
  }
  S.kernel_live = false;
  if (e != cudaSuccess) return cuda_err(e, "serving kernel");
  RunCtl hc;
  e = cudaMemcpy(&hc, S.g->ctl, sizeof hc, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_err(e, "serving kernel status");
  if (hc.error) return fail(hc.error, "serving kernel raised device error %d", hc.error);
  return TDFS_OK;
}

// Admit pending queries into slots (scheduler thread, lock held by caller
// only while taking from `pending`).
int admit(Server &S, std::vector<Pending> &batch) {
  if (batch.empty()) return TDFS_OK;
  SlotTable *h = S.g->htab;
  const int first = S.next_slot;
  for (const Pending &q : batch) {
    const int s = S.next_slot++;
    SlotInfo &in = h->info[s];
    level0_range(S.g, q.plan, 0, S.g->nedges, S.opt.launch.label_index >= 0, &in);
    in.stride = 1;
    in.phase = 0;
    in.chunk = auto_chunk(in.e_end - in.e_begin, 1, S.shape.blocks * S.shape.warps_per_block, S.opt.launch.edge_chunk);
    in.ntickets = (in.e_end - in.e_begin + in.chunk - 1) / in.chunk;
    in.budget = S.opt.launch.work_budget;
    std::memset(&h->hot[s], 0, sizeof h->hot[s]);
    h->hot[s].state = in.ntickets > 0 ? kSlotActive : kSlotDone;  // labels no edge has: done at once
    h->plan[s] = q.plan;
    S.slot_ticket[s] = q.ticket;
    S.slot_bytes[s] = q.bytes;
    S.slot_submit[s] = q.submitted;
    S.slot_done[s] = 0;
    S.used_bytes += q.bytes;
    ++S.inflight;
  }
  const int n = S.next_slot - first;
  SlotTable *d = S.g->tab;
  cudaError_t e = cudaMemcpyAsync(d->hot + first, h->hot + first, sizeof(SlotHot) * n, cudaMemcpyHostToDevice,
                                  S.cstream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d->info + first, h->info + first, sizeof(SlotInfo) * n, cudaMemcpyHostToDevice, S.cstream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d->plan + first, h->plan + first, sizeof(DevPlan) * n, cudaMemcpyHostToDevice, S.cstream);
  // the records are complete on the device before `admitted` exposes them
  h->ctl.admitted = (unsigned long long)S.next_slot;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&d->ctl.admitted, &h->ctl.admitted, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                        S.cstream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S.cstream);
  if (e != cudaSuccess) return cuda_err(e, "server admission");
  return TDFS_OK;
}

// Poll the in-flight slots; deliver finished ones.
int poll(Server &S) {
  if (S.lo_slot >= S.next_slot) return TDFS_OK;
  const int lo = S.lo_slot, n = S.next_slot - lo;
  cudaError_t e =
      cudaMemcpyAsync(S.mirror + lo, S.g->tab->hot + lo, sizeof(SlotHot) * n, cudaMemcpyDeviceToHost, S.cstream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S.cstream);
  if (e != cudaSuccess) return cuda_err(e, "server poll");
  const auto now = Clock::now();
  std::lock_guard<std::mutex> lk(S.mu);
  for (int s = lo; s < S.next_slot; ++s) {
    if (S.slot_done[s] || S.mirror[s].state != kSlotDone) continue;
    S.slot_done[s] = 1;
    Result &r = S.results[S.slot_ticket[s]];
    r.done = true;
    if (S.mirror[s].aborted) {
      r.error = TDFS_ERR_TIMEOUT;  // ran out of its work budget: no valid count
      ++S.aborted;
    } else {
      r.count = (uint64_t)(S.mirror[s].count * (unsigned long long)S.g->htab->plan[s].multiplicity);
    }
    r.latency_us = std::chrono::duration<double, std::micro>(now - S.slot_submit[s]).count();
    S.latencies.push_back(r.latency_us);
    S.used_bytes -= S.slot_bytes[s];
    --S.inflight;
    ++S.completed;
    S.last_done = now;
  }
  while (S.lo_slot < S.next_slot && S.slot_done[S.lo_slot]) ++S.lo_slot;
  S.cv_done.notify_all();
  return TDFS_OK;
}

void fail_all(Server &S, int rc) {
  std::lock_guard<std::mutex> lk(S.mu);
  S.fatal = rc;
  S.fatal_msg = tdfs_last_error();
  for (auto &kv : S.results)
    if (!kv.second.done) {
      kv.second.done = true;
      kv.second.error = rc;
    }
  for (const Pending &q : S.pending) S.results[q.ticket] = Result{true, rc, 0, 0};
  S.pending.clear();
  S.cv_done.notify_all();
}

void scheduler(Server *SP) {
  Server &S = *SP;
  cudaSetDevice(S.g->device);
  int rc = open_epoch(S);
  while (!rc) {
    std::vector<Pending> batch;
    bool stop = false;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      if (S.pending.empty() && S.inflight == 0 && !S.stopping)
        S.cv_work.wait_for(lk, std::chrono::milliseconds(5));
      stop = S.stopping && S.pending.empty() && S.inflight == 0;
      // admission: in-flight places, memory budget, and room left in the table
      while (!S.pending.empty() && S.inflight + (int)batch.size() < S.opt.max_inflight &&
             S.next_slot + (int)batch.size() < kMaxSlots) {
        size_t bytes = 0;
        for (const Pending &q : batch) bytes += q.bytes;
        if (S.used_bytes + bytes + S.pending.front().bytes > S.opt.mem_budget) break;
        batch.push_back(S.pending.front());
        S.pending.pop_front();
      }
    }
    if (stop) break;
    if (!batch.empty()) {
      if ((rc = admit(S, batch))) break;
    }
    bool running = false;
    if ((rc = kernel_state(S, &running))) break;
    if (!running && S.inflight > 0) {
      if ((rc = launch_kernel(S))) break;
    }
    if ((rc = poll(S))) break;
    // a spent table: close it, let the kernel drain, open the next epoch
    if (S.next_slot + 1 >= kMaxSlots && S.inflight == 0) {
      int one = 1;
      cudaError_t e = cudaMemcpyAsync(&S.g->tab->ctl.shutdown, &one, sizeof one, cudaMemcpyHostToDevice, S.cstream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(S.cstream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(S.kstream);
      if (e != cudaSuccess) {
        rc = cuda_err(e, "server epoch close");
        break;
      }
      S.kernel_live = false;
      if ((rc = open_epoch(S))) break;
    }
    if (batch.empty() && S.inflight > 0) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  if (rc) {
    fail_all(S, rc);
    return;
  }
  // drain: close the table so the kernel retires
  int one = 1;
  cudaMemcpyAsync(&S.g->tab->ctl.shutdown, &one, sizeof one, cudaMemcpyHostToDevice, S.cstream);
  cudaStreamSynchronize(S.cstream);
  cudaStreamSynchronize(S.kstream);
}

}  // namespace

int server_create(tdfs_graph *g, const tdfs_server_options *o, Server **out) {
  auto S = std::make_unique<Server>();
  S->g = g;
  tdfs_server_options_default(&S->opt);
  if (o) S->opt = *o;
  if (S->opt.max_k < 3 || S->opt.max_k > kMaxK) return fail(TDFS_ERR_ARG, "max_k must lie in [3, 7]");
  if (S->opt.max_inflight < 1 || S->opt.max_inflight > kMaxSlots / 2)
    return fail(TDFS_ERR_ARG, "max_inflight must lie in [1, %d]", kMaxSlots / 2);
  if (S->opt.idle_exit_ms < 1) S->opt.idle_exit_ms = 50;
  S->labeled = S->opt.labeled != 0;
  if (S->labeled && !g->labeled) return fail(TDFS_ERR_ARG, "labeled server on a graph opened without labels");
  cudaError_t e = cudaSetDevice(g->device);
  if (e != cudaSuccess) return cuda_err(e, "cudaSetDevice");
  tdfs_options lo = S->opt.launch;
  int rc = launch_shape(g, S->opt.max_k, S->labeled, lo, &S->shape);
  if (rc) return rc;
  if ((rc = acquire_workspace(g))) return rc;
  S->cap = S->shape.cfg.cap;
  if (S->opt.mem_budget == 0)
    S->opt.mem_budget = (size_t)S->opt.max_inflight * query_bytes(S->opt.max_k, S->cap, S->shape.warps_per_block);
  e = cudaStreamCreateWithFlags(&S->kstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->cstream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMallocHost(&S->mirror, sizeof(SlotHot) * kMaxSlots);
  if (e != cudaSuccess) return cuda_err(e, "server streams");
  S->slot_ticket.assign(kMaxSlots, 0);
  S->slot_bytes.assign(kMaxSlots, 0);
  S->slot_submit.assign(kMaxSlots, Clock::time_point{});
  S->slot_done.assign(kMaxSlots, 0);
  Server *raw = S.release();
  raw->th = std::thread(scheduler, raw);
  *out = raw;
  return TDFS_OK;
}

int server_submit(Server *S, const DevPlan &plan, uint64_t *ticket) {
  if (plan.labeled != (int)S->labeled)
    return fail(TDFS_ERR_ADMISSION, "query mode (labeled=%d) differs from the server's", plan.labeled);
  if (plan.k > S->opt.max_k)
    return fail(TDFS_ERR_ADMISSION, "pattern with %d vertices exceeds the server's stack layout (max_k=%d)", plan.k,
                S->opt.max_k);
  const size_t bytes = query_bytes(plan.k, S->cap, S->shape.warps_per_block);
  if (bytes > S->opt.mem_budget)
    return fail(TDFS_ERR_ADMISSION, "query needs %zu bytes, the server budget is %zu", bytes, S->opt.mem_budget);
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal) return fail(S->fatal, "server stopped: %s", S->fatal_msg.c_str());
  if (S->stopping) return fail(TDFS_ERR_ARG, "server is shutting down");
  const uint64_t t = S->next_ticket++;
  if (S->completed == 0 && S->latencies.empty() && S->first_submit == Clock::time_point{})
    S->first_submit = Clock::now();
  S->pending.push_back(Pending{t, plan, bytes, Clock::now()});
  S->results[t] = Result{};
  *ticket = t;
  S->cv_work.notify_one();
  return TDFS_OK;
}

int server_wait(Server *S, uint64_t ticket, uint64_t *count, double *latency_us) {
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->results.find(ticket);
  if (it == S->results.end()) return fail(TDFS_ERR_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  S->cv_done.wait(lk, [&] { return S->results[ticket].done; });
  Result r = S->results[ticket];
  S->results.erase(ticket);
  if (latency_us) *latency_us = r.latency_us;
  if (r.error == TDFS_ERR_TIMEOUT && !S->fatal)
    return fail(r.error, "query %llu ran out of its work budget (%lld units)", (unsigned long long)ticket,
                (long long)S->opt.launch.work_budget);
  if (r.error) return fail(r.error, "query failed: %s", S->fatal_msg.c_str());
  if (count) *count = r.count;
  if (latency_us) *latency_us = r.latency_us;
  return TDFS_OK;
}

int server_stats(Server *S, tdfs_serve_stats *st) {
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(st, 0, sizeof *st);
  st->completed = S->completed;
  st->aborted = S->aborted;
  st->pending = S->pending.size();
  st->inflight = S->inflight;
  std::vector<double> l = S->latencies;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto q = [&](double f) { return l[std::min(l.size() - 1, (size_t)(f * (l.size() - 1) + 0.5))]; };
    st->p50_us = q(0.50);
    st->p99_us = q(0.99);
    st->max_us = l.back();
    const double span = std::chrono::duration<double>(S->last_done - S->first_submit).count();
    st->queries_per_s = span > 0 ? S->completed / span : 0;
  }
  return TDFS_OK;
}

int server_destroy(Server *S) {
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
    S->cv_work.notify_all();
  }
  if (S->th.joinable()) S->th.join();
  cudaStreamDestroy(S->kstream);
  cudaStreamDestroy(S->cstream);
  cudaFreeHost(S->mirror);
  const int rc = S->fatal;
  delete S;
  return rc;
}

}  // namespace tdfs
