// static_count.cu -- counting without any device allocation.
//
// Some callers cannot call cudaMalloc: a host process whose device memory is
// carved up by another runtime (an inference server's caching allocator, a
// plugin loaded into an application that owns every byte of the GPU).  For them,
// tdfs_count_static runs the same match kernel as tdfs_count with all of its
// working memory taken from one fixed array that lives in the library's
// device image: kScratchBytes per GPU, held from the first use of the library
// on that GPU until the process exits.
//
// The caller passes the inputs (the CSR of the data graph in device memory,
// optionally its vertex labels, the compiled pattern) and receives the
// output (the count).  The CSR is not checked: it must follow the rules that
// tdfs_graph_from_csr enforces (rowptr spans [0, E], rows strictly
// increasing, ids in [0, n), labels in [0, 254]; labels are checked).  Everything else -- the control block, the split ring,
// the query slot, the edge-to-source map, the neighbour-degree maxima and the
// 8-bit labels -- is carved out of the scratch array, so the graph may have
// at most as many vertices and edges as fit in what is left after the fixed
// parts; larger graphs are rejected with TDFS_ERR_CAPACITY.
//
// All calls share the one array and leave their contents in it: the parts
// that must start at zero are cleared at the start of every call.  Two calls
// whose work overlaps on the GPU (different streams or host threads) race on
// the array; callers must serialise them.
//
// colidx must start on a 16-byte boundary: the kernel stages adjacency
// windows with 16-byte vector loads at offsets rounded down to 4 ints, and a
// misaligned base would fault.  Such a pointer (a sub-allocation, a slice
// like colidx + 1) is rejected with TDFS_ERR_ARG before any GPU work.  The
// same loads round the end of a window up to 4 ints, so when E is not a
// multiple of 4 they could read up to 3 ints past colidx[E-1], outside the
// caller's buffer; for those graphs the staged windows are turned off (the
// kernel searches the lists directly; the count is the same).
//
// The first call on each device looks up the array's device address
// (cudaGetSymbolAddress, with that device current).  The call copies its
// query record from host stack memory and waits for the kernel, so it cannot
// be recorded into a CUDA graph: a call on a stream that is being captured
// is rejected with TDFS_ERR_ARG.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "graph.h"
#include "match.cuh"
#include "plan.h"
#include "serve.h"

namespace tdfs {

namespace {

constexpr size_t kScratchBytes = size_t(48) << 20;  // 48 MiB per GPU
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char *g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mu;

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Report a failed CUDA call (what: "<call>: %s") and clear the runtime's
// last-error slot, so the error cannot resurface in a later launch check.
int cuda_fail_static(const char *what, cudaError_t e) {
  (void)cudaGetLastError();
  return fail(TDFS_ERR_CUDA, what, cudaGetErrorString(e));
}

// Fixed layout of the array (offsets in bytes).
struct Layout {
  size_t ctl, bad, units, qhdr, tab, src, maxnd, label, end;
};

Layout layout(int64_t n, int64_t nedges) {
  Layout L;
  size_t o = 0;
  L.ctl = o;   o = align_up(o + sizeof(RunCtl));
  L.bad = o;   o = align_up(o + sizeof(int32_t));
  L.units = o; o = align_up(o + sizeof(SplitUnit) * kQueueCap);
  L.qhdr = o;  o = align_up(o + sizeof(QueueHdr));
  L.tab = o;   o = align_up(o + sizeof(SlotTable));
  L.src = o;   o = align_up(o + sizeof(int32_t) * (size_t)(nedges > 0 ? nedges : 1));
  L.maxnd = o; o = align_up(o + sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  L.label = o; o = align_up(o + (size_t)(n > 0 ? n : 1));
  L.end = o;
  return L;
}

}  // namespace
}  // namespace tdfs

using namespace tdfs;

extern "C" int tdfs_count_static(int device, int64_t n, int64_t nedges, const int64_t *d_rowptr,
                                 const int32_t *d_colidx, const int32_t *d_labels, const tdfs_plan *p,
                                 const tdfs_options *opt, uint64_t *count) {
  if (!d_rowptr || (!d_colidx && nedges) || !p || !count) return fail(TDFS_ERR_ARG, "null argument");
  if (device < 0 || device >= kMaxDevices) return fail(TDFS_ERR_ARG, "device %d out of range", device);
  if (n < 0 || n > INT32_MAX - 1 || nedges < 0) return fail(TDFS_ERR_ARG, "bad graph size");
  if (reinterpret_cast<uintptr_t>(d_colidx) & 15)
    return fail(TDFS_ERR_ARG, "colidx must be 16-byte aligned (the kernel reads it with 16-byte vector loads)");
  const DevPlan &plan = plan_device_table(p);
  if (plan.labeled && !d_labels) return fail(TDFS_ERR_ARG, "labeled pattern without vertex labels");
  const Layout L = layout(n, nedges);
  if (L.end > kScratchBytes)
    return fail(TDFS_ERR_CAPACITY,
                "graph needs %zu bytes of scratch (n=%lld, E=%lld); the fixed array holds %zu bytes", L.end,
                (long long)n, (long long)nedges, kScratchBytes);
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail_static("cudaSetDevice: %s", e);
  unsigned char *base;
  {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[device]) {
      void *addr = nullptr;
      e = cudaGetSymbolAddress(&addr, g_scratch);
      if (e != cudaSuccess) return cuda_fail_static("cudaGetSymbolAddress: %s", e);
      g_scratch_addr[device] = static_cast<unsigned char *>(addr);
    }
    base = g_scratch_addr[device];
  }
  tdfs_options o;
  if (opt) o = *opt; else tdfs_options_default(&o);
  cudaStream_t st = static_cast<cudaStream_t>(o.stream);
  {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return cuda_fail_static("cudaStreamIsCapturing: %s", e);
    if (cs != cudaStreamCaptureStatusNone)
      return fail(TDFS_ERR_ARG, "tdfs_count_static cannot be called on a stream that is being captured");
  }
  // 16-byte window loads may round the last list's end up to 4 ints: without
  // that slack after colidx[E-1], search the lists directly instead
  if (nedges % 4 != 0) o.merge_window = -1;
  RunCtl *ctl = reinterpret_cast<RunCtl *>(base + L.ctl);
  SplitUnit *units = reinterpret_cast<SplitUnit *>(base + L.units);
  QueueHdr *qh = reinterpret_cast<QueueHdr *>(base + L.qhdr);
  SlotTable *tab = reinterpret_cast<SlotTable *>(base + L.tab);
  int32_t *src = reinterpret_cast<int32_t *>(base + L.src);
  int32_t *maxnd = reinterpret_cast<int32_t *>(base + L.maxnd);
  uint8_t *label8 = plan.labeled ? reinterpret_cast<uint8_t *>(base + L.label) : nullptr;
  // derived graph arrays, written into the scratch (each call recomputes them)
  int32_t *bad = reinterpret_cast<int32_t *>(base + L.bad);
  e = cudaMemsetAsync(bad, 0, sizeof(int32_t), st);
  if (e != cudaSuccess) return cuda_fail_static("scratch clear: %s", e);
  int rc = prepare_graph_arrays(d_rowptr, d_colidx, (int32_t)n, plan.labeled ? d_labels : nullptr, src, maxnd,
                                label8, bad, st);
  if (rc) return rc;
  DevGraph g;
  g.rowptr = d_rowptr;
  g.colidx = d_colidx;
  g.src = src;
  g.label = label8;
  g.maxnd = maxnd;
  g.lperm = nullptr;  // no label index here: labeled slots walk the edge ids
  g.colidx_l = nullptr;  // nor label-partitioned rows: labeled plans test labels per candidate
  g.loff = nullptr;
  g.nlab = 0;
  g.nedges = nedges;
  g.n = (int32_t)n;
  g.max_degree = 0;
  LaunchShape s;
  tdfs_graph probe;  // launch_shape reads only the device index
  std::memset(&probe, 0, sizeof probe);
  probe.device = device;
  rc = launch_shape(&probe, plan.k, plan.labeled != 0, o, &s);
  if (rc) return rc;
  // one query slot over the option's edge range, dealt like tdfs_count deals it
  // (host staging is on the stack: pageable, nothing is allocated)
  const int64_t eb = std::max<int64_t>(0, o.edge_begin);
  const int64_t ee = std::max(eb, (o.edge_end < 0 || o.edge_end > nedges) ? nedges : o.edge_end);
  const int stride = o.edge_stride > 0 ? o.edge_stride : 1;
  if (o.edge_phase < 0 || o.edge_phase >= stride) return fail(TDFS_ERR_ARG, "edge_phase must lie in [0, edge_stride)");
  SlotCtl h_ctl;
  SlotHot h_hot;
  SlotInfo h_info;
  RunCtl h_run;
  std::memset(&h_ctl, 0, sizeof h_ctl);
  h_ctl.admitted = 1;
  h_ctl.shutdown = 1;
  std::memset(&h_hot, 0, sizeof h_hot);
  std::memset(&h_info, 0, sizeof h_info);
  std::memset(&h_run, 0, sizeof h_run);
  h_info.e_begin = eb;
  h_info.e_end = ee;
  h_info.stride = stride;
  h_info.phase = o.edge_phase;
  h_info.chunk = auto_chunk(ee - eb, stride, s.blocks * s.warps_per_block, o.edge_chunk);
  const int64_t chunks = (ee - eb + h_info.chunk - 1) / h_info.chunk;
  h_info.ntickets = chunks <= o.edge_phase ? 0 : (chunks - o.edge_phase + stride - 1) / stride;
  h_hot.state = h_info.ntickets > 0 ? kSlotActive : kSlotDone;
  if (h_info.ntickets == 0) h_ctl.completed = 1;
  e = cudaMemcpyAsync(&tab->ctl, &h_ctl, sizeof h_ctl, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&tab->hot[0], &h_hot, sizeof h_hot, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&tab->info[0], &h_info, sizeof h_info, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&tab->plan[0], &plan, sizeof plan, cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return cuda_fail_static("slot upload: %s", e);
  init_launch(ctl, qh, st);  // clears the control block and the split ring
  rc = launch_match(plan.labeled != 0, g, ctl, tab, units, qh, s.cfg, s.blocks, s.warps_per_block, st);
  if (rc) return rc;
  int32_t h_bad = 0;
  e = cudaMemcpyAsync(&h_hot, &tab->hot[0], sizeof h_hot, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_bad, bad, sizeof h_bad, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_run, ctl, sizeof h_run, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail_static("match kernel: %s", e);
  if (h_bad) return fail(TDFS_ERR_FORMAT, "vertex labels must lie in [0, 254]");
  if (h_run.error) return fail(h_run.error, "device error %d", h_run.error);
  if (h_hot.state != kSlotDone) return fail(TDFS_ERR_TIMEOUT, "the query did not complete");
  *count = (uint64_t)(h_hot.count * (unsigned long long)plan.multiplicity);
  return TDFS_OK;
}
