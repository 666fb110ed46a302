// graph.cu -- device-resident data graph: upload and one-time preprocessing.
//
// Replaces GraphPreprocessor::to_gpu (src/graph.h:34-50) and build_src_vtx
// (src/graph.h:195-212).  HBM layout:
//   rowptr  int64[n+1]        as in the file
//   colidx  int32[E + pad]    as in the file; padded by kColPad ints so that
//                             16-byte vector loads at the end stay in bounds
//   src     int32[E]          edge -> source vertex (built on the device)
//   maxnd   int32[n]          max degree over the neighbours of each vertex,
//                             so the level-0 test "some neighbour of c has
//                             degree >= deg(pattern vertex 2)"
//                             (src/gpu_match.cu:541-548) is one load
//   label   uint8[n]          labeled graphs only (labels must be < 255)
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "csr.h"
#include "graph.h"

namespace tdfs {

namespace {

// One warp per vertex: writes the vertex id over its edge range.
__global__ void build_src_kernel(const int64_t *__restrict__ rowptr, int32_t n, int32_t *__restrict__ src) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; v < n; v += warps) {
    const int64_t b = rowptr[v], e = rowptr[v + 1];
    for (int64_t j = b + lane; j < e; j += 32) src[j] = (int32_t)v;
  }
}

// One warp per vertex: max over neighbours w of deg(w).
__global__ void max_nbr_deg_kernel(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                                   int32_t n, int32_t *__restrict__ maxnd) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * blockDim.x / 32;
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / 32; v < n; v += warps) {
    const int64_t b = rowptr[v], e = rowptr[v + 1];
    int32_t m = -1;
    for (int64_t j = b + lane; j < e; j += 32) {
      const int32_t w = colidx[j];
      m = max(m, (int32_t)(rowptr[w + 1] - rowptr[w]));
    }
    m = __reduce_max_sync(0xffffffffu, (unsigned)(m + 1)) - 1;
    if (lane == 0) maxnd[v] = m;
  }
}

__global__ void narrow_labels_kernel(const int32_t *__restrict__ in, int32_t n, uint8_t *__restrict__ out,
                                     int32_t *__restrict__ bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t l = in[i];
    if (l < 0 || l > 254) atomicExch(bad, 1);
    out[i] = (uint8_t)(l < 0 || l > 254 ? 255 : l);
  }
}

// Report a failed CUDA call and clear the runtime's last-error slot, so the
// error cannot resurface in a later launch check.
int cuda_fail(cudaError_t e, const char *what) {
  (void)cudaGetLastError();
  return fail(TDFS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace

// Derived per-graph arrays into caller-provided device memory, no allocation:
// edge -> source, neighbour-degree maxima and (when labels is not null) 8-bit
// labels.  *bad becomes nonzero when a label lies outside [0, 254].
int prepare_graph_arrays(const int64_t *rowptr, const int32_t *colidx, int32_t n, const int32_t *labels,
                         int32_t *src, int32_t *maxnd, uint8_t *label8, int32_t *bad, cudaStream_t st) {
  (void)cudaGetLastError();  // the check below must see these launches' errors only
  if (n > 0) {
    const int threads = 256;
    const int64_t want = ((int64_t)n * 32 + threads - 1) / threads;
    const int blocks = (int)std::min<int64_t>(want, 148 * 16);
    build_src_kernel<<<blocks, threads, 0, st>>>(rowptr, n, src);
    max_nbr_deg_kernel<<<blocks, threads, 0, st>>>(rowptr, colidx, n, maxnd);
    if (labels) narrow_labels_kernel<<<148 * 4, 256, 0, st>>>(labels, n, label8, bad);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? TDFS_OK : cuda_fail(e, "graph preparation kernels");
}

namespace {

// ---- launch workspaces, pooled per device ---------------------------------
std::mutex g_pool_mu;
std::vector<Workspace *> g_pool;        // idle workspaces (any device)
constexpr int kIdlePerDevice = 4;       // idle workspaces kept per device; more are freed

void free_workspace(Workspace *w) {
  cudaFree(w->ctl);
  cudaFreeHost(w->htab);
  if (w->gstream) cudaStreamDestroy(static_cast<cudaStream_t>(w->gstream));
  delete w;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

int acquire_workspace(tdfs_graph *g) {
  if (g->ws) return TDFS_OK;
  Workspace *w = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (size_t i = 0; i < g_pool.size(); ++i)
      if (g_pool[i]->device == g->device) {
        w = g_pool[i];
        g_pool.erase(g_pool.begin() + (long)i);
        break;
      }
  }
  if (!w) {
    // one device allocation (control block, ring, slot table) and one pinned
    // host allocation (staging copies of the slot table and control block)
    const size_t o_queue = align256(sizeof(RunCtl));
    const size_t o_tab = o_queue + align256(sizeof(SplitUnit) * kQueueCap + sizeof(QueueHdr));
    const size_t dev_bytes = o_tab + align256(sizeof(SlotTable));
    const size_t o_hctl = align256(sizeof(SlotTable));
    w = new Workspace{};
    w->device = g->device;
    char *d = nullptr, *h = nullptr;
    cudaError_t e = cudaMalloc(&d, dev_bytes);
    if (e == cudaSuccess) {
      e = cudaMallocHost(&h, o_hctl + sizeof(RunCtl));
      if (e != cudaSuccess) cudaFree(d);
    }
    if (e != cudaSuccess) {
      delete w;
      return cuda_fail(e, "launch workspace");
    }
    w->ctl = reinterpret_cast<RunCtl *>(d);
    w->queue = reinterpret_cast<SplitUnit *>(d + o_queue);
    w->tab = reinterpret_cast<SlotTable *>(d + o_tab);
    w->htab = reinterpret_cast<SlotTable *>(h);
    w->hctl = reinterpret_cast<RunCtl *>(h + o_hctl);
  }
  g->ws = w;
  g->ctl = w->ctl;
  g->queue = w->queue;
  g->tab = w->tab;
  g->htab = w->htab;
  g->hctl = w->hctl;
  return TDFS_OK;
}

namespace {

void release_workspace(tdfs_graph *g) {
  Workspace *w = g->ws;
  if (!w) return;
  g->ws = nullptr;
  g->ctl = nullptr;
  g->queue = nullptr;
  g->tab = nullptr;
  g->htab = nullptr;
  g->hctl = nullptr;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  int idle = 0;
  for (Workspace *x : g_pool) idle += x->device == w->device;
  if (idle < kIdlePerDevice) g_pool.push_back(w);
  else free_workspace(w);
}

}  // namespace

// The graph arrays live in one device allocation:
//   rowptr int64[n+1] | colidx int32[E + kColPad] | src int32[E] | maxnd int32[n] | label uint8[n]
// each part starting on a 256-byte boundary.  Labels are checked and
// narrowed to 8 bits on the host, so the upload is a few stream-ordered
// copies and two preprocessing kernels, synchronised once at the end.
int graph_upload(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx, const int32_t *labels,
                 int device, int32_t max_degree, tdfs_graph **out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(TDFS_ERR_CUDA, "no CUDA device visible (the tdfs engine has no CPU path)");
  if (device < 0 || device >= ndev) return fail(TDFS_ERR_ARG, "device %d out of range", device);
  std::vector<uint8_t> lab8;
  std::unique_ptr<LabelIndex> lindex;
  if (labels) {
    lab8.resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      if (labels[i] < 0 || labels[i] > 254)
        return fail(TDFS_ERR_FORMAT, "vertex labels must lie in [0, 254] for the device label array");
      lab8[(size_t)i] = (uint8_t)labels[i];
    }
    // level-0 label index: a stable counting sort of the edge ids by
    // (label(src), label(dst))
    lindex.reset(new LabelIndex);
    std::vector<int64_t> &off = lindex->off;
    off.assign(65537, 0);
    for (int64_t v = 0; v < n; ++v) {
      const int ls = lab8[(size_t)v] << 8;
      for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j) ++off[(size_t)(ls | lab8[(size_t)colidx[j]]) + 1];
    }
    for (size_t k = 1; k < off.size(); ++k) off[k] += off[k - 1];
    std::vector<int64_t> at(off.begin(), off.end() - 1);
    lindex->perm.resize((size_t)nedges);
    for (int64_t v = 0; v < n; ++v) {
      const int ls = lab8[(size_t)v] << 8;
      for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j)
        lindex->perm[(size_t)at[(size_t)(ls | lab8[(size_t)colidx[j]])]++] = (int32_t)j;
    }
  }
  // label-partitioned rows, for graphs with at most kSegLabels labels: each
  // row re-sorted by (label, id), a stable counting sort per row, with the
  // start of every label's segment relative to the row start.  A labeled
  // plan then scans only the segment of the label it needs.
  int nlab = 0;
  std::vector<int32_t> col_l, loff;
  if (labels) {
    for (int64_t v = 0; v < n; ++v) nlab = std::max(nlab, lab8[(size_t)v] + 1);
    if (nlab > kSegLabels) nlab = 0;
  }
  if (nlab > 0) {
    col_l.resize((size_t)nedges);
    loff.assign((size_t)n * (nlab + 1), 0);
    std::vector<int32_t> cnt(nlab + 1);
    for (int64_t v = 0; v < n; ++v) {
      std::fill(cnt.begin(), cnt.end(), 0);
      for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j) ++cnt[lab8[(size_t)colidx[j]] + 1];
      int32_t *o = loff.data() + (size_t)v * (nlab + 1);
      for (int l = 0; l < nlab; ++l) o[l + 1] = o[l] + cnt[l + 1];
      for (int l = 0; l < nlab; ++l) cnt[l] = o[l];
      for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j)
        col_l[(size_t)(rowptr[v] + cnt[lab8[(size_t)colidx[j]]]++)] = colidx[j];
    }
  }
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  static_assert(kColPad % 4 == 0, "padding keeps 16-byte loads aligned");
  const size_t o_col = align256(sizeof(int64_t) * (size_t)(n + 1));
  const size_t o_src = o_col + align256(sizeof(int32_t) * (size_t)(nedges + kColPad));
  const size_t o_maxnd = o_src + align256(sizeof(int32_t) * (size_t)(nedges ? nedges : 1));
  const size_t o_label = o_maxnd + align256(sizeof(int32_t) * (size_t)(n ? n : 1));
  const size_t o_perm = o_label + align256((size_t)(labels && n ? n : 1));
  const size_t o_coll = o_perm + align256(sizeof(int32_t) * (size_t)(labels && nedges ? nedges : 1));
  const size_t o_loff = o_coll + align256(sizeof(int32_t) * (size_t)(nlab ? nedges + kColPad : 1));
  const size_t total = o_loff + align256(sizeof(int32_t) * (nlab ? loff.size() : 1));
  char *base = nullptr;
  e = cudaMalloc(&base, total);
  if (e != cudaSuccess) return cuda_fail(e, "graph arrays");
  auto *g = new tdfs_graph;
  std::memset(g, 0, sizeof *g);
  g->device = device;
  g->n = n;
  g->nedges = nedges;
  g->max_degree = max_degree;
  g->labeled = labels != nullptr;
  g->arrays = base;
  g->rowptr = reinterpret_cast<int64_t *>(base);
  g->colidx = reinterpret_cast<int32_t *>(base + o_col);
  g->src = reinterpret_cast<int32_t *>(base + o_src);
  g->maxnd = reinterpret_cast<int32_t *>(base + o_maxnd);
  g->label = labels ? reinterpret_cast<uint8_t *>(base + o_label) : nullptr;
  g->lperm = labels ? reinterpret_cast<int32_t *>(base + o_perm) : nullptr;
  g->colidx_l = nlab ? reinterpret_cast<int32_t *>(base + o_coll) : nullptr;
  g->loff = nlab ? reinterpret_cast<int32_t *>(base + o_loff) : nullptr;
  g->nlab = nlab;
  g->bytes = total;
  const cudaStream_t st = cudaStreamPerThread;
  e = cudaMemcpyAsync(g->rowptr, rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nedges)
    e = cudaMemcpyAsync(g->colidx, colidx, sizeof(int32_t) * nedges, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->colidx + nedges, 0x7f, sizeof(int32_t) * kColPad, st);
  if (e == cudaSuccess && labels && n)
    e = cudaMemcpyAsync(g->label, lab8.data(), (size_t)n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && labels && nedges)
    e = cudaMemcpyAsync(g->lperm, lindex->perm.data(), sizeof(int32_t) * nedges, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nlab) {
    if (nedges) e = cudaMemcpyAsync(g->colidx_l, col_l.data(), sizeof(int32_t) * nedges, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(g->colidx_l + nedges, 0x7f, sizeof(int32_t) * kColPad, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(g->loff, loff.data(), sizeof(int32_t) * loff.size(), cudaMemcpyHostToDevice, st);
  }
  int rc = TDFS_OK;
  if (e == cudaSuccess && n > 0) {
    (void)cudaGetLastError();  // the check below must see these launches' errors only
    const int threads = 256;
    const int64_t want = ((int64_t)n * 32 + threads - 1) / threads;
    const int blocks = (int)std::min<int64_t>(want, 148 * 16);
    build_src_kernel<<<blocks, threads, 0, st>>>(g->rowptr, (int32_t)n, g->src);
    max_nbr_deg_kernel<<<blocks, threads, 0, st>>>(g->rowptr, g->colidx, (int32_t)n, g->maxnd);
    e = cudaGetLastError();
  }
  // the host label copy and the caller's arrays must outlive the copies
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) rc = cuda_fail(e, "graph upload");
  if (rc) {
    cudaFree(base);
    delete g;
    return rc;
  }
  g->lindex = lindex.release();
  *out = g;
  return TDFS_OK;
}

void label_range(const LabelIndex &x, int l0, int l1, int64_t eb, int64_t ee, int64_t *b, int64_t *e) {
  *b = *e = 0;
  if (l0 < 0 || l0 > 254 || l1 < 0 || l1 > 254) return;  // a label no vertex has: nothing to do
  const size_t key = (size_t)(l0 << 8 | l1);
  const int32_t *g0 = x.perm.data() + x.off[key], *g1 = x.perm.data() + x.off[key + 1];
  // ids ascend within a group: the edge-id range is a position range
  *b = x.off[key] + (std::lower_bound(g0, g1, (int32_t)std::min<int64_t>(eb, INT32_MAX)) - g0);
  *e = x.off[key] + (std::lower_bound(g0, g1, (int32_t)std::min<int64_t>(ee, INT32_MAX)) - g0);
  if (ee > INT32_MAX) *e = x.off[key + 1];
}

void graph_release(tdfs_graph *g) {
  if (!g) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(g->device);
  release_graphs(g);
  release_workspace(g);
  cudaFree(g->arrays);
  delete g->lindex;
  cudaSetDevice(cur);
  delete g;
}

DevGraph graph_view(const tdfs_graph *g) {
  DevGraph v;
  v.rowptr = g->rowptr;
  v.colidx = g->colidx;
  v.src = g->src;
  v.label = g->label;
  v.maxnd = g->maxnd;
  v.lperm = g->lperm;
  v.colidx_l = g->colidx_l;
  v.loff = g->loff;
  v.nlab = g->nlab;
  v.nedges = g->nedges;
  v.n = (int32_t)g->n;
  v.max_degree = g->max_degree;
  return v;
}

}  // namespace tdfs
