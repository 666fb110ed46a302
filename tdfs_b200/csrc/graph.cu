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
#include <thread>
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

__device__ __forceinline__ unsigned lanes_below() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// ---- label rows and label index on the device (at most kSegLabels labels) --
// Both are stable counting sorts.  Within a warp, the lanes holding the same
// key are found with __match_any_sync; each lane's rank among them (lanes
// below it) plus the counts of the earlier chunks gives its position, so the
// output keeps the input order within every key, as a sequential pass would.

// Edge ids per tile of the label-index sort: small tiles for parallelism
// (one warp walks a tile in order), at most kMaxTiles of them so the
// (key, tile) histogram stays a few MB.
constexpr int64_t kMinTileEdges = 512;
constexpr int64_t kMaxTiles = 8192;
inline int64_t tile_edges(int64_t nedges) {
  const int64_t t = (nedges + kMaxTiles - 1) / kMaxTiles;
  return std::max(kMinTileEdges, (t + 31) & ~int64_t(31));
}
constexpr int kBuildWarps = 8;    // warps per CTA of the build kernels

// One warp per vertex: its row again, stably partitioned by neighbour label
// (col_l), and each label's segment start relative to the row start (loff,
// nl + 1 per vertex, the last one the row length).  Two passes over the row:
// the label counts, then the scatter.
__global__ void label_rows_kernel(const int64_t *__restrict__ rowptr, const int32_t *__restrict__ colidx,
                                  const uint8_t *__restrict__ lab, int32_t n, int nl, int32_t *__restrict__ col_l,
                                  int32_t *__restrict__ loff) {
  __shared__ int32_t cnt_s[kBuildWarps][kSegLabels];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int32_t *cnt = cnt_s[wib];
  const int64_t warps = (int64_t)gridDim.x * kBuildWarps;
  for (int64_t v = (int64_t)blockIdx.x * kBuildWarps + wib; v < n; v += warps) {
    const int64_t b = rowptr[v], e = rowptr[v + 1];
    if (lane < kSegLabels) cnt[lane] = 0;
    __syncwarp();
    for (int64_t c0 = b; c0 < e; c0 += 32) {
      const int64_t j = c0 + lane;
      const bool valid = j < e;
      const int key = valid ? (int)lab[colidx[j]] : -1;
      const unsigned m = __match_any_sync(0xffffffffu, key);
      if (valid && lane == __ffs(m) - 1) cnt[key] += __popc(m);
      __syncwarp();
    }
    const int32_t c = lane < nl ? cnt[lane] : 0;
    int32_t incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    const int32_t excl = incl - c;  // lane nl: the row length
    if (lane <= nl) loff[v * (nl + 1) + lane] = excl;
    __syncwarp();
    if (lane < nl) cnt[lane] = excl;  // scatter cursors
    __syncwarp();
    for (int64_t c0 = b; c0 < e; c0 += 32) {
      const int64_t j = c0 + lane;
      const bool valid = j < e;
      const int32_t w = valid ? colidx[j] : 0;
      const int key = valid ? (int)lab[w] : -1;
      const unsigned m = __match_any_sync(0xffffffffu, key);
      if (valid) col_l[b + cnt[key] + __popc(m & lanes_below())] = w;
      __syncwarp();
      if (valid && lane == __ffs(m) - 1) cnt[key] += __popc(m);
      __syncwarp();
    }
  }
}

// One warp per tile of `tile` consecutive edge ids: the number of the
// tile's edges with each group key nl * label(src) + label(dst), written
// key-major (hist[key * ntiles + tile]) so that one exclusive scan gives every
// (key, tile) its first position in the label index.
__global__ void edge_hist_kernel(const int32_t *__restrict__ src, const int32_t *__restrict__ colidx,
                                 const uint8_t *__restrict__ lab, int64_t nedges, int64_t tile, int nl,
                                 int32_t ntiles, int32_t *__restrict__ hist) {
  __shared__ int32_t cnt_s[kBuildWarps][kSegLabels * kSegLabels];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int32_t *cnt = cnt_s[wib];
  const int G = nl * nl;
  const int64_t warps = (int64_t)gridDim.x * kBuildWarps;
  for (int64_t t = (int64_t)blockIdx.x * kBuildWarps + wib; t < ntiles; t += warps) {
    for (int k = lane; k < G; k += 32) cnt[k] = 0;
    __syncwarp();
    const int64_t b = t * tile, e = b + tile < nedges ? b + tile : nedges;
    for (int64_t c0 = b; c0 < e; c0 += 32) {
      const int64_t j = c0 + lane;
      const bool valid = j < e;
      const int key = valid ? (int)lab[src[j]] * nl + (int)lab[colidx[j]] : -1;
      const unsigned m = __match_any_sync(0xffffffffu, key);
      if (valid && lane == __ffs(m) - 1) cnt[key] += __popc(m);
      __syncwarp();
    }
    for (int k = lane; k < G; k += 32) hist[(int64_t)k * ntiles + t] = cnt[k];
    __syncwarp();
  }
}

// One CTA of 1024 threads: exclusive scan of the histogram in place (each
// thread a contiguous run, then a scan of the run sums in shared memory), and
// the group offsets goff[key] (goff[G] = the edge count).
__global__ void __launch_bounds__(1024) index_scan_kernel(int32_t *__restrict__ a, int64_t N, int G,
                                                          int32_t ntiles, int64_t nedges,
                                                          int64_t *__restrict__ goff) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int64_t per = (N + 1023) / 1024;
  const int64_t b = t * per < N ? t * per : N, e = b + per < N ? b + per : N;
  int64_t s = 0;
  for (int64_t i = b; i < e; ++i) s += a[i];
  part[t] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int64_t v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int64_t run = part[t] - s;
  for (int64_t i = b; i < e; ++i) {
    const int32_t x = a[i];
    a[i] = (int32_t)run;
    run += x;
  }
  __syncthreads();
  for (int k = t; k < G; k += 1024) goff[k] = a[(int64_t)k * ntiles];
  if (t == 0) goff[G] = nedges;
}

// One warp per tile: every edge id to its place in the label index, from the
// scanned (key, tile) starts, in edge-id order within each key.
__global__ void edge_scatter_kernel(const int32_t *__restrict__ src, const int32_t *__restrict__ colidx,
                                    const uint8_t *__restrict__ lab, int64_t nedges, int64_t tile, int nl,
                                    int32_t ntiles, const int32_t *__restrict__ start,
                                    int32_t *__restrict__ perm) {
  __shared__ int32_t cur_s[kBuildWarps][kSegLabels * kSegLabels];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  int32_t *cur = cur_s[wib];
  const int G = nl * nl;
  const int64_t warps = (int64_t)gridDim.x * kBuildWarps;
  for (int64_t t = (int64_t)blockIdx.x * kBuildWarps + wib; t < ntiles; t += warps) {
    for (int k = lane; k < G; k += 32) cur[k] = start[(int64_t)k * ntiles + t];
    __syncwarp();
    const int64_t b = t * tile, e = b + tile < nedges ? b + tile : nedges;
    for (int64_t c0 = b; c0 < e; c0 += 32) {
      const int64_t j = c0 + lane;
      const bool valid = j < e;
      const int key = valid ? (int)lab[src[j]] * nl + (int)lab[colidx[j]] : -1;
      const unsigned m = __match_any_sync(0xffffffffu, key);
      if (valid) perm[cur[key] + __popc(m & lanes_below())] = (int32_t)j;
      __syncwarp();
      if (valid && lane == __ffs(m) - 1) cur[key] += __popc(m);
      __syncwarp();
    }
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
  if (idle < kIdlePerDevice) g_pool.insert(g_pool.end(), 1, w);
  else free_workspace(w);
}

}  // namespace

namespace {

// ---- cached allocations ----------------------------------------------------
// A freed graph's device block and pinned staging block are kept for the next
// upload, so a create/free cycle of a small graph pays no cudaMalloc,
// cudaMallocHost or cudaFree (each costs more than the rest of its upload).
class BlockCache {
 public:
  BlockCache(bool pinned, size_t cap) : pinned_(pinned), cap_(cap) {}

  // A block of at least `need` bytes for `device` (the current device):
  // the smallest idle one within twice that, else a new allocation (after
  // returning this device's idle blocks when memory is short).
  cudaError_t take(int device, size_t need, void **p, size_t *bytes) {
    need = (need + kGrain - 1) & ~(kGrain - 1);
    {
      std::lock_guard<std::mutex> lk(mu_);
      int best = -1;
      for (size_t i = 0; i < idle_.size(); ++i) {
        const Block &b = idle_[i];
        if (b.device == device && b.bytes >= need && b.bytes <= 2 * need &&
            (best < 0 || b.bytes < idle_[(size_t)best].bytes))
          best = (int)i;
      }
      if (best >= 0) {
        *p = idle_[(size_t)best].p;
        *bytes = idle_[(size_t)best].bytes;
        idle_bytes_ -= *bytes;
        idle_.erase(idle_.begin() + best);
        return cudaSuccess;
      }
    }
    cudaError_t e = alloc(p, need);
    if (e == cudaErrorMemoryAllocation) {
      (void)cudaGetLastError();
      drop(device);
      e = alloc(p, need);
    }
    if (e == cudaSuccess) *bytes = need;
    return e;
  }

  // Keep a block for reuse (within the cache's byte cap), else free it.
  void give(int device, void *p, size_t bytes) {
    if (!p) return;
    {
      std::lock_guard<std::mutex> lk(mu_);
      int mine = 0;
      for (const Block &b : idle_) mine += b.device == device;
      if (idle_bytes_ + bytes <= cap_ && mine < kPerDevice) {
        idle_.push_back(Block{device, bytes, p});
        idle_bytes_ += bytes;
        return;
      }
    }
    release(p);
  }

 private:
  struct Block {
    int device;
    size_t bytes;
    void *p;
  };
  static constexpr size_t kGrain = size_t(1) << 20;  // sizes rounded to 1 MiB, so re-uploads fit exactly
  static constexpr int kPerDevice = 4;

  cudaError_t alloc(void **p, size_t bytes) { return pinned_ ? cudaMallocHost(p, bytes) : cudaMalloc(p, bytes); }
  void release(void *p) {
    if (pinned_) cudaFreeHost(p); else cudaFree(p);
  }
  void drop(int device) {
    std::vector<Block> mine;
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t i = 0; i < idle_.size();) {
        if (idle_[i].device == device) {
          idle_bytes_ -= idle_[i].bytes;
          mine.push_back(idle_[i]);
          idle_.erase(idle_.begin() + (long)i);
        } else {
          ++i;
        }
      }
    }
    for (const Block &b : mine) release(b.p);
  }

  std::mutex mu_;
  std::vector<Block> idle_;
  size_t idle_bytes_ = 0;
  const bool pinned_;
  const size_t cap_;
};

// never destroyed: the blocks may outlive the CUDA runtime at process exit
BlockCache &device_blocks() {
  static BlockCache *c = new BlockCache(false, size_t(512) << 20);
  return *c;
}
BlockCache &pinned_blocks() {
  static BlockCache *c = new BlockCache(true, size_t(256) << 20);
  return *c;
}

int host_threads() {
  const unsigned t = std::thread::hardware_concurrency();
  return t ? (int)std::min(t, 32u) : 4;
}

// The label index and the label rows, written by the host straight into the
// pinned staging block they are uploaded from:
//  * perm: a stable counting sort of the edge ids by the group key
//    nl * label(src) + label(dst), with its group offsets `off`;
//  * with nlab > 0 (at most kSegLabels labels, nlab == nl): col_l, every row
//    re-sorted by (label, id), and loff, each row's segment starts relative
//    to the row start (nlab + 1 per vertex).
// Two passes over the edges (count, then scatter).  Large graphs split the
// rows over host threads in contiguous runs of about equal edge counts; each
// run scatters from its own group offsets, so the order stays stable.
void build_label_arrays(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx, const uint8_t *lab,
                        int nl, int nlab, int32_t *perm, int32_t *col_l, int32_t *loff, std::vector<int64_t> &off) {
  const int G = nl * nl;
  const int T = nedges < (int64_t(1) << 20) ? 1 : (int)std::min<int64_t>(host_threads(), nedges >> 19);
  std::vector<int64_t> rb((size_t)T + 1, 0);
  rb[(size_t)T] = n;
  for (int t = 1; t < T; ++t) {
    const int64_t want = nedges * t / T;
    rb[(size_t)t] = std::max(rb[(size_t)t - 1], (int64_t)(std::upper_bound(rowptr, rowptr + n + 1, want) - rowptr) - 1);
  }
  std::vector<int64_t> cnt((size_t)T * G, 0);  // per run and group: edges, then the run's scatter cursor
  auto count_run = [&](int t) {
    int64_t *c = cnt.data() + (size_t)t * G;
    for (int64_t v = rb[(size_t)t]; v < rb[(size_t)t + 1]; ++v) {
      int64_t *cv = c + (size_t)lab[v] * nl;
      if (nlab) {
        int32_t k[kSegLabels] = {0};
        for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j) ++k[lab[colidx[j]]];
        int32_t *o = loff + (size_t)v * (nlab + 1);
        o[0] = 0;
        for (int l = 0; l < nlab; ++l) {
          o[l + 1] = o[l] + k[l];
          cv[l] += k[l];
        }
      } else {
        for (int64_t j = rowptr[v]; j < rowptr[v + 1]; ++j) ++cv[lab[colidx[j]]];
      }
    }
  };
  auto scatter_run = [&](int t) {
    int64_t *at = cnt.data() + (size_t)t * G;
    for (int64_t v = rb[(size_t)t]; v < rb[(size_t)t + 1]; ++v) {
      int64_t *av = at + (size_t)lab[v] * nl;
      const int64_t b = rowptr[v], e = rowptr[v + 1];
      if (nlab) {
        int32_t k[kSegLabels];
        const int32_t *o = loff + (size_t)v * (nlab + 1);
        for (int l = 0; l < nlab; ++l) k[l] = o[l];
        for (int64_t j = b; j < e; ++j) {
          const int32_t x = colidx[j];
          const int l = lab[x];
          perm[av[l]++] = (int32_t)j;
          col_l[b + k[l]++] = x;
        }
      } else {
        for (int64_t j = b; j < e; ++j) perm[av[lab[colidx[j]]]++] = (int32_t)j;
      }
    }
  };
  auto run = [&](auto &&f) {
    if (T == 1) {
      f(0);
      return;
    }
    std::vector<std::thread> th;
    for (int t = 0; t < T; ++t) th.emplace_back(f, t);
    for (auto &x : th) x.join();
  };
  run(count_run);
  off.assign((size_t)G + 1, 0);
  for (int gk = 0; gk < G; ++gk) {
    int64_t s = off[(size_t)gk];
    for (int t = 0; t < T; ++t) {  // run t scatters group gk from here
      const int64_t c = cnt[(size_t)t * G + gk];
      cnt[(size_t)t * G + gk] = s;
      s += c;
    }
    off[(size_t)gk + 1] = s;
  }
  run(scatter_run);
}

}  // namespace

// The graph arrays live in one device allocation, each part starting on a
// 256-byte boundary:
//   rowptr int64[n+1] | colidx int32[E + kColPad] | src int32[E] | maxnd int32[n]
//   | label uint8[n] | lperm int32[E] | colidx_l int32[E + kColPad] | loff int32[n (nlab+1)]
// The parts from `label` on are derived on the host into one pinned staging
// block laid out the same way and uploaded with one copy.  The CSR copies and
// the two preprocessing kernels are queued first, so the device works while
// the host sorts; one synchronisation at the end.
int graph_upload(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx, const int32_t *labels,
                 int device, int32_t max_degree, tdfs_graph **out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(TDFS_ERR_CUDA, "no CUDA device visible (the tdfs engine has no CPU path)");
  if (device < 0 || device >= ndev) return fail(TDFS_ERR_ARG, "device %d out of range", device);
  int nl = 0;
  if (labels) {
    for (int64_t i = 0; i < n; ++i) {
      if (labels[i] < 0 || labels[i] > 254)
        return fail(TDFS_ERR_FORMAT, "vertex labels must lie in [0, 254] for the device label array");
      nl = std::max(nl, labels[i] + 1);
    }
    if (nedges > INT32_MAX) return fail(TDFS_ERR_CAPACITY, "labeled graphs hold at most 2^31 - 1 directed edges");
  }
  // label-partitioned rows for graphs with at most kSegLabels labels
  const int nlab = labels && nl <= kSegLabels ? nl : 0;
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
  const size_t nloff = nlab ? (size_t)n * (size_t)(nlab + 1) : 0;
  // with label rows the label arrays are built on the device, which needs
  // scratch for the index sort: the (key, tile) histogram and the group
  // offsets; otherwise the host builds them into the staging block
  const bool dev_build = nlab > 0;
  const int G = nl * nl;
  const int64_t tile = tile_edges(nedges);
  const int32_t ntiles = dev_build ? (int32_t)((nedges + tile - 1) / tile) : 0;
  const size_t o_hist = o_loff + align256(sizeof(int32_t) * (nloff ? nloff : 1));
  const size_t o_goff = o_hist + align256(sizeof(int32_t) * (size_t)(dev_build && ntiles ? (int64_t)G * ntiles : 1));
  const size_t total = dev_build ? o_goff + align256(sizeof(int64_t) * (size_t)(G + 1)) : o_hist;
  void *arrays = nullptr, *stage = nullptr;
  size_t array_bytes = 0, stage_bytes = 0;
  e = device_blocks().take(device, total, &arrays, &array_bytes);
  if (e != cudaSuccess) return cuda_fail(e, "graph arrays");
  if (labels) {
    e = pinned_blocks().take(device, dev_build ? (size_t)std::max<int64_t>(n, 1) : total - o_label, &stage,
                             &stage_bytes);
    if (e != cudaSuccess) {
      device_blocks().give(device, arrays, array_bytes);
      return cuda_fail(e, "pinned staging for the label arrays");
    }
  }
  char *base = static_cast<char *>(arrays);
  auto *g = new tdfs_graph;
  std::memset(g, 0, sizeof *g);
  g->device = device;
  g->n = n;
  g->nedges = nedges;
  g->max_degree = max_degree;
  g->labeled = labels != nullptr;
  g->arrays = arrays;
  g->array_bytes = array_bytes;
  g->staging = stage;
  g->staging_bytes = stage_bytes;
  g->rowptr = reinterpret_cast<int64_t *>(base);
  g->colidx = reinterpret_cast<int32_t *>(base + o_col);
  g->src = reinterpret_cast<int32_t *>(base + o_src);
  g->maxnd = reinterpret_cast<int32_t *>(base + o_maxnd);
  g->label = labels ? reinterpret_cast<uint8_t *>(base + o_label) : nullptr;
  g->lperm = labels ? reinterpret_cast<int32_t *>(base + o_perm) : nullptr;
  g->colidx_l = nlab ? reinterpret_cast<int32_t *>(base + o_coll) : nullptr;
  g->loff = nlab ? reinterpret_cast<int32_t *>(base + o_loff) : nullptr;
  g->nlab = nlab;
  g->bytes = dev_build ? o_hist : total;  // the scratch is not part of the graph
  const cudaStream_t st = cudaStreamPerThread;
  e = cudaMemcpyAsync(g->rowptr, rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nedges)
    e = cudaMemcpyAsync(g->colidx, colidx, sizeof(int32_t) * nedges, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(g->colidx + nedges, 0x7f, sizeof(int32_t) * kColPad, st);
  if (e == cudaSuccess && n > 0) {
    (void)cudaGetLastError();  // the check below must see these launches' errors only
    const int threads = 256;
    const int64_t want = ((int64_t)n * 32 + threads - 1) / threads;
    const int blocks = (int)std::min<int64_t>(want, 148 * 16);
    build_src_kernel<<<blocks, threads, 0, st>>>(g->rowptr, (int32_t)n, g->src);
    max_nbr_deg_kernel<<<blocks, threads, 0, st>>>(g->rowptr, g->colidx, (int32_t)n, g->maxnd);
    e = cudaGetLastError();
  }
  std::unique_ptr<LabelIndex> lindex;
  if (e == cudaSuccess && labels) {
    char *h = static_cast<char *>(stage);
    auto *lab8 = reinterpret_cast<uint8_t *>(h);
    for (int64_t i = 0; i < n; ++i) lab8[i] = (uint8_t)labels[i];
    lindex.reset(new LabelIndex);
    lindex->nl = nl;
    lindex->nedges = nedges;
    if (dev_build) {
      // label rows and label index by the kernels above, after the CSR's
      // preprocessing in stream order; the host keeps the group offsets
      lindex->dev_perm = g->lperm;
      lindex->off.assign((size_t)G + 1, 0);
      e = cudaMemcpyAsync(g->label, lab8, (size_t)n, cudaMemcpyHostToDevice, st);
      if (e == cudaSuccess) e = cudaMemsetAsync(g->colidx_l + nedges, 0x7f, sizeof(int32_t) * kColPad, st);
      if (e == cudaSuccess && n > 0) {
        const int blocks = (int)std::min<int64_t>((n + kBuildWarps - 1) / kBuildWarps, 148 * 16);
        label_rows_kernel<<<blocks, 32 * kBuildWarps, 0, st>>>(g->rowptr, g->colidx, g->label, (int32_t)n, nl,
                                                              g->colidx_l, g->loff);
        e = cudaGetLastError();
      }
      if (e == cudaSuccess && ntiles > 0) {
        auto *hist = reinterpret_cast<int32_t *>(base + o_hist);
        auto *goff = reinterpret_cast<int64_t *>(base + o_goff);
        const int blocks = (int)std::min<int64_t>((ntiles + kBuildWarps - 1) / kBuildWarps, 148 * 16);
        edge_hist_kernel<<<blocks, 32 * kBuildWarps, 0, st>>>(g->src, g->colidx, g->label, nedges, tile, nl,
                                                             ntiles, hist);
        index_scan_kernel<<<1, 1024, 0, st>>>(hist, (int64_t)G * ntiles, G, ntiles, nedges, goff);
        edge_scatter_kernel<<<blocks, 32 * kBuildWarps, 0, st>>>(g->src, g->colidx, g->label, nedges, tile, nl,
                                                                ntiles, hist, g->lperm);
        e = cudaGetLastError();
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(lindex->off.data(), goff, sizeof(int64_t) * (size_t)(G + 1), cudaMemcpyDeviceToHost,
                              st);
      }
    } else {
      // while the device copies and preprocesses the CSR
      auto *perm = reinterpret_cast<int32_t *>(h + (o_perm - o_label));
      auto *col_l = reinterpret_cast<int32_t *>(h + (o_coll - o_label));
      auto *loff = reinterpret_cast<int32_t *>(h + (o_loff - o_label));
      lindex->perm = perm;
      build_label_arrays(n, nedges, rowptr, colidx, lab8, nl, nlab, perm, col_l, loff, lindex->off);
      if (nlab) std::memset(col_l + nedges, 0x7f, sizeof(int32_t) * kColPad);
      e = cudaMemcpyAsync(base + o_label, h, total - o_label, cudaMemcpyHostToDevice, st);
    }
  }
  // the staging block and the caller's arrays must outlive the copies
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    const int rc = cuda_fail(e, "graph upload");
    cudaStreamSynchronize(st);
    pinned_blocks().give(device, stage, stage_bytes);
    device_blocks().give(device, arrays, array_bytes);
    delete g;
    return rc;
  }
  g->lindex = lindex.release();
  *out = g;
  return TDFS_OK;
}

bool label_range(LabelIndex &x, int l0, int l1, int64_t eb, int64_t ee, int64_t *b, int64_t *e) {
  *b = *e = 0;
  if (l0 < 0 || l0 >= x.nl || l1 < 0 || l1 >= x.nl) return true;  // a label no vertex has: nothing to do
  const size_t key = (size_t)l0 * (size_t)x.nl + (size_t)l1;
  if (eb <= 0 && ee >= x.nedges) {
    *b = x.off[key];
    *e = x.off[key + 1];
    return true;
  }
  std::call_once(x.fetch_once, [&x] {
    if (x.perm || !x.dev_perm) return;
    x.fetched.resize((size_t)x.nedges);
    if (cudaMemcpy(x.fetched.data(), x.dev_perm, sizeof(int32_t) * (size_t)x.nedges, cudaMemcpyDeviceToHost) ==
        cudaSuccess)
      x.perm = x.fetched.data();
    else
      (void)cudaGetLastError();
  });
  if (!x.perm) return false;
  const int32_t *g0 = x.perm + x.off[key], *g1 = x.perm + x.off[key + 1];
  // ids ascend within a group: the edge-id range is a position range
  *b = x.off[key] + (std::lower_bound(g0, g1, (int32_t)std::min<int64_t>(eb, INT32_MAX)) - g0);
  *e = x.off[key] + (std::lower_bound(g0, g1, (int32_t)std::min<int64_t>(ee, INT32_MAX)) - g0);
  if (ee > INT32_MAX) *e = x.off[key + 1];
  return true;
}

void graph_release(tdfs_graph *g) {
  if (!g) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(g->device);
  release_graphs(g);
  release_workspace(g);
  // the blocks go back to the caches, not to the driver: wait for anything
  // still reading them, as cudaFree would
  cudaDeviceSynchronize();
  device_blocks().give(g->device, g->arrays, g->array_bytes);
  pinned_blocks().give(g->device, g->staging, g->staging_bytes);
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
