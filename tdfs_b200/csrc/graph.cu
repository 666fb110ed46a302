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

#include <cstring>
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

int cuda_fail(cudaError_t e, const char *what) {
  return fail(TDFS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace

// Derived per-graph arrays into caller-provided device memory, no allocation:
// edge -> source, neighbour-degree maxima and (when labels is not null) 8-bit
// labels.  *bad becomes nonzero when a label lies outside [0, 254].
int prepare_graph_arrays(const int64_t *rowptr, const int32_t *colidx, int32_t n, const int32_t *labels,
                         int32_t *src, int32_t *maxnd, uint8_t *label8, int32_t *bad, cudaStream_t st) {
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

#define CK(x)                                    \
  do {                                           \
    cudaError_t e_ = (x);                        \
    if (e_ != cudaSuccess) {                     \
      release(g);                                \
      delete g;                                  \
      return cuda_fail(e_, #x);                  \
    }                                            \
  } while (0)

void release(tdfs_graph *g) {
  if (!g) return;
  cudaFree(g->rowptr);
  cudaFree(g->colidx);
  cudaFree(g->src);
  cudaFree(g->maxnd);
  cudaFree(g->label);
  cudaFree(g->ctl);
  cudaFree(g->queue);
  cudaFree(g->tab);
  if (g->htab) cudaFreeHost(g->htab);
  if (g->hctl) cudaFreeHost(g->hctl);
  g->hctl = nullptr;
  g->tab = nullptr;
  g->htab = nullptr;
  g->rowptr = nullptr;
  g->colidx = nullptr;
  g->src = nullptr;
  g->maxnd = nullptr;
  g->label = nullptr;
  g->ctl = nullptr;
  g->queue = nullptr;
}

int graph_upload(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx, const int32_t *labels,
                 int device, int32_t max_degree, tdfs_graph **out) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(TDFS_ERR_CUDA, "no CUDA device visible (the tdfs engine has no CPU path)");
  if (device < 0 || device >= ndev) return fail(TDFS_ERR_ARG, "device %d out of range", device);
  auto *g = new tdfs_graph;
  std::memset(g, 0, sizeof *g);
  g->device = device;
  g->n = n;
  g->nedges = nedges;
  g->max_degree = max_degree;
  g->labeled = labels != nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    delete g;
    return cuda_fail(e, "cudaSetDevice");
  }
  static_assert(kColPad % 4 == 0, "padding keeps 16-byte loads aligned");
  CK(cudaMalloc(&g->rowptr, sizeof(int64_t) * (n + 1)));
  CK(cudaMalloc(&g->colidx, sizeof(int32_t) * (nedges + kColPad)));
  CK(cudaMalloc(&g->src, sizeof(int32_t) * (nedges ? nedges : 1)));
  CK(cudaMalloc(&g->maxnd, sizeof(int32_t) * (n ? n : 1)));
  CK(cudaMalloc(&g->ctl, sizeof(RunCtl)));
  CK(cudaMalloc(&g->queue, sizeof(SplitUnit) * kQueueCap + sizeof(QueueHdr)));
  CK(cudaMalloc(&g->tab, sizeof(SlotTable)));
  CK(cudaMallocHost(&g->htab, sizeof(SlotTable)));
  CK(cudaMallocHost(&g->hctl, sizeof(RunCtl)));
  CK(cudaMemcpy(g->rowptr, rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(g->colidx, colidx, sizeof(int32_t) * nedges, cudaMemcpyHostToDevice));
  CK(cudaMemset(g->colidx + nedges, 0x7f, sizeof(int32_t) * kColPad));
  g->bytes = sizeof(int64_t) * (n + 1) + sizeof(int32_t) * (2 * nedges + kColPad + n);
  if (n > 0) {
    const int threads = 256;
    const int64_t want = ((int64_t)n * 32 + threads - 1) / threads;
    const int blocks = (int)std::min<int64_t>(want, 148 * 16);
    build_src_kernel<<<blocks, threads>>>(g->rowptr, (int32_t)n, g->src);
    max_nbr_deg_kernel<<<blocks, threads>>>(g->rowptr, g->colidx, (int32_t)n, g->maxnd);
    CK(cudaGetLastError());
  }
  if (labels) {
    int32_t *tmp = nullptr, *bad = nullptr;
    CK(cudaMalloc(&g->label, n ? n : 1));
    CK(cudaMalloc(&tmp, sizeof(int32_t) * (n + 1)));
    bad = tmp + n;
    CK(cudaMemcpy(tmp, labels, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
    CK(cudaMemset(bad, 0, sizeof(int32_t)));
    if (n > 0) narrow_labels_kernel<<<148 * 4, 256>>>(tmp, (int32_t)n, g->label, bad);
    int32_t hbad = 0;
    CK(cudaMemcpy(&hbad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost));
    cudaFree(tmp);
    if (hbad) {
      release(g);
      delete g;
      return fail(TDFS_ERR_FORMAT, "vertex labels must lie in [0, 254] for the device label array");
    }
    g->bytes += n;
  }
  CK(cudaDeviceSynchronize());
  *out = g;
  return TDFS_OK;
}

void graph_release(tdfs_graph *g) {
  if (!g) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(g->device);
  release_graphs(g);
  if (g->gstream) cudaStreamDestroy(static_cast<cudaStream_t>(g->gstream));
  g->gstream = nullptr;
  release(g);
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
  v.nedges = g->nedges;
  v.n = (int32_t)g->n;
  v.max_degree = g->max_degree;
  return v;
}

}  // namespace tdfs
