// refshard.cu -- TEST INFRASTRUCTURE: runs the reference's own kernel
// (_parallel_match, src/gpu_match.cu compiled unchanged) over contiguous
// level-0 edge ranges, so the reference can be timed on the same bounded
// slices of a workload as this repository's engine.
//
//   refshard_{ulb,lb} <graph prefix> <pattern.g> [-w K] [-f] <begin> <end> [<begin> <end> ...]
//
// With -w K the first K ranges are warm-up launches in the same process
// (module loading and first-touch costs land there) and are neither timed
// nor counted.  With -f a 256 MB buffer is written before every launch,
// outside the timed event pair, so each timed launch starts with an L2
// that holds none of the graph (B200's L2 is 126 MB).
//
// Set-up follows the reference driver (cu_test.cu:14-78): the reference's
// GraphPreprocessor / PatternPreprocessor / build_src_vtx / to_gpu, per-warp
// call stacks of MAX_SLOT_NUM x GRAPH_DEGREE ints, the timeout queue, and the
// <<<GRID_DIM, BLOCK_DIM>>> launch timed by a cudaEvent pair (cu_test.cu:81-97).
// Per range, the device Graph's nedges is set to `end` and the job queue's
// cursor to `begin`: the kernel reads nedges only as the end of its edge
// scan (src/gpu_match.cu:524-530) and the job queue only through `cur`.  The
// per-warp counts are summed after every launch and the total is multiplied
// by |Aut| when unlabeled (cu_test.cu:100-105).
//
// Prints "<pattern>\t<sum of kernel ms>\t<count>" like cu_test.cu:107.
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "src/gpu_match.cuh"

using namespace STMatch;

#define CK(x)                                                                      \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); \
      return 1;                                                                    \
    }                                                                              \
  } while (0)

static const int kQueueCapTriples = 1000000;  // TIMEOUT_QUEUE_CAP, cu_test.cu:8

int main(int argc, char **argv) {
  int first = 3, warm = 0;
  bool flush = false;
  while (first < argc && argv[first][0] == '-') {
    if (std::strcmp(argv[first], "-w") == 0 && first + 1 < argc) {
      warm = std::atoi(argv[first + 1]);
      first += 2;
    } else if (std::strcmp(argv[first], "-f") == 0) {
      flush = true;
      first += 1;
    } else {
      break;
    }
  }
  if (argc < first + 2 || (argc - first) % 2 || warm < 0) {
    fprintf(stderr, "usage: %s <prefix> <pattern.g> [-w K] [-f] <begin> <end> [<begin> <end> ...]\n", argv[0]);
    return 2;
  }
  CK(cudaSetDevice(0));
  GraphPreprocessor g(argv[1]);
  PatternPreprocessor p(argv[2]);
  g.build_src_vtx(p);
  Graph *gpu_graph = g.to_gpu();
  Pattern *gpu_pattern = p.to_gpu();

  JobQueue jq;
  std::memset(&jq, 0, sizeof jq);
  JobQueue *gpu_queue = nullptr;
  CK(cudaMalloc(&gpu_queue, sizeof(JobQueue)));

  graph_node_t *slot_storage = nullptr;
  CK(cudaMalloc(&slot_storage, sizeof(graph_node_t) * NWARPS_TOTAL * MAX_SLOT_NUM * GRAPH_DEGREE));
  std::vector<CallStack> stk(NWARPS_TOTAL);
  for (int i = 0; i < NWARPS_TOTAL; i++) {
    std::memset(stk[i].iter, 0, sizeof(stk[i].iter));
    std::memset(stk[i].slot_size, 0, sizeof(stk[i].slot_size));
    stk[i].slot_storage =
        (graph_node_t(*)[GRAPH_DEGREE])((char *)slot_storage + (size_t)i * sizeof(graph_node_t) * MAX_SLOT_NUM * GRAPH_DEGREE);
  }
  CallStack *gpu_callstack = nullptr;
  CK(cudaMalloc(&gpu_callstack, NWARPS_TOTAL * sizeof(CallStack)));
  CK(cudaMemcpy(gpu_callstack, stk.data(), sizeof(CallStack) * NWARPS_TOTAL, cudaMemcpyHostToDevice));

  size_t *gpu_res = nullptr;
  CK(cudaMalloc(&gpu_res, sizeof(size_t) * NWARPS_TOTAL));
  std::vector<size_t> res(NWARPS_TOTAL);
  int *idle_warps, *idle_warps_count, *global_mutex;
  CK(cudaMalloc(&idle_warps, sizeof(int) * GRID_DIM));
  CK(cudaMemset(idle_warps, 0, sizeof(int) * GRID_DIM));
  CK(cudaMalloc(&idle_warps_count, sizeof(int)));
  CK(cudaMemset(idle_warps_count, 0, sizeof(int)));
  CK(cudaMalloc(&global_mutex, sizeof(int) * GRID_DIM));
  CK(cudaMemset(global_mutex, 0, sizeof(int) * GRID_DIM));
  int *queue_space = nullptr;
  CK(cudaMalloc(&queue_space, sizeof(int) * kQueueCapTriples * (STOP_LEVEL + 1)));
  Queue *tq = nullptr;
  CK(cudaMallocManaged(&tq, sizeof(Queue)));
  tq->queue_ = queue_space;
  tq->size_ = kQueueCapTriples * (STOP_LEVEL + 1);
  tq->resetQueue();

  void *l2flush = nullptr;
  const size_t kFlushBytes = size_t(256) << 20;
  if (flush) CK(cudaMalloc(&l2flush, kFlushBytes));
  cudaEvent_t start, stop;
  CK(cudaEventCreate(&start));
  CK(cudaEventCreate(&stop));
  unsigned long long total = 0;
  double total_ms = 0;
  for (int a = first, r = 0; a + 1 < argc; a += 2, ++r) {
    const long begin = std::atol(argv[a]), end = std::atol(argv[a + 1]);
    if (begin < 0 || end < begin || end > g.g.nedges) {
      fprintf(stderr, "bad range %ld %ld\n", begin, end);
      return 2;
    }
    jq.cur = (unsigned long long)begin;
    CK(cudaMemcpy(gpu_queue, &jq, sizeof jq, cudaMemcpyHostToDevice));
    const graph_edge_t ne = end;
    CK(cudaMemcpy((char *)gpu_graph + offsetof(Graph, nedges), &ne, sizeof ne, cudaMemcpyHostToDevice));
    CK(cudaMemset(gpu_res, 0, sizeof(size_t) * NWARPS_TOTAL));
    if (l2flush) CK(cudaMemset(l2flush, r & 0xff, kFlushBytes));
    CK(cudaDeviceSynchronize());
    CK(cudaEventRecord(start));
    _parallel_match<<<GRID_DIM, BLOCK_DIM>>>(gpu_graph, gpu_pattern, gpu_callstack, gpu_queue, gpu_res, idle_warps,
                                             idle_warps_count, global_mutex, tq);
    CK(cudaEventRecord(stop));
    CK(cudaEventSynchronize(stop));
    CK(cudaGetLastError());
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, start, stop));
    CK(cudaMemcpy(res.data(), gpu_res, sizeof(size_t) * NWARPS_TOTAL, cudaMemcpyDeviceToHost));
    if (r < warm) continue;  // warm-up launch
    total_ms += ms;
    for (int i = 0; i < NWARPS_TOTAL; i++) total += res[i];
  }
  if (!LABELED) total *= p.PatternMultiplicity;
  printf("%s\t%f\t%llu\n", argv[2], total_ms, total);
  return 0;
}
