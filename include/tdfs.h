/*
 * tdfs.h -- C ABI of the B200 subgraph-enumeration engine (libtdfs_b200.so).
 *
 * Drop-in for the hot path of lyuheng/tdfs: the reference has no library API;
 * its seam is graph load -> pattern plan -> one kernel launch -> u64 sum
 * (cu_test.cu:14-107).  Each entry point below names the reference code it
 * replaces.  Plain C types only; handles are opaque and caller-owned.  Every
 * function returns 0 on success or a TDFS_ERR_* code, with a message from
 * tdfs_last_error() (thread-local).  Calls on one handle must come from one
 * host thread at a time.
 */
#ifndef TDFS_B200_H
#define TDFS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TDFS_MAX_PATTERN 7 /* src/config.h:11 PAT_SIZE */

enum {
  TDFS_OK = 0,
  TDFS_ERR_IO = 1,        /* missing/unreadable file (src/graph.h:127-130 exits) */
  TDFS_ERR_FORMAT = 2,    /* malformed graph or pattern file */
  TDFS_ERR_PATTERN = 3,   /* pattern outside the supported class */
  TDFS_ERR_CUDA = 4,      /* CUDA runtime failure */
  TDFS_ERR_CAPACITY = 5,  /* a device buffer limit was exceeded */
  TDFS_ERR_TIMEOUT = 6,   /* a bounded device wait ran out */
  TDFS_ERR_ARG = 7,       /* invalid argument */
  TDFS_ERR_ADMISSION = 8  /* serving: query rejected by the memory budget */
};

typedef struct tdfs_graph tdfs_graph; /* device-resident data graph */
typedef struct tdfs_plan tdfs_plan;   /* compiled pattern plan */
typedef struct tdfs_csr tdfs_csr;     /* host CSR (generators, file reader) */

/* Launch knobs.  Zero means "choose automatically". */
typedef struct {
  int warps_per_block;  /* warps per CTA */
  int blocks_per_sm;    /* resident CTAs per SM */
  int chunk_cap;        /* candidate slots per DFS level (multiple of 32; 0 auto: 128 for patterns
                           of at most 4 vertices, 512 for 5, 256 for 6 and 7, per launch) */
  int steal;            /* 1: intra-block work stealing + global split queue; 0: off; -1 auto */
  int merge_window;     /* merge-window size in ints (0 auto, -1 = binary search only) */
  int64_t edge_begin;   /* level-0 directed-edge range [edge_begin, edge_end) */
  int64_t edge_end;     /*   (0, -1 = all edges) */
  int edge_stride;      /* level-0 chunks are dealt round-robin over edge_stride */
  int edge_phase;       /*   shards; this call takes chunks == edge_phase (mod) */
  void *stream;         /* cudaStream_t; NULL = legacy default stream */
  int steal_min;        /* steal only levels with >= steal_min items left (0 auto = 2) */
  int merge_ratio;      /* merge a list whose length <= merge_ratio x the scanned span, else
                           search it (0 auto = 4) */
  int graph_capture;    /* 1: launch through a cached CUDA graph (upload, reset, kernel,
                           read-back captured once per launch shape and batch size) */
  int edge_chunk;       /* directed edges per level-0 ticket: 1, 2, 4, ..., 32 (0 auto; 32 whenever
                           edge_stride > 1, the chunk the round-robin dealing is defined on) */
  int fixed_stage;      /* last vertex: stage the intersection of its backward neighbours
                           other than the parent once per parent in shared memory
                           (0 auto = on, -1 off) */
  int split_after_us;   /* a warp's subtree becomes stealable after this many microseconds
                           on it, donatable to the HBM ring after 4x (0 auto = 150, -1 = at once) */
  int steal_first;      /* an idle warp first takes a level with >= steal_first items from a warp
                           of its CTA, then a unit of the split ring, and only then a level
                           with >= steal_min items (0 auto = 8) */
  int lane_list;        /* last level with a staged fixed set: up to 32 siblings are counted in
                           one flattened warp pass over their adjacency lists laid end to end;
                           lists longer than max(lane_list, 4 x the fixed set) are counted one by
                           one (0 auto = 32, -1 off: one warp pass per sibling) */
  int64_t work_budget;  /* work units each pattern (or served query) may spend, 0 = unlimited: one
                           unit per DFS node claimed and per 32-wide adjacency scan step.  A pattern
                           that runs out is abandoned on the device and reported with
                           TDFS_ERR_TIMEOUT; the others complete normally */
  int wait_limit_ms;    /* bound on a warp's idle wait for work before the launch reports
                           TDFS_ERR_TIMEOUT (0 auto = 30000) */
  int split_rush_us;    /* > 0: once a quarter of the grid's warps are idle (the tail of a launch),
                           subtrees may be split after this many microseconds instead of
                           split_after_us (0 = off) */
  int leaf_steal_min;   /* items of the last stored level (each only counts leaves) are stolen or
                           donated only while at least this many are left (0 auto = 64, -1 = 2) */
  int label_index;      /* labeled plans take level-0 tickets over the graph's label index: only
                           the edges whose end labels match the plan's first two vertices
                           (0 auto = on, -1 off: every edge id, filtered) */
  int level_hoist;      /* a stored level whose backward neighbours all lie above its parent keeps
                           its candidate set (as of its deepest backward neighbour) and reuses it
                           for every node below, cut by the conditions in between
                           (0 auto = on, -1 off) */
  int label_rows;       /* labeled plans on a graph with at most 16 labels read only the label
                           segment of each adjacency row they scan (rows kept a second time,
                           sorted by label then id) (0 auto = on, -1 off: whole rows, labels
                           tested per candidate) */
  int tail_count;       /* when the last 2 or 3 pattern vertices hang only on vertices up to some
                           level s (no edge among them, and on unlabeled plans no order condition
                           between them), a node at level s counts the leaves below it as the
                           tuples of distinct vertices from their candidate sets, by
                           inclusion-exclusion, instead of enumerating them (0 auto = on, -1 off) */
  int dead_prune;       /* a node at level a is not descended when a later pattern vertex whose
                           backward neighbours all lie at or above a has no candidate under the
                           conditions so far: no leaf can lie below it (0 auto = on, -1 off) */
} tdfs_options;

const char *tdfs_last_error(void);
int tdfs_version(void);
void tdfs_options_default(tdfs_options *opt);

/* ---- data graph: replaces GraphPreprocessor(prefix) + to_gpu()
 *      (src/graph.h:26-50, read_bin_file src/graph.h:136-193) ---------------
 * Reads <prefix>.meta.txt / .vertex.bin / .edge.bin (and .label.bin when
 * labeled) and uploads the CSR to `device`.  Rows must be strictly increasing
 * (the reference asserts no duplicates, src/graph.h:186-192). */
int tdfs_graph_open(const char *prefix, int labeled, int device, tdfs_graph **out);
/* Same from caller host buffers (copied; labels may be NULL when unlabeled). */
int tdfs_graph_from_csr(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx,
                        const int32_t *labels, int device, tdfs_graph **out);
int tdfs_graph_info(const tdfs_graph *g, int64_t *n, int64_t *nedges, int32_t *max_degree,
                    int *labeled, size_t *device_bytes);
int tdfs_graph_free(tdfs_graph *g);

/* ---- pattern plan: replaces PatternPreprocessor(gfile) + to_gpu()
 *      (src/pattern.h:90-108) ------------------------------------------------
 * Matching order = file order; symmetry conditions from the full
 * automorphism group; reuse levels; labels.  labeled selects lb semantics. */
int tdfs_plan_compile(const char *gpath, int labeled, tdfs_plan **out);
int tdfs_plan_from_text(const char *text, int labeled, tdfs_plan **out);
/* JSON with the plan fields the reference kernel reads (for known-answer
 * tests against src/pattern.h).  Returns the needed size in *len. */
int tdfs_plan_dump(const tdfs_plan *p, char *buf, size_t cap, size_t *len);
int tdfs_plan_info(const tdfs_plan *p, int *k, int *labeled, int64_t *multiplicity);
int tdfs_plan_free(tdfs_plan *p);

/* ---- count: replaces the _parallel_match launch + host reduction
 *      (cu_test.cu:81-105; kernel src/gpu_match.cu:951-1080) ----------------
 * *count = the number ulb/lb print (unlabeled totals already x |Aut|).
 * *kernel_ms (nullable) = device time of the match kernel(s), as the
 * reference's cudaEvent pair measures it (cu_test.cu:81-97). */
int tdfs_count(tdfs_graph *g, const tdfs_plan *p, const tdfs_options *opt, uint64_t *count,
               float *kernel_ms);

/* ---- batched launch (no reference counterpart) ----------------------------
 * All plans run in one persistent launch; counts[i] belongs to plans[i]. */
int tdfs_count_batch(tdfs_graph *g, const tdfs_plan *const *plans, int nplans,
                     const tdfs_options *opt, uint64_t *counts, float *kernel_ms);
/* Same, with a status per plan: status[i] = TDFS_OK, or TDFS_ERR_TIMEOUT when
 * plan i ran out of opt->work_budget (counts[i] is then 0).  Returns TDFS_OK
 * when the launch itself succeeded.  tdfs_count_batch returns TDFS_ERR_TIMEOUT
 * when any plan ran out. */
int tdfs_count_batch_status(tdfs_graph *g, const tdfs_plan *const *plans, int nplans,
                            const tdfs_options *opt, uint64_t *counts, int *status, float *kernel_ms);

/* ---- diagnostics of the last count launch on a graph (no reference
 *      counterpart; the reference computes clock64 spans and discards them,
 *      src/gpu_match.cu:1001,1069-1075) ---------------------------------------
 * For a batched count over both modes, the launch of the labeled plans. */
typedef struct {
  uint64_t steals;       /* intra-CTA steals */
  uint64_t splits;       /* subtree units that went through the split ring */
  int64_t warps;         /* warps in the persistent grid */
  double idle_fraction;  /* share of the warps' running time spent without work */
  double mean_warp_ms;   /* mean time a warp ran, first instruction to retirement */
} tdfs_launch_stats;
int tdfs_last_launch(const tdfs_graph *g, tdfs_launch_stats *st);

/* ---- bounded device waits, shown to run out (no reference counterpart) ----
 * Launches the match kernel over a slot that can never complete (admitted,
 * no level-0 tickets, no work held), so every warp waits for work until its
 * wait_limit_ms bound runs out, then the kernel returns.  Returns the status
 * the launch reports -- TDFS_ERR_TIMEOUT when the bound works -- and the
 * kernel's duration in *kernel_ms.  The context stays usable afterwards. */
int tdfs_selftest_wait_limit(tdfs_graph *g, int wait_limit_ms, float *kernel_ms);

/* ---- autotuner (no reference counterpart; the reference's shape is fixed at
 *      compile time, src/config.h:15-27) ---------------------------------------
 * Times launch shapes on a sample of the batch (the level-0 chunks t with
 * t % sample_stride == 0) by coordinate descent over warps per CTA, candidate
 * chunk depth, the steal threshold, stealing on/off, the merge window and the
 * merge/search switch point, and returns the fastest as *best (base's edge
 * range and stream kept).  *best_ms = its sample time.  Under a work budget
 * (base->work_budget) the score is the sample time per completed plan, so a
 * shape that abandons plans early does not win by it. */
int tdfs_autotune(tdfs_graph *g, const tdfs_plan *const *plans, int nplans, const tdfs_options *base,
                  int sample_stride, tdfs_options *best, float *best_ms);

/* ---- serving (no reference counterpart) -----------------------------------
 * A continuous-batching server over one device-resident graph: queries
 * submitted at any time are admitted into a running persistent kernel as
 * in-flight places and device memory free up, so their work overlaps on the
 * GPU.  Admission charges each query its slot record plus one CTA's DFS stack
 * for its pattern size; a query that can never fit is rejected at submit with
 * TDFS_ERR_ADMISSION.  While a server is attached, the graph handle must not
 * be used for tdfs_count / tdfs_count_batch. */
typedef struct tdfs_server tdfs_server;

typedef struct {
  int max_inflight;     /* queries on the device at once (<= 8192) */
  int max_k;            /* largest pattern the stack layout holds (3..7) */
  int labeled;          /* lb (1) or ulb (0) queries */
  int idle_exit_ms;     /* the kernel retires after this long idle; relaunched on demand */
  size_t mem_budget;    /* device bytes charged to in-flight queries (0 = max_inflight x a 7-vertex query) */
  tdfs_options launch;  /* launch knobs; the edge range is ignored */
} tdfs_server_options;

typedef struct {
  uint64_t completed;   /* finished queries, those that ran out of their budget included */
  uint64_t pending;     /* submitted, not yet admitted */
  uint64_t inflight;    /* admitted, not yet complete */
  double p50_us, p99_us, max_us;  /* submit -> completion seen on the host */
  double queries_per_s; /* completed / (last completion - first submit) */
  uint64_t aborted;     /* queries that ran out of the work budget (launch.work_budget) */
} tdfs_serve_stats;

void tdfs_server_options_default(tdfs_server_options *opt);
int tdfs_server_create(tdfs_graph *g, const tdfs_server_options *opt, tdfs_server **out);
int tdfs_server_submit(tdfs_server *s, const tdfs_plan *p, uint64_t *ticket); /* thread-safe */
int tdfs_server_wait(tdfs_server *s, uint64_t ticket, uint64_t *count, double *latency_us);
int tdfs_server_stats(tdfs_server *s, tdfs_serve_stats *st);
int tdfs_server_destroy(tdfs_server *s); /* drains admitted queries, stops the kernel */

/* ---- counting without device allocation (no counterpart in the reference) --
 * For callers that cannot call cudaMalloc: a plugin whose host process hands
 * all device memory to its own allocator, or code that runs where allocating
 * is not allowed.  Same kernel and counts as tdfs_count; the graph is passed
 * as device pointers (not checked: the rules of tdfs_graph_from_csr; labels
 * int32, needed for a labeled pattern) and every working buffer lives in one fixed 48 MiB array inside the
 * library's device image, held on each GPU that uses the library until the
 * process exits.  Graphs whose derived arrays do not fit in it are rejected
 * with TDFS_ERR_CAPACITY (about 4*E + 5*n bytes, up to ~28 MiB, must fit).
 * d_colidx must be 16-byte aligned (TDFS_ERR_ARG otherwise): the kernel reads
 * adjacency windows with 16-byte loads.  When E is not a multiple of 4 those
 * windows are turned off, so nothing past colidx[E-1] is read.  The first
 * call on a device looks up the array's address.  A call waits for its
 * kernel and cannot be recorded into a CUDA graph: on a capturing stream it
 * returns TDFS_ERR_ARG.  Calls share the array: calls that overlap on the
 * GPU race, so serialise them.  opt may be NULL; opt->stream is honoured. */
int tdfs_count_static(int device, int64_t n, int64_t nedges, const int64_t *d_rowptr, const int32_t *d_colidx,
                      const int32_t *d_labels, const tdfs_plan *p, const tdfs_options *opt, uint64_t *count);

/* ---- host CSR: generators and file writer (graph_converter/ output format,
 *      graph_converter/compactify.cpp:172-195, labelize.cpp:130-133) ------- */
int tdfs_csr_read(const char *prefix, int labeled, tdfs_csr **out);
int tdfs_csr_view(const tdfs_csr *c, int64_t *n, int64_t *nedges, const int64_t **rowptr,
                  const int32_t **colidx, const int32_t **labels, int32_t *max_degree);
int tdfs_csr_write(const tdfs_csr *c, const char *prefix); /* .label.bin too when labelled */
int tdfs_csr_set_labels(tdfs_csr *c, int nlabels, uint64_t seed); /* uniform [0, nlabels) */
int tdfs_csr_free(tdfs_csr *c);
/* Host CSR from caller arrays (copied; labels may be NULL), checked as
 * tdfs_graph_from_csr checks them: replaces reading a converted graph back
 * (src/graph.h:136-193) for graphs already in memory. */
int tdfs_csr_from_arrays(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx,
                         const int32_t *labels, tdfs_csr **out);
/* Descending-degree relabelling of any graph (graph_converter/relabel.cpp:
 * 11-71): new vertex i is the i-th of the (degree, id) pairs sorted in
 * descending order, rows re-sorted; labels move with their vertices. */
int tdfs_csr_relabel(const tdfs_csr *in, tdfs_csr **out);
/* Degree orientation of any graph (graph_converter/halve.cpp:10-42): edge
 * (s, d) is kept when deg(d) > deg(s), or they tie and d > s; max_degree
 * becomes the largest kept row.  Vertex ids and labels are unchanged. */
int tdfs_csr_halve(const tdfs_csr *in, tdfs_csr **out);
/* Erdos-Renyi G(n, p), p = avg_degree / (n - 1) */
int tdfs_gen_er(int64_t n, double avg_degree, uint64_t seed, tdfs_csr **out);
/* Chung-Lu power law: ~undirected_edges edges, exponent gamma, degree cap,
 * relabelled in descending-degree order (graph_converter/relabel.cpp:27-35) */
int tdfs_gen_chung_lu(int64_t n, int64_t undirected_edges, double gamma, int32_t max_degree,
                      uint64_t seed, tdfs_csr **out);
/* R-MAT: 2^scale vertices, edge_factor * 2^scale samples, deduplicated and
 * symmetrised, self-loops dropped */
int tdfs_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                  tdfs_csr **out);
/* random connected pattern in valid matching order (vertex i>0 has an earlier
 * neighbour, vertex 2 is adjacent to vertex 1) written as .g text */
int tdfs_gen_pattern(int k, double density, int nlabels, uint64_t seed, char *buf, size_t cap);

/* ---- cost estimate before a count (no counterpart in the reference) -------
 * Knuth's random-probe estimator of the DFS tree the match kernel walks, run
 * on the host copy of the graph: `probes` random root-to-leaf paths with the
 * kernel's exact candidate rules (level-0 edge filter, symmetry conditions or
 * labels, injectivity).  Unbiased for matches and per-depth node counts; the
 * relative standard errors say how far to trust them.  Used to admit or
 * schedule queries by expected work; deterministic for a given seed.  The
 * level-0 edge range [edge_begin, edge_end) is as in tdfs_options (0, -1 =
 * every edge): the estimate of what tdfs_count counts over that range. */
typedef struct tdfs_estimate_result {
  double matches;                  /* expected count, as tdfs_count reports it */
  double nodes[TDFS_MAX_PATTERN];  /* expected partial matches at each depth 1..k-1 */
  double scanned;                  /* expected adjacency entries the set scans read */
  double matches_rse;              /* relative standard error of `matches` */
  double scanned_rse;              /* relative standard error of `scanned` */
  int64_t probes;
} tdfs_estimate_result;
int tdfs_estimate(const tdfs_csr *c, const tdfs_plan *p, int64_t edge_begin, int64_t edge_end, int64_t probes,
                  uint64_t seed, tdfs_estimate_result *out);

#ifdef __cplusplus
}
#endif
#endif
