/*
 * oracle.h -- CPU oracle for the tdfs subgraph-counting hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (lyuheng/tdfs): the pattern plan compiler of src/pattern.h and the
 * count semantics of the DFS kernel in src/gpu_match.cu.  It is used by the
 * tests as the parity checker and by bench.py as the timed CPU baseline.  The
 * product (tdfs_b200/) never links, loads or calls it.
 *
 * Parity pins: the plan is checked field by field against the reference's own
 * PatternPreprocessor (oracle/refdump.cpp compiled against src/pattern.h and
 * bliss from source), and the counts against closed forms on complete graphs,
 * a brute-force injective-map counter, and counts printed by the reference's
 * own CUDA build (tests/golden/).
 */
#ifndef TDFS_ORACLE_H
#define TDFS_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_PAT_SIZE 7  /* src/config.h:11 PAT_SIZE */

/* condition operators, numbered as src/pattern.h:21 CondOperator */
#define ORC_LESS_THAN 0
#define ORC_LARGER_THAN 1
#define ORC_NON_EQUAL 2

typedef struct {
  int k;                          /* pattern vertices */
  int labeled;                    /* 1: lb semantics, 0: ulb semantics */
  int adj[ORC_PAT_SIZE][ORC_PAT_SIZE];   /* raw edge labels from the .g file */
  int vlabel[ORC_PAT_SIZE];       /* vertex labels (all 1 when unlabeled) */
  int degree[ORC_PAT_SIZE];       /* pattern degree (adj > 0) */
  int nbn[ORC_PAT_SIZE];          /* backward neighbours */
  int bn[ORC_PAT_SIZE][ORC_PAT_SIZE];
  int shared_lvl[ORC_PAT_SIZE];   /* reuse source vertex, -1 = none */
  int nbn_sh[ORC_PAT_SIZE];       /* extra backward neighbours under reuse */
  int bn_sh[ORC_PAT_SIZE][ORC_PAT_SIZE];
  int cond_op[ORC_PAT_SIZE][ORC_PAT_SIZE]; /* cond_op[i][j], j < i */
  int ncond_pairs;                /* symmetry-breaking pairs (a < b) */
  int cond_a[64], cond_b[64];
  int orient;                     /* partial_ori[0][0]: level-0 edge r<c */
  long long multiplicity;         /* PatternMultiplicity (brute-force |Aut|) */
  int aut_size;                   /* |Aut| under the bliss (adj > 0) relation */
} orc_plan;

typedef struct {
  int64_t n;
  int64_t nedges;                 /* directed edge count */
  int64_t *rowptr;                /* n + 1 */
  int32_t *colidx;                /* nedges */
  int32_t *label;                 /* n, or NULL */
  int32_t max_degree;
} orc_graph;

/* status codes */
#define ORC_OK 0
#define ORC_ERR_IO 1
#define ORC_ERR_FORMAT 2
#define ORC_ERR_PATTERN 3

const char *orc_last_error(void);

int orc_plan_from_text(const char *text, int labeled, orc_plan *out);
int orc_plan_from_file(const char *path, int labeled, orc_plan *out);

int orc_graph_load(const char *prefix, int labeled, orc_graph *out);
/* wraps caller memory (not copied, not freed by orc_graph_free) */
void orc_graph_wrap(int64_t n, int64_t nedges, int64_t *rowptr, int32_t *colidx,
                    int32_t *label, orc_graph *out);
void orc_graph_free(orc_graph *g);

/* The reference count for (graph, plan): what ulb/lb print.  Level-0 edges
 * [edge_begin, edge_end) only (pass 0, -1 for all).  threads <= 0: all cores.
 * bytes_out (nullable) receives the merge-model algorithmic bytes. */
int orc_count(const orc_graph *g, const orc_plan *p, int threads,
              int64_t edge_begin, int64_t edge_end,
              unsigned long long *count_out, unsigned long long *bytes_out);

/* Number of injective, edge-preserving (non-induced) maps, and label
 * preserving when p->labeled, by exhaustive search.  Tiny graphs only. */
int orc_bruteforce(const orc_graph *g, const orc_plan *p,
                   unsigned long long *count_out);

#ifdef __cplusplus
}
#endif
#endif
