/*
 * oracle.c -- CPU oracle for the tdfs subgraph-counting hot path.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference
 * algorithm, used by tests/ as the parity checker and by bench.py as the timed
 * CPU baseline.  Nothing in the product (tdfs_b200/) links or calls it.
 *
 * Every function cites the reference file:line (paths inside lyuheng/tdfs)
 * whose behaviour it restates.  The restatement follows the reference's
 * *semantics*; the data structures are this file's own (flat arrays, a
 * recursive DFS over fully materialised candidate sets, pthreads).
 *
 * Parity pins (see tests/): plan fields against the reference's own
 * PatternPreprocessor (oracle/refdump.cpp), counts against closed forms on
 * K_n, against orc_bruteforce() and against counts printed by the
 * reference's own CUDA build (tests/golden/).
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <errno.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

static __thread char g_err[512];

const char *orc_last_error(void) { return g_err; }

static int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

/* ------------------------------------------------------------------------- */
/* .g parsing -- src/pattern.h:110-143 (readfile)                              */
/* ------------------------------------------------------------------------- */

/* Leading '#' lines are skipped; then a run of "v <id> <label>" lines whose
 * labels are taken in line order (the id is ignored, as in the reference);
 * then "e <u> <v> <label>" lines setting adj[u][v] = adj[v][u] = label.
 * Unlabeled mode forces every vertex label to 1 (src/pattern.h:124-129).
 * Blank lines are skipped (the reference would read garbage from them). */
static int parse_g(const char *text, int labeled, orc_plan *p) {
  memset(p, 0, sizeof *p);
  p->labeled = labeled ? 1 : 0;
  const char *s = text;
  int phase = 0; /* 0: header, 1: vertices, 2: edges */
  int lineno = 0;
  while (*s) {
    const char *e = strchr(s, '\n');
    size_t len = e ? (size_t)(e - s) : strlen(s);
    char line[256];
    if (len >= sizeof line) return fail(ORC_ERR_FORMAT, "line %d too long", lineno + 1);
    memcpy(line, s, len);
    line[len] = 0;
    s = e ? e + 1 : s + len;
    lineno++;
    char *q = line;
    while (*q == ' ' || *q == '\t' || *q == '\r') q++;
    if (*q == 0) continue;
    if (phase == 0 && line[0] == '#') continue;
    if (phase == 0) phase = 1;
    if (phase == 1 && line[0] != 'v') phase = 2;
    if (phase == 1) {
      int id, lab;
      if (sscanf(line + 1, "%d %d", &id, &lab) != 2)
        return fail(ORC_ERR_FORMAT, "line %d: bad vertex line", lineno);
      if (p->k >= ORC_PAT_SIZE)
        return fail(ORC_ERR_PATTERN, "pattern has more than %d vertices", ORC_PAT_SIZE);
      p->vlabel[p->k] = labeled ? lab : 1;
      p->k++;
    } else {
      int u, v, lab;
      if (line[0] != 'e' || sscanf(line + 1, "%d %d %d", &u, &v, &lab) != 3)
        return fail(ORC_ERR_FORMAT, "line %d: bad edge line", lineno);
      if (u < 0 || v < 0 || u >= p->k || v >= p->k)
        return fail(ORC_ERR_PATTERN, "line %d: edge endpoint out of range", lineno);
      if (u == v) return fail(ORC_ERR_PATTERN, "line %d: self-loop in pattern", lineno);
      p->adj[u][v] = lab;
      p->adj[v][u] = lab;
    }
  }
  if (p->k < 3) return fail(ORC_ERR_PATTERN, "pattern needs at least 3 vertices");
  return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Permutation groups                                                          */
/* ------------------------------------------------------------------------- */

typedef struct {
  int n;        /* number of perms */
  int k;
  signed char (*perm)[ORC_PAT_SIZE];
} permset;

static int next_perm(int *a, int k) { /* lexicographic next permutation */
  int i = k - 2;
  while (i >= 0 && a[i] >= a[i + 1]) i--;
  if (i < 0) return 0;
  int j = k - 1;
  while (a[j] <= a[i]) j--;
  int t = a[i]; a[i] = a[j]; a[j] = t;
  for (int l = i + 1, r = k - 1; l < r; l++, r--) { t = a[l]; a[l] = a[r]; a[r] = t; }
  return 1;
}

/* The brute-force group of src/pattern.h:274-310: a permutation pp is kept
 * when, for every i, {j : adj[i][j] == 1} equals adj_tmp[i], where
 * adj_tmp[pp[i]] = {pp[j] : adj[i][j] != 0}.  Note the asymmetric `== 1` /
 * `!= 0` tests, restated as they are: with edge label 1 this is Aut(P). */
static int in_bf_group(const orc_plan *p, const int *pp) {
  int k = p->k;
  int tmp[ORC_PAT_SIZE][ORC_PAT_SIZE];
  memset(tmp, 0, sizeof tmp);
  for (int i = 0; i < k; i++)
    for (int j = 0; j < k; j++)
      if (p->adj[i][j] != 0) tmp[pp[i]][pp[j]] = 1;
  for (int i = 0; i < k; i++) {
    int c = 0, sz = 0;
    for (int j = 0; j < k; j++) {
      sz += tmp[i][j];
      if (p->adj[i][j] == 1) {
        c++;
        if (!tmp[i][j]) return 0;
      }
    }
    if (c != sz) return 0;
  }
  return 1;
}

/* The group bliss reports generators for (src/pattern.h:581-594: bliss graph
 * with an edge wherever adj > 0, all vertices one colour), closed under
 * products by src/pattern.h:603-663.  The closure of a generating set of a
 * finite group is the group, so it is enumerated here directly. */
static int in_bliss_group(const orc_plan *p, const int *pp) {
  for (int i = 0; i < p->k; i++)
    for (int j = 0; j < p->k; j++)
      if ((p->adj[i][j] > 0) != (p->adj[pp[i]][pp[j]] > 0)) return 0;
  return 1;
}

/* GetConditions -- src/pattern.h:665-707.  Repeatedly take the orbit class
 * with the smallest representative that has more than one member; n0 is its
 * minimum; for every group element perm add (n0, argmin_{m in class, m != n0}
 * perm[m]); restrict the group to the stabiliser of n0.  Finally sort and
 * deduplicate.  The result depends only on the group as a set. */
static void get_conditions(orc_plan *p, permset *aut) {
  int k = p->k;
  /* at most |G| pairs per round and the group at least halves each round */
  int na = 0, capn = 2 * aut->n + 8;
  int *ca = malloc(sizeof(int) * capn), *cb = malloc(sizeof(int) * capn);
  for (;;) {
    int cls = -1;
    unsigned orbit_mask = 0;
    for (int v = 0; v < k && cls < 0; v++) {
      unsigned m = 0;
      for (int a = 0; a < aut->n; a++) m |= 1u << aut->perm[a][v];
      int rep = __builtin_ctz(m ? m : 1u);
      if (m && rep == v && __builtin_popcount(m) > 1) { cls = v; orbit_mask = m; }
    }
    if (cls < 0) break;
    int n0 = cls;
    for (int a = 0; a < aut->n; a++) {
      int best = -1;
      for (int m = 0; m < k; m++) {
        if (m == n0 || !(orbit_mask >> m & 1)) continue;
        if (best < 0 || aut->perm[a][m] < aut->perm[a][best]) best = m;
      }
      ca[na] = n0;
      cb[na] = best;
      na++;
    }
    int w = 0;
    for (int a = 0; a < aut->n; a++)
      if (aut->perm[a][n0] == n0) memcpy(aut->perm[w++], aut->perm[a], ORC_PAT_SIZE);
    aut->n = w;
  }
  /* sort + unique (lexicographic on pairs) */
  for (int i = 1; i < na; i++) {
    int a = ca[i], b = cb[i], j = i - 1;
    while (j >= 0 && (ca[j] > a || (ca[j] == a && cb[j] > b))) {
      ca[j + 1] = ca[j]; cb[j + 1] = cb[j]; j--;
    }
    ca[j + 1] = a; cb[j + 1] = b;
  }
  p->ncond_pairs = 0;
  for (int i = 0; i < na; i++) {
    if (i > 0 && ca[i] == ca[i - 1] && cb[i] == cb[i - 1]) continue;
    p->cond_a[p->ncond_pairs] = ca[i];
    p->cond_b[p->ncond_pairs] = cb[i];
    p->ncond_pairs++;
  }
  free(ca);
  free(cb);
}

/* ------------------------------------------------------------------------- */
/* Plan compile -- src/pattern.h:90-101 and the steps it calls                 */
/* ------------------------------------------------------------------------- */

static int compile_plan(orc_plan *p) {
  int k = p->k;
  /* pattern degrees, src/pattern.h:189-195 (matching order is the identity,
   * src/pattern.h:184-187) */
  for (int i = 0; i < k; i++) {
    int d = 0;
    for (int j = 0; j < k; j++) d += p->adj[i][j] > 0;
    p->degree[i] = d;
  }

  /* both groups by enumeration of all k! permutations */
  static const int maxperm = 5040;
  permset bliss = {0, k, malloc(sizeof(signed char[ORC_PAT_SIZE]) * maxperm)};
  int a[ORC_PAT_SIZE];
  for (int i = 0; i < k; i++) a[i] = i;
  long long nbf = 0;
  int orient = 0;
  do {
    if (in_bf_group(p, a)) {
      nbf++;
      if (a[0] == 1) orient = 1; /* src/pattern.h:312-340 partial_ori[0][0] */
    }
    if (in_bliss_group(p, a)) {
      for (int i = 0; i < ORC_PAT_SIZE; i++) bliss.perm[bliss.n][i] = (signed char)(i < k ? a[i] : i);
      bliss.n++;
    }
  } while (next_perm(a, k));
  p->multiplicity = nbf;      /* src/pattern.h:310 PatternMultiplicity */
  p->orient = orient;
  p->aut_size = bliss.n;
  get_conditions(p, &bliss);
  free(bliss.perm);

  /* condition_order, src/pattern.h:416-448 with SetConditions
   * src/pattern.h:709-719: for j < i the operator is LARGER_THAN when (j, i)
   * is a condition pair, else NON_EQUAL. */
  for (int i = 0; i < k; i++)
    for (int j = 0; j < i; j++) {
      int op = ORC_NON_EQUAL;
      for (int c = 0; c < p->ncond_pairs; c++) {
        if (p->cond_a[c] == j && p->cond_b[c] == i) { op = ORC_LARGER_THAN; break; }
        if (p->cond_a[c] == i && p->cond_b[c] == j) { op = ORC_LESS_THAN; break; }
      }
      p->cond_op[i][j] = op;
    }

  /* backward neighbours, src/pattern.h:342-358 */
  for (int i = 1; i < k; i++) {
    p->nbn[i] = 0;
    for (int j = 0; j < i; j++)
      if (p->adj[i][j] > 0) p->bn[i][p->nbn[i]++] = j;
  }
  for (int i = 2; i < k; i++)
    if (p->nbn[i] == 0)
      return fail(ORC_ERR_PATTERN, "pattern vertex %d has no earlier neighbour", i);

  /* reuse levels, src/pattern.h:370-413 */
  int nbr_bits[ORC_PAT_SIZE] = {0};
  p->shared_lvl[0] = p->shared_lvl[1] = -1;
  for (int i = 1; i < k; i++) {
    for (int j = 0; j < i; j++)
      if (p->adj[j][i] > 0) nbr_bits[i] |= 1 << j;
    if (i == 1) continue;
    p->shared_lvl[i] = -1;
    for (int j = i - 1; j >= 1; j--) {
      if ((nbr_bits[i] & nbr_bits[j]) == nbr_bits[j] && p->nbn[i] >= 2 && p->nbn[j] >= 2 &&
          p->vlabel[i] == p->vlabel[j]) {
        p->shared_lvl[i] = j;
        break;
      }
    }
  }
  for (int i = 0; i < k; i++) {
    int dep = p->shared_lvl[i];
    p->nbn_sh[i] = 0;
    if (dep == -1) continue;
    for (int j = i - 1; j >= 0; j--)
      if ((nbr_bits[i] >> j & 1) && !(nbr_bits[dep] >> j & 1)) p->bn_sh[i][p->nbn_sh[i]++] = j;
  }
  /* unlabeled: reuse is dropped unless every condition of dep appears among
   * the conditions of i, src/pattern.h:460-480 */
  if (!p->labeled) {
    for (int i = 0; i < k; i++) {
      int dep = p->shared_lvl[i];
      if (dep == -1) continue;
      for (int j = 0; j < dep; j++)
        if (p->cond_op[dep][j] != p->cond_op[i][j]) p->shared_lvl[i] = -1;
    }
  }
  return ORC_OK;
}

int orc_plan_from_text(const char *text, int labeled, orc_plan *out) {
  int rc = parse_g(text, labeled, out);
  if (rc) return rc;
  return compile_plan(out);
}

int orc_plan_from_file(const char *path, int labeled, orc_plan *out) {
  FILE *f = fopen(path, "rb");
  if (!f) return fail(ORC_ERR_IO, "cannot open %s", path);
  char buf[8192];
  size_t n = fread(buf, 1, sizeof buf - 1, f);
  fclose(f);
  buf[n] = 0;
  return orc_plan_from_text(buf, labeled, out);
}

/* ------------------------------------------------------------------------- */
/* Graph files -- src/graph.h:136-193 (read_bin_file)                          */
/* ------------------------------------------------------------------------- */

static int read_exact(const char *path, void *dst, size_t bytes) {
  FILE *f = fopen(path, "rb");
  if (!f) return fail(ORC_ERR_IO, "cannot open %s", path);
  size_t got = fread(dst, 1, bytes, f);
  fclose(f);
  if (got != bytes) return fail(ORC_ERR_FORMAT, "%s: short file", path);
  return ORC_OK;
}

int orc_graph_load(const char *prefix, int labeled, orc_graph *g) {
  memset(g, 0, sizeof *g);
  char path[4096];
  snprintf(path, sizeof path, "%s.meta.txt", prefix);
  FILE *f = fopen(path, "r");
  if (!f) return fail(ORC_ERR_IO, "cannot open %s", path);
  long long n, e, vid, maxd;
  int ok = fscanf(f, "%lld %lld %lld %lld", &n, &e, &vid, &maxd) == 4;
  fclose(f);
  if (!ok || n < 0 || e < 0 || vid != 4)
    return fail(ORC_ERR_FORMAT, "%s: bad meta (need n, E, vid_size=4, max_degree)", path);
  g->n = n;
  g->nedges = e;
  g->rowptr = malloc(sizeof(int64_t) * (n + 1));
  g->colidx = malloc(sizeof(int32_t) * (e ? e : 1));
  int rc;
  snprintf(path, sizeof path, "%s.vertex.bin", prefix);
  if ((rc = read_exact(path, g->rowptr, sizeof(int64_t) * (n + 1)))) goto bad;
  snprintf(path, sizeof path, "%s.edge.bin", prefix);
  if ((rc = read_exact(path, g->colidx, sizeof(int32_t) * e))) goto bad;
  if (labeled) {
    g->label = malloc(sizeof(int32_t) * (n ? n : 1));
    snprintf(path, sizeof path, "%s.label.bin", prefix);
    if ((rc = read_exact(path, g->label, sizeof(int32_t) * n))) goto bad;
  }
  if (g->rowptr[0] != 0 || g->rowptr[n] != e) {
    rc = fail(ORC_ERR_FORMAT, "rowptr does not span [0, E]");
    goto bad;
  }
  int32_t md = 0;
  for (int64_t v = 0; v < n; v++) {
    int64_t b = g->rowptr[v], t = g->rowptr[v + 1];
    if (t < b) { rc = fail(ORC_ERR_FORMAT, "rowptr decreases at %lld", (long long)v); goto bad; }
    if (t - b > md) md = (int32_t)(t - b);
    for (int64_t j = b; j < t; j++) {
      if (g->colidx[j] < 0 || g->colidx[j] >= n) {
        rc = fail(ORC_ERR_FORMAT, "neighbour id out of range at edge %lld", (long long)j);
        goto bad;
      }
      /* src/graph.h:186-192 asserts no duplicates; sortedness is required by
       * the binary search of src/gpu_match.cu:160-185 */
      if (j + 1 < t && g->colidx[j] >= g->colidx[j + 1]) {
        rc = fail(ORC_ERR_FORMAT, "adjacency of %lld not strictly increasing", (long long)v);
        goto bad;
      }
    }
  }
  g->max_degree = md;
  return ORC_OK;
bad:
  orc_graph_free(g);
  return rc;
}

void orc_graph_wrap(int64_t n, int64_t nedges, int64_t *rowptr, int32_t *colidx, int32_t *label,
                    orc_graph *g) {
  g->n = n;
  g->nedges = nedges;
  g->rowptr = rowptr;
  g->colidx = colidx;
  g->label = label;
  int32_t md = 0;
  for (int64_t v = 0; v < n; v++)
    if (rowptr[v + 1] - rowptr[v] > md) md = (int32_t)(rowptr[v + 1] - rowptr[v]);
  g->max_degree = md;
}

void orc_graph_free(orc_graph *g) {
  free(g->rowptr);
  free(g->colidx);
  free(g->label);
  memset(g, 0, sizeof *g);
}

/* ------------------------------------------------------------------------- */
/* DFS count -- semantics of src/gpu_match.cu:496-949 and cu_test.cu:100-105   */
/* ------------------------------------------------------------------------- */

typedef struct {
  const orc_graph *g;
  const orc_plan *p;
  int32_t *cand[ORC_PAT_SIZE];
  int32_t cn[ORC_PAT_SIZE];
  int32_t *tmp;
  int32_t phi[ORC_PAT_SIZE];
  unsigned long long bytes;
} dfs_ctx;

static inline int64_t deg(const orc_graph *g, int32_t v) { return g->rowptr[v + 1] - g->rowptr[v]; }

/* check_validity of src/gpu_match.cu:277-327: unlabeled -> the condition
 * operators against every earlier vertex; labeled -> vertex label equality
 * plus injectivity against every earlier vertex. */
static inline int valid(const dfs_ctx *c, int i, int32_t x) {
  const orc_plan *p = c->p;
  if (!p->labeled) {
    for (int j = 0; j < i; j++) {
      int32_t m = c->phi[j];
      int op = p->cond_op[i][j];
      if (op == ORC_LESS_THAN) { if (m <= x) return 0; }
      else if (op == ORC_LARGER_THAN) { if (m >= x) return 0; }
      else if (m == x) return 0;
    }
    return 1;
  }
  if (c->g->label[x] != p->vlabel[i]) return 0;
  for (int j = 0; j < i; j++)
    if (c->phi[j] == x) return 0;
  return 1;
}

/* in-place intersection of sorted `a` (length na) with sorted `b`; when
 * `filter_i` >= 0 elements of `a` failing valid() are dropped first. */
static int32_t isect(dfs_ctx *c, int filter_i, const int32_t *a, int32_t na, const int32_t *b,
                     int64_t nb, int32_t *out) {
  int32_t w = 0;
  int64_t j = 0;
  for (int32_t t = 0; t < na; t++) {
    int32_t x = a[t];
    if (filter_i >= 0 && !valid(c, filter_i, x)) continue;
    /* gallop in b */
    int64_t step = 1, lo = j;
    while (lo + step < nb && b[lo + step] < x) { lo += step; step <<= 1; }
    int64_t hi = lo + step < nb ? lo + step : nb;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (b[mid] < x) lo = mid + 1; else hi = mid;
    }
    j = lo;
    if (j < nb && b[j] == x) out[w++] = x;
  }
  return w;
}

static int32_t filter_copy(dfs_ctx *c, int i, const int32_t *a, int64_t na, int32_t *out) {
  int32_t w = 0;
  for (int64_t t = 0; t < na; t++)
    if (valid(c, i, a[t])) out[w++] = a[t];
  return w;
}

/* extend of src/gpu_match.cu:623-779 for pattern vertex i: the candidate set
 * into c->cand[i]; returns its size.  The sequence of set operations (which
 * list is scanned, which is searched, reuse of an earlier level's set) is the
 * reference's, so that the merge-model byte count follows its plan. */
static int32_t extend(dfs_ctx *c, int i) {
  const orc_plan *p = c->p;
  const orc_graph *g = c->g;
  int32_t *res = c->cand[i];
  int dep = p->shared_lvl[i];
  if (dep == -1) {
    if (p->nbn[i] == 1) { /* arr_copy, :340-416 */
      int32_t t = c->phi[p->bn[i][0]];
      int64_t d = deg(g, t);
      c->bytes += 16 + 4 * (unsigned long long)d;
      return c->cn[i] = filter_copy(c, i, g->colidx + g->rowptr[t], d, res);
    }
    /* smallest backward-neighbour list is scanned (strict <, first wins),
     * :646-663 */
    int imin = 0;
    int64_t dmin = deg(g, c->phi[p->bn[i][0]]);
    for (int b = 1; b < p->nbn[i]; b++) {
      int64_t d = deg(g, c->phi[p->bn[i][b]]);
      if (d < dmin) { dmin = d; imin = b; }
    }
    c->bytes += 16ull * p->nbn[i];
    int32_t tmin = c->phi[p->bn[i][imin]];
    int first = imin != 0 ? 0 : 1;
    int32_t s1 = c->phi[p->bn[i][first]];
    int64_t d1 = deg(g, s1);
    c->bytes += 16 + 4ull * (unsigned long long)(d1 + dmin);
    int32_t n = isect(c, i, g->colidx + g->rowptr[tmin], (int32_t)dmin, g->colidx + g->rowptr[s1], d1, res);
    for (int b = first + 1; b < p->nbn[i]; b++) {
      if (b == imin) continue;
      int32_t s = c->phi[p->bn[i][b]];
      int64_t d = deg(g, s);
      c->bytes += 16 + 4ull * (unsigned long long)(d + n);
      n = isect(c, -1, res, n, g->colidx + g->rowptr[s], d, res);
    }
    return c->cn[i] = n;
  }
  /* reuse of the candidate set of pattern vertex dep, :733-776 */
  const int32_t *src = c->cand[dep];
  int32_t ns = c->cn[dep];
  if (p->nbn_sh[i] == 0) { /* arr_copy_shared, :418-494 */
    c->bytes += 4ull * (unsigned long long)ns;
    return c->cn[i] = filter_copy(c, i, src, ns, res);
  }
  int32_t s1 = c->phi[p->bn_sh[i][0]];
  int64_t d1 = deg(g, s1);
  c->bytes += 16 + 4ull * (unsigned long long)(d1 + ns);
  int32_t n = isect(c, i, src, ns, g->colidx + g->rowptr[s1], d1, res);
  for (int b = 1; b < p->nbn_sh[i]; b++) {
    int32_t s = c->phi[p->bn_sh[i][b]];
    int64_t d = deg(g, s);
    c->bytes += 16 + 4ull * (unsigned long long)(d + n);
    n = isect(c, -1, res, n, g->colidx + g->rowptr[s], d, res);
  }
  return c->cn[i] = n;
}

/* match, src/gpu_match.cu:830-949: iterate the candidates of every vertex
 * but the last; at the last vertex add the candidate-set size. */
static unsigned long long dfs(dfs_ctx *c, int i) {
  int32_t n = extend(c, i);
  if (i == c->p->k - 1) return (unsigned long long)n;
  unsigned long long s = 0;
  for (int32_t t = 0; t < n; t++) {
    c->phi[i] = c->cand[i][t];
    s += dfs(c, i + 1);
  }
  return s;
}

/* get_job's per-edge filter, src/gpu_match.cu:531-556.  The "some neighbour
 * of c has degree >= degree[2]" test is the reference's (:541-548). */
static int job_ok(const orc_graph *g, const orc_plan *p, int32_t r, int32_t c) {
  if (!p->labeled && p->orient == 1 && !(r < c)) return 0;
  if (p->labeled && !(g->label[r] == p->vlabel[0] && g->label[c] == p->vlabel[1])) return 0;
  if (deg(g, r) < p->degree[0] || deg(g, c) < p->degree[1]) return 0;
  for (int64_t d = g->rowptr[c]; d < g->rowptr[c + 1]; d++)
    if (deg(g, g->colidx[d]) >= p->degree[2]) return 1;
  return 0;
}

typedef struct {
  const orc_graph *g;
  const orc_plan *p;
  int64_t begin, end;
  int64_t next; /* atomic */
  unsigned long long count, bytes;
  pthread_mutex_t mu;
} job_t;

#define ORC_CHUNK 256

static void *worker(void *arg) {
  job_t *J = arg;
  const orc_graph *g = J->g;
  dfs_ctx c;
  memset(&c, 0, sizeof c);
  c.g = g;
  c.p = J->p;
  size_t cap = (size_t)g->max_degree + 1;
  for (int i = 0; i < ORC_PAT_SIZE; i++) c.cand[i] = malloc(sizeof(int32_t) * cap);
  unsigned long long cnt = 0;
  for (;;) {
    int64_t e0 = __atomic_fetch_add(&J->next, ORC_CHUNK, __ATOMIC_RELAXED);
    if (e0 >= J->end) break;
    int64_t e1 = e0 + ORC_CHUNK < J->end ? e0 + ORC_CHUNK : J->end;
    /* source vertex of edge e0: the reference keeps an edge->source array
     * (src/graph.h:195-212); a binary search over rowptr gives the same */
    int64_t lo = 0, hi = g->n;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (g->rowptr[mid + 1] <= e0) lo = mid + 1; else hi = mid;
    }
    int32_t r = (int32_t)lo;
    for (int64_t e = e0; e < e1; e++) {
      while (g->rowptr[r + 1] <= e) r++;
      int32_t cc = g->colidx[e];
      c.bytes += 8;
      if (!job_ok(g, J->p, r, cc)) continue;
      c.phi[0] = r;
      c.phi[1] = cc;
      cnt += dfs(&c, 2);
    }
  }
  for (int i = 0; i < ORC_PAT_SIZE; i++) free(c.cand[i]);
  pthread_mutex_lock(&J->mu);
  J->count += cnt;
  J->bytes += c.bytes;
  pthread_mutex_unlock(&J->mu);
  return NULL;
}

int orc_count(const orc_graph *g, const orc_plan *p, int threads, int64_t edge_begin,
              int64_t edge_end, unsigned long long *count_out, unsigned long long *bytes_out) {
  if (p->labeled && !g->label) return fail(ORC_ERR_FORMAT, "labeled count needs vertex labels");
  if (edge_end < 0 || edge_end > g->nedges) edge_end = g->nedges;
  if (edge_begin < 0) edge_begin = 0;
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  job_t J;
  memset(&J, 0, sizeof J);
  J.g = g;
  J.p = p;
  J.begin = edge_begin;
  J.end = edge_end;
  J.next = edge_begin;
  pthread_mutex_init(&J.mu, NULL);
  pthread_t *th = malloc(sizeof(pthread_t) * threads);
  int started = 0;
  for (int t = 0; t < threads; t++)
    if (pthread_create(&th[t], NULL, worker, &J) == 0) started++;
    else break;
  if (started == 0) worker(&J);
  for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&J.mu);
  /* cu_test.cu:100-105: unlabeled totals are multiplied by |Aut| */
  unsigned long long total = J.count;
  if (!p->labeled) total *= (unsigned long long)p->multiplicity;
  *count_out = total;
  if (bytes_out) *bytes_out = J.bytes;
  return ORC_OK;
}

/* ------------------------------------------------------------------------- */
/* Brute force: injective edge-preserving maps (independent of the plan)       */
/* ------------------------------------------------------------------------- */

static int has_edge(const orc_graph *g, int32_t u, int32_t v) {
  int64_t lo = g->rowptr[u], hi = g->rowptr[u + 1];
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (g->colidx[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo < g->rowptr[u + 1] && g->colidx[lo] == v;
}

static unsigned long long bf_rec(const orc_graph *g, const orc_plan *p, int i, int32_t *phi) {
  if (i == p->k) return 1;
  unsigned long long s = 0;
  for (int32_t x = 0; x < g->n; x++) {
    int ok = 1;
    for (int j = 0; j < i && ok; j++) {
      if (phi[j] == x) ok = 0;
      else if (p->adj[i][j] > 0 && !has_edge(g, phi[j], x)) ok = 0;
    }
    if (ok && p->labeled && g->label[x] != p->vlabel[i]) ok = 0;
    if (!ok) continue;
    phi[i] = x;
    s += bf_rec(g, p, i + 1, phi);
  }
  return s;
}

int orc_bruteforce(const orc_graph *g, const orc_plan *p, unsigned long long *count_out) {
  if (p->labeled && !g->label) return fail(ORC_ERR_FORMAT, "labeled count needs vertex labels");
  int32_t phi[ORC_PAT_SIZE];
  *count_out = bf_rec(g, p, 0, phi);
  return ORC_OK;
}
