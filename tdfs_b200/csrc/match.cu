// match.cu -- the sm_100a DFS subgraph-counting kernel (design notes in
// match.cuh).  Count semantics follow src/gpu_match.cu and cu_test.cu:
//   unlabeled: edges (r, c) with r < c when vertices 0 and 1 are symmetric,
//              every later vertex i drawn from the intersection of its
//              backward neighbours' lists, phi(j) < phi(i) for each
//              symmetry pair (j, i) and phi(j) != phi(i) for other j < i;
//              the host multiplies the total by |Aut|.
//   labeled:   vertex labels must match and every vertex differs from all
//              earlier ones; no multiplier.
//   both:      the level-0 degree filter of get_job (src/gpu_match.cu:540-548).
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <mutex>

#include "match.cuh"

namespace tdfs {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxLists = kMaxK - 1;
constexpr int kCasLimit = 1 << 20;
constexpr int kStoredMax = kMaxK;  // level index bound (stored levels are 2..k-2)
constexpr int kFlatUnroll = 4;     // positions per lane in flight in the flattened last-level pass

struct LevelHdr {
  const int32_t *src;            // source list: global adjacency list or an smem buffer
  const int32_t *mlist[kMaxLists];
  int32_t mlen[kMaxLists];
  int32_t mcur[kMaxLists];
  int32_t spos, send;            // source cursor
  int32_t lo, hi;                // x > lo, x < hi (unlabeled)
  int32_t nm;                    // membership lists
  int32_t nneq;
  int32_t neqv[kMaxK];           // excluded vertices
  int32_t nprod;                 // candidates produced into the buffer (first fill)
  int32_t complete;              // buffer holds the whole candidate set
  uint32_t merge_mask;           // bit m: list m uses the staged-window merge
  int32_t core;                  // hoisted level: the buffer holds the level's core set (see hoist_anchor)
};

struct alignas(16) WarpSmem {
  unsigned long long word[kStoredMax];  // per level 1..k-2: gen:32 | next:16 | end:16
  DevPlan plan;                  // plan of the query this warp works on
  int32_t slot;                  // its slot (-1: none)
  int32_t pad0_[3];
  int32_t phi[kMaxK + 1];
  int32_t er[kEdgeChunk];        // level-1 items: edge pairs (phi(0), phi(1))
  int32_t ec[kEdgeChunk];
  LevelHdr h[kMaxK];
  LevelHdr hf;                   // scan of the last vertex's fixed lists
  int32_t fvalid;                // 0: stale, 1: F holds the fixed set, 2: too large
  int32_t fn;                    // |F|
  int32_t xneq[kMaxK];           // values the last vertex must differ from, between F's anchor and the parent
  int32_t tn[3];                 // count_tail: sizes of the tail's base sets
  int8_t tanc[4];                //   and the level each base's conditions reach
  // derived from the plan once per plan switch (derive_plan)
  int8_t hanchor[kMaxK];         // per level: anchor of a hoisted level, -1 when not hoisted
  uint8_t hneq[kMaxK];           // per hoisted level: bit j = candidates must differ from phi(j)
  int8_t fanchor;                // anchor of the last vertex's fixed set
  int8_t lastmode;               // last vertex: 2 parent-free fixed set, 1 fixed set with the parent,
                                 // 3 the parent its one backward neighbour (label segments), 0 none of these
  uint8_t hoistmask;             // bit i: level i is hoisted
  int8_t tail;                   // level whose nodes count their independent tail in closed form, -1 none
  uint8_t deadmask[kMaxK];       // per level a: bit j = vertex j's candidates depend on phi(0..a) only and
                                 // are checked for emptiness at each level-a node (dead-subtree pruning)
  unsigned long long t_base;     // globaltimer when the current base work was taken
  // lane 0's bookkeeping, kept here rather than in registers every lane holds
  unsigned long long idle_since; // bounded idle wait: start of the current wait
  unsigned long long idle_start; // diagnostics: start of the current idle span
  unsigned long long idle_total; // diagnostics: idle time so far
  unsigned long long t_start;    // diagnostics: when this warp started
  int32_t hungry_seen;           // the grid's idle-warp count as last read (maybe_donate)
  int32_t pad_h_;
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ void raise_error(RunCtl *ctl, int code) { atomicCAS(&ctl->error, 0, code); }

// first index in a[lo, hi) with a[idx] >= x
__device__ __forceinline__ int32_t lower_bound(const int32_t *a, int32_t lo, int32_t hi, int32_t x) {
  while (lo < hi) {
    const int32_t mid = (lo + hi) >> 1;
    if (a[mid] < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// first index in a[lo, hi) with a[idx] > x, by 32-ary warp search
__device__ int32_t warp_upper_bound(const int32_t *a, int32_t lo, int32_t hi, int32_t x) {
  const int lane = lane_id();
  while (hi - lo > 32) {
    const int32_t step = (hi - lo + 31) >> 5;
    const int32_t idx = lo + lane * step;
    const bool le = idx < hi && a[idx] <= x;
    const int c = __popc(__ballot_sync(kFull, le));
    if (c == 0) return lo;
    const int32_t nlo = lo + (c - 1) * step + 1;
    hi = min(hi, lo + c * step);
    lo = nlo;
  }
  const int32_t idx = lo + lane;
  const bool le = idx < hi && a[idx] <= x;
  return lo + __popc(__ballot_sync(kFull, le));
}

template <bool LAB>
__device__ __forceinline__ bool pass_filter(int32_t x, const LevelHdr &H, int i, const DevPlan &P,
                                            const DevGraph &G, bool segmented) {
  if (LAB) {
    // reading label segments, every source holds i's label only
    if (!segmented && (int32_t)G.label[x] != P.label[i]) return false;
  } else {
    if (x <= H.lo || x >= H.hi) return false;
  }
#pragma unroll
  for (int t = 0; t < kMaxK; ++t)
    if (t < H.nneq && H.neqv[t] == x) return false;
  return true;
}

// Stage L[cur .. cur + window) of membership list m in shared memory with
// 16-byte loads from the aligned offset below cur, no further than the list's
// end.  Returns the staged extent; the caller syncs the warp before reading.
struct Window {
  int32_t first;  // index of the cursor position inside win
  int32_t last;   // exclusive end of valid entries in win
};

__device__ __forceinline__ Window stage_window(const int32_t *L, int32_t len, int32_t cur, int32_t *win,
                                               int window, const int32_t *colidx) {
  const int lane = lane_id();
  const int64_t off = (int64_t)(L - colidx) + cur;
  const int64_t a0 = off & ~(int64_t)3;
  const int64_t wend = (int64_t)(L - colidx) + len - a0;
  Window w;
  w.last = (int32_t)(wend < (int64_t)window ? wend : (int64_t)window);
  w.first = (int32_t)(off - a0);
  const int4 *gsrc = reinterpret_cast<const int4 *>(colidx + a0);
  const int nvec = (max(w.last, 0) + 3) >> 2;
  for (int t = lane; t < nvec; t += 32) reinterpret_cast<int4 *>(win)[t] = __ldg(gsrc + t);
  return w;
}

// Membership of each lane's x in the level's other lists.  `ok` lanes are
// tested; cursors advance monotonically (the source is sorted).  List 0's
// window may already be staged (`w0`, issued together with the source load
// so the two memory round trips overlap); `win` is the warp's staging area.
__device__ __forceinline__ bool test_lists(bool ok, int32_t x, const LevelHdr &H,
                                           int32_t (&cur)[kMaxLists], int32_t *win, int window,
                                           const int32_t *colidx, bool staged0, Window w0) {
#pragma unroll
  for (int m = 0; m < kMaxLists; ++m) {
    if (m >= H.nm) break;
    const int32_t *L = H.mlist[m];
    const int32_t len = H.mlen[m];
    int32_t p = 0;
    const bool searched = ok;
    const bool merge = H.merge_mask >> m & 1;
    if (merge && ((m == 0 && staged0) || __any_sync(kFull, ok))) {
      const Window w = (m == 0 && staged0) ? w0 : stage_window(L, len, cur[m], win, window, colidx);
      __syncwarp();
      if (ok) {
        if (w.first < w.last && x <= win[w.last - 1]) {
          const int32_t q = lower_bound(win, w.first, w.last, x);
          p = cur[m] + (q - w.first);
          ok = win[q] == x;
        } else {
          const int32_t from = cur[m] + max(0, w.last - w.first);
          p = lower_bound(L, from, len, x);
          ok = p < len && L[p] == x;
        }
      }
      __syncwarp();
    } else if (ok) {
      p = lower_bound(L, cur[m], len, x);
      ok = p < len && L[p] == x;
    }
    const unsigned mx = __reduce_max_sync(kFull, searched ? (unsigned)p : 0u);
    cur[m] = max(cur[m], (int32_t)mx);
  }
  return ok;
}

template <bool LAB>
struct Engine {
  const DevPlan &P;  // W.plan
  const DevGraph &G;
  const KernelCfg &cfg;
  RunCtl *ctl;
  SlotTable *tab;
  SplitUnit *units;
  QueueHdr *qh;
  WarpSmem &W;
  int32_t *bufs;  // stored level l at bufs + (l - 2) * cap
  int32_t *win;   // merge staging (cfg.window ints)
  unsigned char *cta;   // this CTA's shared memory (warp regions cfg.warp_bytes apart)
  size_t hdr_bytes;     // WarpSmem rounded to 16 bytes
  unsigned long long count = 0;
  unsigned work = 0;  // work units since the last flush: one per claim and per 32-wide scan step
  int lane;

  __device__ Engine(const DevGraph &g, const KernelCfg &c, RunCtl *ct, SlotTable *tb, SplitUnit *u, QueueHdr *q,
                    WarpSmem &w, int32_t *b, int32_t *wn)
      : P(w.plan), G(g), cfg(c), ctl(ct), tab(tb), units(u), qh(q), W(w), bufs(b), win(wn), lane(lane_id()) {
    extern __shared__ __align__(16) unsigned char smem[];
    cta = smem;
    hdr_bytes = (sizeof(WarpSmem) + 15) & ~(size_t)15;
  }

  __device__ __forceinline__ int32_t *buf(int l) { return bufs + (l - 2) * cfg.cap; }
  __device__ __forceinline__ int32_t *fbuf() { return win + cfg.window; }  // F (cfg.fixed)
  __device__ __forceinline__ int64_t deg(int32_t v) { return G.rowptr[v + 1] - G.rowptr[v]; }

  // Adjacency rows as pattern vertex i sees them.  On a label-partitioned
  // graph a labeled plan reads only the segment of a row that carries vertex
  // i's label (every candidate of i must carry it); otherwise the whole row.
  __device__ __forceinline__ bool segmented() const { return LAB && cfg.segments && G.colidx_l != nullptr; }
  __device__ __forceinline__ const int32_t *lbase() const { return segmented() ? G.colidx_l : G.colidx; }
  __device__ __forceinline__ void row_for(int32_t v, int i, int64_t &b, int64_t &e) const {
    if (segmented()) {
      const int l = P.label[i];
      const int64_t r = G.rowptr[v];
      if (l >= G.nlab) {  // a label no vertex carries
        b = e = r;
        return;
      }
      const int32_t *o = G.loff + (int64_t)v * (G.nlab + 1) + l;
      b = r + o[0];
      e = r + o[1];
    } else {
      b = G.rowptr[v];
      e = G.rowptr[v + 1];
    }
  }

  // Set up the candidate scan of pattern vertex i from phi(0..i-1).
  __device__ void setup(int i, bool allow_reuse) {
    stale_from(i - 1);
    setup_into(W.h[i], i, allow_reuse, i - 1);
  }

  // phi(j) just changed: the sets built on phi(0..j) -- the last vertex's
  // fixed set and the core sets of hoisted levels anchored at j or deeper --
  // are stale.
  __device__ void stale_from(int j) {
    if (lane == 0) {
      if (W.fanchor >= j) W.fvalid = 0;
      unsigned m = (unsigned)W.hoistmask >> (j + 1) << (j + 1);
      while (m) {
        const int t = __ffs(m) - 1;
        m &= m - 1;
        if (W.hanchor[t] >= j) W.h[t].core = 0;
      }
    }
    __syncwarp();  // every lane reads the flags next, to take the same path
  }

  // ---- hoisted levels --------------------------------------------------------
  // A stored level i whose backward neighbours all lie at or above level a <
  // i - 1 (a = its deepest one, at least 1) has a candidate set that depends
  // on phi(0..a) only, except for the conditions on the vertices between a
  // and i: the "core" set -- the backward neighbours' lists intersected and
  // filtered by the conditions on phi(0..a) -- is produced once per node at
  // level a into the level's buffer and reused for every node below it.  Each
  // reuse publishes the sub-range of the sorted core set inside the bounds of
  // the conditions between a and i (two searches in shared memory); values
  // that must differ from one of those vertices are skipped when claimed
  // (item_ok).  Returns a, or -1 when level i is not hoisted.
  __device__ int hoist_anchor_of(int i) const {
    if (!cfg.hoist || i < 2 || i > P.k - 2 || P.dep[i] >= 0) return -1;
    int a = 1;
    for (int t = 0; t < P.nbn[i]; ++t) a = max(a, (int)P.bn[i][t]);
    return a < i - 1 ? a : -1;
  }
  __device__ __forceinline__ int hoist_anchor(int i) const { return W.hanchor[i]; }

  // The plan's derived tables (anchors, masks, last-level mode), written by
  // lane 0 whenever W.plan changes, so the DFS loop reads them instead of
  // recomputing them from the plan at every node.
  __device__ void derive_plan() {
    if (lane == 0) {
      unsigned hm = 0;
      for (int i = 0; i < kMaxK; ++i) {
        const int a = hoist_anchor_of(i);
        W.hanchor[i] = (int8_t)a;
        unsigned m = 0;
        if (a >= 0) {
          hm |= 1u << i;
          for (int j = a + 1; j < i; ++j)
            if (LAB || !((P.larger[i] | P.less[i]) >> j & 1)) m |= 1u << j;
        }
        W.hneq[i] = (uint8_t)m;
      }
      W.hoistmask = (uint8_t)hm;
      const int last = P.k - 1;
      W.fanchor = (int8_t)fixed_anchor(last);
      W.lastmode = (int8_t)(free_applies(last) ? 2 : fixed_applies(last) ? 1 : single_applies(last) ? 3 : 0);
      W.tail = (int8_t)tail_level();
      for (int a = 0; a < kMaxK; ++a) W.deadmask[a] = 0;
      if (LAB && cfg.prune) {  // labeled plans: sparse label sets make empty ones common
        for (int j = 3; j < P.k; ++j) {
          int a = 1;  // level-1 items set phi(0) and phi(1) together
          for (int t = 0; t < P.nbn[j]; ++t) a = max(a, (int)P.bn[j][t]);
          if (j >= a + 2) W.deadmask[a] |= (uint8_t)(1u << j);
        }
      }
    }
    __syncwarp();
  }

  // ---- dead subtrees ---------------------------------------------------------
  // A vertex j whose backward neighbours all lie at or above level a < j-1
  // has, below a node at level a, candidates that are a subset of its
  // backward neighbours' lists filtered by the conditions on phi(0..a).  When
  // that set is empty, no node below has a leaf: the node is not descended.
  // The check scans only until its first candidate.
  __device__ bool subtree_dead(int a) {
    unsigned m = W.deadmask[a];
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      if (collect(j, a, nullptr) == 0) return true;
    }
    return false;
  }

  // ---- independent tail ------------------------------------------------------
  // The last t = k-1-s pattern vertices (2 <= t <= 3, s >= 2) form an
  // independent tail when every backward neighbour of each lies at or above
  // level s, and -- on unlabeled plans -- no order condition ties two of them.
  // Below a node at level s their candidate sets A_j are then fixed (the
  // backward neighbours' lists, filtered by the conditions on phi(0..s)), and
  // the leaves the DFS would count are exactly the tuples of distinct
  // vertices drawn one from each set; count_tail counts them by
  // inclusion-exclusion instead of enumerating levels s+1..k-1.  The smallest
  // such s is taken.  Returns s, or -1.
  __device__ int tail_level() const {
    if (!cfg.tail || !cfg.fixed) return -1;
    const int k = P.k;
    for (int s = max(2, k - 4); s <= k - 3; ++s) {
      bool ok = true;
      for (int j = s + 1; j < k; ++j) {
        for (int t = 0; t < P.nbn[j]; ++t) ok &= P.bn[j][t] <= s;
        if (!LAB) ok &= ((unsigned)(P.larger[j] | P.less[j]) >> (s + 1)) == 0;
      }
      if (ok) return s;
    }
    return -1;
  }

  // Lane-wise: may candidate x of level l be claimed under the current
  // prefix?  Only a hoisted level has candidates that can fail: those equal
  // to a vertex between the anchor and l that l must differ from.
  __device__ __forceinline__ bool item_ok(int l, int32_t x) const {
    unsigned m = W.hneq[l];
    while (m) {
      const int j = __ffs(m) - 1;
      m &= m - 1;
      if (W.phi[j] == x) return false;
    }
    return true;
  }

  // Produce level i's core set into its buffer when the smallest source list
  // fits (the whole set then lands in one chunk); false otherwise, and the
  // caller produces the level the ordinary way.
  __device__ bool build_core(int i, int a) {
    LevelHdr &H = W.h[i];
    setup_into(H, i, false, a);
    if (H.send - H.spos > cfg.cap - 32) return false;
    produce(i);
    if (lane == 0) {
      H.core = 1;
      H.complete = 0;  // not the candidate set of the current prefix: no reuse from it
    }
    __syncwarp();
    return true;
  }

  // Publish the part of level i's core set inside the bounds of the
  // conditions on the vertices between the anchor a and i.
  __device__ void publish_core(int i, int a) {
    int32_t lo = -1, hi = INT_MAX;
    if (!LAB && lane > a && lane < i) {
      if (P.larger[i] >> lane & 1) lo = W.phi[lane];
      else if (P.less[i] >> lane & 1) hi = W.phi[lane];
    }
    lo = (int32_t)__reduce_max_sync(kFull, (unsigned)(lo + 1)) - 1;
    hi = (int32_t)__reduce_min_sync(kFull, (unsigned)hi);
    if (lane == 0) {
      const int32_t *c = buf(i);
      const int32_t n = W.h[i].nprod;
      const int32_t b = lo >= 0 ? upper_bound_smem(c, n, lo) : 0;
      const int32_t e = hi < INT_MAX ? lower_bound(c, 0, n, hi) : n;
      const unsigned long long gen = (W.word[i] >> 32) + 1;
      __threadfence_block();
      atomicExch(&W.word[i], (gen << 32) | ((unsigned long long)b << 16) | (unsigned long long)max(b, e));
    }
    __syncwarp();
  }

  // The level the last vertex i's fixed set F hangs on: its deepest backward
  // neighbour other than the parent (vertex i-1), at least 1 (level-1 items
  // change phi(0) and phi(1) together).  F is built with the backward
  // neighbours and conditions of vertices up to the anchor only, so it stays
  // valid for every node below the anchor; the conditions on the vertices
  // between the anchor and the parent are applied per count (extra_conds).
  __device__ int fixed_anchor(int i) const {
    int a = 1;
    for (int t = 0; t < P.nbn[i]; ++t) {
      const int b = P.bn[i][t];
      if (b != i - 1 && b > a) a = b;
    }
    return a;
  }

  // Set up a scan for vertex i into header H over the backward neighbours and
  // conditions of the vertices up to `limit` (i - 1: all of them; smaller:
  // the fixed part of the last vertex's candidate set, see build_fixed).
  __device__ void setup_into(LevelHdr &H, int i, bool allow_reuse, int limit) {
    const int dep = P.dep[i];
    const bool full = limit >= i - 1;
    const bool reuse = full && allow_reuse && dep >= 2 && W.h[dep].complete;
    const int32_t *src;
    int32_t slen;
    int nm = 0;
    int mylen = -1, myslot = -1;  // this lane's membership list, if any
    if (reuse) {
      src = buf(dep);
      slen = W.h[dep].nprod;
      nm = P.nsh[i];
      if (lane < nm) {
        const int32_t v = W.phi[P.bnsh[i][lane]];
        int64_t b, e;
        row_for(v, i, b, e);
        mylen = (int32_t)(e - b);
        myslot = lane;
        H.mlist[lane] = lbase() + b;
        H.mlen[lane] = mylen;
        H.mcur[lane] = 0;
      }
    } else {
      // scan the smallest backward-neighbour list (first on ties, as
      // src/gpu_match.cu:646-663)
      const int nbn = P.nbn[i];
      const bool part = lane < nbn && P.bn[i][lane] <= limit;
      const unsigned pmask = __ballot_sync(kFull, part);
      unsigned long long key = ~0ull;
      int64_t b = 0, e = 0;
      if (part) {
        const int32_t v = W.phi[P.bn[i][lane]];
        row_for(v, i, b, e);
        key = ((unsigned long long)(e - b) << 8) | (unsigned)lane;
      }
      unsigned long long best = key;
#pragma unroll
      for (int s = 16; s >= 1; s >>= 1) {
        const unsigned long long o = __shfl_xor_sync(kFull, best, s);
        best = o < best ? o : best;
      }
      const int bmin = (int)(best & 0xff);
      const int64_t sb = __shfl_sync(kFull, b, bmin);
      slen = (int32_t)(best >> 8);
      src = lbase() + sb;
      nm = __popc(pmask) - 1;
      if (part && lane != bmin) {
        const int rank = __popc(pmask & lanemask_lt());
        const int rmin = __popc(pmask & ((1u << bmin) - 1u));
        myslot = rank < rmin ? rank : rank - 1;
        mylen = (int32_t)(e - b);
        H.mlist[myslot] = lbase() + b;
        H.mlen[myslot] = mylen;
        H.mcur[myslot] = 0;
      }
    }
    // bounds from the symmetry conditions; the excluded vertices are packed
    // into shared memory by ballot (lane j looks at phi(j))
    int32_t lo = -1, hi = INT_MAX;
    bool isneq = false;
    int32_t myphi = 0;
    if (lane < i && lane <= limit) {
      myphi = W.phi[lane];
      if (LAB) {
        isneq = true;
      } else if (P.larger[i] >> lane & 1) {
        lo = myphi;
      } else if (P.less[i] >> lane & 1) {
        hi = myphi;
      } else {
        isneq = true;
      }
    }
    lo = __reduce_max_sync(kFull, (unsigned)(lo + 1)) - 1;  // lo >= -1
    hi = (int32_t)__reduce_min_sync(kFull, (unsigned)hi);
    const unsigned nmask = __ballot_sync(kFull, isneq);
    const int nneq = __popc(nmask);
    if (isneq) H.neqv[__popc(nmask & lanemask_lt())] = myphi;
    // skip the prefix <= lo by a 32-ary search; a short source is cheaper to
    // filter in the scan, except when the closed-form count needs the bound
    int32_t spos = 0;
    const bool closed = !LAB && nm == 0 && hi == INT_MAX && i == P.k - 1 && full;
    if (!LAB && lo >= 0 && slen > 0 && (slen > 64 || closed)) spos = warp_upper_bound(src, 0, slen, lo);
    // merge (staged window) or per-lane search, per list, by degree ratio
    uint32_t mm = 0;
    if (cfg.window > 0 && myslot >= 0 && (int64_t)mylen <= (int64_t)cfg.merge_ratio * max(1, slen - spos)) mm = 1u << myslot;
    mm = __reduce_or_sync(kFull, mm);
    if (lane == 0) {
      H.src = src;
      H.send = slen;
      H.spos = spos;
      H.lo = lo;
      H.hi = hi;
      H.nm = nm;
      H.nneq = nneq;
      H.complete = 0;
      H.nprod = -1;
      H.merge_mask = mm;
    }
    __syncwarp();
  }

  // Fill the level-i buffer with the next chunk of candidates and publish it.
  __device__ void produce(int i) {
    LevelHdr &H = W.h[i];
    int32_t *out = buf(i);
    const int32_t *src = H.src;
    int32_t spos = H.spos;
    const int32_t send = H.send;
    int32_t cur[kMaxLists];
#pragma unroll
    for (int m = 0; m < kMaxLists; ++m) cur[m] = m < H.nm ? H.mcur[m] : 0;
    int32_t n = 0;
    const int32_t cap = cfg.cap;
    while (n <= cap - 32 && spos < send) {
      const int32_t idx = spos + lane;
      const bool valid = idx < send;
      const int32_t x = valid ? src[idx] : 0;
      const bool st0 = H.nm > 0 && (H.merge_mask & 1u);
      Window w0 = {0, 0};
      if (st0) w0 = stage_window(H.mlist[0], H.mlen[0], cur[0], win, cfg.window, lbase());
      bool ok = valid && pass_filter<LAB>(x, H, i, P, G, segmented());
      ok = test_lists(ok, x, H, cur, win, cfg.window, lbase(), st0, w0);
      const unsigned mask = __ballot_sync(kFull, ok);
      if (ok) out[n + __popc(mask & lanemask_lt())] = x;
      n += __popc(mask);
      spos += 32;
      ++work;
    }
    __syncwarp();
    if (lane == 0) {
      const bool first = H.nprod < 0;
      H.spos = spos;
#pragma unroll
      for (int m = 0; m < kMaxLists; ++m)
        if (m < H.nm) H.mcur[m] = cur[m];
      if (first) {
        H.nprod = n;
        H.complete = spos >= send;
      } else {
        H.complete = 0;
      }
      const unsigned long long gen = (W.word[i] >> 32) + 1;
      __threadfence_block();
      atomicExch(&W.word[i], (gen << 32) | (unsigned long long)n);
    }
    __syncwarp();
  }

  // Count the candidates of the last pattern vertex (not stored).
  // The last vertex's backward neighbours other than its parent (vertex i-1)
  // are the same for every sibling at level i-1: their filtered intersection
  // F is built once per parent into shared memory, and each sibling then
  // counts |F ∩ N(phi(i-1))| under the one condition that involves the
  // parent.  Applies when the parent is a backward neighbour, at least one
  // other backward neighbour exists and the plan does not reuse a level.
  __device__ bool fixed_applies(int i) {
    if (!cfg.fixed || i < 3 || P.dep[i] >= 0 || P.nbn[i] < 2) return false;
    bool has_parent = false;
    for (int t = 0; t < P.nbn[i]; ++t) has_parent |= P.bn[i][t] == i - 1;
    return has_parent;
  }

  // Scan vertex i's candidates under the backward neighbours and conditions
  // of the vertices up to `limit` into `out` (scratch header W.hf).  Returns
  // their number, or -1 when they might not fit in `cap` entries.  With
  // out == nullptr nothing is stored and the scan stops at the first
  // candidate (the result is then 0 or more).
  __device__ int32_t collect(int i, int limit, int32_t *out) {
    LevelHdr &H = W.hf;
    setup_into(H, i, false, limit);
    const int32_t *src = H.src;
    const int32_t send = H.send;
    int32_t cur[kMaxLists];
#pragma unroll
    for (int m = 0; m < kMaxLists; ++m) cur[m] = m < H.nm ? H.mcur[m] : 0;
    int32_t n = 0;
    bool over = false;
    for (int32_t spos = H.spos; spos < send; spos += 32) {
      ++work;
      if (out && n > cfg.cap - 32) {  // a full step could write past the buffer: give up
        over = true;
        break;
      }
      const int32_t idx = spos + lane;
      const bool valid = idx < send;
      const int32_t x = valid ? src[idx] : 0;
      bool ok = valid && pass_filter<LAB>(x, H, i, P, G, segmented());
      ok = test_lists(ok, x, H, cur, win, cfg.window, lbase(), false, Window{0, 0});
      const unsigned mask = __ballot_sync(kFull, ok);
      if (ok && out) out[n + __popc(mask & lanemask_lt())] = x;
      n += __popc(mask);
      if (!out && n > 0) break;
    }
    __syncwarp();
    return over ? -1 : n;
  }

  __device__ void build_fixed(int i) {
    const int32_t n = collect(i, W.fanchor, fbuf());
    if (lane == 0) {
      W.fn = max(n, 0);
      W.fvalid = n < 0 ? 2 : 1;
    }
    __syncwarp();
  }

  // |a ∩ b| of two sorted sets in shared memory (lanes search the smaller
  // one's elements in the larger); with c, |a ∩ b ∩ c|.
  __device__ int32_t common_count(const int32_t *a, int32_t na, const int32_t *b, int32_t nb,
                                  const int32_t *c = nullptr, int32_t nc = 0) {
    if (na > nb) {
      const int32_t *t = a; a = b; b = t;
      const int32_t u = na; na = nb; nb = u;
    }
    int32_t r = 0;
    for (int32_t pos = 0; pos < na; pos += 32) {
      const int32_t idx = pos + lane;
      bool ok = idx < na;
      if (ok) {
        const int32_t y = a[idx];
        const int32_t q = lower_bound(b, 0, nb, y);
        ok = q < nb && b[q] == y;
        if (ok && c) {
          const int32_t q2 = lower_bound(c, 0, nc, y);
          ok = q2 < nc && c[q2] == y;
        }
      }
      r += __popc(__ballot_sync(kFull, ok));
    }
    return r;
  }

  // Leaves below the current node at level s = W.tail: the tuples of
  // distinct vertices from the tail's candidate sets A_{s+1}, .., A_{k-1},
  // built into the buffers of levels s+1.. and F's buffer.  With t = 2:
  // |A||B| - |A ∩ B|; with t = 3: |A||B||C| - |A ∩ B||C| - |A ∩ C||B|
  // - |B ∩ C||A| + 2|A ∩ B ∩ C|.  On labeled plans two tail vertices with
  // different labels never meet, so their intersection term is dropped.
  // Returns -1 when a set might not fit its buffer; the caller then descends
  // the ordinary way (the buffers' previous contents are marked stale here).
  // Unlabeled plans: every tail set built per node, with the conditions on
  // phi(0..s) (order conditions included), so no base needs a correction.
  __device__ long long count_tail_per_node(int s) {
    const int k = P.k;
    const int t = k - 1 - s;
    if (lane == 0) {
      W.fvalid = 0;
      for (int l = s + 1; l <= k - 2; ++l) W.h[l].core = W.h[l].complete = 0;
    }
    __syncwarp();
#pragma unroll 1
    for (int u = 0; u < t; ++u) {
      const int32_t n = collect(s + 1 + u, s, u == t - 1 ? fbuf() : buf(s + 1 + u));
      if (n <= 0) return n;  // -1: might not fit; 0: an empty set, no leaves
      if (lane == 0) W.tn[u] = n;
    }
    __syncwarp();
    const int32_t *A0 = buf(s + 1), *A1 = t == 2 ? fbuf() : buf(s + 2), *A2 = fbuf();
    const int32_t n0 = W.tn[0], n1 = W.tn[1], n2 = t == 3 ? W.tn[2] : 1;
    long long c = (long long)n0 * n1 * n2 - (long long)common_count(A0, n0, A1, n1) * n2;
    if (t == 2) return c;
    c -= (long long)common_count(A0, n0, A2, n2) * n1;
    c -= (long long)common_count(A1, n1, A2, n2) * n0;
    c += 2ll * common_count(A0, n0, A1, n1, A2, n2);
    return c;
  }

  __device__ long long count_tail(int s) {
    if (!LAB) return count_tail_per_node(s);
    const int k = P.k;
    const int t = k - 1 - s;
    // phi(s) just changed: the sets anchored at s or deeper are stale
    stale_from(s);
    // Each tail set is taken from a base that may be shared by all nodes
    // below an earlier level: a hoisted level's core set (anchor hanchor[j])
    // or the last vertex's fixed set F (anchor fanchor), built once per anchor
    // node.  A base anchored at a holds the set under the conditions on
    // phi(0..a); the vertices phi(a+1..s) it may still hold are removed from
    // the counts below.  Other sets are built per node.  One call site of
    // collect for all of them (the kernel's code stays small).
#pragma unroll 1
    for (int u = 0; u < t; ++u) {
      const int j = s + 1 + u;
      // 0: built per node; 1: the last vertex's F; 2: a hoisted level's core
      const int kind = (LAB && j == k - 1) ? 1 : (LAB && j < k - 1 && W.hanchor[j] >= 0) ? 2 : 0;
      const int anc = kind == 1 ? W.fanchor : kind == 2 ? W.hanchor[j] : s;
      int32_t n;
      if (kind == 1 && W.fvalid == 2) return -1;  // F does not fit
      if ((kind == 1 && W.fvalid == 1) || (kind == 2 && W.h[j].core)) {
        n = kind == 1 ? W.fn : W.h[j].nprod;
      } else {
        n = collect(j, anc, j == k - 1 ? fbuf() : buf(j));
        if (lane == 0) {
          if (kind == 1) {  // as build_fixed leaves it
            W.fn = max(n, 0);
            W.fvalid = n < 0 ? 2 : 1;
          } else if (kind == 2 && n >= 0) {  // as build_core leaves it, without publishing any item
            LevelHdr &H = W.h[j];
            H.nprod = n;
            H.core = 1;
            H.complete = 0;
            H.spos = H.send = 0;
          } else if (j == k - 1) {
            W.fvalid = 0;  // F's buffer now holds this node's set
          } else {
            W.h[j].complete = 0;
          }
        }
        __syncwarp();
        if (n < 0) return -1;
      }
      if (n == 0) return 0;  // an empty set: no leaves
      if (lane == 0) {
        W.tn[u] = n;
        W.tanc[u] = (int8_t)anc;
      }
      __syncwarp();
    }
    const long long s0 = tail_size(s, t, 0), s1 = tail_size(s, t, 1);
    const bool e01 = !LAB || P.label[s + 1] == P.label[s + 2];
    if (t == 2) return s0 * s1 - (e01 ? tail_common(s, t, 3u) : 0);
    const long long s2 = tail_size(s, t, 2);
    long long c = s0 * s1 * s2;
    const bool e02 = !LAB || P.label[s + 1] == P.label[s + 3];
    const bool e12 = !LAB || P.label[s + 2] == P.label[s + 3];
    if (e01) c -= tail_common(s, t, 3u) * s2;
    if (e02) c -= tail_common(s, t, 5u) * s1;
    if (e12) c -= tail_common(s, t, 6u) * s0;
    if (e01 && e02) c += 2ll * tail_common(s, t, 7u);
    return c;
  }

  // Base set u of the tail rooted at level s (t sets): buffer and size.
  __device__ __forceinline__ const int32_t *tail_base(int s, int t, int u) {
    return u == t - 1 ? fbuf() : buf(s + 1 + u);
  }
  // Does base u hold phi(m) for this lane's m (m <= s)?  Such a value is not
  // in the node's set when m lies after the base's anchor.
  __device__ __forceinline__ bool tail_holds(int s, int t, int u) {
    if (!LAB || lane > s) return false;  // unlabeled bases are built per node
    const int32_t *B = tail_base(s, t, u);
    const int32_t nb = W.tn[u], x = W.phi[lane];
    const int32_t q = lower_bound(B, 0, nb, x);
    return q < nb && B[q] == x;
  }
  __device__ long long tail_size(int s, int t, int u) {
    const bool lost = lane > W.tanc[u] && tail_holds(s, t, u);
    return (long long)W.tn[u] - __popc(__ballot_sync(kFull, lost));
  }
  // |intersection of the node's sets in `mask`| (bits of u; two or three sets)
  __device__ long long tail_common(int s, int t, unsigned mask) {
    const int u = __ffs(mask) - 1, v = __ffs(mask & (mask - 1)) - 1;
    const int w = mask == 7u ? 2 : -1;
    long long c = common_count(tail_base(s, t, u), W.tn[u], tail_base(s, t, v), W.tn[v],
                               w >= 0 ? tail_base(s, t, w) : nullptr, w >= 0 ? W.tn[w] : 0);
    if (LAB) {
      int after = max((int)W.tanc[u], (int)W.tanc[v]);
      if (w >= 0) after = max(after, (int)W.tanc[w]);
      const bool lost = lane > after && tail_holds(s, t, u) && tail_holds(s, t, v) && (w < 0 || tail_holds(s, t, w));
      c -= __popc(__ballot_sync(kFull, lost));
    }
    return c;
  }

  // Conditions of the last vertex i on the vertices between F's anchor and
  // its parent, (anchor, i-2], for the current prefix: a lower and an upper
  // bound (unlabeled symmetry conditions) and the values it must differ from
  // (W.xneq[0..n)).  F was built without them; they are applied per count.
  struct Extra {
    int32_t lo, hi;
    int n;
  };

  __device__ Extra extra_conds(int i) {
    const int a = W.fanchor;
    int32_t lo = -1, hi = INT_MAX, v = 0;
    bool isneq = false;
    if (lane > a && lane <= i - 2) {
      v = W.phi[lane];
      if (LAB) {
        isneq = true;
      } else if (P.larger[i] >> lane & 1) {
        lo = v;
      } else if (P.less[i] >> lane & 1) {
        hi = v;
      } else {
        isneq = true;
      }
    }
    Extra X;
    X.lo = (int32_t)__reduce_max_sync(kFull, (unsigned)(lo + 1)) - 1;
    X.hi = (int32_t)__reduce_min_sync(kFull, (unsigned)hi);
    const unsigned m = __ballot_sync(kFull, isneq);
    if (isneq) W.xneq[__popc(m & lanemask_lt())] = v;
    X.n = __popc(m);
    __syncwarp();
    return X;
  }

  __device__ __forceinline__ bool extra_ok(const Extra &X, int32_t y) const {
    if (y <= X.lo || y >= X.hi) return false;
    for (int t = 0; t < X.n; ++t)
      if (W.xneq[t] == y) return false;
    return true;
  }

  __device__ __forceinline__ bool in_fixed(int32_t y) {
    const int32_t *F = fbuf();
    const int32_t q = lower_bound(F, 0, W.fn, y);
    return q < W.fn && F[q] == y;
  }

  __device__ unsigned long long count_fixed(int i) {
    const int32_t x = W.phi[i - 1];
    if (W.fn == 0) return 0;
    const Extra X = extra_conds(i);
    int64_t b = 0, e = 0;
    if (lane == 0) row_for(x, i, b, e);
    b = __shfl_sync(kFull, b, 0);
    e = __shfl_sync(kFull, e, 0);
    return count_fixed_list(i, x, b, e, X);
  }

  // The condition between the last vertex i and its parent: 1 = y > x,
  // 2 = y < x, 0 = y != x.
  __device__ __forceinline__ int parent_rel(int i) const {
    return LAB ? 0 : (P.larger[i] >> (i - 1) & 1) ? 1 : (P.less[i] >> (i - 1) & 1) ? 2 : 0;
  }

  // Last level over a batch of b siblings (items[0..b), b <= 32) that share
  // the fixed set F, in one flattened warp-wide pass: the siblings' adjacency
  // lists are laid end to end (an exclusive scan of their lengths) and lane t
  // takes positions t, t + 32, ... of that sequence, kFlatUnroll positions at
  // once, so the loads are coalesced within each list and several rounds of
  // them are in flight together -- one pass over the batch instead of a
  // dependent rowptr -> list -> search chain per sibling.  Lists longer than
  // max(cfg.lane_list, 4 |F|) (hubs) are counted one by one afterwards by
  // count_fixed_list, which searches F's elements in them instead.
  __device__ unsigned long long count_fixed_flat(int i, const int32_t *items, int b) {
    const int32_t *F = fbuf();
    const int32_t nF = W.fn;
    if (nF == 0) return 0;
    const int rel = parent_rel(i);
    const Extra X = extra_conds(i);
    const bool mine = lane < b && item_ok(i - 1, items[lane]);
    const int32_t x = mine ? items[lane] : 0;
    int64_t rb = 0, re = 0;
    if (mine) row_for(x, i, rb, re);
    const int64_t lim = cfg.lane_list > 4 * nF ? (int64_t)cfg.lane_list : 4ll * nF;
    const bool flat = mine && re - rb <= lim;
    const int32_t len = flat ? (int32_t)(re - rb) : 0;
    int32_t incl = len;
#pragma unroll
    for (int s = 1; s < 32; s <<= 1) {
      const int32_t t = __shfl_up_sync(kFull, incl, s);
      if (lane >= s) incl += t;
    }
    const int32_t off = incl - len;  // exclusive prefix: first position of this lane's list
    const int32_t total = __shfl_sync(kFull, incl, 31);
    unsigned c = 0;
    for (int32_t base = 0; base < total; base += 32 * kFlatUnroll) {
      work += kFlatUnroll;
      int32_t y[kFlatUnroll], xo[kFlatUnroll];
      bool v[kFlatUnroll];
#pragma unroll
      for (int u = 0; u < kFlatUnroll; ++u) {
        const int32_t pos = base + u * 32 + lane;
        // owner: the last sibling whose list starts at or before pos
        int j = 0;
#pragma unroll
        for (int s = 16; s >= 1; s >>= 1) {
          const int32_t oc = __shfl_sync(kFull, off, j + s);
          if (oc <= pos) j += s;
        }
        const int32_t oj = __shfl_sync(kFull, off, j);
        const int64_t bj = __shfl_sync(kFull, rb, j);
        xo[u] = __shfl_sync(kFull, x, j);
        v[u] = pos < total;
        y[u] = v[u] ? lbase()[bj + (pos - oj)] : 0;
      }
#pragma unroll
      for (int u = 0; u < kFlatUnroll; ++u) {
        const int32_t yy = y[u], xx = xo[u];
        if (v[u] && (rel == 1 ? yy > xx : rel == 2 ? yy < xx : yy != xx) && extra_ok(X, yy)) {
          const int32_t q = lower_bound(F, 0, nF, yy);
          c += q < nF && F[q] == yy;
        }
      }
    }
    unsigned long long sum = __reduce_add_sync(kFull, c);
    unsigned rest = __ballot_sync(kFull, mine && !flat);
    while (rest) {
      const int j = __ffs(rest) - 1;
      rest &= rest - 1;
      sum += count_fixed_list(i, __shfl_sync(kFull, x, j), __shfl_sync(kFull, rb, j), __shfl_sync(kFull, re, j), X);
    }
    return sum;
  }

  // The last vertex i when its parent (vertex i-1) is not one of its backward
  // neighbours: its candidate set is F (built once per anchor-level node by
  // build_fixed) cut by the conditions on the vertices after the anchor --
  // the fixed ones between the anchor and the parent (extra_conds) and the
  // parent's own (y > x, y < x, or y != x: unlabeled symmetry conditions, or
  // injectivity when labeled).  F is sorted, so sibling x counts a range of
  // F by two binary searches in shared memory, less the excluded values that
  // fall in it; lane j takes sibling j.
  // Last vertex i whose one backward neighbour is its parent, on a labeled
  // plan reading label segments: sibling x's candidates are the label-L(i)
  // segment of N(x) minus the prefix vertices, so each sibling's count is a
  // segment length and a few searches (count_single_batch).
  __device__ bool single_applies(int i) {
    return LAB && segmented() && i >= 3 && P.nbn[i] == 1 && P.bn[i][0] == i - 1;
  }

  // Lane t counts sibling t of the batch: the length of the label-L(i)
  // segment of N(x), minus the vertices of phi(0..i-2) and x itself (the
  // values the labeled DFS excludes) that carry that label and are found in
  // the segment by binary search.
  __device__ unsigned long long count_single_batch(int i, const int32_t *items, int b) {
    unsigned c = 0;
    if (lane < b && item_ok(i - 1, items[lane])) {
      const int32_t x = items[lane];
      int64_t rb, re;
      row_for(x, i, rb, re);
      const int32_t *L = lbase() + rb;
      const int32_t len = (int32_t)(re - rb);
      int32_t cnt = len;
      for (int j = 0; j < i; ++j) {
        const int32_t v = j < i - 1 ? W.phi[j] : x;
        if ((int32_t)G.label[v] != P.label[i]) continue;  // not in this segment
        const int32_t q = lower_bound(L, 0, len, v);
        if (q < len && L[q] == v) --cnt;
      }
      c = (unsigned)cnt;
    }
    return __reduce_add_sync(kFull, c);
  }

  __device__ bool free_applies(int i) {
    if (!cfg.fixed || i < 3) return false;
    for (int t = 0; t < P.nbn[i]; ++t)
      if (P.bn[i][t] == i - 1) return false;
    return true;
  }

  __device__ unsigned long long count_free_batch(int i, const int32_t *items, int b) {
    const int32_t *F = fbuf();
    const int32_t nF = W.fn;
    if (nF == 0) return 0;
    const int rel = parent_rel(i);
    const Extra X = extra_conds(i);
    unsigned c = 0;
    if (lane < b && item_ok(i - 1, items[lane])) {
      const int32_t x = items[lane];
      int32_t lo = X.lo, hi = X.hi;  // candidates lie strictly between
      if (rel == 1) lo = max(lo, x);
      else if (rel == 2) hi = min(hi, x);
      int32_t cnt = 0;
      if (lo < hi) {
        cnt = max(0, lower_bound(F, 0, nF, hi) - upper_bound_smem(F, nF, lo));
        for (int t = 0; t < X.n; ++t) {
          const int32_t e = W.xneq[t];
          if (e > lo && e < hi && in_fixed(e)) --cnt;
        }
        if (rel == 0 && x > lo && x < hi && in_fixed(x)) --cnt;
      }
      c = (unsigned)cnt;
    }
    return __reduce_add_sync(kFull, c);
  }

  // |F ∩ N(x)| under the parent condition, the warp together; N(x) is
  // colidx[b, e).
  __device__ unsigned long long count_fixed_list(int i, int32_t x, int64_t b, int64_t e, const Extra &X) {
    const int32_t *F = fbuf();
    const int32_t nF = W.fn;
    const int32_t *L = lbase() + b;
    const int32_t len = (int32_t)(e - b);
    const int rel = parent_rel(i);
    unsigned long long c = 0;
    if ((int64_t)len <= 4ll * nF) {
      // scan N(x) (coalesced), look each y up in F (shared memory)
      int32_t start = 0;
      if (rel == 1 && len > 64) start = warp_upper_bound(L, 0, len, x);
      for (int32_t pos = start; pos < len; pos += 32) {
        ++work;
        const int32_t idx = pos + lane;
        const bool valid = idx < len;
        const int32_t y = valid ? L[idx] : 0;
        bool ok = valid && (rel == 1 ? y > x : rel == 2 ? y < x : y != x) && extra_ok(X, y);
        if (ok) {
          const int32_t q = lower_bound(F, 0, nF, y);
          ok = q < nF && F[q] == y;
        }
        c += __popc(__ballot_sync(kFull, ok));
      }
    } else {
      // scan F, search each y in N(x) from a monotone cursor
      int32_t start = rel == 1 ? upper_bound_smem(F, nF, x) : 0;
      int32_t curp = 0;
      for (int32_t pos = start; pos < nF; pos += 32) {
        ++work;
        const int32_t idx = pos + lane;
        const bool valid = idx < nF;
        const int32_t y = valid ? F[idx] : 0;
        bool ok = valid && (rel == 1 ? y > x : rel == 2 ? y < x : y != x) && extra_ok(X, y);
        const bool searched = ok;
        int32_t p = 0;
        if (ok) {
          p = lower_bound(L, curp, len, y);
          ok = p < len && L[p] == y;
        }
        curp = max(curp, (int32_t)__reduce_max_sync(kFull, searched ? (unsigned)p : 0u));
        c += __popc(__ballot_sync(kFull, ok));
      }
    }
    return c;
  }

  __device__ __forceinline__ int32_t upper_bound_smem(const int32_t *a, int32_t n, int32_t x) {
    int32_t lo = 0, hi = n;
    while (lo < hi) {
      const int32_t mid = (lo + hi) >> 1;
      if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
  }

  __device__ unsigned long long count_last(int i) {
    if (W.lastmode == 1) {
      if (W.fvalid == 0) build_fixed(i);
      if (W.fvalid == 1) return count_fixed(i);
    }
    setup(i, true);
    const LevelHdr &H = W.h[i];
    const int32_t *src = H.src;
    const int32_t send = H.send;
    int32_t spos = H.spos;
    if (!LAB && H.nm == 0 && H.hi == INT_MAX) {
      // closed form: everything above the bound except the excluded vertices
      int32_t hit = 0;
      if (lane < H.nneq) {
        const int32_t v = H.neqv[lane];
        bool dup = false;  // equal excluded vertices are excluded once
        for (int t = 0; t < lane; ++t) dup |= H.neqv[t] == v;
        if (v > H.lo && !dup) {
          const int32_t q = lower_bound(src, spos, send, v);
          hit = q < send && src[q] == v;
        }
      }
      const int32_t excl = __popc(__ballot_sync(kFull, hit));
      return (unsigned long long)(send - spos - excl);
    }
    int32_t cur[kMaxLists];
#pragma unroll
    for (int m = 0; m < kMaxLists; ++m) cur[m] = m < H.nm ? H.mcur[m] : 0;
    unsigned long long c = 0;
    for (; spos < send; spos += 32) {
      ++work;
      const int32_t idx = spos + lane;
      const bool valid = idx < send;
      const int32_t x = valid ? src[idx] : 0;
      const bool st0 = H.nm > 0 && (H.merge_mask & 1u);
      Window w0 = {0, 0};
      if (st0) w0 = stage_window(H.mlist[0], H.mlen[0], cur[0], win, cfg.window, lbase());
      bool ok = valid && pass_filter<LAB>(x, H, i, P, G, segmented());
      ok = test_lists(ok, x, H, cur, win, cfg.window, lbase(), st0, w0);
      c += __popc(__ballot_sync(kFull, ok));
    }
    return c;
  }

  // Claim up to 32 consecutive buffered candidates of stored level l (one
  // CAS): all of them while no warp is hungry, else at most half of what is
  // left, so that the other half stays stealable.  Returns the first index
  // and sets *b to how many (0 when none).
  __device__ int32_t claim_batch(int l, int *b) {
    int32_t r = -1, got = 0;
    if (lane == 0) {
      const bool share = cfg.steal && W.hungry_seen > 0;
      unsigned long long w = *(volatile unsigned long long *)&W.word[l];
      for (int tries = 0;; ++tries) {
        const uint32_t it = (uint32_t)(w >> 16) & 0xffffu, n = (uint32_t)w & 0xffffu;
        if (it >= n) break;
        if (tries >= kCasLimit) {
          raise_error(ctl, TDFS_ERR_TIMEOUT);
          break;
        }
        // leaving half only helps while what is left can still be stolen
        const bool half = share && n - it >= 2u * (uint32_t)cfg.leaf_min;
        const uint32_t take = min(32u, half ? max(1u, (n - it) / 2) : n - it);
        const unsigned long long old = atomicCAS(&W.word[l], w, w + ((unsigned long long)take << 16));
        if (old == w) {
          r = (int32_t)it;
          got = (int)take;
          break;
        }
        w = old;
      }
    }
    *b = __shfl_sync(kFull, got, 0);
    return __shfl_sync(kFull, r, 0);
  }

  // Claim the next buffered candidate of stored level l; -1 when none.
  __device__ int32_t claim(int l) {
    int32_t r = -1;
    if (lane == 0) {
      unsigned long long w = *(volatile unsigned long long *)&W.word[l];
      int tries = 0;
      for (;; ++tries) {
        const uint32_t it = (uint32_t)(w >> 16) & 0xffffu, n = (uint32_t)w & 0xffffu;
        if (it >= n) break;
        if (tries >= kCasLimit) {
          raise_error(ctl, TDFS_ERR_TIMEOUT);
          break;
        }
        const unsigned long long old = atomicCAS(&W.word[l], w, w + (1ull << 16));
        if (old == w) {
          r = (int32_t)it;
          break;
        }
        w = old;
      }
    }
    return __shfl_sync(kFull, r, 0);
  }

  // ---- query slots ----------------------------------------------------------

  __device__ __forceinline__ unsigned long long now_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
  }

  // Copy slot s's plan into this warp's shared memory (all lanes).
  __device__ void load_plan(int s) {
    if (W.slot == s) return;
    __syncwarp();
    // the host may have written this slot while the kernel runs (serving):
    // read it through L2 (ld.cg), never from a stale L1 line
    const int32_t *srcw = reinterpret_cast<const int32_t *>(&tab->plan[s]);
    int32_t *dstw = reinterpret_cast<int32_t *>(&W.plan);
    for (int t = lane; t < (int)(sizeof(DevPlan) / 4); t += 32) dstw[t] = __ldcg(srcw + t);
    if (lane == 0) W.slot = s;
    __syncwarp();
    derive_plan();
  }

  // Give up this warp's hold on slot s (lane 0).  Its count is added first;
  // the warp that drops the last hold after the tickets ran out completes the
  // slot, exactly once (CAS on the state).
  __device__ void release_lane0(int s) {
    SlotHot &h = tab->hot[s];
    if (count) {
      atomicAdd(&h.count, count);
      count = 0;
    }
    __threadfence();
    const int old = atomicSub(&h.holders, 1);
    if (old == 1) {
      const unsigned long long t = *(volatile unsigned long long *)&h.ticket;
      if ((long long)t >= __ldcg(&tab->info[s].ntickets) &&
          atomicCAS(&h.state, kSlotActive, kSlotDone) == kSlotActive) {
        h.t_done = now_ns();
        __threadfence();
        atomicAdd(&tab->ctl.completed, 1ull);
      }
    }
  }

  // Level-0 chunk t of slot s: up to 32 directed edges (the slot's chunk
  // size), filtered as get_job
  // (src/gpu_match.cu:531-556), published as level-1 items (pairs phi(0),
  // phi(1)).  Returns false when no edge of the chunk passes the filter.
  __device__ bool fetch_chunk(int s, long long t) {
    const SlotInfo &in = tab->info[s];
    const int chunk = __ldcg(&in.chunk);
    const int64_t e0 = __ldcg(&in.e_begin) + (t * __ldcg(&in.stride) + __ldcg(&in.phase)) * (int64_t)chunk;
    const int64_t e = e0 + lane;
    bool ok = lane < chunk && e < __ldcg(&in.e_end);
    int32_t r = 0, c = 0;
    if (ok) {
      // labeled plans may walk the label index: positions map to edge ids
      const int64_t ed = __ldcg(&in.perm) ? (int64_t)G.lperm[e] : e;
      r = G.src[ed];
      c = G.colidx[ed];
      if (!LAB && P.orient && !(r < c)) ok = false;
      if (LAB && ok && ((int32_t)G.label[r] != P.label[0] || (int32_t)G.label[c] != P.label[1])) ok = false;
      if (ok && (deg(r) < P.deg[0] || deg(c) < P.deg[1] || G.maxnd[c] < P.deg[2])) ok = false;
    }
    const unsigned mask = __ballot_sync(kFull, ok);
    if (ok) {
      const int slot = __popc(mask & lanemask_lt());
      W.er[slot] = r;
      W.ec[slot] = c;
    }
    __syncwarp();
    if (!mask) return false;
    if (lane == 0) {
      W.fvalid = 0;
      W.t_base = now_ns();
      for (int j = 2; j < kMaxK; ++j) W.h[j].complete = W.h[j].core = 0;
      publish(1, __popc(mask));
    }
    __syncwarp();
    return true;
  }

  // Take level-0 tickets from open slots until a chunk yields edges.  On
  // success this warp holds the slot; false when no slot has tickets left.
  __device__ bool take_tickets() {
    SlotCtl &C = tab->ctl;
    for (;;) {
      int s = -1;
      long long t = 0;
      if (lane == 0) {
        const unsigned long long adm = *(volatile unsigned long long *)&C.admitted;
        unsigned long long lo = *(volatile unsigned long long *)&C.first_open;
        for (unsigned long long q = lo; q < adm && s < 0; ++q) {
          SlotHot &h = tab->hot[q];
          const long long nt = __ldcg(&tab->info[q].ntickets);
          if ((long long)*(volatile unsigned long long *)&h.ticket >= nt) {
            if (q == lo) {  // advance the hint past exhausted slots
              atomicMax(&C.first_open, q + 1);
              lo = q + 1;
            }
            continue;
          }
          atomicAdd(&h.holders, 1);  // hold before taking: completion needs holders == 0
          const unsigned long long tk = atomicAdd(&h.ticket, 1ull);
          if ((long long)tk < nt) {
            if (tk == 0) atomicCAS(&h.t_first, 0ull, now_ns());
            s = (int)q;
            t = (long long)tk;
          } else {
            release_lane0((int)q);  // nothing to flush: this warp holds no work
          }
        }
      }
      s = __shfl_sync(kFull, s, 0);
      t = __shfl_sync(kFull, t, 0);
      if (s < 0) return false;
      load_plan(s);
      // keep taking tickets of this slot until a chunk yields edges
      for (;;) {
        if (fetch_chunk(s, t)) return true;
        long long nt = 0;
        if (lane == 0) {
          const unsigned long long tk = atomicAdd(&tab->hot[s].ticket, 1ull);
          nt = (long long)tk < __ldcg(&tab->info[s].ntickets) ? (long long)tk : -1;
          if (nt < 0) release_lane0(s);
        }
        nt = __shfl_sync(kFull, nt, 0);
        if (nt < 0) break;  // this slot is spent: look at the others
        t = nt;
      }
    }
  }

  // A warp that holds slot W.slot and has finished its subtree keeps the hold
  // and takes the slot's next level-0 ticket directly: one atomic per ticket
  // instead of a release, a new hold and a take on the slot's lines.  Returns
  // false when the slot has no tickets left; the hold is then dropped (and
  // the count flushed).
  __device__ bool next_ticket_same_slot() {
    const int s = W.slot;
    for (;;) {
      long long t = -1;
      if (lane == 0) {
        const unsigned long long tk = atomicAdd(&tab->hot[s].ticket, 1ull);
        t = (long long)tk < __ldcg(&tab->info[s].ntickets) ? (long long)tk : -1;
        if (t < 0) release_lane0(s);
      }
      t = __shfl_sync(kFull, t, 0);
      if (t < 0) return false;
      if (fetch_chunk(s, t)) return true;
    }
  }

  // New batch of `n` items at level l (1 = edge pairs, >= 2 candidates).
  __device__ __forceinline__ void publish(int l, int n) {
    const unsigned long long gen = (W.word[l] >> 32) + 1;
    __threadfence_block();
    atomicExch(&W.word[l], (gen << 32) | (unsigned long long)n);
  }

  // ---- work stealing and the global split queue ---------------------------

  __device__ __forceinline__ WarpSmem &warp_at(int v) {
    return *reinterpret_cast<WarpSmem *>(cta + (size_t)v * cfg.warp_bytes);
  }
  __device__ __forceinline__ int32_t *buf_of(int v, int l) {
    return reinterpret_cast<int32_t *>(cta + (size_t)v * cfg.warp_bytes + hdr_bytes) + cfg.window +
           (cfg.fixed ? cfg.cap : 0) +
           (l - 2) * cfg.cap;
  }

  // Make `cnt` items of level l (already in this warp's level-l storage,
  // prefix already in W.phi, plan in W.plan) this warp's new base subtree.
  __device__ void install(int l, int cnt) {
    if (lane == 0) {
      W.fvalid = 0;
      W.t_base = now_ns();
      for (int j = 2; j < kMaxK; ++j) W.h[j].complete = W.h[j].core = 0;
      if (l >= 2) {
        W.h[l].spos = W.h[l].send = 0;  // no source left: only the given candidates
        W.h[l].nprod = cnt;
      }
      publish(l, cnt);
    }
    __syncwarp();
  }

  // How long a warp's base subtree must have run before others may split it:
  // cfg.split_after_ns normally (small subtrees finish where they started),
  // cfg.rush_ns once at least cfg.rush_hungry warps of the grid are idle --
  // the tail of a launch, where a few large subtrees hold all the work left
  // and every split is worth more than it costs.
  __device__ __forceinline__ unsigned long long split_gate() {
    if (cfg.rush_hungry > 0 && *(volatile int32_t *)&ctl->hungry >= cfg.rush_hungry)
      return (unsigned long long)cfg.rush_ns;
    return (unsigned long long)cfg.split_after_ns;
  }

  // Steal half of the remaining items at the shallowest level of another
  // warp of this CTA.  The thief copies the victim's plan, prefix and the
  // upper half of its items, takes a hold on the victim's slot, then CASes
  // the victim's word (gen | next | end) down to the split point.  The copy is
  // valid iff the CAS succeeds: a warp rewrites its items, prefix, plan or
  // slot only after bumping gen.  Returns the level (1 = edge pairs) or 0.
  __device__ int steal_local(int nwarps, int me, int min_items) {
    // one pass: lane v scans warp v's levels and offers its shallowest level
    // with at least min_items items; the warp takes the shallowest offer,
    // the largest one on ties
    unsigned long long key = 0;
    const unsigned long long now = now_ns();
    const unsigned long long gate = split_gate();
    if (lane < nwarps && lane != me && now - *(volatile const unsigned long long *)&warp_at(lane).t_base >= gate) {
      const WarpSmem &V = warp_at(lane);
      const int vk = *(volatile const int32_t *)&V.plan.k;
      for (int l = 1; l <= kMaxK - 2; ++l) {
        const unsigned long long w = *(volatile const unsigned long long *)&V.word[l];
        const int rem = (int)((uint32_t)w & 0xffffu) - (int)((uint32_t)(w >> 16) & 0xffffu);
        if (rem >= (l >= 2 && l == vk - 2 ? max(min_items, cfg.leaf_min) : min_items)) {
          key = ((unsigned long long)(kMaxK - l) << 40) | ((unsigned long long)rem << 8) | (unsigned)lane;
          break;
        }
      }
    }
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
      const unsigned long long o = __shfl_xor_sync(kFull, key, s);
      key = o > key ? o : key;
    }
    if (!key) return 0;
    const int l = kMaxK - (int)(key >> 40);
    const int vic = (int)(key & 0xff);
    WarpSmem &V = warp_at(vic);
    unsigned long long w = 0;
    if (lane == 0) w = *(volatile unsigned long long *)&V.word[l];
    w = __shfl_sync(kFull, w, 0);
    __threadfence_block();
    const int it = (int)((uint32_t)(w >> 16) & 0xffffu), n = (int)((uint32_t)w & 0xffffu);
    const int vk = *(volatile const int32_t *)&V.plan.k;
    if (n - it < (l >= 2 && l == vk - 2 ? max(min_items, cfg.leaf_min) : min_items)) return 0;
    const int vslot = *(volatile int32_t *)&V.slot;
    if (vslot < 0) return 0;
    const int take = (n - it) / 2;
    const int from = n - take;
    {  // plan
      const volatile int32_t *sp = reinterpret_cast<const volatile int32_t *>(&V.plan);
      int32_t *dp = reinterpret_cast<int32_t *>(&W.plan);
      for (int t = lane; t < (int)(sizeof(DevPlan) / 4); t += 32) dp[t] = sp[t];
    }
    if (l == 1) {
      if (lane < take) {
        W.er[lane] = ((volatile int32_t *)V.er)[from + lane];
        W.ec[lane] = ((volatile int32_t *)V.ec)[from + lane];
      }
    } else {
      const volatile int32_t *vb = buf_of(vic, l);
      int32_t *mb = buf(l);
      for (int t = lane; t < take; t += 32) mb[t] = vb[from + t];
      if (lane < l) W.phi[lane] = ((volatile int32_t *)V.phi)[lane];
    }
    __threadfence_block();
    __syncwarp();
    int won = 0;
    if (lane == 0) {
      atomicAdd(&tab->hot[vslot].holders, 1);
      won = atomicCAS(&V.word[l], w, (w & ~0xffffull) | (unsigned long long)from) == w;
      if (won) {
        // the victim's largest grain was just halved: it cools down for a
        // full gate before it can be split again
        *(volatile unsigned long long *)&V.t_base = now_ns();
        W.slot = vslot;
      } else {
        release_lane0(vslot);  // nothing to flush: this warp holds no work
        W.slot = -1;           // the plan copy above overwrote the old one
      }
    }
    won = __shfl_sync(kFull, won, 0);
    __syncwarp();
    if (!won) return 0;
    derive_plan();  // the plan came from the victim
    install(l, take);
    if (lane == 0) atomicAdd(&ctl->steals, 1ull);
    return l;
  }

  // Bounded MPMC ring with per-slot sequence numbers (lane 0 only).  A slot
  // is reserved before its unit is written, so a donation can never be left
  // without a place; consumers skip units with no items.
  __device__ long long queue_reserve() {
    unsigned long long pos = *(volatile unsigned long long *)&qh->tail;
    for (int tries = 0; tries < 64; ++tries) {
      const unsigned long long seq = *(volatile unsigned long long *)&qh->seq[pos & (kQueueCap - 1)];
      const long long dif = (long long)(seq - pos);
      if (dif == 0) {
        const unsigned long long old = atomicCAS(&qh->tail, pos, pos + 1);
        if (old == pos) return (long long)pos;
        pos = old;
      } else if (dif < 0) {
        return -1;  // full
      } else {
        pos = *(volatile unsigned long long *)&qh->tail;
      }
    }
    return -1;
  }

  // Write a unit: slot, level l, prefix W.phi[0..l-1], items [from, from+cnt)
  // of level l (pairs when l == 1).  A unit with items carries one hold on
  // its slot.
  __device__ void queue_publish(unsigned long long pos, int l, int from, int cnt) {
    SplitUnit &u = units[pos & (kQueueCap - 1)];
    u.level = l;
    u.nitems = cnt;
    u.slot = W.slot;
    if (l == 1) {
      for (int t = 0; t < cnt; ++t) {
        u.items[2 * t] = W.er[from + t];
        u.items[2 * t + 1] = W.ec[from + t];
      }
    } else {
      for (int j = 0; j < l; ++j) u.phi[j] = W.phi[j];
      const int32_t *b = buf(l);
      for (int t = 0; t < cnt; ++t) u.items[t] = b[from + t];
    }
    __threadfence();
    atomicExch(&qh->seq[pos & (kQueueCap - 1)], pos + 1);
  }

  // Pop one unit into this warp's state; returns its level or 0.  The
  // unit's hold on its slot passes to this warp.
  __device__ int queue_pop() {
    int l = 0, cnt = 0, us = -1;
    if (lane == 0) {
      unsigned long long pos = *(volatile unsigned long long *)&qh->head;
      for (int tries = 0; tries < 64; ++tries) {
        const unsigned long long slot = pos & (kQueueCap - 1);
        const unsigned long long seq = *(volatile unsigned long long *)&qh->seq[slot];
        const long long dif = (long long)(seq - (pos + 1));
        if (dif == 0) {
          const unsigned long long old = atomicCAS(&qh->head, pos, pos + 1);
          if (old == pos) {
            __threadfence();
            const volatile SplitUnit &u = units[slot];
            l = u.level;
            cnt = u.nitems;
            us = u.slot;
            if (us < 0 || cnt <= 0 || l < 1 || l > kMaxK - 2 || (l == 1 ? 2 * cnt : cnt) > kUnitItems) {
              l = 0;  // an empty reservation (it carries no hold)
            } else if (l == 1) {
              for (int t = 0; t < cnt; ++t) {
                W.er[t] = u.items[2 * t];
                W.ec[t] = u.items[2 * t + 1];
              }
            } else {
              for (int j = 0; j < l; ++j) W.phi[j] = u.phi[j];
              int32_t *mb = buf(l);  // buffer placement does not depend on the plan
              for (int t = 0; t < cnt; ++t) mb[t] = u.items[t];
            }
            __threadfence();
            atomicExch(&qh->seq[slot], pos + kQueueCap);
            break;
          }
          pos = old;
        } else if (dif < 0) {
          break;  // empty
        } else {
          pos = *(volatile unsigned long long *)&qh->head;
        }
      }
    }
    l = __shfl_sync(kFull, l, 0);
    cnt = __shfl_sync(kFull, cnt, 0);
    us = __shfl_sync(kFull, us, 0);
    __syncwarp();
    if (!l) return 0;
    load_plan(us);
    install(l, cnt);
    return l;
  }

  // Busy warp: when some warp is hungry, move up to a unit's worth of the
  // shallowest remaining items into the global ring.
  __device__ void maybe_donate(int level) {
    int hungry = 0;
    if (lane == 0) {
      // the one read of the grid-wide idle count on the busy path, every few
      // claims; claim_batch works from this copy
      W.hungry_seen = *(volatile int32_t *)&ctl->hungry;
      if (now_ns() - W.t_base >= 4ull * split_gate()) hungry = W.hungry_seen;
    }
    hungry = __shfl_sync(kFull, hungry, 0);
    if (hungry <= 0) return;
    if (lane == 0) {
      int l = 1;
      for (; l <= level; ++l) {
        const unsigned long long w = *(volatile unsigned long long *)&W.word[l];
        const int rem = (int)((uint32_t)w & 0xffffu) - (int)((uint32_t)(w >> 16) & 0xffffu);
        if (rem >= (l >= 2 && l == P.k - 2 ? max(2, cfg.leaf_min) : 2)) break;
      }
      if (l <= level) {
        const long long pos = queue_reserve();
        if (pos >= 0) {
          const int maxtake = l == 1 ? kUnitItems / 2 : kUnitItems;
          int cnt = 0, from = 0;
          unsigned long long w = *(volatile unsigned long long *)&W.word[l];
          for (int t = 0; t < kCasLimit; ++t) {
            const int it = (int)((uint32_t)(w >> 16) & 0xffffu), n = (int)((uint32_t)w & 0xffffu);
            if (n - it < 2) break;
            const int take = min((n - it) / 2, maxtake);
            const unsigned long long old =
                atomicCAS(&W.word[l], w, (w & ~0xffffull) | (unsigned long long)(n - take));
            if (old == w) {
              cnt = take;
              from = n - take;
              break;
            }
            w = old;
          }
          if (cnt) atomicAdd(&tab->hot[W.slot].holders, 1);  // the unit's hold
          queue_publish((unsigned long long)pos, l, from, cnt);
          if (cnt) atomicAdd(&ctl->splits, 1ull);
        }
      }
    }
    __syncwarp();
  }

  // ---- work budget (budgeted launches) -------------------------------------
  // Every warp counts work units (one per claim and per 32-wide scan step) and
  // adds them to its slot's counter every few claims.  The flush that takes
  // the counter past the slot's budget marks the slot aborted and closes its
  // level-0 tickets; every warp holding work of an aborted slot drops it at
  // its next check, and the slot then completes through the usual holds with
  // `aborted` set (its count is not valid).  Returns true when the slot this
  // warp works on is aborted.
  __device__ bool over_budget() {
    int ab = 0;
    if (lane == 0 && W.slot >= 0) {
      const int s = W.slot;
      SlotHot &h = tab->hot[s];
      const long long budget = __ldcg(&tab->info[s].budget);
      if (budget > 0) {
        const unsigned long long tot = atomicAdd(&h.work, (unsigned long long)work) + work;
        if ((long long)tot > budget && atomicCAS(&h.aborted, 0, 1) == 0)
          atomicMax(&h.ticket, (unsigned long long)__ldcg(&tab->info[s].ntickets));
        ab = *(volatile int32_t *)&h.aborted;
      }
    }
    work = 0;
    return __shfl_sync(kFull, ab, 0) != 0;
  }

  // Drop the subtree this warp holds at levels base..level: every level word
  // gets a new generation with no items, so no thief can take them either.
  __device__ void abandon(int base, int level) {
    if (lane == 0)
      for (int l = base; l <= level; ++l) publish(l, 0);
    __syncwarp();
  }

  // ---- main loop ------------------------------------------------------------
  // level 1 iterates edge pairs, 2..k-2 iterate buffered candidates, the last
  // vertex k-1 is counted in place.  `base` is the shallowest level this warp
  // owns: below it the warp releases its slot and acquires new work (level-0
  // tickets of an open slot, a steal from its CTA, or a unit from the ring).
  __device__ void run(int nwarps, int me) {
    int level = 0, base = 1;
    if (lane == 0) W.t_start = now_ns();
    bool hungry = false;  // counted in ctl->hungry (warps polling for work)
    bool holding = false;
    unsigned claims = 0;
    if (lane == 0) {
      for (int l = 0; l < kStoredMax; ++l) W.word[l] = 0;
      for (int l = 0; l < kMaxK; ++l) W.h[l].complete = W.h[l].core = 0;
      W.slot = -1;
      W.fvalid = 0;
      W.t_base = 0;
      W.idle_since = W.idle_start = W.idle_total = 0;
      W.hungry_seen = 0;
    }
    __syncwarp();
    for (;;) {
      if (level < base) {
        // ---- the finished subtree: the next ticket of the same slot, else
        // release and acquire new work ----
        level = 0;
        if (holding) {
          holding = false;
          if (next_ticket_same_slot()) level = base = 1;
          __syncwarp();
        }
        if (!level && take_tickets()) level = base = 1;
        if (!level && cfg.steal) {
          // largest grains first: a big share of a CTA neighbour's level, a
          // split unit from the ring (work of other SMs), then any remainder
          int l = steal_local(nwarps, me, max(cfg.steal_first, cfg.steal_min));
          if (!l) {
            int nonempty = 0;
            if (lane == 0) {
              const unsigned long long h = *(volatile unsigned long long *)&qh->head;
              const unsigned long long t = *(volatile unsigned long long *)&qh->tail;
              nonempty = h < t;
            }
            if (__shfl_sync(kFull, nonempty, 0)) l = queue_pop();
          }
          if (!l && cfg.steal_min < cfg.steal_first) l = steal_local(nwarps, me, cfg.steal_min);
          if (l) level = base = l;
        }
        if (level) {
          holding = true;
          if (hungry && lane == 0) atomicSub(&ctl->hungry, 1);
          hungry = false;
          if (lane == 0) {
            W.idle_since = 0;
            if (W.idle_start) {
              W.idle_total += now_ns() - W.idle_start;
              W.idle_start = 0;
            }
          }
          nap = 256;
          continue;
        }
        // ---- idle: retire when every admitted slot is done and no more will
        // come, or -- without stealing -- as soon as admissions are closed and
        // no tickets are left (nothing else could reach this warp); otherwise
        // wait (bounded) for splits or admissions
        int done = 0;
        if (lane == 0) {
          if (!hungry && cfg.steal) atomicAdd(&ctl->hungry, 1);
          const SlotCtl &C = tab->ctl;
          const unsigned long long adm = *(volatile unsigned long long *)&C.admitted;
          const unsigned long long cmp = *(volatile unsigned long long *)&C.completed;
          const int shut = *(volatile int32_t *)&C.shutdown;
          if (shut && (cmp >= adm || !cfg.steal)) done = 1;
        }
        hungry = cfg.steal != 0;
        done = __shfl_sync(kFull, done, 0);
        if (done) break;
        if (!wait_for_work()) break;
        continue;
      }
      if (level >= 2 && level + 1 == P.k - 1) {
        // last stored level: batches of up to 32 siblings against the fixed
        // part of the last vertex's candidates (built once per grandparent)
        const int i = level + 1;
        const int lm = W.lastmode;
        // (mode 3 exists on labeled plans only: kept out of the unlabeled kernel)
        const int mode = lm == 2 ? 2 : (cfg.lane_list > 0 && (lm == 1 || (LAB && lm == 3))) ? lm : 0;
        if (mode) {
          if (mode != 3 && W.fvalid == 0) build_fixed(i);
          if (mode == 3 || W.fvalid == 1) {
            int b = 0;
            const int32_t first = claim_batch(level, &b);
            if (b > 0) {
              work += b;
              if (cfg.budgeted && ((++claims & 7u) == 0) && over_budget()) {
                abandon(base, level);
                level = base - 1;
                continue;
              }
              count += mode == 2           ? count_free_batch(i, buf(level) + first, b)
                       : (!LAB || mode == 1) ? count_fixed_flat(i, buf(level) + first, b)
                                             : count_single_batch(i, buf(level) + first, b);
              if (cfg.steal && (cfg.budgeted ? (claims & 7u) == 0 : (++claims & 7u) == 0)) maybe_donate(level);
              continue;
            }
          }
        }
      }
      const int32_t idx = claim(level);
      if (idx >= 0) {
        if (level == 1) {
          const int32_t r = W.er[idx], c = W.ec[idx];
          __syncwarp();
          if (lane == 0) {
            W.phi[0] = r;
            W.phi[1] = c;
          }
        } else {
          const int32_t x = buf(level)[idx];
          __syncwarp();
          if (!item_ok(level, x)) continue;  // a hoisted core value this prefix excludes
          if (lane == 0) W.phi[level] = x;
        }
        __syncwarp();
        ++work;
        if ((++claims & 7u) == 0) {
          if (cfg.budgeted && over_budget()) {
            abandon(base, level);
            level = base - 1;
            continue;
          }
          if (cfg.steal) maybe_donate(level);
        }
        if (level == W.tail) {
          const long long c = count_tail(level);
          if (c >= 0) {
            count += (unsigned long long)c;
            continue;
          }
        }
        if (level + 1 == P.k - 1) {
          count += count_last(P.k - 1);
        } else if (LAB && W.deadmask[level] && subtree_dead(level)) {
          continue;  // no leaf below this node
        } else {
          const int i = level + 1;
          const int a = hoist_anchor(i);
          stale_from(level);
          if (a >= 0 && (W.h[i].core || build_core(i, a))) {
            publish_core(i, a);
          } else {
            setup(i, true);
            produce(i);
          }
          ++level;
        }
        continue;
      }
      if (level >= 2 && W.h[level].spos < W.h[level].send) {
        produce(level);
        continue;
      }
      --level;
    }
    if (hungry && lane == 0) atomicSub(&ctl->hungry, 1);
    if (lane == 0) {
      const unsigned long long t = now_ns();
      if (W.idle_start) W.idle_total += t - W.idle_start;
      atomicAdd(&ctl->idle_ns, W.idle_total);
      atomicAdd(&ctl->warp_ns, t - W.t_start);
    }
    __syncwarp();
  }

  // Bounded idle wait between acquisition attempts: exponential back-off.
  // Returns false (retire) after too long without work: in a launch whose
  // admissions are closed that means a busy warp stalled and is reported as
  // a timeout; a serving launch simply retires and the host relaunches it.
  unsigned nap = 256;
  __device__ bool wait_for_work() {
    int ok = 1;
    if (lane == 0) {
      const unsigned long long t = now_ns();
      if (!W.idle_since) W.idle_since = t;
      if (!W.idle_start) W.idle_start = t;
      const SlotCtl &C = tab->ctl;
      const int shut = *(volatile int32_t *)&C.shutdown;
      // serving: the idle clock runs only while every admitted query is
      // complete -- a warp that retired while one query was still running
      // would leave the grid short for the queries admitted after it
      if (!shut && *(volatile unsigned long long *)&C.completed < *(volatile unsigned long long *)&C.admitted)
        W.idle_since = t;
      const unsigned long long limit_ms = shut ? (unsigned long long)cfg.idle_ms : (unsigned long long)C.idle_exit_ms;
      if (t - W.idle_since > limit_ms * 1000000ull) {
        if (shut) raise_error(ctl, TDFS_ERR_TIMEOUT);
        ok = 0;
      }
    }
    ok = __shfl_sync(kFull, ok, 0);
    if (ok) {
      __nanosleep(nap);
      nap = min(nap * 2, 8192u);
    }
    return ok;
  }
};

// Two register budgets of one kernel: MINB = 4 CTAs of 256 threads per SM
// caps it at 64 registers (with a few spills), MINB = 3 gives it 80 and no
// spills.  A launch whose shared memory already limits it to <= 3 CTAs per
// SM runs the 80-register build at no cost in occupancy.
template <bool LAB, int MINB>
__global__ void __launch_bounds__(256, MINB) match_kernel(const __grid_constant__ DevGraph G,
                                                    const __grid_constant__ KernelCfg cfg, RunCtl *ctl,
                                                    SlotTable *tab, SplitUnit *units, QueueHdr *qh) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int me = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  unsigned char *base = smem + (size_t)me * cfg.warp_bytes;
  WarpSmem &W = *reinterpret_cast<WarpSmem *>(base);
  const size_t hdr = (sizeof(WarpSmem) + 15) & ~(size_t)15;
  int32_t *win = reinterpret_cast<int32_t *>(base + hdr);
  int32_t *bufs = win + cfg.window + (cfg.fixed ? cfg.cap : 0);
  Engine<LAB> eng(G, cfg, ctl, tab, units, qh, W, bufs, win);
  eng.run(nwarps, me);
}

__global__ void init_kernel(RunCtl *ctl, QueueHdr *qh) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    ctl->hungry = 0;
    ctl->steals = 0;
    ctl->splits = 0;
    ctl->idle_ns = 0;
    ctl->warp_ns = 0;
    ctl->error = 0;
    qh->head = 0;
    qh->tail = 0;
  }
  for (int i = t; i < kQueueCap; i += gridDim.x * blockDim.x) qh->seq[i] = (unsigned long long)i;
}

}  // namespace

size_t warp_smem_bytes(int k, int cap, int window, bool fixed) {
  const size_t hdr = (sizeof(WarpSmem) + 15) & ~(size_t)15;
  const int stored = k > 3 ? k - 3 : 0;
  return hdr + sizeof(int32_t) * ((size_t)window + (size_t)(stored + (fixed ? 1 : 0)) * cap);
}

namespace {

// The dynamic shared-memory limit of each kernel instance only ever grows:
// setting it lower for a small launch would make a later, larger launch of
// the same instance fail with an invalid argument.  Tracked per device and
// instance, raised under a lock.
template <bool LAB, int MINB>
cudaError_t ensure_dynamic_smem(size_t smem) {
  static std::mutex mu;
  static size_t set_to[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) return e != cudaSuccess ? e : cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (smem <= set_to[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(match_kernel<LAB, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) set_to[dev] = smem;
  return e;
}

template <bool LAB, int MINB>
cudaError_t occupancy(int *n, int warps_per_block, size_t smem) {
  cudaError_t e = ensure_dynamic_smem<LAB, MINB>(smem);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, match_kernel<LAB, MINB>, warps_per_block * 32, smem);
  return e;
}

}  // namespace

int resident_blocks_per_sm(bool labeled, int warps_per_block, size_t smem, bool wide) {
  int n = 0;
  cudaError_t e;
  if (labeled)
    e = wide ? occupancy<true, 3>(&n, warps_per_block, smem) : occupancy<true, 4>(&n, warps_per_block, smem);
  else
    e = wide ? occupancy<false, 3>(&n, warps_per_block, smem) : occupancy<false, 4>(&n, warps_per_block, smem);
  return e == cudaSuccess ? n : -1;
}

void init_launch(RunCtl *ctl, QueueHdr *qh, cudaStream_t stream) {
  init_kernel<<<64, 256, 0, stream>>>(ctl, qh);
}

int launch_match(bool labeled, const DevGraph &g, RunCtl *ctl, SlotTable *tab, SplitUnit *units, QueueHdr *qh,
                 const KernelCfg &cfg, int blocks, int warps_per_block, cudaStream_t stream) {
  const size_t smem = (size_t)cfg.warp_bytes * warps_per_block;
  const dim3 grid(blocks), block(warps_per_block * 32);
  cudaError_t a;
  if (labeled)
    a = cfg.wide_regs ? ensure_dynamic_smem<true, 3>(smem) : ensure_dynamic_smem<true, 4>(smem);
  else
    a = cfg.wide_regs ? ensure_dynamic_smem<false, 3>(smem) : ensure_dynamic_smem<false, 4>(smem);
  if (a != cudaSuccess) return fail(TDFS_ERR_CUDA, "match kernel shared memory: %s", cudaGetErrorString(a));
  (void)cudaGetLastError();  // the check below must see this launch's error only
  if (labeled) {
    if (cfg.wide_regs) match_kernel<true, 3><<<grid, block, smem, stream>>>(g, cfg, ctl, tab, units, qh);
    else match_kernel<true, 4><<<grid, block, smem, stream>>>(g, cfg, ctl, tab, units, qh);
  } else {
    if (cfg.wide_regs) match_kernel<false, 3><<<grid, block, smem, stream>>>(g, cfg, ctl, tab, units, qh);
    else match_kernel<false, 4><<<grid, block, smem, stream>>>(g, cfg, ctl, tab, units, qh);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TDFS_ERR_CUDA, "match kernel launch: %s", cudaGetErrorString(e));
  return TDFS_OK;
}

}  // namespace tdfs
