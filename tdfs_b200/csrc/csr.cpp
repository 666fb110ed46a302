// csr.cpp -- host CSR: the reference's binary graph format and the seeded
// synthetic generators (Erdos-Renyi, Chung-Lu power law, R-MAT, labels,
// random connected patterns).
//
// File format (written by graph_converter/compactify.cpp:172-195, read by
// src/graph.h:136-193): <prefix>.meta.txt holds "n E vid_size max_degree"
// whitespace separated (vid_size must be 4); <prefix>.vertex.bin is int64
// rowptr[n+1]; <prefix>.edge.bin is int32 colidx[E], every row sorted with no
// duplicates; <prefix>.label.bin is int32 label[n] (graph_converter/
// labelize.cpp:130-133).
#include "csr.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <unordered_set>

namespace tdfs {

namespace {

int hw_threads() {
  unsigned t = std::thread::hardware_concurrency();
  return t ? (int)std::min(t, 64u) : 4;
}

// f(b, e) over [0, n) split across host threads; `work` (default n) is the
// total cost in elementary steps: below ~2M steps one thread does it all,
// since starting threads would cost more than they save.
template <class F>
void parallel_for(int64_t n, F f, int64_t work = -1) {
  int T = hw_threads();
  if ((work < 0 ? n : work) < (1 << 21)) T = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([=] {
      int64_t b = n * t / T, e = n * (t + 1) / T;
      f(b, e);
    });
  for (auto &x : th) x.join();
}

template <class T>
int read_array(const std::string &path, T *dst, size_t count) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(TDFS_ERR_IO, "cannot open %s", path.c_str());
  f.read(reinterpret_cast<char *>(dst), sizeof(T) * count);
  if ((size_t)f.gcount() != sizeof(T) * count) return fail(TDFS_ERR_FORMAT, "%s: short file", path.c_str());
  return TDFS_OK;
}

template <class T>
int write_array(const std::string &path, const T *src, size_t count) {
  std::ofstream f(path, std::ios::binary);
  if (!f) return fail(TDFS_ERR_IO, "cannot create %s", path.c_str());
  f.write(reinterpret_cast<const char *>(src), sizeof(T) * count);
  if (!f) return fail(TDFS_ERR_IO, "write failed: %s", path.c_str());
  return TDFS_OK;
}

}  // namespace

int validate_csr(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx,
                 int32_t *max_degree) {
  if (n < 0 || n > INT32_MAX - 1 || nedges < 0) return fail(TDFS_ERR_FORMAT, "bad graph size");
  if (rowptr[0] != 0 || rowptr[n] != nedges) return fail(TDFS_ERR_FORMAT, "rowptr must span [0, E]");
  std::atomic<int> bad{0};
  std::atomic<int64_t> where{-1};
  std::vector<int32_t> part_max(hw_threads() + 1, 0);
  std::atomic<int> slot{0};
  parallel_for(
      n, [&](int64_t b, int64_t e) {
    int32_t md = 0;
    for (int64_t v = b; v < e && !bad.load(std::memory_order_relaxed); ++v) {
      int64_t lo = rowptr[v], hi = rowptr[v + 1];
      if (hi < lo || hi - lo > INT32_MAX) { bad = 1; where = v; break; }
      md = std::max<int32_t>(md, (int32_t)(hi - lo));
      for (int64_t j = lo; j < hi; ++j) {
        int32_t c = colidx[j];
        if (c < 0 || c >= n) { bad = 2; where = v; break; }
        if (j + 1 < hi && c >= colidx[j + 1]) { bad = 3; where = v; break; }
      }
    }
    part_max[slot++] = md;
  }, n + nedges);
  if (bad == 1) return fail(TDFS_ERR_FORMAT, "rowptr decreases at vertex %lld", (long long)where.load());
  if (bad == 2) return fail(TDFS_ERR_FORMAT, "neighbour id out of range in row %lld", (long long)where.load());
  if (bad == 3)
    return fail(TDFS_ERR_FORMAT, "row %lld not strictly increasing (unsorted or duplicate edge)",
                (long long)where.load());
  if (max_degree) *max_degree = *std::max_element(part_max.begin(), part_max.end());
  return TDFS_OK;
}

void csr_from_pairs(int64_t n, std::vector<std::pair<uint32_t, uint32_t>> &pairs, tdfs_csr *out) {
  // counting sort by source over both directions, then per-row sort + unique
  std::vector<std::atomic<int64_t>> deg(n + 1);
  for (auto &d : deg) d.store(0, std::memory_order_relaxed);
  const int64_t m = (int64_t)pairs.size();
  parallel_for(m, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      auto [u, v] = pairs[i];
      if (u == v) continue;
      deg[u].fetch_add(1, std::memory_order_relaxed);
      deg[v].fetch_add(1, std::memory_order_relaxed);
    }
  });
  std::vector<int64_t> off(n + 1, 0);
  for (int64_t v = 0; v < n; ++v) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
  std::vector<int32_t> raw(off[n]);
  for (int64_t v = 0; v < n; ++v) deg[v].store(off[v], std::memory_order_relaxed);
  parallel_for(m, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      auto [u, v] = pairs[i];
      if (u == v) continue;
      raw[deg[u].fetch_add(1, std::memory_order_relaxed)] = (int32_t)v;
      raw[deg[v].fetch_add(1, std::memory_order_relaxed)] = (int32_t)u;
    }
  });
  std::vector<std::pair<uint32_t, uint32_t>>().swap(pairs);
  std::vector<int64_t> newdeg(n, 0);
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v) {
      auto *lo = raw.data() + off[v], *hi = raw.data() + off[v + 1];
      std::sort(lo, hi);
      newdeg[v] = std::unique(lo, hi) - lo;
    }
  });
  out->n = n;
  out->rowptr.assign(n + 1, 0);
  for (int64_t v = 0; v < n; ++v) out->rowptr[v + 1] = out->rowptr[v] + newdeg[v];
  out->nedges = out->rowptr[n];
  out->colidx.resize(out->nedges);
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t v = b; v < e; ++v)
      std::memcpy(out->colidx.data() + out->rowptr[v], raw.data() + off[v], sizeof(int32_t) * newdeg[v]);
  });
  int32_t md = 0;
  for (int64_t v = 0; v < n; ++v) md = std::max<int32_t>(md, (int32_t)newdeg[v]);
  out->max_degree = md;
}

// Descending-degree relabelling as graph_converter/relabel.cpp:27-58 does
// it: (degree, id) pairs sorted with std::greater, so ties go to the larger
// old id first; vertex i of the output is order[i] of the input, every row
// is mapped through the new ids and sorted again.  Labels move with their
// vertices.
void relabel_by_degree(const tdfs_csr &g, tdfs_csr *c) {
  const int64_t n = g.n;
  std::vector<std::pair<int64_t, int64_t>> order(n);
  for (int64_t v = 0; v < n; ++v) order[v] = {g.rowptr[v + 1] - g.rowptr[v], v};
  std::sort(order.begin(), order.end(), std::greater<>());
  std::vector<int32_t> newid(n);
  for (int64_t i = 0; i < n; ++i) newid[order[i].second] = (int32_t)i;
  c->n = n;
  c->nedges = g.nedges;
  c->max_degree = g.max_degree;
  c->rowptr.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) c->rowptr[i + 1] = c->rowptr[i] + order[i].first;
  c->colidx.resize(g.nedges);
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) {
      int64_t old = order[i].second;
      int32_t *dst = c->colidx.data() + c->rowptr[i];
      int64_t d = g.rowptr[old + 1] - g.rowptr[old];
      for (int64_t t = 0; t < d; ++t) dst[t] = newid[g.colidx[g.rowptr[old] + t]];
      std::sort(dst, dst + d);
    }
  });
  c->labels.clear();
  if (!g.labels.empty()) {
    c->labels.resize(n);
    for (int64_t i = 0; i < n; ++i) c->labels[i] = g.labels[order[i].second];
  }
}

// Degree orientation as graph_converter/halve.cpp:17-32 does it: edge (s, d)
// is kept when deg(d) > deg(s), or the degrees tie and d > s, so each
// undirected edge of a symmetric graph survives in exactly one direction.
// Rows stay sorted; vertex ids and labels are unchanged.
void halve_by_degree(const tdfs_csr &g, tdfs_csr *c) {
  const int64_t n = g.n;
  auto deg = [&](int64_t v) { return g.rowptr[v + 1] - g.rowptr[v]; };
  std::vector<int64_t> keep(n, 0);
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t s = b; s < e; ++s) {
      const int64_t ds = deg(s);
      int64_t k = 0;
      for (int64_t j = g.rowptr[s]; j < g.rowptr[s + 1]; ++j) {
        const int64_t d = g.colidx[j], dd = deg(d);
        k += dd > ds || (dd == ds && d > s);
      }
      keep[s] = k;
    }
  });
  c->n = n;
  c->rowptr.assign(n + 1, 0);
  int64_t md = 0;
  for (int64_t v = 0; v < n; ++v) {
    c->rowptr[v + 1] = c->rowptr[v] + keep[v];
    md = std::max(md, keep[v]);
  }
  c->nedges = c->rowptr[n];
  c->max_degree = (int32_t)md;
  c->colidx.resize(c->nedges);
  parallel_for(n, [&](int64_t b, int64_t e) {
    for (int64_t s = b; s < e; ++s) {
      const int64_t ds = deg(s);
      int32_t *out = c->colidx.data() + c->rowptr[s];
      for (int64_t j = g.rowptr[s]; j < g.rowptr[s + 1]; ++j) {
        const int64_t d = g.colidx[j], dd = deg(d);
        if (dd > ds || (dd == ds && d > s)) *out++ = (int32_t)d;
      }
    }
  });
  c->labels = g.labels;
}

}  // namespace tdfs

using namespace tdfs;

extern "C" {

int tdfs_csr_from_arrays(int64_t n, int64_t nedges, const int64_t *rowptr, const int32_t *colidx,
                         const int32_t *labels, tdfs_csr **out) {
  if (!rowptr || (!colidx && nedges) || !out) return fail(TDFS_ERR_ARG, "null argument");
  int32_t md = 0;
  int rc = validate_csr(n, nedges, rowptr, colidx, &md);
  if (rc) return rc;
  auto *c = new tdfs_csr;
  c->n = n;
  c->nedges = nedges;
  c->max_degree = md;
  c->rowptr.assign(rowptr, rowptr + n + 1);
  c->colidx.assign(colidx, colidx + nedges);
  if (labels) c->labels.assign(labels, labels + n);
  *out = c;
  return TDFS_OK;
}

int tdfs_csr_relabel(const tdfs_csr *in, tdfs_csr **out) {
  if (!in || !out) return fail(TDFS_ERR_ARG, "null argument");
  auto *c = new tdfs_csr;
  relabel_by_degree(*in, c);
  *out = c;
  return TDFS_OK;
}

int tdfs_csr_halve(const tdfs_csr *in, tdfs_csr **out) {
  if (!in || !out) return fail(TDFS_ERR_ARG, "null argument");
  auto *c = new tdfs_csr;
  halve_by_degree(*in, c);
  *out = c;
  return TDFS_OK;
}

int tdfs_csr_read(const char *prefix, int labeled, tdfs_csr **out) {
  if (!prefix || !out) return fail(TDFS_ERR_ARG, "null argument");
  std::string p(prefix);
  std::ifstream meta(p + ".meta.txt");
  if (!meta) return fail(TDFS_ERR_IO, "cannot open %s.meta.txt", prefix);
  long long n, e, vid, maxd;
  if (!(meta >> n >> e >> vid >> maxd)) return fail(TDFS_ERR_FORMAT, "%s.meta.txt: need n E vid_size max_degree", prefix);
  if (vid != 4) return fail(TDFS_ERR_FORMAT, "%s.meta.txt: vid_size must be 4 (got %lld)", prefix, vid);
  if (n < 0 || e < 0) return fail(TDFS_ERR_FORMAT, "%s.meta.txt: negative size", prefix);
  auto *c = new tdfs_csr;
  c->n = n;
  c->nedges = e;
  c->rowptr.resize(n + 1);
  c->colidx.resize(e);
  int rc = read_array(p + ".vertex.bin", c->rowptr.data(), n + 1);
  if (!rc) rc = read_array(p + ".edge.bin", c->colidx.data(), e);
  if (!rc && labeled) {
    c->labels.resize(n);
    rc = read_array(p + ".label.bin", c->labels.data(), n);
  }
  if (!rc) rc = validate_csr(n, e, c->rowptr.data(), c->colidx.data(), &c->max_degree);
  if (rc) {
    delete c;
    return rc;
  }
  *out = c;
  return TDFS_OK;
}

int tdfs_csr_view(const tdfs_csr *c, int64_t *n, int64_t *nedges, const int64_t **rowptr,
                  const int32_t **colidx, const int32_t **labels, int32_t *max_degree) {
  if (!c) return fail(TDFS_ERR_ARG, "null csr");
  if (n) *n = c->n;
  if (nedges) *nedges = c->nedges;
  if (rowptr) *rowptr = c->rowptr.data();
  if (colidx) *colidx = c->colidx.data();
  if (labels) *labels = c->labels.empty() ? nullptr : c->labels.data();
  if (max_degree) *max_degree = c->max_degree;
  return TDFS_OK;
}

int tdfs_csr_write(const tdfs_csr *c, const char *prefix) {
  if (!c || !prefix) return fail(TDFS_ERR_ARG, "null argument");
  std::string p(prefix);
  {
    std::ofstream meta(p + ".meta.txt");
    if (!meta) return fail(TDFS_ERR_IO, "cannot create %s.meta.txt", prefix);
    meta << c->n << "\n" << c->nedges << "\n" << 4 << "\n" << c->max_degree << "\n";
  }
  int rc = write_array(p + ".vertex.bin", c->rowptr.data(), c->rowptr.size());
  if (!rc) rc = write_array(p + ".edge.bin", c->colidx.data(), c->colidx.size());
  if (!rc && !c->labels.empty()) rc = write_array(p + ".label.bin", c->labels.data(), c->labels.size());
  return rc;
}

int tdfs_csr_set_labels(tdfs_csr *c, int nlabels, uint64_t seed) {
  if (!c || nlabels < 1 || nlabels > 255) return fail(TDFS_ERR_ARG, "labels: need 1 <= nlabels <= 255");
  c->labels.resize(c->n);
  parallel_for(c->n, [&](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) c->labels[i] = (int32_t)(hash64(seed, (uint64_t)i) % (uint64_t)nlabels);
  });
  return TDFS_OK;
}

int tdfs_csr_free(tdfs_csr *c) {
  delete c;
  return TDFS_OK;
}

// G(n, p) by geometric skipping over the pairs (i < j) in row-major order.
int tdfs_gen_er(int64_t n, double avg_degree, uint64_t seed, tdfs_csr **out) {
  if (!out || n < 2 || n > (1ll << 31) - 2 || avg_degree <= 0 || avg_degree >= n - 1)
    return fail(TDFS_ERR_ARG, "er: need n >= 2 and 0 < avg_degree < n - 1");
  const double p = avg_degree / (double)(n - 1);
  const double lq = std::log1p(-p);
  Rng rng(seed);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  pairs.reserve((size_t)(n * avg_degree / 2 * 1.1) + 16);
  int64_t i = 0, j = 0;  // current pair index: row i, column j (> i)
  int64_t pos = -1;      // linear position within row i of column j-(i+1)
  for (;;) {
    double r = 1.0 - rng.uniform();  // (0, 1]
    int64_t skip = (int64_t)std::floor(std::log(r) / lq);
    pos += 1 + skip;
    while (i < n - 1 && pos >= n - 1 - i) {
      pos -= n - 1 - i;
      ++i;
    }
    if (i >= n - 1) break;
    j = i + 1 + pos;
    pairs.emplace_back((uint32_t)i, (uint32_t)j);
  }
  auto *c = new tdfs_csr;
  csr_from_pairs(n, pairs, c);
  *out = c;
  return TDFS_OK;
}

// Chung-Lu: expected degree w_i = C (i + i0)^(-1/(gamma-1)), with w_0 equal
// to the cap and sum(w) = 2 * undirected_edges; endpoints are drawn from w
// until the target number of distinct edges is reached (no loops, no
// duplicates, no vertex above the cap); then the ids are relabelled by
// descending degree, ties by descending old id, as graph_converter/
// relabel.cpp:27-35 sorts (degree, id) pairs with std::greater.
int tdfs_gen_chung_lu(int64_t n, int64_t m, double gamma, int32_t cap, uint64_t seed, tdfs_csr **out) {
  if (!out || n < 2 || n > (1ll << 31) - 2 || m < 1 || gamma <= 1.0 || cap < 1 || m > n * (int64_t)cap / 2)
    return fail(TDFS_ERR_ARG, "chung_lu: bad arguments");
  const double alpha = 1.0 / (gamma - 1.0);
  auto total = [&](double i0) {
    double s = 0;
    for (int64_t i = 0; i < n; ++i) s += std::pow((i + i0) / i0, -alpha);
    return s * cap;
  };
  // find i0 with sum(w) = 2m (total decreases as i0 shrinks)
  double lo = 1e-6, hi = (double)n;
  for (int it = 0; it < 100; ++it) {
    double mid = std::sqrt(lo * hi);
    if (total(mid) > 2.0 * m) hi = mid; else lo = mid;
  }
  const double i0 = std::sqrt(lo * hi);
  std::vector<double> cdf(n);
  double s = 0;
  for (int64_t i = 0; i < n; ++i) {
    s += cap * std::pow((i + i0) / i0, -alpha);
    cdf[i] = s;
  }
  Rng rng(seed);
  auto draw = [&]() {
    double x = rng.uniform() * s;
    return (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
  };
  std::unordered_set<uint64_t> seen;
  seen.reserve((size_t)m * 2);
  std::vector<int32_t> deg(n, 0);
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  pairs.reserve(m);
  int64_t attempts = 0, limit = 200 * m;
  while ((int64_t)pairs.size() < m && attempts++ < limit) {
    uint32_t u = draw(), v = draw();
    if (u == v) continue;
    if (u > v) std::swap(u, v);
    if (deg[u] >= cap || deg[v] >= cap) continue;
    if (!seen.insert((uint64_t)u << 32 | v).second) continue;
    ++deg[u];
    ++deg[v];
    pairs.emplace_back(u, v);
  }
  tdfs_csr g;
  csr_from_pairs(n, pairs, &g);
  auto *c = new tdfs_csr;
  relabel_by_degree(g, c);
  *out = c;
  return TDFS_OK;
}

// R-MAT: each sample descends `scale` levels choosing quadrant a/b/c/d; the
// samples are split into 256 fixed blocks with their own streams so the
// result does not depend on the thread count.
int tdfs_gen_rmat(int scale, int edge_factor, double a, double b, double c, uint64_t seed,
                  tdfs_csr **out) {
  if (!out || scale < 1 || scale > 30 || edge_factor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1)
    return fail(TDFS_ERR_ARG, "rmat: bad arguments");
  const int64_t n = 1ll << scale;
  const int64_t m = (int64_t)edge_factor << scale;
  const int kBlocks = 256;
  const uint32_t ta = (uint32_t)std::llround(a * 65536.0), tb = (uint32_t)std::llround((a + b) * 65536.0),
                 tc = (uint32_t)std::llround((a + b + c) * 65536.0);
  std::vector<std::pair<uint32_t, uint32_t>> pairs(m);
  std::atomic<int> next{0};
  int T = hw_threads();
  std::vector<std::thread> th;
  for (int t = 0; t < T; ++t)
    th.emplace_back([&] {
      for (int blk; (blk = next++) < kBlocks;) {
        Rng rng(hash64(seed, (uint64_t)blk));
        int64_t lo = m * blk / kBlocks, hi = m * (blk + 1) / kBlocks;
        for (int64_t i = lo; i < hi; ++i) {
          uint32_t u = 0, v = 0;
          uint64_t bits = 0;
          for (int l = 0; l < scale; ++l) {
            if ((l & 3) == 0) bits = rng.next();
            uint32_t r = (uint32_t)(bits & 0xFFFF);
            bits >>= 16;
            uint32_t q = r < ta ? 0 : r < tb ? 1 : r < tc ? 2 : 3;
            u = (u << 1) | (q >> 1);
            v = (v << 1) | (q & 1);
          }
          pairs[i] = {u, v};
        }
      }
    });
  for (auto &x : th) x.join();
  auto *g = new tdfs_csr;
  csr_from_pairs(n, pairs, g);
  *out = g;
  return TDFS_OK;
}

int tdfs_gen_pattern(int k, double density, int nlabels, uint64_t seed, char *buf, size_t cap) {
  if (k < 3 || k > kMaxK || nlabels < 1 || !buf) return fail(TDFS_ERR_ARG, "pattern: need 3 <= k <= 7");
  Rng rng(seed);
  bool e[kMaxK][kMaxK] = {};
  // spanning edges in matching order: 2 ~ 1, every other i > 0 ~ random earlier
  for (int i = 1; i < k; ++i) {
    int j = (i == 2) ? 1 : (int)rng.below(i);
    e[i][j] = e[j][i] = true;
  }
  const int pairs = k * (k - 1) / 2;
  double extra = (density * pairs - (k - 1)) / (double)(pairs - (k - 1));
  extra = std::min(1.0, std::max(0.0, extra));
  for (int i = 0; i < k; ++i)
    for (int j = i + 1; j < k; ++j)
      if (!e[i][j] && rng.uniform() < extra) e[i][j] = e[j][i] = true;
  std::string s = "# t 1\n";
  for (int i = 0; i < k; ++i) s += "v " + std::to_string(i) + " " + std::to_string(rng.below(nlabels)) + "\n";
  for (int i = 0; i < k; ++i)
    for (int j = i + 1; j < k; ++j)
      if (e[i][j]) s += "e " + std::to_string(i) + " " + std::to_string(j) + " 1\n";
  if (s.size() + 1 > cap) return fail(TDFS_ERR_ARG, "pattern: buffer too small");
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return TDFS_OK;
}

}  // extern "C"
