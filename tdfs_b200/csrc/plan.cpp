// plan.cpp -- compile a .g pattern into the plan table the DFS kernel reads.
//
// Restates the reference's PatternPreprocessor (src/pattern.h:65-720) for the
// fields its kernel reads (src/gpu_match.cu): matching order = file order,
// backward neighbours, pattern degrees, symmetry-breaking conditions from the
// full automorphism group, the level-0 edge-orientation bit, reuse levels and
// vertex labels.  The reference gets automorphism generators from bliss and
// closes them under products (src/pattern.h:603-663); with at most 7! = 5040
// permutations the group is enumerated here directly, which yields the same
// set and therefore the same conditions.
#include "plan.h"

#include <algorithm>
#include <functional>
#include <cstdio>
#include <cstring>
#include <map>
#include <numeric>
#include <set>
#include <sstream>

namespace tdfs {

namespace {

using Perm = std::array<int, kMaxK>;

// .g reader, src/pattern.h:110-143.  '#' header lines, then "v id label"
// lines (labels in line order; the id is not used, as in the reference), then
// "e u v label" lines.  Blank lines are ignored.
int parse(const std::string &text, bool labeled, HostPlan *p) {
  std::istringstream in(text);
  std::string line;
  int stage = 0, lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    if (stage == 0 && line[0] == '#') continue;
    if (stage == 0) stage = 1;
    if (stage == 1 && line[0] != 'v') stage = 2;
    std::istringstream ls(line.substr(1));
    if (stage == 1) {
      int id, lab;
      if (!(ls >> id >> lab)) return fail(TDFS_ERR_FORMAT, "pattern line %d: bad vertex line", lineno);
      if (p->k == kMaxK) return fail(TDFS_ERR_PATTERN, "pattern has more than %d vertices", kMaxK);
      p->vlabel[p->k++] = labeled ? lab : 1;  // unlabeled: all 1 (src/pattern.h:124-129)
    } else {
      int u, v, lab;
      if (line[0] != 'e' || !(ls >> u >> v >> lab))
        return fail(TDFS_ERR_FORMAT, "pattern line %d: bad edge line", lineno);
      if (u < 0 || v < 0 || u >= p->k || v >= p->k)
        return fail(TDFS_ERR_PATTERN, "pattern line %d: endpoint out of range", lineno);
      if (u == v) return fail(TDFS_ERR_PATTERN, "pattern line %d: self-loop", lineno);
      p->adj[u][v] = p->adj[v][u] = lab;
    }
  }
  if (p->k < 3) return fail(TDFS_ERR_PATTERN, "pattern needs at least 3 vertices (has %d)", p->k);
  return TDFS_OK;
}

// PatternMultiplicity test, src/pattern.h:281-308: permutation pp maps the
// edge set {adj != 0} onto a set that must equal {adj == 1} row by row.
bool keeps_labelled_edges(const HostPlan &p, const Perm &pp) {
  std::array<unsigned, kMaxK> image{};
  for (int i = 0; i < p.k; ++i)
    for (int j = 0; j < p.k; ++j)
      if (p.adj[i][j] != 0) image[pp[i]] |= 1u << pp[j];
  for (int i = 0; i < p.k; ++i) {
    unsigned ones = 0;
    for (int j = 0; j < p.k; ++j)
      if (p.adj[i][j] == 1) ones |= 1u << j;
    if (ones != image[i]) return false;
  }
  return true;
}

// Automorphism of the simple graph {adj > 0} (the bliss graph built by
// src/pattern.h:581-594, all vertices one colour).
bool is_automorphism(const HostPlan &p, const Perm &pp) {
  for (int i = 0; i < p.k; ++i)
    for (int j = i + 1; j < p.k; ++j)
      if ((p.adj[i][j] > 0) != (p.adj[pp[i]][pp[j]] > 0)) return false;
  return true;
}

// Every permutation pp of 0..k-1 with ok(i, j, pp[i], pp[j]) for all i, j,
// by depth-first extension of consistent prefixes.
template <class Ok, class Emit>
void search_perms(int k, const Ok &ok, const Emit &emit) {
  Perm pp{};
  unsigned used = 0;
  std::function<void(int)> go = [&](int d) {
    if (d == k) {
      emit(pp);
      return;
    }
    for (int v = 0; v < k; ++v) {
      if (used >> v & 1) continue;
      bool fine = ok(d, d, v, v);
      for (int i = 0; fine && i < d; ++i) fine = ok(i, d, pp[i], v) && ok(d, i, v, pp[i]);
      if (!fine) continue;
      pp[d] = v;
      used |= 1u << v;
      go(d + 1);
      used &= ~(1u << v);
    }
  };
  go(0);
}

// GetConditions, src/pattern.h:665-707.
std::vector<std::pair<int, int>> symmetry_conditions(int k, std::vector<Perm> group) {
  std::vector<std::pair<int, int>> out;
  for (;;) {
    // orbit classes keyed by their smallest member
    std::map<int, std::set<int>> classes;
    for (int v = 0; v < k; ++v) {
      std::set<int> orbit;
      for (const Perm &g : group) orbit.insert(g[v]);
      if (!orbit.empty()) classes[*orbit.begin()].insert(orbit.begin(), orbit.end());
    }
    auto it = std::find_if(classes.begin(), classes.end(),
                           [](const auto &c) { return c.second.size() > 1; });
    if (it == classes.end()) break;
    const std::set<int> &cls = it->second;
    const int n0 = *cls.begin();
    for (const Perm &g : group) {
      int best = -1;
      for (int m : cls)
        if (m != n0 && (best < 0 || g[m] < g[best])) best = m;
      out.emplace_back(n0, best);
    }
    group.erase(std::remove_if(group.begin(), group.end(), [n0](const Perm &g) { return g[n0] != n0; }),
                group.end());
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return out;
}

int derive(HostPlan *p) {
  const int k = p->k;
  for (int i = 0; i < k; ++i) {
    int d = 0;
    for (int j = 0; j < k; ++j) d += p->adj[i][j] > 0;
    p->degree[i] = d;  // src/pattern.h:189-195
  }

  // Both groups by backtracking over partial permutations: a prefix
  // pp[0..d) extends only while every pair among its vertices already obeys
  // the relation, so the search visits the group's members and few dead ends
  // instead of all k! permutations.  Every full permutation reached is
  // checked once more by the whole-permutation test, and the group comes out
  // as the same set (the conditions depend on the set only).
  std::vector<Perm> aut;
  p->multiplicity = 0;
  p->orient = 0;
  search_perms(k, [&](int i, int j, int pi, int pj) { return (p->adj[i][j] != 0) == (p->adj[pi][pj] == 1); },
               [&](const Perm &pp) {
                 if (!keeps_labelled_edges(*p, pp)) return;
                 ++p->multiplicity;
                 if (pp[0] == 1) p->orient = 1;  // L_adj[0][1], src/pattern.h:312-340
               });
  search_perms(k, [&](int i, int j, int pi, int pj) { return i == j || (p->adj[i][j] > 0) == (p->adj[pi][pj] > 0); },
               [&](const Perm &pp) {
                 if (is_automorphism(*p, pp)) aut.push_back(pp);
               });
  p->conditions = symmetry_conditions(k, std::move(aut));

  // condition_order, src/pattern.h:416-448 (SetConditions :709-719).
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < i; ++j) {
      int op = kNonEqual;
      for (auto [a, b] : p->conditions) {
        if (a == j && b == i) { op = kLarger; break; }
        if (a == i && b == j) { op = kLess; break; }
      }
      p->cond[i][j] = op;
    }

  // Backward neighbours, src/pattern.h:342-358.
  for (int i = 1; i < k; ++i) {
    p->bn[i].clear();
    for (int j = 0; j < i; ++j)
      if (p->adj[i][j] > 0) p->bn[i].push_back(j);
  }
  // The reference asserts on a vertex without earlier neighbour
  // (src/gpu_match.cu:638-639); here it is a compile error.
  for (int i = 2; i < k; ++i)
    if (p->bn[i].empty())
      return fail(TDFS_ERR_PATTERN, "pattern vertex %d has no earlier neighbour (not in connected order)", i);

  // Reuse levels, src/pattern.h:370-413, and their removal for unlabeled
  // patterns whose conditions differ, src/pattern.h:460-480.
  std::array<unsigned, kMaxK> nb{};
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < i; ++j)
      if (p->adj[j][i] > 0) nb[i] |= 1u << j;
  p->shared_lvl.fill(-1);
  for (int i = 2; i < k; ++i) {
    for (int j = i - 1; j >= 1; --j) {
      if ((nb[i] & nb[j]) == nb[j] && p->bn[i].size() >= 2 && p->bn[j].size() >= 2 &&
          p->vlabel[i] == p->vlabel[j]) {
        p->shared_lvl[i] = j;
        break;
      }
    }
    int dep = p->shared_lvl[i];
    p->bn_sh[i].clear();
    if (dep < 0) continue;
    for (int j = i - 1; j >= 0; --j)
      if ((nb[i] >> j & 1) && !(nb[dep] >> j & 1)) p->bn_sh[i].push_back(j);
    if (!p->labeled)
      for (int j = 0; j < dep; ++j)
        if (p->cond[dep][j] != p->cond[i][j]) p->shared_lvl[i] = -1;
  }
  return TDFS_OK;
}

}  // namespace

int compile_pattern(const std::string &text, bool labeled, HostPlan *out) {
  HostPlan p;
  p.labeled = labeled;
  p.text = text;
  int rc = parse(text, labeled, &p);
  if (rc) return rc;
  rc = derive(&p);
  if (rc) return rc;
  *out = std::move(p);
  return TDFS_OK;
}

DevPlan HostPlan::to_device() const {
  DevPlan d;
  std::memset(&d, 0, sizeof d);
  d.k = k;
  d.labeled = labeled;
  d.orient = labeled ? 0 : orient;  // the r<c filter applies to ulb only (src/gpu_match.cu:536)
  for (int i = 0; i < 3; ++i) d.deg[i] = degree[i];
  for (int i = 0; i < kMaxK; ++i) {
    d.label[i] = (i < k && vlabel[i] >= 0 && vlabel[i] < 255) ? vlabel[i] : 255;
    d.dep[i] = -1;
  }
  for (int i = 1; i < k; ++i) {
    d.nbn[i] = (int)bn[i].size();
    for (size_t t = 0; t < bn[i].size(); ++t) d.bn[i][t] = (int8_t)bn[i][t];
    if (shared_lvl[i] >= 0) {
      d.dep[i] = shared_lvl[i];
      d.nsh[i] = (int)bn_sh[i].size();
      for (size_t t = 0; t < bn_sh[i].size(); ++t) d.bnsh[i][t] = (int8_t)bn_sh[i][t];
    }
    for (int j = 0; j < i; ++j) {
      if (labeled) {
        d.neq[i] |= 1u << j;  // labeled: injectivity against all earlier (:315-325)
      } else if (cond[i][j] == kLarger) {
        d.larger[i] |= 1u << j;
      } else if (cond[i][j] == kLess) {
        d.less[i] |= 1u << j;
      } else {
        d.neq[i] |= 1u << j;
      }
    }
  }
  d.multiplicity = labeled ? 1 : (uint64_t)multiplicity;
  return d;
}

std::string HostPlan::dump_json() const {
  std::ostringstream o;
  auto list = [&](const char *name, auto f, int n) {
    o << ", \"" << name << "\": [";
    for (int i = 0; i < n; ++i) o << (i ? ", " : "") << f(i);
    o << "]";
  };
  auto vec = [](const std::vector<int> &v) {
    std::string s = "[";
    for (size_t i = 0; i < v.size(); ++i) s += (i ? ", " : "") + std::to_string(v[i]);
    return s + "]";
  };
  o << "{\"k\": " << k << ", \"labeled\": " << (int)labeled << ", \"multiplicity\": " << multiplicity
    << ", \"orient\": " << orient;
  list("degree", [&](int i) { return degree[i]; }, k);
  list("vertex_labels", [&](int i) { return vlabel[i]; }, k);
  list("num_BN", [&](int i) { return i ? (int)bn[i].size() : 0; }, k);
  list("backward_neighbors", [&](int i) { return i ? vec(bn[i]) : std::string("[]"); }, k);
  list("shared_lvl", [&](int i) { return shared_lvl[i]; }, k);
  list("backward_neighbors_sh", [&](int i) { return shared_lvl[i] >= 0 ? vec(bn_sh[i]) : std::string("[]"); }, k);
  list("condition_cnt", [&](int i) { return i; }, k);
  list("condition_order", [&](int i) {
    std::string s = "[";
    for (int j = 0; j < i; ++j) s += (j ? ", [" : "[") + std::to_string(cond[i][j]) + ", " + std::to_string(j) + "]";
    return s + "]";
  }, k);
  o << ", \"conditions\": [";
  for (size_t c = 0; c < conditions.size(); ++c)
    o << (c ? ", [" : "[") << conditions[c].first << ", " << conditions[c].second << "]";
  o << "]}";
  return o.str();
}

}  // namespace tdfs
