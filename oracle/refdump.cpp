// refdump.cpp -- TEST INFRASTRUCTURE: prints every plan field of the
// reference's own PatternPreprocessor (src/pattern.h) as one JSON line after
// the marker "@@PLAN".  It is compiled by oracle/Makefile against the
// reference sources where they lie, with bliss built from its sources, and
// never enters the product.  Its output pins the oracle's plan restatement.
#include <cuda_runtime.h>
#include <cstring>
#include <cstdio>
#include "src/pattern.h"

int main(int argc, char** argv) {
  if (argc != 2) {
    fprintf(stderr, "usage: %s <pattern.g>\n", argv[0]);
    return 2;
  }
  STMatch::PatternPreprocessor p(argv[1]);
  const STMatch::Pattern& t = p.pat;
  int k = t.nnodes;
  printf("@@PLAN {\"k\": %d, \"labeled\": %d, \"multiplicity\": %d, \"orient\": %u", k,
         (int)LABELED, p.PatternMultiplicity, t.partial_ori[0][0]);
  auto arr = [&](const char* name, const int* a, int n) {
    printf(", \"%s\": [", name);
    for (int i = 0; i < n; i++) printf("%s%d", i ? ", " : "", a[i]);
    printf("]");
  };
  arr("degree", t.degree, k);
  arr("vertex_labels", t.vertex_labels, k);
  arr("num_BN", t.num_BN, k);
  printf(", \"backward_neighbors\": [");
  for (int i = 0; i < k; i++) {
    printf("%s[", i ? ", " : "");
    for (int j = 0; j < t.num_BN[i]; j++) printf("%s%d", j ? ", " : "", t.backward_neighbors[i][j]);
    printf("]");
  }
  printf("]");
  arr("shared_lvl", t.shared_lvl, k);
  printf(", \"backward_neighbors_sh\": [");
  for (int i = 0; i < k; i++) {
    printf("%s[", i ? ", " : "");
    if (t.shared_lvl[i] != -1)
      for (int j = 0; j < t.num_BN_sh[i]; j++) printf("%s%d", j ? ", " : "", t.backward_neighbors_sh[i][j]);
    printf("]");
  }
  printf("]");
  arr("condition_cnt", t.condition_cnt, k);
  printf(", \"condition_order\": [");
  for (int i = 0; i < k; i++) {
    printf("%s[", i ? ", " : "");
    for (int j = 0; j < t.condition_cnt[i]; j++)
      printf("%s[%d, %d]", j ? ", " : "", t.condition_order[i * STMatch::PAT_SIZE * 2 + 2 * j],
             t.condition_order[i * STMatch::PAT_SIZE * 2 + 2 * j + 1]);
    printf("]");
  }
  printf("]");
  printf(", \"conditions\": [");
  bool first = true;
  for (int i = 0; i < k; i++)
    for (auto& c : p.order_[i])
      if (c.first == STMatch::LESS_THAN) {
        printf("%s[%d, %d]", first ? "" : ", ", i, c.second);
        first = false;
      }
  printf("]}\n");
  return 0;
}
