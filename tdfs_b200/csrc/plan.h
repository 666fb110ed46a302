// plan.h -- host-side pattern plan compiler.
#pragma once

#include <array>
#include <string>
#include <utility>
#include <vector>

#include "common.h"

namespace tdfs {

// A parsed .g pattern plus everything derived from it.  Field meanings follow
// the reference's Pattern struct (src/pattern.h:43-62) and
// PatternPreprocessor (src/pattern.h:65-720).
struct HostPlan {
  int k = 0;
  bool labeled = false;
  std::array<std::array<int, kMaxK>, kMaxK> adj{};  // raw edge labels
  std::array<int, kMaxK> vlabel{};
  std::array<int, kMaxK> degree{};
  std::array<std::vector<int>, kMaxK> bn;      // backward neighbours
  std::array<int, kMaxK> shared_lvl{};         // reuse source or -1
  std::array<std::vector<int>, kMaxK> bn_sh;   // extra BNs under reuse
  std::array<std::array<int, kMaxK>, kMaxK> cond{};  // cond[i][j], j < i
  std::vector<std::pair<int, int>> conditions;  // pairs (a, b): phi(a) < phi(b)
  int orient = 0;                               // partial_ori[0][0]
  long long multiplicity = 0;                   // PatternMultiplicity
  std::string text;                             // source .g text

  DevPlan to_device() const;
  std::string dump_json() const;
};

// Parse + compile; returns TDFS_OK or an error code (message via set_error).
int compile_pattern(const std::string &text, bool labeled, HostPlan *out);

}  // namespace tdfs
