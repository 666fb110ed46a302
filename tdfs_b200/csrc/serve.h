// serve.h -- continuous-batching query server (serve.cpp).
#pragma once

#include <cstddef>
#include <cstdint>

#include "common.h"
#include "graph.h"
#include "match.cuh"

namespace tdfs {

// Launch shape of the persistent match kernel (capi.cpp).
struct LaunchShape {
  int warps_per_block;
  int blocks;
  KernelCfg cfg;
};
int launch_shape(const tdfs_graph *g, int kmax, bool labeled, const tdfs_options &o, LaunchShape *out);

// The level-0 range of a slot over edge ids [eb, ee), through the graph's
// label index for labeled plans when use_index is set (capi.cpp).
void level0_range(const tdfs_graph *g, const DevPlan &p, int64_t eb, int64_t ee, bool use_index, SlotInfo *in);

// The device plan table of a compiled pattern (capi.cpp).
const DevPlan &plan_device_table(const tdfs_plan *p);

struct Server;
size_t query_bytes(int k, int cap, int warps_per_block);
int server_create(tdfs_graph *g, const tdfs_server_options *o, Server **out);
int server_submit(Server *s, const DevPlan &plan, uint64_t *ticket);
int server_wait(Server *s, uint64_t ticket, uint64_t *count, double *latency_us);
int server_stats(Server *s, tdfs_serve_stats *st);
int server_destroy(Server *s);

}  // namespace tdfs
