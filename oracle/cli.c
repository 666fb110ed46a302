/*
 * cli.c -- command-line front end of the CPU oracle (TEST INFRASTRUCTURE).
 *
 *   oracle_count [--labeled] [--threads N] [--bytes] [--brute] <prefix> <p.g>
 *
 * Prints "<pattern path>\t<ms>\t<count>\n", the line format of the
 * reference's driver (cu_test.cu:107).
 */
#include "oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static double now_ms(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec / 1e6;
}

int main(int argc, char **argv) {
  int labeled = 0, threads = 0, bytes = 0, brute = 0;
  const char *prefix = NULL, *gpath = NULL;
  for (int i = 1; i < argc; i++) {
    if (!strcmp(argv[i], "--labeled")) labeled = 1;
    else if (!strcmp(argv[i], "--threads") && i + 1 < argc) threads = atoi(argv[++i]);
    else if (!strcmp(argv[i], "--bytes")) bytes = 1;
    else if (!strcmp(argv[i], "--brute")) brute = 1;
    else if (!prefix) prefix = argv[i];
    else if (!gpath) gpath = argv[i];
  }
  if (!prefix || !gpath) {
    fprintf(stderr, "usage: %s [--labeled] [--threads N] [--bytes] [--brute] <graph prefix> <pattern.g>\n", argv[0]);
    return 2;
  }
  orc_graph g;
  orc_plan p;
  if (orc_graph_load(prefix, labeled, &g)) { fprintf(stderr, "%s\n", orc_last_error()); return 1; }
  if (orc_plan_from_file(gpath, labeled, &p)) { fprintf(stderr, "%s\n", orc_last_error()); return 1; }
  unsigned long long cnt = 0, nb = 0;
  double t0 = now_ms();
  int rc = brute ? orc_bruteforce(&g, &p, &cnt) : orc_count(&g, &p, threads, 0, -1, &cnt, &nb);
  double t1 = now_ms();
  if (rc) { fprintf(stderr, "%s\n", orc_last_error()); return 1; }
  printf("%s\t%f\t%llu\n", gpath, t1 - t0, cnt);
  if (bytes) printf("bytes\t%llu\n", nb);
  orc_graph_free(&g);
  return 0;
}
