/* Command-line front end of the CPU oracle (test infrastructure only).
 *   cpg_oracle seq     FILE K OUT   SEQUENTIAL costs, 9 significant digits
 *   cpg_oracle closure FILE K OUT   closure-at-split costs
 *   cpg_oracle sfxt    FILE OUT     "succ dist" per vertex
 * Prints the wall time of the SFXT and PFXT stages on stderr. */
#define _POSIX_C_SOURCE 199309L
#include "cpg_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static double now_ms(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    fprintf(stderr, "usage: cpg_oracle seq|closure FILE K OUT | sfxt FILE OUT\n");
    return 2;
  }
  orc_graph g;
  if (orc_read_text(argv[2], 0, &g) != 0) {
    fprintf(stderr, "cannot read %s\n", argv[2]);
    return 1;
  }
  int32_t* dist = malloc(sizeof(int32_t) * (size_t)(g.n + 1));
  int32_t* succ = malloc(sizeof(int32_t) * (size_t)(g.n + 1));
  double t0 = now_ms();
  orc_sfxt(&g, dist, succ, NULL);
  double t1 = now_ms();
  if (strcmp(argv[1], "sfxt") == 0) {
    FILE* f = fopen(argv[3], "w");
    for (int32_t v = 0; v < g.n; ++v) fprintf(f, "%d %d\n", succ[v], dist[v]);
    fclose(f);
    fprintf(stderr, "sfxt_ms=%.3f\n", t1 - t0);
    return 0;
  }
  if (argc < 5) return 2;
  long long k = atoll(argv[3]);
  orc_node* out = malloc(sizeof(orc_node) * (size_t)(k > 0 ? k : 1));
  int64_t n = 0;
  float split = 0.0f;
  if (strcmp(argv[1], "seq") == 0)
    n = orc_sequential(&g, dist, succ, k, out);
  else
    n = orc_closure_topk(&g, dist, succ, k, out, &split);
  double t2 = now_ms();
  if (n < 0) {
    fprintf(stderr, "oracle failed\n");
    return 1;
  }
  FILE* f = fopen(argv[4], "w");
  for (int64_t i = 0; i < n; ++i) fprintf(f, "%.9g\n", (double)out[i].slack);
  fclose(f);
  fprintf(stderr, "sfxt_ms=%.3f pfxt_ms=%.3f paths=%lld split=%.9g\n", t1 - t0,
          t2 - t1, (long long)n, (double)split);
  return 0;
}
