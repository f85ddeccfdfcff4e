/*
 * CPU oracle for the critical-path-generation hot path.  TEST INFRASTRUCTURE
 * ONLY: see cpg_oracle.h for what it restates and who may call it.
 */
#include "cpg_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- ingestion */

static int grow(void** p, size_t* cap, size_t need, size_t elem) {
  if (need <= *cap) return 0;
  size_t c = *cap ? *cap : 1024;
  while (c < need) c *= 2;
  void* q = realloc(*p, c * elem);
  if (!q) return -1;
  *p = q;
  *cap = c;
  return 0;
}

/* Edges are grouped per source (and per destination) in file order, the way
 * read_input's unordered_map<int, vector<pair>> keeps them (gpucpg.cu:500-541). */
int orc_build_csr(int32_t n, int32_t m, const int32_t* src, const int32_t* dst,
                  const float* w, orc_graph* g) {
  memset(g, 0, sizeof(*g));
  g->n = n;
  g->m = m;
  g->adjp = calloc((size_t)n + 1, sizeof(int32_t));
  g->iadjp = calloc((size_t)n + 1, sizeof(int32_t));
  g->adj = malloc(sizeof(int32_t) * (size_t)(m ? m : 1));
  g->w = malloc(sizeof(float) * (size_t)(m ? m : 1));
  g->iadj = malloc(sizeof(int32_t) * (size_t)(m ? m : 1));
  int32_t* fill = calloc((size_t)n + 1, sizeof(int32_t));
  if (!g->adjp || !g->iadjp || !g->adj || !g->w || !g->iadj || !fill) {
    free(fill);
    orc_free_graph(g);
    return -1;
  }
  for (int32_t e = 0; e < m; ++e) {
    if (src[e] < 0 || src[e] >= n || dst[e] < 0 || dst[e] >= n) {
      free(fill);
      orc_free_graph(g);
      return -2;
    }
    g->adjp[src[e] + 1]++;
    g->iadjp[dst[e] + 1]++;
  }
  for (int32_t v = 0; v < n; ++v) {
    g->adjp[v + 1] += g->adjp[v];
    g->iadjp[v + 1] += g->iadjp[v];
  }
  for (int32_t e = 0; e < m; ++e) {
    int32_t p = g->adjp[src[e]] + fill[src[e]]++;
    g->adj[p] = dst[e];
    g->w[p] = w[e];
  }
  memset(fill, 0, sizeof(int32_t) * ((size_t)n + 1));
  for (int32_t e = 0; e < m; ++e) {
    int32_t p = g->iadjp[dst[e]] + fill[dst[e]]++;
    g->iadj[p] = src[e];
  }
  free(fill);
  return 0;
}

void orc_free_graph(orc_graph* g) {
  free(g->adjp);
  free(g->adj);
  free(g->w);
  free(g->iadjp);
  free(g->iadj);
  memset(g, 0, sizeof(*g));
}

/* Text format of read_input (gpucpg.cu:453-548): first line N, then N vertex
 * name lines (skipped), then one edge per line: the first quoted token is the
 * tail, the second the head; if the line holds a ',' the text between it and
 * ';' is the delay (std::stof), else the delay is 1.0.  Blank lines are
 * skipped here (the reference would throw on them). */
int orc_read_text(const char* path, int ignore_wgts, orc_graph* g) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  char* line = NULL;
  size_t lcap = 0;
  ssize_t len;
  int rc = 0;
  long n = -1;
  if ((len = getline(&line, &lcap, f)) <= 0) {
    rc = -2;
    goto done;
  }
  n = strtol(line, NULL, 10);
  if (n < 0 || n > INT_MAX - 2) {
    rc = -2;
    goto done;
  }
  for (long i = 0; i < n; ++i) {
    if (getline(&line, &lcap, f) < 0) {
      rc = -2;
      goto done;
    }
  }
  int32_t *src = NULL, *dst = NULL;
  float* wt = NULL;
  size_t cs = 0, cd = 0, cw = 0, m = 0;
  while ((len = getline(&line, &lcap, f)) >= 0) {
    char* q1 = strchr(line, '"');
    if (!q1) {
      int blank = 1;
      for (char* c = line; *c; ++c)
        if (*c != ' ' && *c != '\t' && *c != '\r' && *c != '\n') blank = 0;
      if (blank) continue;
      rc = -2;
      break;
    }
    char* q2 = strchr(q1 + 1, '"');
    char* q3 = q2 ? strchr(q2 + 1, '"') : NULL;
    char* q4 = q3 ? strchr(q3 + 1, '"') : NULL;
    if (!q4) {
      rc = -2;
      break;
    }
    long u = strtol(q1 + 1, NULL, 10);
    long v = strtol(q3 + 1, NULL, 10);
    float w = 1.0f;
    if (!ignore_wgts && strchr(line, ',')) {
      char* c = strchr(q4 + 1, ',');
      if (c) w = strtof(c + 1, NULL);
    }
    if (u < 0 || u >= n || v < 0 || v >= n) {
      rc = -2;
      break;
    }
    if (grow((void**)&src, &cs, m + 1, sizeof(int32_t)) ||
        grow((void**)&dst, &cd, m + 1, sizeof(int32_t)) ||
        grow((void**)&wt, &cw, m + 1, sizeof(float))) {
      rc = -1;
      break;
    }
    src[m] = (int32_t)u;
    dst[m] = (int32_t)v;
    wt[m] = w;
    ++m;
  }
  if (rc == 0) rc = orc_build_csr((int32_t)n, (int32_t)m, src, dst, wt, g);
  free(src);
  free(dst);
  free(wt);
done:
  free(line);
  fclose(f);
  return rc;
}

/* ---------------------------------------------------------------- SFXT */

/* CpGen::levelize (gpucpg.cu:21368-21407): Kahn over the fan-in CSR with the
 * out-degree as the dependency count; sinks are level 0. */
int32_t orc_levelize(const orc_graph* g, int32_t* order, int32_t* lvlp,
                     int32_t* level_of) {
  const int32_t n = g->n;
  int32_t* deps = malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
  if (!deps) return -1;
  int32_t tail = 0;
  for (int32_t v = 0; v < n; ++v) {
    deps[v] = g->adjp[v + 1] - g->adjp[v];
    if (level_of) level_of[v] = -1;
    if (deps[v] == 0) order[tail++] = v;
  }
  int32_t head = 0, levels = 0;
  lvlp[0] = 0;
  while (head < tail) {
    int32_t end = tail;
    for (; head < end; ++head) {
      int32_t v = order[head];
      if (level_of) level_of[v] = levels;
      for (int32_t e = g->iadjp[v]; e < g->iadjp[v + 1]; ++e) {
        int32_t u = g->iadj[e];
        if (--deps[u] == 0) order[tail++] = u;
      }
    }
    lvlp[++levels] = end;
  }
  free(deps);
  return levels;
}

static inline int32_t fixed_delay(float w) { return (int32_t)(w * ORC_SCALE_UP); }

/* relax_bu_step (gpucpg.cu:1167-1188); int32 adds wrap like the device's. */
void orc_relax(const orc_graph* g, const int32_t* order, const int32_t* lvlp,
               int32_t n_levels, int32_t* dist) {
  for (int32_t v = 0; v < g->n; ++v) dist[v] = INT_MAX;
  if (n_levels <= 0) return;
  for (int32_t i = lvlp[0]; i < lvlp[1]; ++i) dist[order[i]] = 0;
  for (int32_t l = 1; l < n_levels; ++l) {
    for (int32_t i = lvlp[l]; i < lvlp[l + 1]; ++i) {
      int32_t v = order[i];
      int32_t best = INT_MAX;
      for (int32_t e = g->adjp[v]; e < g->adjp[v + 1]; ++e) {
        int32_t c = (int32_t)((uint32_t)dist[g->adj[e]] + (uint32_t)fixed_delay(g->w[e]));
        if (c < best) best = c;
      }
      dist[v] = best;
    }
  }
}

/* update_successors_bu (gpucpg.cu:2606-2628). */
void orc_successors(const orc_graph* g, const int32_t* dist, int32_t* succ) {
  for (int32_t v = 0; v < g->n; ++v) {
    int32_t s = -1;
    for (int32_t e = g->adjp[v]; e < g->adjp[v + 1]; ++e) {
      int32_t nb = g->adj[e];
      int32_t c = (int32_t)((uint32_t)dist[nb] + (uint32_t)fixed_delay(g->w[e]));
      if (dist[v] == c && nb > s) s = nb;
    }
    succ[v] = s;
  }
}

int32_t orc_sfxt(const orc_graph* g, int32_t* dist, int32_t* succ,
                 int32_t* level_of) {
  int32_t* order = malloc(sizeof(int32_t) * (size_t)(g->n + 1));
  int32_t* lvlp = malloc(sizeof(int32_t) * (size_t)(g->n + 2));
  if (!order || !lvlp) {
    free(order);
    free(lvlp);
    return -1;
  }
  int32_t nl = orc_levelize(g, order, lvlp, level_of);
  orc_relax(g, order, lvlp, nl, dist);
  orc_successors(g, dist, succ);
  free(order);
  free(lvlp);
  return nl;
}

/* ---------------------------------------------------------------- PFXT */

static inline float dist_to_float(int32_t d) {
  return (float)d / (float)ORC_SCALE_UP;
}

/* new_slack = slack + dist_neighbor + wgt - dist_v, evaluated left to right
 * (gpucpg.cu:3271-3276). */
float orc_child_cost(float parent, int32_t dist_n, float w, int32_t dist_v) {
  float a = parent + dist_to_float(dist_n);
  float b = a + w;
  return b - dist_to_float(dist_v);
}

int32_t orc_deviation_csr(int32_t n, const int32_t* adjp, const int32_t* adj,
                          const float* w, const int32_t* succ,
                          const int32_t* dist, int32_t* offsets, int32_t* dsts,
                          float* deltas) {
  int32_t c = 0;
  for (int32_t v = 0; v < n; ++v) {
    offsets[v] = c;
    for (int32_t e = adjp[v]; e < adjp[v + 1]; ++e) {
      int32_t h = adj[e];
      if (h == succ[v] || dist[h] == INT_MAX || dist[v] == INT_MAX) continue;
      dsts[c] = h;
      deltas[c] = dist_to_float(dist[h]) + w[e] - dist_to_float(dist[v]);
      ++c;
    }
  }
  offsets[n] = c;
  return c;
}

/* --- min-heap of orc_node keyed by slack (std::priority_queue with the
 *     comparator a.slack > b.slack) */
typedef struct {
  orc_node* a;
  size_t n, cap;
} heap_t;

static int heap_push(heap_t* h, orc_node x) {
  if (grow((void**)&h->a, &h->cap, h->n + 1, sizeof(orc_node))) return -1;
  size_t i = h->n++;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (!(h->a[p].slack > x.slack)) break;
    h->a[i] = h->a[p];
    i = p;
  }
  h->a[i] = x;
  return 0;
}

static void heap_pop(heap_t* h) {
  orc_node x = h->a[--h->n];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1, r = l + 1, s = i;
    float best = x.slack;
    if (l < h->n && h->a[l].slack < best) {
      s = l;
      best = h->a[l].slack;
    }
    if (r < h->n && h->a[r].slack < best) s = r;
    if (s == i) break;
    h->a[i] = h->a[s];
    i = s;
  }
  if (h->n) h->a[i] = x;
}

static int cmp_node_slack(const void* pa, const void* pb) {
  const orc_node* a = pa;
  const orc_node* b = pb;
  if (a->slack < b->slack) return -1;
  if (a->slack > b->slack) return 1;
  return 0;
}

static int32_t* find_sources(const orc_graph* g, int32_t* ns) {
  int32_t* s = malloc(sizeof(int32_t) * (size_t)(g->n ? g->n : 1));
  *ns = 0;
  if (!s) return NULL;
  for (int32_t v = 0; v < g->n; ++v)
    if (g->iadjp[v + 1] == g->iadjp[v]) s[(*ns)++] = v;
  return s;
}

/* SEQUENTIAL (gpucpg.cu:21230-21300).  Like the reference, the children of
 * the top node are pushed before the top is popped, and every source is
 * seeded (the reference does not filter unreachable sources here). */
int64_t orc_sequential(const orc_graph* g, const int32_t* dist,
                       const int32_t* succ, int64_t k, orc_node* out) {
  heap_t h = {0};
  int32_t ns = 0;
  int32_t* srcs = find_sources(g, &ns);
  if (!srcs) return -1;
  for (int32_t i = 0; i < ns; ++i) {
    orc_node r = {0, -1, srcs[i], -1, 0, dist_to_float(dist[srcs[i]])};
    if (heap_push(&h, r)) return -1;
  }
  free(srcs);
  orc_node* paths = malloc(sizeof(orc_node) * (size_t)(k > 0 ? k : 1));
  if (!paths) return -1;
  int64_t np = 0;
  for (int64_t i = 0; i < k; ++i) {
    if (h.n == 0) break;
    orc_node top = h.a[0];
    paths[np++] = top;
    int32_t v = top.to;
    while (v != -1) {
      for (int32_t e = g->adjp[v]; e < g->adjp[v + 1]; ++e) {
        int32_t nb = g->adj[e];
        if (nb == succ[v]) continue;
        if (dist[nb] == INT_MAX) continue;
        orc_node c = {top.level + 1, v, nb, -1, 0,
                      orc_child_cost(top.slack, dist[nb], g->w[e], dist[v])};
        if (heap_push(&h, c)) return -1;
        paths[np - 1].num_children++;
      }
      v = succ[v];
    }
    heap_pop(&h);
  }
  free(h.a);
  /* stable ascending sort then the zero-cost filter (21323-21360) */
  qsort(paths, (size_t)np, sizeof(orc_node), cmp_node_slack);
  int64_t w = 0;
  for (int64_t i = 0; i < np; ++i)
    if (paths[i].slack != 0.0f) out[w++] = paths[i];
  free(paths);
  return w;
}

/* --- closure at a split */
typedef struct {
  orc_node* a;
  size_t n, cap;
} vec_t;

/* Pruning tables (orc_closure_topk_paths, prune != 0): each vertex's
 * deviation edges ordered by exact delta, and the least delta on each
 * vertex's suffix chain. */
typedef struct {
  int32_t* off;     /* n+1 row offsets */
  int32_t* edge;    /* fan-out edge of each deviation, rows ordered by delta */
  double* delta;    /* exact delta of each deviation */
  double* chain;    /* least delta on the suffix chain from v; +inf if none */
  double emax;      /* 2 max dist/10000 + max |w| */
} prune_t;

typedef struct {
  double d;
  int32_t e;
} dev_key;

static int cmp_dev(const void* pa, const void* pb) {
  const dev_key* a = pa;
  const dev_key* b = pb;
  if (a->d < b->d) return -1;
  if (a->d > b->d) return 1;
  return (a->e > b->e) - (a->e < b->e);
}

static void prune_free(prune_t* p) {
  free(p->off);
  free(p->edge);
  free(p->delta);
  free(p->chain);
}

static int prune_build(const orc_graph* g, const int32_t* dist, const int32_t* succ,
                       prune_t* p) {
  const int32_t n = g->n;
  memset(p, 0, sizeof(*p));
  p->off = malloc(sizeof(int32_t) * ((size_t)n + 1));
  p->edge = malloc(sizeof(int32_t) * (g->m ? (size_t)g->m : 1));
  p->delta = malloc(sizeof(double) * (g->m ? (size_t)g->m : 1));
  p->chain = malloc(sizeof(double) * (n ? (size_t)n : 1));
  dev_key* row = malloc(sizeof(dev_key) * (g->m ? (size_t)g->m : 1));
  int32_t* stack = malloc(sizeof(int32_t) * (n ? (size_t)n : 1));
  unsigned char* done = calloc(n ? (size_t)n : 1, 1);
  if (!p->off || !p->edge || !p->delta || !p->chain || !row || !stack || !done) {
    free(row);
    free(stack);
    free(done);
    prune_free(p);
    return -1;
  }
  double dmax = 0.0, wmax = 0.0;
  int32_t c = 0;
  for (int32_t v = 0; v < n; ++v) {
    p->off[v] = c;
    if (dist[v] != INT_MAX && fabs(dist[v] / 1e4) > dmax) dmax = fabs(dist[v] / 1e4);
    int32_t r = 0;
    for (int32_t e = g->adjp[v]; e < g->adjp[v + 1]; ++e) {
      const int32_t nb = g->adj[e];
      if (fabs((double)g->w[e]) > wmax) wmax = fabs((double)g->w[e]);
      if (nb == succ[v] || dist[nb] == INT_MAX) continue;
      row[r].d = ((double)dist[nb] - (double)dist[v]) / 1e4 + (double)g->w[e];
      row[r].e = e;
      ++r;
    }
    qsort(row, (size_t)r, sizeof(dev_key), cmp_dev);
    for (int32_t i = 0; i < r; ++i) {
      p->edge[c + i] = row[i].e;
      p->delta[c + i] = row[i].d;
    }
    c += r;
  }
  p->off[n] = c;
  p->emax = 2.0 * dmax + wmax;
  /* chain minima, memoised along successor chains (a cycle in succ cannot
   * occur: dist strictly decreases along it unless delays are zero, and the
   * walk stops at vertices already on the stack) */
  for (int32_t v = 0; v < n; ++v) {
    if (done[v]) continue;
    int32_t top = 0;
    for (int32_t u = v; u >= 0 && !done[u]; u = succ[u]) {
      done[u] = 2;
      stack[top++] = u;
    }
    while (top > 0) {
      const int32_t u = stack[--top];
      double m = p->off[u + 1] > p->off[u] ? p->delta[p->off[u]] : INFINITY;
      const int32_t s = succ[u];
      if (s >= 0 && done[s] == 1 && p->chain[s] < m) m = p->chain[s];
      p->chain[u] = m;
      done[u] = 1;
    }
  }
  free(row);
  free(stack);
  free(done);
  return 0;
}

static inline double prune_bound(const prune_t* p, float s) {
  return 0x1p-20 * (fabs((double)s) + p->emax);
}

/* Accept every path whose cost is <= lim, expanding accepted paths along their
 * suffix chain.  Returns 0 on success, 1 if more than cap paths were accepted,
 * -1 on allocation failure.  *complete is set when no child was rejected.
 * With pr, rows and chain tails that cannot hold a child costing <= lim are
 * skipped (counted as rejected). */
static int closure(const orc_graph* g, const int32_t* dist, const int32_t* succ,
                   const int32_t* srcs, int32_t ns, float lim, size_t cap,
                   const prune_t* pr, vec_t* acc, int* complete) {
  acc->n = 0;
  *complete = 1;
  for (int32_t i = 0; i < ns; ++i) {
    orc_node r = {0, -1, srcs[i], -1, 0, dist_to_float(dist[srcs[i]])};
    if (!(r.slack <= lim)) {
      *complete = 0;
      continue;
    }
    if (grow((void**)&acc->a, &acc->cap, acc->n + 1, sizeof(orc_node))) return -1;
    acc->a[acc->n++] = r;
  }
  for (size_t i = 0; i < acc->n; ++i) {
    orc_node p = acc->a[i];
    if (pr) {
      const double room = (double)lim - (double)p.slack + prune_bound(pr, p.slack);
      for (int32_t v = p.to; v != -1; v = succ[v]) {
        if (pr->chain[v] > room) {
          if (pr->chain[v] != INFINITY) *complete = 0;
          break;
        }
        for (int32_t j = pr->off[v]; j < pr->off[v + 1]; ++j) {
          if (pr->delta[j] > room) {
            *complete = 0;
            break;
          }
          const int32_t e = pr->edge[j], nb = g->adj[e];
          float c = orc_child_cost(p.slack, dist[nb], g->w[e], dist[v]);
          if (!(c <= lim)) {
            *complete = 0;
            continue;
          }
          if (acc->n >= cap) return 1;
          if (grow((void**)&acc->a, &acc->cap, acc->n + 1, sizeof(orc_node))) return -1;
          orc_node x = {p.level + 1, v, nb, (int32_t)i, 0, c};
          acc->a[acc->n++] = x;
        }
      }
      continue;
    }
    for (int32_t v = p.to; v != -1; v = succ[v]) {
      for (int32_t e = g->adjp[v]; e < g->adjp[v + 1]; ++e) {
        int32_t nb = g->adj[e];
        if (nb == succ[v] || dist[nb] == INT_MAX) continue;
        float c = orc_child_cost(p.slack, dist[nb], g->w[e], dist[v]);
        if (!(c <= lim)) {
          *complete = 0;
          continue;
        }
        if (acc->n >= cap) return 1;
        if (grow((void**)&acc->a, &acc->cap, acc->n + 1, sizeof(orc_node))) return -1;
        orc_node x = {p.level + 1, v, nb, (int32_t)i, 0, c};
        acc->a[acc->n++] = x;
      }
    }
  }
  return 0;
}

static size_t count_le(const vec_t* acc, float t) {
  size_t c = 0;
  for (size_t i = 0; i < acc->n; ++i)
    if (acc->a[i].slack <= t && acc->a[i].slack != 0.0f) ++c;
  return c;
}

typedef struct {
  float slack;
  int64_t idx;
} rank_t;

static int cmp_rank(const void* pa, const void* pb) {
  const rank_t* a = pa;
  const rank_t* b = pb;
  if (a->slack < b->slack) return -1;
  if (a->slack > b->slack) return 1;
  return (a->idx > b->idx) - (a->idx < b->idx);
}

static int cmp_float(const void* pa, const void* pb) {
  float a = *(const float*)pa, b = *(const float*)pb;
  return (a > b) - (a < b);
}

/* Roots in source-id order with finite distance; with ref_roots, the
 * reference's initial-split truncation applied (gpucpg.cu:19136-19179). */
static int32_t* seed_roots(const orc_graph* g, const int32_t* dist, int ref_roots,
                           int32_t* ns_out) {
  int32_t ns = 0;
  int32_t* all = find_sources(g, &ns);
  if (!all) return NULL;
  int32_t r = 0;
  for (int32_t i = 0; i < ns; ++i)
    if (dist[all[i]] != INT_MAX) all[r++] = all[i];
  if (ref_roots && r > 0) {
    float* sorted = malloc(sizeof(float) * (size_t)r);
    if (!sorted) {
      free(all);
      return NULL;
    }
    for (int32_t i = 0; i < r; ++i) sorted[i] = dist_to_float(dist[all[i]]);
    qsort(sorted, (size_t)r, sizeof(float), cmp_float);
    const float perc = 0.005f;
    const float split = sorted[(size_t)(perc * r)];
    const int32_t n_short = (int32_t)(perc * r + 1);
    free(sorted);
    int32_t kept = 0, short_seen = 0;
    for (int32_t i = 0; i < r; ++i) {
      float c = dist_to_float(dist[all[i]]);
      if (c > split) {
        all[kept++] = all[i];
      } else if (short_seen < n_short) {
        ++short_seen;
        all[kept++] = all[i];
      }
    }
    r = kept;
  }
  *ns_out = r;
  return all;
}

int64_t orc_closure_topk(const orc_graph* g, const int32_t* dist,
                         const int32_t* succ, int64_t k, orc_node* out,
                         float* split_out) {
  return orc_closure_topk_ex(g, dist, succ, k, 0, out, split_out);
}

int64_t orc_closure_topk_ex(const orc_graph* g, const int32_t* dist,
                            const int32_t* succ, int64_t k, int ref_roots,
                            orc_node* out, float* split_out) {
  return orc_closure_topk_paths(g, dist, succ, k, ref_roots, 1, out, split_out, NULL, NULL, 0);
}

int64_t orc_closure_topk_paths(const orc_graph* g, const int32_t* dist,
                               const int32_t* succ, int64_t k, int ref_roots, int prune,
                               orc_node* out, float* split_out, int64_t* path_off,
                               int32_t* verts, int64_t verts_cap) {
  if (k <= 0) {
    if (path_off) path_off[0] = 0;
    return 0;
  }
  int32_t ns = 0;
  int32_t* srcs = seed_roots(g, dist, ref_roots, &ns);
  if (!srcs) return -1;
  float c0 = INFINITY, dmax = 1.0f;
  for (int32_t i = 0; i < ns; ++i) {
    float c = dist_to_float(dist[srcs[i]]);
    if (c < c0) c0 = c;
  }
  for (int32_t v = 0; v < g->n; ++v)
    if (dist[v] != INT_MAX && fabsf(dist_to_float(dist[v])) > dmax)
      dmax = fabsf(dist_to_float(dist[v]));
  vec_t acc = {0};
  if (c0 == INFINITY) {
    free(srcs);
    if (path_off) path_off[0] = 0;
    return 0;
  }
  prune_t pt;
  const prune_t* pr = NULL;
  if (prune) {
    if (prune_build(g, dist, succ, &pt)) {
      free(srcs);
      return -1;
    }
    pr = &pt;
  }
  /* Children may cost a few ulps less than their parent after rounding; the
   * margin keeps such descendants in the closure. */
  size_t cap = (size_t)(8 * k + 4096);
  float lo = 0.0f, hi = 0.0f, d = 1e-4f * fmaxf(1.0f, fabsf(c0)), t = c0;
  int have_hi = 0, complete = 0, rc = 0, done = 0;
  for (int iter = 0; iter < 400 && !done; ++iter) {
    t = c0 + d;
    float m = fmaxf(fmaxf(fabsf(t), 2.0f * dmax), 1.0f) * 0x1p-17f;
    rc = closure(g, dist, succ, srcs, ns, t + m, cap, pr, &acc, &complete);
    if (rc < 0) break;
    if (rc == 1) { /* over the cap: bisect down, or grow the cap on a tie wall */
      hi = d;
      have_hi = 1;
      float mid = 0.5f * (lo + hi);
      if (c0 + mid == c0 + lo || c0 + mid == c0 + hi) {
        cap *= 4;
      } else {
        d = mid;
      }
      continue;
    }
    size_t c = count_le(&acc, t);
    if (c >= (size_t)k || complete) {
      done = 1;
      break;
    }
    lo = d;
    if (have_hi) {
      float mid = 0.5f * (lo + hi);
      if (c0 + mid == c0 + lo || c0 + mid == c0 + hi) {
        d = hi;
        cap *= 4;
      } else {
        d = mid;
      }
    } else {
      d = 2.0f * d;
    }
  }
  if (!done && rc == 0) rc = -1;
  free(srcs);
  if (pr) prune_free(&pt);
  if (rc != 0) {
    free(acc.a);
    return -1;
  }
  if (split_out) *split_out = t;
  rank_t* r = malloc(sizeof(rank_t) * (acc.n ? acc.n : 1));
  int64_t* pos = malloc(sizeof(int64_t) * (acc.n ? acc.n : 1));
  if (!r || !pos) {
    free(r);
    free(pos);
    free(acc.a);
    return -1;
  }
  size_t nr = 0;
  for (size_t i = 0; i < acc.n; ++i) {
    pos[i] = -1;
    if (acc.a[i].slack != 0.0f) {
      r[nr].slack = acc.a[i].slack;
      r[nr].idx = (int64_t)i;
      ++nr;
    }
  }
  qsort(r, nr, sizeof(rank_t), cmp_rank);
  int64_t nout = (int64_t)nr < k ? (int64_t)nr : k;
  for (int64_t j = 0; j < nout; ++j) pos[r[j].idx] = j;
  for (int64_t j = 0; j < nout; ++j) {
    orc_node x = acc.a[r[j].idx];
    x.parent = x.parent >= 0 ? (int32_t)pos[x.parent] : -1;
    out[j] = x;
  }
  int64_t status = nout;
  if (path_off) {
    /* vertex sequence: deviations from the root down, then the chain walk
     * that leaves the chain at each deviation's tail for its head */
    int64_t w = 0;
    int32_t* devs = NULL;
    size_t dcap = 0;
    path_off[0] = 0;
    for (int64_t j = 0; j < nout && status >= 0; ++j) {
      size_t nd = 0;
      int64_t cur = r[j].idx;
      while (acc.a[cur].parent >= 0) {
        if (grow((void**)&devs, &dcap, 2 * (nd + 1), sizeof(int32_t))) {
          status = -1;
          break;
        }
        devs[2 * nd] = acc.a[cur].from;
        devs[2 * nd + 1] = acc.a[cur].to;
        ++nd;
        cur = acc.a[cur].parent;
      }
      if (status < 0) break;
      int32_t v = acc.a[cur].to;
      size_t d = nd;
      while (v >= 0) {
        if (w >= verts_cap) {
          status = -2;
          break;
        }
        verts[w++] = v;
        if (d > 0 && devs[2 * (d - 1)] == v) {
          v = devs[2 * (d - 1) + 1];
          --d;
        } else {
          v = succ[v];
        }
      }
      path_off[j + 1] = w;
    }
    free(devs);
  }
  free(r);
  free(pos);
  free(acc.a);
  return status;
}

/* ------------------------------------------------------------ BVSS checks */

void orc_bfs_levels(int32_t n, const int32_t* adjp, const int32_t* adj,
                    const int32_t* sinks, int32_t n_sinks, int32_t* levels) {
  /* fan-in lists, then a plain queue BFS from the sinks */
  int32_t* ip = calloc((size_t)n + 1, sizeof(int32_t));
  int32_t* ia = malloc(sizeof(int32_t) * (adjp[n] ? (size_t)adjp[n] : 1));
  int32_t* fill = malloc(sizeof(int32_t) * (n ? (size_t)n : 1));
  int32_t* q = malloc(sizeof(int32_t) * (n ? (size_t)n : 1));
  for (int32_t u = 0; u < n; ++u)
    for (int32_t e = adjp[u]; e < adjp[u + 1]; ++e) ip[adj[e] + 1]++;
  for (int32_t v = 0; v < n; ++v) ip[v + 1] += ip[v];
  for (int32_t v = 0; v < n; ++v) fill[v] = ip[v];
  for (int32_t u = 0; u < n; ++u)
    for (int32_t e = adjp[u]; e < adjp[u + 1]; ++e) ia[fill[adj[e]]++] = u;
  for (int32_t v = 0; v < n; ++v) levels[v] = -1;
  int32_t qh = 0, qt = 0;
  for (int32_t i = 0; i < n_sinks; ++i) {
    const int32_t t = sinks[i];
    if (t < 0 || t >= n || levels[t] >= 0) continue;
    levels[t] = 0;
    q[qt++] = t;
  }
  while (qh < qt) {
    const int32_t v = q[qh++];
    for (int32_t e = ip[v]; e < ip[v + 1]; ++e) {
      const int32_t u = ia[e];
      if (levels[u] < 0) {
        levels[u] = levels[v] + 1;
        q[qt++] = u;
      }
    }
  }
  free(ip);
  free(ia);
  free(fill);
  free(q);
}

static int cmp_pair(const void* a, const void* b) {
  const int32_t* x = (const int32_t*)a;
  const int32_t* y = (const int32_t*)b;
  if (x[0] != y[0]) return x[0] < y[0] ? -1 : 1;
  if (x[1] != y[1]) return x[1] < y[1] ? -1 : 1;
  return 0;
}

int64_t orc_adev_pairs(int32_t n, const int32_t* adjp, const int32_t* adj,
                       const int32_t* succ, const int32_t* sources, int32_t n_sources,
                       int32_t* pairs, int64_t max_pairs) {
  unsigned char* is_src = calloc(n ? (size_t)n : 1, 1);
  for (int32_t i = 0; i < n_sources; ++i)
    if (sources[i] >= 0 && sources[i] < n) is_src[sources[i]] = 1;
  int64_t cap = adjp[n] ? adjp[n] : 1;
  int32_t* all = malloc(sizeof(int32_t) * 2 * (size_t)cap);
  int64_t cnt = 0;
  for (int32_t u = 0; u < n; ++u) {
    if (!is_src[u]) continue;
    for (int32_t e = adjp[u]; e < adjp[u + 1]; ++e) {
      if (adj[e] == succ[u]) continue;
      all[2 * cnt] = u;
      all[2 * cnt + 1] = adj[e];
      ++cnt;
    }
  }
  qsort(all, (size_t)cnt, 2 * sizeof(int32_t), cmp_pair);
  int64_t uniq = 0;
  for (int64_t i = 0; i < cnt; ++i) {
    if (uniq > 0 && all[2 * i] == all[2 * (uniq - 1)] && all[2 * i + 1] == all[2 * (uniq - 1) + 1])
      continue;
    all[2 * uniq] = all[2 * i];
    all[2 * uniq + 1] = all[2 * i + 1];
    ++uniq;
  }
  for (int64_t i = 0; i < uniq && i < max_pairs; ++i) {
    pairs[2 * i] = all[2 * i];
    pairs[2 * i + 1] = all[2 * i + 1];
  }
  free(all);
  free(is_src);
  return uniq;
}
