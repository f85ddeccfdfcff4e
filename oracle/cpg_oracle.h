/*
 * CPU oracle for the critical-path-generation hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the gpu-cpg_b200 library,
 * its C ABI or its C++ shim) links, loads or calls this code.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and only as
 * the checker or the timed CPU port.
 *
 * It restates, in plain C, the reference gpu-cpg algorithm for this path
 * (file:line cites are into the reference tree, gpucpg/gpucpg.cu unless noted):
 *   - text ingestion                      CpGen::read_input        453-548
 *   - reverse levelisation (CPU Kahn)     CpGen::levelize          21368-21407
 *   - fixed-point relax                   relax_bu_step            1167-1188
 *   - successor (max id among arg-mins)   update_successors_bu     2606-2628
 *   - root seeding                        report_paths             18502-18520
 *   - child cost, left-to-right fp32      expand_short_pile        3234-3306
 *   - SEQUENTIAL priority-queue PFXT      report_paths             21230-21300
 *   - closure at a split (the set GPG's   SHORT_LONG driver        19134-20850
 *     short pile holds when it stops:
 *     every path whose ancestors and itself cost <= split)
 *   - zero-cost filter + ascending sort   report_paths             21323-21360
 *
 * Division: (float)dist / 10000 is IEEE round-to-nearest here (the reference's
 * host-side root seeding uses the same); the reference's device kernels are
 * built with --use_fast_math, so device-side quotients may differ in the last
 * bit.  Parity against the device is therefore exact only where the device is
 * asked for IEEE division, and within tolerance otherwise.
 */
#ifndef CPG_ORACLE_H
#define CPG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_SCALE_UP 10000

typedef struct {
  int32_t n, m;
  int32_t* adjp;   /* fan-out row offsets, n+1 */
  int32_t* adj;    /* fan-out heads, m */
  float* w;        /* fan-out delays, m */
  int32_t* iadjp;  /* fan-in row offsets, n+1 */
  int32_t* iadj;   /* fan-in tails, m */
} orc_graph;

/* PfxtNode (gpucpg.cuh:74-107) with a parent index valid in the output list. */
typedef struct {
  int32_t level, from, to, parent, num_children;
  float slack;
} orc_node;

/* Parse the reference's text format ("N", N name lines, "u" -> "v"[, w];).
 * Returns 0 on success, -1 on I/O error, -2 on a malformed line. */
int orc_read_text(const char* path, int ignore_wgts, orc_graph* g);

/* Build both CSRs from an edge list in file order (row order = file order). */
int orc_build_csr(int32_t n, int32_t m, const int32_t* src, const int32_t* dst,
                  const float* w, orc_graph* g);
void orc_free_graph(orc_graph* g);

/* Reverse levelisation: sinks are level 0.  order[] lists vertices level by
 * level, lvlp[0..n_levels] are the level offsets.  Vertices never levelled
 * (on or above a cycle) are left out.  Returns the number of levels. */
int32_t orc_levelize(const orc_graph* g, int32_t* order, int32_t* lvlp,
                     int32_t* level_of);

/* dist[v] = min over out-edges (v,n) of dist[n] + (int)(w*10000.0f). */
void orc_relax(const orc_graph* g, const int32_t* order, const int32_t* lvlp,
               int32_t n_levels, int32_t* dist);
/* succ[v] = max n with dist[v] == dist[n] + (int)(w*10000.0f), else -1. */
void orc_successors(const orc_graph* g, const int32_t* dist, int32_t* succ);
/* All three in one call. */
int32_t orc_sfxt(const orc_graph* g, int32_t* dist, int32_t* succ,
                 int32_t* level_of);

/* The reference's SEQUENTIAL path: K pops of a min-heap, children pushed
 * before the pop exactly as gpucpg.cu:21249-21296 does.  Writes at most k
 * nodes sorted ascending with zero-cost nodes removed; returns the count. */
int64_t orc_sequential(const orc_graph* g, const int32_t* dist,
                       const int32_t* succ, int64_t k, orc_node* out);

/* Closure at a split: the k smallest non-zero costs among all paths, found by
 * expanding every path whose cost is <= split + margin with the reference's
 * suffix-chain walk and raising the split until >= k paths cost <= split.
 * Writes at most k nodes sorted ascending, parents indexed into out[] (-1 if
 * the parent is a root or not in the list).  Returns the count, or -1 on
 * allocation failure.  *split_out receives the final split. */
int64_t orc_closure_topk(const orc_graph* g, const int32_t* dist,
                         const int32_t* succ, int64_t k, orc_node* out,
                         float* split_out);

/* Same, with the reference G-PathGen's root seeding when ref_roots != 0:
 * the roots are sorted, split = cost at index (size_t)(0.005f * R), the short
 * pile is resized to (int)(0.005f * R + 1) after removing the roots above the
 * split, so roots at or below the split beyond that count (in source-id
 * order) are dropped (gpucpg.cu:19134-19179). */
int64_t orc_closure_topk_ex(const orc_graph* g, const int32_t* dist,
                            const int32_t* succ, int64_t k, int ref_roots,
                            orc_node* out, float* split_out);

/* orc_closure_topk_ex with two additions.
 *
 * prune != 0 gives the same set faster.  Each vertex's deviation edges are
 * ordered by their exact cost delta (dist_head - dist_tail)/10000 + w in
 * double precision, and each vertex keeps the least delta on its suffix
 * chain.  A parent of cost s stops scanning a row, or walking its chain, once
 * s + delta exceeds the limit by more than a float-rounding bound
 * E = 2^-20 (|s| + 2 max dist/10000 + max |w|).  The fp32 child cost
 * ((s + a) + w) - b is at least the exact s + delta minus about 6 ulps of
 * those magnitudes, so no child that could cost <= the limit is skipped.
 * The closure's set, the split search and the float costs are unchanged;
 * only the work per accepted path drops from the whole chain times the
 * degree to the children that are accepted plus a few.
 *
 * When path_off is not NULL, the vertex sequence of returned path j (source to
 * sink: the root's source, the suffix chain up to each deviation's tail, the
 * deviation's head, and so on) is written to verts[path_off[j] ..
 * path_off[j+1]).  path_off holds k+1 entries.  At most verts_cap vertices are
 * written; the call returns -2 if they do not fit.
 *
 * Returns the number of paths, -1 on allocation failure, -2 if verts_cap is
 * too small. */
int64_t orc_closure_topk_paths(const orc_graph* g, const int32_t* dist,
                               const int32_t* succ, int64_t k, int ref_roots, int prune,
                               orc_node* out, float* split_out, int64_t* path_off,
                               int32_t* verts, int64_t verts_cap);

/* Parameters of the seeded levelised DAG (field order of the product's
 * cpg_gen_params, so the same settings describe both generators). */
typedef struct {
  uint64_t seed;
  int32_t n_pins, n_levels, n_first, n_last, level_span;
  int32_t degree_kind; /* 0: uniform {deg_lo..deg_hi}; 1: geometric of mean deg_mean */
  int32_t deg_lo, deg_hi;
  double deg_mean;
  int32_t deg_cap;
  int32_t weight_kind; /* 0: fp32 uniform [w_lo, w_hi]; 1: integers {iw_lo..iw_hi} */
  float w_lo, w_hi;
  int32_t iw_lo, iw_hi;
  int32_t add_virtual; /* super-source n_pins and super-sink n_pins+1 */
} orc_gen_params;

/* Seeded levelised DAG (cpg_gen.c).  On success *src, *dst, *w hold *m_out
 * edges (free each with orc_free) and *n_out vertices; returns 0, -1 on
 * allocation failure, -2 on bad parameters. */
int orc_generate(const orc_gen_params* p, int32_t* n_out, int64_t* m_out, int32_t** src,
                 int32_t** dst, float** w);
void orc_free(void* p);

/* Deviation edges of every vertex: fan-out edges whose head is not the
 * successor and whose head and tail distances are finite, with their cost
 * delta dist_head/10000 + w - dist_tail/10000 (build_compact_static_deviation_csr,
 * tc_pfxt_candidates.cuh:713-750).  offsets has n+1 entries; dsts/deltas at
 * most m.  Returns the number of deviation edges. */
int32_t orc_deviation_csr(int32_t n, const int32_t* adjp, const int32_t* adj,
                          const float* w, const int32_t* succ,
                          const int32_t* dist, int32_t* offsets, int32_t* dsts,
                          float* deltas);

/* Cost of one child, left to right as expand_short_pile writes it. */
float orc_child_cost(float parent, int32_t dist_n, float w, int32_t dist_v);

/* Pull BFS levels from the sinks over a fan-out CSR: a vertex gets level L+1
 * the first time one of its heads has level L; -1 if never reached
 * (run_scalar_bvss_pull_bfs_levels, tc_sfxt_bvss.cuh:418-495, restated on the
 * CSR instead of the packed slices). */
void orc_bfs_levels(int32_t n, const int32_t* adjp, const int32_t* adj,
                    const int32_t* sinks, int32_t n_sinks, int32_t* levels);

/* Distinct deviation pairs (u, v) leaving the sources: fan-out edges u -> v
 * of a source u with v != succ[u] (discover_pairs_for_sources,
 * tc_pfxt_bvss.cuh:582-636).  Writes at most max_pairs pairs sorted by
 * (u, v) as 2 int32 each; returns the full count. */
int64_t orc_adev_pairs(int32_t n, const int32_t* adjp, const int32_t* adj,
                       const int32_t* succ, const int32_t* sources, int32_t n_sources,
                       int32_t* pairs, int64_t max_pairs);

#ifdef __cplusplus
}
#endif
#endif
