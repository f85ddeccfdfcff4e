/*
 * Seeded levelised DAG generator, restated for the CPU oracle.
 *
 * TEST AND BENCH INFRASTRUCTURE ONLY.  The product library has its own
 * generator (cpg_dag_generate); this restatement lets the oracle's golden
 * pins, the tests' oracle side and bench.py's reference arm build the same
 * synthetic workloads without loading the product.  tests/test_oracle.py
 * checks that both give identical edge lists for the same parameters.
 *
 * The workload shape follows the reference's text-format conventions
 * (read_input, gpucpg/gpucpg.cu:453-548): pins in levels, edges from level i
 * to a uniformly chosen level in i+1..i+span, a repair pass so that only
 * level-0 pins are sources, and an explicit virtual super-source (id n_pins)
 * and super-sink (id n_pins+1) joined by zero-delay edges.
 *
 * Random numbers: MT19937-64 (Matsumoto and Nishimura, ACM TOMACS 2000; the
 * engine C++ names std::mt19937_64), default-seeded with `seed`.  uniform()
 * takes the top 53 bits of a draw; below(n) scales uniform() by n.
 */
#include "cpg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MT_N 312
#define MT_M 156

typedef struct {
  uint64_t s[MT_N];
  int i;
} mt64;

static void mt_seed(mt64* r, uint64_t seed) {
  r->s[0] = seed;
  for (int i = 1; i < MT_N; ++i)
    r->s[i] = 6364136223846793005ULL * (r->s[i - 1] ^ (r->s[i - 1] >> 62)) + (uint64_t)i;
  r->i = MT_N;
}

static uint64_t mt_next(mt64* r) {
  static const uint64_t A = 0xB5026F5AA96619E9ULL, UP = 0xFFFFFFFF80000000ULL,
                        LO = 0x7FFFFFFFULL;
  if (r->i >= MT_N) {
    for (int k = 0; k < MT_N; ++k) {
      const uint64_t x = (r->s[k] & UP) | (r->s[(k + 1) % MT_N] & LO);
      r->s[k] = r->s[(k + MT_M) % MT_N] ^ (x >> 1) ^ ((x & 1) ? A : 0);
    }
    r->i = 0;
  }
  uint64_t x = r->s[r->i++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}

static double uniform(mt64* r) { return (double)(mt_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static int64_t below(mt64* r, int64_t n) { return (int64_t)(uniform(r) * (double)n) % n; }

typedef struct {
  int32_t *src, *dst;
  float* w;
  int64_t m, cap;
} edges_t;

static int push_edge(edges_t* e, int32_t u, int32_t v, float w) {
  if (e->m == e->cap) {
    int64_t c = e->cap ? 2 * e->cap : 1 << 16;
    int32_t* s = realloc(e->src, sizeof(int32_t) * (size_t)c);
    if (s) e->src = s;
    int32_t* d = realloc(e->dst, sizeof(int32_t) * (size_t)c);
    if (d) e->dst = d;
    float* x = realloc(e->w, sizeof(float) * (size_t)c);
    if (x) e->w = x;
    if (!s || !d || !x) return -1;
    e->cap = c;
  }
  e->src[e->m] = u;
  e->dst[e->m] = v;
  e->w[e->m] = w;
  ++e->m;
  return 0;
}

static int32_t sample_degree(mt64* r, const orc_gen_params* p) {
  if (p->degree_kind == 0) return p->deg_lo + (int32_t)below(r, p->deg_hi - p->deg_lo + 1);
  const double q = 1.0 - 1.0 / p->deg_mean;
  if (q <= 0.0) return 1;
  double u = uniform(r);
  if (u <= 0.0) u = 1e-300;
  int64_t k = 1 + (int64_t)floor(log(u) / log(q));
  if (k > p->deg_cap) k = p->deg_cap;
  return (int32_t)k;
}

static float sample_weight(mt64* r, const orc_gen_params* p) {
  if (p->weight_kind == 1) return (float)(p->iw_lo + below(r, p->iw_hi - p->iw_lo + 1));
  return p->w_lo + (p->w_hi - p->w_lo) * (float)uniform(r);
}

/* Open-addressed set of the heads already chosen for one tail: at least four
 * slots per possible head keep it sparse. */
typedef struct {
  int32_t* key;
  int32_t* used;
  uint32_t mask;
  int n_used;
} head_set;

static int set_insert(head_set* s, int32_t v) {
  uint32_t h = ((uint32_t)v * 2654435761u) & s->mask;
  while (s->key[h] != -1) {
    if (s->key[h] == v) return 0;
    h = (h + 1) & s->mask;
  }
  s->key[h] = v;
  s->used[s->n_used++] = (int32_t)h;
  return 1;
}

static void set_clear(head_set* s) {
  for (int i = 0; i < s->n_used; ++i) s->key[s->used[i]] = -1;
  s->n_used = 0;
}

int orc_generate(const orc_gen_params* p, int32_t* n_out, int64_t* m_out, int32_t** src,
                 int32_t** dst, float** w) {
  *src = *dst = NULL;
  *w = NULL;
  if (p->n_levels < 2 || p->n_first < 1 || p->n_last < 1 ||
      p->n_pins < p->n_first + p->n_last + (p->n_levels - 2) || p->level_span < 1)
    return -2;
  if (p->degree_kind == 0 && (p->deg_lo < 1 || p->deg_hi < p->deg_lo)) return -2;
  if (p->degree_kind == 1 && (p->deg_mean < 1.0 || p->deg_cap < 1)) return -2;
  const int32_t max_deg = p->degree_kind == 0 ? p->deg_hi : p->deg_cap;
  uint32_t slots = 64;
  while (slots < 4u * (uint32_t)max_deg) slots *= 2;
  mt64* r = malloc(sizeof(mt64));
  head_set hs = {malloc(sizeof(int32_t) * slots), malloc(sizeof(int32_t) * slots), slots - 1, 0};
  const int32_t L = p->n_levels, np = p->n_pins;
  int64_t* lstart = malloc(sizeof(int64_t) * (size_t)(L + 1));
  int32_t* perm = malloc(sizeof(int32_t) * (size_t)np);
  int32_t* chosen = malloc(sizeof(int32_t) * (size_t)max_deg);
  unsigned char* has_in = calloc((size_t)np, 1);
  edges_t e = {0};
  int rc = -1;
  if (!r || !hs.key || !hs.used || !lstart || !perm || !chosen || !has_in) goto out;
  mt_seed(r, p->seed);
  memset(hs.key, 0xff, sizeof(int32_t) * slots);
  const int64_t mid = (int64_t)np - p->n_first - p->n_last;
  lstart[0] = 0;
  for (int32_t l = 0; l < L; ++l) {
    int64_t sz;
    if (l == 0)
      sz = p->n_first;
    else if (l == L - 1)
      sz = p->n_last;
    else
      sz = mid / (L - 2) + ((l - 1) < (mid % (L - 2)) ? 1 : 0);
    lstart[l + 1] = lstart[l] + sz;
  }
  /* the i-th pin in level order is perm[i] (Fisher-Yates from the top) */
  for (int32_t i = 0; i < np; ++i) perm[i] = i;
  for (int32_t i = np - 1; i > 0; --i) {
    const int32_t j = (int32_t)below(r, i + 1);
    const int32_t t = perm[i];
    perm[i] = perm[j];
    perm[j] = t;
  }
  for (int32_t l = 0; l + 1 < L; ++l) {
    const int32_t lmax = (L - 1 < l + p->level_span) ? L - 1 : l + p->level_span;
    const int64_t span_pins = lstart[lmax + 1] - lstart[l + 1];
    for (int64_t i = lstart[l]; i < lstart[l + 1]; ++i) {
      const int32_t u = perm[i];
      int32_t deg = sample_degree(r, p);
      if (deg > span_pins) deg = (int32_t)span_pins;
      int nc = 0;
      for (int32_t k = 0; k < deg; ++k) {
        for (int attempt = 0; attempt < 64; ++attempt) {
          const int32_t tl = l + 1 + (int32_t)below(r, lmax - l);
          const int64_t sz = lstart[tl + 1] - lstart[tl];
          const int32_t v = perm[lstart[tl] + below(r, sz)];
          if (set_insert(&hs, v)) {
            chosen[nc++] = v;
            break;
          }
        }
      }
      set_clear(&hs);
      for (int c = 0; c < nc; ++c) {
        if (push_edge(&e, u, chosen[c], sample_weight(r, p))) goto out;
        has_in[chosen[c]] = 1;
      }
    }
  }
  /* repair: every pin above level 0 gets an in-edge from the level below */
  for (int32_t l = 1; l < L; ++l) {
    for (int64_t i = lstart[l]; i < lstart[l + 1]; ++i) {
      const int32_t v = perm[i];
      if (has_in[v]) continue;
      const int64_t sz = lstart[l] - lstart[l - 1];
      const int32_t u = perm[lstart[l - 1] + below(r, sz)];
      if (push_edge(&e, u, v, sample_weight(r, p))) goto out;
      has_in[v] = 1;
    }
  }
  if (p->add_virtual) {
    for (int64_t i = lstart[0]; i < lstart[1]; ++i)
      if (push_edge(&e, np, perm[i], 0.0f)) goto out;
    for (int64_t i = lstart[L - 1]; i < lstart[L]; ++i)
      if (push_edge(&e, perm[i], np + 1, 0.0f)) goto out;
  }
  *n_out = np + (p->add_virtual ? 2 : 0);
  *m_out = e.m;
  *src = e.src;
  *dst = e.dst;
  *w = e.w;
  e.src = e.dst = NULL;
  e.w = NULL;
  rc = 0;
out:
  free(e.src);
  free(e.dst);
  free(e.w);
  free(r);
  free(hs.key);
  free(hs.used);
  free(lstart);
  free(perm);
  free(chosen);
  free(has_in);
  return rc;
}

void orc_free(void* p) { free(p); }
