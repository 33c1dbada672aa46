/*
 * Multi-core CPU list ranking -- TEST INFRASTRUCTURE and CPU BASELINE ONLY.
 *
 * A shared-memory (POSIX threads) restatement, over all host cores, of two
 * of the reference's distributed list rankers, so that the GPU library has a
 * CPU baseline beside the sequential GatherChase when the reference's MPI
 * binary cannot be built.  The product library never links or calls this
 * file.
 *
 *  - cpu_sparse_ruling_set: the reference's sparse ruling set
 *    (lib/kascade/sparse_ruling_set.cpp:45-331) in its post-invert form
 *    (chase forward from the rulers, no list reversal): every leaf and every
 *    root is a ruler, further rulers are sampled (a counter hash stands in
 *    for the shuffled permutation of sparse_ruling_set.cpp:106-136); each
 *    ruler's chain is walked until the next ruler or root, each reached
 *    element recording (ruler, distance from the ruler) in place of
 *    (succ, rank) as work_on_item does (sparse_ruling_set.cpp:147-273); the
 *    ruler sublist is ranked recursively (sparse_ruling_set.cpp:335-392, base
 *    case: the sequential chase); finally each element takes its ruler's
 *    root and rank (ruler_propagation.hpp:148-256, pull mode): rank =
 *    rank(ruler) - distance from the ruler.  Each thread walks several chains
 *    at once, so that their random reads overlap.
 *  - cpu_pointer_doubling: synchronous pointer doubling
 *    (pointer_doubling_generic.hpp:609-700) with double-buffered rounds over
 *    the active elements.
 *
 * Contract of both: the reference's in-place one (succ -> root, rank:
 * distance to the successor in -> distance to the root out; roots keep their
 * input rank in the ruling set, whose chase never adds a root's rank).  Lists
 * only for the ruling set (the reference asserts is_list,
 * sparse_ruling_set.cpp:52); forests as well for pointer doubling.  Both
 * return a negative value on an index out of range; pointer doubling also on
 * a rootless cycle (more than 64 rounds), the ruling set on a walk longer
 * than n (a rootless cycle that no leaf leads into is not seen, as in the
 * sequential chase).
 *
 * Threads: all online cores, or KASCADE_CPU_THREADS.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <sched.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../kascade_b200/csrc/gen_common.h"

#define ORACLE_API __attribute__((visibility("default")))
#define MAX_THREADS 1024

int oracle_local_pointer_chasing(uint64_t* succ, int64_t* rank, uint64_t n);

ORACLE_API int cpu_threads(void) {
  const char* env = getenv("KASCADE_CPU_THREADS");
  if (env && atoi(env) > 0) return atoi(env) < MAX_THREADS ? atoi(env) : MAX_THREADS;
  cpu_set_t set;
  int n = 0;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) n = CPU_COUNT(&set);
  if (n <= 0) n = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (n <= 0) n = 1;
  return n < MAX_THREADS ? n : MAX_THREADS;
}

/* ---- a minimal fork-join: fn(arg, t, nt) on nt threads ------------------ */
typedef void (*par_fn)(void* arg, int t, int nt);
typedef struct {
  par_fn fn;
  void* arg;
  int t, nt;
} par_job;

static void* par_entry(void* p) {
  par_job* j = (par_job*)p;
  j->fn(j->arg, j->t, j->nt);
  return NULL;
}

static void par_run(int nt, par_fn fn, void* arg) {
  pthread_t th[MAX_THREADS];
  par_job jobs[MAX_THREADS];
  int started[MAX_THREADS];
  for (int t = 0; t < nt; ++t) {
    jobs[t] = (par_job){fn, arg, t, nt};
    started[t] = 0;
  }
  for (int t = 1; t < nt; ++t) started[t] = pthread_create(&th[t], NULL, par_entry, &jobs[t]) == 0;
  fn(arg, 0, nt);
  /* a thread that could not start: its share runs here */
  for (int t = 1; t < nt; ++t) {
    if (started[t])
      pthread_join(th[t], NULL);
    else
      fn(arg, t, nt);
  }
}

static inline void span_of(uint64_t n, int t, int nt, uint64_t* lo, uint64_t* hi) {
  *lo = n * (uint64_t)t / (uint64_t)nt;
  *hi = n * (uint64_t)(t + 1) / (uint64_t)nt;
}

/* ---- sparse ruling set --------------------------------------------------- */
/* Ruler ids are 32-bit; levels at or below this size go to the sequential
 * chase. */
#define SRS_SEQ_MAX (1u << 16)
#define SRS_CHAINS 8
#define SRS_CHUNK 256

typedef struct {
  uint64_t* succ;
  int64_t* rank;
  uint64_t n, m;
  uint32_t spacing;
  uint64_t seed;
  uint8_t* has_pred;
  uint8_t* is_ruler;
  uint32_t* id;
  uint64_t* part; /* per-thread counts, then offsets */
  uint64_t* succ2;
  int64_t* rank2;
  uint64_t* elem_of;
  uint64_t next_ruler;
  int err;
} srs_ctx;

static void srs_mark_preds(void* a, int t, int nt) {
  srs_ctx* c = (srs_ctx*)a;
  uint64_t lo, hi;
  span_of(c->n, t, nt, &lo, &hi);
  int err = 0;
  for (uint64_t i = lo; i < hi; ++i) {
    const uint64_t s = c->succ[i];
    if (s >= c->n) {
      err = 1;
      continue;
    }
    if (s != i) __atomic_store_n(&c->has_pred[s], (uint8_t)1, __ATOMIC_RELAXED);
  }
  if (err) __atomic_store_n(&c->err, 1, __ATOMIC_RELAXED);
}

/* rulers: roots, leaves (sparse_ruling_set.cpp:61-86) and a hashed sample */
static void srs_count_rulers(void* a, int t, int nt) {
  srs_ctx* c = (srs_ctx*)a;
  uint64_t lo, hi, cnt = 0;
  span_of(c->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i) {
    const uint8_t r = (c->succ[i] == i) || !c->has_pred[i] || ks_bounded(ks_hash3(c->seed, 77, i), c->spacing) == 0;
    c->is_ruler[i] = r;
    cnt += r;
  }
  c->part[t] = cnt;
}

static void srs_number_rulers(void* a, int t, int nt) {
  srs_ctx* c = (srs_ctx*)a;
  uint64_t lo, hi, k = c->part[t];
  span_of(c->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i)
    if (c->is_ruler[i]) {
      c->id[i] = (uint32_t)k;
      c->elem_of[k] = i;
      k++;
    }
}

static void srs_chase(void* a, int t, int nt) {
  (void)t;
  (void)nt;
  srs_ctx* c = (srs_ctx*)a;
  uint64_t* succ = c->succ;
  int64_t* rank = c->rank;
  const uint8_t* is_ruler = c->is_ruler;
  const uint64_t n = c->n, m = c->m;
  uint64_t k[SRS_CHAINS], cur[SRS_CHAINS], hops[SRS_CHAINS];
  int64_t d[SRS_CHAINS];
  int live[SRS_CHAINS];
  uint64_t pos = 0, end = 0;
  int active = 0, err = 0, exhausted = 0;
  for (int s = 0; s < SRS_CHAINS; ++s) live[s] = 0;
  for (;;) {
    /* refill the empty slots with the next rulers */
    for (int s = 0; s < SRS_CHAINS && !exhausted; ++s) {
      while (!live[s]) {
        if (pos == end) {
          pos = __atomic_fetch_add(&c->next_ruler, SRS_CHUNK, __ATOMIC_RELAXED);
          if (pos >= m) {
            exhausted = 1;
            break;
          }
          end = pos + SRS_CHUNK < m ? pos + SRS_CHUNK : m;
        }
        const uint64_t kk = pos++;
        const uint64_t r = c->elem_of[kk];
        const uint64_t nx = succ[r];
        const int64_t w = rank[r];
        succ[r] = kk;
        rank[r] = 0;
        if (nx == r) { /* a root: a chain of its own; the rank stays */
          c->succ2[kk] = kk;
          c->rank2[kk] = w;
          continue;
        }
        k[s] = kk;
        cur[s] = nx;
        d[s] = w;
        hops[s] = 0;
        live[s] = 1;
        active++;
        __builtin_prefetch(&succ[nx]);
        __builtin_prefetch(&is_ruler[nx]);
      }
    }
    if (!active) break;
    /* one hop of every live chain */
    for (int s = 0; s < SRS_CHAINS; ++s) {
      if (!live[s]) continue;
      const uint64_t x = cur[s];
      if (is_ruler[x]) { /* the chain ends at the next ruler (or a root) */
        c->succ2[k[s]] = c->id[x];
        c->rank2[k[s]] = d[s];
        live[s] = 0;
        active--;
        continue;
      }
      const uint64_t nx = succ[x];
      const int64_t w = rank[x];
      succ[x] = k[s];
      rank[x] = d[s];
      d[s] += w;
      cur[s] = nx;
      if (nx >= n || ++hops[s] > n) {
        err = 1;
        live[s] = 0;
        active--;
        continue;
      }
      __builtin_prefetch(&succ[nx]);
      __builtin_prefetch(&is_ruler[nx]);
    }
  }
  if (err) __atomic_store_n(&c->err, 1, __ATOMIC_RELAXED);
}

/* pull propagation: each element takes its ruler's root and rank */
static void srs_propagate(void* a, int t, int nt) {
  srs_ctx* c = (srs_ctx*)a;
  uint64_t lo, hi;
  span_of(c->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i) {
    const uint64_t kk = c->succ[i];
    c->rank[i] = c->rank2[kk] - c->rank[i];
    c->succ[i] = c->elem_of[c->succ2[kk]];
  }
}

static int srs_level(uint64_t* succ, int64_t* rank, uint64_t n, uint32_t spacing, uint64_t seed, int depth, int nt) {
  if (n <= SRS_SEQ_MAX || depth >= 12 || n >= (1ull << 32) || nt <= 1)
    return oracle_local_pointer_chasing(succ, rank, n) == 0 ? 0 : -1;
  srs_ctx c;
  memset(&c, 0, sizeof(c));
  c.succ = succ;
  c.rank = rank;
  c.n = n;
  c.spacing = spacing;
  c.seed = seed;
  c.has_pred = (uint8_t*)calloc(n, 1);
  c.is_ruler = (uint8_t*)malloc(n);
  c.id = (uint32_t*)malloc(sizeof(uint32_t) * n);
  c.part = (uint64_t*)calloc((size_t)nt + 1, sizeof(uint64_t));
  int rc = -1;
  if (!c.has_pred || !c.is_ruler || !c.id || !c.part) goto out;
  par_run(nt, srs_mark_preds, &c);
  if (c.err) goto out;
  par_run(nt, srs_count_rulers, &c);
  {
    uint64_t acc = 0;
    for (int t = 0; t < nt; ++t) {
      const uint64_t x = c.part[t];
      c.part[t] = acc;
      acc += x;
    }
    c.m = acc;
  }
  free(c.has_pred);
  c.has_pred = NULL;
  c.succ2 = (uint64_t*)malloc(sizeof(uint64_t) * c.m);
  c.rank2 = (int64_t*)malloc(sizeof(int64_t) * c.m);
  c.elem_of = (uint64_t*)malloc(sizeof(uint64_t) * c.m);
  if (!c.succ2 || !c.rank2 || !c.elem_of) goto out;
  par_run(nt, srs_number_rulers, &c);
  par_run(nt, srs_chase, &c);
  if (c.err) goto out;
  if (srs_level(c.succ2, c.rank2, c.m, spacing, ks_mix64(seed), depth + 1, nt) != 0) goto out;
  par_run(nt, srs_propagate, &c);
  rc = 0;
out:
  free(c.has_pred);
  free(c.is_ruler);
  free(c.id);
  free(c.part);
  free(c.succ2);
  free(c.rank2);
  free(c.elem_of);
  return rc;
}

ORACLE_API int cpu_sparse_ruling_set(uint64_t* succ, int64_t* rank, uint64_t n, uint32_t spacing, uint64_t seed,
                                     int threads) {
  if (spacing < 2) spacing = 2;
  if (threads <= 0) threads = cpu_threads();
  if (threads > MAX_THREADS) threads = MAX_THREADS;
  return srs_level(succ, rank, n, spacing, seed, 0, threads);
}

/* ---- synchronous pointer doubling ----------------------------------------
 * Roots flagged with the MSB (initialize_active_vertices,
 * pointer_doubling_generic.hpp:418-438), then rounds over the active
 * elements, each reading (succ, rank) of its successor as it stood at the
 * start of the round (:43-60, :171-212); an element retires once its new
 * successor is a flagged root; the flag is cleared at the end. */
#define PD_ROOT_FLAG (1ull << 63)

typedef struct {
  uint64_t* succ;
  int64_t* rank;
  uint64_t n, na;
  uint64_t *s2, *act, *act2;
  int64_t* r2;
  uint64_t* part;
  int err;
} pd_ctx;

static void pd_flag(void* a, int t, int nt) {
  pd_ctx* c = (pd_ctx*)a;
  uint64_t lo, hi, cnt = 0;
  int err = 0;
  span_of(c->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i) {
    if (c->succ[i] >= c->n) err = 1;
    if (c->succ[i] == i)
      c->succ[i] |= PD_ROOT_FLAG;
    else
      cnt++;
  }
  c->part[t] = cnt;
  if (err) __atomic_store_n(&c->err, 1, __ATOMIC_RELAXED);
}

static void pd_init_active(void* a, int t, int nt) {
  pd_ctx* c = (pd_ctx*)a;
  uint64_t lo, hi, k = c->part[t];
  span_of(c->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i)
    if (!(c->succ[i] & PD_ROOT_FLAG)) c->act[k++] = i;
}

static void pd_read(void* a, int t, int nt) {
  pd_ctx* c = (pd_ctx*)a;
  uint64_t lo, hi, cnt = 0;
  span_of(c->na, t, nt, &lo, &hi);
  for (uint64_t j = lo; j < hi; ++j) {
    const uint64_t i = c->act[j];
    const uint64_t s = c->succ[i] & ~PD_ROOT_FLAG;
    c->s2[j] = c->succ[s];
    c->r2[j] = c->rank[i] + c->rank[s];
    cnt += !(c->s2[j] & PD_ROOT_FLAG);
  }
  c->part[t] = cnt;
}

static void pd_write(void* a, int t, int nt) {
  pd_ctx* c = (pd_ctx*)a;
  uint64_t lo, hi, k = c->part[t];
  span_of(c->na, t, nt, &lo, &hi);
  for (uint64_t j = lo; j < hi; ++j) {
    const uint64_t i = c->act[j];
    c->succ[i] = c->s2[j];
    c->rank[i] = c->r2[j];
    if (!(c->s2[j] & PD_ROOT_FLAG)) c->act2[k++] = i;
  }
}

static void pd_unflag(void* a, int t, int nt) {
  pd_ctx* c = (pd_ctx*)a;
  uint64_t lo, hi;
  span_of(c->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i) c->succ[i] &= ~PD_ROOT_FLAG;
}

static uint64_t exclusive_scan(uint64_t* part, int nt) {
  uint64_t acc = 0;
  for (int t = 0; t < nt; ++t) {
    const uint64_t x = part[t];
    part[t] = acc;
    acc += x;
  }
  return acc;
}

/* Returns the number of rounds, or -1. */
ORACLE_API int cpu_pointer_doubling(uint64_t* succ, int64_t* rank, uint64_t n, int threads) {
  int nt = threads > 0 ? threads : cpu_threads();
  if (nt > MAX_THREADS) nt = MAX_THREADS;
  pd_ctx c;
  memset(&c, 0, sizeof(c));
  c.succ = succ;
  c.rank = rank;
  c.n = n;
  const uint64_t cap = n ? n : 1;
  c.s2 = (uint64_t*)malloc(sizeof(uint64_t) * cap);
  c.r2 = (int64_t*)malloc(sizeof(int64_t) * cap);
  c.act = (uint64_t*)malloc(sizeof(uint64_t) * cap);
  c.act2 = (uint64_t*)malloc(sizeof(uint64_t) * cap);
  c.part = (uint64_t*)calloc((size_t)nt + 1, sizeof(uint64_t));
  int rounds = -1;
  if (c.s2 && c.r2 && c.act && c.act2 && c.part) {
    par_run(nt, pd_flag, &c);
    if (!c.err) {
      c.na = exclusive_scan(c.part, nt);
      par_run(nt, pd_init_active, &c);
      rounds = 0;
      while (c.na > 0) {
        if (rounds >= 64) {
          rounds = -1;
          break;
        }
        par_run(nt, pd_read, &c);
        const uint64_t na2 = exclusive_scan(c.part, nt);
        par_run(nt, pd_write, &c);
        uint64_t* tmp = c.act;
        c.act = c.act2;
        c.act2 = tmp;
        c.na = na2;
        rounds++;
      }
    }
    par_run(nt, pd_unflag, &c);
  }
  free(c.s2);
  free(c.r2);
  free(c.act);
  free(c.act2);
  free(c.part);
  return rounds;
}

/* ---- parallel forms of the seeded generators ------------------------------
 * The same per-index functions the oracle and the device generators use, so
 * that full-size baseline inputs need not be built on one core. */
typedef struct {
  uint64_t n, seed, blocks, spine;
  uint32_t layout_or_kind, wbits;
  uint64_t* out;
  uint32_t* w;
  ks_perm p;
} gen_ctx;

static void gen_list_part(void* a, int t, int nt) {
  gen_ctx* g = (gen_ctx*)a;
  uint64_t lo, hi;
  span_of(g->n, t, nt, &lo, &hi);
  for (uint64_t k = lo; k < hi; ++k) {
    const uint64_t e = ks_list_elem(&g->p, g->layout_or_kind, g->n, k);
    g->out[e] = (k + 1 < g->n) ? ks_list_elem(&g->p, g->layout_or_kind, g->n, k + 1) : e;
  }
}

static void gen_weights_part(void* a, int t, int nt) {
  gen_ctx* g = (gen_ctx*)a;
  uint64_t lo, hi;
  span_of(g->n, t, nt, &lo, &hi);
  for (uint64_t i = lo; i < hi; ++i) g->w[i] = ks_weight(g->seed, i, g->wbits);
}

static void gen_forest_part(void* a, int t, int nt) {
  gen_ctx* g = (gen_ctx*)a;
  uint64_t lo, hi;
  span_of(g->n, t, nt, &lo, &hi);
  for (uint64_t v = lo; v < hi; ++v) {
    uint64_t at, par;
    ks_forest_edge(&g->p, g->layout_or_kind, g->n, g->blocks, g->spine, g->seed, v, &at, &par);
    g->out[at] = par;
  }
}

ORACLE_API void cpu_gen_list(uint64_t n, uint64_t seed, uint32_t layout, uint64_t* succ) {
  if (n == 0) return;
  gen_ctx g = {n, seed, 0, 0, layout, 0, succ, NULL, ks_list_perm(n, seed, layout)};
  par_run(cpu_threads(), gen_list_part, &g);
}

ORACLE_API void cpu_gen_weights(uint64_t n, uint64_t seed, uint32_t wbits, uint32_t* w) {
  gen_ctx g;
  memset(&g, 0, sizeof(g));
  g.n = n;
  g.seed = seed;
  g.wbits = wbits;
  g.w = w;
  par_run(cpu_threads(), gen_weights_part, &g);
}

ORACLE_API void cpu_gen_forest(uint64_t n, uint64_t seed, uint32_t kind, uint64_t blocks, uint64_t spine,
                               uint64_t* parent) {
  if (n == 0) return;
  gen_ctx g = {n, seed, blocks, spine, kind, 0, parent, NULL, ks_forest_perm(n, seed)};
  par_run(cpu_threads(), gen_forest_part, &g);
}
