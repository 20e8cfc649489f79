/* Test infrastructure (oracle), not product code. See ngap_oracle.h.
 *
 * One OpenMP task per (group, segment), as the reference runs one thread per
 * (group, segment) (code/src/ngap/ngap.cu:2182-2199). Per segment:
 *   frontier(seg start) = start-of-data states (segment 0, or every segment
 *                         when the stream was duplicated) + always-active states
 *                         (ngap.cu:2201-2210);
 *   for each position: every frontier state whose symbol class holds the byte
 *   reports (if it is a report state) and contributes its CSR successors; the
 *   always-active states are appended to the next frontier (ngap.cu:2212-2258,
 *   DEBUG_PL_ADVANCE_CONCAT is defined in code/src/ngap/ngap_buffer.h:19);
 *   the loop stops at the segment end or when the frontier is empty.
 * With validator_quirk the odd-start rule of the validator's loop condition
 * (see ngap_oracle.h) is reproduced too.
 */
#define _GNU_SOURCE
#include "ngap_oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t* v;
  int64_t n, cap;
} vec64;

static void vpush64(vec64* a, uint64_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 256;
    a->v = (uint64_t*)realloc(a->v, (size_t)a->cap * sizeof(uint64_t));
  }
  a->v[a->n++] = x;
}

typedef struct {
  int32_t* v;
  int64_t n, cap;
} vec32;

static void vpush32(vec32* a, int32_t x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? a->cap * 2 : 256;
    a->v = (int32_t*)realloc(a->v, (size_t)a->cap * sizeof(int32_t));
  }
  a->v[a->n++] = x;
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static int cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return (x > y) - (x < y);
}

static inline int accepts(const oracle_group* g, int32_t v, uint8_t s) {
  return (g->bits[(int64_t)v * 8 + (s >> 5)] >> (s & 31)) & 1u;
}

/* key ordering (offset, id) as compareResult (ngap.cu:19-30) */
static inline uint64_t to_key(uint32_t id, uint32_t off) { return ((uint64_t)off << 32) | id; }

static void run_unit(const oracle_group* g, int gi, const uint8_t* input, int64_t seg,
                     int64_t seg_len, int is_dup, int64_t first_seg, int mode, int unique,
                     int quirk, vec64* rep, oracle_stats* st) {
  const int64_t lo = seg * seg_len, hi = lo + seg_len;
  /* the reference validator's first test reads frontiers[iter % 2] with iter
     the segment's first global position (ngap.cu:2212) */
  if (quirk && ((first_seg + seg) * seg_len) % 2 != 0) return;
  const uint32_t gbits = (uint32_t)gi << 22;
  vec32 cur = {0}, nxt = {0};
  uint8_t* mark = NULL;
  if (mode == 1) mark = (uint8_t*)calloc((size_t)g->V + 1, 1);
  if (first_seg + seg == 0 || is_dup)
    for (int i = 0; i < g->nstart; i++) vpush32(&cur, g->starts[i]);
  for (int i = 0; i < g->naas; i++) vpush32(&cur, g->aas[i]);
  if (mode == 1) { /* deduplicate the initial frontier */
    int64_t k = 0;
    for (int64_t i = 0; i < cur.n; i++)
      if (!mark[cur.v[i]]) {
        mark[cur.v[i]] = 1;
        cur.v[k++] = cur.v[i];
      }
    cur.n = k;
    for (int64_t i = 0; i < cur.n; i++) mark[cur.v[i]] = 0;
  }
  int64_t iter = lo;
  while (cur.n > 0 && iter < hi) {
    const uint8_t sym = input[iter];
    nxt.n = 0;
    st->frontier += (uint64_t)cur.n;
    for (int64_t k = 0; k < cur.n; k++) {
      int32_t v = cur.v[k];
      if (!accepts(g, v, sym)) continue;
      int32_t e0 = g->row_offsets[v], e1 = g->row_offsets[v + 1];
      st->matched++;
      st->matched_deg += (uint64_t)(e1 - e0);
      if (g->attrs[v] & 2) {
        vpush64(rep, to_key((uint32_t)v | gbits, (uint32_t)iter));
        st->reports_raw++;
      }
      for (int32_t e = e0; e < e1; e++) {
        int32_t u = g->cols[e];
        if (mode == 1) {
          if (mark[u]) continue;
          mark[u] = 1;
        }
        vpush32(&nxt, u);
      }
    }
    if (mode == 0 && unique && nxt.n > 1) {
      qsort(nxt.v, (size_t)nxt.n, sizeof(int32_t), cmp_i32);
      int64_t k = 1;
      for (int64_t i = 1; i < nxt.n; i++)
        if (nxt.v[i] != nxt.v[k - 1]) nxt.v[k++] = nxt.v[i];
      nxt.n = k;
    }
    for (int i = 0; i < g->naas; i++) {
      int32_t a = g->aas[i];
      if (mode == 1) {
        if (mark[a]) continue;
        mark[a] = 1;
      }
      vpush32(&nxt, a);
    }
    if (mode == 1)
      for (int64_t i = 0; i < nxt.n; i++) mark[nxt.v[i]] = 0;
    vec32 t = cur;
    cur = nxt;
    nxt = t;
    iter++;
  }
  free(cur.v);
  free(nxt.v);
  free(mark);
}

static int64_t g_last_needed = 0;

int64_t oracle_last_needed(void) { return g_last_needed; }

int64_t oracle_match(const oracle_group* groups, int ngroups, const uint8_t* input,
                     int64_t num_seg, int64_t seg_len, int is_dup, int64_t first_seg, int mode,
                     int unique, int validator_quirk, int nthreads, uint64_t* out, int64_t cap,
                     oracle_stats* stats) {
  const int64_t units = (int64_t)ngroups * num_seg;
  vec64* reps = (vec64*)calloc((size_t)(units > 0 ? units : 1), sizeof(vec64));
  oracle_stats* sts = (oracle_stats*)calloc((size_t)(units > 0 ? units : 1), sizeof(oracle_stats));
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int64_t u = 0; u < units; u++) {
    int gi = (int)(u / num_seg);
    int64_t seg = u % num_seg;
    run_unit(&groups[gi], gi, input, seg, seg_len, is_dup, first_seg, mode, unique,
             validator_quirk, &reps[u], &sts[u]);
  }
  int64_t total = 0;
  oracle_stats acc = {0, 0, 0, 0};
  for (int64_t u = 0; u < units; u++) {
    total += reps[u].n;
    acc.matched += sts[u].matched;
    acc.matched_deg += sts[u].matched_deg;
    acc.reports_raw += sts[u].reports_raw;
    acc.frontier += sts[u].frontier;
  }
  uint64_t* all = (uint64_t*)malloc((size_t)(total > 0 ? total : 1) * sizeof(uint64_t));
  int64_t k = 0;
  for (int64_t u = 0; u < units; u++) {
    if (reps[u].n) memcpy(all + k, reps[u].v, (size_t)reps[u].n * sizeof(uint64_t));
    k += reps[u].n;
    free(reps[u].v);
  }
  free(reps);
  free(sts);
  qsort(all, (size_t)total, sizeof(uint64_t), cmp_u64);
  int64_t n = 0;
  for (int64_t i = 0; i < total; i++)
    if (n == 0 || all[i] != all[n - 1]) all[n++] = all[i];
  if (stats) *stats = acc;
  g_last_needed = n;
  if (n > cap) {
    free(all);
    return -1;
  }
  for (int64_t i = 0; i < n; i++) {
    uint64_t key = all[i];
    uint32_t off = (uint32_t)(key >> 32), id = (uint32_t)key;
    out[i] = ((uint64_t)id << 32) | off;
  }
  free(all);
  return n;
}
