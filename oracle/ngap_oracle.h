/* Test infrastructure (oracle), not product code.
 *
 * CPU restatement of the reference's CPU matcher and validator:
 *   automataGroupsReference   code/src/ngap/ngap.cu:2171-2268
 *   automataValidation        code/src/ngap/ngap.cu:2270-2344 (sort + unique)
 *   compareResult             code/src/ngap/ngap.cu:19-30     (order by offset, then id)
 * Parity is pinned against the reference's known-answer test (small_dataset/
 * apple.anml, README.md:156-186) and against group graphs produced by the
 * reference's own front-end (oracle/_ref/ref_frontend). Only tests, the smoke
 * check and the CPU-baseline leg of the benchmark use it.
 */
#ifndef NGAP_ORACLE_H_
#define NGAP_ORACLE_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_group {
  int32_t V;
  const int32_t* row_offsets; /* V + 1 */
  const int32_t* cols;        /* row_offsets[V] */
  const uint32_t* bits;       /* V * 8 */
  const uint8_t* attrs;       /* bit0 always-active, bit1 report */
  int32_t naas;
  const int32_t* aas;
  int32_t nstart;
  const int32_t* starts;
} oracle_group;

typedef struct oracle_stats {
  uint64_t matched;      /* sum over positions of matched frontier states */
  uint64_t matched_deg;  /* sum of out-degrees of those states */
  uint64_t reports_raw;  /* reports before deduplication */
  uint64_t frontier;     /* sum over positions of frontier sizes (states tested) */
} oracle_stats;

/* mode 0: the reference loop as written (vector frontier, duplicates kept,
 *         `unique` sorts and deduplicates each next frontier like --unique);
 * mode 1: same report set with a bitmap-deduplicated frontier (bounded work).
 * Reports are written as the reference packs them, ((sid | g << 22) << 32) |
 * offset, sorted by (offset, id) and deduplicated. Returns the number of
 * unique reports, or -1 when more than `cap` would be written (stats and the
 * return of oracle_last_needed() still give the count). first_seg is the
 * global index of the first segment (start-of-data states belong to global
 * segment 0 unless is_dup).
 *
 * validator_quirk = 1 reproduces the reference CPU validator exactly as it
 * runs, including its loop condition `while (!frontiers[iter % 2].empty() ...)`
 * (ngap.cu:2212): iter starts at the segment's first global position and the
 * initial states go to frontiers[0], so a segment that starts at an odd
 * position (odd seg_len, odd segment index) tests the empty frontiers[1] and
 * reports nothing. The reference's GPU matchers report those segments; with
 * validator_quirk = 0 (the default, the engine's semantics) they are matched
 * like every other segment. */
int64_t oracle_match(const oracle_group* groups, int ngroups, const uint8_t* input,
                     int64_t num_seg, int64_t seg_len, int is_dup, int64_t first_seg, int mode,
                     int unique, int validator_quirk, int nthreads, uint64_t* out, int64_t cap,
                     oracle_stats* stats);

int64_t oracle_last_needed(void);

#ifdef __cplusplus
}
#endif
#endif
