/*
 * gapped.h -- CPU oracle of the gapped stage (score-only gapped X-drop
 * extension of the ungapped HSPs).  TEST INFRASTRUCTURE ONLY; see gapped.c
 * for its status (unpinned: NCBI's GetGappedScore is not in the reference).
 *
 * Conventions (the device kernel follows them exactly):
 *
 * Order and skipping.  A subject's ungapped HSPs are taken by descending
 * score, equal scores in discovery order.  One whose query range
 * [hsp_q, hsp_q + len) and subject range [hsp_s, hsp_s + len) both lie inside
 * the ranges of a gapped HSP already reported for the subject is skipped.
 *
 * Seed.  An HSP of at most OR_GWINDOW (11) letters is seeded at its middle
 * letter (offset len / 2); a longer one at offset k + 5 of the first k whose
 * 11-letter window scores highest.
 *
 * Extension.  Left: A = query[q_seed], query[q_seed - 1], ..., query[0] and
 * B = subject[s_seed], ..., subject[0] (the seed pair aligned first); right:
 * the letters after the seed on both sides.  Cells (i, j): i letters of A and
 * j of B taken.  H(0,0) = 0;
 *   E(i,j) = max(H(i,j-1) - open, E(i,j-1)) - extend     (gap in A)
 *   F(i,j) = max(H(i-1,j) - open, F(i-1,j)) - extend     (gap in B)
 *   H(i,j) = max(H(i-1,j-1) + S(a_i, b_j), E(i,j), F(i,j))
 * (a gap of k letters costs open + k * extend).  Dead cells hold OR_GNEG and
 * start no path; every value is clamped at OR_GNEG.  Row 0 is the origin and
 * then the cells E(0,j) while they are >= -xdrop.  Row i >= 1 is computed
 * from the first live column lo of row i-1 through one past its last live
 * column, then further right while E(i,j) >= best - xdrop (best as of row
 * i-1); after the whole row, best = max(best, the row's maximum) and every
 * cell of the row below best - xdrop becomes dead.  The extension ends at a
 * row with no live cell, or after the last row.  It returns best and the
 * first cell holding it (lowest row, then lowest column) -- row 0's origin
 * (0 letters) when no cell beats 0.
 *
 * Result.  score = left best + right best; the gapped HSP spans
 * query [q_seed + 1 - li, q_seed + 1 + ri) and subject
 * [s_seed + 1 - lj, s_seed + 1 + rj); reported when score >= cutoff.
 */
#ifndef BLASTP_ORACLE_GAPPED_H
#define BLASTP_ORACLE_GAPPED_H

#include <stdint.h>

#include "oracle.h"

#ifdef __cplusplus
extern "C" {
#endif

#define OR_GWINDOW 11
#define OR_GNEG (-(1 << 28))

typedef struct or_gparams {
    int32_t gap_open, gap_extend, xdrop, cutoff;   /* raw scores */
} or_gparams;

typedef struct or_ghsp {
    int32_t score;
    int32_t q_start, q_end;      /* query range, end exclusive */
    int32_t s_start, s_end;      /* subject range, end exclusive */
    int32_t q_seed, s_seed;      /* the seed pair */
    int32_t ungapped;            /* index of the ungapped HSP within its subject */
} or_ghsp;

/* One extension over A (M letters) and B (N letters), read at A[dir * i] and
 * B[dir * j]; H, F are work buffers of N + 1 ints.  Returns the best score,
 * with the letters it covers on each side in *bi, *bj. */
int32_t or_gapped_extend(const int8_t* matrix28, const uint8_t* A, int32_t M, const uint8_t* B, int32_t N,
                         int32_t dir, int32_t xdrop, int32_t open, int32_t extend, int32_t* H, int32_t* F,
                         int32_t* bi, int32_t* bj);

/* The seed pair of an ungapped HSP. */
void or_gapped_seed(const int8_t* matrix28, const uint8_t* query, const uint8_t* subject, int32_t hsp_q,
                    int32_t hsp_s, int32_t len, int32_t* q_seed, int32_t* s_seed);

/* The gapped stage over a database: the ungapped HSPs of each subject
 * (CSR hsp_off / hsps, per subject in discovery order) in, the reported
 * gapped HSPs out (CSR goff [n+1] / out, per subject in processing order).
 * Returns the total, which may exceed cap (then only goff is complete). */
int64_t or_gapped(const uint8_t* db, const int64_t* db_off, int32_t n_subjects, const uint8_t* query, int32_t qlen,
                  const int64_t* hsp_off, const or_hsp* hsps, const int8_t* matrix28, const or_gparams* p,
                  int32_t n_threads, int64_t* goff, or_ghsp* out, int64_t cap);

#ifdef __cplusplus
}
#endif
#endif
