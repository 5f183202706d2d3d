/*
 * oracle.h -- CPU oracle for blastp's two-hit word finder + ungapped X-drop
 * extension.  TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the
 * CPU-baseline leg of bench.py use it as the checker; the product path never
 * links, loads or calls it.
 *
 * Parity status: PINNED to the reference's own code.  The reference (GPU-BLAST
 * 1.1 over NCBI BLAST+ 2.2.28) ships no tests or golden vectors, and its GPU
 * build needs the absent NCBI toolkit; but its kernel source
 * (gpu_blastp_kernel.cu) is host-compiled unmodified into oracle/_ref by
 * ref_driver.cpp, and tests/test_ref_pinned.py requires this oracle's
 * counters and complete HSP sets to equal that kernel's on config-sized and
 * edge-case inputs.  Also pinned: the scoring table (the reference's BLOSUM62
 * held as a fixture) and hand-computed known-answer cases in tests/.  Still
 * unpinned: NCBI's own neighbour-word rule and cutoff formula, which the
 * reference calls but does not ship.
 *
 * Semantics restated (file:line into the reference project):
 *   word scan + presence test + cell fetch   gpu_blastp_kernel.cu:151-192
 *   two-hit diagonal state machine           gpu_blastp_kernel.cu:194-297
 *   context selection, cutoff, HSP record    gpu_blastp_kernel.cu:238-276
 *   per-subject counters                     gpu_blastp_kernel.cu:310-312
 *   s_BlastAaExtendTwoHit                    gpu_blastp_kernel.cu:341-415
 *   s_BlastAaExtendLeft                      gpu_blastp_kernel.cu:435-481
 *   s_BlastAaExtendRight                     gpu_blastp_kernel.cu:503-549
 *   record layout GPUBlastInitHitList        ncbi_blast_files/gpu_cpu_common.h:29-38
 * The neighbour-word table follows NCBI's rule (all words scoring >= T against
 * a query word; the exact word is added when its self-score is below T), as
 * consumed by the kernel at gpu_blastp_kernel.cu:182-192.
 */
#ifndef BLASTP_ORACLE_H
#define BLASTP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_ALPHA 28            /* NCBIstdaa alphabet size */
#define OR_NCELL 32768         /* 3 letters x 5 bits */

typedef struct or_hsp {         /* same field order as GPUBlastInitHitList */
    int32_t hsp_q, hsp_s, query_offset, subject_offset, hsp_len, score;
} or_hsp;

/* Neighbour-word table as CSR keyed by the packed code r0<<10|r1<<5|r2.
 * cell_start has OR_NCELL+1 entries; entries of a cell are ascending query
 * offsets.  Returns the number of entries, or -1 if cap is too small (the
 * cell_start array is still complete in that case). */
int64_t or_build_table(const uint8_t* query, int32_t qlen, const int8_t* matrix28,
                       int32_t threshold, uint32_t* cell_start, uint16_t* entries,
                       int64_t cap);

/* Scan subjects [0, n_subjects) of a flat database against one query.
 *  db/db_off         residues (NCBIstdaa) and n_subjects+1 offsets
 *  ctx_*             n_ctx contexts: first query offset, x-drop, cutoff (raw)
 *  diag_mask         power-of-two-minus-one mask of the diagonal array
 *  counters          out, n_subjects*3: hits, successful extensions, extensions
 *  hsp_off           out, n_subjects+1: CSR offsets into hsps
 *  hsps              out, capacity hsp_cap, per subject in discovery order
 * Returns the total number of HSPs (may exceed hsp_cap; then only the counts
 * and offsets are complete and the caller re-runs with a larger buffer). */
int64_t or_scan(const uint8_t* db, const int64_t* db_off, int32_t n_subjects,
                const uint8_t* query, int32_t qlen,
                const uint32_t* cell_start, const uint16_t* entries,
                int32_t n_ctx, const int32_t* ctx_offset, const int32_t* ctx_xdrop,
                const int32_t* ctx_cutoff, int32_t window, int32_t diag_mask,
                const int8_t* matrix28, int32_t n_threads,
                int32_t* counters, int64_t* hsp_off, or_hsp* hsps, int64_t hsp_cap);

/* One two-hit extension, exposed for known-answer tests. */
void or_extend_two_hit(const int8_t* matrix28, const uint8_t* subject, int32_t slen,
                       const uint8_t* query, int32_t qlen, int32_t s_left,
                       int32_t s_right, int32_t q_right, int32_t xdrop,
                       int32_t out[6] /* hsp_q, hsp_s, len, score, s_last, right_ext */);

#ifdef __cplusplus
}
#endif
#endif
