/*
 * oracle.c -- CPU oracle for blastp's two-hit word finder + ungapped X-drop
 * extension.  TEST INFRASTRUCTURE ONLY (see oracle.h): the product path never
 * links, loads or calls this file.  Pinned to the reference's own kernel
 * source, host-compiled into oracle/_ref (ref_driver.cpp), by
 * tests/test_ref_pinned.py; also by the scoring table and hand-computed cases.
 *
 * Plain C99 + pthreads.  Subjects are independent, so threads take chunks of
 * subjects from an atomic cursor; each thread owns one diagonal array and
 * reuses it across its subjects with the diagonal-offset trick the reference
 * kernel uses (gpu_blastp_kernel.cu:204-229,308).
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define WORD 3
#define FLAG 0x80000000u

static inline int sc(const int8_t* m, int a, int b) { return m[a * OR_ALPHA + b]; }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }
static inline uint32_t code3(int a, int b, int c) { return ((uint32_t)a << 10) | ((uint32_t)b << 5) | (uint32_t)c; }

/* Neighbour words of every query word: all w with score(qword, w) >= T over
 * the letters 1..27 (letter 0 scores -128 against everything), plus the exact
 * word when its self-score is below T.  Cells list query offsets ascending. */
int64_t or_build_table(const uint8_t* query, int32_t qlen, const int8_t* m,
                       int32_t threshold, uint32_t* cell_start, uint16_t* entries,
                       int64_t cap)
{
    uint32_t* cnt = (uint32_t*)calloc(OR_NCELL, sizeof(uint32_t));
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            uint32_t acc = 0;
            for (int c = 0; c < OR_NCELL; ++c) { cell_start[c] = acc; acc += cnt[c]; cnt[c] = 0; }
            cell_start[OR_NCELL] = acc;
            if ((int64_t)acc > cap) { free(cnt); return -1; }
        }
        for (int q = 0; q + WORD <= qlen; ++q) {
            int a = query[q], b = query[q + 1], c = query[q + 2];
            int self = sc(m, a, a) + sc(m, b, b) + sc(m, c, c);
            for (int r0 = 1; r0 < OR_ALPHA; ++r0) {
                int s0 = sc(m, a, r0);
                for (int r1 = 1; r1 < OR_ALPHA; ++r1) {
                    int s1 = s0 + sc(m, b, r1);
                    for (int r2 = 1; r2 < OR_ALPHA; ++r2) {
                        int s2 = s1 + sc(m, c, r2);
                        int take = s2 >= threshold ||
                                   (self < threshold && r0 == a && r1 == b && r2 == c);
                        if (!take) continue;
                        uint32_t w = code3(r0, r1, r2);
                        if (pass == 1) entries[cell_start[w] + cnt[w]] = (uint16_t)q;
                        cnt[w]++;
                    }
                }
            }
        }
    }
    int64_t total = cell_start[OR_NCELL];
    free(cnt);
    return total;
}

/* gpu_blastp_kernel.cu:341-415 with :435-481 and :503-549 inlined.  The
 * reference scores the 3-letter start as matrix[s][q] and the walks as
 * matrix[q][s]; BLOSUM62 is symmetric (checked by the tests). */
void or_extend_two_hit(const int8_t* m, const uint8_t* s, int32_t slen,
                       const uint8_t* q, int32_t qlen, int32_t s_left,
                       int32_t s_right, int32_t q_right, int32_t xdrop, int32_t out[6])
{
    /* one beyond the best-scoring prefix of the second word */
    int score = 0, left_score = 0, shift = 0;
    for (int i = 0; i < WORD; ++i) {
        score += sc(m, q[q_right + i], s[s_right + i]);
        if (score > left_score) { left_score = score; shift = i + 1; }
    }
    q_right += shift;
    s_right += shift;

    /* left walk from (s_right-1, q_right-1) towards the sequence starts */
    int s_off = s_right - 1, q_off = q_right - 1;
    int n = imin(s_off, q_off);
    int run = 0, best = 0, best_k = -1;
    for (int k = 0; k <= n; ++k) {
        run += sc(m, q[q_off - k], s[s_off - k]);
        if (run > best) { best = run; best_k = k; }
        if (best - run >= xdrop) break;
    }
    int left_d = best_k + 1;
    left_score = best;

    int right_ext = 0, right_d = 0, right_score = 0, s_last = s_right;
    if (left_d >= s_right - s_left) {
        right_ext = 1;
        int n2 = imin(slen - s_right, qlen - q_right);
        int rbest = left_score, rrun = left_score, rbest_i = -1, i;
        for (i = 0; i < n2; ++i) {
            rrun += sc(m, q[q_right + i], s[s_right + i]);
            if (rrun > rbest) { rbest = rrun; rbest_i = i; }
            if (rrun <= 0 || rbest - rrun >= xdrop) break;
        }
        right_d = rbest_i + 1;
        right_score = rbest;
        s_last = s_right + i;
    }
    out[0] = q_right - left_d;
    out[1] = s_right - left_d;
    out[2] = left_d + right_d;
    out[3] = imax(left_score, right_score);
    out[4] = s_last;
    out[5] = right_ext;
}

typedef struct { int32_t oid; or_hsp h; } rec_t;

typedef struct {
    /* shared, read-only */
    const uint8_t* db; const int64_t* db_off; int32_t n;
    const uint8_t* query; int32_t qlen;
    const uint32_t* cell_start; const uint16_t* entries;
    int32_t n_ctx; const int32_t* ctx_offset; const int32_t* ctx_xdrop; const int32_t* ctx_cutoff;
    int32_t window, diag_mask; const int8_t* m;
    int32_t* counters;
    int32_t* cursor;
} job_t;

typedef struct { job_t* job; rec_t* recs; int64_t nrec, caprec; } worker_t;

static void push(worker_t* w, int32_t oid, const or_hsp* h)
{
    if (w->nrec == w->caprec) {
        w->caprec = w->caprec ? 2 * w->caprec : 1024;
        w->recs = (rec_t*)realloc(w->recs, (size_t)w->caprec * sizeof(rec_t));
    }
    w->recs[w->nrec].oid = oid;
    w->recs[w->nrec].h = *h;
    w->nrec++;
}

static int context_of(const job_t* j, int q)
{
    int k = j->n_ctx - 1;               /* last context starting at or before q */
    while (k > 0 && q < j->ctx_offset[k]) --k;
    return k;
}

#define CHUNK 64

static void* worker_main(void* arg)
{
    worker_t* w = (worker_t*)arg;
    const job_t* j = w->job;
    int32_t L = j->diag_mask + 1;
    uint32_t* diag = (uint32_t*)calloc((size_t)L, sizeof(uint32_t));
    int64_t base = j->window;
    for (;;) {
        int32_t first = __atomic_fetch_add(j->cursor, CHUNK, __ATOMIC_RELAXED);
        if (first >= j->n) break;
        int32_t last = imin(first + CHUNK, j->n);
        for (int32_t oid = first; oid < last; ++oid) {
            const uint8_t* sub = j->db + j->db_off[oid];
            int32_t slen = (int32_t)(j->db_off[oid + 1] - j->db_off[oid]);
            if (base + slen + j->window > (1 << 30)) {
                memset(diag, 0, (size_t)L * sizeof(uint32_t));
                base = j->window;
            }
            int32_t hits = 0, succ = 0, ext = 0;
            for (int32_t s = 0; s <= slen - WORD; ++s) {
                uint32_t c = code3(sub[s], sub[s + 1], sub[s + 2]);
                uint32_t e0 = j->cell_start[c], e1 = j->cell_start[c + 1];
                hits += (int32_t)(e1 - e0);
                for (uint32_t e = e0; e < e1; ++e) {
                    int32_t q = j->entries[e];
                    int32_t d = (q - s) & j->diag_mask;
                    uint32_t v = diag[d];
                    int32_t stamp = (int32_t)(s + base);
                    if (v & FLAG) {
                        if (stamp < (int32_t)(v & ~FLAG)) continue;
                        diag[d] = (uint32_t)stamp;
                        continue;
                    }
                    int32_t prev = (int32_t)v - (int32_t)base;
                    int32_t diff = s - prev;
                    if (diff >= j->window) { diag[d] = (uint32_t)stamp; continue; }
                    if (diff < WORD) continue;
                    int k = context_of(j, q);
                    int32_t r[6];
                    or_extend_two_hit(j->m, sub, slen, j->query, j->qlen, prev + WORD, s, q,
                                      j->ctx_xdrop[k], r);
                    ++ext;
                    if (r[3] >= j->ctx_cutoff[k]) {
                        or_hsp h = { r[0], r[1], q, s, r[2], r[3] };
                        push(w, oid, &h);
                        ++succ;
                    }
                    if (r[5]) diag[d] = ((uint32_t)(r[4] - (WORD - 1) + base)) | FLAG;
                    else diag[d] = (uint32_t)stamp;
                }
            }
            base += slen + j->window;
            j->counters[3 * (int64_t)oid + 0] = hits;
            j->counters[3 * (int64_t)oid + 1] = succ;
            j->counters[3 * (int64_t)oid + 2] = ext;
        }
    }
    free(diag);
    return NULL;
}

int64_t or_scan(const uint8_t* db, const int64_t* db_off, int32_t n_subjects,
                const uint8_t* query, int32_t qlen,
                const uint32_t* cell_start, const uint16_t* entries,
                int32_t n_ctx, const int32_t* ctx_offset, const int32_t* ctx_xdrop,
                const int32_t* ctx_cutoff, int32_t window, int32_t diag_mask,
                const int8_t* matrix28, int32_t n_threads,
                int32_t* counters, int64_t* hsp_off, or_hsp* hsps, int64_t hsp_cap)
{
    if (n_threads <= 0) n_threads = (int32_t)sysconf(_SC_NPROCESSORS_ONLN);
    if (n_threads < 1) n_threads = 1;
    int32_t cursor = 0;
    job_t job = { db, db_off, n_subjects, query, qlen, cell_start, entries,
                  n_ctx, ctx_offset, ctx_xdrop, ctx_cutoff, window, diag_mask,
                  matrix28, counters, &cursor };
    worker_t* ws = (worker_t*)calloc((size_t)n_threads, sizeof(worker_t));
    pthread_t* th = (pthread_t*)calloc((size_t)n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        ws[t].job = &job;
        if (n_threads == 1) worker_main(&ws[t]);
        else pthread_create(&th[t], NULL, worker_main, &ws[t]);
    }
    if (n_threads > 1)
        for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);

    int64_t acc = 0;
    for (int32_t i = 0; i < n_subjects; ++i) { hsp_off[i] = acc; acc += counters[3 * (int64_t)i + 1]; }
    hsp_off[n_subjects] = acc;
    for (int t = 0; t < n_threads; ++t) {
        int32_t cur = -1; int64_t rank = 0;
        for (int64_t r = 0; r < ws[t].nrec; ++r) {
            const rec_t* x = &ws[t].recs[r];
            if (x->oid != cur) { cur = x->oid; rank = 0; }
            int64_t dst = hsp_off[cur] + rank++;
            if (dst < hsp_cap) hsps[dst] = x->h;
        }
        free(ws[t].recs);
    }
    free(ws);
    free(th);
    return acc;
}
