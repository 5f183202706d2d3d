/*
 * gapped.c -- CPU oracle of the gapped stage that consumes the ungapped
 * HSPs: score-only gapped X-drop extension with affine gaps from a seed in
 * each ungapped HSP.  TEST INFRASTRUCTURE ONLY: the tests use it as the
 * checker of the device's gapped stage; the product never links it.
 *
 * Parity status: UNPINNED.  The reference hands its ungapped HSPs to NCBI
 * BLAST+ 2.2.28's GetGappedScore (ncbi_blast_files/blast_engine.c:588-591),
 * whose code (blast_gapalign.c) is not in the reference tree.  This file
 * restates the published algorithm (Altschul et al. 1997, Nucleic Acids Res.
 * 25:3389-3402, "Gapped BLAST and PSI-BLAST": a seed at the centre of the
 * best 11-letter segment of an ungapped HSP, then X-drop dynamic programming
 * with affine gap costs in both directions) with the exact conventions of
 * gapped.h, which the device kernel follows bit for bit.  It is not NCBI's
 * code and is not claimed to reproduce NCBI's outputs.
 */
#define _GNU_SOURCE
#include "gapped.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static inline int sc(const int8_t* m, int a, int b) { return m[a * OR_ALPHA + b]; }
static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int32_t cl(int32_t v) { return v < OR_GNEG ? OR_GNEG : v; }

/* One extension (gapped.h, "extension").  H and F hold N+1 ints each. */
int32_t or_gapped_extend(const int8_t* m, const uint8_t* A, int32_t M, const uint8_t* B, int32_t N, int32_t dir,
                         int32_t xdrop, int32_t open, int32_t ext, int32_t* H, int32_t* F, int32_t* bi,
                         int32_t* bj)
{
    int32_t best = 0, best_i = 0, best_j = 0;
    /* row 0: the origin, then gap cells while >= -xdrop */
    H[0] = 0;
    F[0] = OR_GNEG;
    int32_t lo = 0, last = 0;
    {
        int32_t e = OR_GNEG, h_left = 0;
        for (int32_t j = 1; j <= N; ++j) {
            e = cl(imax(h_left - open, e) - ext);
            if (e < -xdrop) break;
            H[j] = e;
            F[j] = OR_GNEG;
            h_left = e;
            last = j;
        }
    }
    for (int32_t i = 1; i <= M; ++i) {
        const int ai = A[dir * (i - 1)];
        const int32_t floor_prev = best - xdrop;
        int32_t row_max = OR_GNEG, row_j = -1;
        int32_t diag = OR_GNEG;                  /* H(i-1, j-1) */
        int32_t e = OR_GNEG, h_left = OR_GNEG;   /* E(i, j-1), H(i, j-1) */
        int32_t j = lo;
        for (; j <= N; ++j) {
            const int in_prev = j <= last;
            const int32_t up_h = in_prev ? H[j] : OR_GNEG;
            const int32_t up_f = in_prev ? F[j] : OR_GNEG;
            const int32_t f = cl(imax(up_h - open, up_f) - ext);
            e = cl(imax(h_left - open, e) - ext);
            const int32_t d = diag == OR_GNEG ? OR_GNEG : diag + sc(m, ai, B[dir * (j - 1)]);
            if (j > last + 1 && e < floor_prev) break;
            const int32_t h = imax(d, imax(e, f));
            H[j] = h;
            F[j] = f;
            diag = up_h;
            h_left = h;
            if (h > row_max) { row_max = h; row_j = j; }
        }
        const int32_t end = j;
        if (row_max > best) { best = row_max; best_i = i; best_j = row_j; }
        const int32_t floor_now = best - xdrop;
        int32_t first_live = -1, last_live = -1;
        for (int32_t k = lo; k < end; ++k) {
            if (H[k] < floor_now) {
                H[k] = OR_GNEG;
                F[k] = OR_GNEG;
            } else {
                if (first_live < 0) first_live = k;
                last_live = k;
            }
        }
        if (first_live < 0) break;
        lo = first_live;
        last = last_live;
    }
    *bi = best_i;
    *bj = best_j;
    return best;
}

void or_gapped_seed(const int8_t* m, const uint8_t* q, const uint8_t* s, int32_t hsp_q, int32_t hsp_s,
                    int32_t len, int32_t* q_seed, int32_t* s_seed)
{
    if (len <= OR_GWINDOW) {
        *q_seed = hsp_q + len / 2;
        *s_seed = hsp_s + len / 2;
        return;
    }
    int32_t w = 0;
    for (int t = 0; t < OR_GWINDOW; ++t) w += sc(m, q[hsp_q + t], s[hsp_s + t]);
    int32_t best = w, best_k = 0;
    for (int32_t k = 1; k + OR_GWINDOW <= len; ++k) {
        w += sc(m, q[hsp_q + k + OR_GWINDOW - 1], s[hsp_s + k + OR_GWINDOW - 1]) - sc(m, q[hsp_q + k - 1], s[hsp_s + k - 1]);
        if (w > best) { best = w; best_k = k; }
    }
    *q_seed = hsp_q + best_k + OR_GWINDOW / 2;
    *s_seed = hsp_s + best_k + OR_GWINDOW / 2;
}

/* The gapped stage for one subject; appends to out (capacity cap) and
 * returns the number of gapped HSPs reported.  H, F: work buffers of
 * slen + 1 ints; order: work array of n_u ints. */
static int32_t gapped_subject(const int8_t* m, const uint8_t* q, int32_t qlen, const uint8_t* s, int32_t slen,
                              const or_hsp* u, int32_t n_u, const or_gparams* p, int32_t* H, int32_t* F,
                              int32_t* order, or_ghsp* out)
{
    /* descending score, discovery order among equals (insertion sort: stable) */
    for (int32_t k = 0; k < n_u; ++k) {
        int32_t t = k;
        while (t > 0 && u[order[t - 1]].score < u[k].score) { order[t] = order[t - 1]; --t; }
        order[t] = k;
    }
    int32_t n_out = 0;
    for (int32_t r = 0; r < n_u; ++r) {
        const or_hsp* h = &u[order[r]];
        int contained = 0;
        for (int32_t g = 0; g < n_out && !contained; ++g)
            contained = out[g].q_start <= h->hsp_q && h->hsp_q + h->hsp_len <= out[g].q_end &&
                        out[g].s_start <= h->hsp_s && h->hsp_s + h->hsp_len <= out[g].s_end;
        if (contained) continue;
        int32_t qs, ss;
        or_gapped_seed(m, q, s, h->hsp_q, h->hsp_s, h->hsp_len, &qs, &ss);
        int32_t li, lj, ri, rj;
        const int32_t L = or_gapped_extend(m, q + qs, qs + 1, s + ss, ss + 1, -1, p->xdrop, p->gap_open,
                                           p->gap_extend, H, F, &li, &lj);
        const int32_t R = or_gapped_extend(m, q + qs + 1, qlen - qs - 1, s + ss + 1, slen - ss - 1, 1, p->xdrop,
                                           p->gap_open, p->gap_extend, H, F, &ri, &rj);
        const int32_t score = L + R;
        if (score < p->cutoff) continue;
        or_ghsp* o = &out[n_out++];
        o->score = score;
        o->q_start = qs + 1 - li;
        o->q_end = qs + 1 + ri;
        o->s_start = ss + 1 - lj;
        o->s_end = ss + 1 + rj;
        o->q_seed = qs;
        o->s_seed = ss;
        o->ungapped = order[r];
    }
    return n_out;
}

typedef struct {
    const uint8_t* db; const int64_t* db_off; int32_t n;
    const uint8_t* q; int32_t qlen;
    const int64_t* hoff; const or_hsp* hsps;
    const int8_t* m; const or_gparams* p;
    int64_t* counts; or_ghsp** per;
    int32_t* cursor;
} gjob_t;

static void* gworker(void* arg)
{
    gjob_t* j = (gjob_t*)arg;
    int32_t cap_len = 0, cap_u = 0;
    int32_t *H = NULL, *F = NULL, *order = NULL;
    for (;;) {
        const int32_t oid = __atomic_fetch_add(j->cursor, 1, __ATOMIC_RELAXED);
        if (oid >= j->n) break;
        const int32_t n_u = (int32_t)(j->hoff[oid + 1] - j->hoff[oid]);
        j->counts[oid] = 0;
        if (n_u == 0) continue;
        const int32_t slen = (int32_t)(j->db_off[oid + 1] - j->db_off[oid]);
        if (slen + 1 > cap_len) {
            cap_len = slen + 1;
            H = (int32_t*)realloc(H, sizeof(int32_t) * cap_len);
            F = (int32_t*)realloc(F, sizeof(int32_t) * cap_len);
        }
        if (n_u > cap_u) {
            cap_u = n_u;
            order = (int32_t*)realloc(order, sizeof(int32_t) * cap_u);
        }
        or_ghsp* out = (or_ghsp*)malloc(sizeof(or_ghsp) * n_u);
        j->counts[oid] = gapped_subject(j->m, j->q, j->qlen, j->db + j->db_off[oid], slen, j->hsps + j->hoff[oid], n_u,
                                        j->p, H, F, order, out);
        j->per[oid] = out;
    }
    free(H);
    free(F);
    free(order);
    return NULL;
}

int64_t or_gapped(const uint8_t* db, const int64_t* db_off, int32_t n_subjects, const uint8_t* query, int32_t qlen,
                  const int64_t* hsp_off, const or_hsp* hsps, const int8_t* matrix28, const or_gparams* p,
                  int32_t n_threads, int64_t* goff, or_ghsp* out, int64_t cap)
{
    int64_t* counts = (int64_t*)calloc((size_t)n_subjects + 1, sizeof(int64_t));
    or_ghsp** per = (or_ghsp**)calloc((size_t)n_subjects + 1, sizeof(or_ghsp*));
    int32_t cursor = 0;
    gjob_t job = {db, db_off, n_subjects, query, qlen, hsp_off, hsps, matrix28, p, counts, per, &cursor};
    if (n_threads < 1) n_threads = 1;
    pthread_t* tid = (pthread_t*)malloc(sizeof(pthread_t) * n_threads);
    for (int t = 0; t < n_threads; ++t) pthread_create(&tid[t], NULL, gworker, &job);
    for (int t = 0; t < n_threads; ++t) pthread_join(tid[t], NULL);
    free(tid);
    int64_t total = 0;
    goff[0] = 0;
    for (int32_t s = 0; s < n_subjects; ++s) {
        for (int64_t k = 0; k < counts[s]; ++k)
            if (total + k < cap) out[total + k] = per[s][k];
        total += counts[s];
        goff[s + 1] = total;
        free(per[s]);
    }
    free(per);
    free(counts);
    return total;
}
