// The gapped stage: score-only gapped X-drop extension with affine gaps from
// a seed in each ungapped HSP of a finished search -- the consumer of the
// ungapped HSPs, which the reference hands to NCBI's GetGappedScore
// (ncbi_blast_files/blast_engine.c:588-591; NCBI's code is not in the
// reference).  The algorithm is the published one (Altschul et al. 1997,
// Nucleic Acids Res. 25:3389: a seed at the centre of the best 11-letter
// segment of the ungapped HSP, then X-drop dynamic programming with affine gap
// costs in both directions); the exact conventions -- order, skipping of
// contained HSPs, seed, band, row-synchronous X-drop, tie-breaking -- are
// stated in include/blastp_b200.h at bp_gapped_run and followed bit for bit.
//
// Mapping: one warp per subject that has ungapped HSPs (subjects come from a
// cursor in blocks of 32, a ballot picks the non-empty ones).  The warp ranks
// the subject's HSPs by score, then takes them in order: a containment test
// against the gapped HSPs reported so far (one lane per earlier HSP), the
// seed (one lane per 11-letter window, a warp arg-max), and the two
// extensions.  An extension runs row by row (one query letter per row); a row
// is computed in blocks of 32 columns (one subject letter per lane):
//   t(j)  = max(H(i-1,j-1) + S, F(i,j))    (diagonal from the previous lane)
//   E(i,j) = max over k < j of t(k) - open - (j-k) extend
//          = an exclusive prefix max of t(k) + k extend across the lanes,
//            carried from block to block
//   H(i,j) = max(t(j), E(i,j))
// (a path that opens a horizontal gap from a cell reached by one is never
// better, gap opening being >= 0).  The previous row's cells are kept in a
// per-warp ring of columns in global memory (L1-resident) and read with the
// X-drop test of that row applied (a cell below best - xdrop is dead), so no
// separate pruning pass is needed; only the first and last live columns of
// the row are looked up after it.  A band wider than the ring aborts the
// subject, which a second launch redoes with a ring as wide as its subject.
#include <string.h>

#include <algorithm>
#include <vector>

#include "bp_internal.h"

#define CK(call, what)                                                    \
    do {                                                                  \
        cudaError_t _err = (call);                                        \
        if (_err != cudaSuccess) return bp_set_cuda_error(e, _err, what); \
    } while (0)

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int32_t kNeg = -(1 << 28);        // a dead cell
constexpr int kWindow = 11;                 // seed window
constexpr int kWarps = 8;                   // warps per CTA

struct GappedArgs {
    const uint8_t* db;
    const int64_t* db_off;
    int32_t first;               // result subject s is database subject first + s
    int32_t n;                   // subjects of the result
    const uint8_t* query;
    int32_t qlen;
    const int8_t* matrix;        // [28][32]
    const int64_t* hoff;         // ungapped CSR
    const bp_hsp* hsps;
    int32_t open, ext, xdrop, cutoff;
    int32_t ring;                // columns per warp (power of two, >= 64)
    int2* rings;                 // (H, F) per column, ring columns per warp
    int32_t* order;              // one per ungapped HSP: the processing order
    bp_gapped_hsp* staging;      // one per ungapped HSP: subject s's reports at hoff[s]..
    int32_t* counters;           // 3 per subject
    uint32_t* cursor;
    uint32_t* n_over;            // subjects whose band outgrew the ring
    int32_t* over;               // their indices
    const int32_t* only;         // when set: process these n_only subjects (one per warp)
    int32_t n_only;
};

__device__ __forceinline__ int32_t cl(int32_t v) { return v < kNeg ? kNeg : v; }

__device__ __forceinline__ int32_t warp_max(int32_t v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ int32_t warp_min(int32_t v) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

struct ExtResult {
    int32_t best, bi, bj;
    bool over;
};

// One extension: A (M letters) and B (N letters) read at A[dir * i], B[dir * j].
__device__ ExtResult extend(const GappedArgs& g, const int8_t* m, const uint8_t* __restrict__ A, int32_t M,
                            const uint8_t* __restrict__ B, int32_t N, int dir, int2* ring, int lane) {
    const int32_t open = g.open, ext = g.ext, xdrop = g.xdrop;
    const int32_t mask = g.ring - 1;
    ExtResult r{0, 0, 0, false};
    // row 0: the origin, then gap cells -(open + j ext) while >= -xdrop
    int32_t last = 0;
    if (open + ext <= xdrop && N > 0) last = min(N, (xdrop - open) / ext);
    if (last + 1 > g.ring) {
        r.over = true;
        return r;
    }
    for (int32_t j = lane; j <= last; j += 32) ring[j & mask] = make_int2(j == 0 ? 0 : -(open + j * ext), kNeg);
    __syncwarp();
    int32_t lo = 0, best = 0;
    for (int32_t i = 1; i <= M; ++i) {
        const int ai = A[dir * (i - 1)];
        const int8_t* mrow = m + ai * BP_MROW;
        const int32_t floor_prev = best - xdrop;
        int32_t carry_e = kNeg, carry_diag = kNeg;
        int32_t lmax = kNeg, lmax_j = 0x7fffffff;      // this lane's best cell of the row
        int32_t end = -1;
        // this lane's cells of the row's first block and of its last two
        // blocks (kNeg where not computed), for the live-range search below
        int32_t h_first = kNeg, h_last = kNeg, h_prev = kNeg;
        int32_t b_last = lo;
        for (int32_t b0 = lo;; b0 += 32) {
            if (b0 + 32 > lo + g.ring) {                // the row would wrap onto itself
                r.over = true;
                return r;
            }
            const int32_t j = b0 + lane;
            const bool valid = j <= N;
            int2 up = make_int2(kNeg, kNeg);
            if (valid && j <= last) {
                up = ring[j & mask];
                if (up.x < floor_prev) up = make_int2(kNeg, kNeg);   // dead in the previous row
            }
            const int32_t f = cl(max(up.x - open, up.y) - ext);
            int32_t diag = __shfl_up_sync(kFull, up.x, 1);
            if (lane == 0) diag = carry_diag;
            int32_t d = kNeg;
            if (valid && diag != kNeg) d = diag + mrow[__ldg(B + dir * (j - 1))];
            const int32_t t = max(d, f);
            // E: exclusive prefix max of t(k) + k ext over the lanes, then the carry
            const int32_t v = t + lane * ext;
            int32_t incl = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t y = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl = max(incl, y);
            }
            int32_t excl = __shfl_up_sync(kFull, incl, 1);
            int32_t e = cl(carry_e - lane * ext);
            if (lane > 0) e = max(e, cl(excl - open - lane * ext));
            const bool stop = !valid || (j > last + 1 && e < floor_prev);
            const unsigned sm = __ballot_sync(kFull, stop);
            const int first_stop = sm ? __ffs(sm) - 1 : 32;
            const int32_t h = max(t, e);
            const int32_t hk = lane < first_stop ? h : kNeg;
            if (b0 == lo) h_first = hk;
            h_prev = h_last;
            h_last = hk;
            b_last = b0;
            if (lane < first_stop) {
                ring[j & mask] = make_int2(h, f);
                if (h > lmax) {
                    lmax = h;
                    lmax_j = j;
                }
            }
            if (first_stop < 32) {
                end = b0 + first_stop;
                break;
            }
            const int32_t vmax = __shfl_sync(kFull, incl, 31);
            carry_e = cl(max(carry_e - 32 * ext, vmax - open - 32 * ext));
            carry_diag = __shfl_sync(kFull, up.x, 31);
        }
        __syncwarp();
        // the row's maximum and the first column holding it
        const int32_t rmax = warp_max(lmax);
        const int32_t rj = warp_min(lmax == rmax ? lmax_j : 0x7fffffff);
        if (rmax > best) {
            best = rmax;
            r.best = rmax;
            r.bi = i;
            r.bj = rj;
        }
        // live range of the row: first and last column >= best - xdrop
        const int32_t floor_now = best - xdrop;
        // (blocks held in registers answer without the ring: the first block
        // for the first live column, the last two for the last one)
        int32_t first_live = -1;
        {
            const unsigned lm = __ballot_sync(kFull, h_first >= floor_now);
            if (lm) first_live = lo + __ffs(lm) - 1;
        }
        for (int32_t b0 = lo + 32; b0 < end && first_live < 0; b0 += 32) {
            const int32_t j = b0 + lane;
            const bool live = j < end && ring[j & mask].x >= floor_now;
            const unsigned lm = __ballot_sync(kFull, live);
            if (lm) first_live = b0 + __ffs(lm) - 1;
        }
        if (first_live < 0) break;
        int32_t last_live = -1;
        {
            const unsigned lm = __ballot_sync(kFull, h_last >= floor_now);
            if (lm) last_live = b_last + (31 - __clz(lm));
        }
        if (last_live < 0 && b_last > lo) {
            const unsigned lm = __ballot_sync(kFull, h_prev >= floor_now);
            if (lm) last_live = b_last - 32 + (31 - __clz(lm));
        }
        for (int32_t b1 = b_last - 32; last_live < 0; b1 -= 32) {
            const int32_t j = b1 - 32 + lane;
            const bool live = j >= first_live && j < end && ring[j & mask].x >= floor_now;
            const unsigned lm = __ballot_sync(kFull, live);
            if (lm) last_live = b1 - 32 + (31 - __clz(lm));
        }
        lo = first_live;
        last = last_live;
        __syncwarp();
    }
    return r;
}

// Subject s of the result (all lanes).  Returns false when a band outgrew the ring.
__device__ bool gapped_subject(const GappedArgs& g, const int8_t* m, int32_t s, int2* ring, int lane) {
    const int64_t base = g.hoff[s];
    const int32_t n_u = (int32_t)(g.hoff[s + 1] - base);
    const bp_hsp* u = g.hsps + base;
    // rank by score, descending; equal scores in discovery order
    for (int32_t k = lane; k < n_u; k += 32) {
        const int32_t sk = u[k].score;
        int32_t rank = 0;
        for (int32_t t = 0; t < n_u; ++t) {
            const int32_t st = u[t].score;
            rank += (st > sk || (st == sk && t < k)) ? 1 : 0;
        }
        g.order[base + rank] = k;
    }
    __syncwarp();
    const int64_t so = g.db_off[g.first + s];
    const uint8_t* sub = g.db + so;
    const int32_t slen = (int32_t)(g.db_off[g.first + s + 1] - so);
    const uint8_t* q = g.query;
    bp_gapped_hsp* out = g.staging + base;
    int32_t n_out = 0, n_ext = 0;
    for (int32_t r = 0; r < n_u; ++r) {
        const int32_t k = g.order[base + r];
        const bp_hsp h = u[k];
        bool inside = false;
        for (int32_t t = lane; t < n_out; t += 32) {
            const bp_gapped_hsp o = out[t];
            inside |= o.q_start <= h.hsp_q && h.hsp_q + h.hsp_len <= o.q_end && o.s_start <= h.hsp_s &&
                      h.hsp_s + h.hsp_len <= o.s_end;
        }
        if (__any_sync(kFull, inside)) continue;
        // seed: the middle of a short HSP, else of its first best 11-letter window
        int32_t qs = h.hsp_q + h.hsp_len / 2, ss = h.hsp_s + h.hsp_len / 2;
        if (h.hsp_len > kWindow) {
            int32_t wbest = kNeg, wk = 0x7fffffff;
            for (int32_t w0 = lane; w0 + kWindow <= h.hsp_len; w0 += 32) {
                int32_t acc = 0;
#pragma unroll
                for (int t = 0; t < kWindow; ++t) acc += m[q[h.hsp_q + w0 + t] * BP_MROW + __ldg(sub + h.hsp_s + w0 + t)];
                if (acc > wbest) {
                    wbest = acc;
                    wk = w0;
                }
            }
            const int32_t wm = warp_max(wbest);
            const int32_t kk = warp_min(wbest == wm ? wk : 0x7fffffff);
            qs = h.hsp_q + kk + kWindow / 2;
            ss = h.hsp_s + kk + kWindow / 2;
        }
        const ExtResult L = extend(g, m, q + qs, qs + 1, sub + ss, ss + 1, -1, ring, lane);
        if (L.over) return false;
        const ExtResult R = extend(g, m, q + qs + 1, g.qlen - qs - 1, sub + ss + 1, slen - ss - 1, 1, ring, lane);
        if (R.over) return false;
        ++n_ext;
        const int32_t score = L.best + R.best;
        if (score >= g.cutoff) {
            if (lane == 0) {
                bp_gapped_hsp o;
                o.score = score;
                o.q_start = qs + 1 - L.bi;
                o.q_end = qs + 1 + R.bi;
                o.s_start = ss + 1 - L.bj;
                o.s_end = ss + 1 + R.bj;
                o.q_seed = qs;
                o.s_seed = ss;
                o.ungapped = k;
                out[n_out] = o;
            }
            ++n_out;
            __syncwarp();
        }
    }
    if (lane == 0) {
        g.counters[3 * (int64_t)s + 0] = n_u;
        g.counters[3 * (int64_t)s + 1] = n_out;
        g.counters[3 * (int64_t)s + 2] = n_ext;
    }
    return true;
}

__global__ void __launch_bounds__(kWarps * 32) gapped_kernel(GappedArgs g) {
    __shared__ int8_t m[28 * BP_MROW];
    for (int i = threadIdx.x; i < 28 * BP_MROW; i += blockDim.x) m[i] = g.matrix[i];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t warp_id = (int64_t)blockIdx.x * kWarps + (threadIdx.x >> 5);
    int2* ring = g.rings + warp_id * g.ring;
    if (g.only) {
        for (int64_t i = warp_id; i < g.n_only; i += (int64_t)gridDim.x * kWarps) {
            const int32_t s = g.only[i];
            // (the ring spans the whole subject here, so no band can outgrow it)
            if (!gapped_subject(g, m, s, ring, lane) && lane == 0) g.counters[3 * (int64_t)s + 1] = 0;
        }
        return;
    }
    for (;;) {
        uint32_t blk = 0;
        if (lane == 0) blk = atomicAdd(g.cursor, 1u);
        blk = __shfl_sync(kFull, blk, 0);
        const int64_t s0 = (int64_t)blk * 32;
        if (s0 >= g.n) break;
        const int32_t s = (int32_t)(s0 + lane);
        bool has = false;
        if (s < g.n) {
            has = g.hoff[s + 1] > g.hoff[s];
            if (!has) {
                g.counters[3 * (int64_t)s + 0] = 0;
                g.counters[3 * (int64_t)s + 1] = 0;
                g.counters[3 * (int64_t)s + 2] = 0;
            }
        }
        unsigned todo = __ballot_sync(kFull, has);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const int32_t sub = (int32_t)(s0 + l);
            if (!gapped_subject(g, m, sub, ring, lane) && lane == 0) {
                g.counters[3 * (int64_t)sub + 0] = (int32_t)(g.hoff[sub + 1] - g.hoff[sub]);
                g.counters[3 * (int64_t)sub + 1] = 0;
                g.counters[3 * (int64_t)sub + 2] = 0;
                g.over[atomicAdd(g.n_over, 1u)] = sub;
            }
            __syncwarp();
        }
    }
}

// Gapped HSPs from their per-subject staging slots (at the ungapped offsets)
// to the dense CSR.
__global__ void gather_gapped(int32_t n, const int64_t* __restrict__ hoff, const int32_t* __restrict__ counters,
                              const int64_t* __restrict__ goff, const bp_gapped_hsp* __restrict__ staging,
                              bp_gapped_hsp* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < n; s += warps) {
        const int32_t c = counters[3 * s + 1];
        for (int32_t k = lane; k < c; k += 32) out[goff[s] + k] = staging[hoff[s] + k];
    }
}

}  // namespace

struct bp_gapped {
    bp_engine* e = nullptr;
    int32_t n = 0;
    int32_t* d_counters = nullptr;
    int64_t* d_off = nullptr;
    bp_gapped_hsp* d_hsps = nullptr;
    int64_t n_hsps = 0;
    float ms = 0.f;
};

void bp_gapped_params_default(bp_gapped_params* p) {
    if (!p) return;
    p->gap_open = 11;
    p->gap_extend = 1;
    p->x_dropoff = 38;
    p->cutoff_score = 0;
}

#define CKG(call, what)                                                        \
    do {                                                                       \
        cudaError_t _err = (call);                                             \
        if (_err != cudaSuccess) {                                             \
            bp_gapped_destroy(gp);                                             \
            for (void* _p : scratch) cudaFree(_p);                             \
            return bp_set_cuda_error(e, _err, what);                           \
        }                                                                      \
    } while (0)

bp_status bp_gapped_run_ring(bp_result* r, const bp_gapped_params* p, int32_t ring_columns, bp_gapped** out) {
    if (!r || !p || !out) return BP_ERR_INVALID;
    if (p->gap_open < 0 || p->gap_open > 65535 || p->gap_extend < 1 || p->gap_extend > 255 || p->x_dropoff < 0 ||
        p->x_dropoff > (1 << 20) || ring_columns < 64 || (ring_columns & (ring_columns - 1)))
        return BP_ERR_INVALID;
    bp_status st = bp_result_wait(r);
    if (st != BP_OK) return st;
    bp_engine* e = r->e;
    if (!r->db || !r->q) return bp_set_error(e, BP_ERR_INVALID, "bp_gapped_run: the search's database or query is gone");
    if (r->q->n_ctx != 1) return bp_set_error(e, BP_ERR_INVALID, "bp_gapped_run: single-context queries only");
    const int32_t n = r->n;
    const int64_t n_u = r->n_hsps;
    std::vector<void*> scratch;
    bp_gapped* gp = new bp_gapped();
    gp->e = e;
    gp->n = n;
    CKG(cudaSetDevice(e->device), "cudaSetDevice");
    cudaStream_t cs = e->stream;
    CKG(cudaMalloc((void**)&gp->d_counters, ((size_t)n + 1) * 3 * sizeof(int32_t)), "cudaMalloc(gapped counters)");
    CKG(cudaMalloc((void**)&gp->d_off, ((size_t)n + 1) * sizeof(int64_t)), "cudaMalloc(gapped offsets)");
    int32_t* d_order = nullptr;
    bp_gapped_hsp* d_staging = nullptr;
    uint32_t* d_words = nullptr;       // [0] cursor, [1] subjects over the ring
    int32_t* d_over = nullptr;
    int32_t* d_fill = nullptr;
    int64_t* d_sums = nullptr;
    const size_t nu = (size_t)std::max<int64_t>(n_u, 1);
    CKG(cudaMalloc((void**)&d_order, nu * sizeof(int32_t)), "cudaMalloc(order)");
    scratch.push_back(d_order);
    CKG(cudaMalloc((void**)&d_staging, nu * sizeof(bp_gapped_hsp)), "cudaMalloc(staging)");
    scratch.push_back(d_staging);
    CKG(cudaMalloc((void**)&d_words, 4 * sizeof(uint32_t)), "cudaMalloc(words)");
    scratch.push_back(d_words);
    CKG(cudaMalloc((void**)&d_over, (size_t)std::max(n, 1) * sizeof(int32_t)), "cudaMalloc(overflow list)");
    scratch.push_back(d_over);
    CKG(cudaMalloc((void**)&d_fill, (size_t)std::max(n, 1) * sizeof(int32_t)), "cudaMalloc(fill)");
    scratch.push_back(d_fill);
    CKG(cudaMalloc((void**)&d_sums, (size_t)bp_order_blocksums_needed(n) * sizeof(int64_t)), "cudaMalloc(sums)");
    scratch.push_back(d_sums);
    CKG(cudaMemsetAsync(d_words, 0, 4 * sizeof(uint32_t), cs), "memset");

    GappedArgs g{};
    g.db = r->db->d_res;
    g.db_off = r->db->d_off;
    g.first = r->first;
    g.n = n;
    g.query = r->q->d_q;
    g.qlen = r->q->qlen;
    g.matrix = e->d_matrix;
    g.hoff = r->d_hsp_off;
    g.hsps = r->d_hsps;
    g.open = p->gap_open;
    g.ext = p->gap_extend;
    g.xdrop = p->x_dropoff;
    g.cutoff = p->cutoff_score;
    g.order = d_order;
    g.staging = d_staging;
    g.counters = gp->d_counters;
    g.cursor = d_words;
    g.n_over = d_words + 1;
    g.over = d_over;
    const int grid = e->sm_count * 4;          // 32 warps per SM
    g.ring = ring_columns;
    int2* d_rings = nullptr;
    CKG(cudaMalloc((void**)&d_rings, (size_t)grid * kWarps * ring_columns * sizeof(int2)), "cudaMalloc(rings)");
    scratch.push_back(d_rings);
    g.rings = d_rings;
    // the reports never outnumber the ungapped HSPs: the output is sized once
    CKG(cudaMalloc((void**)&gp->d_hsps, nu * sizeof(bp_gapped_hsp)), "cudaMalloc(gapped hsps)");
    // kernel, offsets and gather enqueued back to back; one read-back at the
    // end says whether any subject needs the wide-ring launch (then the
    // offsets and gather run again behind it)
    auto finish = [&]() -> cudaError_t {
        cudaError_t err = bp_launch_offsets(e, cs, n, gp->d_counters, gp->d_off, d_fill, d_sums);
        if (err == cudaSuccess && n > 0) {
            gather_gapped<<<e->sm_count * 4, 256, 0, cs>>>(n, r->d_hsp_off, gp->d_counters, gp->d_off, d_staging,
                                                          gp->d_hsps);
            e->launches += 1;
            err = cudaGetLastError();
        }
        return err;
    };
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    CKG(cudaEventCreate(&t0), "cudaEventCreate");
    CKG(cudaEventCreate(&t1), "cudaEventCreate");
    struct Events {
        cudaEvent_t& a;
        cudaEvent_t& b;
        ~Events() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } events{t0, t1};
    uint32_t* h_words = bp_pinned_get(e);
    if (!h_words) {
        bp_gapped_destroy(gp);
        for (void* q : scratch) cudaFree(q);
        return bp_set_error(e, BP_ERR_NOMEM, "bp_gapped_run: pinned read-back slot");
    }
    struct Slot {
        bp_engine* e;
        uint32_t* p;
        ~Slot() { bp_pinned_put(e, p); }
    } slot{e, h_words};
    CKG(cudaEventRecord(t0, cs), "cudaEventRecord");
    if (n > 0) {
        gapped_kernel<<<grid, kWarps * 32, 0, cs>>>(g);
        e->launches += 1;
        CKG(cudaGetLastError(), "gapped kernel launch");
    }
    CKG(finish(), "gapped offsets and gather");
    CKG(cudaEventRecord(t1, cs), "cudaEventRecord");
    CKG(cudaMemcpyAsync(h_words, d_words, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, cs), "read overflow count");
    CKG(cudaStreamSynchronize(cs), "gapped stage");
    cudaEventElapsedTime(&gp->ms, t0, t1);
    const uint32_t n_over = h_words[1];
    if (n_over > 0) {
        // subjects whose band outgrew the ring: again, one warp each, with a
        // ring as wide as the longest of them
        std::vector<int32_t> over(n_over);
        CKG(cudaMemcpy(over.data(), d_over, n_over * sizeof(int32_t), cudaMemcpyDeviceToHost), "read overflow list");
        int64_t widest = 64;
        std::vector<int64_t> offs(2);
        for (int32_t s : over) {
            CKG(cudaMemcpy(offs.data(), r->db->d_off + r->first + s, 2 * sizeof(int64_t), cudaMemcpyDeviceToHost),
                "read subject span");
            widest = std::max<int64_t>(widest, offs[1] - offs[0] + 2);
        }
        int64_t ring2 = 64;
        while (ring2 < widest + 32) ring2 <<= 1;
        const int64_t budget = (int64_t)1 << 30;   // bytes of rings for the second launch
        int64_t warps2 = std::max<int64_t>(1, std::min<int64_t>((int64_t)n_over, budget / (ring2 * 8)));
        warps2 = std::min<int64_t>(warps2, (int64_t)e->sm_count * 8 * kWarps);
        const int grid2 = (int)((warps2 + kWarps - 1) / kWarps);
        int2* d_rings2 = nullptr;
        CKG(cudaMalloc((void**)&d_rings2, (size_t)grid2 * kWarps * ring2 * sizeof(int2)), "cudaMalloc(wide rings)");
        scratch.push_back(d_rings2);
        GappedArgs g2 = g;
        g2.ring = (int32_t)ring2;
        g2.rings = d_rings2;
        g2.only = d_over;
        g2.n_only = (int32_t)n_over;
        CKG(cudaEventRecord(t0, cs), "cudaEventRecord");
        gapped_kernel<<<grid2, kWarps * 32, 0, cs>>>(g2);
        e->launches += 1;
        CKG(cudaGetLastError(), "gapped kernel launch (wide rings)");
        CKG(finish(), "gapped offsets and gather");
        CKG(cudaEventRecord(t1, cs), "cudaEventRecord");
        CKG(cudaStreamSynchronize(cs), "gapped stage (wide rings)");
        float ms2 = 0.f;
        cudaEventElapsedTime(&ms2, t0, t1);
        gp->ms += ms2;
    }
    CKG(cudaMemcpy(&gp->n_hsps, gp->d_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost), "read gapped count");
    for (void* q : scratch) cudaFree(q);
    *out = gp;
    return BP_OK;
}

bp_status bp_gapped_run(bp_result* r, const bp_gapped_params* p, bp_gapped** out) {
    return bp_gapped_run_ring(r, p, 2048, out);
}

int64_t bp_gapped_hsps(const bp_gapped* g) { return g ? g->n_hsps : -1; }
float bp_gapped_ms(const bp_gapped* g) { return g ? g->ms : 0.f; }

bp_status bp_gapped_copy(bp_gapped* g, int32_t* counters, int64_t* off, bp_gapped_hsp* hsps) {
    if (!g) return BP_ERR_INVALID;
    bp_engine* e = g->e;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    if (counters && g->n > 0)
        CK(cudaMemcpy(counters, g->d_counters, (size_t)g->n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost),
           "copy gapped counters");
    if (off) CK(cudaMemcpy(off, g->d_off, ((size_t)g->n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost), "copy offsets");
    if (hsps && g->n_hsps > 0)
        CK(cudaMemcpy(hsps, g->d_hsps, (size_t)g->n_hsps * sizeof(bp_gapped_hsp), cudaMemcpyDeviceToHost),
           "copy gapped hsps");
    return BP_OK;
}

void bp_gapped_destroy(bp_gapped* g) {
    if (!g) return;
    if (g->e) cudaSetDevice(g->e->device);
    cudaFree(g->d_counters);
    cudaFree(g->d_off);
    cudaFree(g->d_hsps);
    delete g;
}
