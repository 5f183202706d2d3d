// Plain scan kernel: one query against a range of subjects.
//
// Semantics follow the reference kernel GPU_BLASTP_kernelTwoHit
// (gpu_blastp_kernel.cu:42-320) and its extenders (:341-549); the mapping to
// the hardware does not:
//  * a warp owns one subject at a time (subjects handed out by an atomic
//    cursor, so length skew does not idle a CTA) instead of a thread per
//    subject;
//  * the warp reads 32 consecutive word positions, looks them up in the
//    presence bitmap (shared memory) and the CSR table, and flattens the
//    resulting word hits into chunks of 32 -- one hit per lane, whatever the
//    per-position hit counts are;
//  * the per-diagonal two-hit state lives in shared memory, one array per
//    warp (the reference keeps it in global memory, one per thread);
//  * hits of one chunk that fall on the same diagonal are ordered with
//    __match_any_sync: they are applied in word-position order, which is the
//    only order the state machine depends on (distinct diagonals are
//    independent);
//  * surviving HSPs are compacted with a warp ballot into one global append
//    buffer, tagged with the subject and the hit's index in the subject's hit
//    stream so a later pass can restore the reference's discovery order.
#include "bp_internal.h"

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr uint32_t kFlag = 0x80000000u;

struct ExtOut {
    int hsp_q, hsp_s, len, score, s_last, right_ext;
};

__device__ __forceinline__ int msc(const int8_t* m, int a, int b) { return m[a * BP_MROW + b]; }

// s_BlastAaExtendTwoHit (gpu_blastp_kernel.cu:341-415) with the left
// (:435-481) and right (:503-549) X-drop walks inlined.  Subject read through
// the read-only path, query and matrix from shared memory.
__device__ ExtOut extend_two_hit(const int8_t* m, const uint8_t* __restrict__ subj, int slen,
                                 const uint8_t* qry, int qlen, int s_left, int s_right,
                                 int q_right, int xdrop) {
    int score = 0, left_score = 0, shift = 0;
#pragma unroll
    for (int i = 0; i < BP_WORD; ++i) {
        score += msc(m, qry[q_right + i], __ldg(subj + s_right + i));
        if (score > left_score) {
            left_score = score;
            shift = i + 1;
        }
    }
    q_right += shift;
    s_right += shift;

    int s_off = s_right - 1, q_off = q_right - 1;
    int n = min(s_off, q_off);
    int run = 0, best = 0, best_k = -1;
    for (int k = 0; k <= n; ++k) {
        run += msc(m, qry[q_off - k], __ldg(subj + s_off - k));
        if (run > best) {
            best = run;
            best_k = k;
        }
        if (best - run >= xdrop) break;
    }
    int left_d = best_k + 1;
    left_score = best;

    ExtOut o;
    o.right_ext = 0;
    o.s_last = s_right;
    int right_d = 0, right_score = 0;
    if (left_d >= s_right - s_left) {
        o.right_ext = 1;
        int n2 = min(slen - s_right, qlen - q_right);
        int rrun = left_score, rbest = left_score, rbest_i = -1, i = 0;
        for (; i < n2; ++i) {
            rrun += msc(m, qry[q_right + i], __ldg(subj + s_right + i));
            if (rrun > rbest) {
                rbest = rrun;
                rbest_i = i;
            }
            if (rrun <= 0 || rbest - rrun >= xdrop) break;
        }
        right_d = rbest_i + 1;
        right_score = rbest;
        o.s_last = s_right + i;
    }
    o.hsp_q = q_right - left_d;
    o.hsp_s = s_right - left_d;
    o.len = left_d + right_d;
    o.score = max(left_score, right_score);
    return o;
}

// Last context whose first query offset is <= q (gpu_blastp_kernel.cu:238-241).
__device__ __forceinline__ int context_of(const int32_t* __restrict__ ctx, int n_ctx, int q) {
    int lo = 0, hi = n_ctx - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(ctx + 3 * mid) <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
scan_plain(ScanArgs a) {
    extern __shared__ __align__(16) uint8_t sm[];
    int8_t* m = reinterpret_cast<int8_t*>(sm);                 // 28 x 32, padded to 1 KB
    uint32_t* pv = reinterpret_cast<uint32_t*>(sm + 1024);     // 1024 words
    uint8_t* qs = sm + 1024 + 4096;
    const int qpad = (a.qlen + 15) & ~15;
    uint32_t* diag_all = reinterpret_cast<uint32_t*>(qs + qpad);
    const int L = a.diag_mask + 1;

    for (int i = threadIdx.x; i < 28 * BP_MROW; i += blockDim.x) m[i] = a.matrix[i];
    for (int i = threadIdx.x; i < BP_NCELL / 32; i += blockDim.x) pv[i] = a.pv[i];
    for (int i = threadIdx.x; i < a.qlen; i += blockDim.x) qs[i] = a.query[i];
    for (int i = threadIdx.x; i < WARPS * L; i += blockDim.x) diag_all[i] = 0;
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t* diag = diag_all + (threadIdx.x >> 5) * L;
    int base = a.window;   // diagonal stamp offset (gpu_blastp_kernel.cu:308)

    for (;;) {
        int oid = 0;
        if (lane == 0) oid = (int)atomicAdd(a.cursor, 1u);
        oid = __shfl_sync(kFull, oid, 0);
        if (oid >= a.n) break;
        const int64_t so = a.db_off[a.first + oid];
        const int slen = (int)(a.db_off[a.first + oid + 1] - so);
        const uint8_t* __restrict__ sub = a.db + so;
        if (base + slen + a.window > (1 << 30)) {
            for (int i = lane; i < L; i += 32) diag[i] = 0;
            __syncwarp();
            base = a.window;
        }
        int hits = 0, ext = 0, succ = 0, key_base = 0;
        for (int s0 = 0; s0 <= slen - BP_WORD; s0 += 32) {
            const int s = s0 + lane;
            uint32_t start = 0, cnt = 0;
            if (s <= slen - BP_WORD) {
                uint32_t c = ((uint32_t)__ldg(sub + s) << 10) | ((uint32_t)__ldg(sub + s + 1) << 5) |
                             (uint32_t)__ldg(sub + s + 2);
                if (pv[c >> 5] & (1u << (c & 31))) {
                    start = __ldg(a.cell_start + c);
                    cnt = __ldg(a.cell_start + c + 1) - start;
                }
            }
            hits += (int)cnt;
            uint32_t incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const uint32_t total = __shfl_sync(kFull, incl, 31);
            for (uint32_t hb = 0; hb < total; hb += 32) {
                const uint32_t j = hb + lane;
                const bool hv = j < total;
                int lo = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    uint32_t v = __shfl_sync(kFull, incl, lo + step - 1);
                    if (v <= j) lo += step;
                }
                const uint32_t o_incl = __shfl_sync(kFull, incl, lo);
                const uint32_t o_cnt = __shfl_sync(kFull, cnt, lo);
                const uint32_t o_start = __shfl_sync(kFull, start, lo);
                const int hs = s0 + lo;
                int hq = 0, d = 0;
                if (hv) {
                    hq = __ldg(a.entries + o_start + (j - (o_incl - o_cnt)));
                    d = (hq - hs) & a.diag_mask;
                }
                const unsigned vmask = __ballot_sync(kFull, hv);
                unsigned peers = 0;
                if (hv) peers = __match_any_sync(vmask, d);
                bool pending = hv, found = false;
                ExtOut r;
                for (;;) {
                    const unsigned pend = __ballot_sync(kFull, pending);
                    if (!pend) break;
                    if (pending && (peers & pend & lt) == 0) {
                        pending = false;
                        const uint32_t v = diag[d];
                        const int stamp = hs + base;
                        if (v & kFlag) {
                            if (stamp >= (int)(v & ~kFlag)) diag[d] = (uint32_t)stamp;
                        } else {
                            const int prev = (int)v - base;
                            const int diff = hs - prev;
                            if (diff >= a.window) {
                                diag[d] = (uint32_t)stamp;
                            } else if (diff >= BP_WORD) {
                                const int k = a.n_ctx == 1 ? 0 : context_of(a.ctx, a.n_ctx, hq);
                                r = extend_two_hit(m, sub, slen, qs, a.qlen, prev + BP_WORD, hs, hq,
                                                   __ldg(a.ctx + 3 * k + 1));
                                ++ext;
                                found = r.score >= __ldg(a.ctx + 3 * k + 2);
                                diag[d] = r.right_ext
                                              ? ((uint32_t)(r.s_last - (BP_WORD - 1) + base) | kFlag)
                                              : (uint32_t)stamp;
                            }
                        }
                    }
                    __syncwarp();
                }
                const unsigned fm = __ballot_sync(kFull, found);
                if (fm) {
                    uint32_t pos0 = 0;
                    if (lane == 0) pos0 = atomicAdd(a.rec_count, (uint32_t)__popc(fm));
                    pos0 = __shfl_sync(kFull, pos0, 0);
                    if (found) {
                        const uint32_t pos = pos0 + (uint32_t)__popc(fm & lt);
                        if (pos < a.rec_cap) {
                            HspRec rec;
                            rec.oid = oid;
                            rec.key = key_base + (int)j;
                            rec.h.hsp_q = r.hsp_q;
                            rec.h.hsp_s = r.hsp_s;
                            rec.h.query_offset = hq;
                            rec.h.subject_offset = hs;
                            rec.h.hsp_len = r.len;
                            rec.h.score = r.score;
                            a.recs[pos] = rec;
                        }
                    }
                    succ += __popc(fm);
                }
            }
            key_base += (int)total;
        }
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            hits += __shfl_xor_sync(kFull, hits, o);
            ext += __shfl_xor_sync(kFull, ext, o);
        }
        if (lane == 0) {
            a.counters[3 * (int64_t)oid + 0] = hits;
            a.counters[3 * (int64_t)oid + 1] = succ;
            a.counters[3 * (int64_t)oid + 2] = ext;
        }
        base += slen + a.window;
    }
}

template <int WARPS>
cudaError_t launch_scan_t(bp_engine* e, const ScanArgs& a) {
    const int L = a.diag_mask + 1;
    size_t smem = 1024 + 4096 + (size_t)((a.qlen + 15) & ~15) + (size_t)WARPS * L * 4;
    cudaError_t err = cudaFuncSetAttribute(scan_plain<WARPS>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (err != cudaSuccess) return err;
    int per_sm = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scan_plain<WARPS>, WARPS * 32, smem);
    if (err != cudaSuccess) return err;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    int grid = e->sm_count * per_sm;
    int need = (a.n + WARPS - 1) / WARPS;
    if (grid > need) grid = need > 0 ? need : 1;
    scan_plain<WARPS><<<grid, WARPS * 32, smem, e->stream>>>(a);
    e->launches += 1;
    return cudaGetLastError();
}

}  // namespace

cudaError_t bp_launch_scan(bp_engine* e, const ScanArgs& a) {
    const int L = a.diag_mask + 1;
    // Keep the per-CTA diagonal arrays within ~96 KB so two CTAs fit an SM.
    if (L <= 2048) return launch_scan_t<8>(e, a);
    if (L <= 8192) return launch_scan_t<2>(e, a);
    return launch_scan_t<1>(e, a);
}
