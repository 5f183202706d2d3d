// Scan kernels: one query against a range of subjects (scan_kernel), and many
// queries against one resident database (scan_batch_kernel).
//
// Semantics follow the reference kernel GPU_BLASTP_kernelTwoHit
// (gpu_blastp_kernel.cu:42-320) and its extenders (:341-549); the mapping to
// the hardware does not:
//  * one persistent CTA per SM with up to 32 warps; the query, the scoring
//    matrix and (when they fit) the compact neighbour-word table are loaded
//    into shared memory and shared by every warp;
//  * a warp owns one subject at a time.  In the plain kernel it takes
//    subjects from a global cursor through a three-stage software pipeline:
//    cursor grab (i+3), offsets load (i+2), cp.async.bulk L2 prefetch of the
//    residues (i+1), scan (i) -- so the database is streamed from HBM into L2
//    ahead of the warp that reads it;
//  * the warp reads 128 consecutive word positions (4 per lane, contiguous),
//    loading the next window's residues while it works on the current one,
//    looks the words up in the table and flattens the resulting word hits
//    into chunks of 32 -- one hit per lane, whatever the per-position hit
//    counts are;
//  * the per-diagonal two-hit state lives in shared memory, one array per
//    warp of L = Q + window entries (rounded up to 32, at least 128),
//    indexed by (q - s) mod L (the reference keeps a power-of-two array in
//    global memory, one per thread);
//  * hits of one chunk on the same diagonal are applied in word-position
//    order (__match_any_sync), the only order the state machine depends on;
//    distinct diagonals are independent;
//  * for queries of 150 letters and more, a hit pair that calls for an
//    extension does not stop the warp: it becomes a task and its diagonal is
//    marked pending; later hits on a pending diagonal wait, in order, in a
//    blocked list.  When the queue fills, or the subject ends, the warp walks
//    the queued extensions -- one lane per extension when there are enough
//    of them, the whole warp per extension otherwise -- writes their outcomes
//    into the diagonal states and replays the blocked hits.  Every diagonal
//    therefore sees exactly the reference's sequence of events; only the
//    interleaving of independent diagonals changes.  Shorter queries extend
//    each pair at once, the whole warp walking 32 letters per step;
//  * surviving HSPs are compacted with a warp ballot into one global append
//    buffer, tagged with the subject and the hit's index in the subject's hit
//    stream, from which the ordering pass restores the discovery order.
#include "bp_internal.h"

extern __shared__ __align__(128) uint8_t bp_smem[];

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kP = 4;                       // word positions per lane per window
// Per-lane position table row: kP hit counts and kP cell starts, padded to an
// odd number of words so that the 32 lanes' rows start in 32 different banks
// (rows read by the hit flattening, by owner lane, stay conflict-free too).
constexpr int kRow = 2 * kP + 1;
constexpr int kMaxWarps = 32;
constexpr int kTaskCap = 64;                // queued extensions per warp
constexpr int kBlkCap = 64;                 // hits waiting behind queued extensions, per warp
constexpr int kLaneWalkMin = 2;             // from this many queued extensions on, one lane walks each
// Queries at least this long queue their extensions (kDefer); shorter ones
// have too few extensions per subject for one-lane-per-extension walks to pay
// for the queue, and extend each pair at once with the whole warp (with the
// score profile and rounds by rank, 160 aa: 3.65 -> 3.51 ms per 1M subjects
// queued; 130 aa gains nothing).
constexpr int kDeferMinQlen = 150;
constexpr int kMaxMembers = 32;             // queries per packed table (BP_MAX_PACK_MEMBERS)
// Diagonal arrays of at most this many entries use 16-bit entries.
constexpr int kNarrowMaxL = 8192;

// One diagonal entry: a stamp (position + the warp's running offset) and two
// flags -- an extension reached past this point, or an extension waits in
// the task queue.  Stamps stay below kMax: the offset is rebased when the
// next window could produce a larger one.  16-bit entries halve the per-warp
// arrays, so long queries keep more warps (and their tables) on chip.
template <typename DiagT>
struct DiagBits;
template <>
struct DiagBits<uint32_t> {
    static constexpr uint32_t kFlag = 0x80000000u, kPend = 0x40000000u, kStamp = 0x3fffffffu;
    static constexpr int kMax = 1 << 30;
};
template <>
struct DiagBits<uint16_t> {
    static constexpr uint32_t kFlag = 0x8000u, kPend = 0x4000u, kStamp = 0x3fffu;
    static constexpr int kMax = 1 << 14;
};

}  // namespace

// Shared-memory layout of one launch (host computes, kernel reads).
struct ScanLayout {
    int warps;
    int cells_mode;        // 0: u16 starts in smem, 1: u32 starts in smem, 2: u32 starts in global
    int entries_smem;
    int L;                 // diagonal entries per warp (the longest query's)
    int off_cells, off_entries, off_query, off_members, off_mof, off_warps, off_ctl;
    int off_stream;        // plain and streaming launches: per-warp subject pipeline
    int off_prof;          // query score profile (0: none): row q holds m[query[q]][0..31]
    int warp_bytes;        // diagonal array + per-lane position table + task queue + blocked list
                           // (+ per-member counters when packed)
    int total;
};

namespace {

// A queued extension (diff = hs - previous hit on the diagonal) or a blocked
// hit (diff = 0).
struct Task {
    int hs, key, d;
    uint32_t hqx;          // query offset | diff << 16
};

struct ExtOut {
    int hsp_q, hsp_s, len, score, s_last, right_ext;
};

__device__ __forceinline__ int msc(const int8_t* m, int a, int b) { return m[a * BP_MROW + b]; }

// The score of query offset q against subject letter s: from the matrix and
// the query, or (kProf) from the query's score profile, row q.
template <bool kProf>
__device__ __forceinline__ int qscore(const int8_t* m, const uint8_t* qry, int q, int s) {
    return kProf ? m[q * BP_MROW + s] : msc(m, qry[q], s);
}

__device__ __forceinline__ int warp_incl_sum(int x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

__device__ __forceinline__ int warp_incl_max(int x, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x = max(x, y);
    }
    return x;
}

// One X-drop walk, 32 letters per iteration.  Letter i (i = 0..n-1) scores
// m[q(i)][s(i)] with q(i) = qry[q0 + dir*i], s(i) = subj[s0 + dir*i].  The
// running score starts at `start`, the best at `start`; the walk stops after
// the first letter where best - run >= xdrop (or, when walking right,
// run <= 0).  Returns the best score, the index of the letter that first
// reached it (-1 if none), and the index of the stopping letter (n if the
// walk ran out of letters).  All lanes return the same values.  kProf: m is
// the query's score profile.
template <bool kRight, bool kProf>
__device__ __forceinline__ void warp_xdrop(const int8_t* m, const uint8_t* __restrict__ subj, const uint8_t* qry,
                                           int s0, int q0, int n, int start, int xdrop, int lane, int& best,
                                           int& best_i, int& stop_i) {
    int carry = start;
    best = start;
    best_i = -1;
    stop_i = n;
    for (int i0 = 0; i0 < n; i0 += 32) {
        const int i = i0 + lane;
        const bool valid = i < n;
        int v = 0;
        if (valid) {
            if (kProf)
                v = kRight ? m[(q0 + i) * BP_MROW + __ldg(subj + s0 + i)]
                           : m[(q0 - i) * BP_MROW + __ldg(subj + s0 - i)];
            else
                v = kRight ? msc(m, qry[q0 + i], __ldg(subj + s0 + i)) : msc(m, qry[q0 - i], __ldg(subj + s0 - i));
        }
        const int run = carry + warp_incl_sum(v, lane);
        const int pm = max(best, warp_incl_max(run, lane));
        const bool stop = valid && ((pm - run >= xdrop) || (kRight && run <= 0));
        const unsigned sb = __ballot_sync(kFull, stop);
        const int last = sb ? (__ffs(sb) - 1) : min(31, n - 1 - i0);
        const int nb = __shfl_sync(kFull, pm, last);
        if (nb > best) {
            const unsigned at = __ballot_sync(kFull, valid && lane <= last && run == nb);
            best_i = i0 + __ffs(at) - 1;
            best = nb;
        }
        carry = __shfl_sync(kFull, run, last);
        if (sb) {
            stop_i = i0 + last;
            break;
        }
    }
}

// The same walk by one lane, with the outcome of the reference's
// letter-by-letter loops (gpu_blastp_kernel.cu:435-481, :503-549): residues
// are fetched four letters at a time so the loads overlap the dependent score
// chain, a group of four is tested for a stop once (the running scores and
// bests of its letters are all known), and only a group that stops, or the
// last partial one, is resolved letter by letter.  kProf: m is the query's
// score profile, stepped one row per letter.
template <bool kRight, bool kProf>
__device__ __forceinline__ void lane_xdrop(const int8_t* m, const uint8_t* __restrict__ subj, const uint8_t* qry,
                                           int s0, int q0, int n, int start, int xdrop, int& best, int& best_i,
                                           int& stop_i) {
    constexpr int D = kRight ? 1 : -1;
    const uint8_t* qp = qry + q0;
    const int8_t* pp = m + (kProf ? q0 * BP_MROW : 0);
    const uint8_t* sp = subj + s0;
    int run = start;
    best = start;
    best_i = -1;
    stop_i = n;
    int i0 = 0;
    for (; i0 + 4 <= n; i0 += 4) {
        int sc[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            sc[k] = kProf ? pp[D * (i0 + k) * BP_MROW + __ldg(sp + D * (i0 + k))]
                          : msc(m, qp[D * (i0 + k)], __ldg(sp + D * (i0 + k)));
        // the group's running scores and bests; one test for a stop anywhere in it
        const int r0 = run + sc[0], r1 = r0 + sc[1], r2 = r1 + sc[2], r3 = r2 + sc[3];
        const int b0 = max(best, r0), b1 = max(b0, r1), b2 = max(b1, r2), b3 = max(b2, r3);
        bool t0 = b0 - r0 >= xdrop, t1 = b1 - r1 >= xdrop, t2 = b2 - r2 >= xdrop, t3 = b3 - r3 >= xdrop;
        if (kRight) {
            t0 |= r0 <= 0;
            t1 |= r1 <= 0;
            t2 |= r2 <= 0;
            t3 |= r3 <= 0;
        }
        if (t0 | t1 | t2 | t3) {
            // the first stopping letter k, with the best (and where it was
            // first reached) as of that letter
            const int k = t0 ? 0 : t1 ? 1 : t2 ? 2 : 3;
            if (r0 > best) {
                best = r0;
                best_i = i0;
            }
            if (k >= 1 && r1 > best) {
                best = r1;
                best_i = i0 + 1;
            }
            if (k >= 2 && r2 > best) {
                best = r2;
                best_i = i0 + 2;
            }
            if (k >= 3 && r3 > best) {
                best = r3;
                best_i = i0 + 3;
            }
            stop_i = i0 + k;
            return;
        }
        // no stop: the group's best was first reached at the first letter equal to it
        if (b3 > best) best_i = i0 + (r0 == b3 ? 0 : r1 == b3 ? 1 : r2 == b3 ? 2 : 3);
        best = b3;
        run = r3;
    }
    for (; i0 < n; ++i0) {
        run += kProf ? pp[D * i0 * BP_MROW + __ldg(sp + D * i0)] : msc(m, qp[D * i0], __ldg(sp + D * i0));
        if (run > best) {
            best = run;
            best_i = i0;
        }
        if (best - run >= xdrop || (kRight && run <= 0)) {
            stop_i = i0;
            return;
        }
    }
}

// s_BlastAaExtendTwoHit (gpu_blastp_kernel.cu:341-415): the word-start shift,
// the left walk, which must reach s_left for the right walk to run, and the
// right walk starting from the left score.  The walks stay within query
// offsets [q_lo, q_hi): the whole query, or one query of a packed table.  kWarp: every lane passes the
// same arguments, the walks use the whole warp and every lane gets the
// result; otherwise each lane extends its own hit pair.  kProf: every score
// comes from the query's score profile, which the layout places right after
// the query (at the next 16-byte boundary; plain and streaming launches, one
// query, so q_hi is its length).
template <bool kWarp, bool kProf = false>
__device__ __forceinline__ ExtOut extend_two_hit(const int8_t* m, const uint8_t* __restrict__ subj, int slen,
                                                 const uint8_t* qry, int q_lo, int q_hi, int s_left, int s_right,
                                                 int q_right, int xdrop, int lane) {
    if (kProf) m = reinterpret_cast<const int8_t*>(qry) + ((q_hi + 15) & ~15);
    int score = 0, left_score = 0, shift = 0;
#pragma unroll
    for (int i = 0; i < BP_WORD; ++i) {
        score += qscore<kProf>(m, qry, q_right + i, __ldg(subj + s_right + i));
        if (score > left_score) {
            left_score = score;
            shift = i + 1;
        }
    }
    q_right += shift;
    s_right += shift;

    int lbest, lbest_k, lstop;
    const int nl = min(s_right, q_right - q_lo);
    if (kWarp)
        warp_xdrop<false, kProf>(m, subj, qry, s_right - 1, q_right - 1, nl, 0, xdrop, lane, lbest, lbest_k, lstop);
    else
        lane_xdrop<false, kProf>(m, subj, qry, s_right - 1, q_right - 1, nl, 0, xdrop, lbest, lbest_k, lstop);
    const int left_d = lbest_k + 1;
    left_score = lbest;

    ExtOut o;
    o.right_ext = 0;
    o.s_last = s_right;
    int right_d = 0, right_score = 0;
    if (left_d >= s_right - s_left) {
        o.right_ext = 1;
        const int nr = min(slen - s_right, q_hi - q_right);
        int rbest, rbest_i, rstop;
        if (kWarp)
            warp_xdrop<true, kProf>(m, subj, qry, s_right, q_right, nr, left_score, xdrop, lane, rbest, rbest_i,
                                    rstop);
        else lane_xdrop<true, kProf>(m, subj, qry, s_right, q_right, nr, left_score, xdrop, rbest, rbest_i, rstop);
        right_d = rbest_i + 1;
        right_score = rbest;
        o.s_last = s_right + rstop;
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
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(ctx + 3 * mid) <= q) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Prefetches the residues [s, e) of a subject into L2 in whole 16-byte
// blocks, none of which reaches past db_bytes (a partial last block is left
// to the warp's own loads).
__device__ __forceinline__ void prefetch_span(const uint8_t* db, long long db_bytes, long long s, long long e) {
    const long long lo = s & ~15LL;
    const long long hi = min((e + 15) & ~15LL, db_bytes & ~15LL);
    if (hi > lo) prefetch_l2(db + lo, (uint32_t)(hi - lo));
}

// Residues r..r+kP+1 of the window starting at `sl` (code-1, or -1 past the
// end).  kCheck: codes of 28 and more (r > 26) are noted in `bad`; every
// residue of a subject passes through some lane's window.
template <bool kCheck = false>
__device__ __forceinline__ void load_window(const uint8_t* __restrict__ sub, int slen, int sl, int (&r)[kP + 2],
                                            uint32_t& bad) {
#pragma unroll
    for (int i = 0; i < kP + 2; ++i) {
        r[i] = (sl + i < slen) ? (int)__ldg(sub + sl + i) - 1 : -1;
        if (kCheck) bad |= r[i] > BP_ALPHABET - 2 ? 1u : 0u;
    }
}

// One warp's view of the subject it is scanning.
// kProf: the launch's layout holds the query's score profile (plain and
// streaming launches only).
template <typename DiagT, bool kProf = false>
struct WarpScan {
    const ScanArgs* a;
    const int8_t* m;
    const uint8_t* qs;
    DiagT* diag;
    Task* tasks;
    Task* blocked;
    const uint8_t* sub;
    int slen, oid, base, lane;   // oid: the subject's segment (packed: its index in the batch's range)
    unsigned lt;
    int nt, nb;            // queued tasks and blocked hits (warp-uniform)
    int ext, succ;         // this lane's share of the subject's counters
    int* wcnt;             // packed: per-member hits, successes, extensions (shared memory)
};

// The query an offset belongs to: its bounds, x-drop and cutoff.  Packed
// tables look the member up in the offset-to-member table; otherwise the
// context is the last one starting at or before the offset.
struct Member {
    int k, q_lo, q_hi, xdrop, cutoff;
};

template <bool kPacked, class W>
__device__ __forceinline__ Member member_at(const W& w, int hq) {
    const ScanArgs& a = *w.a;
    Member r;
    if (kPacked) {
        r.k = a.member_of[hq];
        const int32_t* mm = a.members + 5 * r.k;
        r.q_lo = mm[1];
        r.q_hi = mm[1] + mm[2];
        r.xdrop = mm[3];
        r.cutoff = mm[4];
    } else {
        r.k = a.n_ctx == 1 ? 0 : context_of(a.ctx, a.n_ctx, hq);
        r.q_lo = 0;
        r.q_hi = a.qlen;
        r.xdrop = __ldg(a.ctx + 3 * r.k + 1);
        r.cutoff = __ldg(a.ctx + 3 * r.k + 2);
    }
    return r;
}

// Appends the reported HSPs of this round (one candidate per lane).  Packed:
// the record goes to its query's segment, with query offsets relative to it.
template <bool kPacked, class W>
__device__ __forceinline__ void emit(W& w, bool found, int key, int hs, int hq, const ExtOut& x) {
    const unsigned fm = __ballot_sync(kFull, found);
    if (!fm) return;
    uint32_t pos0 = 0;
    if (w.lane == 0) pos0 = atomicAdd(w.a->rec_count, (uint32_t)__popc(fm));
    pos0 = __shfl_sync(kFull, pos0, 0);
    if (found) {
        int seg = w.oid, q0 = 0;
        if (kPacked) {
            const int k = w.a->member_of[hq];
            seg = w.a->members[5 * k] * w.a->seg_stride + w.oid;
            q0 = w.a->members[5 * k + 1];
            atomicAdd(&w.wcnt[3 * k + 1], 1);
        } else {
            ++w.succ;
        }
        const uint32_t pos = pos0 + (uint32_t)__popc(fm & w.lt);
        if (pos < w.a->rec_cap) {
            HspRec rec;
            rec.oid = seg;
            rec.key = key;
            rec.h.hsp_q = x.hsp_q - q0;
            rec.h.hsp_s = x.hsp_s;
            rec.h.query_offset = hq - q0;
            rec.h.subject_offset = hs;
            rec.h.hsp_len = x.len;
            rec.h.score = x.score;
            w.a->recs[pos] = rec;
        }
    }
}

// The diagonal's entry after an extension of the pair ending at hs: past the
// right walk's last letter when it ran, else the hit itself.
template <typename DiagT>
__device__ __forceinline__ DiagT diag_after(const ExtOut& x, int hs, int base) {
    return (DiagT)(x.right_ext ? ((uint32_t)(x.s_last - (BP_WORD - 1) + base) | DiagBits<DiagT>::kFlag)
                               : (uint32_t)(hs + base));
}

// Applies up to 32 hits (one per lane, in hit-stream order by lane) to the
// diagonal states.  Hits on the same diagonal go one per round in lane order.
// kDefer: a pair within the window becomes a task and marks its diagonal
// pending, and a hit on a pending diagonal joins the blocked list (needs room
// for 32 more tasks and 32 more blocked hits).  Otherwise each pair is
// extended at once by the whole warp, one after the other.
template <bool kDefer, bool kPacked, typename DiagT, bool kProf>
__device__ __forceinline__ void apply_hits(WarpScan<DiagT, kProf>& w, bool hv, int hs, int hq, int d, int key,
                                           bool count) {
    using B = DiagBits<DiagT>;
    const unsigned vmask = __ballot_sync(kFull, hv);
    if (!vmask) return;
    if (kPacked && count && hv) atomicAdd(&w.wcnt[3 * w.a->member_of[hq]], 1);   // word hits per query
    unsigned peers = 0;
    if (hv) peers = __match_any_sync(vmask, d);
    // a hit goes in the round of its rank among the chunk's hits on its
    // diagonal (the lanes before it with the same d), so every diagonal sees
    // its hits in lane order and one round holds one hit per diagonal
    // (packed tables keep asking each round which hits are still pending:
    // there the rank's registers cost the kernel more than the ballots)
    const int rank = (!kPacked && hv) ? __popc(peers & w.lt) : -1;
    const int rounds = kPacked ? 0 : (int)__reduce_max_sync(kFull, (unsigned)(rank + 1));
    bool pending = kPacked && hv, found = false;
    ExtOut res{0, 0, 0, 0, 0, 0};
    const int window = w.a->window;
    for (int round = 0;; ++round) {
        bool go;
        if (kPacked) {
            const unsigned pend = __ballot_sync(kFull, pending);
            if (!pend) break;
            go = pending && (peers & pend & w.lt) == 0;
            if (go) pending = false;
        } else {
            if (round >= rounds) break;
            go = rank == round;
        }
        bool need = false, blk = false;
        int diff = 0;
        if (go) {
            const uint32_t v = w.diag[d];
            const int stamp = hs + w.base;
            if (kDefer && (v & B::kPend)) {
                blk = true;
            } else if (v & B::kFlag) {
                // an extension already covered this hit; the first hit past it restarts the diagonal
                if (stamp >= (int)(v & B::kStamp)) w.diag[d] = (DiagT)stamp;
            } else {
                diff = hs - ((int)v - w.base);
                if (diff >= window) w.diag[d] = (DiagT)stamp;
                else if (diff >= BP_WORD) need = true;
            }
        }
        if (kDefer) {
            const unsigned bm = __ballot_sync(kFull, blk);
            if (blk) w.blocked[w.nb + __popc(bm & w.lt)] = Task{hs, key, d, (uint32_t)hq};
            w.nb += __popc(bm);
            const unsigned nm = __ballot_sync(kFull, need);
            if (need) {
                w.tasks[w.nt + __popc(nm & w.lt)] = Task{hs, key, d, (uint32_t)hq | ((uint32_t)diff << 16)};
                w.diag[d] = (DiagT)(B::kPend | (uint32_t)(hs + w.base));
                if (kPacked) atomicAdd(&w.wcnt[3 * w.a->member_of[hq] + 2], 1);
                else ++w.ext;
            }
            w.nt += __popc(nm);
        } else {
            // this round's extensions, one after the other, each by the whole warp
            unsigned E = __ballot_sync(kFull, need);
            while (E) {
                const int leader = __ffs(E) - 1;
                E &= E - 1;
                const int e_s = __shfl_sync(kFull, hs, leader);
                const int e_q = __shfl_sync(kFull, hq, leader);
                const int e_diff = __shfl_sync(kFull, diff, leader);
                const Member mb = member_at<kPacked>(w, e_q);
                const ExtOut x = extend_two_hit<true>(w.m, w.sub, w.slen, w.qs, mb.q_lo, mb.q_hi,
                                                      e_s - e_diff + BP_WORD, e_s, e_q, mb.xdrop, w.lane);
                if (w.lane == leader) {
                    res = x;
                    if (kPacked) atomicAdd(&w.wcnt[3 * mb.k + 2], 1);
                    else ++w.ext;
                    found = x.score >= mb.cutoff;
                    w.diag[d] = diag_after<DiagT>(x, hs, w.base);
                }
            }
            __syncwarp();
        }
    }
    if (!kDefer) emit<kPacked>(w, found, key, hs, hq, res);
}

// Walks every queued extension and writes its outcome into its diagonal.
template <bool kPacked, typename DiagT, bool kProf>
__device__ void flush_tasks(WarpScan<DiagT, kProf>& w) {
    const int nt = w.nt;
    if (nt >= kLaneWalkMin) {
        for (int t0 = 0; t0 < nt; t0 += 32) {
            const int t = t0 + w.lane;
            bool found = false;
            Task tk{0, 0, 0, 0};
            ExtOut x{0, 0, 0, 0, 0, 0};
            if (t < nt) {
                tk = w.tasks[t];
                const int hq = (int)(tk.hqx & 0xffffu), diff = (int)(tk.hqx >> 16);
                const Member mb = member_at<kPacked>(w, hq);
                if (kProf)
                    x = extend_two_hit<false, true>(w.m, w.sub, w.slen, w.qs, mb.q_lo, mb.q_hi, tk.hs - diff + BP_WORD,
                                                    tk.hs, hq, mb.xdrop, w.lane);
                else
                    x = extend_two_hit<false>(w.m, w.sub, w.slen, w.qs, mb.q_lo, mb.q_hi, tk.hs - diff + BP_WORD,
                                              tk.hs, hq, mb.xdrop, w.lane);
                found = x.score >= mb.cutoff;
                w.diag[tk.d] = diag_after<DiagT>(x, tk.hs, w.base);
            }
            emit<kPacked>(w, found, tk.key, tk.hs, (int)(tk.hqx & 0xffffu), x);
        }
    } else {
        for (int t = 0; t < nt; ++t) {
            const Task tk = w.tasks[t];
            const int hq = (int)(tk.hqx & 0xffffu), diff = (int)(tk.hqx >> 16);
            const Member mb = member_at<kPacked>(w, hq);
            const ExtOut x =
                kProf
                    ? extend_two_hit<true, true>(w.m, w.sub, w.slen, w.qs, mb.q_lo, mb.q_hi, tk.hs - diff + BP_WORD,
                                                 tk.hs, hq, mb.xdrop, w.lane)
                    : extend_two_hit<true>(w.m, w.sub, w.slen, w.qs, mb.q_lo, mb.q_hi, tk.hs - diff + BP_WORD, tk.hs,
                                           hq, mb.xdrop, w.lane);
            const bool found = w.lane == 0 && x.score >= mb.cutoff;
            if (w.lane == 0) w.diag[tk.d] = diag_after<DiagT>(x, tk.hs, w.base);
            emit<kPacked>(w, found, tk.key, tk.hs, hq, x);
        }
    }
    __syncwarp();
    w.nt = 0;
}

// Resolves the queued extensions, then replays the blocked hits once, in
// order.  A replayed hit may queue a new extension (and block the hits after
// it on its diagonal again); the blocked list is rewritten in place.
template <bool kPacked, typename DiagT, bool kProf>
__device__ void resolve(WarpScan<DiagT, kProf>& w) {
    flush_tasks<kPacked>(w);
    const int n = w.nb;
    w.nb = 0;
    for (int r = 0; r < n; r += 32) {
        const int i = r + w.lane;
        const bool hv = i < n;
        Task b{0, 0, 0, 0};
        if (hv) b = w.blocked[i];
        __syncwarp();
        apply_hits<true, kPacked>(w, hv, b.hs, (int)(b.hqx & 0xffffu), b.d, b.key, false);
    }
    __syncwarp();
}

// Scans one subject.  oid: the subject's counter/record segment; packed: its
// index in the batch's subject range (each query's segment is derived).
// Moves the stamp offset so that position s0 gets stamp `window`: every entry
// moves down by delta = base + s0 - window with its flag, and an entry that
// would go below zero -- a hit or an extension end more than `window` before
// s0 -- becomes 0, which every later hit reads the same way (a diagonal whose
// last event is out of reach).  Nothing may be pending.  All n entries are
// swept, the batched kernel's longer arrays included, so no older stamp can
// look recent after the move.
template <typename DiagT>
__device__ __forceinline__ void rebase_diag(DiagT* diag, int n, int delta, int lane) {
    using B = DiagBits<DiagT>;
    for (int i = lane; i < n; i += 32) {
        const uint32_t v = diag[i];
        const int st = (int)(v & B::kStamp);
        diag[i] = st >= delta ? (DiagT)((uint32_t)(st - delta) | (v & B::kFlag)) : (DiagT)0;
    }
    __syncwarp();
}

// Scans one subject.  The stamps written while a window starting at s0 is
// processed (hits, pending marks, extension ends) are at most
// base + s0 + 128 + qlen (a hit lies before s0 + 128 and a right walk ends
// within qlen letters of it), so the offset is reset when that bound could
// reach DiagBits::kMax.  clear_len: entries of the warp's whole array.
template <typename CellT, bool kDefer, bool kPacked, typename DiagT, bool kCheck = false, bool kProf = false>
__device__ void scan_subject(const ScanArgs& a, const int8_t* m, const uint8_t* qs, const CellT* cells,
                             const uint16_t* entries, DiagT* diag, int clear_len, uint32_t* lane_pos, Task* tasks,
                             Task* blocked, int* wcnt, int oid, const uint8_t* __restrict__ sub, int slen, int& base,
                             int lane) {
    using B = DiagBits<DiagT>;
    const int L = a.diag_len;
    if (base + a.qlen + 129 >= B::kMax) {
        // every entry is older than this subject: start the offset again
        for (int i = lane; i < clear_len; i += 32) diag[i] = 0;
        __syncwarp();
        base = a.window;
    }
    WarpScan<DiagT, kProf> w;
    w.a = &a;
    w.m = m;
    w.qs = qs;
    w.diag = diag;
    w.tasks = tasks;
    w.blocked = blocked;
    w.sub = sub;
    w.slen = slen;
    w.oid = oid;
    w.base = base;
    w.lane = lane;
    w.lt = (1u << lane) - 1u;
    w.nt = w.nb = 0;
    w.ext = w.succ = 0;
    w.wcnt = wcnt;
    if (kPacked) {
        for (int i = lane; i < 3 * a.n_members; i += 32) wcnt[i] = 0;
        __syncwarp();
    }
    int hits = 0, key_base = 0;
    int s0m = 0;                         // s0 mod L
    const int last_pos = slen - BP_WORD;
    const uint32_t* my_row = lane_pos - lane * kRow;
    int r[kP + 2];
    uint32_t bad = 0;
    load_window<kCheck>(sub, slen, lane * kP, r, bad);
    for (int s0 = 0; s0 <= last_pos; s0 += 32 * kP) {
        if (base + s0 + 129 + a.qlen >= B::kMax) {
            // long subject: settle every queued extension, then move the offset
            if (kDefer)
                while (w.nt > 0 || w.nb > 0) resolve<kPacked>(w);
            rebase_diag(diag, clear_len, base + s0 - a.window, lane);
            base = a.window - s0;
            w.base = base;
        }
        int rn[kP + 2];
        load_window<kCheck>(sub, slen, s0 + 32 * kP + lane * kP, rn, bad);   // next window, in flight meanwhile
        const int sl = s0 + lane * kP;
        uint32_t lane_cnt = 0;
#pragma unroll
        for (int p = 0; p < kP; ++p) {
            uint32_t start = 0, cnt = 0;
            if (sl + p <= last_pos && (unsigned)r[p] < 27u && (unsigned)r[p + 1] < 27u && (unsigned)r[p + 2] < 27u) {
                const int c = r[p] * 729 + r[p + 1] * 27 + r[p + 2];
                start = cells[c];
                cnt = (uint32_t)cells[c + 1] - start;
            }
            lane_pos[p] = lane_cnt;        // hits of this lane before position p
            lane_pos[kP + p] = start;
            lane_cnt += cnt;
        }
        hits += (int)lane_cnt;
        const uint32_t incl = (uint32_t)warp_incl_sum((int)lane_cnt, lane);
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        __syncwarp();
        for (uint32_t hb = 0; hb < total; hb += 32) {
            if (kDefer)
                while (w.nt > kTaskCap - 32 || w.nb > kBlkCap - 32) resolve<kPacked>(w);
            const uint32_t j = hb + lane;
            const bool hv = j < total;
            // owner lane: first lane whose inclusive prefix exceeds j
            int lo = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const uint32_t v = __shfl_sync(kFull, incl, lo + step - 1);
                if (v <= j) lo += step;
            }
            const uint32_t o_incl = __shfl_sync(kFull, incl, lo);
            const uint32_t o_cnt = __shfl_sync(kFull, lane_cnt, lo);
            int hs = 0, hq = 0, d = 0;
            if (hv) {
                const uint32_t local = j - (o_incl - o_cnt);
                const uint32_t* op = my_row + lo * kRow;
                int p = 0;
#pragma unroll
                for (int t = 1; t < kP; ++t)
                    if (op[t] <= local) p = t;
                hs = s0 + lo * kP + p;
                hq = entries[op[kP + p] + (local - op[p])];
                // (hq - hs) mod L, from s0 mod L: lo*kP + p < 128 <= L
                int hm = s0m + lo * kP + p;
                if (hm >= L) hm -= L;
                d = hq - hm;
                if (d < 0) d += L;
            }
            apply_hits<kDefer, kPacked>(w, hv, hs, hq, d, key_base + (int)j, true);
        }
        key_base += (int)total;
        s0m += 32 * kP;
        if (s0m >= L) s0m -= L;
        __syncwarp();
#pragma unroll
        for (int i = 0; i < kP + 2; ++i) r[i] = rn[i];
    }
    if (kDefer)
        while (w.nt > 0 || w.nb > 0) resolve<kPacked>(w);
    if (kPacked) {
        // every query of the packed table gets its own counters for this subject
        __syncwarp();
        for (int k = lane; k < a.n_members; k += 32) {
            const int64_t seg = (int64_t)a.members[5 * k] * a.seg_stride + oid;
            a.counters[3 * seg + 0] = wcnt[3 * k + 0];
            a.counters[3 * seg + 1] = wcnt[3 * k + 1];
            a.counters[3 * seg + 2] = wcnt[3 * k + 2];
        }
        __syncwarp();
        base += slen + a.window;
        return;
    }
    if (kCheck && __any_sync(kFull, bad != 0) && lane == 0) atomicOr(a.error, 1u);
    int ext = w.ext, succ = w.succ;
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        hits += __shfl_xor_sync(kFull, hits, o);
        ext += __shfl_xor_sync(kFull, ext, o);
        succ += __shfl_xor_sync(kFull, succ, o);
    }
    if (lane == 0) {
        a.counters[3 * (int64_t)oid + 0] = hits;
        a.counters[3 * (int64_t)oid + 1] = succ;
        a.counters[3 * (int64_t)oid + 2] = ext;
    }
    base += slen + a.window;
}

// Longest first (see ScanArgs::long_ids): cursor slot s < n_long is the
// range's s-th long subject, slot n_long + i is subject i of the range,
// skipped there when it is long (it was scanned in the first pass).
constexpr uint32_t kSecond = 0x80000000u;   // a second-pass slot
constexpr uint32_t kNone = 0x7fffffffu;     // past the last slot

__device__ __forceinline__ uint32_t slot_subject(const ScanArgs& a, int n_long, uint32_t slot) {
    if (slot < (uint32_t)n_long) return (uint32_t)(__ldg(a.long_ids + slot) - a.first);
    slot -= (uint32_t)n_long;
    return slot < (uint32_t)a.n ? (slot | kSecond) : kNone;
}

__device__ __forceinline__ bool in_range(const ScanArgs& a, uint32_t id) { return (id & ~kSecond) < (uint32_t)a.n; }

// A second-pass slot of a subject the first pass scanned.
__device__ __forceinline__ bool done_first(const ScanArgs& a, int n_long, uint32_t id, long long len) {
    return (id & kSecond) && n_long > 0 && len >= a.long_min;
}

// Per-warp regions: diagonal array, lane position table, task queue, blocked
// list, and (packed layouts) per-member counters.
template <typename DiagT>
struct WarpRegions {
    DiagT* diag;
    uint32_t* lane_pos;
    Task* tasks;
    Task* blocked;
    int* wcnt;
};

template <typename DiagT>
__device__ __forceinline__ WarpRegions<DiagT> warp_regions(const ScanLayout& lay, int warp, int lane) {
    uint8_t* wr = bp_smem + lay.off_warps + (size_t)warp * lay.warp_bytes;
    const size_t db = (size_t)lay.L * sizeof(DiagT);     // L is a multiple of 32: 16-byte aligned
    WarpRegions<DiagT> r;
    r.diag = reinterpret_cast<DiagT*>(wr);
    r.lane_pos = reinterpret_cast<uint32_t*>(wr + db) + lane * kRow;
    r.tasks = reinterpret_cast<Task*>(wr + db + 32 * kRow * 4);
    r.blocked = r.tasks + kTaskCap;
    r.wcnt = reinterpret_cast<int*>(r.blocked + kBlkCap);
    return r;
}

// The scoring matrix, the query and (when they fit) the compact table, into
// shared memory for every warp of the CTA (callers synchronise after).
template <typename CellT, bool kCellsSmem>
__device__ __forceinline__ void load_tables(const ScanArgs& a, const ScanLayout& lay, const int8_t*& m,
                                            const uint8_t*& qs, const CellT*& cells, const uint16_t*& entries) {
    uint8_t* sm = bp_smem;
    int8_t* mm = reinterpret_cast<int8_t*>(sm);
    uint8_t* q = sm + lay.off_query;
    for (int i = threadIdx.x; i < 28 * BP_MROW; i += blockDim.x) mm[i] = a.matrix[i];
    if (kCellsSmem) {
        CellT* c = reinterpret_cast<CellT*>(sm + lay.off_cells);
        for (int i = threadIdx.x; i <= BP_NC; i += blockDim.x) c[i] = (CellT)a.cells[i];
    }
    if (lay.entries_smem) {
        uint16_t* e = reinterpret_cast<uint16_t*>(sm + lay.off_entries);
        for (int i = threadIdx.x; i < a.n_entries; i += blockDim.x) e[i] = a.entries[i];
    }
    for (int i = threadIdx.x; i < a.qlen; i += blockDim.x) q[i] = a.query[i];
    if (lay.off_prof) {
        int8_t* pf = reinterpret_cast<int8_t*>(sm + lay.off_prof);
        for (int i = threadIdx.x; i < a.qlen * BP_MROW; i += blockDim.x)
            pf[i] = a.matrix[(int)__ldg(a.query + i / BP_MROW) * BP_MROW + i % BP_MROW];
    }
    m = mm;
    qs = q;
    cells = kCellsSmem ? reinterpret_cast<const CellT*>(sm + lay.off_cells) : reinterpret_cast<const CellT*>(a.cells);
    entries = lay.entries_smem ? reinterpret_cast<const uint16_t*>(sm + lay.off_entries) : a.entries;
}

// Lane 0's subject pipeline (shared memory, one per warp, plain and
// streaming launches): a ring of three subjects -- the one being scanned,
// the next (span known, residues prefetched), the one after (id known) -- so
// that little lives in registers across the scan of a subject (in registers
// this state made the scan spill).
struct StreamSubj {
    long long s, e;        // device span of the residues
    uint32_t id;           // subject of the range (>= n: none)
    int c;                 // chunk
    int ok;                // offsets inside the chunk
    int pad;
};
struct StreamCtl {
    StreamSubj q[3];
    int hint, ready;       // chunk hint of locate(); highest chunk known to be there
};

template <typename CellT, bool kCellsSmem, bool kDefer, typename DiagT, bool kProf>
__global__ void __launch_bounds__(kMaxWarps * 32, 1)
scan_kernel(ScanArgs a, ScanLayout lay) {
    // an earlier check on the device refused the inputs: nothing to scan
    if (a.abort_if && *a.abort_if) return;
    const int n_long = a.n_long_at ? *a.n_long_at : a.n_long;
    const int8_t* m;
    const uint8_t* qs;
    const CellT* cells;
    const uint16_t* entries;
    load_tables<CellT, kCellsSmem>(a, lay, m, qs, cells, entries);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpRegions<DiagT> wr = warp_regions<DiagT>(lay, warp, lane);
    for (int i = lane; i < lay.L; i += 32) wr.diag[i] = 0;
    __syncthreads();

    // Subject pipeline, kept by lane 0 in a per-warp ring in shared memory:
    // the subject being scanned, the next (offsets known, residues
    // prefetched into L2), the one after (id known, offsets loaded this
    // round); a new id is taken from the cursor after each scan.
    // slot_subject: subject index in the range, kSecond on second-pass
    // slots, kNone past the end.
    StreamCtl* sc = reinterpret_cast<StreamCtl*>(bp_smem + lay.off_stream) + warp;
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) {
            StreamSubj& q = sc->q[k];
            q.id = slot_subject(a, n_long, atomicAdd(a.cursor, 1u));
            if (k < 2 && in_range(a, q.id)) {
                q.s = a.db_off[a.first + (q.id & ~kSecond)];
                q.e = a.db_off[a.first + (q.id & ~kSecond) + 1];
            }
        }
    }
    __syncwarp();
    int base = a.window;   // diagonal stamp offset (gpu_blastp_kernel.cu:308)
    for (int i = 0;; i = i == 2 ? 0 : i + 1) {
        const int i1 = i == 2 ? 0 : i + 1, i2 = i1 == 2 ? 0 : i1 + 1;
        int go = 0;
        if (lane == 0) {
            const StreamSubj& cur = sc->q[i];
            const StreamSubj& nx = sc->q[i1];
            StreamSubj& nx2 = sc->q[i2];
            if (!in_range(a, cur.id)) {
                go = -1;
            } else {
                if (in_range(a, nx.id) && nx.e > nx.s && !done_first(a, n_long, nx.id, nx.e - nx.s))
                    prefetch_span(a.db, a.db_bytes, nx.s, nx.e);
                if (in_range(a, nx2.id)) {
                    nx2.s = a.db_off[a.first + (nx2.id & ~kSecond)];
                    nx2.e = a.db_off[a.first + (nx2.id & ~kSecond) + 1];
                }
                go = done_first(a, n_long, cur.id, cur.e - cur.s) ? 0 : 1;
            }
        }
        go = __shfl_sync(kFull, go, 0);
        if (go < 0) break;
        __syncwarp();
        if (go) {
            const StreamSubj& cur = sc->q[i];
            const long long s0 = cur.s, e0 = cur.e;
            scan_subject<CellT, kDefer, false, DiagT, false, kProf>(a, m, qs, cells, entries, wr.diag, lay.L,
                                                                  wr.lane_pos, wr.tasks,
                                               wr.blocked, wr.wcnt, a.oid_base + (int)(cur.id & ~kSecond), a.db + s0,
                                               (int)(e0 - s0), base, lane);
        }
        __syncwarp();
        if (lane == 0) sc->q[i].id = slot_subject(a, n_long, atomicAdd(a.cursor, 1u));
        __syncwarp();
    }
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Lane 0 of a streaming launch: whether chunk c's residues are there.  The
// wait is bounded by a.wait_ns and by a poll count; when either runs out, or
// another warp has given up already, *stalled is set and the warp stops.
__device__ bool wait_chunk(const ScanArgs& a, int c) {
    const volatile uint32_t* f = a.chunk_flag + c;
    if (*f != a.gen) {
        const volatile uint32_t* st = a.stalled;
        const uint64_t t0 = global_ns();
        uint32_t polls = 0;
        while (*f != a.gen) {
            if (*st || ++polls >= (1u << 26) || global_ns() - t0 > a.wait_ns) {
                atomicOr(a.stalled, 1u);
                return false;
            }
            __nanosleep(256);
        }
    }
    __threadfence();
    return true;
}

// Lane 0 of a streaming launch: the device span [s, e) of subject id of the
// range and its chunk c; false when its offsets leave the chunk (out of
// order).  A warp's subjects come in increasing order, so the chunk hint
// only moves forward.
__device__ __forceinline__ bool locate(const ScanArgs& a, uint32_t id, int& hint, long long& s, long long& e,
                                       int& c) {
    while (hint + 1 < a.n_chunks && (int)id >= a.chunk_first[hint + 1]) ++hint;
    c = hint;
    const long long lo = a.db_off[a.first + id], hi = a.db_off[a.first + id + 1];
    const long long clo = a.chunk_lo[c], chi = a.chunk_lo[c + 1];
    if (lo < clo || hi < lo || hi > chi || hi - lo > (1LL << 29)) return false;
    s = a.chunk_base[c] + (lo - clo);
    e = s + (hi - lo);
    return true;
}

// Streaming form of scan_kernel for the host-to-host search: one launch over
// all subjects while their residues are still being uploaded in chunks.  The
// subjects go in index order through the same three-stage pipeline; before
// a subject is scanned, lane 0 waits (bounded) for its chunk's flag, which
// the upload stream writes with a 4-byte copy after the chunk's data.  Each
// chunk starts on a 128-byte boundary of the device buffer, so no cache
// line read after a flag can hold bytes loaded before it.  Residue codes are
// checked as they are read; offsets are checked against their chunk before
// any residue of the subject is touched.
template <typename CellT, bool kCellsSmem, bool kDefer, bool kProf>
__global__ void __launch_bounds__(kMaxWarps * 32, 1)
scan_stream_kernel(ScanArgs a, ScanLayout lay) {
    const int8_t* m;
    const uint8_t* qs;
    const CellT* cells;
    const uint16_t* entries;
    load_tables<CellT, kCellsSmem>(a, lay, m, qs, cells, entries);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpRegions<uint16_t> wr = warp_regions<uint16_t>(lay, warp, lane);
    for (int i = lane; i < lay.L; i += 32) wr.diag[i] = 0;
    StreamCtl* sc = reinterpret_cast<StreamCtl*>(bp_smem + lay.off_stream) + warp;
    const uint32_t n = (uint32_t)a.n;
    if (lane == 0) {
        sc->hint = 0;
        sc->ready = -1;
        for (int k = 0; k < 3; ++k) {
            StreamSubj& q = sc->q[k];
            q.id = atomicAdd(a.cursor, 1u);
            q.ok = 0;
            if (k < 2 && q.id < n) q.ok = locate(a, q.id, sc->hint, q.s, q.e, q.c);
        }
    }
    __syncthreads();
    int base = a.window;
    for (int i = 0;; i = i == 2 ? 0 : i + 1) {
        const int i1 = i == 2 ? 0 : i + 1, i2 = i1 == 2 ? 0 : i1 + 1;
        int go = 0;
        if (lane == 0) {
            StreamSubj& cur = sc->q[i];
            StreamSubj& nx = sc->q[i1];
            StreamSubj& nx2 = sc->q[i2];
            if (cur.id >= n) {
                go = -2;                                     // nothing left
            } else {
                if (nx.id < n && nx.ok && nx.c <= sc->ready && nx.e > nx.s)
                    prefetch_span(a.db, a.db_bytes, nx.s, nx.e);
                if (nx2.id < n) nx2.ok = locate(a, nx2.id, sc->hint, nx2.s, nx2.e, nx2.c);
                if (!cur.ok) {
                    atomicOr(a.bad_off, 1u);
                } else if (cur.c <= sc->ready) {
                    go = 1;
                } else if (wait_chunk(a, cur.c)) {
                    sc->ready = cur.c;
                    go = 1;
                } else {
                    go = -1;                                 // the upload stalled: the host reports it
                }
            }
        }
        go = __shfl_sync(kFull, go, 0);
        if (go < 0) break;
        __syncwarp();
        const StreamSubj& cur = sc->q[i];
        if (go) {
            const long long s0 = cur.s, e0 = cur.e;
            scan_subject<CellT, kDefer, false, uint16_t, true, kProf>(a, m, qs, cells, entries, wr.diag, lay.L,
                                                                    wr.lane_pos, wr.tasks, wr.blocked, wr.wcnt,
                                                                    a.oid_base + (int)cur.id, a.db + s0,
                                                                    (int)(e0 - s0), base, lane);
        }
        __syncwarp();
        if (lane == 0) sc->q[i].id = atomicAdd(a.cursor, 1u);   // becomes the one after next
        __syncwarp();
    }
}

// Per-CTA control block of the batched kernel (shared memory).
struct BatchCtl {
    ScanArgs args;         // the current query's view, read by scan_subject
    int item;              // work item in hand (-1: none left)
    unsigned sub_ctr;      // next subject of the item
};

// Batched form: many queries against one resident database in one launch.
// Work items are (unit, subject chunk) pairs, a unit being one query or (kPacked)
// a packed table of several short queries; a CTA takes items from its own
// queue (per-CTA schedule) or from a global cursor, loads a unit's table
// into shared memory only when the unit changes, prefetches the chunk's
// residues into L2, and its warps share the chunk's subjects.  Each
// (query, subject) pair sees exactly the plain kernel's sequence of events,
// so every query's result is its single-query result; counters and records
// are indexed by segment = query * n_subjects + subject.
template <typename CellT, bool kCellsSmem, bool kDefer, bool kPacked, typename DiagT, bool kProf = false>
__global__ void __launch_bounds__(kMaxWarps * 32, 1)
scan_batch_kernel(BatchArgs b, ScanLayout lay) {
    uint8_t* sm = bp_smem;
    int8_t* m = reinterpret_cast<int8_t*>(sm);
    uint8_t* qs = sm + lay.off_query;
    BatchCtl* ctl = reinterpret_cast<BatchCtl*>(sm + lay.off_ctl);
    for (int i = threadIdx.x; i < 28 * BP_MROW; i += blockDim.x) m[i] = b.matrix[i];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpRegions<DiagT> wr = warp_regions<DiagT>(lay, warp, lane);
    for (int i = lane; i < lay.L; i += 32) wr.diag[i] = 0;
    int base = b.window;   // diagonal stamp offset, carried across queries (stale stamps stay stale)
    int cur_q = -1;
    const CellT* cells = nullptr;
    const uint16_t* entries = nullptr;
    int qpos = 0, qend = 0;
    if (b.queue_off) {
        qpos = b.queue_off[blockIdx.x];
        qend = b.queue_off[blockIdx.x + 1];
    }
    for (;;) {
        if (threadIdx.x == 0) {
            int it = -1;
            if (b.queue_off) {
                if (qpos < qend) it = b.queue_items[qpos++];
            } else {
                const int k = (int)atomicAdd(b.item_cursor, 1u);
                if (k < b.n_items) it = b.cursor_order ? b.cursor_order[k] : k;
            }
            ctl->item = it;
            ctl->sub_ctr = 0;
        }
        __syncthreads();
        const int it = ctl->item;
        if (it < 0) break;
        const WorkItem wi = b.items[it];
        if (wi.qid != cur_q) {
            const BatchQuery bq = b.queries[wi.qid];
            for (int i = threadIdx.x; i < bq.qlen; i += blockDim.x) qs[i] = bq.query[i];
            if (kProf) {
                // this query's profile, right after it (inside the region the
                // layout sized for the class's longest query)
                int8_t* pf = reinterpret_cast<int8_t*>(qs + ((bq.qlen + 15) & ~15));
                for (int i = threadIdx.x; i < bq.qlen * BP_MROW; i += blockDim.x)
                    pf[i] = b.matrix[(int)__ldg(bq.query + i / BP_MROW) * BP_MROW + i % BP_MROW];
            }
            if (kCellsSmem) {
                CellT* c = reinterpret_cast<CellT*>(sm + lay.off_cells);
                for (int i = threadIdx.x; i <= BP_NC; i += blockDim.x) c[i] = (CellT)bq.cells[i];
                cells = c;
            } else {
                cells = reinterpret_cast<const CellT*>(bq.cells);
            }
            if (lay.entries_smem) {
                uint16_t* e = reinterpret_cast<uint16_t*>(sm + lay.off_entries);
                for (int i = threadIdx.x; i < bq.n_entries; i += blockDim.x) e[i] = bq.entries[i];
                entries = e;
            } else {
                entries = bq.entries;
            }
            if (kPacked) {
                int32_t* mm = reinterpret_cast<int32_t*>(sm + lay.off_members);
                for (int i = threadIdx.x; i < 5 * bq.n_members; i += blockDim.x) mm[i] = bq.members[i];
                uint8_t* mof = sm + lay.off_mof;
                for (int i = threadIdx.x; i < bq.qlen; i += blockDim.x) mof[i] = bq.member_of[i];
            }
            if (threadIdx.x == 0) {
                ScanArgs& a = ctl->args;
                a.members = reinterpret_cast<const int32_t*>(sm + lay.off_members);
                a.member_of = sm + lay.off_mof;
                a.n_members = bq.n_members;
                a.seg_stride = b.n_subjects;
                a.query = bq.query;
                a.qlen = bq.qlen;
                a.ctx = bq.ctx;
                a.n_ctx = bq.n_ctx;
                a.window = b.window;
                a.diag_len = bq.diag_len;
                a.counters = b.counters;
                a.recs = b.recs;
                a.rec_cap = b.rec_cap;
                a.rec_count = b.rec_count;
            }
            cur_q = wi.qid;
            __syncthreads();
        }
        if (threadIdx.x == 0 && wi.count > 0) {
            // stream the chunk's residues into L2 ahead of the warps
            long long lo = b.db_off[wi.first] & ~15LL;
            const long long hi = (b.db_off[wi.first + wi.count] + 15) & ~15LL;
            while (lo < hi) {
                const long long n = min(hi - lo, (long long)(1 << 20));
                prefetch_l2(b.db + lo, (uint32_t)n);
                lo += n;
            }
        }
        const BatchQuery* unit = b.queries + wi.qid;
        const long long seg0 = kPacked ? 0 : (long long)__ldg(&unit->seg_query) * b.n_subjects;
        for (;;) {
            unsigned s = 0;
            if (lane == 0) s = atomicAdd(&ctl->sub_ctr, 1u);
            s = __shfl_sync(kFull, s, 0);
            // longest first: the item's long subjects, then the others in order
            if (s >= (unsigned)(wi.n_long + wi.count)) break;
            const bool second = s >= (unsigned)wi.n_long;
            const int oid = second ? wi.first + (int)s - wi.n_long : __ldg(b.long_ids + wi.long_first + (int)s);
            const long long so = b.db_off[oid], eo = b.db_off[oid + 1];
            if (second && wi.n_long > 0 && eo - so >= b.long_min) continue;   // scanned in the first pass
            // (offset resets clear the launch's whole array, lay.L entries:
            // queries with a longer array than this one read past its end)
            scan_subject<CellT, kDefer, kPacked, DiagT, false, kProf>(ctl->args, m, qs, cells, entries, wr.diag, lay.L,
                                                                      wr.lane_pos, wr.tasks, wr.blocked, wr.wcnt,
                                                                      (int)(seg0 + oid - b.subject_first), b.db + so,
                                                                      (int)(eo - so), base, lane);
        }
        __syncthreads();
    }
}

ScanLayout make_layout(int qlen, int L, int64_t n_entries, int warps, int cells_mode, int entries_smem,
                       bool packed, bool stream = false, bool prof = false) {
    ScanLayout l{};
    l.warps = warps;
    l.cells_mode = cells_mode;
    l.entries_smem = entries_smem;
    l.L = L;
    auto al = [](long long x, long long a) { return (x + a - 1) / a * a; };
    long long off = 1024;                             // matrix 28 x 32
    l.off_cells = (int)off;
    if (cells_mode == 0) off = al(off + (BP_NC + 1) * 2LL, 16);
    else if (cells_mode == 1) off = al(off + (BP_NC + 1) * 4LL, 16);
    l.off_entries = (int)off;
    if (entries_smem) off = al(off + n_entries * 2, 16);
    const long long big = 1LL << 30;                  // anything this large cannot fit
    if (off > big) off = big;
    l.off_query = (int)off;
    off = al(off + qlen, 16);
    if (prof) {   // right after the query: the walks find it from the query's address
        l.off_prof = (int)off;
        off = al(off + (long long)BP_MROW * qlen, 16);
    }
    l.off_members = (int)off;
    l.off_mof = (int)off;
    if (packed) {
        off = al(off + 5 * 4 * kMaxMembers, 16);
        l.off_mof = (int)off;
        off = al(off + qlen, 16);
    }
    l.off_warps = (int)off;
    const long long diag_bytes = (long long)L * (L <= kNarrowMaxL ? 2 : 4);
    const long long wb = al(diag_bytes + 32 * kRow * 4 + (kTaskCap + kBlkCap) * (long long)sizeof(Task) +
                                (packed ? 3 * 4 * kMaxMembers : 0),
                            16);
    l.warp_bytes = (int)(wb > big ? big : wb);
    off += (long long)warps * wb;
    off = al(off, 16);
    l.off_ctl = (int)(off > big ? big : off);
    off += 512;                                       // batched kernel's control block
    l.off_stream = (int)(off > big ? big : off);
    if (stream) off += kMaxWarps * (long long)sizeof(StreamCtl);
    l.total = (int)(off > big ? big : off);
    return l;
}

// Picks the layout with the most warps, preferring the whole table in shared
// memory as long as that still leaves at least 16 warps.  Plain and streaming
// launches of queries whose extensions are queued (one lane walks each) also
// get the query's score profile when it costs at most one warp and moves
// nothing out of shared memory: the walks then read one profile byte per
// letter instead of the query letter and the matrix entry (250 aa: 4.47 ->
// 4.38 ms, 500 aa: 6.50 -> 6.38 ms per 1M subjects; at 700 aa it would cost
// two warps, 8.37 -> 8.76 ms, at 1,000 aa the table's place in shared
// memory, 12.6 -> 15.3 ms).
// The same layout with the query's score profile added, at the same warps or
// one fewer; unchanged when that does not fit (or the array is 32-bit wide).
ScanLayout with_profile(const ScanLayout& l, int qlen, int64_t n_entries, int smem_optin, bool packed, bool stream) {
    if (l.L > kNarrowMaxL) return l;
    for (int wp = l.warps; wp >= l.warps - 1 && wp >= 1; --wp) {
        const ScanLayout lp = make_layout(qlen, l.L, n_entries, wp, l.cells_mode, l.entries_smem, packed, stream, true);
        if (lp.total <= smem_optin) return lp;
    }
    return l;
}

bool choose_layout(int qlen, int L, int64_t n_entries, int smem_optin, ScanLayout* out, bool packed = false,
                   bool stream = false) {
    const int cell_modes[2] = {n_entries < 65536 ? 0 : 1, 2};
    for (int min_w : {16, 8, 1})
        for (int cm : cell_modes)
            for (int es = 1; es >= 0; --es) {
                if (es && cm == 2) continue;
                for (int w = kMaxWarps; w >= min_w; --w) {
                    const ScanLayout l = make_layout(qlen, L, n_entries, w, cm, es, packed, stream);
                    if (l.total <= smem_optin) {
                        *out = l;
                        if (stream && !packed && qlen >= kDeferMinQlen)
                            *out = with_profile(l, qlen, n_entries, smem_optin, packed, stream);
                        return true;
                    }
                }
            }
    return false;
}

template <typename CellT, bool kCellsSmem, bool kDefer, typename DiagT, bool kProf = false>
cudaError_t launch(bp_engine* e, cudaStream_t stream, const ScanArgs& a, const ScanLayout& lay) {
    auto kern = scan_kernel<CellT, kCellsSmem, kDefer, DiagT, kProf>;
    // the largest allowed size, not this launch's: launches of one instance
    // with different layouts (batch classes, captured graph nodes replayed
    // later) must all stay valid whatever order the attribute was set in
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem_optin);
    if (err != cudaSuccess) return err;
    int grid = e->sm_count;
    const int need = (a.n + lay.warps - 1) / lay.warps;   // no more CTAs than subjects to feed them
    if (grid > need) grid = need > 0 ? need : 1;
    kern<<<grid, lay.warps * 32, lay.total, stream>>>(a, lay);
    e->launches += 1;
    return cudaGetLastError();
}

template <typename CellT, bool kCellsSmem, bool kDefer, bool kProf = false>
cudaError_t launch_stream(bp_engine* e, cudaStream_t stream, const ScanArgs& a, const ScanLayout& lay) {
    auto kern = scan_stream_kernel<CellT, kCellsSmem, kDefer, kProf>;
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem_optin);
    if (err != cudaSuccess) return err;
    int grid = e->sm_count;
    const int need = (a.n + lay.warps - 1) / lay.warps;
    if (grid > need) grid = need > 0 ? need : 1;
    kern<<<grid, lay.warps * 32, lay.total, stream>>>(a, lay);
    e->launches += 1;
    return cudaGetLastError();
}

template <typename CellT, bool kCellsSmem, bool kDefer, bool kPacked, typename DiagT, bool kProf = false>
cudaError_t launch_batch(bp_engine* e, cudaStream_t stream, const BatchArgs& b, const ScanLayout& lay, int grid) {
    auto kern = scan_batch_kernel<CellT, kCellsSmem, kDefer, kPacked, DiagT, kProf>;
    // the largest allowed size, not this launch's: launches of one instance
    // with different layouts (batch classes, captured graph nodes replayed
    // later) must all stay valid whatever order the attribute was set in
    cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem_optin);
    if (err != cudaSuccess) return err;
    kern<<<grid, lay.warps * 32, lay.total, stream>>>(b, lay);
    e->launches += 1;
    return cudaGetLastError();
}

}  // namespace

static_assert(sizeof(BatchCtl) <= 512, "batched control block must fit its shared-memory slot");
static_assert(sizeof(Task) == 16, "task layout");
static_assert(sizeof(BatchCtl) % 8 == 0 && 512 % 8 == 0, "stream control blocks stay 8-byte aligned");
static_assert((32 * kRow * 4) % 16 == 0, "the task queue after the position table stays 16-byte aligned");
static_assert(kRow % 2 == 1, "odd row stride: one bank per lane");
static_assert(kMaxMembers == BP_MAX_PACK_MEMBERS, "pack size limit");

int bp_diag_len(int qlen, int window) {
    const long long n = ((long long)qlen + window + 31) / 32 * 32;
    return (int)(n < 128 ? 128 : (n > (1LL << 30) ? (1LL << 30) : n));
}

// Diagonal arrays longer than kNarrowMaxL (query + window above about 8,000)
// use 32-bit entries and always queue their extensions (the results are the
// same either way).
template <bool kPacked>
cudaError_t launch_batch_layout(bp_engine* e, cudaStream_t stream, const BatchArgs& b, const ScanLayout& lay,
                                int grid, bool defer) {
    using N = uint16_t;
    if (!kPacked && lay.L > kNarrowMaxL) {
        if (lay.cells_mode == 0) return launch_batch<uint16_t, true, true, false, uint32_t>(e, stream, b, lay, grid);
        if (lay.cells_mode == 1) return launch_batch<uint32_t, true, true, false, uint32_t>(e, stream, b, lay, grid);
        return launch_batch<uint32_t, false, true, false, uint32_t>(e, stream, b, lay, grid);
    }
    if (lay.L > kNarrowMaxL) return cudaErrorInvalidValue;   // packed tables are short
    if constexpr (!kPacked) {
        if (defer && lay.off_prof) {
            if (lay.cells_mode == 0) return launch_batch<uint16_t, true, true, false, N, true>(e, stream, b, lay, grid);
            if (lay.cells_mode == 1) return launch_batch<uint32_t, true, true, false, N, true>(e, stream, b, lay, grid);
            return launch_batch<uint32_t, false, true, false, N, true>(e, stream, b, lay, grid);
        }
    }
    if (defer) {
        if (lay.cells_mode == 0) return launch_batch<uint16_t, true, true, kPacked, N>(e, stream, b, lay, grid);
        if (lay.cells_mode == 1) return launch_batch<uint32_t, true, true, kPacked, N>(e, stream, b, lay, grid);
        return launch_batch<uint32_t, false, true, kPacked, N>(e, stream, b, lay, grid);
    }
    if (lay.cells_mode == 0) return launch_batch<uint16_t, true, false, kPacked, N>(e, stream, b, lay, grid);
    if (lay.cells_mode == 1) return launch_batch<uint32_t, true, false, kPacked, N>(e, stream, b, lay, grid);
    return launch_batch<uint32_t, false, false, kPacked, N>(e, stream, b, lay, grid);
}

cudaError_t bp_launch_scan_batch(bp_engine* e, cudaStream_t stream, const BatchArgs& b, int32_t max_qlen,
                                 int32_t max_diag_len, int64_t max_entries, int grid, int max_warps, bool packed) {
    ScanLayout lay;
    if (!choose_layout(max_qlen, max_diag_len, max_entries, e->smem_optin, &lay, packed)) return cudaErrorInvalidValue;
    if (max_warps > 0 && lay.warps > max_warps) {
        lay = make_layout(max_qlen, max_diag_len, max_entries, max_warps, lay.cells_mode, lay.entries_smem, packed);
    }
    const bool defer = max_qlen >= kDeferMinQlen;
    if (!packed && defer) lay = with_profile(lay, max_qlen, max_entries, e->smem_optin, false, false);
    return packed ? launch_batch_layout<true>(e, stream, b, lay, grid, defer)
                  : launch_batch_layout<false>(e, stream, b, lay, grid, defer);
}

int bp_scan_warps(int32_t qlen, int32_t diag_len, int64_t n_entries, int smem_optin, bool packed) {
    ScanLayout l;
    return choose_layout(qlen, diag_len, n_entries, smem_optin, &l, packed) ? l.warps : 0;
}

bool bp_scan_defers(int32_t qlen) { return qlen >= kDeferMinQlen; }

bool bp_scan_fits(int32_t qlen, int32_t diag_len, int64_t n_entries, int smem_optin) {
    // (with the per-warp subject pipelines the plain and streaming launches reserve)
    ScanLayout l;
    return choose_layout(qlen, diag_len, n_entries, smem_optin, &l, false, true);
}

cudaError_t bp_launch_scan(bp_engine* e, const ScanArgs& a) { return bp_launch_scan_on(e, e->stream, a); }

bool bp_scan_streams(int32_t diag_len) { return diag_len <= kNarrowMaxL; }

cudaError_t bp_launch_scan_stream(bp_engine* e, cudaStream_t st, const ScanArgs& a) {
    ScanLayout lay;
    if (!choose_layout(a.qlen, a.diag_len, a.n_entries, e->smem_optin, &lay, false, true))
        return cudaErrorInvalidValue;
    if (lay.L > kNarrowMaxL || a.n_chunks < 1) return cudaErrorNotSupported;
    if (a.qlen >= kDeferMinQlen && lay.off_prof) {
        if (lay.cells_mode == 0) return launch_stream<uint16_t, true, true, true>(e, st, a, lay);
        if (lay.cells_mode == 1) return launch_stream<uint32_t, true, true, true>(e, st, a, lay);
        return launch_stream<uint32_t, false, true, true>(e, st, a, lay);
    }
    if (a.qlen >= kDeferMinQlen) {
        if (lay.cells_mode == 0) return launch_stream<uint16_t, true, true>(e, st, a, lay);
        if (lay.cells_mode == 1) return launch_stream<uint32_t, true, true>(e, st, a, lay);
        return launch_stream<uint32_t, false, true>(e, st, a, lay);
    }
    if (lay.cells_mode == 0) return launch_stream<uint16_t, true, false>(e, st, a, lay);
    if (lay.cells_mode == 1) return launch_stream<uint32_t, true, false>(e, st, a, lay);
    return launch_stream<uint32_t, false, false>(e, st, a, lay);
}

cudaError_t bp_launch_scan_on(bp_engine* e, cudaStream_t st, const ScanArgs& a) {
    ScanLayout lay;
    if (!choose_layout(a.qlen, a.diag_len, a.n_entries, e->smem_optin, &lay, false, true))
        return cudaErrorInvalidValue;
    using N = uint16_t;
    if (lay.L > kNarrowMaxL) {
        // (32-bit arrays always queue their extensions: a query that is short
        // but has a very large window gets the same results either way)
        if (lay.cells_mode == 0) return launch<uint16_t, true, true, uint32_t>(e, st, a, lay);
        if (lay.cells_mode == 1) return launch<uint32_t, true, true, uint32_t>(e, st, a, lay);
        return launch<uint32_t, false, true, uint32_t>(e, st, a, lay);
    }
    if (a.qlen >= kDeferMinQlen && lay.off_prof) {
        if (lay.cells_mode == 0) return launch<uint16_t, true, true, N, true>(e, st, a, lay);
        if (lay.cells_mode == 1) return launch<uint32_t, true, true, N, true>(e, st, a, lay);
        return launch<uint32_t, false, true, N, true>(e, st, a, lay);
    }
    if (a.qlen >= kDeferMinQlen) {
        if (lay.cells_mode == 0) return launch<uint16_t, true, true, N>(e, st, a, lay);
        if (lay.cells_mode == 1) return launch<uint32_t, true, true, N>(e, st, a, lay);
        return launch<uint32_t, false, true, N>(e, st, a, lay);
    }
    if (lay.cells_mode == 0) return launch<uint16_t, true, false, N>(e, st, a, lay);
    if (lay.cells_mode == 1) return launch<uint32_t, true, false, N>(e, st, a, lay);
    return launch<uint32_t, false, false, N>(e, st, a, lay);
}
