// Batched search: many queries against one HBM-resident database in one
// persistent launch (scan_batch_kernel), optionally captured in a CUDA graph
// and replayed.
//
// The reference searches one query per kernel launch (gpu_blastp.cu:197-210,
// the query in constant memory, contexts capped at 4096).  Here a batch of
// queries, each with its own device table, is cut into work items
// (query, subject chunk); the items are handed to the CTAs either through a
// global cursor, or through per-CTA queues filled statically (round robin) or
// from predicted costs (longest-processing-time-first into the least loaded
// queue).  Queries are grouped into classes by diagonal-array size, so a
// short query does not run with the shared-memory layout (and the lower warp
// count) of the longest one; each class is one persistent launch, the
// classes on parallel streams (parallel graph branches) so one class's tail
// overlaps the next class's start.  Every (query, subject) pair is scanned
// exactly as in the single-query kernel, so each query's result equals its
// single-query result.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <queue>
#include <vector>

#include "bp_internal.h"

#define CKB(call, what)                                                   \
    do {                                                                  \
        cudaError_t _err = (call);                                        \
        if (_err != cudaSuccess) return bp_set_cuda_error(e, _err, what); \
    } while (0)

struct bp_batch {
    bp_engine* e = nullptr;
    const bp_db* db = nullptr;
    int32_t nq = 0, n = 0, first = 0;    // n subjects from `first`
    int64_t nseg = 0;
    std::vector<const bp_query*> queries;
    bp_batch_options opt{};
    std::vector<int32_t> chunk_first;        // n_chunks + 1 subject boundaries
    // device
    BatchQuery* d_queries = nullptr;
    WorkItem* d_items = nullptr;
    int32_t* d_queue_off = nullptr;
    int32_t* d_queue_items = nullptr;
    int32_t* d_counters = nullptr;
    int64_t* d_hsp_off = nullptr;
    bp_hsp* d_hsps = nullptr;
    int32_t* d_keys = nullptr;
    uint32_t cap = 0;                        // capacity of d_hsps / d_keys / d_recs
    uint32_t alloc_cap = 0;
    HspRec* d_recs = nullptr;                // batch-owned scratch, so a captured graph
    int32_t* d_fill = nullptr;               // never points at engine buffers that a
    int64_t* d_blocksums = nullptr;          // later search may regrow
    uint32_t* d_counts = nullptr;            // [0] records, [1] item cursor
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t wait_first = nullptr;   // the first launch's device work waits for this event
    uint64_t launches_per_run = 0;
    float last_ms = 0.f;
    uint32_t* h_count = nullptr;
    int64_t n_hsps = -1;
    int32_t n_items = 0;
    struct Class {
        int32_t max_qlen = 0, max_len = 0;      // longest query and diagonal array
        int64_t max_entries = 0;
        int32_t item_lo = 0, item_hi = 0;      // its items in d_items
        int32_t queue_lo = 0;                  // its queue offsets start at d_queue_off[queue_lo]
        int32_t order_lo = 0;                  // BP_SCHED_COST_ORDER: its items in cursor order at d_queue_items[order_lo]
        int32_t grid = 0;
        double est = 0;                        // expected word hits, to order the launches
        bool packed = false;                   // its units are packed tables
        std::vector<int32_t> units;            // its units (indices into h_units)
    };
    std::vector<BatchQuery> h_units;         // every unit's tables (plain_unpacked launches)
    std::vector<Class> classes;
    std::vector<cudaStream_t> side;          // one per class after the first
    std::vector<cudaEvent_t> ev_join;
    cudaEvent_t ev_fork = nullptr;
    bool capturing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<double> queue_cost;         // predicted cost per CTA queue (cost schedules)
    std::vector<int32_t> item_queue;        // caller's item index -> queue (-1: dynamic)
    std::vector<void*> pack_mem;            // device buffers of the packed tables
    int32_t n_units = 0, n_packs = 0;
};

namespace {

constexpr int32_t kBaseChunk = 1 << 16;   // the cost model's chunk (residues)

// Chunk boundaries over subjects [s0, s1): each chunk holds at least one
// subject, then as many more as keep it within chunk_residues residues.
void plan_direct(const bp_db* db, int32_t s0, int32_t s1, int32_t chunk_residues, std::vector<int32_t>& first) {
    first.clear();
    first.push_back(s0);
    const int64_t* off = db->h_off.data();
    int32_t s = s0;
    while (s < s1) {
        const int64_t limit = off[s] + std::max<int64_t>(chunk_residues, 1);
        int32_t t = (int32_t)(std::upper_bound(off + s + 1, off + s1 + 1, limit) - off) - 1;
        if (t <= s) t = s + 1;
        if (t > s1) t = s1;
        first.push_back(t);
        s = t;
    }
}

// Chunks of at least two base chunks are unions of consecutive base chunks
// (64Ki residues, the cost model's unit), so an item's predicted cost is the
// sum of its base chunks' predictions.
void plan_chunks(const bp_db* db, int32_t s0, int32_t s1, int32_t chunk_residues, std::vector<int32_t>& first) {
    if (chunk_residues < 2 * kBaseChunk) {
        plan_direct(db, s0, s1, chunk_residues, first);
        return;
    }
    std::vector<int32_t> base;
    plan_direct(db, s0, s1, kBaseChunk, base);
    const size_t k = (size_t)chunk_residues / kBaseChunk;
    first.clear();
    for (size_t i = 0; i + 1 < base.size(); i += k) first.push_back(base[i]);
    first.push_back(base.back());
}

bool resolve_range(const bp_db* db, int32_t first, int32_t count, int32_t* s0, int32_t* s1) {
    if (first < 0 || first > db->n) return false;
    if (count < 0) count = db->n - first;
    if ((int64_t)first + count > db->n) return false;
    *s0 = first;
    *s1 = first + count;
    return true;
}

// Enqueues the batch's device work on the engine stream: one persistent
// launch per class (forked onto side streams), then the ordering pass.
bp_status enqueue(bp_batch* b) {
    bp_engine* e = b->e;
    const uint64_t l0 = e->launches;
    CKB(cudaMemsetAsync(b->d_counts, 0, (4 + b->classes.size() + b->h_units.size()) * sizeof(uint32_t), e->stream),
        "memset(counts)");
    // inside a capture a timing event must be an external record node
    const unsigned rec_flags = b->capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    CKB(cudaEventRecordWithFlags(b->ev0, e->stream, rec_flags), "cudaEventRecord");
    CKB(cudaEventRecord(b->ev_fork, e->stream), "cudaEventRecord");
    for (size_t c = 0; c < b->classes.size(); ++c) {
        const bp_batch::Class& k = b->classes[c];
        cudaStream_t st = c == 0 ? e->stream : b->side[c - 1];
        if (c > 0) CKB(cudaStreamWaitEvent(st, b->ev_fork, 0), "cudaStreamWaitEvent");
        BatchArgs a;
        a.db = b->db->d_res;
        a.db_off = b->db->d_off;
        a.n_subjects = b->n;
        a.subject_first = b->first;
        a.queries = b->d_queries;
        a.n_queries = b->nq;
        a.items = b->d_items + k.item_lo;
        a.n_items = k.item_hi - k.item_lo;
        const bool cursor = b->opt.schedule == BP_SCHED_DYNAMIC || b->opt.schedule == BP_SCHED_COST_ORDER;
        a.queue_off = cursor ? nullptr : b->d_queue_off + k.queue_lo;
        a.queue_items = b->d_queue_items;
        a.cursor_order = b->opt.schedule == BP_SCHED_COST_ORDER ? b->d_queue_items + k.order_lo : nullptr;
        a.item_cursor = b->d_counts + 4 + c;
        a.matrix = e->d_matrix;
        a.window = b->queries[0]->p.window;
        a.counters = b->d_counters;
        a.recs = b->d_recs;
        a.rec_cap = b->cap;
        a.rec_count = b->d_counts;
        a.long_ids = b->db->d_long;
        a.long_min = b->db->long_min;
        if (b->opt.plain_unpacked && !k.packed) {
            // each query of the class as the plain single-query scan over the
            // batch's subjects (its own cursor), into the same segments
            for (int32_t ui : k.units) {
                const BatchQuery& u = b->h_units[(size_t)ui];
                ScanArgs p{};
                p.db = b->db->d_res;
                p.db_bytes = ((b->db->nres + 15) & ~15LL) + 32;   // the allocation's zero padding included
                p.db_off = b->db->d_off;
                p.first = b->first;
                p.n = b->n;
                p.query = u.query;
                p.qlen = u.qlen;
                p.cells = u.cells;
                p.entries = u.entries;
                p.n_entries = u.n_entries;
                p.ctx = u.ctx;
                p.n_ctx = u.n_ctx;
                p.matrix = e->d_matrix;
                p.window = a.window;
                p.diag_len = u.diag_len;
                p.counters = b->d_counters;
                p.oid_base = u.seg_query * b->n;
                p.recs = b->d_recs;
                p.rec_cap = b->cap;
                p.rec_count = b->d_counts;
                p.cursor = b->d_counts + 4 + b->classes.size() + ui;
                int32_t long_lo = 0;
                bp_long_slice(b->db->h_long, b->first, b->n, &long_lo, &p.n_long);
                p.long_ids = b->db->d_long ? b->db->d_long + long_lo : nullptr;
                p.long_min = b->db->long_min;
                if (p.n > 0) CKB(bp_launch_scan_on(e, st, p), "plain scan launch");
            }
        } else if (a.n_items > 0) {
            CKB(bp_launch_scan_batch(e, st, a, k.max_qlen, k.max_len, k.max_entries, k.grid, b->opt.max_warps,
                                     k.packed),
                "batched scan launch");
        }
        if (c > 0) {
            CKB(cudaEventRecord(b->ev_join[c - 1], st), "cudaEventRecord");
            CKB(cudaStreamWaitEvent(e->stream, b->ev_join[c - 1], 0), "cudaStreamWaitEvent");
        }
    }
    CKB(cudaEventRecordWithFlags(b->ev1, e->stream, rec_flags), "cudaEventRecord");
    CKB(bp_launch_order(e, (int32_t)b->nseg, b->d_counters, b->d_hsp_off, b->d_recs, b->cap, b->d_counts,
                        b->d_fill, b->d_hsps, b->d_keys, b->d_blocksums),
        "order kernels launch");
    CKB(cudaMemcpyAsync(b->h_count, b->d_counts, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream),
        "copy counts");
    b->launches_per_run = e->launches - l0;
    return BP_OK;
}

// Sizes the batch's scratch and outputs for the current record capacity.
bp_status prepare(bp_batch* b) {
    bp_engine* e = b->e;
    if (!b->d_counts) {
        CKB(cudaMallocAsync((void**)&b->d_counts, (4 + b->classes.size() + b->h_units.size()) * sizeof(uint32_t),
                            e->stream),
            "cudaMalloc(counts)");
        CKB(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming), "cudaEventCreate");
        for (size_t c = 1; c < b->classes.size(); ++c) {
            cudaStream_t st = nullptr;
            cudaEvent_t ev = nullptr;
            CKB(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
            b->side.push_back(st);
            CKB(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
            b->ev_join.push_back(ev);
        }
        CKB(cudaMallocAsync((void**)&b->d_fill, (size_t)std::max<int64_t>(b->nseg, 1) * sizeof(int32_t), e->stream), "cudaMalloc(fill)");
        CKB(cudaMallocAsync((void**)&b->d_blocksums,
                            (size_t)std::max(bp_order_blocksums_needed((int32_t)b->nseg), 1) * sizeof(int64_t),
                            e->stream),
            "cudaMalloc(sums)");
        CKB(cudaEventCreate(&b->ev0), "cudaEventCreate");
        CKB(cudaEventCreate(&b->ev1), "cudaEventCreate");
    }
    if (b->alloc_cap < b->cap || !b->d_hsps) {
        if (b->d_recs) cudaFreeAsync(b->d_recs, e->stream);
        if (b->d_hsps) cudaFreeAsync(b->d_hsps, e->stream);
        if (b->d_keys) cudaFreeAsync(b->d_keys, e->stream);
        b->d_recs = nullptr;
        b->d_hsps = nullptr;
        b->d_keys = nullptr;
        b->alloc_cap = 0;
        const size_t n = std::max<uint32_t>(b->cap, 1);
        CKB(cudaMallocAsync((void**)&b->d_recs, n * sizeof(HspRec), e->stream), "cudaMalloc(records)");
        CKB(cudaMallocAsync((void**)&b->d_hsps, n * sizeof(bp_hsp), e->stream), "cudaMalloc(hsps)");
        CKB(cudaMallocAsync((void**)&b->d_keys, n * sizeof(int32_t), e->stream), "cudaMalloc(keys)");
        b->alloc_cap = b->cap;
    }
    return BP_OK;
}

bp_status capture(bp_batch* b) {
    bp_engine* e = b->e;
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    CKB(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeRelaxed), "begin capture");
    const uint64_t l0 = e->launches;
    b->capturing = true;
    bp_status st = enqueue(b);
    b->capturing = false;
    e->launches = l0;   // captured, not run
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamEndCapture(e->stream, &g);
    if (st != BP_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    CKB(err, "end capture");
    b->graph = g;
    CKB(cudaGraphInstantiate(&b->exec, g, 0), "instantiate graph");
    return BP_OK;
}

bp_status launch_batch(bp_batch* b) {
    bp_engine* e = b->e;
    b->n_hsps = -1;
    if (b->wait_first) {
        // after the host tables' copies: those come from pageable memory and
        // would hold the host until the stream reached them
        CKB(cudaStreamWaitEvent(e->stream, b->wait_first, 0), "cudaStreamWaitEvent");
        b->wait_first = nullptr;
    }
    if (b->opt.use_graph) {
        if (!b->exec) {
            bp_status st = capture(b);
            if (st != BP_OK) return st;
        }
        CKB(cudaGraphLaunch(b->exec, e->stream), "graph launch");
        e->launches += b->launches_per_run;   // the kernels captured in the graph
        return BP_OK;
    }
    return enqueue(b);
}

// Builds one packed table on the device: the members' residues end to end
// with `window` offsets between them (so no two members' hits can meet on one
// diagonal within the window), their tables merged cell by cell, the member
// of every offset, and each member's {index, offset, length, x-drop, cutoff}.
bp_status build_pack(bp_batch* b, const std::vector<BatchQuery>& hq, const bp_query* const* queries,
                     const std::vector<int32_t>& g, int window, BatchQuery* out) {
    bp_engine* e = b->e;
    cudaStream_t es = e->stream;
    std::vector<int32_t> members;
    std::vector<PackSrc> src;
    int32_t P = 0;
    int64_t n_entries = 0;
    for (size_t i = 0; i < g.size(); ++i) {
        const bp_query* q = queries[g[i]];
        if (i) P += window;
        members.insert(members.end(), {g[i], P, q->qlen, q->p.x_dropoff, q->p.cutoff_score});
        src.push_back(PackSrc{q->d_cells, q->d_entries, P, 0});
        P += q->qlen;
        n_entries += q->n_entries;
    }
    const int32_t L = bp_diag_len(P, window);
    if (P > 65535 || n_entries >= (1LL << 31) || bp_scan_warps(P, L, n_entries, e->smem_optin, true) == 0)
        return BP_ERR_TOO_LARGE;
    std::vector<uint8_t> mof((size_t)P, 0xff);
    for (size_t i = 0; i < g.size(); ++i)
        memset(mof.data() + members[5 * i + 1], (int)i, (size_t)members[5 * i + 2]);
    uint8_t* d_q = nullptr;
    uint8_t* d_mof = nullptr;
    uint32_t* d_cells = nullptr;
    uint32_t* d_tmp = nullptr;
    uint16_t* d_entries = nullptr;
    int32_t* d_members = nullptr;
    PackSrc* d_src = nullptr;
    auto track = [&](void* p) { b->pack_mem.push_back(p); };
    CKB(cudaMallocAsync((void**)&d_q, (size_t)((P + 15) & ~15) + 16, es), "cudaMallocAsync(pack)");
    track(d_q);
    CKB(cudaMallocAsync((void**)&d_mof, (size_t)P + 16, es), "cudaMallocAsync(pack)");
    track(d_mof);
    CKB(cudaMallocAsync((void**)&d_cells, (BP_NC + 1) * sizeof(uint32_t), es), "cudaMallocAsync(pack)");
    track(d_cells);
    CKB(cudaMallocAsync((void**)&d_tmp, BP_NC * sizeof(uint32_t), es), "cudaMallocAsync(pack)");
    track(d_tmp);
    CKB(cudaMallocAsync((void**)&d_entries, (size_t)std::max<int64_t>(n_entries, 1) * sizeof(uint16_t), es),
        "cudaMallocAsync(pack)");
    track(d_entries);
    CKB(cudaMallocAsync((void**)&d_members, members.size() * sizeof(int32_t), es), "cudaMallocAsync(pack)");
    track(d_members);
    CKB(cudaMallocAsync((void**)&d_src, src.size() * sizeof(PackSrc), es), "cudaMallocAsync(pack)");
    track(d_src);
    CKB(cudaMemsetAsync(d_q, 0, (size_t)((P + 15) & ~15) + 16, es), "memset(pack)");
    for (size_t i = 0; i < g.size(); ++i)
        if (hq[g[i]].qlen > 0)
            CKB(cudaMemcpyAsync(d_q + members[5 * i + 1], hq[g[i]].query, (size_t)hq[g[i]].qlen,
                                cudaMemcpyDeviceToDevice, es),
                "pack residues");
    CKB(cudaMemcpyAsync(d_mof, mof.data(), (size_t)P, cudaMemcpyHostToDevice, es), "pack members");
    CKB(cudaMemcpyAsync(d_members, members.data(), members.size() * sizeof(int32_t), cudaMemcpyHostToDevice, es),
        "pack members");
    CKB(cudaMemcpyAsync(d_src, src.data(), src.size() * sizeof(PackSrc), cudaMemcpyHostToDevice, es), "pack tables");
    CKB(bp_launch_pack_table(e, es, d_src, (int)g.size(), d_tmp, d_cells, d_entries), "pack table launch");
    BatchQuery u;
    u.query = d_q;
    u.cells = d_cells;
    u.entries = d_entries;
    u.ctx = nullptr;
    u.qlen = P;
    u.n_entries = (int32_t)n_entries;
    u.n_ctx = 1;
    u.diag_len = L;
    u.members = d_members;
    u.member_of = d_mof;
    u.n_members = (int32_t)g.size();
    u.seg_query = -1;
    *out = u;
    return BP_OK;
}

}  // namespace

extern "C" {

void bp_batch_options_default(bp_batch_options* o) {
    memset(o, 0, sizeof(*o));
    o->chunk_residues = 1 << 18;
    o->schedule = BP_SCHED_DYNAMIC;
    o->use_graph = 1;
    o->subject_first = 0;
    o->subject_count = -1;
    o->pack_residues = 512;
}

bp_status bp_batch_plan(const bp_db* db, int32_t subject_first, int32_t subject_count, int32_t chunk_residues,
                        int32_t* chunk_first, int32_t* n_chunks) {
    int32_t s0 = 0, s1 = 0;
    if (!db || !n_chunks || !resolve_range(db, subject_first, subject_count, &s0, &s1)) return BP_ERR_INVALID;
    std::vector<int32_t> first;
    plan_chunks(db, s0, s1, chunk_residues, first);
    *n_chunks = (int32_t)first.size() - 1;
    if (chunk_first) memcpy(chunk_first, first.data(), first.size() * sizeof(int32_t));
    return BP_OK;
}

bp_status bp_search_batch(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                          const bp_batch_options* opt, bp_batch** out) {
    return bp_search_batch_behind(e, db, queries, n_queries, opt, nullptr, out);
}

}  // extern "C"

bp_status bp_search_batch_behind(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                                 const bp_batch_options* opt, cudaEvent_t after, bp_batch** out) {
    if (!e || !db || !queries || n_queries < 0 || !out) return bp_set_error(e, BP_ERR_INVALID, "bp_search_batch: bad argument");
    *out = nullptr;
    bp_batch_options o;
    if (opt) o = *opt;
    else bp_batch_options_default(&o);
    if ((o.schedule == BP_SCHED_COSTS || o.schedule == BP_SCHED_COST_ORDER) && !o.item_costs)
        return bp_set_error(e, BP_ERR_INVALID, "bp_search_batch: cost schedule without item costs");
    if (o.schedule < BP_SCHED_DYNAMIC || o.schedule > BP_SCHED_COST_ORDER)
        return bp_set_error(e, BP_ERR_INVALID, "bp_search_batch: unknown schedule");
    int32_t s0 = 0, s1 = 0;
    if (!resolve_range(db, o.subject_first, o.subject_count, &s0, &s1))
        return bp_set_error(e, BP_ERR_INVALID, "bp_search_batch: subject range outside the database");
    if ((int64_t)n_queries * (s1 - s0) >= (1LL << 31) - 1)
        return bp_set_error(e, BP_ERR_TOO_LARGE, "bp_search_batch: queries x subjects must stay below 2^31");
    CKB(cudaSetDevice(e->device), "cudaSetDevice");
    bp_batch* b = new bp_batch();
    b->e = e;
    b->db = db;
    b->nq = n_queries;
    b->first = s0;
    b->n = s1 - s0;
    b->nseg = (int64_t)n_queries * b->n;
    b->opt = o;
    b->queries.assign(queries, queries + n_queries);
    plan_chunks(db, s0, s1, o.chunk_residues, b->chunk_first);
    const int32_t n_chunks = (int32_t)b->chunk_first.size() - 1;

    std::vector<BatchQuery> hq(n_queries);
    double hits_sum = 0;
    int window = -1;
    for (int32_t i = 0; i < n_queries; ++i) {
        const bp_query* q = queries[i];
        if (window >= 0 && q->p.window != window) {
            delete b;
            return bp_set_error(e, BP_ERR_INVALID, "bp_search_batch: all queries must share one window");
        }
        window = q->p.window;
        hq[i].query = q->d_q;
        hq[i].cells = q->d_cells;
        hq[i].entries = q->d_entries;
        hq[i].ctx = q->d_ctx;
        hq[i].qlen = q->qlen;
        hq[i].n_entries = (int32_t)q->n_entries;
        hq[i].n_ctx = q->n_ctx;
        hq[i].diag_len = q->diag_len;
        hq[i].members = nullptr;
        hq[i].member_of = nullptr;
        hq[i].n_members = 0;
        hq[i].seg_query = i;
        if (!bp_scan_fits(q->qlen, q->diag_len, q->n_entries, e->smem_optin)) {
            delete b;
            return bp_set_error(e, BP_ERR_TOO_LARGE, "bp_search_batch: a query is too long for the diagonal array");
        }
        hits_sum += q->hits_per_residue;
    }
    // units: short queries packed into shared tables, the others alone
    std::vector<std::vector<int32_t>> unit_queries;
    std::vector<BatchQuery> units;
    {
        const int32_t pmax = std::min(o.pack_residues, 65535);
        std::vector<char> packed(n_queries, 0);
        if (pmax > 0) {
            std::vector<int32_t> cand;
            for (int32_t i = 0; i < n_queries; ++i)
                if (hq[i].qlen <= pmax / 2 && queries[i]->n_ctx == 1) cand.push_back(i);
            std::stable_sort(cand.begin(), cand.end(), [&](int32_t x, int32_t y) { return hq[x].qlen < hq[y].qlen; });
            std::vector<std::vector<int32_t>> groups;
            int32_t P = 0;
            for (int32_t qi : cand) {
                const int32_t need = hq[qi].qlen + (groups.empty() || groups.back().empty() ? 0 : window);
                if (groups.empty() || (int)groups.back().size() == BP_MAX_PACK_MEMBERS || P + need > pmax) {
                    groups.emplace_back();
                    P = 0;
                }
                P += hq[qi].qlen + (groups.back().empty() ? 0 : window);
                groups.back().push_back(qi);
            }
            for (const auto& g : groups) {
                if (g.size() < 2) continue;
                BatchQuery u;
                bp_status st = build_pack(b, hq, queries, g, window, &u);
                if (st == BP_ERR_TOO_LARGE) continue;            // does not fit shared memory: leave unpacked
                if (st != BP_OK) {
                    bp_batch_destroy(b);
                    return st;
                }
                for (int32_t qi : g) packed[qi] = 1;
                units.push_back(u);
                unit_queries.push_back(g);
                b->n_packs += 1;
            }
        }
        for (int32_t i = 0; i < n_queries; ++i)
            if (!packed[i]) {
                units.push_back(hq[i]);
                unit_queries.push_back(std::vector<int32_t>(1, i));
            }
    }
    const int32_t n_units = (int32_t)units.size();
    b->n_units = n_units;
    b->h_units = units;
    // classes: a launch's layout is sized for its longest unit, so units share
    // a launch only when that leaves each of them the warps per CTA it would
    // get alone, and when they extend the same way; longest first
    auto own_warps = [&](int32_t i) {
        return bp_scan_warps(units[i].qlen, units[i].diag_len, units[i].n_entries, e->smem_optin,
                             units[i].n_members > 0);
    };
    std::vector<int32_t> order(n_units);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
        const bool px = units[x].n_members > 0, py = units[y].n_members > 0;
        if (px != py) return px;
        return units[x].diag_len != units[y].diag_len ? units[x].diag_len > units[y].diag_len
                                                       : units[x].n_entries > units[y].n_entries;
    });
    std::vector<WorkItem> items;
    items.reserve((size_t)n_units * n_chunks);
    std::vector<int32_t> item_pos((size_t)n_queries * n_chunks);   // caller's item index -> position
    for (size_t i = 0; i < order.size();) {
        bp_batch::Class k;
        k.item_lo = (int32_t)items.size();
        const int32_t u0 = order[i];
        const bool defers = bp_scan_defers(units[u0].qlen);
        k.packed = units[u0].n_members > 0;
        int warps = 0;
        for (; i < order.size(); ++i) {
            const int32_t ui = order[i];
            const BatchQuery& u = units[ui];
            if (ui != u0) {
                if ((u.n_members > 0) != k.packed || bp_scan_defers(u.qlen) != defers || own_warps(ui) != warps) break;
                const int w = bp_scan_warps(std::max(k.max_qlen, u.qlen), std::max(k.max_len, u.diag_len),
                                            std::max<int64_t>(k.max_entries, u.n_entries), e->smem_optin, k.packed);
                if (w != warps) break;
            }
            k.max_len = std::max(k.max_len, u.diag_len);
            k.max_qlen = std::max(k.max_qlen, u.qlen);
            k.max_entries = std::max<int64_t>(k.max_entries, u.n_entries);
            k.units.push_back(ui);
            if (ui == u0) warps = own_warps(ui);
            for (int32_t qi : unit_queries[ui]) k.est += queries[qi]->hits_per_residue;
            for (int32_t c = 0; c < n_chunks; ++c) {
                for (int32_t qi : unit_queries[ui]) item_pos[(size_t)qi * n_chunks + c] = (int32_t)items.size();
                WorkItem w{};
                w.qid = ui;
                w.first = b->chunk_first[c];
                w.count = b->chunk_first[c + 1] - b->chunk_first[c];
                bp_long_slice(db->h_long, w.first, w.count, &w.long_first, &w.n_long);
                items.push_back(w);
            }
        }
        k.item_hi = (int32_t)items.size();
        b->classes.push_back(k);
    }
    b->n_items = (int32_t)items.size();
    // per-CTA queues of each class (indices local to the class)
    const int grid_max = o.ctas > 0 ? o.ctas : e->sm_count;
    std::vector<int32_t> local_queue(items.size(), -1);
    std::vector<int32_t> qoff(1, 0), qitems;
    b->queue_cost.clear();
    for (bp_batch::Class& k : b->classes) {
        const int32_t nk = k.item_hi - k.item_lo;
        k.grid = std::max(1, std::min(grid_max, nk));
        k.queue_lo = (int32_t)qoff.size() - 1;
        std::vector<std::vector<int32_t>> qs(k.grid);
        std::vector<double> load(k.grid, 0.0);
        if (o.schedule == BP_SCHED_COST_ORDER) {
            // one cursor for the class over its items, longest predicted first
            // (ties in index order); the CTAs take them dynamically
            std::vector<int32_t> loc(nk);
            std::iota(loc.begin(), loc.end(), 0);
            std::vector<float> cost(nk, 0.f);
            for (int32_t qi = 0; qi < n_queries; ++qi)
                for (int32_t c = 0; c < n_chunks; ++c) {
                    const int32_t pos = item_pos[(size_t)qi * n_chunks + c];
                    if (pos >= k.item_lo && pos < k.item_hi)
                        cost[pos - k.item_lo] += std::max(0.f, o.item_costs[(size_t)qi * n_chunks + c]);
                }
            std::stable_sort(loc.begin(), loc.end(), [&](int32_t x, int32_t y) { return cost[x] > cost[y]; });
            k.order_lo = (int32_t)qitems.size();
            qitems.insert(qitems.end(), loc.begin(), loc.end());
            qoff.push_back(qoff.back() + nk);
            b->queue_cost.push_back(0.0);
            continue;
        }
        if (o.schedule == BP_SCHED_COSTS) {
            // longest predicted item first, into the least loaded queue; each
            // queue then runs its items in order, query by query, so a CTA
            // reloads a query's table only when the query changes
            std::vector<int32_t> loc(nk);
            std::iota(loc.begin(), loc.end(), 0);
            std::vector<float> cost(nk, 0.f);
            for (int32_t qi = 0; qi < n_queries; ++qi)
                for (int32_t c = 0; c < n_chunks; ++c) {
                    const int32_t pos = item_pos[(size_t)qi * n_chunks + c];
                    if (pos >= k.item_lo && pos < k.item_hi)   // a packed item costs its queries' sum
                        cost[pos - k.item_lo] += std::max(0.f, o.item_costs[(size_t)qi * n_chunks + c]);
                }
            std::stable_sort(loc.begin(), loc.end(), [&](int32_t x, int32_t y) { return cost[x] > cost[y]; });
            typedef std::pair<double, int> Load;
            std::priority_queue<Load, std::vector<Load>, std::greater<Load>> heap;
            for (int c = 0; c < k.grid; ++c) heap.push(Load(0.0, c));
            for (int32_t i : loc) {
                Load l = heap.top();
                heap.pop();
                qs[l.second].push_back(i);
                l.first += cost[i];
                load[l.second] = l.first;
                heap.push(l);
            }
            for (auto& q : qs) std::sort(q.begin(), q.end());
        } else {
            for (int32_t i = 0; i < nk; ++i) qs[i % k.grid].push_back(i);
        }
        for (int c = 0; c < k.grid; ++c) {
            qoff.push_back(qoff.back() + (int32_t)qs[c].size());
            qitems.insert(qitems.end(), qs[c].begin(), qs[c].end());
            b->queue_cost.push_back(load[c]);
            if (o.schedule != BP_SCHED_DYNAMIC)
                for (int32_t li : qs[c]) local_queue[(size_t)(k.item_lo + li)] = k.queue_lo + c;
        }
    }
    b->item_queue.resize(item_pos.size());
    for (size_t i = 0; i < item_pos.size(); ++i) b->item_queue[i] = local_queue[(size_t)item_pos[i]];
    // record capacity: 2.5e-4 HSPs per expected word hit (about 1e-4 are
    // reported on background sequence with homologs planted at 0.2-0.5 %);
    // grown and re-run on overflow, then kept for later runs
    const double span_res = (double)(db->h_off[s1] - db->h_off[s0]);
    b->cap = (uint32_t)std::min<double>(1 << 28, std::max(65536.0, 2.5e-4 * hits_sum * span_res));
    cudaStream_t es = e->stream;
    cudaError_t err = cudaMallocAsync((void**)&b->d_queries, std::max<size_t>(1, units.size()) * sizeof(BatchQuery), es);
    if (err == cudaSuccess) err = cudaMallocAsync((void**)&b->d_items, std::max<size_t>(1, items.size()) * sizeof(WorkItem), es);
    if (err == cudaSuccess) err = cudaMallocAsync((void**)&b->d_queue_off, qoff.size() * sizeof(int32_t), es);
    if (err == cudaSuccess) err = cudaMallocAsync((void**)&b->d_queue_items, std::max<size_t>(1, qitems.size()) * sizeof(int32_t), es);
    if (err == cudaSuccess) err = cudaMallocAsync((void**)&b->d_counters, (size_t)std::max<int64_t>(b->nseg, 1) * 3 * sizeof(int32_t), es);
    if (err == cudaSuccess) err = cudaMallocAsync((void**)&b->d_hsp_off, ((size_t)b->nseg + 1) * sizeof(int64_t), es);
    if (err == cudaSuccess && !(b->h_count = bp_pinned_get(e))) err = cudaErrorMemoryAllocation;
    // the host tables are pageable: copy synchronously with respect to the host
    // (cudaMemcpyAsync from pageable memory returns once staged)
    if (err == cudaSuccess && !units.empty())
        err = cudaMemcpyAsync(b->d_queries, units.data(), units.size() * sizeof(BatchQuery), cudaMemcpyHostToDevice, es);
    if (err == cudaSuccess && !items.empty())
        err = cudaMemcpyAsync(b->d_items, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice, es);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(b->d_queue_off, qoff.data(), qoff.size() * sizeof(int32_t), cudaMemcpyHostToDevice, es);
    if (err == cudaSuccess && !qitems.empty())
        err = cudaMemcpyAsync(b->d_queue_items, qitems.data(), qitems.size() * sizeof(int32_t), cudaMemcpyHostToDevice, es);
    if (err != cudaSuccess) {
        bp_batch_destroy(b);
        return bp_set_cuda_error(e, err, "bp_search_batch: allocate");
    }
    bp_status st = prepare(b);
    b->wait_first = after;
    if (st == BP_OK) st = launch_batch(b);
    if (st != BP_OK) {
        bp_batch_destroy(b);
        return st;
    }
    *out = b;
    return BP_OK;
}

extern "C" {

bp_status bp_batch_run(bp_batch* b) {
    if (!b) return BP_ERR_INVALID;
    bp_engine* e = b->e;
    CKB(cudaSetDevice(e->device), "cudaSetDevice");
    return launch_batch(b);
}

bp_status bp_batch_wait(bp_batch* b) {
    if (!b) return BP_ERR_INVALID;
    bp_engine* e = b->e;
    if (b->n_hsps >= 0) return BP_OK;
    CKB(cudaSetDevice(e->device), "cudaSetDevice");
    for (int attempt = 0; attempt < 4; ++attempt) {
        CKB(cudaStreamSynchronize(e->stream), "batched search");
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, b->ev0, b->ev1) == cudaSuccess) {
            b->last_ms = ms;
            e->last_scan_ms = ms;
        }
        cudaGetLastError();
        const uint32_t count = b->h_count[0];
        if (count <= b->cap) {
            b->n_hsps = count;
            return BP_OK;
        }
        b->cap = count + count / 4 + 1024;
        bp_status st = prepare(b);
        if (st == BP_OK && b->opt.use_graph) st = capture(b);   // buffers moved: capture again
        if (st == BP_OK) st = launch_batch(b);
        if (st != BP_OK) {
            cudaStreamSynchronize(e->stream);   // nothing of the batch left running
            cudaGetLastError();
            return st;
        }
    }
    cudaStreamSynchronize(e->stream);
    cudaGetLastError();
    return bp_set_error(e, BP_ERR_CUDA, "bp_batch_wait: record buffer kept overflowing");
}

int64_t bp_batch_hsps(const bp_batch* b) { return b ? b->n_hsps : -1; }
float bp_batch_last_scan_ms(const bp_batch* b) { return b ? b->last_ms : 0.f; }
int32_t bp_batch_items(const bp_batch* b) { return b ? b->n_items : 0; }

bp_status bp_batch_copy_query(bp_batch* b, int32_t qi, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                              int64_t* n_hsps) {
    if (!b || qi < 0 || qi >= b->nq) return BP_ERR_INVALID;
    bp_status st = bp_batch_wait(b);
    if (st != BP_OK) return st;
    bp_engine* e = b->e;
    const size_t s0 = (size_t)qi * b->n;
    int64_t lo = 0, hi = 0;
    CKB(cudaMemcpy(&lo, b->d_hsp_off + s0, sizeof(int64_t), cudaMemcpyDeviceToHost), "copy offsets");
    CKB(cudaMemcpy(&hi, b->d_hsp_off + s0 + b->n, sizeof(int64_t), cudaMemcpyDeviceToHost), "copy offsets");
    if (n_hsps) *n_hsps = hi - lo;
    if (counters && b->n > 0)
        CKB(cudaMemcpy(counters, b->d_counters + 3 * s0, (size_t)b->n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost),
            "copy counters");
    if (hsp_off) {
        CKB(cudaMemcpy(hsp_off, b->d_hsp_off + s0, ((size_t)b->n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost),
            "copy offsets");
        for (int32_t i = 0; i <= b->n; ++i) hsp_off[i] -= lo;
    }
    if (hsps && hi > lo)
        CKB(cudaMemcpy(hsps, b->d_hsps + lo, (size_t)(hi - lo) * sizeof(bp_hsp), cudaMemcpyDeviceToHost), "copy hsps");
    return BP_OK;
}

bp_status bp_batch_digest(bp_batch* b, int32_t qi, uint64_t out[2]) {
    if (!b || qi < 0 || qi >= b->nq || !out) return BP_ERR_INVALID;
    bp_status st = bp_batch_wait(b);
    if (st != BP_OK) return st;
    const size_t s0 = (size_t)qi * b->n;
    return bp_digest_range(b->e, b->e->stream, b->d_counters + 3 * s0, b->n, b->d_hsp_off + s0, b->d_hsps, out);
}

}  // extern "C"

bp_status bp_batch_digest_sums(bp_batch* b, int32_t qi, bp_engine* e, cudaStream_t st, int64_t first,
                               int64_t rec_base, bool last, uint64_t sums[2]) {
    if (!b || qi < 0 || qi >= b->nq || !sums) return BP_ERR_INVALID;
    bp_status s = bp_batch_wait(b);
    if (s != BP_OK) return s;
    if (!e) {
        e = b->e;
        st = e->stream;
    }
    const size_t s0 = (size_t)qi * b->n;
    return bp_digest_sums(e, st, b->d_counters + 3 * s0, b->n, b->d_hsp_off + s0, b->d_hsps, first, rec_base, last,
                          sums);
}

extern "C" {

bp_status bp_batch_queue_costs(const bp_batch* b, double* costs, int32_t* n_queues) {
    if (!b || !n_queues) return BP_ERR_INVALID;
    *n_queues = (int32_t)b->queue_cost.size();
    if (costs) memcpy(costs, b->queue_cost.data(), b->queue_cost.size() * sizeof(double));
    return BP_OK;
}

bp_status bp_batch_item_queues(const bp_batch* b, int32_t* queue_of_item) {
    if (!b || !queue_of_item) return BP_ERR_INVALID;
    memcpy(queue_of_item, b->item_queue.data(), b->item_queue.size() * sizeof(int32_t));
    return BP_OK;
}

void bp_batch_destroy(bp_batch* b) {
    if (!b) return;
    bp_engine* e = b->e;
    if (e) {
        cudaSetDevice(e->device);
        cudaStreamSynchronize(e->stream);
    }
    bp_batch_destroy_finished(b);
}

}  // extern "C"

// The batch's work has completed (bp_batch_wait returned): its memory goes
// back stream-ordered without waiting for whatever the engine's stream runs
// now.
void bp_batch_destroy_finished(bp_batch* b) {
    if (!b) return;
    bp_engine* e = b->e;
    if (e) cudaSetDevice(e->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (void* p : {(void*)b->d_queries, (void*)b->d_items, (void*)b->d_queue_off, (void*)b->d_queue_items,
                    (void*)b->d_counters, (void*)b->d_hsp_off, (void*)b->d_hsps, (void*)b->d_keys, (void*)b->d_recs,
                    (void*)b->d_fill, (void*)b->d_blocksums, (void*)b->d_counts})
        if (p && e) cudaFreeAsync(p, e->stream);
    for (void* p : b->pack_mem)
        if (p && e) cudaFreeAsync(p, e->stream);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    for (cudaEvent_t ev : b->ev_join) cudaEventDestroy(ev);
    for (cudaStream_t st : b->side) cudaStreamDestroy(st);
    if (e) bp_pinned_put(e, b->h_count);
    cudaGetLastError();
    delete b;
}

// ---- cost prediction and autotuning ---------------------------------------

extern "C" {

bp_status bp_batch_predict_costs(bp_engine* e, bp_mlp* model, const float* weights, const bp_db* db,
                                 const bp_query* const* queries, int32_t n_queries, const int32_t* chunk_first,
                                 int32_t n_chunks, float planted_density, float* costs) {
    if (!e || !model || !weights || !db || !chunk_first || !costs || n_queries < 0 || n_chunks < 0)
        return BP_ERR_INVALID;
    if ((size_t)n_queries * n_chunks == 0) return BP_OK;
    // predict on base chunks when the chunks are unions of them, else directly
    std::vector<int32_t> base;
    plan_direct(db, chunk_first[0], chunk_first[n_chunks], kBaseChunk, base);
    std::vector<int32_t> owner(base.size() - 1);
    bool aligned = true;
    for (size_t i = 0, c = 0; i + 1 < base.size(); ++i) {
        while (c < (size_t)n_chunks && chunk_first[c + 1] <= base[i]) ++c;
        if (c >= (size_t)n_chunks || base[i + 1] > chunk_first[c + 1]) { aligned = false; break; }
        owner[i] = (int32_t)c;
    }
    const int32_t* f = aligned ? base.data() : chunk_first;
    const int32_t nf = aligned ? (int32_t)base.size() - 1 : n_chunks;
    const size_t n = (size_t)n_queries * nf;
    std::vector<float> X(n * BP_COST_FEATURES), Y(n * 2);
    bp_status st = bp_batch_features(e, db, queries, n_queries, f, nf, planted_density, X.data());
    if (st == BP_OK) st = bp_mlp_predict(model, X.data(), (int32_t)n, Y.data());
    if (st != BP_OK) return st;
    std::vector<double> acc((size_t)n_queries * n_chunks, 0.0);
    for (size_t i = 0; i < n; ++i) {
        const double res = expm1((double)X[i * BP_COST_FEATURES + 2]);
        const double hits = expm1(std::max(0.0, (double)Y[2 * i]));
        const double ext = expm1(std::max(0.0, (double)Y[2 * i + 1]));
        const size_t q = i / nf, c = i % nf;
        acc[q * n_chunks + (aligned ? owner[c] : c)] += weights[0] * res + weights[1] * hits + weights[2] * ext;
    }
    for (size_t i = 0; i < acc.size(); ++i) costs[i] = (float)acc[i];
    return BP_OK;
}

void bp_autotune_options_default(bp_autotune_options* o) {
    memset(o, 0, sizeof(*o));
    o->pack_sizes = nullptr;
    o->schedules_mask = (1 << BP_SCHED_DYNAMIC) | (1 << BP_SCHED_STATIC) | (1 << BP_SCHED_COSTS) |
                        (1 << BP_SCHED_COST_ORDER);
    o->reps = 2;
}

// Times every candidate (chunk size x warp cap x schedule) on a sample of the
// subjects with the whole query set, and returns the fastest as *best.  The
// cost schedule is tried only with a model; its costs for the full run come
// from bp_batch_predict_costs with the chosen chunk size.
bp_status bp_batch_autotune(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                            const bp_autotune_options* opt, bp_batch_options* best, bp_autotune_trial* trials,
                            int32_t trials_cap, int32_t* n_trials) {
    if (!e || !db || !queries || n_queries < 1 || !best) return bp_set_error(e, BP_ERR_INVALID, "bp_batch_autotune");
    bp_autotune_options o;
    if (opt) o = *opt;
    else bp_autotune_options_default(&o);
    static const int32_t kChunks[] = {1 << 16, 1 << 18, 1 << 20, 1 << 22};
    static const int32_t kWarps[] = {0, 16};
    static const int32_t kPacks[] = {0, 512, 1024};
    const int32_t* chunks = o.chunk_sizes ? o.chunk_sizes : kChunks;
    const int n_chunk_sizes = o.chunk_sizes ? o.n_chunk_sizes : 4;
    const int32_t* warps = o.warp_caps ? o.warp_caps : kWarps;
    const int n_warp_caps = o.warp_caps ? o.n_warp_caps : 2;
    const int32_t* packs = o.pack_sizes ? o.pack_sizes : kPacks;
    const int n_pack_sizes = o.pack_sizes ? o.n_pack_sizes : 3;
    const int32_t sample = o.sample_subjects > 0 ? std::min(o.sample_subjects, db->n) : std::max(1, db->n / 16);
    const int reps = std::max(1, o.reps);
    bp_batch_options_default(best);
    float best_ms = 1e30f;
    int32_t nt = 0;
    std::vector<float> costs;
    int32_t costs_chunk = -1;
    auto trial = [&](int32_t chunk, int32_t pack, int sched, int32_t max_warps, int32_t plain = 0) -> bp_status {
        bp_batch_options bo;
        bp_batch_options_default(&bo);
        bo.chunk_residues = chunk;
        bo.pack_residues = pack;
        bo.plain_unpacked = plain;
        bo.schedule = sched;
        bo.max_warps = max_warps;
        bo.subject_first = 0;
        bo.subject_count = sample;
        if (sched == BP_SCHED_COSTS || sched == BP_SCHED_COST_ORDER) {
            if (costs_chunk != chunk) {
                std::vector<int32_t> first;
                plan_chunks(db, 0, sample, chunk, first);
                costs.assign((size_t)n_queries * (first.size() - 1), 0.f);
                bp_status st = bp_batch_predict_costs(e, o.model, o.cost_weights, db, queries, n_queries,
                                                      first.data(), (int32_t)first.size() - 1, o.planted_density,
                                                      costs.data());
                if (st != BP_OK) return st;
                costs_chunk = chunk;
            }
            bo.item_costs = costs.data();
        }
        bp_batch* b = nullptr;
        bp_status st = bp_search_batch(e, db, queries, n_queries, &bo, &b);
        if (st == BP_OK) st = bp_batch_wait(b);
        float ms = 1e30f;
        for (int r = 0; r < reps && st == BP_OK; ++r) {
            st = bp_batch_run(b);
            if (st == BP_OK) st = bp_batch_wait(b);
            if (st == BP_OK) ms = std::min(ms, b->last_ms);
        }
        bp_batch_destroy(b);
        if (st != BP_OK) return st;
        if (trials && nt < trials_cap) {
            trials[nt].chunk_residues = chunk;
            trials[nt].schedule = sched;
            trials[nt].max_warps = max_warps;
            trials[nt].ms = ms;
            trials[nt].pack_residues = pack;
            trials[nt].plain_unpacked = plain;
        }
        ++nt;
        if (ms < best_ms) {
            best_ms = ms;
            *best = bo;
            best->item_costs = nullptr;
            best->subject_first = 0;
            best->subject_count = -1;
        }
        return BP_OK;
    };
    // stage 1: chunk size x packing, dynamic schedule, all warps
    const int sched0 = (o.schedules_mask & (1 << BP_SCHED_DYNAMIC)) ? BP_SCHED_DYNAMIC
                       : (o.schedules_mask & (1 << BP_SCHED_STATIC)) ? BP_SCHED_STATIC : BP_SCHED_COSTS;
    if (sched0 == BP_SCHED_COSTS && !o.model) return bp_set_error(e, BP_ERR_INVALID, "bp_batch_autotune: no schedule");
    for (int ci = 0; ci < n_chunk_sizes; ++ci)
        for (int pi = 0; pi < n_pack_sizes; ++pi) {
            bp_status st = trial(chunks[ci], packs[pi], sched0, 0);
            if (st != BP_OK) return st;
        }
    // stage 2: the other schedules, then the warp caps, at the best chunk and packing
    const int32_t chunk = best->chunk_residues, pack = best->pack_residues;
    for (int sched = 0; sched <= BP_SCHED_COST_ORDER; ++sched) {
        const bool needs_model = sched == BP_SCHED_COSTS || sched == BP_SCHED_COST_ORDER;
        if (sched == sched0 || !(o.schedules_mask & (1 << sched)) || (needs_model && !o.model)) continue;
        bp_status st = trial(chunk, pack, sched, 0);
        if (st != BP_OK) return st;
    }
    const int sched = best->schedule;
    for (int wi = 0; wi < n_warp_caps; ++wi) {
        if (warps[wi] == 0) continue;
        bp_status st = trial(chunk, pack, sched, warps[wi]);
        if (st != BP_OK) return st;
    }
    // stage 3: the queries that are not packed as plain single-query scans
    {
        const bp_batch_options b0 = *best;
        bp_status st = trial(b0.chunk_residues, b0.pack_residues, b0.schedule, b0.max_warps, 1);
        if (st != BP_OK) return st;
    }
    if (n_trials) *n_trials = nt;
    return BP_OK;
}

}  // extern "C"

// ---- GPU/CPU co-scheduling -------------------------------------------------

extern "C" {

// The chunk index k that balances the device's share [0, k) against the CPU's
// share [k, n): minimises max(sum_{c<k} cost_c, cpu_factor * sum_{c>=k} cost_c),
// costs being device time per chunk and cpu_factor the CPU's time per unit of
// device time.  Replaces the reference's fixed GPU fraction of the OIDs
// (functions.cpp:125-149, :1059).
int32_t bp_cosched_split_costs(const double* chunk_costs, int32_t n_chunks, double cpu_factor) {
    if (!chunk_costs || n_chunks <= 0) return 0;
    if (!(cpu_factor > 0)) return n_chunks;                 // no CPU share
    double total = 0;
    for (int32_t c = 0; c < n_chunks; ++c) total += std::max(0.0, chunk_costs[c]);
    double gpu = 0, best = 1e300;
    int32_t best_k = n_chunks;
    for (int32_t k = 0; k <= n_chunks; ++k) {
        const double m = std::max(gpu, cpu_factor * (total - gpu));
        if (m < best) {
            best = m;
            best_k = k;
        }
        if (k < n_chunks) gpu += std::max(0.0, chunk_costs[k]);
    }
    return best_k;
}

// The first subject the CPU should take when the device searches subjects
// [0, split) and the CPU the rest, from the cost model's predictions for these
// queries over 64Ki-residue chunks.
bp_status bp_cosched_split(bp_engine* e, bp_mlp* model, const float* weights, const bp_db* db,
                           const bp_query* const* queries, int32_t n_queries, float planted_density, double cpu_factor,
                           int32_t* split_subject) {
    if (!e || !model || !weights || !db || !queries || n_queries < 1 || !split_subject) return BP_ERR_INVALID;
    std::vector<int32_t> first;
    plan_direct(db, 0, db->n, kBaseChunk, first);
    const int32_t nc = (int32_t)first.size() - 1;
    if (nc == 0) {
        *split_subject = 0;
        return BP_OK;
    }
    std::vector<float> costs((size_t)n_queries * nc);
    bp_status st = bp_batch_predict_costs(e, model, weights, db, queries, n_queries, first.data(), nc,
                                          planted_density, costs.data());
    if (st != BP_OK) return st;
    std::vector<double> per_chunk(nc, 0.0);
    for (int32_t q = 0; q < n_queries; ++q)
        for (int32_t c = 0; c < nc; ++c) per_chunk[c] += costs[(size_t)q * nc + c];
    *split_subject = first[bp_cosched_split_costs(per_chunk.data(), nc, cpu_factor)];
    return BP_OK;
}

}  // extern "C"
