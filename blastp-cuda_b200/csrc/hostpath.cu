// bp_blastp_host: one search from host buffers to host buffers, with the
// database upload overlapped with the scan.
//
// The reference copies the whole database to the device and only then
// launches its kernel (gpu_blastp.cu:139-210).  Here the subjects are cut
// into chunks (8, 16, 32, then 64 MiB of residues); a copy stream uploads them one
// after the other, each followed by an event, and the engine stream checks
// and scans every chunk as soon as its event has fired, so the transfer of
// chunk k+1 runs under the scan of chunk k.
//
// Queries whose diagonal arrays take 16-bit entries (all but those of about
// 8,000 letters and more) are scanned by ONE streaming launch
// (scan_stream_kernel): it starts once the offsets are up and takes the
// subjects in order, each warp waiting (bounded) for its subject's chunk,
// whose arrival a 4-byte copy queued after the chunk's data announces.  No
// kernel runs on the upload stream, so the copies never wait for SMs the
// scan holds; chunks start on 128-byte boundaries of the device buffer;
// residue codes and offsets are checked by the scan itself.
//
// Otherwise each chunk gets its own scan launch.  The host checks only the chunk
// boundaries (they bound the copies); every subject's length is checked on
// the device, chunk by chunk, by the kernel that also lists the chunk's long
// subjects for the scan to take first, and a chunk whose check failed is not
// scanned.  Checks run on their own stream and consecutive chunks' scans on
// two streams, so a chunk's checks and its scan's first CTAs take the SMs
// that the previous scan's last subjects leave idle.  The query's table is
// built on the engine stream meanwhile.  All chunks write one set
// of per-subject counters and one record buffer (subject index = chunk start
// + index in the chunk), ordered once at the end; into pinned host memory
// each chunk's counters go back as soon as its scan ends.  Device buffers are
// grow-only and kept by the engine, so repeated calls allocate nothing once
// warm.
#include <string.h>

#include <algorithm>
#include <vector>

#include "bp_internal.h"

#define CKH(call, what)                                                   \
    do {                                                                  \
        cudaError_t _err = (call);                                        \
        if (_err != cudaSuccess) return bp_set_cuda_error(e, _err, what); \
    } while (0)

struct HostPath {
    cudaStream_t copy = nullptr;        // uploads
    cudaStream_t back = nullptr;        // per-chunk counter read-back
    cudaStream_t checks = nullptr;      // per-chunk residue and offsets checks
    cudaStream_t scan2 = nullptr;       // odd chunks' scans (even ones: the engine stream)
    cudaEvent_t fork = nullptr, join = nullptr;
    std::vector<cudaEvent_t> ready;     // one per chunk slot: uploaded
    std::vector<cudaEvent_t> checked;   // one per chunk slot: checked
    std::vector<cudaEvent_t> scanned;   // one per chunk slot: scanned
    uint8_t* d_res = nullptr;
    size_t res_cap = 0;
    int64_t* d_off = nullptr;
    size_t off_cap = 0;
    int32_t* d_counters = nullptr;
    int64_t* d_hsp_off = nullptr;
    size_t subj_cap = 0;
    // [0] records, [1] bad residue, [2] bad offsets, [3] a streaming chunk
    // stalled, [4 .. 4 + chunks) chunk cursors (streaming: [4] only), then the
    // chunks' long-subject counts
    uint32_t* d_words = nullptr;
    size_t words_cap = 0;
    uint32_t* h_words = nullptr;        // pinned read-back
    int32_t* d_long = nullptr;          // chunk k's long subjects at d_long + its first subject
    size_t long_cap = 0;
    // streaming: chunk tables (first subjects, first offsets, device bases),
    // arrival flags, and the value this call's flag copies write
    uint8_t* d_tab = nullptr;
    size_t tab_cap = 0;
    uint8_t* h_tab = nullptr;
    size_t h_tab_cap = 0;
    uint32_t* d_flags = nullptr;
    size_t flags_cap = 0;
    uint32_t* h_gen = nullptr;
    uint32_t gen = 0;
    cudaEvent_t tabs_ready = nullptr;
};

namespace {

constexpr int64_t kChunkResidues = (int64_t)64 << 20;
// Streaming launch: chunks of this many residues throughout.  A chunk costs
// only its arrival flag, and the scan, which runs about as fast as the
// transfer, trails it by at most one chunk.
constexpr int64_t kStreamChunkResidues = (int64_t)8 << 20;

// First index t in [lo, hi] with off[t] > limit, for non-decreasing off; on
// any other array still some index in [lo, hi] (the caller checks the
// boundaries it gets before trusting them).
int32_t first_above(const int64_t* off, int32_t lo, int32_t hi, int64_t limit) {
    while (lo < hi) {
        const int32_t mid = lo + (hi - lo) / 2;
        if (off[mid] <= limit) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}


bool is_pinned(const void* p) {
    cudaPointerAttributes pa;
    const bool pinned = p && cudaPointerGetAttributes(&pa, p) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    return pinned;
}

template <class T>
cudaError_t grow_buf(T** p, size_t* cap, size_t need) {
    if (*p && *cap >= need) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    const size_t n = std::max(need, *cap + *cap / 2);
    cudaError_t err = cudaMalloc((void**)p, n * sizeof(T));
    *cap = err == cudaSuccess ? n : 0;
    return err;
}

}  // namespace

void bp_host_path_free(bp_engine* e) {
    HostPath* h = e->host_path;
    if (!h) return;
    for (cudaStream_t s : {h->copy, h->back, h->checks, h->scan2})
        if (s) cudaStreamSynchronize(s);
    for (cudaEvent_t ev : h->ready) cudaEventDestroy(ev);
    for (cudaEvent_t ev : h->checked) cudaEventDestroy(ev);
    for (cudaEvent_t ev : h->scanned) cudaEventDestroy(ev);
    for (cudaEvent_t ev : {h->fork, h->join})
        if (ev) cudaEventDestroy(ev);
    for (cudaStream_t s : {h->copy, h->back, h->checks, h->scan2})
        if (s) cudaStreamDestroy(s);
    cudaFree(h->d_res);
    cudaFree(h->d_off);
    cudaFree(h->d_counters);
    cudaFree(h->d_hsp_off);
    cudaFree(h->d_words);
    cudaFree(h->d_long);
    cudaFree(h->d_tab);
    cudaFree(h->d_flags);
    if (h->h_words) cudaFreeHost(h->h_words);
    if (h->h_tab) cudaFreeHost(h->h_tab);
    if (h->h_gen) cudaFreeHost(h->h_gen);
    if (h->tabs_ready) cudaEventDestroy(h->tabs_ready);
    delete h;
    e->host_path = nullptr;
}

extern "C" bp_status bp_blastp_host(bp_engine* e, const uint8_t* query, int32_t qlen, const bp_params* p,
                                    const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                                    int32_t n_subjects, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                                    int64_t hsp_cap, int64_t* n_hsps) {
    if (!e || !offsets || n_subjects < 0 || n_residues < 0 || (n_residues > 0 && !residues) || !p ||
        (qlen > 0 && !query) || qlen < 0)
        return bp_set_error(e, BP_ERR_INVALID, "bp_blastp_host: bad argument");
    if (offsets[0] != 0 || offsets[n_subjects] != n_residues)
        return bp_set_error(e, BP_ERR_INVALID, "bp_blastp_host: offsets must run from 0 to n_residues");
    CKH(cudaSetDevice(e->device), "cudaSetDevice");
    // streaming: one launch for every chunk (16-bit diagonal entries, residues
    // in pinned memory, so that every copy is queued before the launch)
    const bool pinned = is_pinned(residues);
    const bool streaming = pinned && n_subjects > 0 && bp_scan_streams(bp_diag_len(qlen, p->window));
    // chunks of whole subjects: streaming, kStreamChunkResidues each;
    // otherwise 8 MiB, 16, 32, then 64 MiB of residues, so the first scan
    // starts after a short upload and later launches stay few
    std::vector<int32_t> cf(1, 0);
    int64_t chunk = streaming ? kStreamChunkResidues : kChunkResidues / 8;
    while (cf.back() < n_subjects) {
        const int32_t s = cf.back();
        const int64_t limit = offsets[s] + chunk;
        if (!streaming) chunk = std::min(kChunkResidues, chunk * 2);
        const int32_t t = first_above(offsets, s + 1, n_subjects + 1, limit) - 1;
        cf.push_back(std::max(t, s + 1));
    }
    const int n_chunks = (int)cf.size() - 1;
    // the chunk boundaries bound every copy: they must be in order and in
    // range before anything is queued (every subject is checked on the device)
    for (int k = 0; k < n_chunks; ++k)
        if (offsets[cf[k]] < 0 || offsets[cf[k + 1]] < offsets[cf[k]] || offsets[cf[k + 1]] > n_residues)
            return bp_set_error(e, BP_ERR_INVALID, "bp_blastp_host: offsets must be non-decreasing, subjects < 2^29");
    if (!e->host_path) e->host_path = new HostPath();
    HostPath* h = e->host_path;
    if (!h->copy) CKH(cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!h->back) CKH(cudaStreamCreateWithFlags(&h->back, cudaStreamNonBlocking), "cudaStreamCreate");
    // whichever way this call returns, no copy is still reading or writing
    // the caller's buffers afterwards
    struct CopiesDone {
        HostPath* h;
        ~CopiesDone() {
            cudaStreamSynchronize(h->copy);
            cudaStreamSynchronize(h->back);
        }
    } copies_done{h};
    if (!h->checks) CKH(cudaStreamCreateWithFlags(&h->checks, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!h->scan2) CKH(cudaStreamCreateWithFlags(&h->scan2, cudaStreamNonBlocking), "cudaStreamCreate");
    if (!h->fork) CKH(cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming), "cudaEventCreate");
    if (!h->join) CKH(cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming), "cudaEventCreate");
    if (!h->h_words) CKH(cudaMallocHost((void**)&h->h_words, 4 * sizeof(uint32_t)), "cudaMallocHost");
    while ((int)h->ready.size() < n_chunks) {
        cudaEvent_t ev = nullptr;
        CKH(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        h->ready.push_back(ev);
        CKH(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        h->checked.push_back(ev);
        CKH(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        h->scanned.push_back(ev);
    }
    // streaming: chunk k's residues at device offset base[k], 128-byte aligned
    std::vector<int64_t> base(n_chunks, 0);
    size_t res_bytes = (size_t)((n_residues + 15) & ~15LL) + 32;
    if (streaming) {
        int64_t at = 0;
        for (int k = 0; k < n_chunks; ++k) {
            base[k] = at;
            at = (at + (offsets[cf[k + 1]] - offsets[cf[k]]) + 127) & ~127LL;
        }
        res_bytes = (size_t)at + 256;
    } else {
        for (int k = 0; k < n_chunks; ++k) base[k] = offsets[cf[k]];
    }
    CKH(grow_buf(&h->d_res, &h->res_cap, res_bytes), "cudaMalloc(database)");
    CKH(grow_buf(&h->d_off, &h->off_cap, (size_t)n_subjects + 1), "cudaMalloc(offsets)");
    if (h->subj_cap < (size_t)n_subjects + 1) {
        cudaFree(h->d_counters);
        cudaFree(h->d_hsp_off);
        h->d_counters = nullptr;
        h->d_hsp_off = nullptr;
        h->subj_cap = 0;
        const size_t n = (size_t)n_subjects + 1;
        CKH(cudaMalloc((void**)&h->d_counters, n * 3 * sizeof(int32_t)), "cudaMalloc(counters)");
        CKH(cudaMalloc((void**)&h->d_hsp_off, n * sizeof(int64_t)), "cudaMalloc(offsets)");
        h->subj_cap = n;
    }
    CKH(grow_buf(&h->d_words, &h->words_cap, 4 + 2 * (size_t)n_chunks), "cudaMalloc(words)");
    CKH(grow_buf(&h->d_long, &h->long_cap, (size_t)std::max(n_subjects, 1)), "cudaMalloc(long subjects)");
    // uploads: from pinned memory every chunk is queued now, so the transfers
    // start under the table build; from pageable memory each copy call returns
    // only once staged, so those copies are interleaved with the scans below
    // (chunked launches only: each chunk's counters go back as its scan ends)
    const bool counters_pinned = !streaming && counters && n_subjects > 0 && is_pinned(counters);
    const int32_t drop_flag = e->drop_flag_chunk;   // fault injection: consumed by this call
    e->drop_flag_chunk = -1;
    auto upload = [&](int k) -> cudaError_t {
        const int64_t lo = offsets[cf[k]], hi = offsets[cf[k + 1]];
        cudaError_t err = cudaSuccess;
        if (hi > lo)
            err = cudaMemcpyAsync(h->d_res + base[k], residues + lo, (size_t)(hi - lo), cudaMemcpyHostToDevice,
                                  h->copy);
        if (err == cudaSuccess) err = cudaEventRecord(h->ready[k], h->copy);
        // streaming: the chunk's arrival flag, after its data in the same stream
        if (err == cudaSuccess && streaming && k != drop_flag)
            err = cudaMemcpyAsync(h->d_flags + k, h->h_gen, sizeof(uint32_t), cudaMemcpyHostToDevice, h->copy);
        return err;
    };
    // chunk tables: first offsets (n + 1), device bases (n), then first subjects (n + 1)
    const size_t tab_bytes = (size_t)(n_chunks + 1) * 8 + (size_t)n_chunks * 8 + (size_t)(n_chunks + 1) * 4;
    if (streaming) {
        // chunk tables and flags; the tables go up first on the upload stream
        // (a copy queued on another stream could wait behind the chunks)
        if (!h->h_gen) CKH(cudaMallocHost((void**)&h->h_gen, sizeof(uint32_t)), "cudaMallocHost");
        if (!h->tabs_ready) CKH(cudaEventCreateWithFlags(&h->tabs_ready, cudaEventDisableTiming), "cudaEventCreate");
        if (h->flags_cap < (size_t)n_chunks) {
            CKH(grow_buf(&h->d_flags, &h->flags_cap, (size_t)n_chunks), "cudaMalloc(flags)");
            CKH(cudaMemsetAsync(h->d_flags, 0, h->flags_cap * sizeof(uint32_t), e->stream), "memset(flags)");
            CKH(cudaStreamSynchronize(e->stream), "memset(flags)");
        }
        CKH(grow_buf(&h->d_tab, &h->tab_cap, tab_bytes), "cudaMalloc(chunk tables)");
        if (h->h_tab_cap < tab_bytes) {
            if (h->h_tab) cudaFreeHost(h->h_tab);
            h->h_tab = nullptr;
            h->h_tab_cap = 0;
            CKH(cudaMallocHost((void**)&h->h_tab, tab_bytes * 2), "cudaMallocHost");
            h->h_tab_cap = tab_bytes * 2;
        }
        int64_t* tlo = (int64_t*)h->h_tab;
        int64_t* tb = tlo + n_chunks + 1;
        int32_t* tf = (int32_t*)(tb + n_chunks);
        for (int k = 0; k <= n_chunks; ++k) {
            tf[k] = cf[k];
            tlo[k] = offsets[cf[k]];
            if (k < n_chunks) tb[k] = base[k];
        }
        *h->h_gen = ++h->gen;
        CKH(cudaMemcpyAsync(h->d_tab, h->h_tab, tab_bytes, cudaMemcpyHostToDevice, h->copy), "upload chunk tables");
    } else {
        CKH(cudaMemsetAsync(h->d_res + n_residues, 0, res_bytes - (size_t)n_residues, h->copy), "memset(pad)");
    }
    CKH(cudaMemcpyAsync(h->d_off, offsets, ((size_t)n_subjects + 1) * 8, cudaMemcpyHostToDevice, h->copy),
        "upload offsets");
    if (streaming) CKH(cudaEventRecord(h->tabs_ready, h->copy), "cudaEventRecord");
    if (pinned)
        for (int k = 0; k < n_chunks; ++k) CKH(upload(k), "upload residues");
    const int32_t long_min = bp_long_threshold(n_residues, n_subjects);
    // the query table (it synchronises the engine stream), then the engine's
    // record scratch
    bp_query* q = nullptr;
    bp_status st = bp_query_create(e, query, qlen, p, &q);
    if (st != BP_OK) {
        cudaStreamSynchronize(h->copy);
        return st;
    }
    if (!bp_scan_fits(q->qlen, q->diag_len, q->n_entries, e->smem_optin)) {
        cudaStreamSynchronize(h->copy);
        bp_query_destroy(q);
        return bp_set_error(e, BP_ERR_TOO_LARGE, "bp_blastp_host: query too long for the diagonal array");
    }
    uint32_t cap = std::max<uint32_t>(e->rec_cap, 65536);
    size_t rc = e->rec_cap;
    CKH(grow_buf(&e->d_recs, &rc, cap), "cudaMalloc(records)");
    e->rec_cap = (uint32_t)rc;
    size_t fc = (size_t)e->fill_cap;
    CKH(grow_buf(&e->d_fill, &fc, (size_t)std::max(n_subjects, 1)), "cudaMalloc(fill)");
    e->fill_cap = (int32_t)fc;
    size_t bc = (size_t)e->blocksum_cap;
    CKH(grow_buf(&e->d_blocksums, &bc, (size_t)bp_order_blocksums_needed(n_subjects)), "cudaMalloc(sums)");
    e->blocksum_cap = (int32_t)bc;
    uint32_t* bad_res = h->d_words + 1;
    uint32_t* bad_off = h->d_words + 2;
    uint32_t* cursors = h->d_words + 4;
    int32_t* long_counts = (int32_t*)(h->d_words + 4 + n_chunks);
    CKH(cudaMemsetAsync(h->d_words, 0, (4 + 2 * (size_t)n_chunks) * sizeof(uint32_t), e->stream), "memset");
    if (streaming) {
        // one launch; it starts once the tables and offsets are up
        CKH(cudaStreamWaitEvent(e->stream, h->tabs_ready, 0), "cudaStreamWaitEvent");
        CKH(cudaEventRecord(e->ev_scan0, e->stream), "cudaEventRecord");
        ScanArgs a{};
        a.db = h->d_res;
        a.db_bytes = (int64_t)h->res_cap;
        a.db_off = h->d_off;
        a.first = 0;
        a.n = n_subjects;
        a.query = q->d_q;
        a.qlen = q->qlen;
        a.cells = q->d_cells;
        a.entries = q->d_entries;
        a.n_entries = (int32_t)q->n_entries;
        a.ctx = q->d_ctx;
        a.n_ctx = q->n_ctx;
        a.matrix = e->d_matrix;
        a.window = q->p.window;
        a.diag_len = q->diag_len;
        a.counters = h->d_counters;
        a.recs = e->d_recs;
        a.rec_cap = e->rec_cap;
        a.rec_count = h->d_words;
        a.cursor = cursors;
        a.error = bad_res;
        a.bad_off = bad_off;
        a.stalled = h->d_words + 3;
        a.n_chunks = n_chunks;
        a.chunk_lo = (const int64_t*)h->d_tab;
        a.chunk_base = a.chunk_lo + n_chunks + 1;
        a.chunk_first = (const int32_t*)(a.chunk_base + n_chunks);
        a.chunk_flag = h->d_flags;
        a.gen = h->gen;
        a.wait_ns = e->upload_wait_ns;   // a chunk later than this: the scan gives up
        CKH(bp_launch_scan_stream(e, e->stream, a), "streaming scan launch");
        CKH(cudaEventRecord(e->ev_scan1, e->stream), "cudaEventRecord");
    } else {
    // chunk k's checks and scan run on the engine stream behind its event
    CKH(cudaEventRecord(e->ev_scan0, e->stream), "cudaEventRecord");
    CKH(cudaEventRecord(h->fork, e->stream), "cudaEventRecord");
    CKH(cudaStreamWaitEvent(h->checks, h->fork, 0), "cudaStreamWaitEvent");
    CKH(cudaStreamWaitEvent(h->scan2, h->fork, 0), "cudaStreamWaitEvent");
    for (int k = 0; k < n_chunks; ++k) {
        const int64_t lo = offsets[cf[k]], hi = offsets[cf[k + 1]];
        if (!pinned) CKH(upload(k), "upload residues");
        CKH(cudaStreamWaitEvent(h->checks, h->ready[k], 0), "cudaStreamWaitEvent");
        CKH(bp_launch_check_residues(e, h->checks, h->d_res + lo, hi - lo, bad_res), "residue check");
        CKH(bp_launch_long_list(e, h->checks, h->d_off, cf[k], cf[k + 1] - cf[k], long_min, h->d_long + cf[k],
                                long_counts + k, bad_off),
            "offsets check");
        CKH(cudaEventRecord(h->checked[k], h->checks), "cudaEventRecord");
        cudaStream_t ss = (k & 1) ? h->scan2 : e->stream;
        CKH(cudaStreamWaitEvent(ss, h->checked[k], 0), "cudaStreamWaitEvent");
        ScanArgs a{};
        a.db = h->d_res;
        a.db_bytes = (int64_t)h->res_cap;
        a.db_off = h->d_off;
        a.first = cf[k];
        a.n = cf[k + 1] - cf[k];
        a.query = q->d_q;
        a.qlen = q->qlen;
        a.cells = q->d_cells;
        a.entries = q->d_entries;
        a.n_entries = (int32_t)q->n_entries;
        a.ctx = q->d_ctx;
        a.n_ctx = q->n_ctx;
        a.matrix = e->d_matrix;
        a.window = q->p.window;
        a.diag_len = q->diag_len;
        a.counters = h->d_counters;
        a.recs = e->d_recs;
        a.rec_cap = e->rec_cap;
        a.rec_count = h->d_words;
        a.cursor = cursors + k;
        a.error = bad_res;
        a.oid_base = cf[k];
        a.long_ids = h->d_long + cf[k];
        a.n_long_at = long_counts + k;
        a.long_min = long_min;
        a.abort_if = bad_off;
        CKH(bp_launch_scan_on(e, ss, a), "scan kernel launch");
        if (counters_pinned && cf[k + 1] > cf[k]) {
            // this chunk's counters are final: back to the host under the next scans
            CKH(cudaEventRecord(h->scanned[k], ss), "cudaEventRecord");
            CKH(cudaStreamWaitEvent(h->back, h->scanned[k], 0), "cudaStreamWaitEvent");
            CKH(cudaMemcpyAsync(counters + 3 * (int64_t)cf[k], h->d_counters + 3 * (int64_t)cf[k],
                                (size_t)(cf[k + 1] - cf[k]) * 12, cudaMemcpyDeviceToHost, h->back),
                "read counters");
        }
    }
    CKH(cudaEventRecord(h->join, h->scan2), "cudaEventRecord");
    CKH(cudaStreamWaitEvent(e->stream, h->join, 0), "cudaStreamWaitEvent");
    CKH(cudaEventRecord(e->ev_scan1, e->stream), "cudaEventRecord");
    }
    // records written and the residue check, then outputs sized by the records
    CKH(cudaMemcpyAsync(h->h_words, h->d_words, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream),
        "read counts");
    CKH(cudaStreamSynchronize(e->stream), "pipelined search");
    // every copy is done too (a scan that skipped a bad subject may not have
    // waited for its chunk): the caller may reuse its buffers on return
    CKH(cudaStreamSynchronize(h->copy), "pipelined search");
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, e->ev_scan0, e->ev_scan1) == cudaSuccess) e->last_scan_ms = ms;
    cudaGetLastError();
    const uint32_t recs = h->h_words[0];
    if (h->h_words[3]) {
        cudaStreamSynchronize(h->copy);
        bp_query_destroy(q);
        return bp_set_error(e, BP_ERR_TIMEOUT, "bp_blastp_host: a chunk of the upload did not arrive in time");
    }
    if (h->h_words[2]) {
        cudaStreamSynchronize(h->back);
        bp_query_destroy(q);
        return bp_set_error(e, BP_ERR_INVALID, "bp_blastp_host: offsets must be non-decreasing, subjects < 2^29");
    }
    if (h->h_words[1]) {
        cudaStreamSynchronize(h->back);
        bp_query_destroy(q);
        return bp_set_error(e, BP_ERR_INVALID, "bp_blastp_host: residue code >= 28");
    }
    if (recs > e->rec_cap) {
        // more HSPs than the record buffer held: the unpipelined path grows and re-runs
        cudaStreamSynchronize(h->back);
        bp_query_destroy(q);
        return bp_blastp_host_staged(e, query, qlen, p, residues, n_residues, offsets, n_subjects, counters, hsp_off,
                                     hsps, hsp_cap, n_hsps);
    }
    bp_hsp* d_hsps = nullptr;
    int32_t* d_keys = nullptr;
    CKH(cudaMallocAsync((void**)&d_hsps, (size_t)std::max<uint32_t>(recs, 1) * sizeof(bp_hsp), e->stream),
        "cudaMallocAsync(hsps)");
    CKH(cudaMallocAsync((void**)&d_keys, (size_t)std::max<uint32_t>(recs, 1) * sizeof(int32_t), e->stream),
        "cudaMallocAsync(keys)");
    CKH(bp_launch_order(e, n_subjects, h->d_counters, h->d_hsp_off, e->d_recs, e->rec_cap, h->d_words, e->d_fill,
                        d_hsps, d_keys, e->d_blocksums),
        "order kernels launch");
    if (n_hsps) *n_hsps = recs;
    cudaError_t err = cudaSuccess;
    if (counters && n_subjects > 0 && !counters_pinned)
        err = cudaMemcpyAsync(counters, h->d_counters, (size_t)n_subjects * 12, cudaMemcpyDeviceToHost, e->stream);
    if (err == cudaSuccess && hsp_off)
        err = cudaMemcpyAsync(hsp_off, h->d_hsp_off, ((size_t)n_subjects + 1) * 8, cudaMemcpyDeviceToHost, e->stream);
    if (hsps && (int64_t)recs > hsp_cap) st = bp_set_error(e, BP_ERR_TOO_LARGE, "bp_blastp_host: hsp_cap too small");
    else if (err == cudaSuccess && hsps && recs > 0)
        err = cudaMemcpyAsync(hsps, d_hsps, (size_t)recs * sizeof(bp_hsp), cudaMemcpyDeviceToHost, e->stream);
    cudaFreeAsync(d_hsps, e->stream);
    cudaFreeAsync(d_keys, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    const cudaError_t err_back = cudaStreamSynchronize(h->back);
    if (err == cudaSuccess) err = err_back;
    bp_query_destroy(q);
    if (err != cudaSuccess) return bp_set_cuda_error(e, err, "bp_blastp_host: results");
    return st;
}
