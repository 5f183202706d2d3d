// Internal declarations shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <vector>

#include "blastp_b200.h"

#define BP_NCELL 32768          // reference layout: 3 letters x 5 bits
#define BP_NC 19683             // compact layout: 27^3 words of letters 1..27
#define BP_WORD 3
#define BP_MROW 32              // device matrix row stride (28 used)
#define BP_MAX_PACK_MEMBERS 32  // queries per packed table

// One reported HSP before ordering: owning subject (relative to the search's
// first subject), its discovery key (index of the triggering word hit in the
// subject's hit stream) and the record itself.
struct HspRec {
    int32_t oid;
    int32_t key;
    bp_hsp h;
};

struct bp_engine {
    int device = 0;
    int sm_count = 0;
    int smem_optin = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_scan0 = nullptr, ev_scan1 = nullptr;
    uint64_t launches = 0;
    float last_scan_ms = 0.f;
    std::string err;
    int8_t* d_matrix = nullptr;          // int8 [28][32]
    // grow-only scratch shared by searches on this engine
    HspRec* d_recs = nullptr;
    uint32_t rec_cap = 0;
    uint32_t* d_counts = nullptr;        // [0] records written, [1] subject cursor, [2] error word
    int32_t* d_fill = nullptr;           // per-subject fill cursors
    int32_t fill_cap = 0;
    int64_t* d_blocksums = nullptr;
    int32_t blocksum_cap = 0;
    // pinned 4-word slots for per-search read-backs (cudaMallocHost is slow)
    uint32_t* h_pool = nullptr;
    std::vector<int> pool_free;
    std::mutex pool_mu;
    struct HostPath* host_path = nullptr;   // buffers and copy stream of bp_blastp_host
    // streaming host-to-host search: how long the scan waits for one upload
    // chunk, and (fault injection, one call) a chunk whose arrival flag is
    // not sent
    uint64_t upload_wait_ns = 20ull * 1000 * 1000 * 1000;
    int32_t drop_flag_chunk = -1;
    unsigned long long* d_digest = nullptr;   // result digests' two sums
};

// Frees bp_blastp_host's buffers (engine destruction).
void bp_host_path_free(bp_engine* e);
extern "C" bp_status bp_blastp_host_staged(bp_engine* e, const uint8_t* query, int32_t qlen, const bp_params* p,
                                           const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                                           int32_t n_subjects, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                                           int64_t hsp_cap, int64_t* n_hsps);
// Sets *bad (device word) when any of n residues is >= 28.
// Subjects [first, first + n): a length outside [0, 2^29] sets *bad; the
// indices of those of at least long_min residues are appended (in no
// particular order) to out, their number added to *count.
cudaError_t bp_launch_long_list(bp_engine* e, cudaStream_t stream, const int64_t* d_off, int32_t first, int32_t n,
                                int32_t long_min, int32_t* out, int32_t* count, uint32_t* bad);
cudaError_t bp_launch_check_residues(bp_engine* e, cudaStream_t stream, const uint8_t* d_res, int64_t n,
                                     uint32_t* d_bad);

// A pinned 4-word slot from the engine's pool (or a fresh pinned block when
// the pool is exhausted); returned with bp_pinned_put.
uint32_t* bp_pinned_get(bp_engine* e);
void bp_pinned_put(bp_engine* e, uint32_t* p);

struct bp_db {
    bp_engine* e = nullptr;
    uint8_t* d_res = nullptr;            // residues + 16 bytes of zero padding
    int64_t* d_off = nullptr;
    int32_t n = 0;
    int64_t nres = 0;
    std::vector<int64_t> h_off;          // host copy of the offsets (chunk planning)
    // subjects of at least long_min residues (ascending indices), scanned
    // first by every launch (see bp_long_subjects)
    std::vector<int32_t> h_long;
    int32_t* d_long = nullptr;
    int32_t long_min = 0;
    // chunk composition histograms of the last chunk plan asked for (the
    // residues never change, so a plan's histograms are computed once; a
    // server asks for the same plan on every batch)
    std::mutex hist_mu;
    std::vector<int32_t> hist_first;
    std::vector<uint32_t> hist;
};

struct bp_query {
    bp_engine* e = nullptr;
    uint8_t* d_q = nullptr;
    int32_t qlen = 0;
    uint32_t* d_cells = nullptr;         // BP_NC + 1 compact cell starts
    uint16_t* d_entries = nullptr;
    int64_t n_entries = 0;
    int32_t n_ctx = 1;
    int32_t* d_ctx = nullptr;            // n_ctx x {query_offset, x_dropoff, cutoff}
    bp_params p{};
    int32_t diag_len = 0;                // diagonal entries (query + window, see bp_diag_len)
    float hits_per_residue = 0.f;        // expected word hits per subject residue (background composition)
};

struct bp_result {
    bp_engine* e = nullptr;
    int32_t n = 0;
    int32_t* d_counters = nullptr;       // 3n
    int64_t* d_hsp_off = nullptr;        // n+1
    bp_hsp* d_hsps = nullptr;
    int32_t* d_keys = nullptr;
    uint32_t cap = 0;
    uint32_t* h_count = nullptr;         // pinned: [0] records written, [1] unused, [2] error word
    int64_t n_hsps = -1;
    // to re-run on overflow
    const bp_db* db = nullptr;
    const bp_query* q = nullptr;
    int32_t first = 0;
};

// Everything the scan kernel reads, by value.
struct ScanArgs {
    const uint8_t* db;
    int64_t db_bytes;           // readable bytes from db: the L2 prefetch of a subject stops there
    const int64_t* db_off;
    int32_t first;              // first subject
    int32_t n;                  // subjects to scan
    const uint8_t* query;
    int32_t qlen;
    const uint32_t* cells;      // BP_NC + 1 compact cell starts
    const uint16_t* entries;
    int32_t n_entries;
    const int32_t* ctx;
    int32_t n_ctx;
    const int8_t* matrix;       // [28][32]
    int32_t window;
    int32_t diag_len;           // diagonal array entries, >= qlen + window
    int32_t* counters;          // 3 per scanned subject
    HspRec* recs;
    uint32_t rec_cap;
    uint32_t* rec_count;
    uint32_t* cursor;           // subject cursor (chunks of 32)
    uint32_t* error;            // set when a bounded wait runs out
    int32_t oid_base;           // plain kernel: counters and records of subject i go to oid_base + i
    // longest first: the range's subjects of at least long_min residues
    // (absolute indices, ascending) are taken before the others, which then
    // skip them; n_long = 0: plain index order
    const int32_t* long_ids;
    int32_t n_long;
    int32_t long_min;
    const int32_t* n_long_at;   // when set, n_long is read from here (a list built on the device)
    const uint32_t* abort_if;   // when set and non-zero at launch, the kernel scans nothing
    // streaming (the host-to-host search's single launch): the range's
    // subjects arrive in n_chunks chunks while the kernel runs.  Chunk c holds
    // subjects [chunk_first[c], chunk_first[c+1]) of the range, whose offsets
    // span [chunk_lo[c], chunk_lo[c+1]); its residues start at db +
    // chunk_base[c] and are there once chunk_flag[c] == gen.  A subject whose
    // offsets leave its chunk sets *bad_off and is skipped; a residue code of
    // 28 or more sets *error; a chunk not there within wait_ns sets *stalled.
    int32_t n_chunks;
    const int32_t* chunk_first;
    const int64_t* chunk_lo;
    const int64_t* chunk_base;
    const uint32_t* chunk_flag;
    uint32_t gen;
    uint64_t wait_ns;
    uint32_t* bad_off;
    uint32_t* stalled;
    // packed tables (batched kernel): per query {id, offset, length, x-drop,
    // cutoff}, the query of every packed offset, and the segment stride
    const int32_t* members;
    const uint8_t* member_of;
    int32_t n_members;
    int32_t seg_stride;
};

// Batched form: one query of a batch, one work item, and the launch arguments.
// A unit of a batch: one query (seg_query = its index in the batch), or a
// packed table of several short queries laid end to end with `window`
// offsets between them (members: 5 int32 per query {index, offset, length,
// x-drop, cutoff}; member_of: the member of every packed offset).
struct BatchQuery {
    const uint8_t* query;
    const uint32_t* cells;
    const uint16_t* entries;
    const int32_t* ctx;
    int32_t qlen, n_entries, n_ctx, diag_len;
    const int32_t* members;
    const uint8_t* member_of;
    int32_t n_members, seg_query;
};
struct WorkItem {
    int32_t qid;            // query of the batch
    int32_t first, count;   // subjects [first, first+count)
    int32_t long_first;     // its long subjects: BatchArgs::long_ids[long_first .. long_first + n_long)
    int32_t n_long;
    int32_t pad[3];
};
struct BatchArgs {
    const uint8_t* db;
    const int64_t* db_off;
    int32_t n_subjects;     // segment stride: segment = query * n_subjects + (subject - subject_first)
    int32_t subject_first;
    const BatchQuery* queries;
    int32_t n_queries;
    const WorkItem* items;
    int32_t n_items;
    const int32_t* queue_off;     // per-CTA queues: items queue_items[queue_off[c] .. queue_off[c+1]) (or null);
                                  // item indices are relative to `items`
    const int32_t* queue_items;
    uint32_t* item_cursor;        // global cursor when queue_off is null
    const int32_t* cursor_order;  // when set, the cursor's k-th item is cursor_order[k] (else item k)
    const int8_t* matrix;
    int32_t window;
    int32_t* counters;            // 3 per segment
    HspRec* recs;
    uint32_t rec_cap;
    uint32_t* rec_count;
    const int32_t* long_ids;      // the database's long subjects (see WorkItem), and their threshold
    int32_t long_min;
};

// ---- host helpers ---------------------------------------------------------
// Database allocation (residues + 32 bytes of zero padding, offsets), and
// the finishing step: padding written, residue codes checked on the device.
extern "C" {
bp_status bp_db_alloc(bp_engine* e, int64_t n_residues, int32_t n_subjects, bp_db** out);
bp_status bp_db_finish(bp_engine* e, bp_db* db);
}
bp_status bp_set_cuda_error(bp_engine* e, cudaError_t err, const char* what);
// Longest-first order: a persistent launch ends when its last warp finishes
// its last subject, so subjects of at least twice the mean length (and at
// least 64 residues) go first.  Returns the threshold and appends the
// indices of [0, n) that reach it, ascending.
int32_t bp_long_subjects(const int64_t* off, int32_t n, std::vector<int32_t>* out);
int32_t bp_long_threshold(int64_t n_residues, int32_t n);
// The part [*lo, *lo + *cnt) of a sorted index list inside [first, first + n).
void bp_long_slice(const std::vector<int32_t>& ids, int32_t first, int32_t n, int32_t* lo, int32_t* cnt);
bp_status bp_set_error(bp_engine* e, bp_status s, const std::string& msg);
void bp_fill_matrix28(int8_t out[28 * 28]);
// Expected word hits per subject residue of a table under the Robinson &
// Robinson background, from its compact cell starts (BP_NC + 1).
float bp_expected_hits_per_residue(const uint32_t* cells);
int bp_cell_to_code15(int cell);
// Diagonal-array length for a query: qlen + window rounded up to 32, at
// least 128.  Any length >= qlen + window gives the same results (two live
// diagonals differ by less than qlen + window, so they never share an entry).
int bp_diag_len(int qlen, int window);
// Whether the scan kernel can take a query (its diagonal array must fit
// shared memory next to the table).
bool bp_scan_fits(int32_t qlen, int32_t diag_len, int64_t n_entries, int smem_optin);
// Warps per CTA the scan kernel runs with for such a query (0: does not fit),
// and whether it queues its extensions (the launch's longest query decides).
int bp_scan_warps(int32_t qlen, int32_t diag_len, int64_t n_entries, int smem_optin, bool packed);
bool bp_scan_defers(int32_t qlen);

// ---- launchers ------------------------------------------------------------
cudaError_t bp_launch_table_build(bp_engine* e, const uint8_t* d_q, int32_t qlen, int32_t threshold,
                                  uint32_t* d_cells, uint16_t* d_entries, uint32_t* d_counts_tmp, int pass);
cudaError_t bp_launch_scan(bp_engine* e, const ScanArgs& a);                       // on the engine stream
cudaError_t bp_launch_scan_on(bp_engine* e, cudaStream_t stream, const ScanArgs& a);
// The streaming scan (ScanArgs::n_chunks >= 1), for diagonal arrays of 16-bit
// entries (bp_scan_streams); cudaErrorNotSupported otherwise.
bool bp_scan_streams(int32_t diag_len);
cudaError_t bp_launch_scan_stream(bp_engine* e, cudaStream_t stream, const ScanArgs& a);
cudaError_t bp_launch_scan_batch(bp_engine* e, cudaStream_t stream, const BatchArgs& b, int32_t max_qlen,
                                 int32_t max_diag_len, int64_t max_entries, int grid, int max_warps, bool packed);
// Packed table of several queries: cells = sum of the members' cells,
// entries = each cell's member entries in member order, shifted by the
// member's offset (d_src: one PackSrc per member, device memory).
struct PackSrc {
    const uint32_t* cells;
    const uint16_t* entries;
    int32_t off;
    int32_t pad;
};
cudaError_t bp_launch_pack_table(bp_engine* e, cudaStream_t stream, const PackSrc* d_src, int n_members,
                                 uint32_t* d_counts_tmp, uint32_t* d_cells, uint16_t* d_entries);
cudaError_t bp_launch_order(bp_engine* e, int32_t n, const int32_t* d_counters, int64_t* d_hsp_off,
                            const HspRec* d_recs, uint32_t rec_cap, const uint32_t* d_rec_count,
                            int32_t* d_fill, bp_hsp* d_out, int32_t* d_keys, int64_t* d_blocksums);
int32_t bp_order_blocksums_needed(int32_t n);
// CSR offsets (n+1) from the second of every three int32 counters per
// subject (the ordering pass's first three launches), on `st`.
cudaError_t bp_launch_offsets(bp_engine* e, cudaStream_t st, int32_t n, const int32_t* d_counters, int64_t* d_off,
                              int32_t* d_fill, int64_t* d_blocksums);
bp_status bp_run_search(bp_engine* e, bp_result* r);
// Grows the engine's search scratch (record buffer, fill cursors, block sums)
// to at least these sizes now: growing later synchronises the device.
bp_status bp_engine_reserve(bp_engine* e, int32_t n_subjects, size_t records);
// Digest of one query's result in device memory: counters (3n), CSR offsets
// (n+1, taken relative to d_hsp_off[0]) and the records they cover; waits
// for `st` (see digest.cu).
bp_status bp_digest_range(bp_engine* e, cudaStream_t st, const int32_t* d_counters, int32_t n,
                          const int64_t* d_hsp_off, const bp_hsp* d_hsps, uint64_t out[2]);
// The raw digest sums of one piece of a result (subjects [first, first + n)
// of the whole, after rec_base of its records; `last`: the piece ends the
// result), and the digest of a whole result of n_subjects from the summed
// sums of its pieces.
bp_status bp_digest_sums(bp_engine* e, cudaStream_t st, const int32_t* d_counters, int32_t n,
                         const int64_t* d_hsp_off, const bp_hsp* d_hsps, int64_t first, int64_t rec_base, bool last,
                         uint64_t sums[2]);
void bp_digest_finish(const uint64_t sums[2], int64_t n_subjects, uint64_t out[2]);
// bp_search_batch whose device work starts only after `after` (an event
// recorded on another stream; null: none); the host-side setup and the
// uploads of its tables do not wait for it.
bp_status bp_search_batch_behind(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                                 const bp_batch_options* opt, cudaEvent_t after, bp_batch** out);
// Frees a batch whose work has completed without synchronising its engine's
// stream (which may already run other work).
void bp_batch_destroy_finished(bp_batch* b);
// Query qi of a finished batch as one piece of a larger result
// (bp_digest_sums), computed with engine e's scratch on stream st (e null:
// the batch's own engine and stream).
bp_status bp_batch_digest_sums(bp_batch* b, int32_t qi, bp_engine* e, cudaStream_t st, int64_t first,
                               int64_t rec_base, bool last, uint64_t sums[2]);
