// Host side of the native C ABI (include/blastp_b200.h).
//
// Replaces the reference's host driver GPU_BLASTP / GPU_BLASTP_get_data /
// GPU_BLASTP_free_memory (gpu_blastp.cu:16-280): instead of per-call
// cudaMalloc of nine buffers, per-block replicas of the presence vector and
// matrix, and a kernel launch without error checks, the engine keeps the
// database and query tables resident, reuses grow-only scratch, allocates
// per-search outputs from the stream-ordered pool, checks every CUDA call and
// returns a status.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bp_internal.h"

#define CK(call, what)                                                    \
    do {                                                                  \
        cudaError_t _err = (call);                                        \
        if (_err != cudaSuccess) return bp_set_cuda_error(e, _err, what); \
    } while (0)

bp_status bp_set_cuda_error(bp_engine* e, cudaError_t err, const char* what) {
    if (e) e->err = std::string(what) + ": " + cudaGetErrorString(err);
    cudaGetLastError();
    return err == cudaErrorMemoryAllocation ? BP_ERR_NOMEM : BP_ERR_CUDA;
}

bp_status bp_set_error(bp_engine* e, bp_status s, const std::string& msg) {
    if (e) e->err = msg;
    return s;
}

namespace {

// Sets *bad when any residue code is >= 28 (16 bytes per thread per step).
// `res` may start anywhere: the bytes before its first 16-byte boundary and
// after its last one are checked one by one, the rest with 16-byte loads.
__global__ void check_residues(const uint8_t* __restrict__ res, int64_t n, uint32_t* bad) {
    const int64_t lead = (int64_t)((16 - ((uintptr_t)res & 15)) & 15);
    const int64_t head = lead < n ? lead : n;
    const uint8_t* body = res + head;                       // 16-byte aligned
    const int64_t n16 = (n - head) / 16;
    uint32_t b = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n16; i += (int64_t)gridDim.x * blockDim.x) {
        const uint4 v = reinterpret_cast<const uint4*>(body)[i];
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            // a byte is >= 28 iff adding 100 sets its high bit or it already has it
            const uint32_t x = w[k];
            b |= (x | ((x & 0x7f7f7f7fu) + 0x64646464u)) & 0x80808080u;
        }
    }
    if (blockIdx.x == 0) {
        for (int64_t i = threadIdx.x; i < head; i += blockDim.x) b |= res[i] >= BP_ALPHABET;
        for (int64_t i = head + n16 * 16 + threadIdx.x; i < n; i += blockDim.x) b |= res[i] >= BP_ALPHABET;
    }
    if (b) atomicOr(bad, 1u);
}

template <class T>
cudaError_t grow(T** p, size_t* cap_elems, size_t need) {
    if (*p && *cap_elems >= need) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    size_t n = std::max(need, *cap_elems * 3 / 2);
    cudaError_t err = cudaMalloc((void**)p, n * sizeof(T));
    *cap_elems = err == cudaSuccess ? n : 0;
    return err;
}

constexpr int kPoolSlots = 1024;

}  // namespace

__global__ void long_list(const int64_t* __restrict__ off, int32_t first, int32_t n, int32_t long_min,
                          int32_t* __restrict__ out, int32_t* count, uint32_t* bad) {
    uint32_t b = 0;
    const int lane = threadIdx.x & 31;
    for (int32_t i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
        const int32_t i = i0 + threadIdx.x;
        bool is_long = false;
        if (i < n) {
            const int64_t d = off[(int64_t)first + i + 1] - off[(int64_t)first + i];
            b |= (d < 0 || d > (1 << 29)) ? 1u : 0u;
            is_long = d >= long_min;
        }
        const unsigned m = __ballot_sync(0xffffffffu, is_long);
        int32_t pos = 0;
        if (lane == 0 && m) pos = atomicAdd(count, __popc(m));
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (is_long) out[pos + __popc(m & ((1u << lane) - 1u))] = first + i;
    }
    if (b) atomicOr(bad, 1u);
}

cudaError_t bp_launch_long_list(bp_engine* e, cudaStream_t stream, const int64_t* d_off, int32_t first, int32_t n,
                                int32_t long_min, int32_t* out, int32_t* count, uint32_t* bad) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<int64_t>((int64_t)e->sm_count * 2, ((int64_t)n + 255) / 256);
    long_list<<<blocks, 256, 0, stream>>>(d_off, first, n, long_min, out, count, bad);
    e->launches += 1;
    return cudaGetLastError();
}

cudaError_t bp_launch_check_residues(bp_engine* e, cudaStream_t stream, const uint8_t* d_res, int64_t n,
                                     uint32_t* d_bad) {
    if (n <= 0) return cudaSuccess;
    const int64_t blocks = std::min<int64_t>((int64_t)e->sm_count * 4, (n / 16 + 255) / 256 + 1);
    check_residues<<<(unsigned)blocks, 256, 0, stream>>>(d_res, n, d_bad);
    e->launches += 1;
    return cudaGetLastError();
}

uint32_t* bp_pinned_get(bp_engine* e) {
    {
        std::lock_guard<std::mutex> lock(e->pool_mu);
        if (e->h_pool && !e->pool_free.empty()) {
            const int i = e->pool_free.back();
            e->pool_free.pop_back();
            return e->h_pool + 4 * i;
        }
    }
    uint32_t* p = nullptr;
    if (cudaMallocHost((void**)&p, 4 * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void bp_pinned_put(bp_engine* e, uint32_t* p) {
    if (!p) return;
    if (e->h_pool && p >= e->h_pool && p < e->h_pool + 4 * kPoolSlots) {
        std::lock_guard<std::mutex> lock(e->pool_mu);
        e->pool_free.push_back((int)((p - e->h_pool) / 4));
    } else {
        cudaFreeHost(p);
    }
}

// Enqueues scan + ordering for r (subjects r->first.. of r->db against r->q)
// on the engine stream.  Scratch is the engine's; outputs are r's.
bp_status bp_engine_reserve(bp_engine* e, int32_t n_subjects, size_t records) {
    if (!e || n_subjects < 0) return BP_ERR_INVALID;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    size_t cap = e->rec_cap;
    CK(grow(&e->d_recs, &cap, std::max<size_t>(records, 65536)), "cudaMalloc(records)");
    e->rec_cap = (uint32_t)cap;
    size_t fcap = (size_t)e->fill_cap;
    CK(grow(&e->d_fill, &fcap, (size_t)std::max(n_subjects, 1)), "cudaMalloc(fill)");
    e->fill_cap = (int32_t)fcap;
    size_t bcap = (size_t)e->blocksum_cap;
    CK(grow(&e->d_blocksums, &bcap, (size_t)bp_order_blocksums_needed(n_subjects)), "cudaMalloc(blocksums)");
    e->blocksum_cap = (int32_t)bcap;
    return BP_OK;
}

bp_status bp_run_search(bp_engine* e, bp_result* r) {
    const bp_db* db = r->db;
    const bp_query* q = r->q;
    const int32_t n = r->n;
    // record capacity from the expected word hits (2.5e-4 HSPs per hit, as
    // batched searches size theirs), so a long query rarely runs twice
    double span = (double)db->nres;
    if (db->h_off.size() == (size_t)db->n + 1) span = (double)(db->h_off[r->first + n] - db->h_off[r->first]);
    const size_t want = (size_t)std::min<double>(1 << 28, std::max(65536.0, 2.5e-4 * q->hits_per_residue * span));
    size_t cap = e->rec_cap;
    CK(grow(&e->d_recs, &cap, std::max<size_t>(r->cap, want)), "cudaMalloc(records)");
    e->rec_cap = (uint32_t)cap;
    size_t fcap = (size_t)e->fill_cap;
    CK(grow(&e->d_fill, &fcap, (size_t)std::max(n, 1)), "cudaMalloc(fill)");
    e->fill_cap = (int32_t)fcap;
    size_t bcap = (size_t)e->blocksum_cap;
    CK(grow(&e->d_blocksums, &bcap, (size_t)bp_order_blocksums_needed(n)), "cudaMalloc(blocksums)");
    e->blocksum_cap = (int32_t)bcap;
    if (r->cap < e->rec_cap || !r->d_hsps) {
        if (r->d_hsps) cudaFreeAsync(r->d_hsps, e->stream);
        if (r->d_keys) cudaFreeAsync(r->d_keys, e->stream);
        r->d_hsps = nullptr;
        r->d_keys = nullptr;
        r->cap = e->rec_cap;
        CK(cudaMallocAsync((void**)&r->d_hsps, (size_t)r->cap * sizeof(bp_hsp), e->stream), "cudaMallocAsync(hsps)");
        CK(cudaMallocAsync((void**)&r->d_keys, (size_t)r->cap * sizeof(int32_t), e->stream), "cudaMallocAsync(keys)");
    }
    CK(cudaMemsetAsync(e->d_counts, 0, 4 * sizeof(uint32_t), e->stream), "memset(counts)");

    ScanArgs a{};
    a.db = db->d_res;
    a.db_bytes = ((db->nres + 15) & ~15LL) + 32;   // the allocation's zero padding included
    a.db_off = db->d_off;
    a.first = r->first;
    a.n = n;
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
    a.counters = r->d_counters;
    a.recs = e->d_recs;
    a.rec_cap = std::min(e->rec_cap, r->cap);
    a.rec_count = e->d_counts;
    a.cursor = e->d_counts + 1;
    a.error = e->d_counts + 2;
    int32_t long_lo = 0;
    bp_long_slice(db->h_long, r->first, n, &long_lo, &a.n_long);
    a.long_ids = db->d_long ? db->d_long + long_lo : nullptr;
    a.long_min = db->long_min;
    CK(cudaEventRecord(e->ev_scan0, e->stream), "cudaEventRecord");
    if (n > 0) CK(bp_launch_scan(e, a), "scan kernel launch");
    CK(cudaEventRecord(e->ev_scan1, e->stream), "cudaEventRecord");
    CK(bp_launch_order(e, n, r->d_counters, r->d_hsp_off, e->d_recs, a.rec_cap, e->d_counts, e->d_fill, r->d_hsps,
                       r->d_keys, e->d_blocksums),
       "order kernels launch");
    CK(cudaMemcpyAsync(r->h_count, e->d_counts, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream),
       "copy counts");
    r->n_hsps = -1;
    return BP_OK;
}

int32_t bp_long_threshold(int64_t n_residues, int32_t n) {
    if (n <= 0) return 0;
    const int64_t t = std::max<int64_t>(64, 2 * (n_residues / n));
    return (int32_t)std::min<int64_t>(t, (int64_t)1 << 30);
}

int32_t bp_long_subjects(const int64_t* off, int32_t n, std::vector<int32_t>* out) {
    if (n <= 0) return 0;
    const int32_t long_min = bp_long_threshold(off[n] - off[0], n);
    for (int32_t i = 0; i < n; ++i)
        if (off[i + 1] - off[i] >= long_min) out->push_back(i);
    return long_min;
}

void bp_long_slice(const std::vector<int32_t>& ids, int32_t first, int32_t n, int32_t* lo, int32_t* cnt) {
    const auto a = std::lower_bound(ids.begin(), ids.end(), first);
    const auto b = std::lower_bound(a, ids.end(), (int32_t)std::min<int64_t>((int64_t)first + n, INT32_MAX));
    *lo = (int32_t)(a - ids.begin());
    *cnt = (int32_t)(b - a);
}

extern "C" {

void bp_params_default(bp_params* p) {
    p->word_length = 3;
    p->threshold = 11;
    p->window = 40;
    p->x_dropoff = 16;
    p->cutoff_score = 41;
}

const char* bp_status_string(bp_status s) {
    switch (s) {
        case BP_OK: return "ok";
        case BP_ERR_INVALID: return "invalid argument";
        case BP_ERR_CUDA: return "CUDA error";
        case BP_ERR_NOMEM: return "out of device memory";
        case BP_ERR_TOO_LARGE: return "input too large";
        case BP_ERR_TIMEOUT: return "device wait timed out";
        case BP_ERR_NOT_READY: return "not ready";
        case BP_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

void bp_blosum62_ncbistdaa(int8_t out[BP_ALPHABET * BP_ALPHABET]) { bp_fill_matrix28(out); }

bp_status bp_engine_create(int device, bp_engine** out) {
    if (!out) return BP_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return BP_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= count) return BP_ERR_INVALID;
    bp_engine* e = new bp_engine();
    e->device = device;
    bp_status st = BP_OK;
    do {
        cudaError_t err;
        if ((err = cudaSetDevice(device)) != cudaSuccess) { st = bp_set_cuda_error(e, err, "cudaSetDevice"); break; }
        if ((err = cudaDeviceGetAttribute(&e->sm_count, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess ||
            (err = cudaDeviceGetAttribute(&e->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device)) !=
                cudaSuccess) {
            st = bp_set_cuda_error(e, err, "cudaDeviceGetAttribute"); break;
        }
        if ((err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "cudaStreamCreate"); break;
        }
        if ((err = cudaEventCreate(&e->ev_scan0)) != cudaSuccess ||
            (err = cudaEventCreate(&e->ev_scan1)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "cudaEventCreate"); break;
        }
        // keep freed stream-ordered allocations cached in the pool
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
        int8_t m28[28 * 28], m32[28 * BP_MROW];
        bp_fill_matrix28(m28);
        for (int a = 0; a < 28; ++a)
            for (int b = 0; b < BP_MROW; ++b) m32[a * BP_MROW + b] = b < 28 ? m28[a * 28 + b] : (int8_t)-128;
        if ((err = cudaMalloc((void**)&e->d_matrix, sizeof(m32))) != cudaSuccess ||
            (err = cudaMemcpy(e->d_matrix, m32, sizeof(m32), cudaMemcpyHostToDevice)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "matrix upload"); break;
        }
        if ((err = cudaMalloc((void**)&e->d_counts, 16 * sizeof(uint32_t))) != cudaSuccess ||
            (err = cudaMallocHost((void**)&e->h_pool, kPoolSlots * 4 * sizeof(uint32_t))) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "counter alloc"); break;
        }
        for (int i = kPoolSlots - 1; i >= 0; --i) e->pool_free.push_back(i);
    } while (0);
    if (st != BP_OK) {
        fprintf(stderr, "bp_engine_create: %s\n", e->err.c_str());
        bp_engine_destroy(e);
        return st;
    }
    *out = e;
    return BP_OK;
}

void bp_engine_destroy(bp_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    bp_host_path_free(e);
    cudaFree(e->d_matrix);
    cudaFree(e->d_recs);
    cudaFree(e->d_counts);
    cudaFree(e->d_fill);
    cudaFree(e->d_blocksums);
    cudaFree(e->d_digest);
    if (e->h_pool) cudaFreeHost(e->h_pool);
    if (e->ev_scan0) cudaEventDestroy(e->ev_scan0);
    if (e->ev_scan1) cudaEventDestroy(e->ev_scan1);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

const char* bp_last_error(const bp_engine* e) { return e ? e->err.c_str() : ""; }
void* bp_engine_stream(bp_engine* e) { return e ? (void*)e->stream : nullptr; }
uint64_t bp_engine_launch_count(const bp_engine* e) { return e ? e->launches : 0; }
float bp_engine_last_scan_ms(const bp_engine* e) { return e ? e->last_scan_ms : 0.f; }

bp_status bp_engine_synchronize(bp_engine* e) {
    if (!e) return BP_ERR_INVALID;
    CK(cudaStreamSynchronize(e->stream), "cudaStreamSynchronize");
    return BP_OK;
}

bp_status bp_engine_set_upload_wait(bp_engine* e, uint32_t ms) {
    if (!e || ms == 0) return BP_ERR_INVALID;
    e->upload_wait_ns = (uint64_t)ms * 1000 * 1000;
    return BP_OK;
}

bp_status bp_engine_drop_chunk_flag(bp_engine* e, int32_t chunk) {
    if (!e) return BP_ERR_INVALID;
    e->drop_flag_chunk = chunk < 0 ? -1 : chunk;
    return BP_OK;
}

bp_status bp_db_alloc(bp_engine* e, int64_t n_residues, int32_t n_subjects, bp_db** out) {
    bp_db* db = new bp_db();
    db->e = e;
    db->n = n_subjects;
    db->nres = n_residues;
    cudaError_t err = cudaMalloc((void**)&db->d_res, (size_t)((n_residues + 15) & ~15LL) + 32);
    if (err == cudaSuccess) err = cudaMalloc((void**)&db->d_off, ((size_t)n_subjects + 1) * sizeof(int64_t));
    if (err != cudaSuccess) {
        bp_db_destroy(db);
        return bp_set_cuda_error(e, err, "cudaMalloc(database)");
    }
    *out = db;
    return BP_OK;
}

// Zero padding after the residues, the residue-code check on the device, and
// the longest-first list (db->h_off must be set).
bp_status bp_db_finish(bp_engine* e, bp_db* db) {
    db->h_long.clear();
    db->long_min = bp_long_subjects(db->h_off.data(), db->n, &db->h_long);
    if (!db->h_long.empty()) {
        CK(cudaMalloc((void**)&db->d_long, db->h_long.size() * sizeof(int32_t)), "cudaMalloc(long subjects)");
        CK(cudaMemcpyAsync(db->d_long, db->h_long.data(), db->h_long.size() * sizeof(int32_t),
                           cudaMemcpyHostToDevice, e->stream),
           "upload long subjects");
    }
    const size_t padded = (size_t)((db->nres + 15) & ~15LL) + 32;
    CK(cudaMemsetAsync(db->d_res + db->nres, 0, padded - (size_t)db->nres, e->stream), "pad database");
    CK(cudaMemsetAsync(e->d_counts + 3, 0, sizeof(uint32_t), e->stream), "memset(check)");
    if (db->nres > 0) {
        check_residues<<<e->sm_count * 4, 256, 0, e->stream>>>(db->d_res, db->nres, e->d_counts + 3);
        e->launches += 1;
        CK(cudaGetLastError(), "residue check launch");
    }
    uint32_t bad = 0;
    CK(cudaMemcpyAsync(&bad, e->d_counts + 3, sizeof(uint32_t), cudaMemcpyDeviceToHost, e->stream), "read check");
    CK(cudaStreamSynchronize(e->stream), "database upload");
    if (bad) return bp_set_error(e, BP_ERR_INVALID, "database: residue code >= 28");
    return BP_OK;
}

bp_status bp_db_create(bp_engine* e, const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                       int32_t n_subjects, bp_db** out) {
    if (!e || !out || !offsets || n_subjects < 0 || n_residues < 0 || (n_residues > 0 && !residues))
        return bp_set_error(e, BP_ERR_INVALID, "bp_db_create: bad argument");
    *out = nullptr;
    if (offsets[0] != 0 || offsets[n_subjects] != n_residues)
        return bp_set_error(e, BP_ERR_INVALID, "bp_db_create: offsets must run from 0 to n_residues");
    for (int32_t i = 0; i < n_subjects; ++i)
        if (offsets[i + 1] < offsets[i] || offsets[i + 1] - offsets[i] > (1 << 29))
            return bp_set_error(e, BP_ERR_INVALID, "bp_db_create: offsets must be non-decreasing, subjects < 2^29");
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    bp_db* db = nullptr;
    bp_status st = bp_db_alloc(e, n_residues, n_subjects, &db);
    if (st != BP_OK) return st;
    cudaError_t err = cudaMemcpyAsync(db->d_res, residues, (size_t)n_residues, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(db->d_off, offsets, ((size_t)n_subjects + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                              e->stream);
    if (err != cudaSuccess) {
        bp_db_destroy(db);
        return bp_set_cuda_error(e, err, "database upload");
    }
    db->h_off.assign(offsets, offsets + (size_t)n_subjects + 1);
    st = bp_db_finish(e, db);
    if (st != BP_OK) {
        bp_db_destroy(db);
        return st;
    }
    *out = db;
    return BP_OK;
}

bp_status bp_db_create_device(bp_engine* e, const uint8_t* d_residues, int64_t n_residues, const int64_t* d_offsets,
                              int32_t n_subjects, bp_db** out) {
    if (!e || !out || !d_offsets || n_subjects < 0 || n_residues < 0)
        return bp_set_error(e, BP_ERR_INVALID, "bp_db_create_device: bad argument");
    *out = nullptr;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    std::vector<int64_t> off((size_t)n_subjects + 1);
    CK(cudaMemcpy(off.data(), d_offsets, off.size() * sizeof(int64_t), cudaMemcpyDeviceToHost), "read offsets");
    if (off[0] != 0 || off[n_subjects] != n_residues)
        return bp_set_error(e, BP_ERR_INVALID, "bp_db_create_device: offsets must run from 0 to n_residues");
    for (int32_t i = 0; i < n_subjects; ++i)
        if (off[i + 1] < off[i] || off[i + 1] - off[i] > (1 << 29))
            return bp_set_error(e, BP_ERR_INVALID, "bp_db_create_device: offsets must be non-decreasing");
    bp_db* db = nullptr;
    bp_status st = bp_db_alloc(e, n_residues, n_subjects, &db);
    if (st != BP_OK) return st;
    cudaError_t err =
        cudaMemcpyAsync(db->d_res, d_residues, (size_t)n_residues, cudaMemcpyDeviceToDevice, e->stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(db->d_off, d_offsets, off.size() * sizeof(int64_t), cudaMemcpyDeviceToDevice, e->stream);
    if (err != cudaSuccess) {
        bp_db_destroy(db);
        return bp_set_cuda_error(e, err, "database copy");
    }
    db->h_off.swap(off);
    st = bp_db_finish(e, db);
    if (st != BP_OK) {
        bp_db_destroy(db);
        return st;
    }
    *out = db;
    return BP_OK;
}

void bp_db_destroy(bp_db* db) {
    if (!db) return;
    cudaFree(db->d_res);
    cudaFree(db->d_off);
    cudaFree(db->d_long);
    delete db;
}

int32_t bp_db_subjects(const bp_db* db) { return db ? db->n : 0; }
int64_t bp_db_residues(const bp_db* db) { return db ? db->nres : 0; }

bp_status bp_query_create(bp_engine* e, const uint8_t* residues, int32_t length, const bp_params* p, bp_query** out) {
    if (!e || !out || !p || length < 0 || (length > 0 && !residues))
        return bp_set_error(e, BP_ERR_INVALID, "bp_query_create: bad argument");
    *out = nullptr;
    if (length > BP_MAX_QUERY_LENGTH)
        return bp_set_error(e, BP_ERR_TOO_LARGE, "bp_query_create: query longer than 65535");
    if (p->word_length != BP_WORD || p->window < 1 || p->window > 65535 || p->x_dropoff < 0)
        return bp_set_error(e, BP_ERR_INVALID,
                            "bp_query_create: word_length must be 3, window 1..65535, x_dropoff >= 0");
    for (int32_t i = 0; i < length; ++i)
        if (residues[i] == 0 || residues[i] >= BP_ALPHABET)
            return bp_set_error(e, BP_ERR_INVALID, "bp_query_create: query residue codes must be 1..27");
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    bp_query* q = new bp_query();
    q->e = e;
    q->qlen = length;
    q->p = *p;
    q->n_ctx = 1;
    q->diag_len = bp_diag_len(length, p->window);
    bp_status st = BP_OK;
    uint32_t* d_tmp = nullptr;
    do {
        cudaError_t err;
        // stream-ordered allocations: no device-wide synchronisation, so a
        // query can be built while searches run on other streams
        if ((err = cudaMallocAsync((void**)&q->d_q, (size_t)((length + 15) & ~15) + 16, e->stream)) != cudaSuccess ||
            (err = cudaMallocAsync((void**)&q->d_cells, (BP_NC + 1) * sizeof(uint32_t), e->stream)) != cudaSuccess ||
            (err = cudaMallocAsync((void**)&q->d_ctx, 3 * sizeof(int32_t), e->stream)) != cudaSuccess ||
            (err = cudaMallocAsync((void**)&d_tmp, BP_NC * sizeof(uint32_t), e->stream)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "cudaMalloc(query)"); break;
        }
        if (length > 0 &&
            (err = cudaMemcpyAsync(q->d_q, residues, (size_t)length, cudaMemcpyHostToDevice, e->stream)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "query upload"); break;
        }
        int32_t ctx[3] = {0, p->x_dropoff, p->cutoff_score};
        if ((err = cudaMemcpyAsync(q->d_ctx, ctx, sizeof(ctx), cudaMemcpyHostToDevice, e->stream)) != cudaSuccess ||
            (err = bp_launch_table_build(e, q->d_q, length, p->threshold, q->d_cells, nullptr, d_tmp, 0)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "table count"); break;
        }
        std::vector<uint32_t> cells(BP_NC + 1);
        if ((err = cudaMemcpyAsync(cells.data(), q->d_cells, cells.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                   e->stream)) != cudaSuccess ||
            (err = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "table size"); break;
        }
        const uint32_t total = cells[BP_NC];
        q->n_entries = total;
        q->hits_per_residue = bp_expected_hits_per_residue(cells.data());
        if ((err = cudaMallocAsync((void**)&q->d_entries, (size_t)std::max<uint32_t>(total, 1) * sizeof(uint16_t),
                                   e->stream)) != cudaSuccess ||
            (err = bp_launch_table_build(e, q->d_q, length, p->threshold, q->d_cells, q->d_entries, d_tmp, 1)) !=
                cudaSuccess ||
            (err = cudaStreamSynchronize(e->stream)) != cudaSuccess) {
            st = bp_set_cuda_error(e, err, "table fill"); break;
        }
    } while (0);
    if (d_tmp) cudaFreeAsync(d_tmp, e->stream);
    if (st != BP_OK) {
        bp_query_destroy(q);
        return st;
    }
    *out = q;
    return BP_OK;
}

void bp_query_destroy(bp_query* q) {
    if (!q) return;
    cudaSetDevice(q->e->device);
    for (void* p : {(void*)q->d_q, (void*)q->d_cells, (void*)q->d_entries, (void*)q->d_ctx})
        if (p) cudaFreeAsync(p, q->e->stream);
    cudaGetLastError();
    delete q;
}

bp_status bp_query_table(bp_query* q, uint32_t* cell_start, uint16_t* entries, int64_t cap, int64_t* n_entries) {
    if (!q) return BP_ERR_INVALID;
    bp_engine* e = q->e;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    CK(cudaStreamSynchronize(e->stream), "sync");
    if (n_entries) *n_entries = q->n_entries;
    if (cell_start) {
        // expand the compact starts to the reference's 15-bit index (same entry order)
        std::vector<uint32_t> cells(BP_NC + 1);
        CK(cudaMemcpy(cells.data(), q->d_cells, cells.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost), "copy table");
        std::vector<uint32_t> cnt(BP_NCELL, 0);
        for (int c = 0; c < BP_NC; ++c) cnt[bp_cell_to_code15(c)] = cells[c + 1] - cells[c];
        uint32_t acc = 0;
        for (int c = 0; c < BP_NCELL; ++c) {
            cell_start[c] = acc;
            acc += cnt[c];
        }
        cell_start[BP_NCELL] = acc;
    }
    if (entries && q->n_entries > 0)
        CK(cudaMemcpy(entries, q->d_entries, (size_t)std::min<int64_t>(cap, q->n_entries) * sizeof(uint16_t),
                      cudaMemcpyDeviceToHost),
           "copy entries");
    return BP_OK;
}

bp_status bp_search(bp_engine* e, const bp_db* db, const bp_query* q, int32_t first, int32_t count, bp_result** out) {
    if (!e || !db || !q || !out || first < 0 || first > db->n)
        return bp_set_error(e, BP_ERR_INVALID, "bp_search: bad argument");
    *out = nullptr;
    if (count < 0 || count > db->n - first) count = db->n - first;
    if (!bp_scan_fits(q->qlen, q->diag_len, q->n_entries, e->smem_optin))
        return bp_set_error(e, BP_ERR_TOO_LARGE, "bp_search: query too long for the shared-memory diagonal array");
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    bp_result* r = new bp_result();
    r->e = e;
    r->n = count;
    r->db = db;
    r->q = q;
    r->first = first;
    r->cap = 0;
    cudaError_t err = cudaMallocAsync((void**)&r->d_counters, (size_t)std::max(count, 1) * 3 * sizeof(int32_t), e->stream);
    if (err == cudaSuccess) err = cudaMallocAsync((void**)&r->d_hsp_off, ((size_t)count + 1) * sizeof(int64_t), e->stream);
    if (err == cudaSuccess && !(r->h_count = bp_pinned_get(e))) err = cudaErrorMemoryAllocation;
    if (err != cudaSuccess) {
        bp_result_destroy(r);
        return bp_set_cuda_error(e, err, "allocate result");
    }
    bp_status st = bp_run_search(e, r);
    if (st != BP_OK) {
        bp_result_destroy(r);
        return st;
    }
    *out = r;
    return BP_OK;
}

bp_status bp_result_wait(bp_result* r) {
    if (!r) return BP_ERR_INVALID;
    bp_engine* e = r->e;
    if (r->n_hsps >= 0) return BP_OK;
    CK(cudaSetDevice(e->device), "cudaSetDevice");
    for (int attempt = 0; attempt < 4; ++attempt) {
        CK(cudaStreamSynchronize(e->stream), "search");
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e->ev_scan0, e->ev_scan1) == cudaSuccess) e->last_scan_ms = ms;
        cudaGetLastError();
        const uint32_t count = r->h_count[0];
        if (count <= r->cap) {
            r->n_hsps = count;
            return BP_OK;
        }
        // record buffer overflowed: enlarge and run again
        r->cap = count + count / 4 + 1024;
        size_t cap = e->rec_cap;
        CK(grow(&e->d_recs, &cap, r->cap), "cudaMalloc(records)");
        e->rec_cap = (uint32_t)cap;
        cudaFreeAsync(r->d_hsps, e->stream);
        cudaFreeAsync(r->d_keys, e->stream);
        r->d_hsps = nullptr;
        r->d_keys = nullptr;
        bp_status st = bp_run_search(e, r);
        if (st != BP_OK) return st;
    }
    return bp_set_error(e, BP_ERR_CUDA, "bp_result_wait: record buffer kept overflowing");
}

int32_t bp_result_subjects(const bp_result* r) { return r ? r->n : 0; }
int64_t bp_result_hsps(const bp_result* r) { return r ? r->n_hsps : -1; }

bp_status bp_result_copy(bp_result* r, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps) {
    if (!r) return BP_ERR_INVALID;
    bp_status st = bp_result_wait(r);
    if (st != BP_OK) return st;
    bp_engine* e = r->e;
    if (counters && r->n > 0)
        CK(cudaMemcpyAsync(counters, r->d_counters, (size_t)r->n * 3 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                           e->stream),
           "copy counters");
    if (hsp_off)
        CK(cudaMemcpyAsync(hsp_off, r->d_hsp_off, ((size_t)r->n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost,
                           e->stream),
           "copy offsets");
    if (hsps && r->n_hsps > 0)
        CK(cudaMemcpyAsync(hsps, r->d_hsps, (size_t)r->n_hsps * sizeof(bp_hsp), cudaMemcpyDeviceToHost, e->stream),
           "copy hsps");
    CK(cudaStreamSynchronize(e->stream), "copy results");
    return BP_OK;
}

void bp_result_destroy(bp_result* r) {
    if (!r) return;
    bp_engine* e = r->e;
    if (r->d_counters) cudaFreeAsync(r->d_counters, e->stream);
    if (r->d_hsp_off) cudaFreeAsync(r->d_hsp_off, e->stream);
    if (r->d_hsps) cudaFreeAsync(r->d_hsps, e->stream);
    if (r->d_keys) cudaFreeAsync(r->d_keys, e->stream);
    bp_pinned_put(e, r->h_count);
    delete r;
}

// The unpipelined form: database upload, then the search (bp_blastp_host
// falls back to it when the pipelined search's record buffer overflows).
bp_status bp_blastp_host_staged(bp_engine* e, const uint8_t* query, int32_t qlen, const bp_params* p,
                                const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                                int32_t n_subjects, int32_t* counters, int64_t* hsp_off, bp_hsp* hsps,
                                int64_t hsp_cap, int64_t* n_hsps) {
    if (!e) return BP_ERR_INVALID;
    bp_db* db = nullptr;
    bp_query* q = nullptr;
    bp_result* r = nullptr;
    bp_status st = bp_db_create(e, residues, n_residues, offsets, n_subjects, &db);
    if (st == BP_OK) st = bp_query_create(e, query, qlen, p, &q);
    if (st == BP_OK) st = bp_search(e, db, q, 0, -1, &r);
    if (st == BP_OK) st = bp_result_wait(r);
    if (st == BP_OK) {
        if (n_hsps) *n_hsps = r->n_hsps;
        if (hsps && r->n_hsps > hsp_cap) st = bp_set_error(e, BP_ERR_TOO_LARGE, "bp_blastp_host: hsp_cap too small");
        else st = bp_result_copy(r, counters, hsp_off, hsps);
    }
    bp_result_destroy(r);
    bp_query_destroy(q);
    bp_db_destroy(db);
    return st;
}

}  // extern "C"
