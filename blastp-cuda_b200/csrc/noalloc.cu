// bp_search_noalloc: the plain search for callers that cannot allocate device
// memory.
//
// Who cannot allocate: code that runs after a fixed device-memory budget has
// been handed out (a serving process that reserves all of HBM at start-up
// for its database and request buffers, where a late cudaMalloc would fail or
// fragment the reservation); code on a latency-critical path, where
// cudaMalloc/cudaFree synchronise the device and stall every other stream;
// and code whose memory comes from an outside allocator that this library
// cannot see.  Such a caller passes its own device buffers for inputs and
// outputs; everything the search needs beyond them -- the neighbour-word
// table, the unordered HSP records, the ordering pass's cursors -- lives in
// one file-scope array below, sized once at compile time.
//
// The array is a __device__ variable: every GPU that loads this library holds
// its 16 MiB until the process exits.  Its name in host code is only a
// host-side stand-in, not a device address, so the first call on each device
// looks up the real address with cudaGetSymbolAddress (that device current)
// and copies the scoring matrix into it.  That first call is therefore
// synchronous set-up work and should come before any stream capture.
//
// All calls share the array and it keeps the last call's contents; each call
// clears what must start at zero.  Calls that overlap on the GPU (two streams,
// or two host threads) race on it: serialise them.
#include <mutex>

#include "bp_internal.h"

namespace {

constexpr int64_t kMaxSubjects = 1 << 20;       // subjects per call
constexpr int32_t kMaxQuery = 4096;             // query length
constexpr int64_t kMaxEntries = 1 << 20;        // neighbour-table entries
constexpr int64_t kMaxRecords = 1 << 18;        // HSPs per call

constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffMatrix = 0;
constexpr size_t kOffCounts = al(kOffMatrix + 28 * BP_MROW);
constexpr size_t kOffCells = al(kOffCounts + 16 * sizeof(uint32_t));
constexpr size_t kOffTmp = al(kOffCells + (BP_NC + 1) * sizeof(uint32_t));
constexpr size_t kOffCtx = al(kOffTmp + BP_NC * sizeof(uint32_t));
constexpr size_t kOffEntries = al(kOffCtx + 4 * sizeof(int32_t));
constexpr size_t kOffRecs = al(kOffEntries + kMaxEntries * sizeof(uint16_t));
constexpr size_t kOffKeys = al(kOffRecs + kMaxRecords * sizeof(HspRec));
constexpr size_t kOffFill = al(kOffKeys + kMaxRecords * sizeof(int32_t));
constexpr size_t kOffSums = al(kOffFill + kMaxSubjects * sizeof(int32_t));
constexpr size_t kScratchBytes = al(kOffSums + ((kMaxSubjects + 4095) / 4096 + 2) * sizeof(int64_t));
static_assert(kScratchBytes <= (16u << 20), "scratch must stay within 16 MiB");

static __device__ __align__(256) uint8_t g_scratch[16u << 20];

struct DeviceSetup {
    bool ready = false;
    uint8_t* base = nullptr;       // device address of g_scratch on this device
    int sm_count = 0;
    int smem_optin = 0;
};
std::mutex g_setup_mu;
DeviceSetup g_setup[64];

// Words of the counts block: [0] records written, [1] subject cursor, [2]
// unused (the plain scan sets no error word), [3] a query residue is 0 or
// >= 28, [4] a database residue is >= 28, [5] the offsets are malformed, [6]
// long subjects listed for the longest-first cursor.
constexpr int kBadQuery = 3, kBadResidue = 4, kBadOffsets = 5, kLongCount = 6;

// Residue codes of the query and the database, and the ends of the offsets
// (off[0] == 0, off[n_subjects] == n); the lengths in between are checked by
// the long-subject listing (each in [0, 2^29]), so together every subject
// lies inside the caller's residue buffer.
__global__ void check_inputs(const uint8_t* __restrict__ q, int32_t qlen, const uint8_t* __restrict__ res,
                             int64_t n, const int64_t* __restrict__ off, int32_t n_subjects, uint32_t* counts) {
    uint32_t bq = 0, bd = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (int64_t i = t; i < qlen; i += stride) bq |= (q[i] == 0 || q[i] >= BP_ALPHABET);
    for (int64_t i = t; i < n; i += stride) bd |= res[i] >= BP_ALPHABET;
    if (bq) atomicOr(counts + kBadQuery, 1u);
    if (bd) atomicOr(counts + kBadResidue, 1u);
    if (t == 0 && (off[0] != 0 || off[n_subjects] != n)) atomicOr(counts + kBadOffsets, 1u);
}

bp_status setup_device(int dev, DeviceSetup** out) {
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.ready) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess) {
            cudaGetLastError();
            return BP_ERR_CUDA;
        }
        if (cudaDeviceGetAttribute(&s.sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&s.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
            cudaGetLastError();
            return BP_ERR_CUDA;
        }
        int8_t m28[28 * 28], m32[28 * BP_MROW];
        bp_fill_matrix28(m28);
        for (int a = 0; a < 28; ++a)
            for (int b = 0; b < BP_MROW; ++b) m32[a * BP_MROW + b] = b < 28 ? m28[a * 28 + b] : (int8_t)-128;
        if (cudaMemcpy((uint8_t*)p + kOffMatrix, m32, sizeof(m32), cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            return BP_ERR_CUDA;
        }
        s.base = (uint8_t*)p;
        s.ready = true;
    }
    *out = &s;
    return BP_OK;
}

}  // namespace

extern "C" bp_status bp_search_noalloc(const uint8_t* d_query, int32_t qlen, const bp_params* p,
                                       const uint8_t* d_residues, int64_t n_residues, const int64_t* d_offsets,
                                       int32_t n_subjects, int32_t* d_counters, int64_t* d_hsp_off, bp_hsp* d_hsps,
                                       int64_t hsp_cap, int64_t* n_hsps, void* stream) {
    if (!p || !d_offsets || !d_counters || !d_hsp_off || !n_hsps || n_subjects < 0 || n_residues < 0 || qlen < 0 ||
        hsp_cap < 0 || (qlen > 0 && !d_query) || (n_residues > 0 && !d_residues) || (hsp_cap > 0 && !d_hsps))
        return BP_ERR_INVALID;
    if (p->word_length != BP_WORD || p->window < 1 || p->window > 65535 || p->x_dropoff < 0) return BP_ERR_INVALID;
    if (n_subjects > kMaxSubjects || qlen > kMaxQuery) return BP_ERR_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return BP_ERR_NO_DEVICE;
    }
    DeviceSetup* s = nullptr;
    bp_status st = setup_device(dev, &s);
    if (st != BP_OK) return st;

    // a launch context over the caller's stream and the static array (no allocation)
    bp_engine e;
    e.device = dev;
    e.sm_count = s->sm_count;
    e.smem_optin = s->smem_optin;
    e.stream = (cudaStream_t)stream;
    e.d_matrix = (int8_t*)(s->base + kOffMatrix);
    uint32_t* counts = (uint32_t*)(s->base + kOffCounts);
    uint32_t* cells = (uint32_t*)(s->base + kOffCells);
    uint32_t* tmp = (uint32_t*)(s->base + kOffTmp);
    int32_t* ctx = (int32_t*)(s->base + kOffCtx);
    uint16_t* entries = (uint16_t*)(s->base + kOffEntries);
    HspRec* recs = (HspRec*)(s->base + kOffRecs);
    int32_t* keys = (int32_t*)(s->base + kOffKeys);
    int32_t* fill = (int32_t*)(s->base + kOffFill);
    int64_t* sums = (int64_t*)(s->base + kOffSums);
    cudaStream_t cs = e.stream;

    const int diag = bp_diag_len(qlen, p->window);
    const int32_t ctx_h[4] = {0, p->x_dropoff, p->cutoff_score, 0};
    uint32_t hostc[7] = {0, 0, 0, 0, 0, 0, 0};
    uint32_t total = 0;
    // longest first, as bp_search schedules: the long subjects' list goes into
    // the fill cursors' slice, which the ordering pass clears after the scan
    const int32_t long_min = bp_long_threshold(n_residues, n_subjects);
    cudaError_t err = cudaMemsetAsync(counts, 0, 16 * sizeof(uint32_t), cs);
    if (err == cudaSuccess) err = cudaMemcpyAsync(ctx, ctx_h, sizeof(ctx_h), cudaMemcpyHostToDevice, cs);
    if (err == cudaSuccess) {
        check_inputs<<<s->sm_count * 4, 256, 0, cs>>>(d_query, qlen, d_residues, n_residues, d_offsets, n_subjects,
                                                      counts);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess)
        err = bp_launch_long_list(&e, cs, d_offsets, 0, n_subjects, long_min, fill, (int32_t*)(counts + kLongCount),
                                  counts + kBadOffsets);
    // the checks must pass before the table build indexes the matrix with
    // query letters and before the scan reads any subject
    if (err == cudaSuccess) err = cudaMemcpyAsync(hostc, counts, sizeof(hostc), cudaMemcpyDeviceToHost, cs);
    if (err == cudaSuccess) err = cudaStreamSynchronize(cs);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return BP_ERR_CUDA;
    }
    if (hostc[kBadQuery] || hostc[kBadResidue] || hostc[kBadOffsets]) return BP_ERR_INVALID;
    err = bp_launch_table_build(&e, d_query, qlen, p->threshold, cells, nullptr, tmp, 0);
    if (err == cudaSuccess) err = cudaMemcpyAsync(&total, cells + BP_NC, sizeof(total), cudaMemcpyDeviceToHost, cs);
    if (err == cudaSuccess) err = cudaStreamSynchronize(cs);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return BP_ERR_CUDA;
    }
    if ((int64_t)total > kMaxEntries) return BP_ERR_TOO_LARGE;
    if (!bp_scan_fits(qlen, diag, total, s->smem_optin)) return BP_ERR_TOO_LARGE;
    err = bp_launch_table_build(&e, d_query, qlen, p->threshold, cells, entries, tmp, 1);

    const uint32_t cap = (uint32_t)(hsp_cap < kMaxRecords ? hsp_cap : kMaxRecords);
    ScanArgs a{};
    a.db = d_residues;
    a.db_bytes = n_residues;   // the caller's buffer: no padding assumed
    a.db_off = d_offsets;
    a.first = 0;
    a.n = n_subjects;
    a.query = d_query;
    a.qlen = qlen;
    a.cells = cells;
    a.entries = entries;
    a.n_entries = (int32_t)total;
    a.ctx = ctx;
    a.n_ctx = 1;
    a.matrix = e.d_matrix;
    a.window = p->window;
    a.diag_len = diag;
    a.counters = d_counters;
    a.recs = recs;
    a.rec_cap = cap;
    a.rec_count = counts;
    a.cursor = counts + 1;
    a.error = counts + 2;
    a.long_ids = fill;
    a.n_long_at = (const int32_t*)(counts + kLongCount);
    a.long_min = long_min;
    if (err == cudaSuccess && n_subjects > 0) err = bp_launch_scan(&e, a);
    if (err == cudaSuccess)
        err = bp_launch_order(&e, n_subjects, d_counters, d_hsp_off, recs, cap, counts, fill, d_hsps, keys, sums);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hostc, counts, 3 * sizeof(uint32_t), cudaMemcpyDeviceToHost, cs);
    if (err == cudaSuccess) err = cudaStreamSynchronize(cs);
    if (err != cudaSuccess) {
        cudaGetLastError();
        return BP_ERR_CUDA;
    }
    *n_hsps = hostc[0];
    if (hostc[0] > cap) return BP_ERR_TOO_LARGE;   // counters and offsets are complete; HSPs were not written
    return BP_OK;
}
