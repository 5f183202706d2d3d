// The reference's GPU entry points (include/gpu_cpu_common_b200.h) served by
// the B200 engine: a drop-in for NCBI's GPU preliminary-search call.
//
// GPU_BLASTP receives what the reference's does (gpu_blastp.cu:16-222): the
// NCBI query, contexts, lookup table, diagonal-table parameters and cutoffs,
// and the GPU-format database volume -- groups of num_blocksx*num_threadsx
// subjects, each padded with zeros to its group's length (a multiple of 64),
// stored 4-byte interleaved (ncbi_blast_files/functions.cpp:428-545).  It
//  1. converts NCBI's presence vector + thick backbone + overflow into the
//     engine's CSR table (host, 32768 cells);
//  2. copies the volume to the device and de-interleaves it there into one
//     flat run per subject (a tiled transpose), keeping the padded length as
//     the subject length, exactly as the reference kernel scans it
//     (gpu_blastp_kernel.cu:138,151,516);
//  3. runs the engine's scan with the caller's contexts, x-drops, cutoffs,
//     window and diagonal mask, writing the per-subject counters straight
//     into the caller's d_Hits.
// GPU_BLASTP_get_data then waits, fills the caller's two-slot HSP ring from
// the ordered HSP set (slot = HSP rank & 1, as gpu_blastp_kernel.cu:274
// leaves it) and copies both arrays to the host.
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>
#include <vector>

#include "bp_internal.h"
#include "gpu_cpu_common_b200.h"

static_assert(sizeof(GPUBlastInitHitList) == sizeof(bp_hsp), "HSP record layouts differ");

namespace {

std::mutex g_mu;
bp_engine* g_engines[64] = {};

struct LegacyJob {
    bp_engine* e = nullptr;
    bp_db db;
    bp_query q;
    bp_result r;
    int32_t n = 0;
    GPUBlastInitHitList* d_list = nullptr;
    int64_t list_cap = 0;
    bool ok = false;
};
std::map<const void*, LegacyJob*> g_jobs;   // keyed by the caller's d_Hits

bp_engine* engine_for_current_device() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    if (!g_engines[dev]) {
        bp_engine* e = nullptr;
        if (bp_engine_create(dev, &e) != BP_OK) return nullptr;
        g_engines[dev] = e;
    }
    return g_engines[dev];
}

// Tiled transpose of one group: source int index base/4 + w*G + i holds
// residues 4w..4w+3 of group member i; destination is member i's flat run.
__global__ void deinterleave(const int32_t* __restrict__ src, uint8_t* __restrict__ dst,
                             const int64_t* __restrict__ group_base, const int32_t* __restrict__ group_len,
                             int32_t group_size, int32_t n_groups, int32_t n_seq) {
    __shared__ int32_t tile[32][33];
    const int g = blockIdx.z;
    if (g >= n_groups) return;
    const int words = group_len[g] >> 2;
    const int w0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
    if (w0 >= words || i0 >= group_size) return;
    const int64_t gb = group_base[g];
    const int64_t first_seq = (int64_t)g * group_size;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int w = w0 + r, i = i0 + threadIdx.x;
        if (w < words && i < group_size && first_seq + i < n_seq)
            tile[r][threadIdx.x] = src[(gb >> 2) + (int64_t)w * group_size + i];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int i = i0 + r, w = w0 + threadIdx.x;
        if (w < words && i < group_size && first_seq + i < n_seq)
            reinterpret_cast<int32_t*>(dst + gb + (int64_t)i * group_len[g])[w] = tile[threadIdx.x][r];
    }
}

// Final two slots per subject: rank r goes to slot r & 1, later ranks
// overwriting earlier ones (gpu_blastp_kernel.cu:274).
__global__ void fill_ring(int32_t n, const int32_t* __restrict__ counters, const int64_t* __restrict__ off,
                          const bp_hsp* __restrict__ hsps, GPUBlastInitHitList* __restrict__ list, int64_t cap) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int32_t succ = counters[3 * (int64_t)s + 1];
        for (int32_t k = succ >= 2 ? succ - 2 : 0; k < succ; ++k) {
            const int64_t slot = 2 * (int64_t)s + (k & 1);
            if (slot < cap) {
                const bp_hsp h = hsps[off[s] + k];
                GPUBlastInitHitList x;
                x.hsp_q = h.hsp_q;
                x.hsp_s = h.hsp_s;
                x.query_offset = h.query_offset;
                x.subject_offset = h.subject_offset;
                x.hsp_len = h.hsp_len;
                x.score = h.score;
                list[slot] = x;
            }
        }
    }
}

// On any failure every subject reports 3 successful extensions, which makes
// the caller re-search it on the CPU (blast_engine.c:529-538).
__global__ void mark_for_cpu(int32_t n, int32_t* counters) {
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        counters[3 * (int64_t)s + 0] = 0;
        counters[3 * (int64_t)s + 1] = MAX_SUCCESSFUL_HITS_PER_SEQUENCE + 1;
        counters[3 * (int64_t)s + 2] = 0;
    }
}

void fail(const char* what, cudaError_t err) {
    fprintf(stderr, "GPU_BLASTP (b200): %s%s%s\n", what, err != cudaSuccess ? ": " : "",
            err != cudaSuccess ? cudaGetErrorString(err) : "");
    cudaGetLastError();
}

}  // namespace

extern "C" {

void Round2Multiple(Int4* MaxLength) {
    const int r = *MaxLength % 64;
    if (r) *MaxLength += 64 - r;
}

Boolean GPU_BLAST_check_availability(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return FALSE;
    }
    return n > 0 ? TRUE : FALSE;
}

Boolean GPU_BLASTP_check_memory(const LookupTableWrap* lookup_wrap, const Blast_ExtendWord* ewp,
                                const BlastGPUOptions* gpu_options, const int h_Database2Dpadded_bytes,
                                const Int4 h_Hits_bytes, const Int4 h_GPUBlastInitHitList_bytes,
                                const Int4 Group_number, const Int4 num_queries, const Int4 query_length) {
    (void)Group_number;
    if (num_queries > NUM_QUERIES_MAX_B200 || query_length > QUERY_LENGTH_MAX_B200) return FALSE;
    const BlastAaLookupTable* lookup = (const BlastAaLookupTable*)lookup_wrap->lut;
    if (lookup->word_length != 3 || lookup->charsize != 5) return FALSE;
    int dev = 0, optin = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return FALSE;
    }
    // any table size fits when it stays in global memory; the diagonal array must fit shared memory
    if (!bp_scan_fits(query_length, bp_diag_len(query_length, ewp->diag_table->window), 1 << 30, optin)) return FALSE;
    const size_t n = (size_t)gpu_options->num_sequences_to;
    size_t need = 2 * (size_t)h_Database2Dpadded_bytes + 8 * (n + 1) + (size_t)h_Hits_bytes +
                  3 * (size_t)h_GPUBlastInitHitList_bytes + (BP_NCELL + 1) * 4 +
                  (size_t)lookup->overflow_size * 2 + 64 * (size_t)query_length + 12 * n + (64u << 20);
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return FALSE;
    }
    return need <= free_b ? TRUE : FALSE;
}

void GPU_BLASTP(const BLAST_SequenceBlk* query, const BlastQueryInfo* query_info,
                const LookupTableWrap* lookup_wrap, const Blast_ExtendWord* ewp,
                const BlastInitialWordParameters* word_params, const BlastGPUOptions* gpu_options,
                const int* Sequence_length_vector, const int h_Database2Dpadded_bytes,
                const char* h_Database2Dpadded, Int4** d_Hits, const Int4 h_Hits_bytes,
                GPUBlastInitHitList** d_GPUBlastInitHitList, const Int4 h_GPUBlastInitHitList_bytes,
                Int4** d_Database2Dpadded, Int4** d_RepeatedSubstitutionMatrix,
                Int4** d_RepeatedSequence_length_vector, PV_ARRAY_TYPE** d_RepeatedPV,
                AaLookupSmallboneCell** d_ThickBackbone, Uint2** d_overflow, Int4** d_RepeatedDiag_array) {
    std::lock_guard<std::mutex> lock(g_mu);
    const int32_t n = gpu_options->num_sequences_to;
    const int32_t G = gpu_options->num_blocksx * gpu_options->num_threadsx;
    const int32_t n_groups = G > 0 ? (n + G - 1) / G : 0;
    const int32_t Q = query->length;
    const int32_t nq = query_info->num_queries;
    const BlastAaLookupTable* lookup = (const BlastAaLookupTable*)lookup_wrap->lut;
    bp_engine* e = engine_for_current_device();
    cudaError_t err = cudaSuccess;

    // d_Hits first, so that a failure below can still tell the caller to use its CPU path.
    if ((err = cudaMalloc((void**)d_Hits, (size_t)h_Hits_bytes)) != cudaSuccess) {
        fail("cudaMalloc(d_Hits)", err);
        return;
    }
    if ((err = cudaMalloc((void**)d_GPUBlastInitHitList, (size_t)h_GPUBlastInitHitList_bytes)) != cudaSuccess ||
        (err = cudaMemset(*d_GPUBlastInitHitList, 0, (size_t)h_GPUBlastInitHitList_bytes)) != cudaSuccess) {
        fail("cudaMalloc(d_GPUBlastInitHitList)", err);
        mark_for_cpu<<<64, 256>>>(h_Hits_bytes / 12, *d_Hits);
        return;
    }
    LegacyJob* job = new LegacyJob();
    job->e = e;
    job->n = n;
    job->d_list = *d_GPUBlastInitHitList;
    job->list_cap = h_GPUBlastInitHitList_bytes / (int64_t)sizeof(GPUBlastInitHitList);
    g_jobs[*d_Hits] = job;

    const char* why = nullptr;
    do {
        if (!e) { why = "no CUDA device"; break; }
        if (lookup->word_length != 3 || lookup->charsize != 5) { why = "only word length 3, 5-bit letters"; break; }
        if (n < 0 || G <= 0 || (int64_t)n * 3 * 4 > h_Hits_bytes) { why = "inconsistent sizes"; break; }
        int64_t vol = 0;
        std::vector<int64_t> gbase((size_t)n_groups + 1);
        for (int32_t g = 0; g < n_groups; ++g) {
            if (Sequence_length_vector[g] < 0 || (Sequence_length_vector[g] & 3)) { why = "bad group length"; break; }
            gbase[g] = vol;
            vol += (int64_t)Sequence_length_vector[g] * G;
        }
        if (why) break;
        gbase[n_groups] = vol;
        if (vol > h_Database2Dpadded_bytes) { why = "database smaller than its group lengths"; break; }
        // 1. NCBI table -> compact CSR over the 27^3 words of letters 1..27 (a
        // word holding the gap letter or a code >= 28 can never be scanned:
        // such words have no cell).  A cell counts only when its presence bit
        // is set, as the reference tests the bit first
        // (gpu_blastp_kernel.cu:182-192).
        const AaLookupSmallboneCell* cells = (const AaLookupSmallboneCell*)lookup->thick_backbone;
        const Uint2* ovf = (const Uint2*)lookup->overflow;
        const PV_ARRAY_TYPE* pv = lookup->pv;
        const int ncell = lookup->backbone_size < BP_NCELL ? lookup->backbone_size : BP_NCELL;
        std::vector<uint32_t> cell_start(BP_NC + 1);
        std::vector<uint16_t> entries;
        for (int cc = 0; cc < BP_NC; ++cc) {
            cell_start[cc] = (uint32_t)entries.size();
            const int c = bp_cell_to_code15(cc);
            if (c >= ncell || !(pv[c >> 5] & (1u << (c & 31)))) continue;
            const int used = cells[c].num_used;
            if (used <= 0) continue;
            const Uint2* src = used <= AA_HITS_PER_CELL ? cells[c].payload.entries
                                                        : ovf + cells[c].payload.overflow_cursor;
            entries.insert(entries.end(), src, src + used);
        }
        cell_start[BP_NC] = (uint32_t)entries.size();
        // every listed offset must start a whole word of the query
        for (uint16_t x : entries)
            if ((int32_t)x + 3 > Q) { why = "lookup table lists an offset beyond the query"; break; }
        if (why) break;
        if (ewp->diag_table->window < 1 || ewp->diag_table->window > 65535) {
            why = "two-hit window outside 1..65535";
            break;
        }
        if (!bp_scan_fits(Q, bp_diag_len(Q, ewp->diag_table->window), (int64_t)cell_start[BP_NC], e->smem_optin)) {
            why = "query too long for the shared-memory diagonal array";
            break;
        }
        if (entries.empty()) entries.push_back(0);

        if (nq < 1) { why = "no query context"; break; }
        std::vector<int32_t> ctx((size_t)3 * nq);
        for (int k = 0; k < nq; ++k) {
            ctx[3 * k + 0] = query_info->contexts[k].query_offset;
            ctx[3 * k + 1] = word_params->cutoffs[k].x_dropoff;
            ctx[3 * k + 2] = word_params->cutoffs[k].cutoff_score;
            if (k > 0 && ctx[3 * k] < ctx[3 * (k - 1)]) { why = "context offsets not ascending"; break; }
        }
        if (why) break;
        std::vector<int64_t> off((size_t)n + 1);
        for (int32_t s = 0; s < n; ++s) {
            const int32_t g = s / G, i = s % G;
            off[s] = gbase[g] + (int64_t)i * Sequence_length_vector[g];
        }
        off[n] = n > 0 ? off[n - 1] + Sequence_length_vector[(n - 1) / G] : 0;

        // 2. device buffers, in the caller's slots
        auto up = [&](void** slot, const void* src, size_t bytes) {
            if (err != cudaSuccess) return;
            err = cudaMalloc(slot, bytes ? bytes : 16);
            if (err == cudaSuccess && bytes) err = cudaMemcpy(*slot, src, bytes, cudaMemcpyHostToDevice);
        };
        int8_t m32[28 * BP_MROW];
        {
            int8_t m28[28 * 28];
            bp_fill_matrix28(m28);
            for (int a = 0; a < 28; ++a)
                for (int b = 0; b < BP_MROW; ++b) m32[a * BP_MROW + b] = b < 28 ? m28[a * 28 + b] : (int8_t)-128;
        }
        up((void**)d_Database2Dpadded, h_Database2Dpadded, (size_t)h_Database2Dpadded_bytes);
        up((void**)d_RepeatedSubstitutionMatrix, m32, sizeof(m32));
        up((void**)d_RepeatedSequence_length_vector, Sequence_length_vector, (size_t)n_groups * 4);
        *d_RepeatedPV = nullptr;   // the compact table needs no presence vector
        up((void**)d_ThickBackbone, cell_start.data(), cell_start.size() * 4);
        up((void**)d_overflow, entries.data(), entries.size() * 2);
        // arena: flat volume | offsets | group bases | query | contexts
        const size_t a_flat = ((size_t)vol + 16 + 255) & ~(size_t)255;
        const size_t a_off = a_flat + (((size_t)n + 1) * 8 + 255 & ~(size_t)255);
        const size_t a_gb = a_off + (((size_t)n_groups + 1) * 8 + 255 & ~(size_t)255);
        const size_t a_q = a_gb + (((size_t)Q + 16 + 255) & ~(size_t)255);
        const size_t a_end = a_q + (size_t)nq * 12 + 16;
        if (err == cudaSuccess) err = cudaMalloc((void**)d_RepeatedDiag_array, a_end);
        if (err != cudaSuccess) { why = "device allocation/upload"; break; }
        uint8_t* arena = (uint8_t*)*d_RepeatedDiag_array;
        uint8_t* d_flat = arena;
        int64_t* d_off = (int64_t*)(arena + a_flat);
        int64_t* d_gb = (int64_t*)(arena + a_off);
        uint8_t* d_q = arena + a_gb;
        int32_t* d_ctx = (int32_t*)(arena + a_q);
        cudaStream_t st = e->stream;
        if ((err = cudaMemsetAsync(d_flat + vol, 0, 16, st)) != cudaSuccess ||
            (err = cudaMemcpyAsync(d_off, off.data(), off.size() * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (err = cudaMemcpyAsync(d_gb, gbase.data(), gbase.size() * 8, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (err = cudaMemcpyAsync(d_q, query->sequence, (size_t)Q, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (err = cudaMemcpyAsync(d_ctx, ctx.data(), ctx.size() * 4, cudaMemcpyHostToDevice, st)) != cudaSuccess) {
            why = "upload";
            break;
        }
        int max_len = 0;
        for (int32_t g = 0; g < n_groups; ++g) max_len = max_len > Sequence_length_vector[g] ? max_len : Sequence_length_vector[g];
        if (n_groups > 0 && max_len > 0) {
            dim3 grid((max_len / 4 + 31) / 32, (G + 31) / 32, n_groups);
            deinterleave<<<grid, dim3(32, 8), 0, st>>>((const int32_t*)*d_Database2Dpadded, d_flat, d_gb,
                                                      *d_RepeatedSequence_length_vector, G, n_groups, n);
            e->launches += 1;
        }

        // 3. scan with the caller's parameters
        job->db.e = e;
        job->db.d_res = d_flat;
        job->db.d_off = d_off;
        job->db.n = n;
        job->db.nres = vol;
        job->q.e = e;
        job->q.d_q = d_q;
        job->q.qlen = Q;
        job->q.d_cells = (uint32_t*)*d_ThickBackbone;
        job->q.d_entries = *d_overflow;
        job->q.n_entries = cell_start[BP_NC];
        job->q.n_ctx = nq;
        job->q.d_ctx = d_ctx;
        job->q.p.word_length = 3;
        job->q.p.window = ewp->diag_table->window;
        // any array of at least Q + window entries gives the reference's results
        // with its power-of-two diag_mask table (gpu_blastp_kernel.cu:202)
        job->q.diag_len = bp_diag_len(Q, ewp->diag_table->window);
        job->q.hits_per_residue = bp_expected_hits_per_residue(cell_start.data());
        job->r.e = e;
        job->r.n = n;
        job->r.db = &job->db;
        job->r.q = &job->q;
        job->r.first = 0;
        job->r.d_counters = *d_Hits;
        if ((err = cudaMalloc((void**)&job->r.d_hsp_off, ((size_t)n + 1) * 8)) != cudaSuccess ||
            !(job->r.h_count = bp_pinned_get(e))) {
            why = "result allocation";
            break;
        }
        if (bp_run_search(e, &job->r) != BP_OK) { why = e->err.c_str(); err = cudaSuccess; break; }
        job->ok = true;
    } while (0);
    if (!job->ok) {
        fail(why ? why : "failed", err);
        mark_for_cpu<<<64, 256>>>(h_Hits_bytes / 12, *d_Hits);
        cudaDeviceSynchronize();
    }
}

void GPU_BLASTP_get_data(Int4* h_Hits, Int4* d_Hits, const Int4 h_Hits_bytes,
                         GPUBlastInitHitList* h_GPUBlastInitHitList,
                         GPUBlastInitHitList* d_GPUBlastInitHitList, Int4 h_GPUBlastInitHitList_bytes,
                         Int4 num_sequences) {
    (void)num_sequences;
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_jobs.find(d_Hits);
    LegacyJob* job = it == g_jobs.end() ? nullptr : it->second;
    if (job && job->ok) {
        bp_engine* e = job->e;
        if (bp_result_wait(&job->r) != BP_OK) {
            fail(e->err.c_str(), cudaSuccess);
            mark_for_cpu<<<64, 256, 0, e->stream>>>(job->n, d_Hits);
        } else if (job->n > 0) {
            fill_ring<<<e->sm_count * 4, 256, 0, e->stream>>>(job->n, job->r.d_counters, job->r.d_hsp_off,
                                                             job->r.d_hsps, d_GPUBlastInitHitList, job->list_cap);
            e->launches += 1;
        }
        cudaStreamSynchronize(e->stream);
    }
    cudaError_t err = cudaMemcpy(h_Hits, d_Hits, (size_t)h_Hits_bytes, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = cudaMemcpy(h_GPUBlastInitHitList, d_GPUBlastInitHitList, (size_t)h_GPUBlastInitHitList_bytes,
                         cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        fail("copy to host", err);
        for (int64_t s = 0; s < h_Hits_bytes / 12; ++s) {
            h_Hits[3 * s + 0] = 0;
            h_Hits[3 * s + 1] = MAX_SUCCESSFUL_HITS_PER_SEQUENCE + 1;
            h_Hits[3 * s + 2] = 0;
        }
    }
}

Boolean GPU_BLASTP_get_hsps(Int4* d_Hits, int64_t* hsp_off, GPUBlastInitHitList* hsps, int64_t hsp_cap,
                            int64_t* n_hsps) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_jobs.find(d_Hits);
    if (it == g_jobs.end() || !it->second->ok) return FALSE;
    LegacyJob* job = it->second;
    if (bp_result_wait(&job->r) != BP_OK) return FALSE;
    const int64_t k = bp_result_hsps(&job->r);
    if (n_hsps) *n_hsps = k;
    if (hsps && k > hsp_cap) return FALSE;
    return bp_result_copy(&job->r, nullptr, hsp_off, reinterpret_cast<bp_hsp*>(hsps)) == BP_OK ? TRUE : FALSE;
}

void GPU_BLASTP_free_memory(Int4** d_Hits, GPUBlastInitHitList** d_GPUBlastInitHitList,
                            Int4** d_Database2Dpadded, Int4** d_RepeatedSubstitutionMatrix,
                            Int4** d_RepeatedSequence_length_vector, PV_ARRAY_TYPE** d_RepeatedPV,
                            AaLookupSmallboneCell** d_ThickBackbone, Uint2** d_overflow,
                            Int4** d_RepeatedDiag_array) {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_jobs.find(*d_Hits);
    if (it != g_jobs.end()) {
        LegacyJob* job = it->second;
        if (job->e) cudaStreamSynchronize(job->e->stream);
        cudaFree(job->r.d_hsp_off);
        if (job->e) {
            if (job->r.d_hsps) cudaFreeAsync(job->r.d_hsps, job->e->stream);
            if (job->r.d_keys) cudaFreeAsync(job->r.d_keys, job->e->stream);
            cudaStreamSynchronize(job->e->stream);
        }
        if (job->e) bp_pinned_put(job->e, job->r.h_count);
        delete job;
        g_jobs.erase(it);
    }
    cudaFree(*d_Hits);
    cudaFree(*d_GPUBlastInitHitList);
    cudaFree(*d_Database2Dpadded);
    cudaFree(*d_RepeatedSubstitutionMatrix);
    cudaFree(*d_RepeatedSequence_length_vector);
    cudaFree(*d_RepeatedPV);
    cudaFree(*d_ThickBackbone);
    cudaFree(*d_overflow);
    cudaFree(*d_RepeatedDiag_array);
    cudaDeviceSynchronize();
}

}  // extern "C"
