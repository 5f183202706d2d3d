/*
 * ref_driver.cpp -- runs the reference's OWN word-finder kernel on the CPU, to
 * pin the oracle (oracle.c) to the reference's code.  TEST INFRASTRUCTURE
 * ONLY: built into oracle/_ref/ by `make -C oracle ref` from the reference
 * tree, loaded by oracle/refkernel.py for the tests; the product never links,
 * loads or calls it.
 *
 * What is compiled: gpu_blastp_kernel.cu as it lies in the reference tree
 * (GPU_BLASTP_kernelTwoHit, gpu_blastp_kernel.cu:42-320, and
 * s_BlastAaExtendTwoHit/Left/Right, :341-549), included below without edits.
 * refshim/cuda_host.h (force-included) turns the CUDA qualifiers into nothing
 * and supplies gridDim/blockDim/blockIdx/threadIdx/__syncthreads; the NCBI
 * names the kernel reads come from refshim/algo/blast/core/*.h, and the
 * GPUBlastInitHitList record and ring size from the reference's own
 * ncbi_blast_files/gpu_cpu_common.h.
 *
 * What this file adds is the host side the reference's GPU_BLASTP
 * (gpu_blastp.cu:16-222) and database writer (functions.cpp:428-545) would do,
 * restated: the 4-byte-interleaved volume of groups of blocks x threads
 * subjects, each group padded with zeros to its longest member rounded up to
 * 64 (Round2Multiple, gpu_blastp.c:11-16 with WIDTH_MULTIPLE 64,
 * gpu_blastp.h:4); per-block copies of the matrix, presence vector and group
 * lengths; the NCBI thick-backbone table (<= 3 inline offsets per cell, the
 * rest in the overflow array) made from a CSR table; zeroed diagonal arrays;
 * the per-context constants.  The kernel is then run block by block, one
 * POSIX thread per CUDA thread of the block (the kernel's shared-memory
 * loading needs all of a block's threads, gpu_blastp_kernel.cu:96-129).
 *
 * Built twice: with the reference's ring of MAX_SUCCESSFUL_HITS_PER_SEQUENCE
 * = 2 records per subject (libref_ring2.so), and with REF_RING=64
 * (libref_ring64.so), which only widens that ring so that every record of a
 * subject with up to 64 successful extensions survives in discovery order.
 */
#include <algo/blast/core/gpu_cpu_common.h>

#if defined(REF_RING)
#undef MAX_SUCCESSFUL_HITS_PER_SEQUENCE
#undef MOD_MAX_SUCCESSFUL_HITS_PER_SEQUENCE
#define MAX_SUCCESSFUL_HITS_PER_SEQUENCE REF_RING
#define MOD_MAX_SUCCESSFUL_HITS_PER_SEQUENCE (REF_RING - 1)
#endif

#include "gpu_blastp_kernel.cu"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <vector>

dim3 gridDim;
dim3 blockDim;
thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
pthread_barrier_t refshim_block_barrier;

/* The kernel's dynamic shared memory (`extern __shared__ int array[]`):
 * one block runs at a time, so one buffer serves every block. */
static const int64_t kSharedInts = 1 << 21;
int array[kSharedInts];

namespace {

const int kWidthMultiple = 64;   /* gpu_blastp.h:4 */
const int kPitch = 16;           /* gpu_cpu_common.h:21 */
const int kNcell = 1 << 15;      /* 3 letters x charsize 5 */

int round_up(int x, int m) { return x % m ? x + (m - x % m) : x; }

struct KernelArgs {
    const int* db;
    const int* matrix;
    int matrix_bytes;
    const PV_ARRAY_TYPE* pv;
    const AaLookupSmallboneCell* backbone;
    const unsigned short* overflow;
    const int* glen;
    int glen_stride;
    int n_subjects;
    int pv_length;
    int qlen;
    int diag_mask;
    int diag_array_length;
    int n_ctx;
    int window;
    int diag_offset;
    int* diag;
    int* hits;
    GPUBlastInitHitList* list;
    int block;
    int tx;
};

void* run_thread(void* p)
{
    const KernelArgs* a = (const KernelArgs*)p;
    blockIdx.x = a->block; blockIdx.y = 0; blockIdx.z = 0;
    threadIdx.x = a->tx; threadIdx.y = 0; threadIdx.z = 0;
    GPU_BLASTP_kernelTwoHit(a->db, a->matrix, a->matrix_bytes, a->pv, a->backbone, a->overflow,
                            a->glen, a->glen_stride, a->n_subjects, a->pv_length, a->qlen,
                            a->diag_mask, a->diag_array_length, a->n_ctx,
                            3 /* word_length */, 5 /* charsize */, kNcell - 1 /* index mask */,
                            a->window, a->diag_offset, a->diag, a->hits, a->list);
    return nullptr;
}

}  // namespace

extern "C" int32_t ref_ring_slots(void) { return MAX_SUCCESSFUL_HITS_PER_SEQUENCE; }

/*
 * Scan subjects [0, n_subjects) of a flat database (residues + n+1 offsets)
 * with the reference kernel.
 *   cell_start/entries  neighbour-word table as CSR keyed by r0<<10|r1<<5|r2
 *                       (32768+1 starts; offsets ascending within a cell)
 *   matrix28/bytes      NCBIstdaa int8 matrix, the first matrix_bytes bytes
 *                       are given to the kernel (the reference ships 640,
 *                       gpu_cpu_common.h:28; 784 is the whole 28x28 table)
 *   ctx_*               per-context first query offset, x-drop, cutoff
 *   diag_offset         the diagonal table's starting offset (NCBI: window)
 *   blocks, threads     the launch shape; threads a multiple of 16
 * Out: hits[n*3] (hits, successful extensions, extensions), ring[n*slots*6]
 * (GPUBlastInitHitList records, slot = rank mod slots, zero when unused),
 * group_len[n] (the padded length each subject was scanned over), and, when
 * kernel_ns is not null, the wall time of the kernel's execution alone (the
 * blocks' threads from start to join; the layout work before it, which the
 * reference does once when it writes its database file, is not included).
 * Returns 0, or a negative code for arguments outside the kernel's limits.
 */
extern "C" int32_t ref_two_hit(const uint8_t* residues, const int64_t* offsets, int32_t n_subjects,
                               const uint8_t* query, int32_t qlen, const uint32_t* cell_start,
                               const uint16_t* entries, const int8_t* matrix28, int32_t matrix_bytes,
                               int32_t n_ctx, const int32_t* ctx_offset, const int32_t* ctx_xdrop,
                               const int32_t* ctx_cutoff, int32_t window, int32_t diag_array_length,
                               int32_t diag_offset, int32_t blocks, int32_t threads, int32_t* hits,
                               int32_t* ring, int32_t* group_len, int64_t* kernel_ns)
{
    if (n_subjects < 0 || qlen < 0 || qlen > QUERY_LENGTH_MAX) return -1;
    if (n_ctx < 1 || n_ctx > NUM_QUERIES_MAX) return -2;
    if (threads < 16 || threads > 1024 || threads % 16 || blocks < 1) return -3;
    if (matrix_bytes < 4 || matrix_bytes > 28 * 28 || matrix_bytes % 4) return -4;
    if (diag_array_length < 1 || (diag_array_length & (diag_array_length - 1))) return -5;

    const int G = blocks * threads;
    const int n_groups = (n_subjects + G - 1) / G;
    std::vector<int> glen(n_groups > 0 ? n_groups : 1, 0);
    for (int s = 0; s < n_subjects; ++s) {
        int64_t len = offsets[s + 1] - offsets[s];
        if (len < 0 || len > (1 << 24)) return -6;
        int g = s / G;
        if ((int)len > glen[g]) glen[g] = (int)len;
    }
    for (int g = 0; g < n_groups; ++g) glen[g] = round_up(glen[g], kWidthMultiple);

    /* interleaved volume (functions.cpp:525-536); the kernel's look-ahead load
     * may read one row past a group, so the tail carries G spare rows */
    std::vector<int64_t> gbase(n_groups + 1, 0);
    for (int g = 0; g < n_groups; ++g) gbase[g + 1] = gbase[g] + (int64_t)glen[g] * G;
    std::vector<int> volume((size_t)(gbase[n_groups] / 4 + 2 * (int64_t)G + 16), 0);
    uint8_t* vb = (uint8_t*)volume.data();
    for (int s = 0; s < n_subjects; ++s) {
        int g = s / G, member = s % G;
        const uint8_t* sub = residues + offsets[s];
        int64_t len = offsets[s + 1] - offsets[s];
        for (int64_t k = 0; k < len; ++k)
            vb[gbase[g] + ((k >> 2) * G + member) * 4 + (k & 3)] = sub[k];
        group_len[s] = glen[g];
    }

    /* per-block copies (gpu_blastp.cu:34-38,42-47,86-89) */
    const int stride = (n_groups / kPitch + (n_groups % kPitch ? 1 : 0)) * kPitch;
    int pv_length = round_up((kNcell >> PV_ARRAY_BTS) + 1, kWidthMultiple);
    std::vector<int> glen_rep((size_t)stride * blocks + 1, 0);
    for (int b = 0; b < blocks; ++b)
        for (int g = 0; g < n_groups; ++g) glen_rep[(size_t)b * stride + g] = glen[g];
    std::vector<PV_ARRAY_TYPE> pv(pv_length, 0);
    std::vector<AaLookupSmallboneCell> backbone(kNcell);
    memset(backbone.data(), 0, sizeof(AaLookupSmallboneCell) * kNcell);
    std::vector<unsigned short> overflow;
    for (int c = 0; c < kNcell; ++c) {
        uint32_t lo = cell_start[c], hi = cell_start[c + 1];
        if (hi == lo) continue;
        pv[c >> PV_ARRAY_BTS] |= (PV_ARRAY_TYPE)1 << (c & PV_ARRAY_MASK);
        backbone[c].num_used = (int)(hi - lo);
        if (hi - lo <= REFSHIM_AA_HITS_PER_CELL) {
            for (uint32_t k = lo; k < hi; ++k) backbone[c].payload.entries[k - lo] = entries[k];
        } else {
            backbone[c].payload.overflow_cursor = (int)overflow.size();
            for (uint32_t k = lo; k < hi; ++k) overflow.push_back(entries[k]);
        }
    }
    overflow.push_back(0);
    std::vector<PV_ARRAY_TYPE> pv_rep((size_t)pv_length * blocks);
    for (int b = 0; b < blocks; ++b) memcpy(&pv_rep[(size_t)b * pv_length], pv.data(), pv_length * 4);
    std::vector<int> matrix_rep((size_t)(matrix_bytes / 4) * blocks);
    for (int b = 0; b < blocks; ++b)
        memcpy(&matrix_rep[(size_t)b * (matrix_bytes / 4)], matrix28, matrix_bytes);

    const int64_t shared_ints = matrix_bytes / 4 + stride + 2 * threads + pv_length;
    if (shared_ints > kSharedInts) return -7;

    /* constant memory (gpu_blastp.cu:189-196) */
    memset(d_Query_const, 0, sizeof(d_Query_const));
    memcpy(d_Query_const, query, qlen);
    for (int k = 0; k < n_ctx; ++k) {
        d_x_dropoff_const[k] = ctx_xdrop[k];
        d_cutoff_score_const[k] = ctx_cutoff[k];
        d_query_offset_const[k] = ctx_offset[k];
    }

    const int slots = MAX_SUCCESSFUL_HITS_PER_SEQUENCE;
    std::vector<int> diag((size_t)diag_array_length * G, 0);
    std::vector<GPUBlastInitHitList> list((size_t)(n_subjects > 0 ? n_subjects : 1) * slots);
    memset(list.data(), 0, list.size() * sizeof(GPUBlastInitHitList));
    memset(hits, 0, sizeof(int32_t) * 3 * (size_t)n_subjects);

    gridDim.x = blocks; gridDim.y = 1; gridDim.z = 1;
    blockDim.x = threads; blockDim.y = 1; blockDim.z = 1;
    std::vector<KernelArgs> args(threads);
    std::vector<pthread_t> tid(threads);
    int rc = 0;
    const auto t0 = std::chrono::steady_clock::now();
    for (int b = 0; b < blocks && rc == 0; ++b) {
        memset(array, 0, sizeof(int) * shared_ints);
        pthread_barrier_init(&refshim_block_barrier, nullptr, threads);
        int started = 0;
        for (int t = 0; t < threads; ++t) {
            KernelArgs& a = args[t];
            a = KernelArgs{volume.data(), matrix_rep.data(), matrix_bytes, pv_rep.data(), backbone.data(),
                           overflow.data(), glen_rep.data(), stride, n_subjects, pv_length, qlen,
                           diag_array_length - 1, diag_array_length, n_ctx, window, diag_offset,
                           diag.data(), hits, list.data(), b, t};
            if (pthread_create(&tid[t], nullptr, run_thread, &a) != 0) { rc = -8; break; }
            ++started;
        }
        /* a thread that could not start would leave the others at the
         * barrier forever; this only happens when thread creation fails */
        if (started != threads) abort();
        for (int t = 0; t < started; ++t) pthread_join(tid[t], nullptr);
        pthread_barrier_destroy(&refshim_block_barrier);
    }
    if (kernel_ns)
        *kernel_ns = std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0)
                         .count();
    memcpy(ring, list.data(), sizeof(int32_t) * 6 * (size_t)n_subjects * slots);
    return rc;
}
