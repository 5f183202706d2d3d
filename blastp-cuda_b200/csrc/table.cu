// Device construction of the query's neighbour-word table.
//
// Replaces the NCBI-built BlastAaLookupTable that the reference copies to the
// GPU (gpu_blastp.cu:45-61, consumed at gpu_blastp_kernel.cu:182-192).  The
// rule is NCBI's: a 3-letter word w is listed under query offset q when
// score(query[q..q+2], w) >= T, and the exact query word is listed even when
// its self-score is below T.  Letters range over 1..27 (the gap letter scores
// -128 against everything and can never qualify).
//
// Layout: CSR keyed by the packed code r0<<10 | r1<<5 | r2 (the reference's
// 15-bit index, gpu_blastp_kernel.cu:149,179): cell_start[32769] (uint32)
// and entries[] (uint16 query offsets, ascending within a cell), plus a
// 32768-bit presence bitmap.  Built in three launches:
//   1. count: one thread per code walks all query words;
//   2. exclusive scan of the counts (one CTA), presence bits;
//   3. fill: the same walk writes the offsets in ascending order.
#include "bp_internal.h"

namespace {

constexpr int kCountThreads = 256;

__device__ __forceinline__ bool word_takes(const int8_t* m, const uint8_t* q, int pos, int r0,
                                           int r1, int r2, int threshold) {
    int a = q[pos], b = q[pos + 1], c = q[pos + 2];
    int s = m[a * BP_MROW + r0] + m[b * BP_MROW + r1] + m[c * BP_MROW + r2];
    if (s >= threshold) return true;
    int self = m[a * BP_MROW + a] + m[b * BP_MROW + b] + m[c * BP_MROW + c];
    return self < threshold && a == r0 && b == r1 && c == r2;
}

// pass 0: counts[code] = number of query words that list `code`.
// pass 1: entries[cell_start[code] + k] = k-th such query offset.
__global__ void __launch_bounds__(kCountThreads)
table_walk(const int8_t* __restrict__ matrix, const uint8_t* __restrict__ query, int qlen,
           int threshold, uint32_t* __restrict__ counts, const uint32_t* __restrict__ cell_start,
           uint16_t* __restrict__ entries, int pass) {
    extern __shared__ uint8_t sm[];
    int8_t* m = reinterpret_cast<int8_t*>(sm);                 // 28 x 32
    uint8_t* q = sm + 28 * BP_MROW;
    for (int i = threadIdx.x; i < 28 * BP_MROW; i += blockDim.x) m[i] = matrix[i];
    for (int i = threadIdx.x; i < qlen; i += blockDim.x) q[i] = query[i];
    __syncthreads();
    int code = blockIdx.x * blockDim.x + threadIdx.x;
    if (code >= BP_NCELL) return;
    int r0 = code >> 10, r1 = (code >> 5) & 31, r2 = code & 31;
    if (r0 == 0 || r1 == 0 || r2 == 0 || r0 >= 28 || r1 >= 28 || r2 >= 28) {
        if (pass == 0) counts[code] = 0;
        return;
    }
    uint32_t k = 0;
    uint32_t base = pass ? cell_start[code] : 0;
    for (int pos = 0; pos + BP_WORD <= qlen; ++pos) {
        if (word_takes(m, q, pos, r0, r1, r2, threshold)) {
            if (pass) entries[base + k] = (uint16_t)pos;
            ++k;
        }
    }
    if (pass == 0) counts[code] = k;
}

// Exclusive scan of BP_NCELL counts with one CTA of 1024 threads (32 cells
// each); writes cell_start[0..BP_NCELL], the presence bitmap and the total.
__global__ void __launch_bounds__(1024)
table_scan(const uint32_t* __restrict__ counts, uint32_t* __restrict__ cell_start,
           uint32_t* __restrict__ pv) {
    __shared__ uint32_t warp_tot[32];
    const int per = BP_NCELL / 1024;  // 32
    int t = threadIdx.x;
    uint32_t local[per];
    uint32_t sum = 0, bits = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        local[i] = counts[t * per + i];
        bits |= (local[i] ? 1u : 0u) << i;
        sum += local[i];
    }
    pv[t] = bits;   // 32 cells per thread = one presence word
    uint32_t incl = sum;
    int lane = t & 31, w = t >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        uint32_t v = warp_tot[lane], x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        warp_tot[lane] = x - v;
    }
    __syncthreads();
    uint32_t run = warp_tot[w] + incl - sum;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        cell_start[t * per + i] = run;
        run += local[i];
    }
    if (t == 1023) cell_start[BP_NCELL] = run;
}

}  // namespace

// pass 0: count + scan (the host then reads cell_start[BP_NCELL] to size the
// entries); pass 1: fill.
cudaError_t bp_launch_table_build(bp_engine* e, const uint8_t* d_q, int32_t qlen, int32_t threshold,
                                  uint32_t* d_cell_start, uint16_t* d_entries, uint32_t* d_pv,
                                  uint32_t* d_counts_tmp, int64_t entry_cap, int pass) {
    (void)entry_cap;
    size_t smem = 28 * BP_MROW + (size_t)qlen;
    if (smem > 48 * 1024) {
        cudaError_t err = cudaFuncSetAttribute(table_walk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem);
        if (err != cudaSuccess) return err;
    }
    int grid = BP_NCELL / kCountThreads;
    if (pass == 0) {
        table_walk<<<grid, kCountThreads, smem, e->stream>>>(e->d_matrix, d_q, qlen, threshold,
                                                             d_counts_tmp, nullptr, nullptr, 0);
        table_scan<<<1, 1024, 0, e->stream>>>(d_counts_tmp, d_cell_start, d_pv);
        e->launches += 2;
    } else {
        table_walk<<<grid, kCountThreads, smem, e->stream>>>(e->d_matrix, d_q, qlen, threshold,
                                                             nullptr, d_cell_start, d_entries, 1);
        e->launches += 1;
    }
    return cudaGetLastError();
}
