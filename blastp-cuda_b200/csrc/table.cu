// Device construction of the query's neighbour-word table.
//
// Replaces the NCBI-built BlastAaLookupTable that the reference copies to the
// GPU (gpu_blastp.cu:45-61, consumed at gpu_blastp_kernel.cu:182-192).  The
// rule is NCBI's: a 3-letter word w is listed under query offset q when
// score(query[q..q+2], w) >= T, and the exact query word is listed even when
// its self-score is below T.  Letters range over 1..27 (the gap letter scores
// -128 against everything and can never qualify).
//
// Layout: CSR over the 27^3 words of letters 1..27, keyed by the compact code
// (r0-1)*729 + (r1-1)*27 + (r2-1): cells[19684] (uint32 starts) and
// entries[] (uint16 query offsets, ascending within a cell).  The compact
// code orders words exactly like the reference's 15-bit index
// r0<<10 | r1<<5 | r2 (gpu_blastp_kernel.cu:149,179), so the entries array is
// the same in both layouts; only the start arrays differ.  Built in three
// launches:
//   1. count: one thread per word walks all query words;
//   2. exclusive scan of the counts (one CTA);
//   3. fill: the same walk writes the offsets in ascending order.
#include "bp_internal.h"

namespace {

constexpr int kCountThreads = 256;

__device__ __forceinline__ bool word_takes(const int8_t* m, const uint8_t* q, int pos, int r0, int r1, int r2,
                                           int threshold) {
    int a = q[pos], b = q[pos + 1], c = q[pos + 2];
    int s = m[a * BP_MROW + r0] + m[b * BP_MROW + r1] + m[c * BP_MROW + r2];
    if (s >= threshold) return true;
    int self = m[a * BP_MROW + a] + m[b * BP_MROW + b] + m[c * BP_MROW + c];
    return self < threshold && a == r0 && b == r1 && c == r2;
}

// pass 0: counts[cell] = number of query words that list the cell's word.
// pass 1: entries[cells[cell] + k] = k-th such query offset.
__global__ void __launch_bounds__(kCountThreads)
table_walk(const int8_t* __restrict__ matrix, const uint8_t* __restrict__ query, int qlen, int threshold,
           uint32_t* __restrict__ counts, const uint32_t* __restrict__ cells, uint16_t* __restrict__ entries,
           int pass) {
    extern __shared__ uint8_t sm[];
    int8_t* m = reinterpret_cast<int8_t*>(sm);                 // 28 x 32
    uint8_t* q = sm + 28 * BP_MROW;
    for (int i = threadIdx.x; i < 28 * BP_MROW; i += blockDim.x) m[i] = matrix[i];
    for (int i = threadIdx.x; i < qlen; i += blockDim.x) q[i] = query[i];
    __syncthreads();
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= BP_NC) return;
    const int r0 = cell / 729 + 1, r1 = (cell / 27) % 27 + 1, r2 = cell % 27 + 1;
    uint32_t k = 0;
    const uint32_t base = pass ? cells[cell] : 0;
    for (int pos = 0; pos + BP_WORD <= qlen; ++pos) {
        if (word_takes(m, q, pos, r0, r1, r2, threshold)) {
            if (pass) entries[base + k] = (uint16_t)pos;
            ++k;
        }
    }
    if (pass == 0) counts[cell] = k;
}

// Exclusive scan of BP_NC counts with one CTA of 1024 threads (20 cells each);
// writes cells[0..BP_NC].
__global__ void __launch_bounds__(1024)
table_scan(const uint32_t* __restrict__ counts, uint32_t* __restrict__ cells) {
    __shared__ uint32_t warp_tot[32];
    constexpr int per = (BP_NC + 1023) / 1024;  // 20
    const int t = threadIdx.x;
    uint32_t local[per];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < per; ++i) {
        const int c = t * per + i;
        local[i] = c < BP_NC ? counts[c] : 0;
        sum += local[i];
    }
    uint32_t incl = sum;
    const int lane = t & 31, w = t >> 5;
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
        const int c = t * per + i;
        if (c <= BP_NC) cells[c] = run;
        run += local[i];
    }
}

// Cells of a packed table: the members' counts summed per cell.
__global__ void pack_count(const PackSrc* __restrict__ src, int n, uint32_t* __restrict__ counts) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= BP_NC) return;
    uint32_t s = 0;
    for (int m = 0; m < n; ++m) s += src[m].cells[c + 1] - src[m].cells[c];
    counts[c] = s;
}

// Entries of a packed table: per cell, each member's entries in member order
// (so offsets stay ascending), shifted to the member's packed offset.
__global__ void pack_fill(const PackSrc* __restrict__ src, int n, const uint32_t* __restrict__ cells,
                          uint16_t* __restrict__ entries) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= BP_NC) return;
    uint32_t pos = cells[c];
    for (int m = 0; m < n; ++m) {
        const uint32_t lo = src[m].cells[c], hi = src[m].cells[c + 1];
        for (uint32_t i = lo; i < hi; ++i) entries[pos++] = (uint16_t)(src[m].entries[i] + src[m].off);
    }
}

}  // namespace

// pass 0: count + scan (the host then reads cells[BP_NC] to size the
// entries); pass 1: fill.
cudaError_t bp_launch_table_build(bp_engine* e, const uint8_t* d_q, int32_t qlen, int32_t threshold,
                                  uint32_t* d_cells, uint16_t* d_entries, uint32_t* d_counts_tmp, int pass) {
    const size_t smem = 28 * BP_MROW + (size_t)qlen;
    if (smem > 48 * 1024) {
        // the device limit, not this query's size, so that concurrent builds
        // for other queries (other threads, other engines) stay valid
        cudaError_t err =
            cudaFuncSetAttribute(table_walk, cudaFuncAttributeMaxDynamicSharedMemorySize, e->smem_optin);
        if (err != cudaSuccess) return err;
    }
    const int grid = (BP_NC + kCountThreads - 1) / kCountThreads;
    if (pass == 0) {
        table_walk<<<grid, kCountThreads, smem, e->stream>>>(e->d_matrix, d_q, qlen, threshold, d_counts_tmp,
                                                             nullptr, nullptr, 0);
        table_scan<<<1, 1024, 0, e->stream>>>(d_counts_tmp, d_cells);
        e->launches += 2;
    } else {
        table_walk<<<grid, kCountThreads, smem, e->stream>>>(e->d_matrix, d_q, qlen, threshold, nullptr,
                                                             d_cells, d_entries, 1);
        e->launches += 1;
    }
    return cudaGetLastError();
}

// 15-bit index code of a compact cell, and back.
int bp_cell_to_code15(int cell) {
    const int r0 = cell / 729 + 1, r1 = (cell / 27) % 27 + 1, r2 = cell % 27 + 1;
    return (r0 << 10) | (r1 << 5) | r2;
}

cudaError_t bp_launch_pack_table(bp_engine* e, cudaStream_t stream, const PackSrc* d_src, int n_members,
                                 uint32_t* d_counts_tmp, uint32_t* d_cells, uint16_t* d_entries) {
    const int grid = (BP_NC + 255) / 256;
    pack_count<<<grid, 256, 0, stream>>>(d_src, n_members, d_counts_tmp);
    table_scan<<<1, 1024, 0, stream>>>(d_counts_tmp, d_cells);
    pack_fill<<<grid, 256, 0, stream>>>(d_src, n_members, d_cells, d_entries);
    e->launches += 3;
    return cudaGetLastError();
}
