// Turns the scan's unordered HSP append buffer into the per-subject CSR the
// API returns, in the reference's discovery order (word position, then the
// order of query offsets in the table cell: gpu_blastp_kernel.cu:151-199).
//
//  1. hsp_off = exclusive scan of the per-subject successful-extension
//     counters (3 launches: block sums, scan of block sums, block scan);
//  2. scatter: each record takes a slot in its subject's segment;
//  3. each subject's segment is sorted by discovery key (segments are short:
//     insertion sort by one thread).
// All launches read the record count from device memory, so the pass can be
// enqueued without a host round trip; on overflow (more records than the
// buffer held) steps 2-3 do nothing and the host re-runs with a larger buffer.
#include "bp_internal.h"

namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;   // subjects per CTA

__device__ __forceinline__ int64_t block_excl_scan(int64_t v, int64_t* tmp, int64_t* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[w] = x;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        int64_t t = lane < nw ? tmp[lane] : 0, u = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int64_t y = __shfl_up_sync(0xffffffffu, u, o);
            if (lane >= o) u += y;
        }
        if (lane < nw) tmp[lane] = u - t;
        if (lane == 31) *total = u;
    }
    __syncthreads();
    int64_t r = tmp[w] + x - v;
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads)
tile_sums(const int32_t* __restrict__ counters, int32_t n, int64_t* __restrict__ sums) {
    __shared__ int64_t tmp[32];
    __shared__ int64_t total;
    int64_t acc = 0;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) acc += counters[3 * (base + i) + 1];
    block_excl_scan(acc, tmp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024)
scan_sums(int64_t* __restrict__ sums, int32_t nb) {
    __shared__ int64_t tmp[32];
    __shared__ int64_t total;
    int64_t carry = 0;
    for (int32_t b0 = 0; b0 < nb; b0 += blockDim.x) {
        const int32_t b = b0 + threadIdx.x;
        const int64_t v = b < nb ? sums[b] : 0;
        const int64_t ex = block_excl_scan(v, tmp, &total);
        if (b < nb) sums[b] = carry + ex;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) sums[nb] = carry;
}

__global__ void __launch_bounds__(kScanThreads)
tile_scan(const int32_t* __restrict__ counters, int32_t n, const int64_t* __restrict__ sums,
          int32_t nb, int64_t* __restrict__ off, int32_t* __restrict__ fill) {
    __shared__ int64_t tmp[32];
    __shared__ int64_t total;
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    int64_t acc = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? counters[3 * (base + i) + 1] : 0;
        acc += v[i];
    }
    int64_t run = sums[blockIdx.x] + block_excl_scan(acc, tmp, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) {
            off[base + i] = run;
            fill[base + i] = 0;
        }
        run += v[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) off[n] = sums[nb];
}

__global__ void scatter_recs(const HspRec* __restrict__ recs, uint32_t cap,
                             const uint32_t* __restrict__ count, const int64_t* __restrict__ off,
                             int32_t* __restrict__ fill, bp_hsp* __restrict__ out,
                             int32_t* __restrict__ keys) {
    const uint32_t c = *count;
    if (c > cap) return;   // overflow: the host re-runs with a larger buffer
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c; i += gridDim.x * blockDim.x) {
        const HspRec r = recs[i];
        const int64_t dst = off[r.oid] + atomicAdd(fill + r.oid, 1);
        out[dst] = r.h;
        keys[dst] = r.key;
    }
}

__global__ void sort_segments(int32_t n, const int64_t* __restrict__ off, const uint32_t* __restrict__ count,
                              uint32_t cap, bp_hsp* __restrict__ out, int32_t* __restrict__ keys) {
    if (*count > cap) return;
    for (int32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const int64_t lo = off[s], hi = off[s + 1];
        for (int64_t i = lo + 1; i < hi; ++i) {
            const int32_t k = keys[i];
            const bp_hsp h = out[i];
            int64_t j = i - 1;
            while (j >= lo && keys[j] > k) {
                keys[j + 1] = keys[j];
                out[j + 1] = out[j];
                --j;
            }
            keys[j + 1] = k;
            out[j + 1] = h;
        }
    }
}

}  // namespace

int32_t bp_order_blocksums_needed(int32_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

cudaError_t bp_launch_offsets(bp_engine* e, cudaStream_t st, int32_t n, const int32_t* d_counters, int64_t* d_off,
                              int32_t* d_fill, int64_t* d_blocksums) {
    const int32_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 0) return cudaMemsetAsync(d_off, 0, sizeof(int64_t), st);
    tile_sums<<<nb, kScanThreads, 0, st>>>(d_counters, n, d_blocksums);
    scan_sums<<<1, 1024, 0, st>>>(d_blocksums, nb);
    tile_scan<<<nb, kScanThreads, 0, st>>>(d_counters, n, d_blocksums, nb, d_off, d_fill);
    e->launches += 3;
    return cudaGetLastError();
}

cudaError_t bp_launch_order(bp_engine* e, int32_t n, const int32_t* d_counters, int64_t* d_hsp_off,
                            const HspRec* d_recs, uint32_t rec_cap, const uint32_t* d_rec_count,
                            int32_t* d_fill, bp_hsp* d_out, int32_t* d_keys, int64_t* d_blocksums) {
    const int32_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb > 0) {
        tile_sums<<<nb, kScanThreads, 0, e->stream>>>(d_counters, n, d_blocksums);
        scan_sums<<<1, 1024, 0, e->stream>>>(d_blocksums, nb);
        tile_scan<<<nb, kScanThreads, 0, e->stream>>>(d_counters, n, d_blocksums, nb, d_hsp_off, d_fill);
    } else {
        cudaMemsetAsync(d_hsp_off, 0, sizeof(int64_t), e->stream);
    }
    int grid = e->sm_count * 4;
    scatter_recs<<<grid, 256, 0, e->stream>>>(d_recs, rec_cap, d_rec_count, d_hsp_off, d_fill, d_out, d_keys);
    sort_segments<<<grid, 256, 0, e->stream>>>(n, d_hsp_off, d_rec_count, rec_cap, d_out, d_keys);
    e->launches += (nb > 0 ? 3 : 0) + 2;
    return cudaGetLastError();
}
