// Result digests: a 128-bit fingerprint of one query's search result --
// per-subject counters, HSP offsets relative to the result's first HSP, and
// the HSP records -- computed on the device.  Two results with equal digests
// are equal with overwhelming probability, so whole result sets (a batch of
// hundreds of queries over millions of subjects, a served request) can be
// compared with a plain search without copying them to the host.  No
// counterpart in the reference.
//
// Each 32-bit word w at position i of one of the three arrays contributes
// mix(tag, i, w) to two independent 64-bit sums (mix: the splitmix64
// finaliser, a published bijective mixer); the sums are order-independent,
// so any grid may compute them, and position- and array-sensitive.  A
// result kept in pieces (consecutive subject ranges, each with its own CSR
// offsets) is digested piece by piece at its global positions and the sums
// added: the same digest as the whole.
#include <string.h>

#include <algorithm>

#include "bp_internal.h"

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

__device__ __forceinline__ void add_word(uint64_t tag, uint64_t i, uint32_t w, uint64_t& a, uint64_t& b) {
    const uint64_t h = mix64((tag << 56) ^ (i << 32) ^ (i >> 32) ^ (uint64_t)w);
    a += h;
    b += mix64(h ^ 0x9e3779b97f4a7c15ull);
}

// counters: 3n words; offsets: n+1 values hoff[i] - hoff[0] (two words
// each; the last one only when `last`); records: (hoff[n] - hoff[0]) x 6
// words from hsps + hoff[0].  The piece starts at subject `first` of the
// whole result, after `rec_base` of its records.
__global__ void digest_kernel(const int32_t* __restrict__ counters, int32_t n, const int64_t* __restrict__ hoff,
                              const bp_hsp* __restrict__ hsps, int64_t first, int64_t rec_base, int last,
                              unsigned long long* out) {
    const int64_t lo = hoff[0];
    const int64_t cnt = hoff[n] - lo;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    uint64_t a = 0, b = 0;
    for (int64_t i = t; i < 3 * (int64_t)n; i += stride)
        add_word(1, (uint64_t)(3 * first + i), (uint32_t)counters[i], a, b);
    for (int64_t i = t; i < (int64_t)n + (last ? 1 : 0); i += stride) {
        const uint64_t v = (uint64_t)(hoff[i] - lo + rec_base);
        add_word(2, 2 * (uint64_t)(first + i), (uint32_t)v, a, b);
        add_word(2, 2 * (uint64_t)(first + i) + 1, (uint32_t)(v >> 32), a, b);
    }
    const uint32_t* w = reinterpret_cast<const uint32_t*>(hsps + lo);
    for (int64_t i = t; i < 6 * cnt; i += stride) add_word(3, (uint64_t)(6 * rec_base + i), w[i], a, b);
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out, (unsigned long long)a);
        atomicAdd(out + 1, (unsigned long long)b);
    }
}

}  // namespace

bp_status bp_digest_sums(bp_engine* e, cudaStream_t st, const int32_t* d_counters, int32_t n,
                         const int64_t* d_hsp_off, const bp_hsp* d_hsps, int64_t first, int64_t rec_base, bool last,
                         uint64_t sums[2]) {
    if (!e || !sums || n < 0 || !d_hsp_off || (n > 0 && !d_counters) || first < 0 || rec_base < 0)
        return BP_ERR_INVALID;
    cudaError_t err = cudaSetDevice(e->device);
    if (err == cudaSuccess && !e->d_digest) err = cudaMalloc((void**)&e->d_digest, 2 * sizeof(unsigned long long));
    if (err != cudaSuccess) return bp_set_cuda_error(e, err, "digest: scratch");
    uint32_t* h = bp_pinned_get(e);
    if (!h) return bp_set_error(e, BP_ERR_NOMEM, "digest: pinned read-back slot");
    err = cudaMemsetAsync(e->d_digest, 0, 2 * sizeof(unsigned long long), st);
    if (err == cudaSuccess) {
        const int64_t words = 5 * (int64_t)n + 2;
        const int blocks = (int)std::min<int64_t>((int64_t)e->sm_count * 8, std::max<int64_t>(1, words / 1024));
        digest_kernel<<<blocks, 256, 0, st>>>(d_counters, n, d_hsp_off, d_hsps, first, rec_base, last ? 1 : 0,
                                              e->d_digest);
        e->launches += 1;
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemcpyAsync(h, e->d_digest, 16, cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err == cudaSuccess) memcpy(sums, h, 16);
    bp_pinned_put(e, h);
    if (err != cudaSuccess) return bp_set_cuda_error(e, err, "digest");
    return BP_OK;
}

void bp_digest_finish(const uint64_t sums[2], int64_t n_subjects, uint64_t out[2]) {
    out[0] = sums[0] ^ ((uint64_t)(uint32_t)n_subjects << 32);
    out[1] = sums[1];
}

bp_status bp_digest_range(bp_engine* e, cudaStream_t st, const int32_t* d_counters, int32_t n,
                          const int64_t* d_hsp_off, const bp_hsp* d_hsps, uint64_t out[2]) {
    if (!out) return BP_ERR_INVALID;
    uint64_t sums[2];
    const bp_status s = bp_digest_sums(e, st, d_counters, n, d_hsp_off, d_hsps, 0, 0, true, sums);
    if (s != BP_OK) return s;
    bp_digest_finish(sums, n, out);
    return BP_OK;
}

bp_status bp_result_digest(bp_result* r, uint64_t out[2]) {
    if (!r || !out) return BP_ERR_INVALID;
    bp_status s = bp_result_wait(r);
    if (s != BP_OK) return s;
    return bp_digest_range(r->e, r->e->stream, r->d_counters, r->n, r->d_hsp_off, r->d_hsps, out);
}
