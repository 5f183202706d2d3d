// Learned cost model for the batched search's schedule: features of each
// (query, subject chunk) work item, and a two-layer MLP (ReLU hidden layer,
// fp32) that predicts the item's word-hit and extension counts, trained on
// the device with the kernels below (forward, backward, Adam).
//
// The reference has no counterpart: it launches one query at a time and
// splits subjects across threads by a fixed stride (gpu_blastp_kernel.cu:64).
//
// Training is deterministic: the per-row pass writes each row's
// pre-activations and error terms, and the weight-gradient pass gives every
// parameter one thread that sums its row terms in row order, so the same
// data and seed give bit-identical weights.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <random>
#include <vector>

#include "bp_internal.h"

#define CKM(call, what)                                                   \
    do {                                                                  \
        cudaError_t _err = (call);                                        \
        if (_err != cudaSuccess) return bp_set_cuda_error(e, _err, what); \
    } while (0)

namespace {

constexpr int kMaxIn = 64, kMaxHidden = 128, kMaxOut = 4;

// Residue counts of each chunk (subjects chunk_first[c] .. chunk_first[c+1]),
// 28 bins.  One CTA per chunk; per-warp private histograms in shared memory.
__global__ void chunk_histogram(const uint8_t* __restrict__ res, const int64_t* __restrict__ off,
                                const int32_t* __restrict__ chunk_first, int32_t n_chunks, uint32_t* __restrict__ out) {
    __shared__ uint32_t h[8][32];
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 8 * 32; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    for (int c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const int64_t lo = off[chunk_first[c]], hi = off[chunk_first[c + 1]];
        const int64_t a16 = (lo + 15) & ~15LL, b16 = hi & ~15LL;
        if (a16 < b16) {
            for (int64_t i = lo + threadIdx.x; i < a16; i += blockDim.x) atomicAdd(&h[warp][res[i]], 1u);
            for (int64_t i = a16 / 16 + threadIdx.x; i < b16 / 16; i += blockDim.x) {
                const uint4 v = reinterpret_cast<const uint4*>(res)[i];
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int j = 0; j < 4; ++j) atomicAdd(&h[warp][(w[k] >> (8 * j)) & 31u], 1u);
            }
            for (int64_t i = b16 + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&h[warp][res[i]], 1u);
        } else {
            for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) atomicAdd(&h[warp][res[i]], 1u);
        }
        __syncthreads();
        if (threadIdx.x < 28) {
            uint32_t s = 0;
            for (int w = 0; w < 8; ++w) s += h[w][threadIdx.x];
            out[(int64_t)c * 28 + threadIdx.x] = s;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < 8 * 32; i += blockDim.x) (&h[0][0])[i] = 0;
        __syncthreads();
    }
}

// Parameter block layout: W1[in][hid], b1[hid], W2[hid][out], b2[out].
struct MlpDims {
    int in, hid, out;
    __host__ __device__ int n_params() const { return in * hid + hid + hid * out + out; }
    __host__ __device__ int w1() const { return 0; }
    __host__ __device__ int b1() const { return in * hid; }
    __host__ __device__ int w2() const { return in * hid + hid; }
    __host__ __device__ int b2() const { return in * hid + hid + hid * out; }
};

// Forward pass of rows idx[0..n) (or 0..n when idx is null); with targets,
// also the backward pass down to the hidden pre-activations:
//   dy = 2 (y - t) / (n * out),  dz = (dy W2^T) * [z > 0].
// Writes x (gathered), z, dz, dy and each row's squared error.
__global__ void mlp_rows(MlpDims d, const float* __restrict__ p, const float* __restrict__ X,
                         const float* __restrict__ T, const int32_t* __restrict__ idx, int n, float* __restrict__ xg,
                         float* __restrict__ Z, float* __restrict__ DZ, float* __restrict__ DY, float* __restrict__ Yout,
                         float* __restrict__ sqerr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int src = idx ? idx[r] : r;
    float x[kMaxIn];
    for (int i = 0; i < d.in; ++i) {
        x[i] = X[(int64_t)src * d.in + i];
        if (xg) xg[(int64_t)r * d.in + i] = x[i];
    }
    float y[kMaxOut];
    for (int o = 0; o < d.out; ++o) y[o] = p[d.b2() + o];
    for (int j = 0; j < d.hid; ++j) {
        float z = p[d.b1() + j];
        for (int i = 0; i < d.in; ++i) z = fmaf(x[i], p[d.w1() + i * d.hid + j], z);
        if (Z) Z[(int64_t)r * d.hid + j] = z;
        const float h = z > 0.f ? z : 0.f;
        for (int o = 0; o < d.out; ++o) y[o] = fmaf(h, p[d.w2() + j * d.out + o], y[o]);
    }
    if (Yout)
        for (int o = 0; o < d.out; ++o) Yout[(int64_t)r * d.out + o] = y[o];
    if (!T) return;
    const float scale = 2.f / ((float)n * (float)d.out);
    float dy[kMaxOut], se = 0.f;
    for (int o = 0; o < d.out; ++o) {
        const float e = y[o] - T[(int64_t)src * d.out + o];
        se = fmaf(e, e, se);
        dy[o] = scale * e;
        DY[(int64_t)r * d.out + o] = dy[o];
    }
    sqerr[r] = se;
    for (int j = 0; j < d.hid; ++j) {
        const float z = Z[(int64_t)r * d.hid + j];
        float g = 0.f;
        if (z > 0.f)
            for (int o = 0; o < d.out; ++o) g = fmaf(dy[o], p[d.w2() + j * d.out + o], g);
        DZ[(int64_t)r * d.hid + j] = g;
    }
}

// Weight gradients: one thread per parameter, summing its row terms in row
// order (deterministic).  Thread n_params sums the squared errors into loss.
__global__ void mlp_param_grads(MlpDims d, const float* __restrict__ xg, const float* __restrict__ Z,
                                const float* __restrict__ DZ, const float* __restrict__ DY,
                                const float* __restrict__ sqerr, int n, float* __restrict__ grad,
                                float* __restrict__ loss) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = d.n_params();
    if (k > np) return;
    float s = 0.f;
    if (k == np) {
        for (int r = 0; r < n; ++r) s += sqerr[r];
        *loss = s / ((float)n * (float)d.out);
        return;
    }
    if (k < d.b1()) {                       // W1[i][j] = sum_r x[r][i] dz[r][j]
        const int i = k / d.hid, j = k % d.hid;
        for (int r = 0; r < n; ++r) s = fmaf(xg[(int64_t)r * d.in + i], DZ[(int64_t)r * d.hid + j], s);
    } else if (k < d.w2()) {                // b1[j] = sum_r dz[r][j]
        const int j = k - d.b1();
        for (int r = 0; r < n; ++r) s += DZ[(int64_t)r * d.hid + j];
    } else if (k < d.b2()) {                // W2[j][o] = sum_r relu(z[r][j]) dy[r][o]
        const int j = (k - d.w2()) / d.out, o = (k - d.w2()) % d.out;
        for (int r = 0; r < n; ++r) {
            const float z = Z[(int64_t)r * d.hid + j];
            if (z > 0.f) s = fmaf(z, DY[(int64_t)r * d.out + o], s);
        }
    } else {                                // b2[o] = sum_r dy[r][o]
        const int o = k - d.b2();
        for (int r = 0; r < n; ++r) s += DY[(int64_t)r * d.out + o];
    }
    grad[k] = s;
}

// Adam (Kingma & Ba 2015), bias-corrected step sizes passed in.
__global__ void adam_step(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                          float* __restrict__ v, int n, float lr_t, float b1, float b2, float eps) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr_t * mk / (sqrtf(vk) + eps);
}

}  // namespace

struct bp_mlp {
    bp_engine* e = nullptr;
    MlpDims d{};
    float* d_p = nullptr;     // parameters
    float* d_g = nullptr;     // gradient
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_loss = nullptr;
    int64_t step = 0;
    // per-row scratch
    int32_t cap = 0;
    float *d_xg = nullptr, *d_z = nullptr, *d_dz = nullptr, *d_dy = nullptr, *d_y = nullptr, *d_se = nullptr;
    int32_t* d_idx = nullptr;
    // data
    int64_t data_cap = 0;
    float *d_X = nullptr, *d_T = nullptr;
    // standardisation (identity until fit sets it)
    std::vector<float> x_mean, x_std, y_mean, y_std;
};

namespace {

bp_status mlp_reserve(bp_mlp* m, int32_t rows) {
    bp_engine* e = m->e;
    if (rows <= m->cap) return BP_OK;
    cudaFree(m->d_xg);
    cudaFree(m->d_z);
    cudaFree(m->d_dz);
    cudaFree(m->d_dy);
    cudaFree(m->d_y);
    cudaFree(m->d_se);
    cudaFree(m->d_idx);
    m->cap = 0;
    const size_t r = (size_t)rows;
    CKM(cudaMalloc((void**)&m->d_xg, r * m->d.in * sizeof(float)), "cudaMalloc(mlp)");
    CKM(cudaMalloc((void**)&m->d_z, r * m->d.hid * sizeof(float)), "cudaMalloc(mlp)");
    CKM(cudaMalloc((void**)&m->d_dz, r * m->d.hid * sizeof(float)), "cudaMalloc(mlp)");
    CKM(cudaMalloc((void**)&m->d_dy, r * m->d.out * sizeof(float)), "cudaMalloc(mlp)");
    CKM(cudaMalloc((void**)&m->d_y, r * m->d.out * sizeof(float)), "cudaMalloc(mlp)");
    CKM(cudaMalloc((void**)&m->d_se, r * sizeof(float)), "cudaMalloc(mlp)");
    CKM(cudaMalloc((void**)&m->d_idx, r * sizeof(int32_t)), "cudaMalloc(mlp)");
    m->cap = rows;
    return BP_OK;
}

bp_status mlp_upload(bp_mlp* m, const float* X, const float* T, int32_t n) {
    bp_engine* e = m->e;
    if (n > m->data_cap) {
        cudaFree(m->d_X);
        cudaFree(m->d_T);
        m->d_X = m->d_T = nullptr;
        m->data_cap = 0;
        CKM(cudaMalloc((void**)&m->d_X, (size_t)n * m->d.in * sizeof(float)), "cudaMalloc(mlp data)");
        CKM(cudaMalloc((void**)&m->d_T, (size_t)n * m->d.out * sizeof(float)), "cudaMalloc(mlp data)");
        m->data_cap = n;
    }
    CKM(cudaMemcpyAsync(m->d_X, X, (size_t)n * m->d.in * sizeof(float), cudaMemcpyHostToDevice, e->stream),
        "upload features");
    if (T)
        CKM(cudaMemcpyAsync(m->d_T, T, (size_t)n * m->d.out * sizeof(float), cudaMemcpyHostToDevice, e->stream),
            "upload targets");
    return BP_OK;
}

// One gradient evaluation over rows idx (device, or null for 0..n) of the
// uploaded data; leaves the gradient in d_g and the loss in d_loss.
bp_status mlp_grad(bp_mlp* m, const int32_t* d_idx, int32_t n) {
    bp_engine* e = m->e;
    mlp_rows<<<(n + 127) / 128, 128, 0, e->stream>>>(m->d, m->d_p, m->d_X, m->d_T, d_idx, n, m->d_xg, m->d_z,
                                                     m->d_dz, m->d_dy, nullptr, m->d_se);
    const int np = m->d.n_params();
    mlp_param_grads<<<(np + 1 + 127) / 128, 128, 0, e->stream>>>(m->d, m->d_xg, m->d_z, m->d_dz, m->d_dy, m->d_se,
                                                                  n, m->d_g, m->d_loss);
    e->launches += 2;
    CKM(cudaGetLastError(), "mlp gradient launch");
    return BP_OK;
}

}  // namespace

extern "C" {

bp_status bp_mlp_create(bp_engine* e, int32_t n_in, int32_t n_hidden, int32_t n_out, uint64_t seed, bp_mlp** out) {
    if (!e || !out || n_in < 1 || n_in > kMaxIn || n_hidden < 1 || n_hidden > kMaxHidden || n_out < 1 ||
        n_out > kMaxOut)
        return bp_set_error(e, BP_ERR_INVALID, "bp_mlp_create: sizes must be in 1..64 / 1..128 / 1..4");
    *out = nullptr;
    CKM(cudaSetDevice(e->device), "cudaSetDevice");
    bp_mlp* m = new bp_mlp();
    m->e = e;
    m->d = MlpDims{n_in, n_hidden, n_out};
    const int np = m->d.n_params();
    // He-uniform first layer, Glorot-uniform second, zero biases
    std::vector<float> p(np, 0.f);
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<float> u(-1.f, 1.f);
    const float a1 = sqrtf(6.f / n_in), a2 = sqrtf(6.f / (n_hidden + n_out));
    for (int k = 0; k < n_in * n_hidden; ++k) p[m->d.w1() + k] = a1 * u(rng);
    for (int k = 0; k < n_hidden * n_out; ++k) p[m->d.w2() + k] = a2 * u(rng);
    m->x_mean.assign(n_in, 0.f);
    m->x_std.assign(n_in, 1.f);
    m->y_mean.assign(n_out, 0.f);
    m->y_std.assign(n_out, 1.f);
    cudaError_t err = cudaMalloc((void**)&m->d_p, np * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc((void**)&m->d_g, np * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc((void**)&m->d_m, np * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc((void**)&m->d_v, np * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc((void**)&m->d_loss, sizeof(float));
    if (err == cudaSuccess) err = cudaMemcpy(m->d_p, p.data(), np * sizeof(float), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(m->d_m, 0, np * sizeof(float));
    if (err == cudaSuccess) err = cudaMemset(m->d_v, 0, np * sizeof(float));
    if (err != cudaSuccess) {
        bp_mlp_destroy(m);
        return bp_set_cuda_error(e, err, "bp_mlp_create");
    }
    *out = m;
    return BP_OK;
}

void bp_mlp_destroy(bp_mlp* m) {
    if (!m) return;
    if (m->e) cudaStreamSynchronize(m->e->stream);
    for (float* p : {m->d_p, m->d_g, m->d_m, m->d_v, m->d_loss, m->d_xg, m->d_z, m->d_dz, m->d_dy, m->d_y, m->d_se,
                     m->d_X, m->d_T})
        cudaFree(p);
    cudaFree(m->d_idx);
    delete m;
}

int32_t bp_mlp_num_params(const bp_mlp* m) { return m ? m->d.n_params() : 0; }

bp_status bp_mlp_get_params(bp_mlp* m, float* params, float* norm) {
    if (!m) return BP_ERR_INVALID;
    bp_engine* e = m->e;
    if (params) {
        CKM(cudaStreamSynchronize(e->stream), "mlp sync");
        CKM(cudaMemcpy(params, m->d_p, m->d.n_params() * sizeof(float), cudaMemcpyDeviceToHost), "read params");
    }
    if (norm) {   // x_mean[in], x_std[in], y_mean[out], y_std[out]
        float* q = norm;
        for (float v : m->x_mean) *q++ = v;
        for (float v : m->x_std) *q++ = v;
        for (float v : m->y_mean) *q++ = v;
        for (float v : m->y_std) *q++ = v;
    }
    return BP_OK;
}

bp_status bp_mlp_set_params(bp_mlp* m, const float* params, const float* norm) {
    if (!m) return BP_ERR_INVALID;
    bp_engine* e = m->e;
    if (params) {
        CKM(cudaStreamSynchronize(e->stream), "mlp sync");
        CKM(cudaMemcpy(m->d_p, params, m->d.n_params() * sizeof(float), cudaMemcpyHostToDevice), "write params");
        CKM(cudaMemset(m->d_m, 0, m->d.n_params() * sizeof(float)), "reset adam");
        CKM(cudaMemset(m->d_v, 0, m->d.n_params() * sizeof(float)), "reset adam");
        m->step = 0;
    }
    if (norm) {
        const float* q = norm;
        for (float& v : m->x_mean) v = *q++;
        for (float& v : m->x_std) v = *q++;
        for (float& v : m->y_mean) v = *q++;
        for (float& v : m->y_std) v = *q++;
    }
    return BP_OK;
}

// Loss L = 1/(n*out) sum (y - t)^2 and its gradient with respect to the raw
// parameters, on raw (unstandardised) inputs and targets.
bp_status bp_mlp_loss_grad(bp_mlp* m, const float* X, const float* T, int32_t n, float* loss, float* grad) {
    if (!m || !X || !T || n < 1) return BP_ERR_INVALID;
    bp_engine* e = m->e;
    CKM(cudaSetDevice(e->device), "cudaSetDevice");
    bp_status st = mlp_reserve(m, n);
    if (st == BP_OK) st = mlp_upload(m, X, T, n);
    if (st == BP_OK) st = mlp_grad(m, nullptr, n);
    if (st != BP_OK) return st;
    if (loss) CKM(cudaMemcpyAsync(loss, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, e->stream), "read loss");
    if (grad)
        CKM(cudaMemcpyAsync(grad, m->d_g, m->d.n_params() * sizeof(float), cudaMemcpyDeviceToHost, e->stream),
            "read grad");
    CKM(cudaStreamSynchronize(e->stream), "mlp gradient");
    return BP_OK;
}

// Standardises X and T (per column), then trains with Adam on shuffled
// minibatches.  loss_curve (optional, epochs entries) gets each epoch's mean
// minibatch loss in standardised units.
bp_status bp_mlp_fit(bp_mlp* m, const float* X, const float* T, int32_t n, int32_t epochs, int32_t batch, float lr,
                     uint64_t seed, float* loss_curve) {
    if (!m || !X || !T || n < 1 || epochs < 0 || batch < 1) return BP_ERR_INVALID;
    bp_engine* e = m->e;
    CKM(cudaSetDevice(e->device), "cudaSetDevice");
    const int in = m->d.in, out = m->d.out;
    std::vector<double> xs(in, 0), xq(in, 0), ys(out, 0), yq(out, 0);
    for (int32_t r = 0; r < n; ++r) {
        for (int i = 0; i < in; ++i) { const double v = X[(int64_t)r * in + i]; xs[i] += v; xq[i] += v * v; }
        for (int o = 0; o < out; ++o) { const double v = T[(int64_t)r * out + o]; ys[o] += v; yq[o] += v * v; }
    }
    for (int i = 0; i < in; ++i) {
        m->x_mean[i] = (float)(xs[i] / n);
        const double var = xq[i] / n - (xs[i] / n) * (xs[i] / n);
        m->x_std[i] = var > 1e-12 ? (float)sqrt(var) : 1.f;
    }
    for (int o = 0; o < out; ++o) {
        m->y_mean[o] = (float)(ys[o] / n);
        const double var = yq[o] / n - (ys[o] / n) * (ys[o] / n);
        m->y_std[o] = var > 1e-12 ? (float)sqrt(var) : 1.f;
    }
    std::vector<float> xn((size_t)n * in), tn((size_t)n * out);
    for (int32_t r = 0; r < n; ++r) {
        for (int i = 0; i < in; ++i) xn[(size_t)r * in + i] = (X[(size_t)r * in + i] - m->x_mean[i]) / m->x_std[i];
        for (int o = 0; o < out; ++o) tn[(size_t)r * out + o] = (T[(size_t)r * out + o] - m->y_mean[o]) / m->y_std[o];
    }
    const int32_t bs = std::min(batch, n);
    bp_status st = mlp_reserve(m, std::max(bs, n));
    if (st == BP_OK) st = mlp_upload(m, xn.data(), tn.data(), n);
    if (st != BP_OK) return st;
    std::vector<int32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(seed);
    const int np = m->d.n_params();
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    std::vector<float> losses;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        CKM(cudaMemcpyAsync(m->d_idx, perm.data(), (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, e->stream),
            "upload permutation");
        double ep_loss = 0;
        int n_batches = 0;
        std::vector<float> bl;
        for (int32_t b0 = 0; b0 + bs <= n; b0 += bs) {   // full minibatches only
            st = mlp_grad(m, m->d_idx + b0, bs);
            if (st != BP_OK) return st;
            ++m->step;
            const float lr_t = lr * (float)(sqrt(1.0 - pow(b2, (double)m->step)) / (1.0 - pow(b1, (double)m->step)));
            adam_step<<<(np + 255) / 256, 256, 0, e->stream>>>(m->d_p, m->d_g, m->d_m, m->d_v, np, lr_t, b1, b2, eps);
            e->launches += 1;
            CKM(cudaGetLastError(), "adam launch");
            if (loss_curve) {
                float l = 0.f;
                CKM(cudaMemcpyAsync(&l, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost, e->stream), "read loss");
                CKM(cudaStreamSynchronize(e->stream), "mlp step");
                ep_loss += l;
            }
            ++n_batches;
        }
        if (loss_curve) loss_curve[ep] = n_batches ? (float)(ep_loss / n_batches) : 0.f;
    }
    CKM(cudaStreamSynchronize(e->stream), "mlp fit");
    return BP_OK;
}

// Predictions for raw features (standardisation applied, outputs mapped back).
bp_status bp_mlp_predict(bp_mlp* m, const float* X, int32_t n, float* Y) {
    if (!m || !X || !Y || n < 0) return BP_ERR_INVALID;
    if (n == 0) return BP_OK;
    bp_engine* e = m->e;
    CKM(cudaSetDevice(e->device), "cudaSetDevice");
    const int in = m->d.in, out = m->d.out;
    std::vector<float> xn((size_t)n * in);
    for (int32_t r = 0; r < n; ++r)
        for (int i = 0; i < in; ++i) xn[(size_t)r * in + i] = (X[(size_t)r * in + i] - m->x_mean[i]) / m->x_std[i];
    bp_status st = mlp_reserve(m, n);
    if (st == BP_OK) st = mlp_upload(m, xn.data(), nullptr, n);
    if (st != BP_OK) return st;
    mlp_rows<<<(n + 127) / 128, 128, 0, e->stream>>>(m->d, m->d_p, m->d_X, nullptr, nullptr, n, nullptr, nullptr,
                                                     nullptr, nullptr, m->d_y, nullptr);
    e->launches += 1;
    CKM(cudaGetLastError(), "mlp forward launch");
    CKM(cudaMemcpyAsync(Y, m->d_y, (size_t)n * out * sizeof(float), cudaMemcpyDeviceToHost, e->stream),
        "read predictions");
    CKM(cudaStreamSynchronize(e->stream), "mlp forward");
    for (int32_t r = 0; r < n; ++r)
        for (int o = 0; o < out; ++o) Y[(size_t)r * out + o] = Y[(size_t)r * out + o] * m->y_std[o] + m->y_mean[o];
    return BP_OK;
}

// Residue counts per chunk (28 bins), computed on the device.
bp_status bp_db_chunk_histograms(bp_engine* e, const bp_db* db, const int32_t* chunk_first, int32_t n_chunks,
                                 uint32_t* counts) {
    if (!e || !db || !chunk_first || n_chunks < 0 || !counts) return BP_ERR_INVALID;
    for (int32_t c = 0; c < n_chunks; ++c)
        if (chunk_first[c] < 0 || chunk_first[c] > chunk_first[c + 1] || chunk_first[c + 1] > db->n)
            return bp_set_error(e, BP_ERR_INVALID, "bp_db_chunk_histograms: bad chunk boundaries");
    if (n_chunks == 0) return BP_OK;
    bp_db* mdb = const_cast<bp_db*>(db);
    {
        std::lock_guard<std::mutex> lock(mdb->hist_mu);
        if (mdb->hist_first.size() == (size_t)n_chunks + 1 &&
            std::equal(mdb->hist_first.begin(), mdb->hist_first.end(), chunk_first)) {
            memcpy(counts, mdb->hist.data(), (size_t)n_chunks * 28 * sizeof(uint32_t));
            return BP_OK;
        }
    }
    CKM(cudaSetDevice(e->device), "cudaSetDevice");
    int32_t* d_first = nullptr;
    uint32_t* d_counts = nullptr;
    CKM(cudaMallocAsync((void**)&d_first, ((size_t)n_chunks + 1) * sizeof(int32_t), e->stream), "cudaMallocAsync");
    CKM(cudaMallocAsync((void**)&d_counts, (size_t)n_chunks * 28 * sizeof(uint32_t), e->stream), "cudaMallocAsync");
    CKM(cudaMemcpyAsync(d_first, chunk_first, ((size_t)n_chunks + 1) * sizeof(int32_t), cudaMemcpyHostToDevice,
                        e->stream),
        "upload chunks");
    chunk_histogram<<<std::min(n_chunks, e->sm_count * 8), 256, 0, e->stream>>>(db->d_res, db->d_off, d_first,
                                                                               n_chunks, d_counts);
    e->launches += 1;
    CKM(cudaGetLastError(), "histogram launch");
    CKM(cudaMemcpyAsync(counts, d_counts, (size_t)n_chunks * 28 * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                        e->stream),
        "read histograms");
    cudaFreeAsync(d_first, e->stream);
    cudaFreeAsync(d_counts, e->stream);
    CKM(cudaStreamSynchronize(e->stream), "histograms");
    std::lock_guard<std::mutex> lock(mdb->hist_mu);
    mdb->hist_first.assign(chunk_first, chunk_first + n_chunks + 1);
    mdb->hist.assign(counts, counts + (size_t)n_chunks * 28);
    return BP_OK;
}

// Cost-model features of every (query, chunk) item, row q * n_chunks + c:
//   [0] log(1 + query length)      [1] log(1 + neighbour-word entries)
//   [2] log(1 + chunk residues)    [3..22] chunk composition over the 20
//   standard residues (fractions)  [23] planted-homolog density (caller's)
bp_status bp_batch_features(bp_engine* e, const bp_db* db, const bp_query* const* queries, int32_t n_queries,
                            const int32_t* chunk_first, int32_t n_chunks, float planted_density, float* X) {
    if (!e || !db || (!queries && n_queries > 0) || n_queries < 0 || !chunk_first || n_chunks < 0 || !X)
        return BP_ERR_INVALID;
    std::vector<uint32_t> h((size_t)n_chunks * 28);
    bp_status st = bp_db_chunk_histograms(e, db, chunk_first, n_chunks, h.data());
    if (st != BP_OK) return st;
    // NCBIstdaa codes of the 20 standard amino acids, alphabetical by letter
    static const int std20[20] = {1, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 22};
    std::vector<float> chunk_f((size_t)n_chunks * 21);
    for (int32_t c = 0; c < n_chunks; ++c) {
        const int64_t len = db->h_off[chunk_first[c + 1]] - db->h_off[chunk_first[c]];
        chunk_f[(size_t)c * 21] = logf(1.f + (float)len);
        for (int k = 0; k < 20; ++k)
            chunk_f[(size_t)c * 21 + 1 + k] = len > 0 ? (float)h[(size_t)c * 28 + std20[k]] / (float)len : 0.f;
    }
    for (int32_t q = 0; q < n_queries; ++q) {
        const float f0 = logf(1.f + (float)queries[q]->qlen), f1 = logf(1.f + (float)queries[q]->n_entries);
        for (int32_t c = 0; c < n_chunks; ++c) {
            float* x = X + ((size_t)q * n_chunks + c) * BP_COST_FEATURES;
            x[0] = f0;
            x[1] = f1;
            memcpy(x + 2, &chunk_f[(size_t)c * 21], 21 * sizeof(float));
            x[23] = planted_density;
        }
    }
    return BP_OK;
}

}  // extern "C"
