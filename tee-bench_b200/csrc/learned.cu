// LRN: learned skew-aware partitioning for sm_100a.
//
// A small FP32 MLP (1 -> 32 -> 32 -> 1, tanh) models the frequency of S's
// keys: log2(rows of S with key k) / 32 as a function of log2(k + 1) / 16 - 1,
// trained per join on the keys a seeded 1% sample of S repeats, by the kernels
// in this file (forward, backward, Adam; the trainer is one 8-CTA thread-block
// cluster that all-reduces gradients through distributed shared memory).
// The model predicts how many S rows each candidate key has; keys predicted
// above a threshold are flagged heavy.  Heavy keys never enter the radix
// partitions: their (R, S) pairs are joined in the histogram read itself,
// split across every CTA that streams S, against a shared-memory table of
// their R rows.  The remaining rows are radix partitioned and joined as in
// RHO.  The model only chooses which keys take the heavy path; every row's
// destination is decided by an exact key comparison, so results are exact
// whatever the model predicts.  When the model predicts too little heavy
// mass, the host falls back to plain radix partitioning.
#include <cooperative_groups.h>

#include "tbg_device.cuh"
#include "tbg_learned.h"

namespace cg = cooperative_groups;

namespace tbg {

// ---------------------------------------------------------------------------
// model
// ---------------------------------------------------------------------------
// parameter layout: W1[H], b1[H], W2[H][H] (row o, column i), b2[H], W3[H], b3
__device__ __forceinline__ float tanh_f(float x) { return tanhf(x); }

__device__ float mlp_forward(const float *__restrict__ p, float x, float *h1, float *h2) {
    const float *W1 = p, *b1 = p + MLP_H, *W2 = p + 2 * MLP_H, *b2 = W2 + MLP_H * MLP_H, *W3 = b2 + MLP_H,
                *b3 = W3 + MLP_H;
#pragma unroll
    for (int i = 0; i < MLP_H; i++) h1[i] = tanh_f(W1[i] * x + b1[i]);
    float out = b3[0];
#pragma unroll 4
    for (int o = 0; o < MLP_H; o++) {
        float z = b2[o];
#pragma unroll
        for (int i = 0; i < MLP_H; i++) z += W2[o * MLP_H + i] * h1[i];
        h2[o] = tanh_f(z);
        out += W3[o] * h2[o];
    }
    return out;
}

__device__ float mlp_eval(const float *__restrict__ p, float x) {
    float h1[MLP_H], h2[MLP_H];
    return mlp_forward(p, x, h1, h2);
}

// Backward of one sample for output gradient dout: fills dz2 (pre-activation
// gradient of layer 2) and dz1 (of layer 1).
__device__ void mlp_backward(const float *__restrict__ p, const float *h1, const float *h2, float dout,
                             float *dz2, float *dz1) {
    const float *W2 = p + 2 * MLP_H, *b2 = W2 + MLP_H * MLP_H, *W3 = b2 + MLP_H;
#pragma unroll
    for (int o = 0; o < MLP_H; o++) dz2[o] = dout * W3[o] * (1.f - h2[o] * h2[o]);
#pragma unroll 4
    for (int i = 0; i < MLP_H; i++) {
        float dh = 0.f;
#pragma unroll
        for (int o = 0; o < MLP_H; o++) dh += W2[o * MLP_H + i] * dz2[o];
        dz1[i] = dh * (1.f - h1[i] * h1[i]);
    }
}

// Per-sample activations of a CTA's batch, stored for the parameter
// gradient reductions: row s = sample s (padded to 33 floats against bank
// conflicts).
struct BatchSmem {
    float h1[MLP_BATCH_CTA][MLP_H + 1];
    float h2[MLP_BATCH_CTA][MLP_H + 1];
    float dz2[MLP_BATCH_CTA][MLP_H + 1];
    float dz1[MLP_BATCH_CTA][MLP_H + 1];
    float x[MLP_BATCH_CTA];
    float dout[MLP_BATCH_CTA];
};

// Sum over s < nb of a[s] * b[s] (or of a[s] when b is null) read with the
// given row strides, in four independent partial sums (the loop is latency
// bound otherwise).
__device__ __forceinline__ float dot_rows(const float *a, int sa, const float *bb, int sb, int nb) {
    float g0 = 0.f, g1 = 0.f, g2 = 0.f, g3 = 0.f;
    int s = 0;
    if (bb) {
        for (; s + 4 <= nb; s += 4) {
            g0 += a[s * sa] * bb[s * sb];
            g1 += a[(s + 1) * sa] * bb[(s + 1) * sb];
            g2 += a[(s + 2) * sa] * bb[(s + 2) * sb];
            g3 += a[(s + 3) * sa] * bb[(s + 3) * sb];
        }
        for (; s < nb; s++) g0 += a[s * sa] * bb[s * sb];
    } else {
        for (; s + 4 <= nb; s += 4) {
            g0 += a[s * sa];
            g1 += a[(s + 1) * sa];
            g2 += a[(s + 2) * sa];
            g3 += a[(s + 3) * sa];
        }
        for (; s < nb; s++) g0 += a[s * sa];
    }
    return (g0 + g1) + (g2 + g3);
}

// Gradient of parameter q summed over the nb samples in `b`.
__device__ __forceinline__ float param_grad(const BatchSmem &b, int q, int nb) {
    constexpr int RS = MLP_H + 1;  // row stride of the activation arrays
    if (q < MLP_H) return dot_rows(&b.dz1[0][q], RS, b.x, 1, nb);                 // W1[i]
    if (q < 2 * MLP_H) return dot_rows(&b.dz1[0][q - MLP_H], RS, nullptr, 0, nb);  // b1[i]
    if (q < 2 * MLP_H + MLP_H * MLP_H) {                                           // W2[o][i]
        const int o = (q - 2 * MLP_H) / MLP_H, i = (q - 2 * MLP_H) % MLP_H;
        return dot_rows(&b.dz2[0][o], RS, &b.h1[0][i], RS, nb);
    }
    if (q < 3 * MLP_H + MLP_H * MLP_H) return dot_rows(&b.dz2[0][q - 2 * MLP_H - MLP_H * MLP_H], RS, nullptr, 0, nb);
    if (q < 4 * MLP_H + MLP_H * MLP_H) return dot_rows(b.dout, 1, &b.h2[0][q - 3 * MLP_H - MLP_H * MLP_H], RS, nb);
    return dot_rows(b.dout, 1, nullptr, 0, nb);                                    // b3
}

// One sample's forward + backward, activations stored in row `s`.
__device__ float sample_fwd_bwd(const float *p, float x, float y, float scale, BatchSmem &b, int s) {
    float h1[MLP_H], h2[MLP_H], dz2[MLP_H], dz1[MLP_H];
    const float out = mlp_forward(p, x, h1, h2);
    const float r = out - y;
    const float dout = 2.f * r * scale;
    mlp_backward(p, h1, h2, dout, dz2, dz1);
#pragma unroll
    for (int i = 0; i < MLP_H; i++) {
        b.h1[s][i] = h1[i];
        b.h2[s][i] = h2[i];
        b.dz2[s][i] = dz2[i];
        b.dz1[s][i] = dz1[i];
    }
    b.x[s] = x;
    b.dout[s] = dout;
    return r * r;
}

// Full-batch gradient and loss sum over n samples (tests and the reported
// training loss): CTAs take MLP_BATCH_CTA samples each and add their partial
// gradients to grad[] with atomics.
__global__ void __launch_bounds__(MLP_BATCH_CTA) k_mlp_grad(const float *__restrict__ params,
                                                            const float *__restrict__ xs,
                                                            const float *__restrict__ ys, uint32_t n,
                                                            float *grad, float *loss_sum) {
    extern __shared__ __align__(16) unsigned char smem[];
    float *p = reinterpret_cast<float *>(smem);
    BatchSmem &b = *reinterpret_cast<BatchSmem *>(p + MLP_PARAMS_PAD);
    for (int q = threadIdx.x; q < MLP_PARAMS; q += MLP_BATCH_CTA) p[q] = params[q];
    __syncthreads();
    const uint32_t s0 = blockIdx.x * MLP_BATCH_CTA;
    const int nb = (int)min((uint32_t)MLP_BATCH_CTA, n - s0);
    float l = 0.f;
    if ((int)threadIdx.x < nb) {
        const uint32_t i = s0 + threadIdx.x;
        l = sample_fwd_bwd(p, xs[i], ys[i], 1.f / (float)n, b, threadIdx.x);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < MLP_PARAMS; q += MLP_BATCH_CTA) atomicAdd(&grad[q], param_grad(b, q, nb));
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss_sum, l);
}

// Trainer: one cluster of MLP_CLUSTER CTAs, persistent over all steps.  Each
// step every CTA draws MLP_BATCH_CTA seeded random training points, computes
// their forward/backward and its partial parameter gradient; after a cluster
// barrier CTA r sums the partials of its parameter slice from every CTA's
// shared memory, applies Adam, and writes the new values into every CTA's
// parameter copy; a second barrier ends the step.
__global__ void __cluster_dims__(MLP_CLUSTER, 1, 1) __launch_bounds__(MLP_BATCH_CTA)
    k_mlp_train(const float *__restrict__ xs, const float *__restrict__ ys, uint32_t n, float *params,
                int steps, float lr0, uint64_t seed) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    extern __shared__ __align__(16) unsigned char smem[];
    float *p = reinterpret_cast<float *>(smem);
    float *gpart = p + MLP_PARAMS_PAD;
    float *am = gpart + MLP_PARAMS_PAD;  // Adam moments of this CTA's slice
    float *av = am + MLP_SLICE;
    BatchSmem &b = *reinterpret_cast<BatchSmem *>(av + MLP_SLICE);
    const int tid = threadIdx.x;
    for (int q = tid; q < MLP_PARAMS; q += MLP_BATCH_CTA) p[q] = params[q];
    for (int q = tid; q < MLP_SLICE; q += MLP_BATCH_CTA) am[q] = av[q] = 0.f;
    cl.sync();
    const float b1c = 0.9f, b2c = 0.999f, eps = 1e-8f;
    const float scale = 1.f / (float)(MLP_BATCH_CTA * MLP_CLUSTER);
    const int q0 = rank * MLP_SLICE, q1 = min(MLP_PARAMS, q0 + MLP_SLICE);
    float pow1 = 1.f, pow2 = 1.f;
    for (int step = 0; step < steps; step++) {
        const uint64_t h = mix64(seed ^ mix64(((uint64_t)step << 20) | (uint64_t)(rank * MLP_BATCH_CTA + tid)));
        const uint32_t i = (uint32_t)(h % n);
        sample_fwd_bwd(p, xs[i], ys[i], scale, b, tid);
        __syncthreads();
        for (int q = tid; q < MLP_PARAMS; q += MLP_BATCH_CTA) gpart[q] = param_grad(b, q, MLP_BATCH_CTA);
        cl.sync();
        pow1 *= b1c;
        pow2 *= b2c;
        // cosine decay from lr0 to lr0 / 10
        const float lr = lr0 * (0.55f + 0.45f * cospif((float)step / (float)(steps > 1 ? steps - 1 : 1)));
        for (int q = q0 + tid; q < q1; q += MLP_BATCH_CTA) {
            float g = 0.f;
            for (int r = 0; r < MLP_CLUSTER; r++) g += cl.map_shared_rank(gpart, r)[q];
            const int k = q - q0;
            am[k] = b1c * am[k] + (1.f - b1c) * g;
            av[k] = b2c * av[k] + (1.f - b2c) * g * g;
            const float mh = am[k] / (1.f - pow1), vh = av[k] / (1.f - pow2);
            const float np = p[q] - lr * mh / (sqrtf(vh) + eps);
            for (int r = 0; r < MLP_CLUSTER; r++) cl.map_shared_rank(p, r)[q] = np;
        }
        cl.sync();
    }
    if (rank == 0)
        for (int q = tid; q < MLP_PARAMS; q += MLP_BATCH_CTA) params[q] = p[q];
}

// Seeded initialisation (uniform Glorot ranges) written to params.
__global__ void k_mlp_init(float *params, uint64_t seed) {
    for (int q = threadIdx.x; q < MLP_PARAMS; q += blockDim.x) {
        const double u = (double)(mix64(seed ^ mix64(0xC0FFEE + q)) >> 11) * (1.0 / 9007199254740992.0);
        float a;
        if (q < MLP_H) a = sqrtf(6.f / (1 + MLP_H)) * 4.f;                     // W1: spread over the key range
        else if (q < 2 * MLP_H) a = 1.f;                                        // b1
        else if (q < 2 * MLP_H + MLP_H * MLP_H) a = sqrtf(6.f / (2 * MLP_H));  // W2
        else if (q < 3 * MLP_H + MLP_H * MLP_H) a = 0.1f;                       // b2
        else if (q < 4 * MLP_H + MLP_H * MLP_H) a = sqrtf(6.f / (MLP_H + 1));  // W3
        else a = 0.f;                                                           // b3
        params[q] = (q == MLP_PARAMS - 1) ? 0.5f : (float)((2.0 * u - 1.0) * a);
    }
}

size_t mlp_train_smem() {
    return (size_t)(2 * MLP_PARAMS_PAD + 2 * MLP_SLICE) * 4 + sizeof(BatchSmem);
}
size_t mlp_grad_smem() { return (size_t)MLP_PARAMS_PAD * 4 + sizeof(BatchSmem); }

cudaError_t launch_mlp_init(float *params, uint64_t seed, cudaStream_t st) {
    k_mlp_init<<<1, 256, 0, st>>>(params, seed);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_mlp_grad(const float *params, const float *xs, const float *ys, uint32_t n, float *grad,
                            float *loss_sum, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(grad, 0, MLP_PARAMS * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(loss_sum, 0, 4, st);
    if (e != cudaSuccess || n == 0) return e;
    const size_t smem = mlp_grad_smem();
    e = smem_limit((const void *)k_mlp_grad, smem);
    if (e != cudaSuccess) return e;
    k_mlp_grad<<<(n + MLP_BATCH_CTA - 1) / MLP_BATCH_CTA, MLP_BATCH_CTA, smem, st>>>(params, xs, ys, n, grad, loss_sum);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_mlp_train(const float *xs, const float *ys, uint32_t n, float *params, int steps, float lr,
                             uint64_t seed, cudaStream_t st) {
    if (n == 0 || steps <= 0) return cudaSuccess;
    const size_t smem = mlp_train_smem();
    cudaError_t e = smem_limit((const void *)k_mlp_train, smem);
    if (e != cudaSuccess) return e;
    k_mlp_train<<<MLP_CLUSTER, MLP_BATCH_CTA, smem, st>>>(xs, ys, n, params, steps, lr, seed);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// sample and training set
// ---------------------------------------------------------------------------
__global__ void k_sample(const Row *__restrict__ in, uint64_t n, Row *__restrict__ out, uint64_t m, uint64_t seed) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = mix64(seed ^ mix64(i + 0x51ED)) % n;
        out[i] = Row{in[j].key, 0u};
    }
}

cudaError_t launch_sample(const Row *in, uint64_t n, Row *out, uint64_t m, uint64_t seed, cudaStream_t st) {
    k_sample<<<(unsigned)umin64((m + 255) / 256, 148 * 8), 256, 0, st>>>(in, n, out, m, seed);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// heavy keys: candidates from the sorted sample, scored by the model
// ---------------------------------------------------------------------------
// Candidates: each distinct key of the sorted sample, with the sample's
// estimate of its S rows (nS * run / m).
// Candidates: the distinct keys of the sorted sample with their sample
// estimate of S rows, written in key order (so the training points, and the
// trained model, do not depend on scheduling).  CTA c owns a contiguous range
// of the sample; k_cand_count counts the run starts in each range, then every
// CTA places its run starts after those of the ranges before it.
constexpr int CAND_THREADS = 256;

__device__ __forceinline__ bool run_start(const Row *sorted, uint64_t i) {
    const uint32_t k = sorted[i].key;
    return k != 0xFFFFFFFFu && (i == 0 || sorted[i - 1].key != k);
}

__global__ void __launch_bounds__(CAND_THREADS) k_cand_count(const Row *__restrict__ sorted, uint64_t m,
                                                            uint64_t chunk, unsigned *cnt) {
    __shared__ uint64_t scratch[CAND_THREADS / 32 + 1];
    const uint64_t lo = (uint64_t)blockIdx.x * chunk, hi = umin64(m, lo + chunk);
    uint64_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += CAND_THREADS) c += run_start(sorted, i);
    uint64_t tot;
    block_excl_scan<CAND_THREADS>(c, &tot, scratch);
    if (threadIdx.x == 0) cnt[blockIdx.x] = (unsigned)tot;
}

__global__ void __launch_bounds__(CAND_THREADS) k_candidates(const Row *__restrict__ sorted, uint64_t m,
                                                            uint64_t chunk, const unsigned *__restrict__ cnt,
                                                            double nS, HeavyCand *cand, unsigned *ncand,
                                                            unsigned cand_cap) {
    __shared__ uint64_t scratch[CAND_THREADS / 32 + 1];
    const uint64_t lo = (uint64_t)blockIdx.x * chunk, hi = umin64(m, lo + chunk);
    uint64_t before = 0;  // run starts in the ranges before this one
    for (unsigned c = threadIdx.x; c < blockIdx.x; c += CAND_THREADS) before += cnt[c];
    uint64_t base;
    block_excl_scan<CAND_THREADS>(before, &base, scratch);
    for (uint64_t t = lo; t < hi; t += CAND_THREADS) {  // block-uniform trip count
        const uint64_t i = t + threadIdx.x;
        const bool start = i < hi && run_start(sorted, i);
        uint64_t tile;
        const uint64_t pos = base + block_excl_scan<CAND_THREADS>(start ? 1 : 0, &tile, scratch);
        if (start) {
            const uint32_t k = sorted[i].key;
            uint64_t a = i + 1, b = m;  // run end: first index with a larger key
            while (a < b) {
                const uint64_t mid = (a + b) >> 1;
                if (sorted[mid].key == k) a = mid + 1;
                else b = mid;
            }
            if (pos < cand_cap) cand[pos] = HeavyCand{k, (float)(nS * (double)(a - i) / (double)m)};
        }
        base += tile;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *ncand = (unsigned)base;
}

cudaError_t launch_candidates(const Row *sorted, uint64_t m, double nS, HeavyCand *cand, unsigned *ncand,
                              unsigned cand_cap, unsigned *scratch_cnt, cudaStream_t st) {
    if (!m) return cudaMemsetAsync(ncand, 0, sizeof(unsigned), st);
    const unsigned g = (unsigned)umin64((m + 4095) / 4096, 148 * 8);
    const uint64_t chunk = (m + g - 1) / g;
    k_cand_count<<<g, CAND_THREADS, 0, st>>>(sorted, m, chunk, scratch_cnt);
    k_candidates<<<g, CAND_THREADS, 0, st>>>(sorted, m, chunk, scratch_cnt, nS, cand, ncand, cand_cap);
    count_launch(2);
    return cudaGetLastError();
}

// Training points of the frequency model: T candidates evenly spread over
// the list; x = key feature, y = log2(sample estimate) / 32.
__global__ void k_freq_points(const HeavyCand *__restrict__ cand, unsigned ncand, float *xs, float *ys, uint32_t T) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const HeavyCand c = cand[(uint64_t)t * ncand / T];
    xs[t] = key_feature((double)c.key);
    ys[t] = log2f(fmaxf(c.count, 1.f)) / 32.f;
}

cudaError_t launch_freq_points(const HeavyCand *cand, unsigned ncand, float *xs, float *ys, uint32_t T,
                               cudaStream_t st) {
    k_freq_points<<<(T + 255) / 256, 256, 0, st>>>(cand, ncand, xs, ys, T);
    count_launch();
    return cudaGetLastError();
}

// Scores every candidate: predicted S rows 2^(32 * M(x)) from the model, or
// the sample estimate (quantile ablation).  Scores at or above tau_min are
// binned by floor(log2(score)): bins[] counts them, mass[] sums the sample's
// estimate of their rows (the model proposes, the sample measures); the score
// replaces cand[].count (0 below tau_min).
__global__ void __launch_bounds__(256) k_heavy_score(HeavyCand *cand, unsigned ncand, const float *__restrict__ params,
                                                     int use_model, double tau_min, double min_sample,
                                                     unsigned *bins, unsigned long long *mass) {
    __shared__ float p[MLP_PARAMS];
    for (int q = threadIdx.x; q < MLP_PARAMS; q += 256) p[q] = params[q];
    __syncthreads();
    for (unsigned i = blockIdx.x * 256 + threadIdx.x; i < ncand; i += gridDim.x * 256) {
        HeavyCand c = cand[i];
        double score = c.count;
        if (c.count < min_sample) score = 0.0;  // seen once in the sample
        else if (use_model) score = exp2(32.0 * (double)mlp_eval(p, key_feature((double)c.key)));
        if (!(score >= tau_min)) score = 0.0;  // also rejects NaN
        score = fmin(score, 4.0e18);
        cand[i].count = (float)score;
        if (score > 0.0) {
            const int bin = min(63, max(0, (int)floor(log2(score))));
            atomicAdd(&bins[bin], 1u);
            atomicAdd(&mass[bin], (unsigned long long)c.count);
        }
    }
}

cudaError_t launch_heavy_score(HeavyCand *cand, unsigned ncand, const float *params, int use_model, double tau_min,
                               double min_sample, unsigned *bins, unsigned long long *mass, cudaStream_t st) {
    if (!ncand) return cudaSuccess;
    k_heavy_score<<<(ncand + 255) / 256, 256, 0, st>>>(cand, ncand, params, use_model, tau_min, min_sample, bins, mass);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// heavy table: open addressing on the key, HEAVY_CAP slots, key EMPTY_KEY
// marks a free slot; val = R rows with the key, start = first of them in the
// heavy R payload list (materialisation).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t heavy_hash(uint32_t k) { return (k * 0x9E3779B1u) >> (32 - HEAVY_LOG2); }
__device__ __forceinline__ uint32_t filter_bit(uint32_t k) { return (k * 0x85EBCA6Bu) >> (32 - FILTER_LOG2); }

__device__ __forceinline__ int heavy_find(const uint32_t *keys, uint32_t k) {
    uint32_t h = heavy_hash(k);
    for (int probe = 0; probe < HEAVY_CAP; probe++) {
        const uint32_t x = keys[h];
        if (x == k) return (int)h;
        if (x == EMPTY_KEY) return -1;
        h = (h + 1) & (HEAVY_CAP - 1);
    }
    return -1;
}

__global__ void k_heavy_build(const HeavyCand *__restrict__ cand, unsigned ncand, float tau, uint32_t *keys,
                              uint32_t *filter, unsigned *inserted) {
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < ncand; i += gridDim.x * blockDim.x) {
        if (!(cand[i].count >= tau)) continue;
        if (atomicAdd(inserted, 1u) >= HEAVY_MAX) continue;
        const uint32_t k = cand[i].key;
        const uint32_t fb = filter_bit(k);
        atomicOr(&filter[fb >> 5], 1u << (fb & 31));
        uint32_t h = heavy_hash(k);
        for (int probe = 0; probe < HEAVY_CAP; probe++) {
            const uint32_t old = atomicCAS(&keys[h], EMPTY_KEY, k);
            if (old == EMPTY_KEY || old == k) break;
            h = (h + 1) & (HEAVY_CAP - 1);
        }
    }
}

cudaError_t launch_heavy_build(const HeavyCand *cand, unsigned ncand, float tau, uint32_t *keys, uint32_t *filter,
                               unsigned *inserted, cudaStream_t st) {
    if (!ncand) return cudaSuccess;
    k_heavy_build<<<(ncand + 255) / 256, 256, 0, st>>>(cand, ncand, tau, keys, filter, inserted);
    count_launch();
    return cudaGetLastError();
}

// R rows of heavy keys: per-slot counts (pass 0) and payload lists (pass 1,
// materialisation only; start[] holds the exclusive prefix of the counts and
// cur[] the fill cursors).
template <int PASS>
__global__ void __launch_bounds__(512) k_heavy_r(const Row *__restrict__ R, uint64_t n, const uint32_t *__restrict__ gkeys,
                                                 const uint32_t *__restrict__ gfilter, unsigned *gcnt,
                                                 const unsigned *__restrict__ start, unsigned *cur, uint32_t *rpay) {
    extern __shared__ __align__(16) unsigned char smem_hr[];
    uint32_t *keys = reinterpret_cast<uint32_t *>(smem_hr);
    unsigned *cnt = keys + HEAVY_CAP;
    uint32_t *filt = cnt + HEAVY_CAP;
    for (int i = threadIdx.x; i < HEAVY_CAP; i += 512) {
        keys[i] = gkeys[i];
        cnt[i] = 0;
    }
    for (int i = threadIdx.x; i < (1 << FILTER_LOG2) / 32; i += 512) filt[i] = gfilter[i];
    __syncthreads();
    // four rows in flight per thread
    const uint64_t stride = (uint64_t)gridDim.x * 512;
    for (uint64_t i0 = (uint64_t)blockIdx.x * 512 + threadIdx.x; i0 < n; i0 += 4 * stride) {
        Row x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t i = i0 + u * stride;
            if (i < n) {
                const uint2 v = ldg_stream(reinterpret_cast<const uint2 *>(R) + i);
                x[u] = Row{v.x, v.y};
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (i0 + u * stride >= n) continue;
            const uint32_t fb = filter_bit(x[u].key);
            if (!(filt[fb >> 5] >> (fb & 31) & 1)) continue;
            const int s = heavy_find(keys, x[u].key);
            if (s < 0) continue;
            if (PASS == 0) atomicAdd(&cnt[s], 1u);
            else rpay[start[s] + atomicAdd(&cur[s], 1u)] = x[u].payload;
        }
    }
    if (PASS == 0) {
        __syncthreads();
        for (int i = threadIdx.x; i < HEAVY_CAP; i += 512)
            if (cnt[i]) atomicAdd(&gcnt[i], cnt[i]);
    }
}

// exclusive prefix of the per-slot R counts (one CTA)
__global__ void k_heavy_prefix(const unsigned *cnt, unsigned *start, unsigned *cur) {
    __shared__ uint64_t scratch[1024 / 32 + 1];
    constexpr int PER = HEAVY_CAP / 1024;
    unsigned local = 0;
    for (int j = 0; j < PER; j++) local += cnt[threadIdx.x * PER + j];
    uint64_t tot;
    unsigned run = (unsigned)block_excl_scan<1024>(local, &tot, scratch);
    for (int j = 0; j < PER; j++) {
        const int s = threadIdx.x * PER + j;
        start[s] = run;
        cur[s] = 0;
        run += cnt[s];
    }
}

// stage 0: per-slot counts of R's heavy rows; stage 1 (materialisation):
// prefix of the counts, then every heavy row's payload into rpay.
cudaError_t launch_heavy_r(const Row *R, uint64_t n, const uint32_t *keys, const uint32_t *filter, unsigned *cnt,
                           unsigned *start, unsigned *cur, uint32_t *rpay, int stage, int nsm, cudaStream_t st) {
    if (!n) return cudaSuccess;
    const unsigned g = (unsigned)umin64((n + 511) / 512, (uint64_t)nsm * 4);
    const size_t smem = (size_t)HEAVY_CAP * 8 + (1 << FILTER_LOG2) / 8;
    cudaError_t e = smem_limit((const void *)k_heavy_r<0>, smem);
    if (e == cudaSuccess) e = smem_limit((const void *)k_heavy_r<1>, smem);
    if (e != cudaSuccess) return e;
    if (stage == 0) {
        k_heavy_r<0><<<g, 512, smem, st>>>(R, n, keys, filter, cnt, nullptr, nullptr, nullptr);
        count_launch();
    } else {
        k_heavy_prefix<<<1, 1024, 0, st>>>(cnt, start, cur);
        k_heavy_r<1><<<g, 512, smem, st>>>(R, n, keys, filter, cnt, start, cur, rpay);
        count_launch(2);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// S histogram with the heavy bypass: per chunk (as k_hist_chunks), rows whose
// key is heavy are joined on the spot against the heavy table (count, or
// rows out), every other row is counted in its radix bin and appended to
// the chunk's region of the compacted S (warp-aggregated, coalesced).
// ---------------------------------------------------------------------------
template <bool MAT>
__global__ void __launch_bounds__(1024) k_hist_bypass(BypassArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *hist = reinterpret_cast<uint32_t *>(smem);
    uint32_t *filt = hist + a.nbins;              // 2^FILTER_LOG2 bits
    uint32_t *hkeys = filt + (1 << FILTER_LOG2) / 32;
    unsigned *hcnt = hkeys + HEAVY_CAP;
    __shared__ unsigned s_keep;
    __shared__ uint64_t scan_scratch[1024 / 32 + 1];
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < a.nbins; i += 1024) hist[i] = 0;
    for (int i = tid; i < (1 << FILTER_LOG2) / 32; i += 1024) filt[i] = a.filter[i];
    for (int i = tid; i < HEAVY_CAP; i += 1024) {
        hkeys[i] = a.hkeys[i];
        hcnt[i] = a.hcnt[i];
    }
    if (tid == 0) s_keep = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * a.chunk;
    const uint64_t hi = umin64(a.n, lo + a.chunk);
    const uint64_t len = hi > lo ? hi - lo : 0;
    const Row *src = a.in + lo;
    uint2 *dst = reinterpret_cast<uint2 *>(a.out + lo);
    const bool vec = (reinterpret_cast<uintptr_t>(src) & 15) == 0;
    unsigned long long matches = 0, heavy_rows = 0;
    // rounds of 8 rows per thread: row pairs p = base/2 + u * 1024 + tid
    for (uint64_t base = 0; base < len; base += 8 * 1024) {
        uint32_t k[8], v[8];
        int slot[8];
        unsigned keep = 0, emit = 0, nheavy = 0;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t r = base + 2 * ((uint64_t)u * 1024 + tid);
            if (vec && r + 1 < len) {
                const uint4 x = ldg_stream(reinterpret_cast<const uint4 *>(src + r));
                k[2 * u] = x.x; v[2 * u] = x.y; k[2 * u + 1] = x.z; v[2 * u + 1] = x.w;
            } else {
                k[2 * u] = k[2 * u + 1] = 0; v[2 * u] = v[2 * u + 1] = 0;
                if (r < len) { const uint2 x = ldg_stream(reinterpret_cast<const uint2 *>(src + r)); k[2 * u] = x.x; v[2 * u] = x.y; }
                if (r + 1 < len) { const uint2 x = ldg_stream(reinterpret_cast<const uint2 *>(src + r + 1)); k[2 * u + 1] = x.x; v[2 * u + 1] = x.y; }
            }
            const uint32_t valid = (r < len ? 1u : 0u) | (r + 1 < len ? 2u : 0u);
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int j = 2 * u + h;
                slot[j] = -1;
                const uint32_t fb = filter_bit(k[j]);
                if ((valid >> h & 1) && (filt[fb >> 5] >> (fb & 31) & 1)) slot[j] = heavy_find(hkeys, k[j]);
                if (slot[j] >= 0) {
                    emit += hcnt[slot[j]];
                    nheavy++;
                } else if (valid >> h & 1) {
                    keep |= 1u << j;
                }
            }
        }
        matches += emit;
        heavy_rows += nheavy;
        // coalesced compaction: one ballot per row slot, one shared atomic per warp
        unsigned m[8], wtot = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            m[j] = __ballot_sync(0xffffffffu, keep >> j & 1);
            wtot += __popc(m[j]);
        }
        unsigned wb = 0;
        if (lane == 0 && wtot) wb = atomicAdd(&s_keep, wtot);
        wb = __shfl_sync(0xffffffffu, wb, 0);
        const unsigned lt = lanemask_lt();
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (keep >> j & 1) {
                atomicAdd(&hist[radix_f(a.rf, k[j])], 1u);
                dst[wb + __popc(m[j] & lt)] = make_uint2(k[j], v[j]);
            }
            wb += __popc(m[j]);
        }
        if (MAT) {
            // heavy rows' output in (row slot, lane) order: coalesced stores
            uint32_t c[8];
#pragma unroll
            for (int j = 0; j < 8; j++) c[j] = slot[j] >= 0 ? hcnt[slot[j]] : 0;
            uint64_t pos[8];
            block_emit_positions<1024, 8>(c, pos, a.rows_ctr, scan_scratch);
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (c[j]) {
                    // R-row starts stay in global memory: only heavy rows read them
                    const unsigned st0 = a.hstart[slot[j]];
                    uint64_t op = pos[j];
                    for (unsigned q = 0; q < c[j]; q++, op++)
                        if (op < a.cap) a.rows[op] = tbg_row_out{k[j], a.rpay[st0 + q], v[j]};
                }
            }
        }
    }
    __syncthreads();
    uint32_t *hdst = a.hist + (uint64_t)blockIdx.x * a.nbins;
    for (int i = tid; i < a.nbins; i += 1024) hdst[i] = hist[i];
    if (tid == 0) a.kept[blockIdx.x] = s_keep;
    const unsigned long long wm = warp_sum_u64(matches), wh = warp_sum_u64(heavy_rows);
    if (lane == 0) {
        if (wm) atomicAdd(a.matches, wm);
        if (wh) atomicAdd(a.heavy_rows, wh);
    }
}

size_t bypass_smem(int nbins, bool mat) {
    (void)mat;  // 2^15 bins + filter + keys + counts: 204,800 B at most
    return (size_t)nbins * 4 + (1 << FILTER_LOG2) / 8 + (size_t)HEAVY_CAP * 4 * 2;
}

cudaError_t launch_hist_bypass(const BypassArgs &a, bool mat, cudaStream_t st) {
    const size_t smem = bypass_smem(a.nbins, mat);
    auto kern = mat ? k_hist_bypass<true> : k_hist_bypass<false>;
    cudaError_t e = smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<a.G, 1024, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
