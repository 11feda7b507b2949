// LRN: learned skew-aware partitioning for sm_100a.
//
// A small FP32 MLP (1 -> 32 -> 32 -> 1, tanh) models the frequency curve of
// S's keys: log2(sample count) of the key of sample rank r (normalised over
// the training points) as a function of log2(r + 1) / 16 - 1 (rank 1 = the
// most frequent key of a seeded 1%
// sample of S).  It is trained per join on that sample's curve by the
// kernels in this file (forward, backward, Adam; the trainer is one 8-CTA
// thread-block cluster that all-reduces gradients through distributed shared
// memory).  The input is a rank the sample measures, never the key's value,
// so the curve is the same whether hot keys are small integers or scattered
// over the key range.  From the trained curve the decision kernel predicts
// the S rows of ranks 1 .. HEAVY_MAX: the ranks predicted above a threshold
// are the heavy keys (taken by sample count), and LRN bypasses only when the
// model predicts they hold enough of S.  Heavy keys never enter the radix
// partitions: their (R, S) pairs are joined in the histogram read itself,
// split across every CTA that streams S, against a shared-memory table of
// their R rows.  The remaining rows are radix partitioned and joined as in
// RHO.  The model only chooses which keys take the heavy path; every row's
// destination is decided by an exact key comparison, so results are exact
// whatever the model predicts.
#include <cooperative_groups.h>

#include "part_dev.cuh"
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
// step every CTA draws MLP_BATCH_CTA seeded random training points (uniformly,
// or in proportion to their weights), computes their forward/backward on its
// first MLP_BATCH_CTA threads and its partial parameter gradient on all
// MLP_TRAIN_THREADS; after a cluster
// barrier CTA r sums the partials of its parameter slice from every CTA's
// shared memory, applies Adam, and writes the new values into every CTA's
// parameter copy; a second barrier ends the step.
__global__ void __cluster_dims__(MLP_CLUSTER, 1, 1) __launch_bounds__(MLP_TRAIN_THREADS)
    k_mlp_train(const float *__restrict__ xs, const float *__restrict__ ys, const float *__restrict__ cw,
                const unsigned *n_dev, uint32_t n_host, float *params, int steps, float lr0, uint64_t seed) {
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    // the point count: from device memory when the caller's kernels made the
    // points (the same value for every CTA), else the host's
    const uint32_t n = n_dev ? *n_dev : n_host;
    if (n == 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    float *p = reinterpret_cast<float *>(smem);
    float *gpart = p + MLP_PARAMS_PAD;
    float *am = gpart + MLP_PARAMS_PAD;  // Adam moments of this CTA's slice
    float *av = am + MLP_SLICE;
    BatchSmem &b = *reinterpret_cast<BatchSmem *>(av + MLP_SLICE);
    const int tid = threadIdx.x;
    for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) p[q] = params[q];
    for (int q = tid; q < MLP_SLICE; q += MLP_TRAIN_THREADS) am[q] = av[q] = 0.f;
    cl.sync();
    const float b1c = 0.9f, b2c = 0.999f, eps = 1e-8f;
    const float scale = 1.f / (float)(MLP_BATCH_CTA * MLP_CLUSTER);
    const int q0 = rank * MLP_SLICE, q1 = min(MLP_PARAMS, q0 + MLP_SLICE);
    const float wtot = cw ? cw[n - 1] : 0.f;
    float pow1 = 1.f, pow2 = 1.f;
    for (int step = 0; step < steps; step++) {
        if (tid < MLP_BATCH_CTA) {  // one sample per thread of the first warps
            const uint64_t h = mix64(seed ^ mix64(((uint64_t)step << 20) | (uint64_t)(rank * MLP_BATCH_CTA + tid)));
            uint32_t i;
            if (cw) {  // the first point whose cumulative weight exceeds u * total
                const float u = (float)((h >> 40) * (1.0 / 16777216.0)) * wtot;
                uint32_t lo = 0, hi = n - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (cw[mid] > u) hi = mid;
                    else lo = mid + 1;
                }
                i = lo;
            } else {
                i = (uint32_t)(h % n);
            }
            sample_fwd_bwd(p, xs[i], ys[i], scale, b, tid);
        }
        __syncthreads();
        for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) gpart[q] = param_grad(b, q, MLP_BATCH_CTA);
        cl.sync();
        pow1 *= b1c;
        pow2 *= b2c;
        // cosine decay from lr0 to lr0 / 10
        const float lr = lr0 * (0.55f + 0.45f * cospif((float)step / (float)(steps > 1 ? steps - 1 : 1)));
        for (int q = q0 + tid; q < q1; q += MLP_TRAIN_THREADS) {
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
        for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) params[q] = p[q];
}

// Seeded initialisation (uniform Glorot ranges) written to params.
__global__ void k_mlp_init(float *params, uint64_t seed) {
    for (int q = threadIdx.x; q < MLP_PARAMS; q += blockDim.x) {
        const double u = (double)(mix64(seed ^ mix64(0xC0FFEE + q)) >> 11) * (1.0 / 9007199254740992.0);
        float a;
        if (q < MLP_H) a = sqrtf(6.f / (1 + MLP_H)) * 4.f;                     // W1: spread over the rank range
        else if (q < 2 * MLP_H) a = 1.f;                                        // b1
        else if (q < 2 * MLP_H + MLP_H * MLP_H) a = sqrtf(6.f / (2 * MLP_H));  // W2
        else if (q < 3 * MLP_H + MLP_H * MLP_H) a = 0.1f;                       // b2
        else if (q < 4 * MLP_H + MLP_H * MLP_H) a = sqrtf(6.f / (MLP_H + 1));  // W3
        else a = 0.f;                                                           // b3
        params[q] = (float)((2.0 * u - 1.0) * a);
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

cudaError_t launch_mlp_train(const float *xs, const float *ys, const float *cw, const unsigned *n_dev, uint32_t n,
                             float *params, int steps, float lr, uint64_t seed, cudaStream_t st) {
    if ((!n_dev && n == 0) || steps <= 0) return cudaSuccess;
    const size_t smem = mlp_train_smem();
    cudaError_t e = smem_limit((const void *)k_mlp_train, smem);
    if (e != cudaSuccess) return e;
    k_mlp_train<<<MLP_CLUSTER, MLP_TRAIN_THREADS, smem, st>>>(xs, ys, cw, n_dev, n, params, steps, lr, seed);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// learning stage: sample, key counts, rank curve, decision
// ---------------------------------------------------------------------------
// The sample: nblocks blocks of SAMPLE_BLOCK consecutive S rows, block j taken
// from the stride-sized stretch j of S at a seeded offset (a stratified 1%
// sample read with coalesced loads).  One warp per block; every block lies
// inside S (stride * nblocks <= nS / SAMPLE_BLOCK).
__global__ void k_sample_blocks(const Row *__restrict__ S, uint32_t *__restrict__ keys, uint64_t nblocks,
                                uint64_t stride, uint64_t seed) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t j = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; j < nblocks; j += nw) {
        const uint64_t sb = j * stride + (stride > 1 ? mix64(seed ^ mix64(j + 0x51ED)) % stride : 0);
        const Row *src = S + sb * SAMPLE_BLOCK;
        const uint2 a = ldg_stream(reinterpret_cast<const uint2 *>(src) + lane);
        const uint2 b = ldg_stream(reinterpret_cast<const uint2 *>(src) + lane + 32);
        keys[j * SAMPLE_BLOCK + lane] = a.x;
        keys[j * SAMPLE_BLOCK + lane + 32] = b.x;
    }
}

cudaError_t launch_sample_blocks(const Row *S, uint64_t nS, uint32_t *keys, uint64_t nblocks, uint64_t stride,
                                 uint64_t seed, cudaStream_t st) {
    (void)nS;
    if (!nblocks) return cudaSuccess;
    const unsigned g = (unsigned)umin64((nblocks * 32 + 255) / 256, 148 * 16);
    k_sample_blocks<<<g, 256, 0, st>>>(S, keys, nblocks, stride, seed);
    count_launch();
    return cudaGetLastError();
}

__device__ __forceinline__ uint32_t count_hash(uint32_t k) { return (k * 0x9E3779B1u) ^ (k >> 15); }

// Adds c to key k's count in the global open-addressing table (tmask + 1
// slots).  A full table drops the key: a key that is not counted is never
// heavy, which only costs speed.
__device__ __forceinline__ void table_add(uint32_t *tk, uint32_t *tc, uint32_t tmask, uint32_t k, uint32_t c) {
    uint32_t h = count_hash(k) & tmask;
    for (uint32_t probe = 0; probe <= tmask && probe < 4096; probe++) {
        const uint32_t old = atomicCAS(&tk[h], EMPTY_KEY, k);
        if (old == EMPTY_KEY || old == k) {
            atomicAdd(&tc[h], c);
            return;
        }
        h = (h + 1) & tmask;
    }
}

// Counts the sample's keys: CTA c aggregates keys [c * CNT_CHUNK, ...) in a
// shared table (equal keys of a warp first combined with __match_any_sync,
// so a hot key costs one shared atomic per warp), then adds each distinct
// key once to the global table.  Key EMPTY_KEY is never counted.
__global__ void __launch_bounds__(CNT_THREADS) k_count_keys(const uint32_t *__restrict__ keys, uint64_t m,
                                                           uint32_t *tk, uint32_t *tc, uint32_t tmask) {
    constexpr int SLOTS = 2 * CNT_CHUNK;
    __shared__ uint32_t lk[SLOTS];
    __shared__ uint32_t lc[SLOTS];
    for (int i = threadIdx.x; i < SLOTS; i += CNT_THREADS) {
        lk[i] = EMPTY_KEY;
        lc[i] = 0;
    }
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * CNT_CHUNK;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int u = 0; u < CNT_CHUNK / CNT_THREADS; u++) {
        const uint64_t i = lo + (uint64_t)u * CNT_THREADS + threadIdx.x;
        const uint32_t k = i < m ? keys[i] : EMPTY_KEY;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        if (k != EMPTY_KEY && lane == __ffs(peers) - 1) {
            uint32_t h = count_hash(k) & (SLOTS - 1);
            for (int probe = 0; probe < SLOTS; probe++) {  // at most CNT_CHUNK keys in 2x the slots
                const uint32_t old = atomicCAS(&lk[h], EMPTY_KEY, k);
                if (old == EMPTY_KEY || old == k) {
                    atomicAdd(&lc[h], (uint32_t)__popc(peers));
                    break;
                }
                h = (h + 1) & (SLOTS - 1);
            }
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < SLOTS; i += CNT_THREADS)
        if (lk[i] != EMPTY_KEY) table_add(tk, tc, tmask, lk[i], lc[i]);
}

cudaError_t launch_count_keys(const LearnBufs &b, uint64_t m, cudaStream_t st) {
    if (!m) return cudaSuccess;
    k_count_keys<<<(unsigned)((m + CNT_CHUNK - 1) / CNT_CHUNK), CNT_THREADS, 0, st>>>(b.keys, m, b.tkeys, b.tcnt,
                                                                                      b.tmask);
    count_launch();
    return cudaGetLastError();
}

// Bin of a sample count: exact below CC_EXACT, then CC_OCT bins per octave.
__host__ __device__ __forceinline__ int cc_bin(uint32_t c) {
    if (c < (uint32_t)CC_EXACT) return (int)c;
#ifdef __CUDA_ARCH__
    const int e = 31 - __clz(c);
#else
    const int e = 31 - __builtin_clz(c);
#endif
    return CC_EXACT + (e - 11) * CC_OCT + (int)((c >> (e - 4)) & (CC_OCT - 1));
}
// Smallest count in bin b.
__host__ __device__ __forceinline__ uint32_t cc_bin_min(int b) {
    if (b < CC_EXACT) return (uint32_t)b;
    const int e = 11 + (b - CC_EXACT) / CC_OCT, f = (b - CC_EXACT) % CC_OCT;
    return (1u << e) | ((uint32_t)f << (e - 4));
}

// Count-of-counts over the table (keys per bin, sample rows per bin) and the
// candidate list: the keys the sample saw at least CAND_MIN_COUNT times.
constexpr int STATS_THREADS = 1024;

__global__ void __launch_bounds__(STATS_THREADS) k_count_stats(const uint32_t *__restrict__ tk, const uint32_t *__restrict__ tc,
                                                    uint32_t tmask, unsigned *bin_keys,
                                                    unsigned long long *bin_rows, HeavyCand *cand,
                                                    unsigned cand_cap, LrnDecision *dec) {
    __shared__ unsigned sk[CC_BINS];
    __shared__ unsigned long long sr[CC_BINS];
    for (int i = threadIdx.x; i < CC_BINS; i += STATS_THREADS) {
        sk[i] = 0;
        sr[i] = 0;
    }
    __syncthreads();
    const uint64_t slots = (uint64_t)tmask + 1;
    const int lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * STATS_THREADS; base < slots; base += (uint64_t)gridDim.x * STATS_THREADS) {
        const uint64_t i = base + threadIdx.x;  // warp-uniform trip count (slots is a multiple of STATS_THREADS)
        const uint32_t k = tk[i], c = tc[i];
        const bool used = k != EMPTY_KEY && c > 0;
        if (used) {
            const int b = cc_bin(c);
            atomicAdd(&sk[b], 1u);
            atomicAdd(&sr[b], (unsigned long long)c);
        }
        const bool is_cand = used && c >= (uint32_t)CAND_MIN_COUNT;
        const unsigned bal = __ballot_sync(0xffffffffu, is_cand);
        unsigned wb = 0;
        if (lane == 0 && bal) wb = atomicAdd(&dec->ncand, (unsigned)__popc(bal));
        wb = __shfl_sync(0xffffffffu, wb, 0);
        const unsigned pos = wb + __popc(bal & lanemask_lt());
        if (is_cand && pos < cand_cap) cand[pos] = HeavyCand{k, c};
    }
    __syncthreads();
    for (int i = threadIdx.x; i < CC_BINS; i += STATS_THREADS) {
        if (sk[i]) {
            atomicAdd(&bin_keys[i], sk[i]);
            atomicAdd(&bin_rows[i], sr[i]);
        }
    }
}

cudaError_t launch_count_stats(const LearnBufs &b, cudaStream_t st) {
    const uint64_t slots = (uint64_t)b.tmask + 1;
    const unsigned g = (unsigned)umin64(slots / STATS_THREADS, 148);
    k_count_stats<<<g, STATS_THREADS, 0, st>>>(b.tkeys, b.tcnt, b.tmask, b.bin_keys, b.bin_rows, b.cand, b.cand_cap, b.dec);
    count_launch();
    return cudaGetLastError();
}

// Training points of the frequency model, one per non-empty count bin in
// decreasing count order: x = rank_feature(mid rank of the bin's keys),
// y = log2(mean sample count of the bin), normalised to zero mean and unit
// spread over the points (so the network starts at the curve's mean and
// learns its shape).  One block; writes the point count and the
// normalisation to dec.
__global__ void __launch_bounds__(1024) k_rank_points(const unsigned *__restrict__ bin_keys,
                                                     const unsigned long long *__restrict__ bin_rows, float *xs,
                                                     float *ys, float *cw, LrnDecision *dec) {
    constexpr int PER = (CC_BINS + 1023) / 1024;
    __shared__ uint64_t scratch[1024 / 32 + 1];
    __shared__ double red[2][32];
    // thread t owns reversed bins [t * PER, t * PER + PER): descending counts
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint64_t keys_here = 0, pts_here = 0;
    for (int j = 0; j < PER; j++) {
        const int r = t * PER + j;
        if (r < CC_BINS) {
            const unsigned nk = bin_keys[CC_BINS - 1 - r];
            keys_here += nk;
            pts_here += nk ? 1 : 0;
        }
    }
    uint64_t tot_keys, tot_pts;
    uint64_t above = block_excl_scan<1024>(keys_here, &tot_keys, scratch);
    uint64_t pt = block_excl_scan<1024>(pts_here, &tot_pts, scratch);
    const uint64_t pt0 = pt;
    double s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < PER; j++) {
        const int r = t * PER + j;
        if (r >= CC_BINS) break;
        const int b = CC_BINS - 1 - r;
        const unsigned nk = bin_keys[b];
        if (!nk) continue;
        const double mid = (double)above + 0.5 * (double)(nk + 1);
        const double y = log2((double)bin_rows[b] / (double)nk);
        xs[pt] = rank_feature(mid);
        ys[pt] = (float)y;
        s1 += y;
        s2 += y * y;
        pt++;
        above += nk;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        red[0][w] = s1;
        red[1][w] = s2;
    }
    __syncthreads();
    double a = 0.0, q = 0.0;
    for (int i = 0; i < 32; i++) {
        a += red[0][i];
        q += red[1][i];
    }
    const double n = tot_pts ? (double)tot_pts : 1.0;
    const double mu = a / n;
    const double sigma = fmax(sqrt(fmax(q / n - mu * mu, 0.0)), 0.25);  // flat curves keep a scale
    for (uint64_t i = pt0; i < pt; i++) ys[i] = (float)(((double)ys[i] - mu) / sigma);
    // sampling weights: half uniform over the points, half in proportion to
    // the sample rows their bin holds (the top ranks, which carry the heavy
    // mass the decision predicts, are fitted more closely); cumulative in
    // point order.  The sample's rows total m (tot_rows below).
    __syncthreads();  // red is reused
    double rows_here = 0.0;
    for (int j = 0; j < PER; j++) {
        const int r = t * PER + j;
        if (r < CC_BINS) rows_here += (double)bin_rows[CC_BINS - 1 - r];
    }
    double rs = rows_here;
    for (int o = 16; o > 0; o >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, o);
    if (lane == 0) red[0][w] = rs;
    __syncthreads();
    double tot_rows = 0.0;
    for (int i = 0; i < 32; i++) tot_rows += red[0][i];
    tot_rows = fmax(tot_rows, 1.0);
    const double wmy = 0.5 * (double)(pt - pt0) / n + 0.5 * rows_here / tot_rows;
    uint64_t dummy;
    // fixed point (2^-40) keeps the block scan in integers
    double run = (double)block_excl_scan<1024>((uint64_t)(wmy * 1099511627776.0), &dummy, scratch) /
                 1099511627776.0;
    uint64_t i = pt0;
    for (int j = 0; j < PER; j++) {
        const int r = t * PER + j;
        if (r >= CC_BINS) break;
        const unsigned nk = bin_keys[CC_BINS - 1 - r];
        if (!nk) continue;
        run += 0.5 / n + 0.5 * (double)bin_rows[CC_BINS - 1 - r] / tot_rows;
        cw[i++] = (float)run;
    }
    if (t == 0) {
        dec->npoints = (unsigned)tot_pts;
        dec->y_mu = (float)mu;
        dec->y_sigma = (float)sigma;
    }
}

cudaError_t launch_rank_points(const LearnBufs &b, cudaStream_t st) {
    k_rank_points<<<1, 1024, 0, st>>>(b.bin_keys, b.bin_rows, b.xs, b.ys, b.cw, b.dec);
    count_launch();
    return cudaGetLastError();
}

// The decision (one block).  pred(r), the predicted S rows of the key of
// sample rank r, comes from the model (2^(mu + sigma M(rank_feature(r))) nS / m,
// mu and sigma the points' normalisation) or,
// for the ablation, from the sample's own count at rank r.  k* = the ranks
// 1 .. HEAVY_MAX whose predicted rows reach tau_min; the heavy keys are the
// sampled keys whose count is at least that of rank k* (the lowest count bin
// that keeps their number <= k*).  Bypass when the model predicts those keys
// to hold at least min_frac of S.  Also the model's loss on the points.
constexpr int DECIDE_THREADS = 512;

__global__ void __launch_bounds__(DECIDE_THREADS) k_decide(const float *__restrict__ params, int use_model,
                                                          const unsigned *__restrict__ bin_keys,
                                                          const unsigned long long *__restrict__ bin_rows,
                                                          const float *__restrict__ xs, const float *__restrict__ ys,
                                                          double nS, double m, double tau_min, double min_frac,
                                                          LrnDecision *dec) {
    __shared__ float p[MLP_PARAMS];
    __shared__ uint32_t cnt_at[HEAVY_MAX + 2];  // sample count of rank r (r = 1 .. HEAVY_MAX + 1)
    __shared__ float lpred[HEAVY_MAX + 2];      // log2 of the predicted S rows of rank r
    // the bins, staged (dynamic shared memory) for the single-thread walks below
    extern __shared__ __align__(16) unsigned char dsm[];
    unsigned long long *sr = reinterpret_cast<unsigned long long *>(dsm);
    unsigned *sk = reinterpret_cast<unsigned *>(sr + CC_BINS);
    __shared__ double red[DECIDE_THREADS / 32];
    __shared__ unsigned s_kstar;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    for (int q = t; q < MLP_PARAMS; q += DECIDE_THREADS) p[q] = params[q];
    for (int r = t; r <= HEAVY_MAX + 1; r += DECIDE_THREADS) cnt_at[r] = 0;
    for (int b = t; b < CC_BINS; b += DECIDE_THREADS) {
        sk[b] = bin_keys[b];
        sr[b] = bin_rows[b];
    }
    if (t == 0) s_kstar = 0;
    __syncthreads();
    // ranks 1 .. HEAVY_MAX + 1 sit in the highest bins: thread 0 walks them
    if (t == 0) {
        unsigned r = 1;
        for (int b = CC_BINS - 1; b >= 1 && r <= (unsigned)HEAVY_MAX + 1; b--) {
            const unsigned nk = sk[b];
            if (!nk) continue;
            const uint32_t c = (uint32_t)(sr[b] / nk);
            for (unsigned j = 0; j < nk && r <= (unsigned)HEAVY_MAX + 1; j++) cnt_at[r++] = c;
        }
    }
    __syncthreads();
    const double lscale = log2(nS / m);
    const double mu = dec->y_mu, sigma = dec->y_sigma;
    for (int r = 1 + t; r <= HEAVY_MAX + 1; r += DECIDE_THREADS)
        lpred[r] = use_model ? (float)(mu + sigma * (double)mlp_eval(p, rank_feature((double)r)) + lscale)
                             : (cnt_at[r] ? (float)(log2((double)cnt_at[r]) + lscale) : -INFINITY);
    __syncthreads();
    // k*: the largest rank <= HEAVY_MAX predicted at or above tau_min among the
    // ranks the sample saw at least CAND_MIN_COUNT times
    const float ltau = (float)log2(tau_min);
    unsigned last_ok = 0;
    for (int r = 1 + t; r <= HEAVY_MAX; r += DECIDE_THREADS)
        if (lpred[r] >= ltau && cnt_at[r] >= (uint32_t)CAND_MIN_COUNT) last_ok = max(last_ok, (unsigned)r);
    for (int o = 16; o > 0; o >>= 1) last_ok = max(last_ok, __shfl_xor_sync(0xffffffffu, last_ok, o));
    if (lane == 0 && last_ok) atomicMax(&s_kstar, last_ok);
    __syncthreads();
    const unsigned kstar = s_kstar;
    double mass = 0.0;
    for (int r = 1 + t; r <= (int)kstar; r += DECIDE_THREADS) mass += exp2((double)lpred[r]);
    // the model's mean squared error on the training points
    const unsigned np = dec->npoints;
    double loss = 0.0;
    for (unsigned i = t; i < np; i += DECIDE_THREADS) {
        const double d = (double)mlp_eval(p, xs[i]) - (double)ys[i];
        loss += d * d;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mass += __shfl_xor_sync(0xffffffffu, mass, o);
        loss += __shfl_xor_sync(0xffffffffu, loss, o);
    }
    if (lane == 0) red[w] = mass;
    __syncthreads();
    double pred_mass = 0.0;
    for (int i = 0; i < DECIDE_THREADS / 32; i++) pred_mass += red[i];
    __syncthreads();
    if (lane == 0) red[w] = loss;
    __syncthreads();
    if (t == 0) {
        double lsum = 0;
        for (int i = 0; i < DECIDE_THREADS / 32; i++) lsum += red[i];
        // count threshold: the lowest bin whose keys, with all above it, number <= k*
        unsigned above = 0, count_min = 0xFFFFFFFFu, heavy = 0;
        unsigned long long rows = 0;
        for (int b = CC_BINS - 1; b >= CAND_MIN_COUNT && kstar; b--) {
            const unsigned nk = sk[b];
            if (!nk) continue;
            if (above + nk > kstar) break;
            above += nk;
            rows += sr[b];
            count_min = cc_bin_min(b);
            heavy = above;
        }
        LrnDecision d = *dec;
        d.k_star = kstar;
        d.count_min = count_min;
        d.heavy_sample = heavy;
        d.pred_mass = pred_mass;
        d.sample_mass = (double)rows * (nS / m);
        d.next_rows = kstar < (unsigned)HEAVY_MAX ? exp2((double)lpred[kstar + 1]) : 0.0;
        d.loss = np ? (float)(lsum / np) : 0.f;
        d.bypass = heavy > 0 && pred_mass >= min_frac * nS ? 1u : 0u;
        *dec = d;
    }
}

cudaError_t launch_decide(const LearnBufs &b, int use_model, double nS, double m, double tau_min, double min_frac,
                          cudaStream_t st) {
    const size_t smem = (size_t)CC_BINS * 12;
    cudaError_t e = smem_limit((const void *)k_decide, smem);
    if (e != cudaSuccess) return e;
    k_decide<<<1, DECIDE_THREADS, smem, st>>>(b.params, use_model, b.bin_keys, b.bin_rows, b.xs, b.ys, nS, m, tau_min, min_frac,
                                 b.dec);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// heavy table: HEAVY_BUCKETS buckets of 4 key slots; key EMPTY_KEY marks a
// free slot (so EMPTY_KEY itself is never heavy).  A key goes to the first
// free slot of its bucket, or of the next buckets when that one is full;
// slots fill in order and are never freed, so a lookup stops at the first
// bucket with a free slot (at <= 50% load almost always the first).  Slot s
// = 4 * bucket + i indexes cnt (R rows with the key) and start (first of them
// in the heavy R payload list, materialisation).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t heavy_bucket(uint32_t k) { return (k * 0x9E3779B1u) >> (32 - HEAVY_LOG2 + 2); }
__device__ __forceinline__ uint32_t filter_bit(uint32_t k) { return (k * 0x85EBCA6Bu) >> (32 - FILTER_LOG2); }

__device__ __forceinline__ int heavy_find(const uint32_t *keys, uint32_t k) {
    if (k == EMPTY_KEY) return -1;
    uint32_t b = heavy_bucket(k);
    for (int probe = 0; probe < HEAVY_BUCKETS; probe++) {
        const uint4 q = reinterpret_cast<const uint4 *>(keys)[b];
        const int i = q.x == k ? 0 : q.y == k ? 1 : q.z == k ? 2 : q.w == k ? 3 : -1;
        if (i >= 0) return (int)(4 * b) + i;
        if (q.w == EMPTY_KEY) return -1;  // slots fill in order: a free last slot ends the search
        b = (b + 1) & (HEAVY_BUCKETS - 1);
    }
    return -1;
}

__device__ __forceinline__ void heavy_insert(uint32_t *keys, uint32_t k) {
    uint32_t b = heavy_bucket(k);
    for (int probe = 0; probe < HEAVY_BUCKETS; probe++) {
        for (int i = 0; i < 4; i++) {
            const uint32_t old = atomicCAS(&keys[4 * b + i], EMPTY_KEY, k);
            if (old == EMPTY_KEY || old == k) return;
        }
        b = (b + 1) & (HEAVY_BUCKETS - 1);
    }
}

// Inserts the candidates whose sample count reaches the decision's
// count_min (at most HEAVY_MAX of them; the decision keeps their number at
// or below k* <= HEAVY_MAX) and sets their filter bits.
__global__ void k_heavy_build(const HeavyCand *__restrict__ cand, unsigned cand_cap, const LrnDecision *dec,
                              uint32_t *keys, uint32_t *filter, unsigned *inserted) {
    const unsigned n = min(dec->ncand, cand_cap);
    const unsigned cmin = dec->count_min;
    if (!dec->bypass) return;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const HeavyCand c = cand[i];
        if (c.count < cmin || c.key == EMPTY_KEY) continue;
        if (atomicAdd(inserted, 1u) >= (unsigned)HEAVY_MAX) continue;
        const uint32_t fb = filter_bit(c.key);
        atomicOr(&filter[fb >> 5], 1u << (fb & 31));
        heavy_insert(keys, c.key);
    }
}

cudaError_t launch_heavy_build(const LearnBufs &b, uint32_t *keys, uint32_t *filter, unsigned *inserted,
                               cudaStream_t st) {
    k_heavy_build<<<148 * 2, 256, 0, st>>>(b.cand, b.cand_cap, b.dec, keys, filter, inserted);
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
// Heavy check of one row against the filter and the table in shared memory:
// the row's slot, or -1.
__device__ __forceinline__ int heavy_slot(const uint32_t *filt, const uint32_t *hkeys, uint32_t k) {
    const uint32_t fb = filter_bit(k);
    if (!((filt[fb >> 5] >> (fb & 31)) & 1u)) return -1;
    return heavy_find(hkeys, k);
}

// One row outside the vector body (the chunk's first row when it starts 8
// bytes past a 16-byte boundary, or its last row): thread 0 only.
template <bool MAT>
__device__ void bypass_edge_row(const BypassArgs &a, const uint32_t *filt, const uint32_t *hkeys,
                                unsigned *hcnt, uint32_t *hist, unsigned *s_keep, uint2 *dst, Row x,
                                unsigned long long &matches, unsigned long long &heavy_rows) {
    const int s = heavy_slot(filt, hkeys, x.key);
    if (s < 0) {
        atomicAdd(&hist[radix_f(a.rf, x.key)], 1u);
        dst[atomicAdd(s_keep, 1u)] = make_uint2(x.key, x.payload);
        return;
    }
    heavy_rows++;
    if (!MAT) {  // counting: hcnt is this block's S rows per heavy slot
        atomicAdd(&hcnt[s], 1u);
        return;
    }
    const unsigned c = hcnt[s];
    matches += c;
    if (c) {
        uint64_t op = atomicAdd(a.rows_ctr, (unsigned long long)c);
        const unsigned st0 = a.hstart[s];
        for (unsigned q = 0; q < c; q++, op++)
            if (op < a.cap) a.rows[op] = tbg_row_out{x.key, a.rpay[st0 + q], x.payload};
    }
}

// Materialising, hcnt holds R's rows per heavy slot and every heavy S row
// emits its pairs on the spot.  Counting, it counts this block's S rows per
// heavy slot instead (added to a.scnt at the end): the join's heavy matches
// are sum_slot S rows x R rows, formed after R's heavy rows are counted on
// the other stream (k_heavy_sum), so that count is off this kernel's path.
template <bool MAT>
__global__ void __launch_bounds__(1024) k_hist_bypass(BypassArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *hkeys = reinterpret_cast<uint32_t *>(smem);  // 16-byte aligned buckets
    unsigned *hcnt = hkeys + HEAVY_CAP;
    uint32_t *filt = hcnt + HEAVY_CAP;                     // 2^FILTER_LOG2 bits
    uint32_t *hist = filt + (1 << FILTER_LOG2) / 32;
    __shared__ unsigned s_keep;
    __shared__ uint64_t scan_scratch[1024 / 32 + 1];
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < a.nbins; i += 1024) hist[i] = 0;
    for (int i = tid; i < (1 << FILTER_LOG2) / 32; i += 1024) filt[i] = a.filter[i];
    for (int i = tid; i < HEAVY_CAP; i += 1024) {
        hkeys[i] = a.hkeys[i];
        hcnt[i] = MAT ? a.hcnt[i] : 0u;
    }
    if (tid == 0) s_keep = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * a.chunk;
    const uint64_t hi = umin64(a.n, lo + a.chunk);
    const uint32_t len = hi > lo ? (uint32_t)(hi - lo) : 0u;  // a chunk holds < 2^32 rows
    const Row *src = a.in + lo;
    uint2 *dst = reinterpret_cast<uint2 *>(a.out + lo);
    const uint32_t head = (len && (reinterpret_cast<uintptr_t>(src) & 15)) ? 1u : 0u;
    const uint32_t npairs = (len - head) / 2;
    const bool tail = ((len - head) & 1) != 0;
    const uint4 *v = reinterpret_cast<const uint4 *>(src + head);
    unsigned long long matches = 0, heavy_rows = 0;
    // rounds of 4 row pairs per thread: pair p = base + u * 1024 + tid
    for (uint32_t base = 0; base < npairs; base += 4 * 1024) {
        uint32_t k[8], pv[8];
        unsigned valid = 0;
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint32_t p = base + u * 1024 + tid;
            k[2 * u] = k[2 * u + 1] = EMPTY_KEY;
            pv[2 * u] = pv[2 * u + 1] = 0;
            if (p < npairs) {
                const uint4 x = ldg_stream(v + p);
                k[2 * u] = x.x;
                pv[2 * u] = x.y;
                k[2 * u + 1] = x.z;
                pv[2 * u + 1] = x.w;
                valid |= 3u << (2 * u);
            }
        }
        int slot[8];
#pragma unroll
        for (int j = 0; j < 8; j++) slot[j] = (valid >> j & 1) ? heavy_slot(filt, hkeys, k[j]) : -1;
        unsigned keep = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            if (slot[j] >= 0) {
                if (MAT) matches += hcnt[slot[j]];
                heavy_rows++;
            } else if (valid >> j & 1) {
                keep |= 1u << j;
            }
        }
        if (!MAT) {  // S rows per heavy slot; a warp's rows of one hot key add once
            const bool dup = warp_has_dups((uint32_t)slot[0], slot[0] >= 0);
#pragma unroll
            for (int j = 0; j < 8; j++) hist_add_warp(hcnt, slot[j] >= 0 ? (uint32_t)slot[j] : 0u, slot[j] >= 0, dup);
        }
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
                dst[wb + __popc(m[j] & lt)] = make_uint2(k[j], pv[j]);
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
                        if (op < a.cap) a.rows[op] = tbg_row_out{k[j], a.rpay[st0 + q], pv[j]};
                }
            }
        }
    }
    __syncthreads();  // every vector row is counted: the edge rows take the next output slots
    if (tid == 0) {
        if (head) bypass_edge_row<MAT>(a, filt, hkeys, hcnt, hist, &s_keep, dst, src[0], matches, heavy_rows);
        if (tail) bypass_edge_row<MAT>(a, filt, hkeys, hcnt, hist, &s_keep, dst, src[len - 1], matches, heavy_rows);
    }
    __syncthreads();
    uint32_t *hdst = a.hist + (uint64_t)blockIdx.x * a.nbins;
    for (int i = tid; i < a.nbins; i += 1024) hdst[i] = hist[i];
    if (!MAT)
        for (int i = tid; i < HEAVY_CAP; i += 1024)
            if (hcnt[i]) atomicAdd(&a.scnt[i], hcnt[i]);
    if (tid == 0) a.kept[blockIdx.x] = s_keep;
    const unsigned long long wm = warp_sum_u64(matches), wh = warp_sum_u64(heavy_rows);
    if (lane == 0) {
        if (wm) atomicAdd(a.matches, wm);
        if (wh) atomicAdd(a.heavy_rows, wh);
    }
}

// Heavy matches of a counting join: sum over slots of R rows x S rows.
__global__ void __launch_bounds__(1024) k_heavy_sum(const unsigned *__restrict__ rcnt,
                                                   const unsigned *__restrict__ scnt, unsigned long long *matches) {
    unsigned long long m = 0;
    for (int i = threadIdx.x; i < HEAVY_CAP; i += 1024) m += (unsigned long long)rcnt[i] * scnt[i];
    m = warp_sum_u64(m);
    if ((threadIdx.x & 31) == 0 && m) atomicAdd(matches, m);
}

cudaError_t launch_heavy_sum(const unsigned *rcnt, const unsigned *scnt, unsigned long long *matches,
                             cudaStream_t st) {
    k_heavy_sum<<<1, 1024, 0, st>>>(rcnt, scnt, matches);
    count_launch();
    return cudaGetLastError();
}

size_t bypass_smem(int nbins, bool mat) {
    (void)mat;  // heavy keys + counts + filter + 2^15 bins: 204,800 B at most
    return (size_t)HEAVY_CAP * 4 * 2 + (1 << FILTER_LOG2) / 8 + (size_t)nbins * 4;
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
