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
constexpr int P_W1 = 0, P_B1 = MLP_H, P_W2 = 2 * MLP_H, P_B2 = P_W2 + MLP_H * MLP_H, P_W3 = P_B2 + MLP_H,
              P_B3 = P_W3 + MLP_H;

// tanh(x) = 1 - 2 / (e^(2x) + 1), through the fast exponential: about 1e-7
// absolute error, a fraction of the instructions of tanhf.  |x| <= 15 keeps
// e^(2x) finite; tanh(15) rounds to 1 in single precision.
__device__ __forceinline__ float tanh_f(float x) {
    x = fminf(fmaxf(x, -15.f), 15.f);
    return 1.f - __fdividef(2.f, __expf(2.f * x) + 1.f);
}

// One evaluation by one thread (the decision's model evaluations).
__device__ float mlp_eval(const float *__restrict__ p, float x) {
    float h1[MLP_H];
#pragma unroll
    for (int i = 0; i < MLP_H; i++) h1[i] = tanh_f(p[P_W1 + i] * x + p[P_B1 + i]);
    float out = p[P_B3];
#pragma unroll 4
    for (int o = 0; o < MLP_H; o++) {
        float z = p[P_B2 + o];
#pragma unroll
        for (int i = 0; i < MLP_H; i++) z += p[P_W2 + o * MLP_H + i] * h1[i];
        out += p[P_W3 + o] * tanh_f(z);
    }
    return out;
}

// A batch of MLP_BATCH_CTA samples is processed by MLP_TRAIN_THREADS threads
// (16 warps).  Forward and backward: warp w serves samples 32 (w / 4) + lane
// and hidden units [8 (w % 4), 8 (w % 4) + 8) of both layers, so the lanes of
// a warp read every weight as a broadcast; the four warps of a sample group
// exchange activations through shared memory under a named barrier.  The
// per-sample rows have a stride of MLP_H + 1 floats: a warp's lanes (one
// sample each) touch distinct banks.
constexpr int RS = MLP_H + 1;
constexpr int MLP_UNITS_WARP = MLP_H / 4;  // hidden units per warp
constexpr int GR_SLICES = 8;               // sample slices of the parameter-gradient sums
static_assert(MLP_TRAIN_THREADS == 4 * MLP_BATCH_CTA, "four warps per 32 samples");
static_assert(MLP_TRAIN_THREADS == 64 * GR_SLICES && MLP_BATCH_CTA % GR_SLICES == 0, "gradient slices");

struct BatchSmem {
    float h1[MLP_BATCH_CTA][RS];
    float h2[MLP_BATCH_CTA][RS];
    float dz2[MLP_BATCH_CTA][RS];
    float dz1[MLP_BATCH_CTA][RS];
    float x[MLP_BATCH_CTA];
    float dout[MLP_BATCH_CTA];
    float part[4][MLP_BATCH_CTA];  // output partial of each unit group
    alignas(16) float red[GR_SLICES][MLP_PARAMS_PAD];  // per-slice gradient partials
};

__device__ __forceinline__ float4 ld4(const float *a) { return *reinterpret_cast<const float4 *>(a); }

// Barrier of the four warps of sample group g (named barriers 1 .. 4, given
// as immediates so that the kernel reserves only those).
__device__ __forceinline__ void group_sync(int g) {
    switch (g) {
        case 0: asm volatile("bar.sync 1, 128;" ::: "memory"); break;
        case 1: asm volatile("bar.sync 2, 128;" ::: "memory"); break;
        case 2: asm volatile("bar.sync 3, 128;" ::: "memory"); break;
        default: asm volatile("bar.sync 4, 128;" ::: "memory"); break;
    }
}

// Dot product of a 16-byte aligned shared row of MLP_H floats with v
// (two accumulators).
__device__ __forceinline__ float dot_row(const float *w, const float (&v)[MLP_H], float acc) {
    float a0 = acc, a1 = 0.f;
#pragma unroll
    for (int i = 0; i < MLP_H; i += 8) {
        const float4 x = ld4(w + i), y = ld4(w + i + 4);
        a0 = fmaf(x.x, v[i], a0);
        a1 = fmaf(x.y, v[i + 1], a1);
        a0 = fmaf(x.z, v[i + 2], a0);
        a1 = fmaf(x.w, v[i + 3], a1);
        a0 = fmaf(y.x, v[i + 4], a0);
        a1 = fmaf(y.y, v[i + 5], a1);
        a0 = fmaf(y.z, v[i + 6], a0);
        a1 = fmaf(y.w, v[i + 7], a1);
    }
    return a0 + a1;
}

// Forward and backward of sample s (input x, target y, loss weight scale) by
// warp j of its sample group g, which owns hidden units [8j, 8j + 8).
// Leaves the sample's activations, pre-activation gradients and output
// gradient in row s; returns the squared error.  Every thread of the group
// calls it (named barriers).
__device__ float group_fwd_bwd(const float *p, BatchSmem &b, float x, float y, float scale, int s, int g, int j) {
    constexpr int U = MLP_UNITS_WARP;
    const int u0 = U * j;
    float *h1 = b.h1[s], *h2 = b.h2[s], *dz2 = b.dz2[s], *dz1 = b.dz1[s];
#pragma unroll
    for (int t = 0; t < U; t++) h1[u0 + t] = tanh_f(p[P_W1 + u0 + t] * x + p[P_B1 + u0 + t]);
    group_sync(g);
    float v[MLP_H];
#pragma unroll
    for (int i = 0; i < MLP_H; i++) v[i] = h1[i];
    float part = 0.f, g2[U];
#pragma unroll
    for (int t = 0; t < U; t++) {
        const int u = u0 + t;
        const float h = tanh_f(dot_row(p + P_W2 + u * MLP_H, v, p[P_B2 + u]));
        h2[u] = h;
        const float w3 = p[P_W3 + u];
        part = fmaf(w3, h, part);
        g2[t] = w3 * (1.f - h * h);
    }
    b.part[j][s] = part;
    group_sync(g);
    const float r = p[P_B3] + ((b.part[0][s] + b.part[1][s]) + (b.part[2][s] + b.part[3][s])) - y;
    const float dout = 2.f * r * scale;
#pragma unroll
    for (int t = 0; t < U; t++) dz2[u0 + t] = dout * g2[t];
    group_sync(g);
#pragma unroll
    for (int o = 0; o < MLP_H; o++) v[o] = dz2[o];
    // dz1[i] = (1 - h1[i]^2) sum_o W2[o][i] dz2[o] for the warp's units i
    float acc[U];
#pragma unroll
    for (int t = 0; t < U; t++) acc[t] = 0.f;
#pragma unroll
    for (int o = 0; o < MLP_H; o++) {
        const float4 a = ld4(p + P_W2 + o * MLP_H + u0), c = ld4(p + P_W2 + o * MLP_H + u0 + 4);
        acc[0] = fmaf(a.x, v[o], acc[0]);
        acc[1] = fmaf(a.y, v[o], acc[1]);
        acc[2] = fmaf(a.z, v[o], acc[2]);
        acc[3] = fmaf(a.w, v[o], acc[3]);
        acc[4] = fmaf(c.x, v[o], acc[4]);
        acc[5] = fmaf(c.y, v[o], acc[5]);
        acc[6] = fmaf(c.z, v[o], acc[6]);
        acc[7] = fmaf(c.w, v[o], acc[7]);
    }
#pragma unroll
    for (int t = 0; t < U; t++) {
        const float a = h1[u0 + t];
        dz1[u0 + t] = acc[t] * (1.f - a * a);
    }
    if (j == 0) {
        b.x[s] = x;
        b.dout[s] = dout;
    }
    return r * r;
}

// Gradient of every parameter summed over samples 0 .. nb of the batch, into
// g[0 .. MLP_PARAMS), by all MLP_TRAIN_THREADS threads (a __syncthreads
// inside).  Slice k of GR_SLICES takes samples [16k, 16k + 16) on 64
// threads: each sums one 4 x 4 tile of W2's gradient and two or three of the
// other parameters over its slice into the slice's partials; then every
// thread adds the slices' partials of its parameters.
__device__ void batch_param_grad(BatchSmem &b, int nb, float *g) {
    constexpr int SPAN = MLP_BATCH_CTA / GR_SLICES;
    const int tid = threadIdx.x, sl = tid >> 6, t = tid & 63;
    const int s0 = sl * SPAN, s1 = min(nb, s0 + SPAN);
    float *red = b.red[sl];
    {
        const int o0 = (t >> 3) * 4, i0 = (t & 7) * 4;
        float acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][c] = 0.f;
        for (int s = s0; s < s1; s++) {
            float d[4], h[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                d[k] = b.dz2[s][o0 + k];
                h[k] = b.h1[s][i0 + k];
            }
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][c] = fmaf(d[a], h[c], acc[a][c]);
        }
#pragma unroll
        for (int a = 0; a < 4; a++)
            *reinterpret_cast<float4 *>(red + P_W2 + (o0 + a) * MLP_H + i0) =
                make_float4(acc[a][0], acc[a][1], acc[a][2], acc[a][3]);
    }
    // the slice's first warp: W1[i] and b2[i]; its second: b1[i] and W3[i];
    // thread 0 also b3 (i = lane, MLP_H = 32)
    {
        static_assert(MLP_H == 32, "one lane per hidden unit");
        const int i = t & 31;
        float a = 0.f, c = 0.f;
        if (t < 32) {
            for (int s = s0; s < s1; s++) {
                a = fmaf(b.dz1[s][i], b.x[s], a);
                c += b.dz2[s][i];
            }
            red[P_W1 + i] = a;
            red[P_B2 + i] = c;
        } else {
            for (int s = s0; s < s1; s++) {
                a += b.dz1[s][i];
                c = fmaf(b.dout[s], b.h2[s][i], c);
            }
            red[P_B1 + i] = a;
            red[P_W3 + i] = c;
        }
        if (t == 0) {
            float d = 0.f;
            for (int s = s0; s < s1; s++) d += b.dout[s];
            red[P_B3] = d;
        }
    }
    __syncthreads();
    for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) {
        float a = 0.f;
#pragma unroll
        for (int k = 0; k < GR_SLICES; k++) a += b.red[k][q];
        g[q] = a;
    }
}

// Full-batch gradient and loss sum over n samples (tests and the reported
// training loss): CTAs take MLP_BATCH_CTA samples each and add their partial
// gradients to grad[] with atomics.
__global__ void __launch_bounds__(MLP_TRAIN_THREADS, 1) k_mlp_grad(const float *__restrict__ params,
                                                                const float *__restrict__ xs,
                                                                const float *__restrict__ ys, uint32_t n,
                                                                float *grad, float *loss_sum) {
    extern __shared__ __align__(16) unsigned char smem[];
    float *p = reinterpret_cast<float *>(smem);
    float *gl = p + MLP_PARAMS_PAD;
    BatchSmem &b = *reinterpret_cast<BatchSmem *>(gl + MLP_PARAMS_PAD);
    const int tid = threadIdx.x, w = tid >> 5, g = w >> 2, j = w & 3, s = 32 * g + (tid & 31);
    for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) p[q] = params[q];
    __syncthreads();
    const uint32_t s0 = blockIdx.x * MLP_BATCH_CTA;
    const int nb = (int)min((uint32_t)MLP_BATCH_CTA, n - s0);
    const bool ok = s < nb;
    // every group runs (named barriers); samples past n add nothing
    const float l = group_fwd_bwd(p, b, ok ? xs[s0 + s] : 0.f, ok ? ys[s0 + s] : 0.f, 1.f / (float)n, s, g, j);
    __syncthreads();
    batch_param_grad(b, nb, gl);
    __syncthreads();
    for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) atomicAdd(&grad[q], gl[q]);
    float lw = (ok && j == 0) ? l : 0.f;
    for (int o = 16; o > 0; o >>= 1) lw += __shfl_xor_sync(0xffffffffu, lw, o);
    if ((tid & 31) == 0) atomicAdd(loss_sum, lw);
}

// Training points staged in the trainer's shared memory (larger point sets
// are read from global memory).
constexpr int MLP_STAGE = CC_BINS;

// Trainer: one cluster of MLP_CLUSTER CTAs, persistent over all steps.  Each
// step every CTA draws MLP_BATCH_CTA seeded random training points (uniformly,
// or in proportion to their weights), runs their forward and backward passes
// and its partial parameter gradient; after a
// cluster barrier CTA r sums the partials of its parameter slice from every
// CTA's shared memory, applies Adam, and writes the new values into every
// CTA's parameter copy; a second barrier ends the step.
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
    float *sx = reinterpret_cast<float *>(&b + 1), *sy = sx + MLP_STAGE, *scw = sy + MLP_STAGE;
    const int tid = threadIdx.x, w = tid >> 5, g = w >> 2, j = w & 3, s = 32 * g + (tid & 31);
    const bool staged = n <= (uint32_t)MLP_STAGE;
    for (int q = tid; q < MLP_PARAMS; q += MLP_TRAIN_THREADS) p[q] = params[q];
    for (int q = tid; q < MLP_SLICE; q += MLP_TRAIN_THREADS) am[q] = av[q] = 0.f;
    if (staged)
        for (uint32_t q = tid; q < n; q += MLP_TRAIN_THREADS) {
            sx[q] = xs[q];
            sy[q] = ys[q];
            if (cw) scw[q] = cw[q];
        }
    const float *px = staged ? sx : xs, *py = staged ? sy : ys, *pw = staged ? scw : cw;
    cl.sync();
    const float b1c = 0.9f, b2c = 0.999f, eps = 1e-8f;
    const float scale = 1.f / (float)(MLP_BATCH_CTA * MLP_CLUSTER);
    const int q0 = rank * MLP_SLICE, q1 = min(MLP_PARAMS, q0 + MLP_SLICE);
    const float wtot = cw ? pw[n - 1] : 0.f;
    float pow1 = 1.f, pow2 = 1.f;
    for (int step = 0; step < steps; step++) {
        // sample s: the group's first warp draws the point, the other three
        // read it after the group barrier
        if (j == 0) {
            const uint64_t hsh = mix64(seed ^ mix64(((uint64_t)step << 20) | (uint64_t)(rank * MLP_BATCH_CTA + s)));
            uint32_t i;
            if (cw) {  // the first point whose cumulative weight exceeds u * total
                const float u = (float)((hsh >> 40) * (1.0 / 16777216.0)) * wtot;
                uint32_t lo = 0, hi = n - 1;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (pw[mid] > u) hi = mid;
                    else lo = mid + 1;
                }
                i = lo;
            } else {
                i = (uint32_t)(hsh % n);
            }
            b.x[s] = px[i];
            b.dout[s] = py[i];  // the target, until the backward pass overwrites it
        }
        group_sync(g);
        group_fwd_bwd(p, b, b.x[s], b.dout[s], scale, s, g, j);
        __syncthreads();
        batch_param_grad(b, MLP_BATCH_CTA, gpart);
        cl.sync();
        pow1 *= b1c;
        pow2 *= b2c;
        // cosine decay from lr0 to lr0 / 10
        const float lr = lr0 * (0.55f + 0.45f * cospif((float)step / (float)(steps > 1 ? steps - 1 : 1)));
        for (int q = q0 + tid; q < q1; q += MLP_TRAIN_THREADS) {
            float gs = 0.f;
            for (int r = 0; r < MLP_CLUSTER; r++) gs += cl.map_shared_rank(gpart, r)[q];
            const int k = q - q0;
            am[k] = b1c * am[k] + (1.f - b1c) * gs;
            av[k] = b2c * av[k] + (1.f - b2c) * gs * gs;
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
    return (size_t)(2 * MLP_PARAMS_PAD + 2 * MLP_SLICE) * 4 + sizeof(BatchSmem) + (size_t)3 * MLP_STAGE * 4;
}
size_t mlp_grad_smem() { return (size_t)2 * MLP_PARAMS_PAD * 4 + sizeof(BatchSmem); }

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
    k_mlp_grad<<<(n + MLP_BATCH_CTA - 1) / MLP_BATCH_CTA, MLP_TRAIN_THREADS, smem, st>>>(params, xs, ys, n, grad,
                                                                                         loss_sum);
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

// The global count table: one 64-bit word per slot, key << 32 | count, so a
// new key is claimed and counted by one compare-and-swap.  CNT_EMPTY (all
// ones) marks a free slot: its key is EMPTY_KEY, which is never counted.
constexpr unsigned long long CNT_EMPTY = ~0ull;
__device__ __forceinline__ unsigned long long cnt_word(uint32_t k, uint32_t c) {
    return ((unsigned long long)k << 32) | c;
}

// Adds c to key k's count, probing from slot h.  A full table drops the key:
// a key that is not counted is never heavy, which only costs speed.
__device__ __forceinline__ void table_add(unsigned long long *t, uint32_t tmask, uint32_t k, uint32_t c, uint32_t h) {
    for (uint32_t probe = 0; probe <= tmask && probe < 4096; probe++) {
        const unsigned long long old = atomicCAS(&t[h], CNT_EMPTY, cnt_word(k, c));
        if (old == CNT_EMPTY) return;
        if ((uint32_t)(old >> 32) == k) {
            atomicAdd(&t[h], (unsigned long long)c);  // the count is the low word; it never carries
            return;
        }
        h = (h + 1) & tmask;
    }
}

// Counts the sample's keys: CTA c aggregates keys [c * CNT_CHUNK, ...) in a
// shared table (equal keys of a warp first combined with __match_any_sync,
// so a hot key costs one shared atomic per warp), then adds each distinct
// key once to the global table: every thread first issues the
// compare-and-swap of each of its slots at the key's home slot, and only the
// slots that met another key probe on.  Key EMPTY_KEY is never counted.
__global__ void __launch_bounds__(CNT_THREADS, 2) k_count_keys(const uint32_t *__restrict__ keys, uint64_t m,
                                                           unsigned long long *table, uint32_t tmask) {
    constexpr int SLOTS = 2 * CNT_CHUNK;
    constexpr int PER = 4;  // flush: slots per thread per batch of compare-and-swaps
    extern __shared__ __align__(16) uint32_t cnt_smem[];
    uint32_t *lk = cnt_smem, *lc = cnt_smem + SLOTS;
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
    for (int base = 0; base < SLOTS; base += PER * CNT_THREADS) {
        uint32_t fk[PER];
        unsigned long long old[PER];
#pragma unroll
        for (int q = 0; q < PER; q++) {  // independent: the compare-and-swaps are all in flight at once
            const int i = base + q * CNT_THREADS + threadIdx.x;
            fk[q] = lk[i];
            old[q] = fk[q] != EMPTY_KEY
                         ? atomicCAS(&table[count_hash(fk[q]) & tmask], CNT_EMPTY, cnt_word(fk[q], lc[i]))
                         : CNT_EMPTY;
        }
#pragma unroll
        for (int q = 0; q < PER; q++) {
            if (fk[q] == EMPTY_KEY || old[q] == CNT_EMPTY) continue;
            const uint32_t h = count_hash(fk[q]) & tmask, c = lc[base + q * CNT_THREADS + threadIdx.x];
            if ((uint32_t)(old[q] >> 32) == fk[q]) atomicAdd(&table[h], (unsigned long long)c);
            else table_add(table, tmask, fk[q], c, (h + 1) & tmask);
        }
    }
}

cudaError_t launch_count_keys(const LearnBufs &b, uint64_t m, cudaStream_t st) {
    if (!m) return cudaSuccess;
    const size_t smem = (size_t)CNT_CHUNK * 2 * 8;
    cudaError_t e = smem_limit((const void *)k_count_keys, smem);
    if (e != cudaSuccess) return e;
    k_count_keys<<<(unsigned)((m + CNT_CHUNK - 1) / CNT_CHUNK), CNT_THREADS, smem, st>>>(b.keys, m, b.table, b.tmask);
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
// Each thread reads STATS_PER consecutive slots per round.  Lanes whose count
// falls in the same exact bin (most of them: counts 1, 2, 3 ...) add to it
// once per warp (__match_any_sync); the candidates' list positions come
// from one global atomic per CTA and round.
constexpr int STATS_THREADS = 1024;
constexpr int STATS_PER = 4;

__global__ void __launch_bounds__(STATS_THREADS, 2) k_count_stats(const unsigned long long *__restrict__ table,
                                                               uint32_t tmask, unsigned *bin_keys,
                                                               unsigned long long *bin_rows, HeavyCand *cand,
                                                               unsigned cand_cap, LrnDecision *dec) {
    __shared__ unsigned sk[CC_BINS];
    __shared__ unsigned long long sr[CC_BINS];
    __shared__ unsigned wbase[STATS_THREADS / 32];
    for (int i = threadIdx.x; i < CC_BINS; i += STATS_THREADS) {
        sk[i] = 0;
        sr[i] = 0;
    }
    __syncthreads();
    const uint64_t groups = ((uint64_t)tmask + 1) / STATS_PER;  // a multiple of STATS_THREADS
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = lanemask_lt();
    for (uint64_t base = (uint64_t)blockIdx.x * STATS_THREADS; base < groups;
         base += (uint64_t)gridDim.x * STATS_THREADS) {
        const uint64_t g = base + threadIdx.x;  // warp- and block-uniform trip count
        const ulonglong2 a = reinterpret_cast<const ulonglong2 *>(table)[2 * g];
        const ulonglong2 c = reinterpret_cast<const ulonglong2 *>(table)[2 * g + 1];
        const unsigned long long wv[STATS_PER] = {a.x, a.y, c.x, c.y};
        unsigned cm = 0;
        // counts 1 and 2 (most keys) by two ballots; a warp holding a larger
        // count groups those lanes by count (__match_any_sync)
        unsigned n1 = 0, n2 = 0;
#pragma unroll
        for (int q = 0; q < STATS_PER; q++) {
            const uint32_t k = (uint32_t)(wv[q] >> 32), n = (uint32_t)wv[q];
            const bool used = k != EMPTY_KEY && n > 0;
            n1 += __popc(__ballot_sync(0xffffffffu, used && n == 1));
            n2 += __popc(__ballot_sync(0xffffffffu, used && n == 2));
            const bool big = used && n > 2;
            if (__ballot_sync(0xffffffffu, big)) {
                const bool exact = big && n < (uint32_t)CC_EXACT;
                const unsigned peers = __match_any_sync(0xffffffffu, exact ? n : 0xFFFFFFFFu);
                if (exact) {
                    if ((peers & lt) == 0) {
                        const unsigned cnt = (unsigned)__popc(peers);
                        atomicAdd(&sk[n], cnt);
                        atomicAdd(&sr[n], (unsigned long long)cnt * n);
                    }
                } else if (big) {
                    const int b = cc_bin(n);
                    atomicAdd(&sk[b], 1u);
                    atomicAdd(&sr[b], (unsigned long long)n);
                }
            }
            if (used && n >= (uint32_t)CAND_MIN_COUNT) cm |= 1u << q;
        }
        if (lane == 0) {
            if (n1) {
                atomicAdd(&sk[1], n1);
                atomicAdd(&sr[1], (unsigned long long)n1);
            }
            if (n2) {
                atomicAdd(&sk[2], n2);
                atomicAdd(&sr[2], 2ull * n2);
            }
        }
        // candidate positions: warp prefix, then one global atomic per CTA
        uint32_t inc = (uint32_t)__popc(cm);
        const uint32_t mine = inc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wbase[w] = inc;
        __syncthreads();
        if (w == 0) {
            const uint32_t t = wbase[lane];
            uint32_t x = t;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            unsigned b0 = 0;
            if (lane == 31 && x) b0 = atomicAdd(&dec->ncand, x);
            b0 = __shfl_sync(0xffffffffu, b0, 31);
            wbase[lane] = b0 + x - t;
        }
        __syncthreads();
        unsigned pos = wbase[w] + inc - mine;
#pragma unroll
        for (int q = 0; q < STATS_PER; q++) {
            if (cm >> q & 1) {
                if (pos < cand_cap) cand[pos] = HeavyCand{(uint32_t)(wv[q] >> 32), (uint32_t)wv[q]};
                pos++;
            }
        }
        __syncthreads();  // wbase is rewritten next round
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
    // four rounds per CTA, two CTAs per SM: one CTA's loads and barriers
    // overlap the other's
    const uint64_t groups = ((uint64_t)b.tmask + 1) / STATS_PER;
    const unsigned g = (unsigned)std::max<uint64_t>(1, groups / (STATS_THREADS * 4));
    k_count_stats<<<g, STATS_THREADS, 0, st>>>(b.table, b.tmask, b.bin_keys, b.bin_rows, b.cand, b.cand_cap, b.dec);
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

// Model evaluations for the decision, spread over many CTAs (one evaluation
// per thread): lpred[r] = log2 of the predicted S rows of sample rank r,
// mu + sigma M(rank_feature(r)) + log2(nS / m), for r = 1 .. HEAVY_MAX + 1
// (mu and sigma the points' normalisation), and the squared error of the
// model on the training points, added to dec->loss_sum.
constexpr int EVAL_THREADS = 256;
constexpr int EVAL_RANKS = HEAVY_MAX + 1;

__global__ void __launch_bounds__(EVAL_THREADS) k_model_eval(const float *__restrict__ params,
                                                            const float *__restrict__ xs,
                                                            const float *__restrict__ ys, double lscale,
                                                            float *lpred, LrnDecision *dec) {
    __shared__ float p[MLP_PARAMS];
    for (int q = threadIdx.x; q < MLP_PARAMS; q += EVAL_THREADS) p[q] = params[q];
    __syncthreads();
    const unsigned np = dec->npoints;
    const int g = blockIdx.x * EVAL_THREADS + threadIdx.x;
    double err = 0.0;
    if (g < EVAL_RANKS) {
        const int r = g + 1;
        lpred[r] = (float)((double)dec->y_mu + (double)dec->y_sigma * (double)mlp_eval(p, rank_feature((double)r)) +
                           lscale);
    } else if ((unsigned)(g - EVAL_RANKS) < np) {
        const unsigned i = (unsigned)(g - EVAL_RANKS);
        const double d = (double)mlp_eval(p, xs[i]) - (double)ys[i];
        err = d * d;
    }
    for (int o = 16; o > 0; o >>= 1) err += __shfl_xor_sync(0xffffffffu, err, o);
    if ((threadIdx.x & 31) == 0 && err > 0.0) atomicAdd(&dec->loss_sum, err);
}

// The decision (one block).  pred(r), the predicted S rows of the key of
// sample rank r, comes from the model (lpred from k_model_eval) or, for the
// ablation, from the sample's own count at rank r.  k* = the ranks
// 1 .. HEAVY_MAX whose predicted rows reach tau_min; the heavy keys are the
// sampled keys whose count is at least that of rank k* (the lowest count bin
// that keeps their number <= k*).  Bypass when the model predicts those keys
// to hold at least min_frac of S.  The bins are read in decreasing count
// order (j = CC_BINS - 1 - bin); above[j] counts the keys of the bins before
// j, so rank r lies in the last j with above[j] < r, found by binary search.
constexpr int DECIDE_THREADS = 1024;
constexpr int DECIDE_PER = (CC_BINS + DECIDE_THREADS - 1) / DECIDE_THREADS;

__global__ void __launch_bounds__(DECIDE_THREADS) k_decide(int use_model, const unsigned *__restrict__ bin_keys,
                                                          const unsigned long long *__restrict__ bin_rows,
                                                          const float *__restrict__ lpred_model, double rows_scale,
                                                          double nS, double tau_min, double min_frac,
                                                          LrnDecision *dec) {
    const double lscale = log2(rows_scale);  // log2(nS / m): sample rows to S rows
    __shared__ float lp[EVAL_RANKS + 1];  // log2 of the predicted S rows of rank r (r = 1 .. HEAVY_MAX + 1)
    __shared__ uint64_t scratch[DECIDE_THREADS / 32 + 1];
    __shared__ double red[DECIDE_THREADS / 32];
    __shared__ unsigned s_kstar, s_jstar;
    extern __shared__ __align__(16) unsigned char dsm[];
    unsigned long long *sr = reinterpret_cast<unsigned long long *>(dsm);  // rows, by j
    unsigned *sk = reinterpret_cast<unsigned *>(sr + CC_BINS);             // keys, by j
    unsigned *above = sk + CC_BINS;                                        // keys before j
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint64_t mine = 0;
#pragma unroll
    for (int q = 0; q < DECIDE_PER; q++) {
        const int j = t * DECIDE_PER + q;
        if (j < CC_BINS) {
            sk[j] = bin_keys[CC_BINS - 1 - j];
            sr[j] = bin_rows[CC_BINS - 1 - j];
            mine += sk[j];
        }
    }
    if (t == 0) {
        s_kstar = 0;
        s_jstar = 0;  // j* + 1 of the last heavy bin; 0: none
    }
    uint64_t total;
    uint64_t run = block_excl_scan<DECIDE_THREADS>(mine, &total, scratch);
#pragma unroll
    for (int q = 0; q < DECIDE_PER; q++) {
        const int j = t * DECIDE_PER + q;
        if (j < CC_BINS) {
            above[j] = (unsigned)run;
            run += sk[j];
        }
    }
    __syncthreads();
    // per rank: the sample count (mean of its bin), the prediction, and the
    // largest rank <= HEAVY_MAX predicted at or above tau_min among the ranks
    // the sample saw at least CAND_MIN_COUNT times
    const float ltau = (float)log2(tau_min);
    unsigned last_ok = 0;
    for (int r = 1 + t; r <= EVAL_RANKS; r += DECIDE_THREADS) {
        uint32_t c = 0;
        if ((uint64_t)r <= total) {
            int lo = 0, hi = CC_BINS - 1;  // last j with above[j] < r
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (above[mid] < (unsigned)r) lo = mid;
                else hi = mid - 1;
            }
            c = sk[lo] ? (uint32_t)(sr[lo] / sk[lo]) : 0u;
        }
        const float l = use_model ? lpred_model[r] : (c ? (float)(log2((double)c) + lscale) : -INFINITY);
        lp[r] = l;
        if (r <= HEAVY_MAX && l >= ltau && c >= (uint32_t)CAND_MIN_COUNT) last_ok = max(last_ok, (unsigned)r);
    }
    for (int o = 16; o > 0; o >>= 1) last_ok = max(last_ok, __shfl_xor_sync(0xffffffffu, last_ok, o));
    if (lane == 0 && last_ok) atomicMax(&s_kstar, last_ok);
    __syncthreads();
    const unsigned kstar = s_kstar;
    // predicted mass of ranks 1 .. k*
    double mass = 0.0;
    for (int r = 1 + t; r <= (int)kstar; r += DECIDE_THREADS) mass += exp2((double)lp[r]);
    // heavy bins: the non-empty bins of count >= CAND_MIN_COUNT whose keys,
    // with all before them, number <= k* (a prefix of j); j* the last of them
#pragma unroll
    for (int q = 0; q < DECIDE_PER; q++) {
        const int j = t * DECIDE_PER + q;
        if (j < CC_BINS && kstar && sk[j] && CC_BINS - 1 - j >= CAND_MIN_COUNT && above[j] + sk[j] <= kstar)
            atomicMax(&s_jstar, (unsigned)j + 1);  // +1: 0 means none
    }
    for (int o = 16; o > 0; o >>= 1) mass += __shfl_xor_sync(0xffffffffu, mass, o);
    if (lane == 0) red[w] = mass;
    __syncthreads();
    const unsigned jst = s_jstar;  // j* + 1, or 0
    double rows = 0.0;
#pragma unroll
    for (int q = 0; q < DECIDE_PER; q++) {
        const int j = t * DECIDE_PER + q;
        if (j < CC_BINS && (unsigned)j < jst) rows += (double)sr[j];
    }
    double pred_mass = 0.0;
    for (int i = 0; i < DECIDE_THREADS / 32; i++) pred_mass += red[i];
    __syncthreads();
    for (int o = 16; o > 0; o >>= 1) rows += __shfl_xor_sync(0xffffffffu, rows, o);
    if (lane == 0) red[w] = rows;
    __syncthreads();
    if (t == 0) {
        double srows = 0.0;
        for (int i = 0; i < DECIDE_THREADS / 32; i++) srows += red[i];
        const unsigned heavy = jst ? above[jst - 1] + sk[jst - 1] : 0u;
        LrnDecision d = *dec;
        d.k_star = kstar;
        d.count_min = jst ? cc_bin_min(CC_BINS - (int)jst) : 0xFFFFFFFFu;
        d.heavy_sample = heavy;
        d.pred_mass = pred_mass;
        d.sample_mass = srows * rows_scale;
        d.next_rows = kstar < (unsigned)HEAVY_MAX ? exp2((double)lp[kstar + 1]) : 0.0;
        d.loss = d.npoints ? (float)(d.loss_sum / d.npoints) : 0.f;
        d.bypass = heavy > 0 && pred_mass >= min_frac * nS ? 1u : 0u;
        *dec = d;
    }
}

cudaError_t launch_decide(const LearnBufs &b, int use_model, double nS, double m, double tau_min, double min_frac,
                          cudaStream_t st) {
    const double lscale = log2(nS / m);
    k_model_eval<<<(EVAL_RANKS + CC_BINS + EVAL_THREADS - 1) / EVAL_THREADS, EVAL_THREADS, 0, st>>>(
        b.params, b.xs, b.ys, lscale, b.lpred, b.dec);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t smem = (size_t)CC_BINS * 16;
    e = smem_limit((const void *)k_decide, smem);
    if (e != cudaSuccess) return e;
    k_decide<<<1, DECIDE_THREADS, smem, st>>>(use_model, b.bin_keys, b.bin_rows, b.lpred, nS / m, nS, tau_min,
                                              min_frac, b.dec);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// heavy table: two tables of HEAVY_BKT buckets of 2 key slots; key EMPTY_KEY
// marks a free slot (so EMPTY_KEY itself is never heavy).  Key k lives in
// bucket heavy_b1(k) of the first table (slots 0 .. HEAVY_CAP / 2) or in
// bucket heavy_b2(k) of the second; slot s indexes cnt (R rows with the key),
// scnt (S rows, counting joins) and start (first of the key's R rows in the
// heavy R payload list, materialisation).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t heavy_b1(uint32_t k) { return (k * 0x9E3779B1u) >> (32 - HEAVY_BKT_LOG2); }
__device__ __forceinline__ uint32_t heavy_b2(uint32_t k) {
    return HEAVY_BKT + ((k * 0x85EBCA6Bu) >> (32 - HEAVY_BKT_LOG2));
}

// Slot of key k, or -1: both buckets are read and compared without branches
// (a key sits in at most one slot).
__device__ __forceinline__ int heavy_lookup(const uint32_t *keys, uint32_t k) {
    const uint32_t b1 = heavy_b1(k), b2 = heavy_b2(k);
    const uint2 x = reinterpret_cast<const uint2 *>(keys)[b1];
    const uint2 y = reinterpret_cast<const uint2 *>(keys)[b2];
    int s = -1;
    s = y.y == k ? (int)(2 * b2 + 1) : s;
    s = y.x == k ? (int)(2 * b2) : s;
    s = x.y == k ? (int)(2 * b1 + 1) : s;
    s = x.x == k ? (int)(2 * b1) : s;
    return k == EMPTY_KEY ? -1 : s;
}

// Inserts k (a key not in the table) by cuckoo displacement: a free slot of
// the key's bucket in the current table, else the key takes a slot whose
// key moves on to its bucket in the other table.  Many threads insert at
// once (atomics only).  Returns false when the walk gave up; the key it
// then holds (k or a displaced one) is left out of the table, which only
// makes that key light.
__device__ bool heavy_insert(uint32_t *keys, uint32_t k) {
    uint32_t cur = k;
    int t = 0;
    for (int it = 0; it < 128; it++) {
        const uint32_t b = t ? heavy_b2(cur) : heavy_b1(cur);
        uint32_t *s = keys + 2 * b;
        if (atomicCAS(&s[0], EMPTY_KEY, cur) == EMPTY_KEY) return true;
        if (atomicCAS(&s[1], EMPTY_KEY, cur) == EMPTY_KEY) return true;
        const uint32_t old = atomicExch(&s[(it >> 1) & 1], cur);
        if (old == EMPTY_KEY) return true;
        cur = old;  // it sat in bucket b of table t: its other bucket is in table t ^ 1
        t ^= 1;
    }
    return false;
}

// Inserts the candidates whose sample count reaches the decision's
// count_min (at most HEAVY_MAX of them; the decision keeps their number at
// or below k* <= HEAVY_MAX); `inserted` ends as the number of keys placed.
__global__ void k_heavy_build(const HeavyCand *__restrict__ cand, unsigned cand_cap, const LrnDecision *dec,
                              uint32_t *keys, unsigned *inserted) {
    const unsigned n = min(dec->ncand, cand_cap);
    const unsigned cmin = dec->count_min;
    if (!dec->bypass) return;
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const HeavyCand c = cand[i];
        if (c.count < cmin || c.key == EMPTY_KEY) continue;
        if (atomicAdd(inserted, 1u) >= (unsigned)HEAVY_MAX) {
            atomicSub(inserted, 1u);
            continue;
        }
        if (!heavy_insert(keys, c.key)) atomicSub(inserted, 1u);
    }
}

cudaError_t launch_heavy_build(const LearnBufs &b, uint32_t *keys, unsigned *inserted, cudaStream_t st) {
    k_heavy_build<<<148 * 2, 256, 0, st>>>(b.cand, b.cand_cap, b.dec, keys, inserted);
    count_launch();
    return cudaGetLastError();
}

// R rows of heavy keys: per-slot counts (pass 0) and payload lists (pass 1,
// materialisation only; start[] holds the exclusive prefix of the counts and
// cur[] the fill cursors).
template <int PASS>
__global__ void __launch_bounds__(512) k_heavy_r(const Row *__restrict__ R, uint64_t n, const uint32_t *__restrict__ gkeys,
                                                 unsigned *gcnt, const unsigned *__restrict__ start, unsigned *cur,
                                                 uint32_t *rpay) {
    extern __shared__ __align__(16) unsigned char smem_hr[];
    uint32_t *keys = reinterpret_cast<uint32_t *>(smem_hr);
    unsigned *cnt = keys + HEAVY_CAP;
    for (int i = threadIdx.x; i < HEAVY_CAP; i += 512) {
        keys[i] = gkeys[i];
        cnt[i] = 0;
    }
    __syncthreads();
    // four rows in flight per thread
    const uint64_t stride = (uint64_t)gridDim.x * 512;
    for (uint64_t i0 = (uint64_t)blockIdx.x * 512 + threadIdx.x; i0 < n; i0 += 4 * stride) {
        Row x[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t i = i0 + u * stride;
            x[u] = Row{EMPTY_KEY, 0};
            if (i < n) {
                const uint2 v = ldg_stream(reinterpret_cast<const uint2 *>(R) + i);
                x[u] = Row{v.x, v.y};
            }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int s = heavy_lookup(keys, x[u].key);  // the padding key EMPTY_KEY is never heavy
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
cudaError_t launch_heavy_r(const Row *R, uint64_t n, const uint32_t *keys, unsigned *cnt, unsigned *start,
                           unsigned *cur, uint32_t *rpay, int stage, int nsm, cudaStream_t st) {
    if (!n) return cudaSuccess;
    const unsigned g = (unsigned)umin64((n + 511) / 512, (uint64_t)nsm * 4);
    const size_t smem = (size_t)HEAVY_CAP * 8;
    cudaError_t e = smem_limit((const void *)k_heavy_r<0>, smem);
    if (e == cudaSuccess) e = smem_limit((const void *)k_heavy_r<1>, smem);
    if (e != cudaSuccess) return e;
    if (stage == 0) {
        k_heavy_r<0><<<g, 512, smem, st>>>(R, n, keys, cnt, nullptr, nullptr, nullptr);
        count_launch();
    } else {
        k_heavy_prefix<<<1, 1024, 0, st>>>(cnt, start, cur);
        k_heavy_r<1><<<g, 512, smem, st>>>(R, n, keys, cnt, start, cur, rpay);
        count_launch(2);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// S histogram with the heavy bypass: per chunk (as k_hist_chunks), every row
// whose key is not heavy is counted in its radix bin and appended to the
// chunk's region of the compacted S (warp-aggregated, coalesced).  Heavy rows
// are joined without partitioning: counting, the kernel counts S rows per
// heavy key (the matches are sum over keys of S rows x R rows, k_heavy_sum);
// materialising, it appends them to the same region from the chunk's end
// down and totals the output rows they make (R rows of their keys), and
// k_heavy_emit writes the pairs while S's kept rows are partitioned.
// ---------------------------------------------------------------------------
// One row outside the vector body (the chunk's first row when it starts 8
// bytes past a 16-byte boundary, or its last row): thread 0 only.
template <bool MAT>
__device__ void bypass_edge_row(const BypassArgs &a, const uint32_t *hkeys, unsigned *hcnt, uint32_t *hist,
                                unsigned *s_keep, unsigned *s_heavy, uint2 *dst, uint2 *dst_end, Row x,
                                unsigned long long &pairs, unsigned &heavy_rows) {
    const int s = heavy_lookup(hkeys, x.key);
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
    pairs += hcnt[s];
    dst_end[-1 - (int64_t)atomicAdd(s_heavy, 1u)] = make_uint2(x.key, x.payload);
}

// The next round's rows are loaded before the current round is processed
// (one round of loads always in flight per thread).
constexpr int BYP_THREADS = 1024;
constexpr int BYP_U = 4;  // 16-byte row pairs per thread per round

// Appends the rows of mask `sel` (bit j: row slot j of this lane) to a
// warp-aggregated region: one ballot per row slot, one shared atomic per
// warp on `ctr`; slot j's rows go to put(j, index).
template <class Put>
__device__ __forceinline__ void warp_append(unsigned sel, unsigned *ctr, Put put) {
    const int lane = threadIdx.x & 31;
    unsigned m[2 * BYP_U], wtot = 0;
#pragma unroll
    for (int j = 0; j < 2 * BYP_U; j++) {
        m[j] = __ballot_sync(0xffffffffu, sel >> j & 1);
        wtot += __popc(m[j]);
    }
    unsigned wb = 0;
    if (lane == 0 && wtot) wb = atomicAdd(ctr, wtot);
    wb = __shfl_sync(0xffffffffu, wb, 0);
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < 2 * BYP_U; j++) {
        if (sel >> j & 1) put(j, wb + __popc(m[j] & lt));
        wb += __popc(m[j]);
    }
}

template <bool MAT>
__global__ void __launch_bounds__(BYP_THREADS, 1) k_hist_bypass(BypassArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *hkeys = reinterpret_cast<uint32_t *>(smem);  // 8-byte aligned buckets
    unsigned *hcnt = hkeys + HEAVY_CAP;
    uint32_t *hist = hcnt + HEAVY_CAP;
    __shared__ unsigned s_keep, s_heavy;
    __shared__ unsigned long long s_pairs;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < a.nbins; i += BYP_THREADS) hist[i] = 0;
    for (int i = tid; i < HEAVY_CAP; i += BYP_THREADS) {
        hkeys[i] = a.hkeys[i];
        hcnt[i] = MAT ? a.hcnt[i] : 0u;
    }
    if (tid == 0) {
        s_keep = 0;
        s_heavy = 0;
        s_pairs = 0;
    }
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * a.chunk;
    const uint64_t hi = umin64(a.n, lo + a.chunk);
    const uint32_t len = hi > lo ? (uint32_t)(hi - lo) : 0u;  // a chunk holds < 2^32 rows
    const Row *src = a.in + lo;
    uint2 *dst = reinterpret_cast<uint2 *>(a.out + lo);
    uint2 *dst_end = reinterpret_cast<uint2 *>(a.out + (lo + len));  // heavy rows, materialising
    const uint32_t head = (len && (reinterpret_cast<uintptr_t>(src) & 15)) ? 1u : 0u;
    const uint32_t npairs = (len - head) / 2;
    const bool tail = ((len - head) & 1) != 0;
    const uint4 *v = reinterpret_cast<const uint4 *>(src + head);
    unsigned long long pairs = 0;  // materialising: output rows of this thread's heavy rows
    unsigned heavy_rows = 0;
    constexpr uint32_t ROUND = BYP_U * BYP_THREADS;
    uint4 nx[BYP_U];
    auto load_round = [&](uint32_t base) {
#pragma unroll
        for (int u = 0; u < BYP_U; u++) {
            const uint32_t p = base + u * BYP_THREADS + tid;
            nx[u] = p < npairs ? ldg_stream(v + p) : make_uint4(EMPTY_KEY, 0, EMPTY_KEY, 0);
        }
    };
    load_round(0);
    // rounds of BYP_U row pairs per thread: pair p = base + u * BYP_THREADS + tid
    for (uint32_t base = 0; base < npairs; base += ROUND) {
        uint32_t k[2 * BYP_U], pv[2 * BYP_U];
        unsigned valid = 0;
#pragma unroll
        for (int u = 0; u < BYP_U; u++) {
            k[2 * u] = nx[u].x;
            pv[2 * u] = nx[u].y;
            k[2 * u + 1] = nx[u].z;
            pv[2 * u + 1] = nx[u].w;
            if (base + u * BYP_THREADS + tid < npairs) valid |= 3u << (2 * u);
        }
        load_round(base + ROUND);  // the next round's loads go out before this round's work
        int slot[2 * BYP_U];
        unsigned hm = 0;
#pragma unroll
        for (int j = 0; j < 2 * BYP_U; j++) {
            slot[j] = heavy_lookup(hkeys, k[j]);
            hm |= (slot[j] >= 0 && (valid >> j & 1)) ? 1u << j : 0u;
        }
        const unsigned km = valid & ~hm;  // rows that go on to the partitions
        heavy_rows += __popc(hm);
        if (!MAT) {  // S rows per heavy slot; a warp's rows of one hot key add once
            const bool dup = warp_has_dups((uint32_t)slot[0], hm & 1u);
#pragma unroll
            for (int j = 0; j < 2 * BYP_U; j++) hist_add_warp(hcnt, (uint32_t)slot[j], hm >> j & 1, dup);
        } else {  // heavy rows from the chunk's end down, and the output rows they make
#pragma unroll
            for (int j = 0; j < 2 * BYP_U; j++) {
                const unsigned c = hcnt[slot[j] >= 0 ? slot[j] : 0];
                pairs += (hm >> j & 1) ? c : 0u;
            }
            warp_append(hm, &s_heavy,
                        [&](int j, unsigned i) { dst_end[-1 - (int64_t)i] = make_uint2(k[j], pv[j]); });
        }
        // kept rows: counted in their radix bin and appended (coalesced)
        warp_append(km, &s_keep, [&](int j, unsigned i) {
            atomicAdd(&hist[radix_f(a.rf, k[j])], 1u);
            dst[i] = make_uint2(k[j], pv[j]);
        });
    }
    __syncthreads();  // every vector row is placed: the edge rows take the next slots
    if (tid == 0) {
        if (head)
            bypass_edge_row<MAT>(a, hkeys, hcnt, hist, &s_keep, &s_heavy, dst, dst_end, src[0], pairs, heavy_rows);
        if (tail)
            bypass_edge_row<MAT>(a, hkeys, hcnt, hist, &s_keep, &s_heavy, dst, dst_end, src[len - 1], pairs,
                                 heavy_rows);
    }
    const unsigned long long wp = warp_sum_u64(pairs), wh = warp_sum_u64((unsigned long long)heavy_rows);
    if (MAT && lane == 0 && wp) atomicAdd(&s_pairs, wp);
    __syncthreads();
    uint32_t *hdst = a.hist + (uint64_t)blockIdx.x * a.nbins;
    for (int i = tid; i < a.nbins; i += BYP_THREADS) hdst[i] = hist[i];
    if (!MAT)
        for (int i = tid; i < HEAVY_CAP; i += BYP_THREADS)
            if (hcnt[i]) atomicAdd(&a.scnt[i], hcnt[i]);
    if (tid == 0) {
        a.kept[blockIdx.x] = s_keep;
        if (MAT) {
            a.hkept[blockIdx.x] = s_heavy;
            a.hpairs[blockIdx.x] = s_pairs;
            if (s_pairs) atomicAdd(a.matches, s_pairs);
        }
    }
    if (lane == 0 && wh) atomicAdd(a.heavy_rows, wh);
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

// First output row of each chunk's heavy pairs (one CTA): exclusive prefix
// of the per-chunk totals, offset by one reservation of their sum.
__global__ void __launch_bounds__(1024) k_heavy_plan(const unsigned long long *__restrict__ hpairs, int G,
                                                    unsigned long long *hbase, unsigned long long *rows_ctr) {
    __shared__ uint64_t scratch[1024 / 32 + 1];
    __shared__ unsigned long long s_base;
    const int per = (G + 1023) / 1024;
    const int c0 = min(G, (int)threadIdx.x * per), c1 = min(G, c0 + per);
    uint64_t sum = 0;
    for (int c = c0; c < c1; c++) sum += hpairs[c];
    uint64_t tot;
    uint64_t run = block_excl_scan<1024>(sum, &tot, scratch);
    if (threadIdx.x == 0) s_base = tot ? atomicAdd(rows_ctr, (unsigned long long)tot) : 0ull;
    __syncthreads();
    for (int c = c0; c < c1; c++) {
        hbase[c] = s_base + run;
        run += hpairs[c];
    }
}

cudaError_t launch_heavy_plan(const unsigned long long *hpairs, int G, unsigned long long *hbase,
                              unsigned long long *rows_ctr, cudaStream_t st) {
    k_heavy_plan<<<1, 1024, 0, st>>>(hpairs, G, hbase, rows_ctr);
    count_launch();
    return cudaGetLastError();
}

// The heavy pairs of a materialising bypass: CTA c reads chunk c's heavy S
// rows (compacted from the chunk's end down), finds each key's slot in the
// heavy table and writes one output row per R row of the key, at
// hbase[c] + a place reserved by its warp (a shared atomic per warp and
// round, no block barriers).  Chunk c's rows fill [hbase[c], hbase[c] +
// hpairs[c]) exactly.  A key's first R payload comes from shared memory
// when it has one R row (the common case: R a key permutation), else its
// list in rpay.
constexpr int EMIT_THREADS = 512;
constexpr int EMIT_U = 4;  // heavy rows per thread per round

__global__ void __launch_bounds__(EMIT_THREADS, 2) k_heavy_emit(HeavyEmitArgs a) {
    extern __shared__ __align__(16) unsigned char smem_he[];
    uint32_t *hkeys = reinterpret_cast<uint32_t *>(smem_he);
    unsigned *hcnt = hkeys + HEAVY_CAP;
    unsigned *hstart = hcnt + HEAVY_CAP;
    __shared__ unsigned long long s_next;
    const int tid = threadIdx.x, lane = tid & 31;
    for (int i = tid; i < HEAVY_CAP; i += EMIT_THREADS) {
        hkeys[i] = a.hkeys[i];
        hcnt[i] = a.hcnt[i];
        hstart[i] = a.hstart[i];
    }
    const int c = blockIdx.x;
    if (tid == 0) s_next = a.hbase[c];
    __syncthreads();
    const uint64_t lo = (uint64_t)c * a.chunk;
    const uint64_t end = umin64(a.n, lo + a.chunk);
    const uint32_t nh = a.hkept[c];
    const uint2 *src = reinterpret_cast<const uint2 *>(a.hs) + (end - nh);
    constexpr uint32_t ROUND = EMIT_U * EMIT_THREADS;
    for (uint32_t base = 0; base < nh; base += ROUND) {
        uint2 x[EMIT_U];
        uint32_t cnt[EMIT_U], st[EMIT_U];
#pragma unroll
        for (int u = 0; u < EMIT_U; u++) {
            const uint32_t i = base + u * EMIT_THREADS + tid;
            x[u] = i < nh ? ldg_stream(src + i) : make_uint2(EMPTY_KEY, 0);
        }
#pragma unroll
        for (int u = 0; u < EMIT_U; u++) {
            const int s = heavy_lookup(hkeys, x[u].x);  // every compacted row is heavy; padding is not
            cnt[u] = s >= 0 ? hcnt[s] : 0u;
            st[u] = s >= 0 ? hstart[s] : 0u;
        }
        // places in (row slot, lane) order, so consecutive lanes store
        // consecutive rows; one reservation per warp and round
        uint32_t pre[EMIT_U], wsum = 0;
#pragma unroll
        for (int u = 0; u < EMIT_U; u++) {
            uint32_t inc = cnt[u];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            pre[u] = wsum + inc - cnt[u];
            wsum += __shfl_sync(0xffffffffu, inc, 31);
        }
        unsigned long long wb = 0;
        if (lane == 0 && wsum) wb = atomicAdd(&s_next, (unsigned long long)wsum);
        wb = __shfl_sync(0xffffffffu, wb, 0);
#pragma unroll
        for (int u = 0; u < EMIT_U; u++) {
            uint64_t op = wb + pre[u];
            for (uint32_t q = 0; q < cnt[u]; q++, op++)
                if (op < a.cap) a.rows[op] = tbg_row_out{x[u].x, a.rpay[st[u] + q], x[u].y};
        }
    }
}

cudaError_t launch_heavy_emit(const HeavyEmitArgs &a, int nsm, cudaStream_t st) {
    (void)nsm;
    if (!a.G) return cudaSuccess;
    const size_t smem = (size_t)HEAVY_CAP * 4 * 3;
    cudaError_t e = smem_limit((const void *)k_heavy_emit, smem);
    if (e != cudaSuccess) return e;
    k_heavy_emit<<<a.G, EMIT_THREADS, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

size_t bypass_smem(int nbins, bool mat) {
    (void)mat;  // heavy keys + counts + 2^15 bins: 196,608 B at most
    return (size_t)HEAVY_CAP * 4 * 2 + (size_t)nbins * 4;
}

cudaError_t launch_hist_bypass(const BypassArgs &a, bool mat, cudaStream_t st) {
    const size_t smem = bypass_smem(a.nbins, mat);
    auto kern = mat ? k_hist_bypass<true> : k_hist_bypass<false>;
    cudaError_t e = smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<a.G, BYP_THREADS, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg

