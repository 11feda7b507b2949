// Declarations of the learned skew-aware partitioner (learned.cu / learned.cpp).
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

#include "tbg_internal.h"

namespace tbg {

// MLP 1 -> MLP_H -> MLP_H -> 1 (tanh); parameter count and padded stride.
constexpr int MLP_H = 32;
// W1, b1 (H each) + W2 (H x H) + b2, W3 (H each) + b3 = 1153 for H = 32
constexpr int MLP_PARAMS = 2 * MLP_H + MLP_H * MLP_H + 2 * MLP_H + 1;
constexpr int MLP_PARAMS_PAD = 1184;  // stride of parameter-sized arrays (>= MLP_PARAMS)
constexpr int MLP_CLUSTER = 8;        // CTAs of the training cluster
constexpr int MLP_BATCH_CTA = 128;    // samples per CTA per step
constexpr int MLP_SLICE = 152;        // parameters updated by each CTA
static_assert(MLP_PARAMS <= MLP_PARAMS_PAD, "parameter stride");
static_assert(MLP_SLICE * MLP_CLUSTER >= MLP_PARAMS, "every parameter belongs to a slice");

// Heavy-key table (open addressing on the key).
constexpr int HEAVY_LOG2 = 13;
constexpr int HEAVY_CAP = 1 << HEAVY_LOG2;
constexpr int HEAVY_MAX = HEAVY_CAP / 2;  // at most half full
constexpr uint32_t EMPTY_KEY = 0xFFFFFFFFu;
constexpr int FILTER_LOG2 = 16;  // bit filter in front of the heavy table (8 KB)

#ifdef __CUDACC__
#define TBG_HD __host__ __device__
#else
#define TBG_HD
#endif
// Model input feature of a key: log2(key + 1) / 16 - 1 maps 0 .. 2^32 onto [-1, 1].
TBG_HD inline float key_feature(double key) { return (float)(log2(key + 1.0) / 16.0 - 1.0); }

struct HeavyCand {
    uint32_t key;
    float count;  // predicted rows of S with this key
};

struct BypassArgs {
    const Row *in;        // S
    uint64_t n;
    uint64_t chunk;
    int G;
    int nbins;
    RadixF rf;
    Row *out;             // compacted S: chunk c's kept rows at [c * chunk, c * chunk + kept[c])
    uint32_t *hist;       // [G][nbins]
    uint32_t *kept;       // [G]
    const uint32_t *filter;
    const uint32_t *hkeys;
    const unsigned *hcnt;
    const unsigned *hstart;
    const uint32_t *rpay;
    unsigned long long *matches;
    unsigned long long *heavy_rows;
    unsigned long long *rows_ctr;
    tbg_row_out *rows;
    uint64_t cap;
};

cudaError_t launch_mlp_init(float *params, uint64_t seed, cudaStream_t st);
cudaError_t launch_mlp_grad(const float *params, const float *xs, const float *ys, uint32_t n, float *grad,
                            float *loss_sum, cudaStream_t st);
cudaError_t launch_mlp_train(const float *xs, const float *ys, uint32_t n, float *params, int steps, float lr,
                             uint64_t seed, cudaStream_t st);
cudaError_t launch_sample(const Row *in, uint64_t n, Row *out, uint64_t m, uint64_t seed, cudaStream_t st);
cudaError_t launch_candidates(const Row *sorted, uint64_t m, double nS, HeavyCand *cand, unsigned *ncand,
                              unsigned cand_cap, unsigned *scratch_cnt, cudaStream_t st);
cudaError_t launch_freq_points(const HeavyCand *cand, unsigned ncand, float *xs, float *ys, uint32_t T,
                               cudaStream_t st);
cudaError_t launch_heavy_score(HeavyCand *cand, unsigned ncand, const float *params, int use_model, double tau_min,
                               double min_sample, unsigned *bins, unsigned long long *mass, cudaStream_t st);
cudaError_t launch_heavy_build(const HeavyCand *cand, unsigned ncand, float tau, uint32_t *keys, uint32_t *filter,
                               unsigned *inserted, cudaStream_t st);
cudaError_t launch_heavy_r(const Row *R, uint64_t n, const uint32_t *keys, const uint32_t *filter, unsigned *cnt,
                           unsigned *start, unsigned *cur, uint32_t *rpay, int stage, int nsm, cudaStream_t st);
cudaError_t launch_hist_bypass(const BypassArgs &a, bool mat, cudaStream_t st);
size_t bypass_smem(int nbins, bool mat);

}  // namespace tbg
