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
constexpr int MLP_TRAIN_THREADS = 512;  // trainer threads per CTA (the gradient sums are spread over them)
constexpr int MLP_SLICE = 152;        // parameters updated by each CTA
static_assert(MLP_PARAMS <= MLP_PARAMS_PAD, "parameter stride");
static_assert(MLP_SLICE * MLP_CLUSTER >= MLP_PARAMS, "every parameter belongs to a slice");

// Heavy-key table: two tables of HEAVY_BKT buckets of 2 key slots (one
// 8-byte load each); a key lives in its bucket of the first table or in its
// bucket of the second (two-choice cuckoo hashing), so a lookup is two loads
// and four compares, without branches.  Slot s (0 .. HEAVY_CAP) indexes the
// per-key arrays (R rows, S rows, payload list starts).
constexpr int HEAVY_LOG2 = 13;
constexpr int HEAVY_CAP = 1 << HEAVY_LOG2;
constexpr int HEAVY_BKT_LOG2 = HEAVY_LOG2 - 2;
constexpr int HEAVY_BKT = 1 << HEAVY_BKT_LOG2;  // buckets per table
constexpr int HEAVY_MAX = HEAVY_CAP / 2;        // at most half full
constexpr uint32_t EMPTY_KEY = 0xFFFFFFFFu;

#ifdef __CUDACC__
#define TBG_HD __host__ __device__
#else
#define TBG_HD
#endif
// Model input: a key's frequency rank r in the sample (1 = most frequent),
// log2(r + 1) / 16 - 1, which maps ranks 0 .. 2^32 onto [-1, 1].  The rank
// comes from the sample's counts, never from the key's value, so the model
// sees the same curve whether hot keys are small integers or scattered over
// the key range.
TBG_HD inline float rank_feature(double rank) { return (float)(log2(rank + 1.0) / 16.0 - 1.0); }

// Sample of S: blocks of SAMPLE_BLOCK consecutive rows (coalesced reads).
constexpr int SAMPLE_BLOCK = 64;
// Per-CTA shared-memory aggregation of the sample's keys before the global
// count table: CNT_CHUNK keys per CTA into 2 * CNT_CHUNK slots (64 KB: two
// CTAs per SM).
constexpr int CNT_THREADS = 1024;
constexpr int CNT_CHUNK = 4096;
// Count-of-counts bins: exact below CC_EXACT, then CC_OCT bins per octave.
constexpr int CC_EXACT = 2048;
constexpr int CC_OCT = 16;
constexpr int CC_BINS = CC_EXACT + CC_OCT * 21;
constexpr int CAND_MIN_COUNT = 2;  // sampled keys seen once are never heavy candidates

struct HeavyCand {
    uint32_t key;
    uint32_t count;  // occurrences in the sample
};

// What the learning stage decided (device memory, read back once).
struct LrnDecision {
    unsigned bypass;          // 1: heavy keys skip partitioning
    unsigned count_min;       // heavy keys: sample count >= count_min
    unsigned k_star;          // ranks whose predicted S rows reach the threshold
    unsigned heavy_sample;    // sampled keys at or above count_min
    unsigned npoints;         // training points (non-empty count bins)
    unsigned ncand;           // candidates listed (sample count >= CAND_MIN_COUNT)
    double pred_mass;         // predicted S rows of ranks 1 .. k_star
    double sample_mass;       // the sample's estimate of the heavy keys' S rows
    double next_rows;         // predicted S rows of rank k_star + 1 (largest key left)
    float loss;               // mean squared error of the model on the (normalised) points
    float y_mu, y_sigma;      // the points' targets are (log2(count) - y_mu) / y_sigma
    unsigned pad;
    double loss_sum;          // squared error of the model summed over the points
};

struct BypassArgs {
    const Row *in;        // S
    uint64_t n;
    uint64_t chunk;
    int G;
    int nbins;
    RadixF rf;
    Row *out;             // compacted S: chunk c's kept rows at [c * chunk, c * chunk + kept[c]);
                          // materialising, its heavy rows from the chunk's end down
    uint32_t *hist;       // [G][nbins]
    uint32_t *kept;       // [G]
    uint32_t *hkept;      // materialising: [G] heavy rows of chunk c
    unsigned long long *hpairs;  // materialising: [G] heavy output rows of chunk c
    const uint32_t *hkeys;
    const unsigned *hcnt;       // materialising: R rows per heavy slot
    unsigned *scnt;             // counting: S rows per heavy slot (added to)
    unsigned long long *matches;
    unsigned long long *heavy_rows;
};

// Output of a materialising bypass: heavy S rows (in the compacted S, from
// each chunk's end down) paired with their keys' R rows.
struct HeavyEmitArgs {
    const Row *hs;              // the compacted S buffer
    uint64_t n, chunk;
    int G;
    const uint32_t *hkept;      // [G] heavy rows of chunk c (at [end - hkept[c], end))
    const unsigned long long *hbase;  // [G] first output row of chunk c
    const uint32_t *hkeys;
    const unsigned *hcnt;       // R rows per heavy slot
    const unsigned *hstart;     // first of them in rpay
    const uint32_t *rpay;
    tbg_row_out *rows;
    uint64_t cap;
};

cudaError_t launch_mlp_init(float *params, uint64_t seed, cudaStream_t st);
cudaError_t launch_mlp_grad(const float *params, const float *xs, const float *ys, uint32_t n, float *grad,
                            float *loss_sum, cudaStream_t st);
// cw (may be null): cumulative sampling weights of the points (cw[n - 1] =
// their total); batches are then drawn in proportion to the weights.
cudaError_t launch_mlp_train(const float *xs, const float *ys, const float *cw, const unsigned *n_dev, uint32_t n,
                             float *params, int steps, float lr, uint64_t seed, cudaStream_t st);
// Learning stage of LRN (all on the device, learned.cu).
struct LearnBufs {
    uint32_t *keys;             // sample keys [m]
    unsigned long long *table;  // global count table [slots]: key << 32 | count
    uint32_t tmask;             // slots - 1
    unsigned *bin_keys;         // [CC_BINS]
    unsigned long long *bin_rows;  // [CC_BINS]
    HeavyCand *cand;            // [cand_cap]
    unsigned cand_cap;
    float *xs, *ys;             // training points [CC_BINS]
    float *cw;                  // their cumulative sampling weights [CC_BINS]
    float *lpred;               // log2 predicted S rows of ranks 0 .. HEAVY_MAX + 1 (entry 0 unused)
    float *params;              // MLP parameters
    LrnDecision *dec;
    unsigned *err;
};
cudaError_t launch_sample_blocks(const Row *S, uint64_t nS, uint32_t *keys, uint64_t nblocks, uint64_t stride,
                                 uint64_t seed, cudaStream_t st);
cudaError_t launch_count_keys(const LearnBufs &b, uint64_t m, cudaStream_t st);
cudaError_t launch_count_stats(const LearnBufs &b, cudaStream_t st);
cudaError_t launch_rank_points(const LearnBufs &b, cudaStream_t st);
cudaError_t launch_decide(const LearnBufs &b, int use_model, double nS, double m, double tau_min, double min_frac,
                          cudaStream_t st);
cudaError_t launch_heavy_build(const LearnBufs &b, uint32_t *keys, unsigned *inserted, cudaStream_t st);
cudaError_t launch_heavy_r(const Row *R, uint64_t n, const uint32_t *keys, unsigned *cnt,
                           unsigned *start, unsigned *cur, uint32_t *rpay, int stage, int nsm, cudaStream_t st);
cudaError_t launch_hist_bypass(const BypassArgs &a, bool mat, cudaStream_t st);
cudaError_t launch_heavy_sum(const unsigned *rcnt, const unsigned *scnt, unsigned long long *matches, cudaStream_t st);
// Exclusive prefix of the chunks' heavy output rows plus one reservation of
// their total from rows_ctr: hbase[c] = first output row of chunk c.
cudaError_t launch_heavy_plan(const unsigned long long *hpairs, int G, unsigned long long *hbase,
                              unsigned long long *rows_ctr, cudaStream_t st);
cudaError_t launch_heavy_emit(const HeavyEmitArgs &a, int nsm, cudaStream_t st);
size_t bypass_smem(int nbins, bool mat);

}  // namespace tbg
