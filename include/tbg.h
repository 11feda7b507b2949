/*
 * tbg.h -- C ABI of tee-bench-b200, a B200 (sm_100a) implementation of the
 * TEEbench equi-join hot path: the radix hash join RHO, its histogram sibling
 * RHT, the sort-merge joins RSM and PSM, and LRN, a learned skew-aware
 * join whose model picks heavy keys that bypass radix partitioning.
 *
 * Two layers:
 *
 * 1. Drop-in entry points with the reference's exact signature
 *        result_t *RHO(relation_t *R, relation_t *S, int nthreads);
 *    and the reference's struct layouts, so a program that linked the
 *    reference's joins (native.cpp:34-46 registry, :125 call) links this
 *    library instead.  Inputs are host buffers; the call copies them to the
 *    GPU, joins there, and returns a malloc'd result_t.  Inputs are NOT
 *    clobbered (the reference writes partitions back into them).
 *
 * 2. A device-resident API (tbg_join_device) on caller-owned device buffers
 *    and a caller stream, used for measurement and by callers that keep data
 *    on the GPU.  All entry points return status codes instead of exiting.
 *
 * Every pointer is plain; `stream` is a cudaStream_t passed as void*.
 */
#ifndef TBG_H
#define TBG_H

#include <stdint.h>
#include <stddef.h>

/* ---- reference types ------------------------------------------------------
 * Identical layouts to Include/data-types.h:32-93 of the reference.  When the
 * reference header was included first (its guard DATA_TYPES_H is defined) its
 * own definitions are used. */
#ifndef DATA_TYPES_H
typedef uint32_t type_key;
typedef uint32_t type_value;
typedef struct row_t tuple_t;
typedef struct table_t relation_t;
typedef struct result_t result_t;
typedef struct threadresult_t threadresult_t;
typedef struct output_list_t output_list_t;

struct row_t {               /* Include/data-types.h:44-47 */
    type_key key;
    type_value payload;
};
struct table_t {             /* Include/data-types.h:49-54 */
    struct row_t *tuples;
    uint64_t num_tuples;
    int ratio_holes;
    int sorted;
};
struct output_list_t {       /* Include/data-types.h:56-61 */
    type_key key;
    type_value Rpayload;
    type_value Spayload;
    struct output_list_t *next;
};
struct threadresult_t {      /* Include/data-types.h:74-78 */
    int64_t nresults;
    output_list_t *results;
    uint32_t threadid;
};
struct result_t {            /* Include/data-types.h:81-85 */
    int64_t totalresults;
    struct threadresult_t *resultlist;
    int nthreads;
};
typedef struct algorithm_t { /* Include/data-types.h:68-71 */
    char name[128];
    result_t *(*join)(struct table_t *, struct table_t *, int);
} algorithm_t;
#endif

#if defined(__GNUC__)
#define TBG_API __attribute__((visibility("default")))
#else
#define TBG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
enum {
    TBG_OK = 0,
    TBG_ERR_ARG = 1,          /* null pointer, bad size or unknown option      */
    TBG_ERR_CUDA = 2,         /* a CUDA runtime call failed                    */
    TBG_ERR_OOM = 3,          /* device or pinned host allocation failed       */
    TBG_ERR_TIMEOUT = 4,      /* a bounded device-side wait gave up            */
    TBG_ERR_CAPACITY = 5,     /* output rows exceed the caller's capacity      */
    TBG_ERR_UNKNOWN_ALGO = 6, /* no join registered under that name            */
    TBG_ERR_NO_DEVICE = 7     /* no CUDA device visible                        */
};

/* ---- drop-in joins (layer 1) ---------------------------------------------
 * Same signature and meaning as the reference entry points:
 *   RHO  Joins/radix_join.h:20-21      (radix join, bucket-chaining table)
 *   RHT  Joins/radix_join.h:23-24      (radix join, histogram table)
 *   RSM  Joins/radix_sortmerge_join.h:4 (radix partitions, sort-merge join)
 *   PSM  Joins/psm/parallel_sortmerge_join.h:61 (global sort, merge join)
 *   LRN  new: radix join whose learned model picks heavy keys that skip
 *        partitioning (joined during S's histogram read), same result
 * totalresults is the exact equi-join cardinality for every algorithm.  The
 * *_mat variants also fill resultlist[t].results with nresults rows each (the
 * JOIN_MATERIALIZE layout of Joins/radix_join.c:1195-1199), NULL-terminated.
 * nthreads sizes resultlist (values < 1 count as 1); the GPU does the work.
 * On error the call logs to stderr and exits with EXIT_FAILURE, as the
 * reference does (Include/util.c:11-18), unless tbg_set_error_mode() chose
 * TBG_ERRMODE_RETURN, in which case it returns NULL. */
TBG_API result_t *RHO(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *RHT(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *RSM(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *PSM(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *LRN(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *RHO_mat(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *RHT_mat(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *RSM_mat(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *PSM_mat(struct table_t *relR, struct table_t *relS, int nthreads);
TBG_API result_t *LRN_mat(struct table_t *relR, struct table_t *relS, int nthreads);

#if defined(JOIN_MATERIALIZE) && !defined(TBG_NO_MATERIALIZE_MAP)
/* A program built with -DJOIN_MATERIALIZE expects rows from RHO & co. */
#define RHO RHO_mat
#define RHT RHT_mat
#define RSM RSM_mat
#define PSM PSM_mat
#define LRN LRN_mat
#endif

/* Name registry replacing native.cpp:34-46 / secure_joins.cpp:103-123. */
TBG_API extern const algorithm_t tbg_algorithms[];
TBG_API extern const int tbg_num_algorithms;
TBG_API const algorithm_t *tbg_find(const char *name); /* NULL when unknown */

/* S slices that RHO and RHT (and their _mat forms) copy to the GPU and join
 * one after another, each slice's join overlapping the next slice's copy;
 * the result is the whole join's.  0 (the default): one slice per 2^26 S
 * rows, at most 16; 1: copy everything, then join.  Returns the previous
 * setting.  No counterpart in the reference (its relations are in host
 * memory already). */
TBG_API int tbg_set_dropin_slices(int k);

/* Host<->device bytes the last drop-in call moved (inputs in, result out). */
TBG_API void tbg_last_transfer_bytes(uint64_t *h2d, uint64_t *d2h);

/* Frees a result_t returned by any drop-in join (lists included). */
TBG_API void tbg_result_free(result_t *res);

enum { TBG_ERRMODE_EXIT = 0, TBG_ERRMODE_RETURN = 1 };
TBG_API int tbg_set_error_mode(int mode);      /* returns the previous mode */
TBG_API int tbg_last_error(void);              /* status of the last failing call  */
TBG_API const char *tbg_last_error_string(void);

/* ---- device-resident API (layer 2) ---------------------------------------- */
enum { TBG_RHO = 0, TBG_RHT = 1, TBG_RSM = 2, TBG_PSM = 3, TBG_LRN = 4 };

/* LRN model choices: how the heavy (frequent) S keys that bypass
 * partitioning are picked from the 1% sample's candidate keys */
enum {
    TBG_MODEL_MLP = 0,        /* FP32 MLP 1->32->32->1, trained on the GPU on
                                 the sample's frequency-by-rank curve; predicts
                                 the S rows of the top ranks                 */
    TBG_MODEL_SAMPLE = 1,     /* ablation: raw sample counts, no model         */
    TBG_MODEL_UNTRAINED = 2,  /* ablation: the MLP at its initialisation       */
    TBG_MODEL_UNIFORM = 3     /* ablation: no heavy keys (plain radix, RHO)    */
};

typedef struct tbg_config {
    int algo;               /* TBG_RHO ...                                     */
    int radix_bits;         /* total partition bits (<= 15), 0 = chosen from |R| */
    int passes;             /* partitioning passes (1 or 2), 0 = automatic     */
    int materialize;        /* 0: count only; 1: write tbg_row_out rows        */
    int skew_split;         /* split oversized partition pairs across CTAs     */
    int model;              /* LRN: TBG_MODEL_*                                */
    int train_steps;        /* LRN: training steps (<= 500)                    */
    int heavy_bypass;       /* LRN: join flagged heavy keys during partitioning */
    double sample_rate;     /* LRN: sampled fraction of S (0: 0.01)            */
    double imbalance_limit; /* LRN: predicted max/mean above which radix is used */
    uint64_t seed;          /* LRN sampling / init seed                        */
    int timing;             /* record per-phase device times into tbg_stats    */
} tbg_config;

typedef struct tbg_row_out { /* one materialised row, 12 bytes */
    uint32_t key;
    uint32_t Rpayload;
    uint32_t Spayload;
} tbg_row_out;

typedef struct tbg_stats {
    uint64_t matches;
    uint64_t partitions;        /* final partitions                          */
    uint64_t work_items;        /* join work items after skew splitting      */
    uint64_t max_part_R, max_part_S;
    double mean_part_R, mean_part_S;
    double imbalance;           /* max / mean of (|R_p| + |S_p|)             */
    double predicted_imbalance; /* LRN: the model's own estimate            */
    int radix_bits, passes;
    int used_fallback;          /* LRN fell back to radix partitioning       */
    uint64_t heavy_keys;        /* LRN: keys joined by the heavy path        */
    uint64_t heavy_rows_S;      /* LRN: S rows that skipped partitioning     */
    int train_steps;
    float train_loss;
    uint32_t kernel_launches;   /* kernels this call launched                */
    float ms_hist, ms_pass1, ms_pass2, ms_join, ms_learn, ms_total;
    double heavy_rows_predicted; /* LRN: S rows the model predicts for the top ranks it flags */
    double heavy_rows_sampled;   /* LRN: the sample's own estimate for the heavy keys taken   */
} tbg_stats;

TBG_API void tbg_config_init(tbg_config *cfg); /* defaults: RHO, automatic, count only */

/* Joins device-resident R and S (rows of struct row_t, any 8-byte alignment)
 * on `stream`.  Waits for the result and returns it in *matches.  With
 * cfg->materialize, rows go to d_rows[0 .. min(matches, rows_cap)); more
 * matches than rows_cap returns TBG_ERR_CAPACITY with *matches exact.
 * Inputs are read only.  Scratch is owned by the library, cached per device
 * and stream, and grown on demand. */
TBG_API int tbg_join_device(const tbg_config *cfg, const struct row_t *dR, uint64_t nR,
                    const struct row_t *dS, uint64_t nS, tbg_row_out *d_rows,
                    uint64_t rows_cap, uint64_t *matches, tbg_stats *stats,
                    void *stream);

/* Same work, fully asynchronous: the match count lands in *d_matches (device
 * memory) and nothing waits.  Errors detected on the device are reported by
 * the next tbg_sync_status() on the same stream. */
TBG_API int tbg_join_device_async(const tbg_config *cfg, const struct row_t *dR, uint64_t nR,
                          const struct row_t *dS, uint64_t nS, tbg_row_out *d_rows,
                          uint64_t rows_cap, uint64_t *d_matches, void *stream);
TBG_API int tbg_sync_status(void *stream);

/* Number of kernels this library launched since load (all entry points). */
TBG_API uint64_t tbg_kernel_launches(void);

/* ---- learned partitioner model (LRN) --------------------------------------
 * The FP32 MLP 1->32->32->1 (tanh) that LRN trains per join, exposed for
 * inspection and tests.  params: W1[32], b1[32], W2[32][32], b2[32], W3[32],
 * b3 (host arrays of tbg_mlp_param_count() floats).  LRN fits the frequency
 * curve of S's keys: x = tbg_mlp_feature(r) for sample rank r (1 = the key
 * the sample saw most often), y = log2(that key's sample count), normalised
 * to zero mean and unit spread over the training points. */
TBG_API int tbg_mlp_param_count(void);
TBG_API float tbg_mlp_feature(uint32_t rank);
/* seeded initialisation, as LRN uses before training */
TBG_API int tbg_mlp_init(float *params, uint64_t seed);
/* mean squared error over n points and its gradient (the GPU backward pass) */
TBG_API int tbg_mlp_grad(const float *params, const float *x, const float *y, uint64_t n,
                         float *grad, float *loss);
/* `steps` Adam steps on the GPU trainer (batches drawn from the n points) */
TBG_API int tbg_mlp_train(float *params, const float *x, const float *y, uint64_t n, int steps,
                          float lr, uint64_t seed);

/* ---- joins split over several GPUs: the exchange step ----------------------
 * The reference splits one join over threads by contiguous chunks of R and S
 * (Joins/radix_join.c:1285-1306).  Across GPUs the split is by key: every
 * rank splits its rows of R and of S by destination shard, an all-to-all
 * (NCCL, in the caller) moves each piece to its shard's rank, every rank joins
 * what it received with tbg_join_device, and the counts are summed (equal keys
 * always meet on one rank).
 *
 * tbg_shard_split writes the n device rows of d_in to d_out grouped by shard:
 * shard d's rows at d_out[offsets[d] .. offsets[d + 1]) (offsets: a host array
 * of nshards + 1 entries, filled; waits for the stream).  1 <= nshards <= 256.
 * tbg_shard_of(key, nshards) is the shard of a key: a multiplicative hash of
 * the key, so shards get even shares of skewed keys too.                    */
TBG_API int tbg_shard_split(const struct row_t *d_in, uint64_t n, int nshards, struct row_t *d_out,
                            uint64_t *offsets, void *stream);
TBG_API uint32_t tbg_shard_of(uint32_t key, int nshards);

/* ---- chained joins on device-resident output --------------------------------
 * to_relation (Enclave/TrustedJoins/secure_joins.cpp:277-301): materialised
 * rows -> relation of (key, payload = R payload) tuples, on the device.     */
TBG_API int tbg_rows_to_relation(const tbg_row_out *d_rows, uint64_t n, struct row_t *d_out,
                                 void *stream);
/* The reference's three-way chain (ecall_three_way_join_sealed_tables,
 * secure_joins.cpp:348-399) without host round trips: out1 = R x S
 * materialised into library memory, rel1 = to_relation(out1), then T x rel1
 * (T on the build side) with cfg's algorithm; its rows go to d_rows2 when it
 * is not NULL (else count only).  *matches1, *matches2: the two counts.    */
TBG_API int tbg_join_three_way(const tbg_config *cfg, const struct row_t *dR, uint64_t nR,
                               const struct row_t *dS, uint64_t nS, const struct row_t *dT,
                               uint64_t nT, tbg_row_out *d_rows2, uint64_t rows2_cap,
                               uint64_t *matches1, uint64_t *matches2, void *stream);

/* ---- batched joins (many independent joins, one persistent launch) -------- *
 * No counterpart in the reference, whose driver runs one join per call
 * (native.cpp:125); each join's count equals RHO's on that join.     */
typedef struct tbg_batch_join {
    const struct row_t *dR; /* device memory, 8-byte aligned                   */
    uint64_t nR;            /* < 2^32                                          */
    const struct row_t *dS;
    uint64_t nS;
} tbg_batch_join;

typedef struct tbg_batch tbg_batch; /* opaque plan: tuned, graph-captured */

/* Plans njoins joins.  cfg (NULL = defaults): algo TBG_RHO or TBG_RHT (RHT
 * fixes the histogram table layout), count only; radix_bits 0 autotunes the
 * partitioning (direct or 1..8 radix bits), table layout, S rows per work
 * item and chunk size per size class by timing the batch's own joins;
 * radix_bits > 0 partitions every join with that many bits (one pass, <= 8);
 * radix_bits < 0 uses the built-in heuristic without timing.  The whole
 * batch is captured as one CUDA graph.  Waits for `stream` (the inputs may be
 * written there), then works on a private stream; the relations must stay
 * allocated, at the same addresses, until tbg_batch_destroy (their contents
 * may change between runs).                                                */
TBG_API int tbg_batch_create(const tbg_batch_join *joins, int njoins, const tbg_config *cfg,
                             void *stream, tbg_batch **out);
/* Replays the graph on `stream` (asynchronous); d_counts[i] (device, may be
 * NULL) receives join i's match count. */
TBG_API int tbg_batch_run(tbg_batch *b, uint64_t *d_counts, void *stream);
/* Waits for the last run; returns its device status (TBG_ERR_TIMEOUT if a
 * bounded wait inside the kernel gave up). */
TBG_API int tbg_batch_sync(tbg_batch *b);
/* JSON summary of the plan (grid, tickets, per-size-class choices and tuned
 * times) into buf[cap]; returns the full length. */
TBG_API int tbg_batch_describe(const tbg_batch *b, char *buf, size_t cap);
TBG_API void tbg_batch_destroy(tbg_batch *b);

/* ---- join count without device allocation ---------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * or cudaFree: engines whose device memory is owned and budgeted by their own
 * pool allocator, and latency-bound pipelines that cannot take the
 * device-wide synchronisation of cudaFree or an out-of-memory failure in the
 * middle of a query.  Count-only RHO of device relations with
 * |R| + |S| <= TBG_STATIC_MAX_ROWS (larger inputs: TBG_ERR_ARG, nothing
 * launched).  Its scratch is one static device array of about 32.3 MiB
 * compiled into the library, which every GPU that loads the library holds
 * until the process exits.  The first call on a device looks the array up
 * (cudaGetSymbolAddress) and sizes the grid: make that first call before any
 * stream capture.  Asynchronous on `stream`: *d_count (device) receives the
 * count and, if d_status is not NULL, *d_status (device) the kernel's status
 * (0, or TBG_ERR_TIMEOUT).  Every call reuses the same array, clearing what
 * must start at zero; calls that overlap on the GPU race, so serialise them. */
#define TBG_STATIC_MAX_ROWS (1ull << 22)
TBG_API int tbg_join_count_static(const struct row_t *dR, uint64_t nR, const struct row_t *dS,
                                  uint64_t nS, uint64_t *d_count, uint32_t *d_status, void *stream);

/* ---- on-GPU seeded generators (App/Lib/generator.cpp semantics) ----------- */
/* pk: keys a seeded permutation of 1..n, payload = row index.               */
TBG_API int tbg_gen_pk(struct row_t *d, uint64_t n, uint64_t seed, void *stream);
/* fk: n / maxid shuffled copies of 1..maxid, then a shuffled prefix of
 * another copy (every key in 1..maxid; generator.cpp:475-514 semantics).    */
TBG_API int tbg_gen_fk(struct row_t *d, uint64_t n, uint64_t maxid, uint64_t seed, void *stream);
/* zipf: keys drawn with P(rank r) ~ r^-z over 1..alphabet; rank -> key is
 * the identity (scatter = 0, the reference's effective mapping) or a seeded
 * permutation (scatter = 1).  z = 0 draws uniformly.                       */
TBG_API int tbg_gen_zipf(struct row_t *d, uint64_t n, uint64_t alphabet, double z, int scatter,
                 uint64_t seed, void *stream);
/* Sum of tbo-style row hashes of d_rows[0..n) (order independent). */
TBG_API int tbg_rows_checksum(const tbg_row_out *d_rows, uint64_t n, uint64_t *checksum,
                      void *stream);

#ifdef __cplusplus
}
#endif
#endif /* TBG_H */
