// Internal declarations shared by the sm_100a kernels and the host runtime of
// tee-bench-b200.  Host code includes this with a plain C++ compiler view
// (no device code is defined here).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/tbg.h"

namespace tbg {

// 8-byte tuple, the layout of struct row_t (uint32 key, uint32 payload).
struct Row {
    uint32_t key;
    uint32_t payload;
};
static_assert(sizeof(Row) == 8, "row layout");

// One unit of join work: an R chunk (fits one CTA's shared memory) against a
// run of S rows of the same partition.
struct Item {
    uint64_t r_off;
    uint64_t s_off;
    uint64_t s_len;
    uint32_t r_len;
    uint32_t part;
};

// Device-side control block, zeroed at the start of every join.
struct Ctrl {
    unsigned long long matches;   // equi-join cardinality
    unsigned long long rows;      // rows reserved in the output
    unsigned int error;           // first TBG_ERR_* raised on the device
    unsigned int nitems;          // join work items written by the planner
    unsigned int tiles[16];       // tile tickets, one slot per scatter launch
    unsigned int item_ctr[4];     // work-item tickets, one slot per join launch
    unsigned long long max_part_R, max_part_S;
    unsigned long long out_of_range;  // keys a range-checked histogram found outside its range
    unsigned long long nonempty;  // partitions with both sides non-empty
    unsigned long long heavy_rows_S;
    unsigned long long heavy_keys;
    unsigned long long pad[3];
};

// Digits per pass of the tile scatter (part_dev.cuh).
constexpr int SCATTER_FMAX = 256;

// Rows per thread per tile of the chunked partitioning passes.
constexpr int PART_THREADS = 512;
constexpr int PART_ITEMS = 8;

// Shared-memory table capacity of the build/probe kernels (rows of R_p).
constexpr int JOIN_THREADS = 512;
constexpr int JOIN_CAPR_DEFAULT = 5120;
constexpr int JOIN_CAPR_FIT = 8192;    // counting joins: the average R partition fills this table
constexpr int JOIN_CAPR_WIDE = 16384;  // ... and partitions up to this size are joined whole
constexpr int JOIN_CAPR_SMALL = 4096;  // count-only tables when every R partition fits it

// Bounded device waits: iterations before a wait gives up with TBG_ERR_TIMEOUT.
constexpr unsigned int SPIN_LIMIT = 1u << 21;

// Radix digit of the final partition index f for a key, pass-major:
// f = ((k & m1) << b2) | ((k >> b1) & m2) with k = key - sub.  With one pass,
// b2 = m2 = 0.
struct RadixF {
    uint32_t m1, b1, m2, b2;
    uint32_t sub = 0;  // digits are taken from key - sub (an order-preserving offset for sorts)
};

// Digit of a key in one partitioning pass: ((key - sub) >> shift) & mask.
struct DigitOp {
    uint32_t shift, mask;
    uint32_t sub = 0;
#ifdef __CUDACC__
    __host__ __device__
#endif
        uint32_t operator()(uint32_t key) const {
        return ((key - sub) >> shift) & mask;
    }
};

// Per-relation partition plan written by the planner kernel.
struct RelPlan {
    uint32_t *hist;       // [P]   final partition sizes
    uint64_t *base;       // [P+1] exclusive prefix, base[P] = n
};

// Arguments of the chunked partitioning passes (partition.cu).
struct PartArgs {
    const Row *in;
    Row *out;
    uint64_t n;               // rows (< 2^32)
    uint64_t chunk;           // rows per pass-1 chunk
    const uint32_t *chunk_len;  // rows of chunk c (null: full chunks of `chunk` rows)
    int G;                    // chunks
    int group;                // pass 2: consecutive chunks per unit
    int b1, b2;               // digit bits of pass 1 and pass 2 (b2 = 0: one pass)
    RadixF rf;
    DigitOp d1, d2;           // digit of pass 1 and of pass 2 (consistent with rf: f = d1 << b2 | d2)
    const uint32_t *pre;      // [G][P] rows of partition f in chunks before c
    const uint32_t *totals;   // [P]
    const uint64_t *base;     // [P+1]
    uint32_t *off1;           // [G][F1] start of unit (c, s) in the pass-1 output
    uint32_t *cnt1;           // [G][F1] rows of unit (c, s)
    unsigned *err;
};

struct JoinArgs {
    const Row *R;
    const Row *S;
    const Item *items;
    const unsigned int *nitems;
    unsigned int *item_ctr;
    int capR;
    int hash_shift;
    int layout;                // 0 bucket chain, 1 histogram (RHT)
    // Launch gate: with `gate` set, the launch does its work only when
    // *gate <= gate_max (gate_le != 0) or *gate > gate_max (gate_le == 0).
    const unsigned long long *gate;
    unsigned long long gate_max;
    int gate_le;
    unsigned long long *matches;
    unsigned long long *rows_ctr;
    tbg_row_out *out;
    uint64_t cap;
    unsigned int *err;
};

struct PlanArgs {
    RelPlan r, s;
    uint64_t nR, nS;
    int P_log2, b1, b2, passes;
    int capR;
    uint64_t capS;            // S rows per work item when splitting (0: no split)
    Item *items;
    uint64_t item_cap;
    Ctrl *ctrl;
};

// ---- launchers (partition.cu, join.cu, gen.cu) ----
cudaError_t launch_hist_chunks(const Row *in, uint64_t n, uint64_t chunk, int G, uint32_t *hist,
                               int P_log2, RadixF rf, cudaStream_t st,
                               unsigned long long *out_of_range = nullptr, uint32_t range_max = 0);
cudaError_t launch_colscan(uint32_t *hist, int G, int P, uint32_t *totals, cudaStream_t st);
cudaError_t launch_plan(const PlanArgs &a, cudaStream_t st);
cudaError_t launch_plan_bases(const uint32_t *totals, uint64_t *base, int P_log2, unsigned long long *maxp,
                              cudaStream_t st);
cudaError_t launch_part_pass1(const PartArgs &a, cudaStream_t st);
cudaError_t launch_part_pass2(const PartArgs &a, cudaStream_t st);
cudaError_t launch_join(const JoinArgs &a, bool materialize, int grid, cudaStream_t st);
size_t join_smem_bytes(int capR);
size_t join_launch_smem(int capR, bool materialize, int layout);
int join_ctas_per_sm(int capR, bool materialize, int layout);

cudaError_t launch_gen_pk(Row *d, uint64_t n, uint64_t seed, cudaStream_t st);
cudaError_t launch_gen_fk(Row *d, uint64_t n, uint64_t maxid, uint64_t seed, cudaStream_t st);
cudaError_t launch_gen_zipf(Row *d, uint64_t n, uint64_t alphabet, double z, int scatter,
                            uint64_t seed, cudaStream_t st);
cudaError_t launch_checksum(const tbg_row_out *rows, uint64_t n, unsigned long long *out,
                            cudaStream_t st);

// Counts kernel launches made by this library (reported by tbg_kernel_launches).
void count_launch(unsigned n = 1);

// Makes `bytes` of dynamic shared memory launchable for kernel `func` on the
// current device.  The limit is process-wide and shared by every host thread,
// so it is only ever raised (under a lock, to the largest size asked for so
// far): a launch that asks for less than the limit stays valid, and one
// thread's smaller launch never lowers the limit under another thread's
// larger one.
cudaError_t smem_limit(const void *func, size_t bytes);

}  // namespace tbg
