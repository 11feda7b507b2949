// Host-side runtime structures of tee-bench-b200 (workspace cache, join run
// record) shared by the C ABI and the per-algorithm pipelines.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <cuda_runtime.h>

#include "tbg_internal.h"

namespace tbg {

// A device buffer that only grows.
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    bool fresh = false;  // set when (re)allocated; consumers that need zeroed memory clear it
    cudaError_t ensure(size_t bytes);
    void release();
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

// Scratch of one (device, stream): reused by consecutive joins on that stream.
struct Workspace {
    int device = 0;
    int nsm = 148;
    DevBuf ctrl, histR, histS, totR, totS, baseR, baseS, off1R, off1S, cnt1R, cnt1S;
    DevBuf tmpR, tmpS, partR, partS, items, misc;
    DevBuf inR, inS, rows;      // drop-in layer: device copies of host inputs and output rows
    DevBuf sc, kept;            // learned path: compacted S and kept rows per chunk
    DevBuf sorthist;            // PSM sort: per-chunk digit histograms and totals
    DevBuf chain_rows, chain_rel;  // chained join: first join's rows and the relation made of them
    DevBuf aux[8];              // algorithm-specific scratch (sort, learned model)
    DevBuf shard;               // shard split: per-chunk histograms and totals
    Ctrl *host_ctrl = nullptr;  // pinned mirror of the control block
    static constexpr size_t HOST_SMALL_BYTES = 4096;
    void *host_small = nullptr;  // pinned HOST_SMALL_BYTES: mid-call read-backs (LRN's decision, shard totals)
    cudaEvent_t ev[8];
    cudaStream_t side = nullptr;       // second stream (learned path), created on first use
    cudaEvent_t fork = nullptr, joined = nullptr, table = nullptr, emit = nullptr;
};

// What one join call did (for stats).
struct JoinRun {
    int B = 0, passes = 0;
    uint64_t P = 0;
    bool timed = false;
    int used_fallback = 0;
    double predicted_imbalance = 0;
    int train_steps = 0;
    float train_loss = 0;
    float ms_learn = 0;
    double heavy_pred = 0, heavy_sampled = 0;
    uint64_t launches = 0;
};

Workspace *workspace_for(cudaStream_t st);
int set_error(int code, const char *fmt, ...);
int cuda_error(cudaError_t e, const char *what);
void choose_radix(const tbg_config &cfg, uint64_t nR, int capR, int *B, int *passes);
int join_capacity(uint64_t nR, bool counting);

int join_device_impl(const tbg_config *cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                     tbg_row_out *d_rows, uint64_t rows_cap, cudaStream_t st, JoinRun *run,
                     Workspace **wout);
int finish_join(const tbg_config &cfg, Workspace &w, cudaStream_t st, const JoinRun &run,
                uint64_t nR, uint64_t nS, uint64_t cap, uint64_t *matches, tbg_stats *stats);

// Heavy-key table used by the S histogram of the learned path (device pointers).
struct SBypass {
    const uint32_t *keys;
    const unsigned *cnt;           // R rows per heavy slot (materialising)
    unsigned *scnt;                // S rows per heavy slot (counting)
    uint32_t *hkept;               // materialising: [G] heavy S rows per chunk
    unsigned long long *hpairs;    // materialising: [G] heavy output rows per chunk
};
struct RadixGeom {
    int B, passes, b1, b2;
    uint64_t P, F1;
    int capR, join_grid;
    uint64_t capS, item_cap;
    int G[2];          // chunks of R, S
    uint64_t ch[2];    // rows per chunk
    uint64_t n[2];     // rows of R, S
    RadixF rf;         // final partition f of a key (histograms)
    DigitOp d1, d2;    // pass-1 and pass-2 digits: f = d1 << b2 | d2
    // S's histogram also counts keys with key - rf.sub > s_range_max into
    // ctrl->out_of_range (S binned by R's key range); 0xFFFFFFFF: no check
    uint32_t s_range_max = 0xFFFFFFFFu;
};
RadixGeom radix_geometry(const tbg_config &cfg, uint64_t nR, uint64_t nS, int capR, Workspace &w);
RadixGeom radix_geometry_msd(uint64_t nR, uint64_t nS, uint32_t sub, int B, int lowbits, Workspace &w);
int ensure_radix_buffers(const RadixGeom &g, bool bypass, Workspace &w);
int part_histogram(int rel, const RadixGeom &g, const Row *d, const tbg_config &cfg, Workspace &w, cudaStream_t st,
                   const SBypass *bypass);
int part_pass(int rel, int which, const RadixGeom &g, const Row *d, Workspace &w, cudaStream_t st, bool bypass);
int plan_items(const RadixGeom &g, Workspace &w, cudaStream_t st);
void mark(Workspace &w, bool timing, int i, cudaStream_t st);
int radix_partition(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                    int capR, Workspace &w, cudaStream_t st, JoinRun *run, int *join_grid_out);
int radix_join_phase(const tbg_config &cfg, tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st,
                     JoinRun *run, int capR, int join_grid);
int lsd_sort_chunked(const Row *in, uint64_t n, uint32_t kmin, uint32_t kmax, DevBuf &a, DevBuf &b, Workspace &w,
                     cudaStream_t st, const Row **out, int *passes);
cudaError_t launch_key_range(const Row *in, uint64_t n, uint32_t *minmax, int nsm, cudaStream_t st);
int run_radix_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                   tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run);
int run_radix_join_sliced(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, const uint64_t *s_lo,
                          int nslices, const std::function<int(int)> &issue, cudaEvent_t r_ready,
                          const cudaEvent_t *s_ready, tbg_row_out *d_rows, uint64_t cap, Workspace &w,
                          cudaStream_t st, JoinRun *run);
int run_sortmerge_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                       tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run);
int run_psm_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                 tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run);
int run_learned_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                     tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run);

}  // namespace tbg
