// Batched joins: many independent equi-joins of uneven sizes in one
// persistent kernel launch.  Device-side plan structures shared by batch.cu
// (kernel) and batch.cpp (planner, autotuner, CUDA graph).
//
// The reference runs one join per process (native.cpp:125 calls the
// algorithm picked by name once; a harness loops RHO over the joins), so
// there is no counterpart to this layout in the reference; each
// join's result equals RHO's count (Joins/radix_join.c:1558-1561) on that
// join's two relations.
#pragma once

#include <cstdint>

#include "tbg_internal.h"

namespace tbg {

constexpr int BATCH_THREADS = 512;
constexpr int BATCH_FMAX = 256;    // one partitioning pass, fan-out <= 256
constexpr int BATCH_CAPR = 8192;   // R rows per shared-memory table
constexpr uint32_t BATCH_SPIN_LIMIT = 1u << 22;

// One join of the batch, in plan order.  B == 0: direct join (no
// partitioning; R is loaded into shared memory capR rows at a time and S is
// probed in slices of capS rows).  B > 0: one radix pass over P = 2^B
// partitions of the low key bits, then build/probe per partition.
struct BatchJoin {
    const Row *R, *S;          // caller's relations (device memory, any 8-byte alignment)
    Row *Rp, *Sp;              // partitioned copies (256-byte aligned regions)
    uint32_t *histR, *histS;   // [GR][P], [GS][P]: per-chunk counts, then per-chunk prefixes
    uint32_t *baseR, *baseS;   // [P] partition starts inside Rp / Sp
    Item *items;               // [item_cap] join work items of this join
    uint64_t nR, nS;
    uint32_t B, P, layout, capS;
    uint32_t GR, GS, chunk, item_cap;
    uint32_t orig;             // index in the caller's array (result slot)
    uint32_t pad;
};

// Per-join progress counters (zeroed before every run).
struct BatchSync {
    unsigned hist_done;  // histogram chunks finished
    unsigned scan_done;  // 1 once bases and items are written
    unsigned scat_done;  // scatter chunks finished
    unsigned nitems;     // items written by the scan
    unsigned item_ctr;   // next item handed to a worker
    unsigned pad[3];
};

// Ticket order: [hist chunks | scans | scatter chunks | join tickets].  A
// ticket depends only on tickets handed out before it, and a handed-out
// ticket belongs to a running CTA, so every wait ends without requiring all
// CTAs to be co-resident.
struct BatchArgs {
    const BatchJoin *joins;
    const uint2 *chunks;     // [n_chunks] {join, rel << 31 | chunk index}
    const uint32_t *scans;   // [n_scans] join
    const uint2 *jt;         // [n_jt] {join, worker or S-slice index}
    BatchSync *sync;         // [njoins]
    unsigned *ticket;
    unsigned *err;
    unsigned long long *counts;  // [njoins] by caller index
    uint32_t n_chunks, n_scans, n_jt, capR;
};

size_t batch_smem_bytes();
int batch_ctas_per_sm();
// Sets k_batch's shared-memory limit on the current device and returns its
// resident CTAs per SM; the status of both CUDA calls is returned.
cudaError_t batch_occupancy(int *per_sm);
cudaError_t launch_batch(const BatchArgs &a, int grid, cudaStream_t st);

}  // namespace tbg
