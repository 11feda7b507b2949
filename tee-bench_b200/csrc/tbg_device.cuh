// Device-side helpers shared by the sm_100a kernels.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#include "tbg_internal.h"

namespace tbg {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__host__ __device__ __forceinline__ uint64_t umin64(uint64_t a, uint64_t b) { return a < b ? a : b; }

__device__ __forceinline__ uint32_t radix_f(const RadixF &rf, uint32_t key) {
    key -= rf.sub;
    return ((key & rf.m1) << rf.b2) | ((key >> rf.b1) & rf.m2);
}

// streaming loads: data read once, keep it out of L1
__device__ __forceinline__ uint4 ldg_stream(const uint4 *p) { return __ldcs(p); }
__device__ __forceinline__ uint2 ldg_stream(const uint2 *p) { return __ldcs(p); }

__device__ __forceinline__ uint64_t ld_relaxed(const uint64_t *p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint64_t *p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned warp_max_u32(unsigned v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Output rows of one block round, NJ row slots per thread: thread t emits
// c[j] rows for slot j.  Positions follow (slot j, warp, lane) order within
// a warp's share, so when each row has at most one match consecutive lanes
// write consecutive rows (coalesced stores).  One atomicAdd on *rows_ctr
// reserves the whole block's rows.  `scratch` holds THREADS / 32 + 1 words;
// every thread of the block must call it; it ends with a barrier.
template <int THREADS, int NJ>
__device__ __forceinline__ void block_emit_positions(const uint32_t (&c)[NJ], uint64_t (&pos)[NJ],
                                                     unsigned long long *rows_ctr, uint64_t *scratch) {
    constexpr int NW = THREADS / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t wpre[NJ];
    uint32_t wtot = 0;
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        uint32_t inc = c[j];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        wpre[j] = wtot + inc - c[j];
        wtot += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) scratch[w] = wtot;
    __syncthreads();
    if (w == 0) {
        const uint64_t mine = lane < NW ? scratch[lane] : 0;
        uint64_t inc = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        const uint64_t total = __shfl_sync(0xffffffffu, inc, 31);
        uint64_t base = 0;
        if (lane == 0 && total) base = atomicAdd(rows_ctr, (unsigned long long)total);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (lane < NW) scratch[lane] = base + inc - mine;
    }
    __syncthreads();
    const uint64_t wbase = scratch[w];
#pragma unroll
    for (int j = 0; j < NJ; j++) pos[j] = wbase + wpre[j];
    __syncthreads();  // scratch is reused by the next round
}

// Lanes of the warp whose value d (< 512) equals this lane's: one ballot per
// bit, so the cost does not depend on how many distinct values the warp
// holds (unlike __match_any_sync).  Every lane of the warp must call it.
__device__ __forceinline__ unsigned warp_peers9(uint32_t d) {
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const bool bit = (d >> k) & 1;
        const unsigned b = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? b : ~b;
    }
    return peers;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide exclusive scan of one uint64 per thread.  Every thread of the
// block must call it.  scratch holds THREADS/32 + 1 words.
template <int THREADS, bool TAIL_SYNC = true>
__device__ __forceinline__ uint64_t block_excl_scan(uint64_t v, uint64_t *total, uint64_t *scratch) {
    constexpr int NW = THREADS / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scratch[w] = x;
    __syncthreads();
    if (w == 0) {
        uint64_t s = lane < NW ? scratch[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < NW) scratch[lane] = s;
    }
    __syncthreads();
    uint64_t before = w ? scratch[w - 1] : 0;
    *total = scratch[NW - 1];
    if (TAIL_SYNC) __syncthreads();  // without it the caller syncs before reusing scratch
    return before + x - v;
}

__device__ __forceinline__ uint32_t next_pow2(uint32_t v) {
    if (v <= 1) return 1;
    return 1u << (32 - __clz(v - 1));
}

// splitmix64 finaliser (Steele, Lea, Flood 2014): a row mixer for checksums
// and a counter-based random source for the generators.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t row_hash(uint32_t key, uint32_t rp, uint32_t sp) {
    return mix64((((uint64_t)key << 32) | rp) ^ mix64((uint64_t)sp));
}

}  // namespace tbg

namespace tbg {

// ---- bulk-copy (TMA) and mbarrier helpers --------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's (and, after a barrier, the CTA's) generic-proxy shared
// memory accesses before later async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global memory into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// this CTA's shared memory to global memory, in this thread's current bulk
// group (no multicast).
__device__ __forceinline__ void bulk_s2g(void *dst, const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// This thread's bulk stores have read their shared-memory sources.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// This thread's bulk stores are complete (their global writes done).
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Bounded wait for phase `parity` of `bar`; false when the limit ran out.
// Bulk prefetch of [p, p + bytes) into L2 (TMA, no destination); the range
// is rounded inward to 16-byte bounds, so it never reaches past the rows.
__device__ __forceinline__ void prefetch_l2(const void *p, uint64_t bytes) {
    const uintptr_t lo = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t hi = (reinterpret_cast<uintptr_t>(p) + bytes) & ~uintptr_t(15);
    for (uintptr_t a = lo; a < hi; a += (1u << 20)) {  // at most 1 MB per instruction
        const uint32_t n = (uint32_t)(hi - a < (1u << 20) ? hi - a : (1u << 20));
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
    }
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace tbg
