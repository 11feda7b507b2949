// Device building blocks of the build/probe join (shared-memory bucket-chain
// or histogram table, count probe), shared by the single-join kernel
// (join.cu) and the batched join (batch.cu).
#pragma once

#include "tbg_device.cuh"

namespace tbg {

// Largest power of two <= x (x >= 1).
__host__ __device__ __forceinline__ uint32_t floor_pow2(uint32_t x) {
    uint32_t p = 1;
    while (p <= x / 2) p <<= 1;
    return p;
}

// Bucket heads of a count-only bucket-chain table of capR rows: the largest
// power of two <= capR + 2, divided by TBG_COUNT_HEAD_DIV (a build option for
// A/B timing: fewer heads, longer chains, a smaller table and so more CTAs
// per SM).
#ifndef TBG_COUNT_HEAD_DIV
#define TBG_COUNT_HEAD_DIV 1
#endif
__host__ __device__ __forceinline__ uint32_t count_head_slots(int capR) {
    const uint32_t h = floor_pow2((uint32_t)capR + 2) / TBG_COUNT_HEAD_DIV;
    return h ? h : 1;
}

// Packed bucket head of a count-only bucket-chain table: the head entry's
// key, its 1-based row and its 1-based next link in one 64-bit word, so a
// probe whose chain has one entry costs one shared load.
__device__ __forceinline__ uint64_t pack_head(uint32_t key, uint32_t row1, uint32_t next1) {
    return ((uint64_t)key << 32) | (row1 << 16) | next1;
}

// Histogram-table probes read the bucket's keys four at a time (a build
// option for A/B timing).
#ifndef TBG_RHT_VEC_PROBE
#define TBG_RHT_VEC_PROBE 1
#endif

struct Table {
    uint32_t *key;    // [capR]
    uint32_t *pay;    // [capR] (unused with head64)
    uint32_t *heads;  // layout 0: [N] 1-based chain heads; layout 1: [Nb+1] starts, then cursors
    uint16_t *next;   // layout 0: [capR] 1-based next links
    uint64_t *head64; // layout 0, count only (else null): [N] packed heads instead of heads
    uint32_t mask;    // bucket mask
    uint32_t hcap;    // head slots available (a power of two <= capR + 2)
    int hs;           // hash shift (radix bits already consumed)
    int layout;

    __device__ __forceinline__ uint32_t bucket(uint32_t k) const { return (k >> hs) & mask; }

    template <class Fn>
    __device__ __forceinline__ void for_each(uint32_t k, Fn fn) const {
        const uint32_t b = bucket(k);
        if (layout == 0) {
            for (uint32_t h = heads[b]; h; h = next[h - 1])
                if (key[h - 1] == k) fn(pay[h - 1]);
        } else {
            for (uint32_t j = heads[b], e = heads[b + 1]; j < e; j++)
                if (key[j] == k) fn(pay[j]);
        }
    }
    __device__ __forceinline__ uint32_t count(uint32_t k) const {
        uint32_t c = 0;
        const uint32_t b = bucket(k);
        if (head64) {
            const uint64_t x = head64[b];
            c = ((x >> 16) & 0xFFFF) != 0 && (uint32_t)(x >> 32) == k;
            for (uint32_t h = (uint32_t)x & 0xFFFF; h; h = next[h - 1]) c += (key[h - 1] == k);
        } else if (layout == 0) {
            for (uint32_t h = heads[b]; h; h = next[h - 1]) c += (key[h - 1] == k);
        } else if (TBG_RHT_VEC_PROBE) {
            // the bucket's keys read as 16-byte words (key[] starts 16-byte
            // aligned): a word's slots before the bucket hold keys of other
            // buckets, which differ from k; slots at or past its end are
            // masked (past the table they may hold stale keys)
            const uint32_t j = heads[b], e = heads[b + 1];
            const uint4 *k4 = reinterpret_cast<const uint4 *>(key);
            for (uint32_t a4 = j & ~3u; a4 < e; a4 += 4) {
                const uint4 q = k4[a4 >> 2];
                c += (q.x == k) + (q.y == k && a4 + 1 < e) + (q.z == k && a4 + 2 < e) + (q.w == k && a4 + 3 < e);
            }
        } else {
            for (uint32_t j = heads[b], e = heads[b + 1]; j < e; j++) c += (key[j] == k);
        }
        return c;
    }
};


// R rows are read with plain loads, or with L2-only loads (CG) when they were
// written earlier in the same kernel launch by other CTAs.
template <bool CG>
__device__ __forceinline__ uint2 ld_row(const Row *R, uint64_t i) {
    const uint2 *p = reinterpret_cast<const uint2 *>(R) + i;
    if (CG) return __ldcg(p);
    return *p;
}
template <bool CG>
__device__ __forceinline__ uint4 ld_pair(const uint4 *p) {
    if (CG) return __ldcg(p);
    return ldg_stream(p);
}

template <int THREADS, bool CG = false>
__device__ void build_table(Table &t, const Row *__restrict__ R, uint64_t r_off, uint32_t r_len,
                            uint64_t *scan_scratch) {
    const int tid = threadIdx.x;
    if (t.head64) {
        // the same buckets and chains with packed heads: a row enters at
        // the head of its chain by compare-and-swap, its next link being the
        // head it displaced
        const uint32_t N = min(next_pow2(r_len), t.hcap);
        t.mask = N - 1;
        for (uint32_t i = tid; i < r_len; i += THREADS) t.key[i] = ld_row<CG>(R, r_off + i).x;
        for (uint32_t i = tid; i < N; i += THREADS) t.head64[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += THREADS) {
            const uint32_t k = t.key[i];
            unsigned long long *slot = reinterpret_cast<unsigned long long *>(&t.head64[t.bucket(k)]);
            unsigned long long old = *slot;
            for (;;) {  // ends: each failed swap means another row entered this chain
                const unsigned long long seen =
                    atomicCAS(slot, old, (unsigned long long)pack_head(k, i + 1, (uint32_t)(old >> 16) & 0xFFFF));
                if (seen == old) break;
                old = seen;
            }
            t.next[i] = (uint16_t)((old >> 16) & 0xFFFF);
        }
        __syncthreads();
    } else if (t.layout == 0) {
        // next_pow2(|R_p|) buckets as in the reference, at most hcap (a
        // longer average chain when capR is not a power of two)
        const uint32_t N = min(next_pow2(r_len), t.hcap);
        t.mask = N - 1;
        for (uint32_t i = tid; i < r_len; i += THREADS) {
            uint2 x = ld_row<CG>(R, r_off + i);
            t.key[i] = x.x;
            t.pay[i] = x.y;
        }
        for (uint32_t i = tid; i < N; i += THREADS) t.heads[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += THREADS) {
            uint32_t b = t.bucket(t.key[i]);
            t.next[i] = (uint16_t)atomicExch(&t.heads[b], i + 1);
        }
        __syncthreads();
    } else {
        uint32_t Nb = next_pow2(r_len) >> 2;
        if (Nb < 4) Nb = 4;
        t.mask = Nb - 1;
        uint32_t *cnt = t.heads;            // [Nb + 1]
        uint32_t *cur = t.heads + Nb + 1;   // cursors, Nb entries (fits: capR + 2 >= 2 Nb + 1)
        for (uint32_t i = tid; i <= Nb; i += THREADS) cnt[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += THREADS)
            atomicAdd(&cnt[t.bucket(ld_row<CG>(R, r_off + i).x)], 1u);
        __syncthreads();
        // exclusive scan of cnt[0..Nb) in place, cnt[Nb] = r_len
        const uint32_t per = (Nb + THREADS - 1) / THREADS;
        const uint32_t lo = min(Nb, tid * per), hi = min(Nb, lo + per);
        uint64_t s = 0;
        for (uint32_t i = lo; i < hi; i++) s += cnt[i];
        uint64_t tot;
        uint64_t run = block_excl_scan<THREADS>(s, &tot, scan_scratch);
        for (uint32_t i = lo; i < hi; i++) {
            uint32_t c = cnt[i];
            cnt[i] = (uint32_t)run;
            cur[i] = (uint32_t)run;
            run += c;
        }
        if (tid == 0) cnt[Nb] = r_len;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += THREADS) {
            uint2 x = ld_row<CG>(R, r_off + i);
            uint32_t pos = atomicAdd(&cur[t.bucket(x.x)], 1u);
            t.key[pos] = x.x;
            if (t.pay) t.pay[pos] = x.y;  // counting tables keep keys only
        }
        __syncthreads();
    }
}

// Matches of S rows [0, len) (row pointer s, any 8-byte alignment) against
// the table, this thread's share: 16-byte loads, four in flight, and with
// TBG_PROBE_AHEAD the next group of four issued before the current group is
// probed (the loads of one group then overlap the probes of the previous).
#ifndef TBG_PROBE_AHEAD
#define TBG_PROBE_AHEAD 1
#endif
template <int THREADS, bool CG = false>
__device__ __forceinline__ unsigned long long probe_count(const Table &t, const Row *s, uint64_t len) {
    unsigned long long local = 0;
    const uint64_t head = ((reinterpret_cast<uintptr_t>(s) & 15) && len) ? 1 : 0;
    const uint64_t body = len - head;
    const uint64_t nv = body / 2;
    const bool tail = body & 1;
    const uint4 *v = reinterpret_cast<const uint4 *>(s + head);
    const int tid = threadIdx.x;
    if (head && tid == 0) local += t.count(ld_row<CG>(s, 0).x);
    if (tail && tid == THREADS - 1) local += t.count(ld_row<CG>(s, len - 1).x);
    uint64_t i = tid;
    if (TBG_PROBE_AHEAD && i + 3 * THREADS < nv) {
        uint4 n0 = ld_pair<CG>(v + i), n1 = ld_pair<CG>(v + i + THREADS);
        uint4 n2 = ld_pair<CG>(v + i + 2 * THREADS), n3 = ld_pair<CG>(v + i + 3 * THREADS);
        for (;;) {
            const uint4 x0 = n0, x1 = n1, x2 = n2, x3 = n3;
            i += 4 * THREADS;
            const bool more = i + 3 * THREADS < nv;
            if (more) {
                n0 = ld_pair<CG>(v + i);
                n1 = ld_pair<CG>(v + i + THREADS);
                n2 = ld_pair<CG>(v + i + 2 * THREADS);
                n3 = ld_pair<CG>(v + i + 3 * THREADS);
            }
            local += t.count(x0.x) + t.count(x0.z) + t.count(x1.x) + t.count(x1.z);
            local += t.count(x2.x) + t.count(x2.z) + t.count(x3.x) + t.count(x3.z);
            if (!more) break;
        }
    }
    for (; i + 3 * THREADS < nv; i += 4 * THREADS) {
        uint4 x0 = ld_pair<CG>(v + i), x1 = ld_pair<CG>(v + i + THREADS);
        uint4 x2 = ld_pair<CG>(v + i + 2 * THREADS), x3 = ld_pair<CG>(v + i + 3 * THREADS);
        local += t.count(x0.x) + t.count(x0.z) + t.count(x1.x) + t.count(x1.z);
        local += t.count(x2.x) + t.count(x2.z) + t.count(x3.x) + t.count(x3.z);
    }
    for (; i < nv; i += THREADS) {
        uint4 x0 = ld_pair<CG>(v + i);
        local += t.count(x0.x) + t.count(x0.z);
    }
    return local;
}

}  // namespace tbg
