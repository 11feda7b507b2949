// Device building blocks of the chunked radix partitioning (warp ranking,
// the TMA-fed digit-sorting tile scatter), shared by the single-join passes
// (partition.cu) and the batched join (batch.cu).
#pragma once

#include "tbg_device.cuh"

namespace tbg {

// ---------------------------------------------------------------------------
// shared helpers
// ---------------------------------------------------------------------------

// True when neighbouring lanes of the warp hold the same digit: a sign of
// skew, for which ranks are aggregated with __match_any_sync.
__device__ __forceinline__ bool warp_has_dups(uint32_t d, bool valid) {
    const int lane = threadIdx.x & 31;
    const uint32_t key = valid ? d : 0xFFFFFFFFu;
    const uint32_t up = __shfl_up_sync(0xffffffffu, key, 1);
    return __any_sync(0xffffffffu, valid && lane > 0 && up == key);
}

// Adds one row's bin to a shared histogram; every lane of the warp calls it
// (valid = false for lanes without a row).  With `dup` (the warp showed
// repeated bins: skew), lanes sharing a bin are merged by __match_any_sync
// into one atomic; otherwise each row pays one shared atomic.
__device__ __forceinline__ void hist_add_warp(uint32_t *h, uint32_t f, bool valid, bool dup) {
    if (!dup) {
        if (valid) atomicAdd(&h[f], 1u);
    } else {
        const unsigned peers = __match_any_sync(0xffffffffu, valid ? f : 0xFFFFFFFFu);
        if (valid && (peers & lanemask_lt()) == 0) atomicAdd(&h[f], (uint32_t)__popc(peers));
    }
}

// Rank of a row on a shared digit counter (returns the old count).
// Correct either way; `dup` only picks the faster path.
__device__ __forceinline__ uint32_t rank_warp(uint32_t *cnt, uint32_t d, bool valid, bool dup) {
    const int lane = threadIdx.x & 31;
    const uint32_t key = valid ? d : 0xFFFFFFFFu;
    uint32_t r = 0;
    if (!dup) {
        if (valid) r = atomicAdd(&cnt[d], 1u);
    } else {
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int leader = __ffs(peers) - 1;
        uint32_t b = 0;
        if (valid && lane == leader) b = atomicAdd(&cnt[d], (uint32_t)__popc(peers));
        b = __shfl_sync(0xffffffffu, b, leader);
        r = b + __popc(peers & lanemask_lt());
    }
    return r;
}

// ---------------------------------------------------------------------------
// tile scatter shared by both passes
// ---------------------------------------------------------------------------
template <int THREADS>
struct PartSmem {
    static constexpr int NW = THREADS / 32;
    static constexpr int T = THREADS * PART_ITEMS;
    Row buf[2][T + 2];                          // input tile (bulk copy), then the same tile digit-sorted
    uint32_t cnt[2][SCATTER_FMAX];              // per-digit counts of the tile, double-buffered
    uint32_t cursor[SCATTER_FMAX];              // next output row of each digit
    uint32_t delta[SCATTER_FMAX];               // cursor - tile offset of the digit
    uint64_t scan[NW + 1];
    uint64_t mbar[2];
};

// Digit of a pass: a bit field of the key (pass 1: bits [0, b1); pass 2:
// bits [b1, b1 + b2); one pass: bits [0, B)).
struct DigitOp {
    uint32_t shift, mask;
    __device__ __forceinline__ uint32_t operator()(uint32_t key) const { return (key >> shift) & mask; }
};

// Where tile rows [t, t + cnt) sit in a shared buffer: the bulk copy moves
// the 16-byte aligned rows [a_lo, a_hi); row r is at buffer index r + off so
// the copy's destination is 16-byte aligned too; edge rows outside the copy
// (at most one at each end) are read from global memory.
struct TileGeo {
    uint64_t t;
    uint32_t cnt, a_lo, a_hi, off;
};

__device__ __forceinline__ TileGeo tile_geo(const Row *in, uint64_t t, uint32_t cnt) {
    TileGeo g;
    g.t = t;
    g.cnt = cnt;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(in + t);
    g.a_lo = (addr & 15) ? 1u : 0u;
    g.a_hi = ((addr + (uintptr_t)cnt * 8) & 15) ? cnt - 1 : cnt;
    if (g.a_hi < g.a_lo) g.a_hi = g.a_lo;  // a single misaligned row: no copy
    g.off = g.a_lo;
    return g;
}

__device__ __forceinline__ void issue_tile(const Row *in, const TileGeo &g, Row *buf, uint64_t *bar) {
    const uint32_t bytes = (g.a_hi - g.a_lo) * 8;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (bytes) bulk_g2s(buf + g.a_lo + g.off, in + g.t + g.a_lo, bytes, bar);
}

// One tile: rows are read from the landed buffer and ranked on one shared
// counter per digit (order inside a digit is free: partitions are
// multisets), one warp prefixes the counts over digits, then the
// tile is staged digit-sorted into the same buffer and written out in slot
// order, so consecutive threads store consecutive rows of each digit's run.
//
// kseq counts the tiles this CTA has processed on the barrier pair `mbar`
// (buffer kseq & 1, phase parity (kseq >> 1) & 1), so a persistent CTA can
// run many ranges without re-initialising the barriers.
template <int THREADS, bool FULL>
__device__ __forceinline__ void part_tile(const Row *__restrict__ in, const TileGeo &g, uint32_t kseq,
                                          bool has_next, const TileGeo &gnext, uint2 *__restrict__ out,
                                          uint32_t out_n, DigitOp dop, int F, PartSmem<THREADS> &sm,
                                          uint64_t *mbar, unsigned *err) {
    constexpr int NW = THREADS / 32;
    (void)NW;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int b = kseq & 1;
    const uint32_t wbase = (uint32_t)w * 32 * PART_ITEMS;
    const uint32_t cnt = g.cnt;
    uint32_t *c = sm.cnt[b];
    if (!mbar_wait(&mbar[b], (kseq >> 1) & 1, SPIN_LIMIT * 16)) atomicCAS(err, 0u, (unsigned)TBG_ERR_TIMEOUT);
    uint2 v[PART_ITEMS];
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        const uint32_t r = wbase + i * 32 + lane;
        if (FULL || r < cnt) {
            if (r >= g.a_lo && r < g.a_hi) {
                const Row x = sm.buf[b][r + g.off];
                v[i] = make_uint2(x.key, x.payload);
            } else {
                v[i] = reinterpret_cast<const uint2 *>(in)[g.t + r];
            }
        }
    }
    for (int i = tid; i < F; i += THREADS) sm.cnt[b ^ 1][i] = 0;
    uint32_t rank[PART_ITEMS];
    const bool dup = warp_has_dups(dop(v[0].x), FULL || wbase + lane < cnt);
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        const bool valid = FULL || wbase + i * 32 + lane < cnt;
        rank[i] = rank_warp(c, valid ? dop(v[i].x) : 0, valid, dup);
    }
    __syncthreads();
    // the other buffer is free (its tile was written out before this barrier)
    if (tid == 0 && has_next) issue_tile(in, gnext, sm.buf[b ^ 1], &mbar[b ^ 1]);
    if (w == 0) {
        // one warp prefixes the digit counts; lane l owns digits l, l + 32, ...
        // and the tile lays digits out in that (lane, i) order: any order
        // works as long as each digit's rows stay contiguous
        constexpr int PER = SCATTER_FMAX / 32;
        uint32_t sum = 0;
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int d = lane + 32 * i;
            sum += d < F ? c[d] : 0;
        }
        uint32_t inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        uint32_t run = inc - sum;
#pragma unroll
        for (int i = 0; i < PER; i++) {
            const int d = lane + 32 * i;
            if (d < F) {
                const uint32_t x = c[d];
                c[d] = run;
                sm.delta[d] = sm.cursor[d] - run;
                sm.cursor[d] += x;
                run += x;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        if (FULL || wbase + i * 32 + lane < cnt) {
            const uint32_t j = c[dop(v[i].x)] + rank[i];
            sm.buf[b][j] = Row{v[i].x, v[i].y};
        }
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < PART_ITEMS; kk++) {
        const uint32_t j = kk * THREADS + tid;
        if (FULL || j < cnt) {
            const Row x = sm.buf[b][j];
            const uint32_t pos = sm.delta[dop(x.key)] + j;
            if (pos < out_n) out[pos] = make_uint2(x.key, x.payload);
            else atomicCAS(err, 0u, (unsigned)TBG_ERR_ARG);
        }
    }
}

// Scatters rows [lo, hi) of `in`, digit by digit, to out[sm.cursor[d]...];
// the caller initialises sm.cursor[0..F) and synchronises.  Tile k + 1 is
// bulk-copied into the second buffer while tile k is processed.  `kseq` is
// the CTA's running tile count on the barrier pair (see part_tile); the
// barriers are initialised once by the caller.
template <int THREADS>
__device__ void part_tiles(const Row *__restrict__ in, uint64_t lo, uint64_t hi, Row *__restrict__ out,
                           uint32_t out_n, DigitOp dop, int F, PartSmem<THREADS> &sm, uint64_t *mbar,
                           uint32_t &kseq, unsigned *err) {
    constexpr int T = THREADS * PART_ITEMS;
    uint2 *o = reinterpret_cast<uint2 *>(out);
    const int ntiles = (int)((hi - lo + T - 1) / T);
    for (int i = threadIdx.x; i < F; i += THREADS) sm.cnt[kseq & 1][i] = 0;
    __syncthreads();
    if (ntiles == 0) return;
    TileGeo g = tile_geo(in, lo, (uint32_t)umin64(T, hi - lo));
    if (threadIdx.x == 0) issue_tile(in, g, sm.buf[kseq & 1], &mbar[kseq & 1]);
    for (int k = 0; k < ntiles; k++, kseq++) {
        const uint64_t t1 = g.t + T;
        const bool more = k + 1 < ntiles;
        const TileGeo gn = more ? tile_geo(in, t1, (uint32_t)umin64(T, hi - t1)) : g;
        if (g.cnt == T) part_tile<THREADS, true>(in, g, kseq, more, gn, o, out_n, dop, F, sm, mbar, err);
        else part_tile<THREADS, false>(in, g, kseq, more, gn, o, out_n, dop, F, sm, mbar, err);
        g = gn;
    }
    __syncthreads();  // the last tile's staging buffer is free again
}

// One range per CTA: initialises the barrier pair held in `sm`.
template <int THREADS>
__device__ void part_range(const Row *__restrict__ in, uint64_t lo, uint64_t hi, Row *__restrict__ out,
                           uint32_t out_n, DigitOp dop, int F, PartSmem<THREADS> &sm, unsigned *err) {
    if (threadIdx.x == 0) {
        mbar_init(&sm.mbar[0], 1);
        mbar_init(&sm.mbar[1], 1);
        fence_mbar_init();
    }
    uint32_t kseq = 0;
    part_tiles<THREADS>(in, lo, hi, out, out_n, dop, F, sm, sm.mbar, kseq, err);
}

}  // namespace tbg
