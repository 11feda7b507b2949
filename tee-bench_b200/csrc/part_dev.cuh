// Device building blocks of the chunked radix partitioning (warp ranking,
// the TMA-fed digit-sorting tile scatter), shared by the single-join passes
// (partition.cu) and the batched join (batch.cu).
#pragma once

#include "tbg_device.cuh"

namespace tbg {

// ---------------------------------------------------------------------------
// shared helpers
// ---------------------------------------------------------------------------

// True when at least four neighbouring lane pairs of the warp hold the same
// digit: a sign of skew, for which the hot values' rows are aggregated (see
// hot_peers).  Fewer repeats (uniform keys over 128-256 digits give a pair
// in about one warp in five) cost less as plain atomics.
__device__ __forceinline__ bool warp_has_dups(uint32_t d, bool valid) {
    const int lane = threadIdx.x & 31;
    const uint32_t key = valid ? d : 0xFFFFFFFFu;
    const uint32_t up = __shfl_up_sync(0xffffffffu, key, 1);
    return __popc(__ballot_sync(0xffffffffu, valid && lane > 0 && up == key)) >= 4;
}

// Under skew a warp holds a few hot values among many distinct ones.  The
// lanes equal to lane 0's or lane 16's value (the likely hot ones) form a
// group: returns its lane mask for this lane, or 0 if this lane is in
// neither group.  Two shuffles and two ballots, whatever the spread.
__device__ __forceinline__ unsigned hot_peers(uint32_t key) {
    const uint32_t c0 = __shfl_sync(0xffffffffu, key, 0);
    const uint32_t c1 = __shfl_sync(0xffffffffu, key, 16);
    const unsigned g0 = __ballot_sync(0xffffffffu, key == c0);
    const unsigned g1 = __ballot_sync(0xffffffffu, key == c1 && key != c0);
    return key == c0 ? g0 : (key == c1 ? g1 : 0u);
}

// Adds one row's bin to a shared histogram; every lane of the warp calls it
// (valid = false for lanes without a row).  With `dup` (the warp showed
// repeated bins: skew), the hot groups add once per group; other rows pay
// one shared atomic each.
__device__ __forceinline__ void hist_add_warp(uint32_t *h, uint32_t f, bool valid, bool dup) {
    if (!dup) {
        if (valid) atomicAdd(&h[f], 1u);
    } else {
        const unsigned peers = hot_peers(valid ? f : 0xFFFFFFFFu);
        if (!valid) return;
        if (!peers) atomicAdd(&h[f], 1u);
        else if ((peers & lanemask_lt()) == 0) atomicAdd(&h[f], (uint32_t)__popc(peers));
    }
}

// Rank of a row on a shared digit counter (returns the old count).
// Correct either way; `dup` only picks the faster path.
__device__ __forceinline__ uint32_t rank_warp(uint32_t *cnt, uint32_t d, bool valid, bool dup) {
    uint32_t r = 0;
    if (!dup) {
        if (valid) r = atomicAdd(&cnt[d], 1u);
    } else {
        const unsigned peers = hot_peers(valid ? d : 0xFFFFFFFFu);
        const int leader = peers ? __ffs(peers) - 1 : 0;
        uint32_t b = 0;
        if (valid) {
            if (!peers) r = atomicAdd(&cnt[d], 1u);
            else if ((int)(threadIdx.x & 31) == leader) b = atomicAdd(&cnt[d], (uint32_t)__popc(peers));
        }
        // every lane joins both shuffles; group members take their leader's base
        const uint32_t b0 = __shfl_sync(0xffffffffu, b, leader);
        if (valid && peers) r = b0 + __popc(peers & lanemask_lt());
    }
    return r;
}

// ---------------------------------------------------------------------------
// tile scatter shared by both passes
// ---------------------------------------------------------------------------
// Tile buffers per CTA (the default): tile q is loaded and ranked while tile
// q - 1 is written out and tile q + 1 is being copied in.
constexpr int PART_NBUF = 3;

// Write-out of a staged tile by bulk stores: every digit run is staged with
// its shared-memory start in the same 16-byte phase as its global
// destination (one spare slot per digit), and one thread per digit stores
// the run's aligned body with one cp.async.bulk store, its edge rows (at most
// one at each end) with plain stores.  The per-row shared loads and global
// stores of the write-out leave the SM's load/store pipe.  An output that
// is not 16-byte aligned takes plain stores for every row.
#ifndef TBG_BULK_STORE
#define TBG_BULK_STORE 0
#endif
constexpr bool PART_BULK = TBG_BULK_STORE != 0;
// A third barrier at the end of every tile (the layout before the tile loop
// was shown not to need it; kept as a build option for A/B timing).
#ifndef TBG_TILE_END_BARRIER
#define TBG_TILE_END_BARRIER 0
#endif
constexpr int PART_PAD = PART_BULK ? SCATTER_FMAX : 0;  // spare slots per staged tile

template <int THREADS, int NBUF = PART_NBUF>
struct PartSmem {
    static constexpr int NW = THREADS / 32;
    static constexpr int T = THREADS * PART_ITEMS;
    Row buf[NBUF][T + 2 + PART_PAD];            // input tiles (bulk copies), each then staged digit-sorted in place
    alignas(16) uint32_t cnt[2][SCATTER_FMAX];  // per-digit counts, then tile offsets, of the two newest tiles
    alignas(16) uint32_t delta[2][SCATTER_FMAX];  // output row - tile slot per digit, of the two newest tiles
    alignas(16) uint32_t cursor[SCATTER_FMAX];  // next output row of each digit
    // bulk write-out: each digit's staged start and row count, of the two newest tiles
    alignas(16) uint32_t rstart[PART_BULK ? 2 : 1][PART_BULK ? SCATTER_FMAX : 4];
    alignas(16) uint32_t rcount[PART_BULK ? 2 : 1][PART_BULK ? SCATTER_FMAX : 4];
    uint64_t scan[NW + 1];
    uint64_t mbar[NBUF];
};

// Digit of a pass: a bit field of the key (pass 1: bits [0, b1); pass 2:
// bits [b1, b1 + b2); one pass: bits [0, B)).

// Destination shard of a key for a join split over n shards (n <= 256): the
// top bits of a multiplicative hash, range-reduced by a multiply-shift, so
// every shard gets an even share of the keys whatever their order or skew,
// and the low key bits that the shards' own radix passes use stay evenly
// spread inside each shard.
struct ShardOp {
    uint32_t n;
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t key) const {
        return (uint32_t)(((uint64_t)(key * 0x9E3779B1u) * n) >> 32);
    }
};

// Where tile rows [t, t + cnt) of an n-row array sit in a shared buffer:
// the bulk copy moves rows [t + c_lo, t + c_hi), a 16-byte aligned span;
// row r (relative to t) is at buffer index r + off, so the copy's
// destination is 16-byte aligned too.  When the tile starts or ends 8 bytes
// past a 16-byte boundary, the copy takes the neighbouring row of the array
// as well, so the whole tile arrives by the bulk copy; only at the array's
// own ends, where no neighbour exists, is an edge row left out of the copy
// (tile rows outside [a_lo, a_hi)) and read from global memory.
struct TileGeo {
    uint64_t t;
    uint32_t cnt, a_lo, a_hi, off;
    int32_t c_lo, c_hi;
};

__device__ __forceinline__ TileGeo tile_geo(const Row *in, uint64_t t, uint32_t cnt, uint64_t n) {
    TileGeo g;
    g.t = t;
    g.cnt = cnt;
    const uintptr_t addr = reinterpret_cast<uintptr_t>(in + t);
    const bool lo_mis = (addr & 15) != 0;
    const bool hi_mis = ((addr + (uintptr_t)cnt * 8) & 15) != 0;
    g.c_lo = lo_mis ? (t >= 1 ? -1 : 1) : 0;
    g.c_hi = hi_mis ? (t + cnt < n ? (int32_t)cnt + 1 : (int32_t)cnt - 1) : (int32_t)cnt;
    if (g.c_hi < g.c_lo) g.c_hi = g.c_lo;  // a single row at an array end: no copy
    g.off = lo_mis ? 1u : 0u;
    g.a_lo = (uint32_t)max(g.c_lo, 0);
    g.a_hi = (uint32_t)min(g.c_hi, (int32_t)cnt);
    if (g.a_hi < g.a_lo) g.a_hi = g.a_lo;
    return g;
}

__device__ __forceinline__ void issue_tile(const Row *in, const TileGeo &g, Row *buf, uint64_t *bar) {
    const uint32_t bytes = (uint32_t)(g.c_hi - g.c_lo) * 8;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (bytes) bulk_g2s(buf + g.c_lo + (int32_t)g.off, in + (int64_t)g.t + g.c_lo, bytes, bar);
}

// A tile's rows are read from its landed buffer and ranked on one shared
// counter per digit (order inside a digit is free: partitions are
// multisets); one warp prefixes the counts over digits while the other warps
// write out the previous tile; then the tile is staged digit-sorted into its
// own buffer, to be written out in slot order (consecutive threads store
// consecutive rows of each digit's run) during the next tile's prefix.
//
// Tile q (the CTA's running tile count, continued across ranges so a
// persistent CTA never re-initialises its barriers) uses buffer q % NB with
// barrier mbar[q % NB] at phase parity (q / NB) & 1, and counters and deltas
// q & 1.

// Waits for tile q and ranks its rows on cnt[q & 1].
template <int THREADS, bool FULL, class Dig, int NB>
__device__ __forceinline__ void tile_load_rank(const Row *__restrict__ in, const TileGeo &g, uint32_t q, Dig dop,
                                               PartSmem<THREADS, NB> &sm, uint64_t *mbar, uint2 (&v)[PART_ITEMS],
                                               uint32_t (&rank)[PART_ITEMS], unsigned *err) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t wbase = (uint32_t)w * 32 * PART_ITEMS;
    const uint32_t cnt = g.cnt;
    const int b = q % NB;
    if (!mbar_wait(&mbar[b], (q / NB) & 1, SPIN_LIMIT * 16)) atomicCAS(err, 0u, (unsigned)TBG_ERR_TIMEOUT);
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
    uint32_t *c = sm.cnt[q & 1];
    const bool dup = warp_has_dups(dop(v[0].x), FULL || wbase + lane < cnt);
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        const bool valid = FULL || wbase + i * 32 + lane < cnt;
        rank[i] = rank_warp(c, valid ? dop(v[i].x) : 0, valid, dup);
    }
}

// Warp 0: digit counts of tile q -> tile offsets (in place), deltas and
// cursors; clears the counters of tile q + 1.  The tile lays the digits out
// in natural order, so neighbouring runs belong to neighbouring digits and a
// warp of the write-out that spans a run boundary reads its deltas from
// different banks.  Lane l owns the 8 consecutive digits [8l, 8l + 8) and
// moves them with 16-byte accesses (conflict-free).  Every counter of all
// SCATTER_FMAX digits is kept at zero outside the F digits in use, so those
// add nothing.
template <int THREADS, int NB>
__device__ __forceinline__ void tile_scan(uint32_t q, int F, PartSmem<THREADS, NB> &sm) {
    (void)F;
    const int lane = threadIdx.x & 31;
    constexpr int PER = SCATTER_FMAX / 32;
    static_assert(PER == 8, "two 16-byte words of counters per lane");
    uint4 *c4 = reinterpret_cast<uint4 *>(sm.cnt[q & 1]) + 2 * lane;
    uint4 *d4 = reinterpret_cast<uint4 *>(sm.delta[q & 1]) + 2 * lane;
    uint4 *u4 = reinterpret_cast<uint4 *>(sm.cursor) + 2 * lane;
    uint4 *n4 = reinterpret_cast<uint4 *>(sm.cnt[(q + 1) & 1]) + 2 * lane;
    const uint4 ca = c4[0], cb = c4[1];
    const uint32_t x[PER] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < PER; i++) sum += x[i];
    if (PART_BULK) sum += PER;  // the lane's digits take one spare slot each
    uint32_t inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    uint32_t run = inc - sum;
    const uint4 ua = u4[0], ub = u4[1];
    uint32_t cur[PER] = {ua.x, ua.y, ua.z, ua.w, ub.x, ub.y, ub.z, ub.w};
    uint32_t off[PER], dl[PER];
#pragma unroll
    for (int i = 0; i < PER; i++) {
        if (PART_BULK) {
            // one spare slot per digit: the run starts in its destination's 16-byte phase
            off[i] = run + ((run ^ cur[i]) & 1u);
            run += x[i] + 1;
        } else {
            off[i] = run;
            run += x[i];
        }
        dl[i] = cur[i] - off[i];
        cur[i] += x[i];
    }
    if (PART_BULK) {
        uint4 *s4 = reinterpret_cast<uint4 *>(sm.rstart[q & 1]) + 2 * lane;
        uint4 *r4 = reinterpret_cast<uint4 *>(sm.rcount[q & 1]) + 2 * lane;
        s4[0] = make_uint4(off[0], off[1], off[2], off[3]);
        s4[1] = make_uint4(off[4], off[5], off[6], off[7]);
        r4[0] = make_uint4(x[0], x[1], x[2], x[3]);
        r4[1] = make_uint4(x[4], x[5], x[6], x[7]);
    }
    c4[0] = make_uint4(off[0], off[1], off[2], off[3]);
    c4[1] = make_uint4(off[4], off[5], off[6], off[7]);
    d4[0] = make_uint4(dl[0], dl[1], dl[2], dl[3]);
    d4[1] = make_uint4(dl[4], dl[5], dl[6], dl[7]);
    u4[0] = make_uint4(cur[0], cur[1], cur[2], cur[3]);
    u4[1] = make_uint4(cur[4], cur[5], cur[6], cur[7]);
    n4[0] = make_uint4(0, 0, 0, 0);
    n4[1] = make_uint4(0, 0, 0, 0);
}

// Stages tile q's rows digit-sorted into its own buffer.
template <int THREADS, bool FULL, class Dig, int NB>
__device__ __forceinline__ void tile_stage(const TileGeo &g, uint32_t q, Dig dop, PartSmem<THREADS, NB> &sm,
                                           const uint2 (&v)[PART_ITEMS], const uint32_t (&rank)[PART_ITEMS]) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t wbase = (uint32_t)w * 32 * PART_ITEMS;
    const uint32_t *c = sm.cnt[q & 1];
    Row *buf = sm.buf[q % NB];
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        if (FULL || wbase + i * 32 + lane < g.cnt) {
            const uint32_t j = c[dop(v[i].x)] + rank[i];
            buf[j] = Row{v[i].x, v[i].y};
        }
    }
    if (PART_BULK) fence_proxy_async_smem();  // the staged rows become visible to the bulk stores
}

// Writes staged tile q (cnt rows) to out, by threads [t0, THREADS).
template <int THREADS, class Dig, int NB>
__device__ __forceinline__ void tile_write(uint32_t q, uint32_t cnt, uint2 *__restrict__ out, uint32_t out_n,
                                           Dig dop, PartSmem<THREADS, NB> &sm, int t0, unsigned *err) {
    if ((int)threadIdx.x < t0) return;
    if (PART_BULK) {
        (void)cnt;
        (void)dop;
        const Row *buf = sm.buf[q % NB];
        const uint32_t *dl = sm.delta[q & 1];
        const uint32_t *rs = sm.rstart[q & 1], *rc = sm.rcount[q & 1];
        const bool aligned = (reinterpret_cast<uintptr_t>(out) & 15) == 0;
        bool issued = false;
        for (int d = (int)threadIdx.x - t0; d < SCATTER_FMAX; d += THREADS - t0) {
            uint32_t n = rc[d];
            if (!n) continue;
            uint32_t s = rs[d];
            uint32_t gpos = dl[d] + s;
            if ((uint64_t)gpos + n > out_n) {
                atomicCAS(err, 0u, (unsigned)TBG_ERR_ARG);
                continue;
            }
            if (!aligned) {
                for (uint32_t r = 0; r < n; r++) out[gpos + r] = make_uint2(buf[s + r].key, buf[s + r].payload);
                continue;
            }
            if (gpos & 1) {  // head row up to the 16-byte boundary (the staged start shares the phase)
                out[gpos] = make_uint2(buf[s].key, buf[s].payload);
                s++;
                gpos++;
                n--;
            }
            const uint32_t body = n & ~1u;
            if (body) {
                bulk_s2g(out + gpos, buf + s, body * 8);
                issued = true;
            }
            if (n & 1) out[gpos + body] = make_uint2(buf[s + body].key, buf[s + body].payload);
        }
        if (issued) {
            bulk_commit();
            bulk_wait_read();  // the buffer is reloaded after the next barrier
        }
        return;
    }
    const Row *buf = sm.buf[q % NB];
    const uint32_t *dl = sm.delta[q & 1];
#pragma unroll 4
    for (uint32_t j = threadIdx.x - t0; j < cnt; j += THREADS - t0) {
        const Row x = buf[j];
        const uint32_t pos = dl[dop(x.key)] + j;
        if (pos < out_n) out[pos] = make_uint2(x.key, x.payload);
        else atomicCAS(err, 0u, (unsigned)TBG_ERR_ARG);
    }
}

__device__ __forceinline__ TileGeo range_tile(const Row *in, uint64_t lo, uint64_t hi, uint64_t n, int k,
                                             uint32_t T) {
    const uint64_t t = lo + (uint64_t)k * T;
    return tile_geo(in, t, (uint32_t)umin64(T, hi - t), n);
}

// Scatters rows [lo, hi) of `in` (in_n rows), digit by digit, to out[sm.cursor[d]...];
// the caller initialises sm.cursor[0..F) and synchronises.  Two barriers
// per tile; the bulk copies run NB - 1 tiles ahead.  `kseq` is the CTA's
// running tile count (see above), and the barriers mbar[0..NB) are
// initialised once by the caller.
template <int THREADS, class Dig, int NB>
__device__ void part_tiles(const Row *__restrict__ in, uint64_t lo, uint64_t hi, uint64_t in_n,
                           Row *__restrict__ out, uint32_t out_n, Dig dop, int F, PartSmem<THREADS, NB> &sm,
                           uint64_t *mbar, uint32_t &kseq, unsigned *err) {
    constexpr uint32_t T = THREADS * PART_ITEMS;
    uint2 *o = reinterpret_cast<uint2 *>(out);
    const int ntiles = (int)((hi - lo + T - 1) / T);
    for (int i = threadIdx.x; i < SCATTER_FMAX; i += THREADS) sm.cnt[kseq & 1][i] = 0;
    __syncthreads();
    if (ntiles == 0) return;
    if (threadIdx.x == 0)
        for (int i = 0; i < NB - 1 && i < ntiles; i++)
            issue_tile(in, range_tile(in, lo, hi, in_n, i, T), sm.buf[(kseq + i) % NB], &mbar[(kseq + i) % NB]);
    uint32_t prev_cnt = 0;
    for (int k = 0; k < ntiles; k++) {
        const uint32_t q = kseq + k;
        const TileGeo g = range_tile(in, lo, hi, in_n, k, T);
        uint2 v[PART_ITEMS];
        uint32_t rank[PART_ITEMS];
        if (g.cnt == T) tile_load_rank<THREADS, true, Dig>(in, g, q, dop, sm, mbar, v, rank, err);
        else tile_load_rank<THREADS, false, Dig>(in, g, q, dop, sm, mbar, v, rank, err);
        __syncthreads();
        if (threadIdx.x < 32) tile_scan<THREADS>(q, F, sm);
        else if (k > 0) tile_write<THREADS, Dig>(q - 1, prev_cnt, o, out_n, dop, sm, 32, err);
        __syncthreads();
        // tile q - 1's buffer is free: copy tile k + NB - 1 into it
        if (threadIdx.x == 0 && k + NB - 1 < ntiles)
            issue_tile(in, range_tile(in, lo, hi, in_n, k + NB - 1, T), sm.buf[(q + NB - 1) % NB],
                       &mbar[(q + NB - 1) % NB]);
        if (g.cnt == T) tile_stage<THREADS, true, Dig>(g, q, dop, sm, v, rank);
        else tile_stage<THREADS, false, Dig>(g, q, dop, sm, v, rank);
        // No barrier here: tile q + 1's load and ranking touch neither tile
        // q's buffer nor its counters, and the next iteration's first barrier
        // orders this staging before tile q's write-out and before the scan
        // that clears cnt[q & 1].
        if (TBG_TILE_END_BARRIER) __syncthreads();
        prev_cnt = g.cnt;
    }
    __syncthreads();  // the last tile is staged
    tile_write<THREADS, Dig>(kseq + ntiles - 1, prev_cnt, o, out_n, dop, sm, 0, err);
    if (PART_BULK) bulk_wait_all();  // this thread's bulk stores have landed
    __syncthreads();  // every buffer is free again
    kseq += ntiles;
}

// One range per CTA: initialises the barriers held in `sm`.
template <int THREADS, class Dig, int NB>
__device__ void part_range(const Row *__restrict__ in, uint64_t lo, uint64_t hi, uint64_t in_n,
                           Row *__restrict__ out, uint32_t out_n, Dig dop, int F, PartSmem<THREADS, NB> &sm,
                           unsigned *err) {
    if (threadIdx.x == 0) {
        for (int i = 0; i < NB; i++) mbar_init(&sm.mbar[i], 1);
        fence_mbar_init();
    }
    uint32_t kseq = 0;
    part_tiles<THREADS, Dig>(in, lo, hi, in_n, out, out_n, dop, F, sm, sm.mbar, kseq, err);
}

}  // namespace tbg
