// One stable LSD radix-sort pass for the PSM sort (7-, 8- or 9-bit digit at
// `shift` of key - sub, sub being the relation's smallest key),
// built like the partitioning passes: CTA c owns chunk c of the input; its
// digit cursors are base[d] + (rows of digit d in chunks before c), from the
// per-chunk histograms (k_hist_chunks) and their column prefix (k_colscan),
// so no CTA waits for another.  Tiles of 512 threads x 8 rows arrive by TMA
// bulk copy; a row's rank within its tile counts the same-digit rows before
// it in tile order (per-(digit, warp) counters advanced row slot by row slot,
// ballot-built peer masks inside a slot); the tile is staged digit-sorted and
// written out in slot order, so stores coalesce.  Chunk order, tile order
// and tile-internal order all follow the input, so the pass is stable.
#include "part_dev.cuh"

namespace tbg {

constexpr int SORT_THREADS = 512;

template <int NB>  // digits per pass: 128, 256 or 512
struct SortSmem {
    static constexpr int NW = SORT_THREADS / 32;
    static constexpr int T = SORT_THREADS * PART_ITEMS;
    Row buf[2][T + 2];               // input tile (bulk copy), then the same tile digit-sorted
    uint16_t cnt[2][NB * NW];        // [warp][digit] counts, then offsets, double-buffered
    uint32_t delta[NB];              // output row - tile slot, per digit
    uint32_t cursor[NB];             // next output row of each digit
    uint64_t scan[NW + 1];
    uint64_t mbar[2];
};

// Lanes of the warp whose value d (< 2^BITS) equals this lane's, from one
// ballot per bit (cost independent of how many values the warp holds).
template <int BITS>
__device__ __forceinline__ unsigned warp_peers_bits(uint32_t d) {
    unsigned peers = 0xffffffffu;
#pragma unroll
    for (int k = 0; k < BITS; k++) {
        const bool bit = (d >> k) & 1;
        const unsigned b = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? b : ~b;
    }
    return peers;
}

template <int NB, int DB, bool FULL>
__device__ __forceinline__ void sort_tile(const Row *__restrict__ in, const TileGeo &g, uint32_t k, bool has_next,
                                          const TileGeo &gnext, uint2 *__restrict__ out, uint32_t out_n,
                                          uint32_t shift, uint32_t sub, SortSmem<NB> &sm, unsigned *err) {
    constexpr int NW = SortSmem<NB>::NW, C = NB * NW / SORT_THREADS, TPD = NW / C;  // TPD threads per digit
    static_assert(C >= 1 && NW % C == 0 && (TPD & (TPD - 1)) == 0 && TPD <= 32,
                  "a thread's counters belong to one digit; a digit's threads share a warp");
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int b = k & 1;
    const uint32_t wbase = (uint32_t)w * 32 * PART_ITEMS;
    const uint32_t cnt = g.cnt;
    uint16_t *c = sm.cnt[b];
    if (!mbar_wait(&sm.mbar[b], (k >> 1) & 1, SPIN_LIMIT * 16)) atomicCAS(err, 0u, (unsigned)TBG_ERR_TIMEOUT);
    uint2 v[PART_ITEMS];
    uint32_t rank[PART_ITEMS];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        const uint32_t r = wbase + i * 32 + lane;
        const bool valid = FULL || r < cnt;
        if (valid) {
            if (r >= g.a_lo && r < g.a_hi) {
                const Row x = sm.buf[b][r + g.off];
                v[i] = make_uint2(x.key, x.payload);
            } else {
                v[i] = reinterpret_cast<const uint2 *>(in)[g.t + r];
            }
        }
        const uint32_t d = valid ? ((v[i].x - sub) >> shift) & (NB - 1) : NB;  // NB: the no-row sentinel
        // a full tile has no sentinel, so its digits need one ballot less
        const unsigned peers = FULL ? warp_peers_bits<DB>(d) : warp_peers_bits<DB + 1>(d);
        uint32_t base = 0;
        if (valid) base = c[w * NB + d];  // warp-major: lanes with different digits hit different banks
        __syncwarp();
        if (valid && (peers & lt) == 0) c[w * NB + d] = (uint16_t)(base + __popc(peers));
        __syncwarp();
        rank[i] = base + __popc(peers & lt);
    }
    for (int i = tid; i < NB * NW; i += SORT_THREADS) sm.cnt[b ^ 1][i] = 0;
    __syncthreads();
    // the other buffer is free (its tile was written out before this barrier)
    if (tid == 0 && has_next) issue_tile(in, gnext, sm.buf[b ^ 1], &sm.mbar[b ^ 1]);
    // exclusive scan over (digit, warp), digit-major; thread t owns the C
    // counters of digit t / TPD for warps (t % TPD) * C ...
    const int dgt = tid / TPD, w0 = (tid % TPD) * C;
    uint32_t sum = 0;
#pragma unroll
    for (int q = 0; q < C; q++) sum += c[(w0 + q) * NB + dgt];
    uint64_t dummy;
    uint32_t run = (uint32_t)block_excl_scan<SORT_THREADS, false>(sum, &dummy, sm.scan);
    const uint32_t dstart = __shfl_sync(0xffffffffu, run, lane & ~(TPD - 1));  // the digit's first offset
    uint32_t dtotal = sum;                                                     // the digit's rows in the tile
#pragma unroll
    for (int o = 1; o < TPD; o <<= 1) dtotal += __shfl_xor_sync(0xffffffffu, dtotal, o);
#pragma unroll
    for (int q = 0; q < C; q++) {
        const uint32_t x = c[(w0 + q) * NB + dgt];
        c[(w0 + q) * NB + dgt] = (uint16_t)run;
        run += x;
    }
    if (tid % TPD == 0) {
        sm.delta[dgt] = sm.cursor[dgt] - dstart;
        sm.cursor[dgt] += dtotal;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PART_ITEMS; i++) {
        if (FULL || wbase + i * 32 + lane < cnt) {
            const uint32_t d = ((v[i].x - sub) >> shift) & (NB - 1);
            sm.buf[b][c[w * NB + d] + rank[i]] = Row{v[i].x, v[i].y};
        }
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < PART_ITEMS; kk++) {
        const uint32_t j = kk * SORT_THREADS + tid;
        if (FULL || j < cnt) {
            const Row x = sm.buf[b][j];
            const uint32_t pos = sm.delta[((x.key - sub) >> shift) & (NB - 1)] + j;
            if (pos < out_n) out[pos] = make_uint2(x.key, x.payload);
            else atomicCAS(err, 0u, (unsigned)TBG_ERR_ARG);
        }
    }
}

// pre: per-chunk digit prefixes [G][NB]; totals: digit totals [NB].
template <int DB>
__global__ void __launch_bounds__(SORT_THREADS, 2) k_sort_pass(const Row *__restrict__ in, Row *__restrict__ out,
                                                               uint64_t n, uint64_t chunk,
                                                               const uint32_t *__restrict__ pre,
                                                               const uint32_t *__restrict__ totals, uint32_t shift,
                                                               uint32_t sub, unsigned *err) {
    constexpr int NB = 1 << DB;
    static_assert(NB <= SORT_THREADS, "one digit total per thread");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<NB> &sm = *reinterpret_cast<SortSmem<NB> *>(smem_raw);
    constexpr int T = SortSmem<NB>::T;
    const int c = blockIdx.x, tid = threadIdx.x;
    // digit bases: exclusive scan of the totals, plus this chunk's prefix
    const uint32_t tot = tid < NB ? totals[tid] : 0;
    uint64_t dummy;
    const uint32_t bse = (uint32_t)block_excl_scan<SORT_THREADS>(tot, &dummy, sm.scan);
    if (tid < NB) sm.cursor[tid] = bse + pre[(uint64_t)c * NB + tid];
    for (int i = tid; i < NB * SortSmem<NB>::NW; i += SORT_THREADS) sm.cnt[0][i] = 0;
    if (tid == 0) {
        mbar_init(&sm.mbar[0], 1);
        mbar_init(&sm.mbar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    const uint64_t lo = (uint64_t)c * chunk;
    const uint64_t hi = umin64(n, lo + chunk);
    if (lo >= hi) return;
    const int ntiles = (int)((hi - lo + T - 1) / T);
    uint2 *o = reinterpret_cast<uint2 *>(out);
    TileGeo g = tile_geo(in, lo, (uint32_t)umin64(T, hi - lo), n);
    if (tid == 0) issue_tile(in, g, sm.buf[0], &sm.mbar[0]);
    for (int k = 0; k < ntiles; k++) {
        const uint64_t t1 = g.t + T;
        const bool more = k + 1 < ntiles;
        const TileGeo gn = more ? tile_geo(in, t1, (uint32_t)umin64(T, hi - t1), n) : g;
        if (g.cnt == T) sort_tile<NB, DB, true>(in, g, (uint32_t)k, more, gn, o, (uint32_t)n, shift, sub, sm, err);
        else sort_tile<NB, DB, false>(in, g, (uint32_t)k, more, gn, o, (uint32_t)n, shift, sub, sm, err);
        g = gn;
    }
}

// digit_bits: 7, 8 or 9
cudaError_t launch_sort_pass(const Row *in, Row *out, uint64_t n, uint64_t chunk, int G, const uint32_t *pre,
                             const uint32_t *totals, uint32_t shift, uint32_t sub, int digit_bits, unsigned *err,
                             cudaStream_t st) {
    cudaError_t e;
    if (digit_bits == 7) {
        const size_t smem = sizeof(SortSmem<128>);
        if ((e = smem_limit((const void *)k_sort_pass<7>, smem)) !=
            cudaSuccess)
            return e;
        k_sort_pass<7><<<G, SORT_THREADS, smem, st>>>(in, out, n, chunk, pre, totals, shift, sub, err);
    } else if (digit_bits == 9) {
        const size_t smem = sizeof(SortSmem<512>);
        if ((e = smem_limit((const void *)k_sort_pass<9>, smem)) !=
            cudaSuccess)
            return e;
        k_sort_pass<9><<<G, SORT_THREADS, smem, st>>>(in, out, n, chunk, pre, totals, shift, sub, err);
    } else {
        const size_t smem = sizeof(SortSmem<256>);
        if ((e = smem_limit((const void *)k_sort_pass<8>, smem)) !=
            cudaSuccess)
            return e;
        k_sort_pass<8><<<G, SORT_THREADS, smem, st>>>(in, out, n, chunk, pre, totals, shift, sub, err);
    }
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// PSM bucket sort.  After the partitioning passes by the top bits of
// key - sub (final partition f = (key - sub) >> lowbits), bucket b holds
// rows [base[b], base[b + 1]) whose keys agree above bit `lowbits`; sorting
// every bucket by the low `lowbits` bits leaves the relation sorted.  One CTA
// per SM walks the buckets.  Per bucket:
//   1. the bucket's histogram over 2^lowbits bins in shared memory (the one
//      read from DRAM) and its exclusive scan;
//   2. one re-read of the bucket (from L2) ranks every row by an atomic on
//      its bin's running offset: a row whose sorted position is below the
//      stage's capacity (27K rows) goes to the stage in shared memory, the
//      others (the bucket's last bins; all but the first 27K rows of a heavy
//      key's bucket) straight to their place in the output; then the stage
//      is written out with coalesced stores.
// Two reads per row.  Before, the bins were cut into parts that each fit
// the stage, with one re-read of the bucket per part (a 32K-row bucket: two
// parts, three reads per row): 8.4 ms for 2^30 rows against 7.3 ms now (ncu
// launch lists).  Staging row indices instead (4 bytes, one part per bucket, the rows
// gathered back from L2 at the write-out) measured 12.8 ms: the gather's
// scattered 8-byte reads cost more L2 sectors than a part's stream.
// Rows of equal keys land in any order, which the merge does not need (a
// join's rows are a multiset).
// ---------------------------------------------------------------------------
// Threads, CTAs per SM and shared memory of the bucket sort (build options
// for A/B timing; the CTAs of one SM hold the buckets in flight in L2).
#ifndef TBG_BSORT_THREADS
#define TBG_BSORT_THREADS 1024
#endif
#ifndef TBG_BSORT_CTAS
#define TBG_BSORT_CTAS 1
#endif
constexpr int BSORT_THREADS = TBG_BSORT_THREADS;
constexpr int BSORT_CTAS = TBG_BSORT_CTAS;
#ifndef TBG_BSORT_GROUPS
#define TBG_BSORT_GROUPS 4
#endif
#ifndef TBG_BSORT_PAIRS
#define TBG_BSORT_PAIRS 2
#endif
constexpr int BSORT_PAIRS = TBG_BSORT_PAIRS;  // 16-byte row pairs per thread per round
constexpr size_t BSORT_SMEM = (BSORT_CTAS == 1 ? 226 : 112) * 1024;  // stage + bins

__device__ __forceinline__ uint32_t bsort_bin(uint32_t key, uint32_t sub, uint32_t mask) { return (key - sub) & mask; }

// A bucket is sorted by a group of BSORT_THREADS / G threads with its own
// bins and stage (G groups per CTA work on G buckets at a time, each at its
// own pace): small buckets (R's 4K rows at 2^27 keys) take G = 4, which keeps
// four buckets' phases overlapping where one group would wait on its
// barriers; large buckets take G = 1 and the whole stage.  The scan of the
// bins reads them as 16-byte words (strided 4-byte reads of a thread's run
// of bins conflicted 4-way at G = 1 and 16-way at G = 4): with it PSM's R
// sort (2^27 rows) took 0.36 ms less at G = 4 than at G = 1.
template <int G>
__device__ __forceinline__ void group_bar(int g) {
    if (G == 1) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(BSORT_THREADS / G) : "memory");
}

// Exclusive scan of one value per thread over a group (scratch: a word per
// warp of the group); every thread of the group calls it.
template <int G>
__device__ __forceinline__ uint32_t group_excl_scan(uint32_t v, uint32_t *total, uint32_t *scratch, int g) {
    constexpr int GT = BSORT_THREADS / G, NW = GT / 32;
    const int lane = threadIdx.x & 31, w = (threadIdx.x % GT) >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scratch[w] = x;
    group_bar<G>(g);
    if (w == 0) {
        uint32_t t = lane < NW ? scratch[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < NW) scratch[lane] = t;
    }
    group_bar<G>(g);
    const uint32_t before = w ? scratch[w - 1] : 0;
    *total = scratch[NW - 1];
    group_bar<G>(g);  // scratch is reused by the next scan
    return before + x - v;
}

// Calls fn(row, index, valid, dup) for every row of the bucket (index: its
// place in the bucket), in group-uniform rounds (so fn may use warp
// collectives); `dup` says the warp saw repeated bins in the round's first
// row slot (skew).  The next round's loads are issued before the current
// round is handed to fn.  The bucket's edge rows (outside the 16-byte
// aligned body) come in a last round of the group's first warp.
template <int GT, class Fn>
__device__ __forceinline__ void bsort_stream(const Row *src, uint32_t len, uint32_t sub, uint32_t mask, int gtid,
                                             Fn fn) {
    const uint32_t head = (reinterpret_cast<uintptr_t>(src) & 15) ? 1u : 0u;
    const uint32_t npairs = (len - head) / 2;
    const bool tail = ((len - head) & 1) != 0;
    const uint4 *v = reinterpret_cast<const uint4 *>(src + head);
    constexpr uint32_t ROUND = BSORT_PAIRS * GT;
    uint4 nx[BSORT_PAIRS];
    auto load = [&](uint32_t p0) {
#pragma unroll
        for (int u = 0; u < BSORT_PAIRS; u++) {
            const uint32_t p = p0 + u * GT + gtid;
            nx[u] = p < npairs ? __ldcg(v + p) : make_uint4(0, 0, 0, 0);
        }
    };
    load(0);
    for (uint32_t p0 = 0; p0 < npairs; p0 += ROUND) {
        uint4 x[BSORT_PAIRS];
#pragma unroll
        for (int u = 0; u < BSORT_PAIRS; u++) x[u] = nx[u];
        load(p0 + ROUND);
        const bool dup = warp_has_dups(bsort_bin(x[0].x, sub, mask), p0 + gtid < npairs);
#pragma unroll
        for (int u = 0; u < BSORT_PAIRS; u++) {
            const uint32_t p = p0 + u * GT + gtid;
            const bool ok = p < npairs;
            fn(Row{x[u].x, x[u].y}, head + 2 * p, ok, dup);
            fn(Row{x[u].z, x[u].w}, head + 2 * p + 1, ok, dup);
        }
    }
    if (gtid < 32) {
        const int lane = gtid;
        const bool ok = (lane == 0 && head) || (lane == 1 && tail);
        const uint32_t i = lane == 0 ? 0u : len - 1;
        const Row r = ok ? src[i] : Row{0, 0};
        fn(r, i, ok, false);
    }
}

// Shared memory of one group: its bins, then its stage.
template <int G>
__host__ __device__ constexpr size_t bsort_group_bytes() {
    return (BSORT_SMEM / G) & ~(size_t)15;
}

template <int G>
__global__ void __launch_bounds__(BSORT_THREADS, BSORT_CTAS)
    k_bucket_sort(const Row *__restrict__ in, Row *__restrict__ out, const uint64_t *__restrict__ base, uint32_t nb,
                  uint32_t sub, int lowbits) {
    extern __shared__ __align__(16) unsigned char bsmem[];
    constexpr int GT = BSORT_THREADS / G;
    const int g = threadIdx.x / GT, gtid = threadIdx.x % GT;
    const uint32_t bins = 1u << lowbits, mask = bins - 1;
    unsigned char *gm = bsmem + g * bsort_group_bytes<G>();
    uint32_t *h = reinterpret_cast<uint32_t *>(gm);          // bins
    uint2 *stage = reinterpret_cast<uint2 *>(gm + 4 * bins);  // cap rows
    const uint32_t cap = (uint32_t)((bsort_group_bytes<G>() - 4 * (size_t)bins) / 8);
    __shared__ uint32_t scratch_all[G][GT / 32];
    uint32_t *scratch = scratch_all[g];
    const uint32_t per = (bins + GT - 1) / GT;
    for (uint32_t b = blockIdx.x * G + g; b < nb; b += gridDim.x * G) {
        const uint64_t lo = base[b], hi = base[b + 1];  // the same for every thread of the group
        if (hi <= lo) continue;
        const Row *src = in + lo;
        uint2 *dst = reinterpret_cast<uint2 *>(out + lo);
        const uint32_t len = (uint32_t)(hi - lo);  // a bucket holds < 2^32 rows
        if (len == 1) {
            if (gtid == 0) dst[0] = make_uint2(src[0].key, src[0].payload);
            continue;
        }
        for (uint32_t q = gtid; q < bins; q += GT) h[q] = 0;
        group_bar<G>(g);
        // 1. histogram and exclusive scan
        bsort_stream<GT>(src, len, sub, mask, gtid, [&](Row r, uint32_t, bool ok, bool dup) {
            hist_add_warp(h, ok ? bsort_bin(r.key, sub, mask) : 0u, ok, dup);
        });
        group_bar<G>(g);
        if (per % 4 == 0) {
            // a thread's bins as 16-byte words: a warp reads consecutive
            // words (one thread's 4 bins each at 1024 threads: no conflicts)
            uint4 *h4 = reinterpret_cast<uint4 *>(h) + gtid * (per / 4);
            uint32_t sum = 0;
            for (uint32_t q = 0; q < per / 4; q++) {
                const uint4 c = h4[q];
                sum += c.x + c.y + c.z + c.w;
            }
            uint32_t tot;
            uint32_t run = group_excl_scan<G>(sum, &tot, scratch, g);
            for (uint32_t q = 0; q < per / 4; q++) {
                const uint4 c = h4[q];
                uint4 o;
                o.x = run;
                o.y = o.x + c.x;
                o.z = o.y + c.y;
                o.w = o.z + c.z;
                run = o.w + c.w;
                h4[q] = o;
            }
        } else {
            const uint32_t b0 = min(bins, gtid * per), b1 = min(bins, b0 + per);
            uint32_t sum = 0;
            for (uint32_t q = b0; q < b1; q++) sum += h[q];
            uint32_t tot;
            uint32_t run = group_excl_scan<G>(sum, &tot, scratch, g);
            for (uint32_t q = b0; q < b1; q++) {
                const uint32_t c = h[q];
                h[q] = run;
                run += c;
            }
        }
        group_bar<G>(g);
        // 2. one re-read of the bucket (from L2) ranks every row: the rows
        // whose sorted position is below the stage's capacity go to the
        // stage, the others (the bucket's last bins) straight to their place
        // in the output; then the stage is written out with coalesced stores
        const uint32_t nstage = min(len, cap);
        bsort_stream<GT>(src, len, sub, mask, gtid, [&](Row r, uint32_t, bool ok, bool dup) {
            const uint32_t pos = rank_warp(h, ok ? bsort_bin(r.key, sub, mask) : 0u, ok, dup);
            if (ok) {
                if (pos < nstage) stage[pos] = make_uint2(r.key, r.payload);
                else dst[pos] = make_uint2(r.key, r.payload);
            }
        });
        group_bar<G>(g);
        for (uint32_t q = gtid; q < nstage; q += GT) dst[q] = stage[q];
        group_bar<G>(g);  // the bins and the stage are reused by the next bucket
    }
}

size_t bucket_sort_smem(int lowbits) {
    (void)lowbits;  // the stage takes what the bins leave
    return BSORT_SMEM;
}

cudaError_t launch_bucket_sort(const Row *in, Row *out, const uint64_t *base, uint32_t nb, uint64_t n, uint32_t sub,
                               int lowbits, int nsm, cudaStream_t st) {
    if (!nb) return cudaSuccess;
    if (lowbits > 14) return cudaErrorInvalidValue;  // the bins must leave room for a stage
    const size_t smem = bucket_sort_smem(lowbits);
    // four groups when their stages hold an average bucket
    constexpr int G4 = BSORT_THREADS >= 1024 ? TBG_BSORT_GROUPS : 1;
    const size_t bins_bytes = (size_t)4 << lowbits;
    const bool small = G4 > 1 && bins_bytes * 2 <= bsort_group_bytes<G4>() &&
                       n / nb <= (bsort_group_bytes<G4>() - bins_bytes) / 8;
    auto kern = small ? k_bucket_sort<G4> : k_bucket_sort<1>;
    cudaError_t e = smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    // one CTA per SM: the buckets in flight (each read from DRAM once and
    // re-read once) stay within L2
    const int G = small ? G4 : 1;
    const unsigned g = (unsigned)std::min<uint64_t>((nb + G - 1) / G, (uint64_t)nsm * BSORT_CTAS);
    kern<<<g, BSORT_THREADS, smem, st>>>(in, out, base, nb, sub, lowbits);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
