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

}  // namespace tbg
