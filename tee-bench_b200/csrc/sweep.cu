// One-sweep stable scatter with decoupled look-back, used by the LSD radix
// sort of the PSM path (every pass a full stable redistribution of the array).
#include "tbg_device.cuh"

namespace tbg {

// ---------------------------------------------------------------------------
// K3 stable scatter, one tile of SCATTER_TILE rows per CTA ticket.
//
//  1. rows are loaded warp-striped: warp w owns a contiguous sub-tile, so the
//     order (warp, item, lane) is the input order (needed for stability);
//  2. each row is ranked inside its warp (ballot-built peer masks) against a
//     warp-private digit counter; a column scan over warps and a scan over
//     digits give every row its slot in the digit-sorted tile;
//  3. the tile publishes its digit counts and looks back over predecessor
//     tiles of the same segment (decoupled look-back, epoch-tagged words,
//     bounded waits) for its global offsets;
//  4. rows are staged digit-sorted in shared memory and written out with
//     consecutive threads on consecutive addresses of each digit run, so the
//     stores coalesce (the software write-combining of radix_join.c:734-827).
// ---------------------------------------------------------------------------
constexpr uint64_t LB_AGG = 1ull << 62;
constexpr uint64_t LB_PRE = 2ull << 62;
constexpr uint64_t LB_VAL = (1ull << 54) - 1;

__device__ __forceinline__ uint64_t lb_pack(uint64_t flag, uint32_t epoch, uint64_t v) {
    return flag | ((uint64_t)(epoch & 0xFF) << 54) | (v & LB_VAL);
}

size_t scatter_smem_bytes() {
    constexpr int NW = SCATTER_THREADS / 32;
    return (size_t)SCATTER_TILE * sizeof(Row)              // stage
           + (size_t)NW * SCATTER_FMAX * sizeof(uint32_t)  // warp digit counters
           + (size_t)SCATTER_FMAX * sizeof(uint32_t)       // tile digit offsets
           + (size_t)SCATTER_FMAX * sizeof(uint64_t)       // global digit positions
           + (size_t)SCATTER_TILE;                         // staged digits
}

__global__ void __launch_bounds__(SCATTER_THREADS) k_scatter(ScatterArgs a) {
    constexpr int NW = SCATTER_THREADS / 32;
    constexpr int T = SCATTER_TILE;
    extern __shared__ __align__(16) unsigned char smem[];
    Row *stage = reinterpret_cast<Row *>(smem);
    uint32_t *wcnt = reinterpret_cast<uint32_t *>(stage + T);
    uint32_t *toff = wcnt + NW * SCATTER_FMAX;
    uint64_t *gpos = reinterpret_cast<uint64_t *>(toff + SCATTER_FMAX);
    uint8_t *dig = reinterpret_cast<uint8_t *>(gpos + SCATTER_FMAX);
    __shared__ uint64_t s_row0, s_rowend;
    __shared__ uint32_t s_tile, s_seg;
    __shared__ int s_first, s_valid, s_abort;
    __shared__ uint64_t scan_scratch[NW + 1];

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int F = 1 << a.dbits;
    const uint32_t dmask = (uint32_t)F - 1;

    if (tid == 0) {
        uint32_t t = atomicAdd(a.tile_ctr, 1u);
        s_tile = t;
        s_abort = 0;
        if (a.seg_start == nullptr) {
            uint64_t ntiles = (a.flat_n + T - 1) / T;
            s_valid = t < ntiles;
            s_seg = 0;
            s_first = (t == 0);
            s_row0 = (uint64_t)t * T;
            s_rowend = umin64(a.flat_n, s_row0 + T);
        } else {
            uint32_t total = a.seg_tile[a.nseg];
            s_valid = t < total;
            if (t < total) {
                // last segment whose first tile is <= t (empty segments share starts)
                uint32_t lo = 0, hi = a.nseg;  // invariant: seg_tile[lo] <= t < seg_tile[hi]
                while (hi - lo > 1) {
                    uint32_t mid = (lo + hi) >> 1;
                    if (a.seg_tile[mid] <= t) lo = mid;
                    else hi = mid;
                }
                uint32_t j = t - a.seg_tile[lo];
                s_seg = lo;
                s_first = (j == 0);
                s_row0 = a.seg_start[lo] + (uint64_t)j * T;
                s_rowend = umin64(a.seg_start[lo + 1], s_row0 + T);
            }
        }
    }
    for (int i = tid; i < NW * F; i += SCATTER_THREADS) wcnt[(i / F) * SCATTER_FMAX + (i % F)] = 0;
    __syncthreads();
    if (!s_valid) return;
    const uint64_t row0 = s_row0, rowend = s_rowend;

    // 1. load (warp-striped within a per-warp contiguous sub-tile)
    uint32_t key[SCATTER_ITEMS], pay[SCATTER_ITEMS], d[SCATTER_ITEMS], rank[SCATTER_ITEMS];
    const uint64_t wbase = row0 + (uint64_t)w * 32 * SCATTER_ITEMS;
#pragma unroll
    for (int i = 0; i < SCATTER_ITEMS; i++) {
        uint64_t r = wbase + (uint64_t)i * 32 + lane;
        if (r < rowend) {
            uint2 x = ldg_stream(reinterpret_cast<const uint2 *>(a.in) + r);
            key[i] = x.x;
            pay[i] = x.y;
            d[i] = (radix_f(a.rf, x.x) >> a.dshift) & dmask;
        } else {
            key[i] = pay[i] = 0;
            d[i] = SCATTER_FMAX;  // sentinel: not a row
        }
    }
    // 2. stable rank within the warp
    uint32_t *myc = wcnt + w * SCATTER_FMAX;
#pragma unroll
    for (int i = 0; i < SCATTER_ITEMS; i++) {
        unsigned peers = warp_peers9(d[i]);  // d < 512: digit or the sentinel
        unsigned lt = peers & lanemask_lt();
        uint32_t c = d[i] < SCATTER_FMAX ? myc[d[i]] : 0;
        rank[i] = c + __popc(lt);
        __syncwarp();
        if (d[i] < SCATTER_FMAX && lt == 0) myc[d[i]] = c + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // column scan over warps (thread = digit), then scan over digits
    uint32_t tot = 0;
    if (tid < F) {
        for (int ww = 0; ww < NW; ww++) {
            uint32_t c = wcnt[ww * SCATTER_FMAX + tid];
            wcnt[ww * SCATTER_FMAX + tid] = tot;
            tot += c;
        }
    }
    uint64_t dummy;
    uint32_t ex = (uint32_t)block_excl_scan<SCATTER_THREADS>(tid < F ? tot : 0, &dummy, scan_scratch);
    if (tid < F) toff[tid] = ex;

    // 3. decoupled look-back within the segment
    if (tid < F) {
        uint64_t *st = a.status + (uint64_t)s_tile * F;
        uint64_t prefix = 0;
        if (s_first) {
            st_relaxed(st + tid, lb_pack(LB_PRE, a.epoch, tot));
        } else {
            st_relaxed(st + tid, lb_pack(LB_AGG, a.epoch, tot));
            int64_t p = (int64_t)s_tile - 1;
            while (p >= 0) {
                const uint64_t *src = a.status + (uint64_t)p * F + tid;
                uint64_t v = ld_relaxed(src);
                unsigned spins = 0;
                while (((v >> 62) == 0) || (((v >> 54) & 0xFF) != (a.epoch & 0xFF))) {
                    if (++spins > SPIN_LIMIT) {
                        atomicCAS(a.err, 0u, (unsigned)TBG_ERR_TIMEOUT);
                        s_abort = 1;
                        v = LB_PRE;  // stop looking back
                        break;
                    }
                    if (spins > 16) __nanosleep(64);
                    v = ld_relaxed(src);
                }
                prefix += v & LB_VAL;
                if ((v >> 62) == 2) break;
                p--;
            }
            st_relaxed(st + tid, lb_pack(LB_PRE, a.epoch, prefix + tot));
        }
        gpos[tid] = a.bases[((uint64_t)s_seg << a.dbits) | tid] + prefix;
    }
    __syncthreads();

    // 4. stage digit-sorted, then coalesced write-out
#pragma unroll
    for (int i = 0; i < SCATTER_ITEMS; i++) {
        if (d[i] < SCATTER_FMAX) {
            uint32_t pos = toff[d[i]] + wcnt[w * SCATTER_FMAX + d[i]] + rank[i];
            stage[pos] = Row{key[i], pay[i]};
            dig[pos] = (uint8_t)d[i];
        }
    }
    __syncthreads();
    if (s_abort) return;
    const int cnt = (int)(rowend - row0);
    for (int j = tid; j < cnt; j += SCATTER_THREADS) {
        uint32_t dd = dig[j];
        uint64_t pos = gpos[dd] + (uint64_t)(j - (int)toff[dd]);
        if (pos < a.out_n) {
            reinterpret_cast<uint2 *>(a.out)[pos] = make_uint2(stage[j].key, stage[j].payload);
        } else {
            atomicCAS(a.err, 0u, (unsigned)TBG_ERR_TIMEOUT);
        }
    }
}

cudaError_t launch_scatter(const ScatterArgs &a, uint64_t max_tiles, cudaStream_t st) {
    if (max_tiles == 0) return cudaSuccess;
    static bool attr_done = false;
    const size_t smem = scatter_smem_bytes();
    if (!attr_done) {
        cudaError_t e = smem_limit((const void *)k_scatter, smem);
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    k_scatter<<<(unsigned)max_tiles, SCATTER_THREADS, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
