// Radix partitioning for sm_100a: histogram, planner, and a stable one-sweep
// scatter with decoupled look-back.
//
// Replaces the reference's partitioning passes (Joins/radix_join.c:630-703
// parallel_radix_partition, :525-562 radix_cluster, :573-619
// serial_radix_partition, the SWWC variant :734-827) and the task queues that
// feed them (Include/task_queue.h).  One histogram read gives the sizes of all
// final partitions of both passes; each pass is then one read and one write.
#include "tbg_device.cuh"

namespace tbg {

// ---------------------------------------------------------------------------
// K1 histogram of the final partition index f over all rows.
// Per-CTA shared-memory histogram; lanes holding the same bin are merged with
// __match_any_sync so a hot key costs one shared atomic per warp, not 32.
// ---------------------------------------------------------------------------
template <bool AGG>
__device__ __forceinline__ void hist_add(uint32_t *h, uint32_t f) {
    if (AGG) {
        unsigned mask = __activemask();
        unsigned peers = __match_any_sync(mask, f);
        if ((peers & lanemask_lt()) == 0) atomicAdd(&h[f], (uint32_t)__popc(peers));
    } else {
        atomicAdd(&h[f], 1u);
    }
}

template <bool AGG>
__global__ void __launch_bounds__(512) k_hist(const Row *__restrict__ in, uint64_t n,
                                              uint32_t *__restrict__ ghist, int nbins,
                                              RadixF rf) {
    extern __shared__ uint32_t sh_hist[];
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) sh_hist[i] = 0;
    __syncthreads();
    const uint64_t head = (reinterpret_cast<uintptr_t>(in) & 15) ? 1 : 0;
    if (head && n && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&sh_hist[radix_f(rf, in[0].key)], 1u);
    const uint64_t body = n > head ? n - head : 0;
    const uint4 *v = reinterpret_cast<const uint4 *>(in + head);
    const uint64_t nv = body / 2;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < nv; i += 4 * stride) {
        uint4 a = ldg_stream(v + i), b = ldg_stream(v + i + stride);
        uint4 c = ldg_stream(v + i + 2 * stride), d = ldg_stream(v + i + 3 * stride);
        hist_add<AGG>(sh_hist, radix_f(rf, a.x));
        hist_add<AGG>(sh_hist, radix_f(rf, a.z));
        hist_add<AGG>(sh_hist, radix_f(rf, b.x));
        hist_add<AGG>(sh_hist, radix_f(rf, b.z));
        hist_add<AGG>(sh_hist, radix_f(rf, c.x));
        hist_add<AGG>(sh_hist, radix_f(rf, c.z));
        hist_add<AGG>(sh_hist, radix_f(rf, d.x));
        hist_add<AGG>(sh_hist, radix_f(rf, d.z));
    }
    for (; i < nv; i += stride) {
        uint4 a = ldg_stream(v + i);
        hist_add<AGG>(sh_hist, radix_f(rf, a.x));
        hist_add<AGG>(sh_hist, radix_f(rf, a.z));
    }
    if ((body & 1) && blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(&sh_hist[radix_f(rf, in[n - 1].key)], 1u);
    __syncthreads();
    for (int j = threadIdx.x; j < nbins; j += blockDim.x)
        if (sh_hist[j]) atomicAdd(&ghist[j], sh_hist[j]);
}

cudaError_t launch_hist(const Row *in, uint64_t n, uint32_t *hist, int P_log2, RadixF rf,
                        bool aggregate, int nsm, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int nbins = 1 << P_log2;
    const size_t smem = (size_t)nbins * sizeof(uint32_t);
    // enough CTAs to cover the GPU, but at least ~16K rows each so the
    // per-CTA histogram flush stays small next to the streaming read
    uint64_t want = (n + 16383) / 16384;
    int per_sm = smem <= 48 * 1024 ? 4 : (smem <= 96 * 1024 ? 2 : 1);
    uint64_t grid = umin64(want, (uint64_t)nsm * per_sm);
    if (grid < 1) grid = 1;
    auto kern = aggregate ? k_hist<true> : k_hist<false>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<(unsigned)grid, 512, smem, st>>>(in, n, hist, nbins, rf);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K2 planner (one CTA): exclusive scans of both histograms into partition
// bases, pass-2 segment/tile tables, and the join work items.  Replaces the
// task creation of Joins/radix_join.c:946-1000 and :609-617 (pairs with both
// sides non-empty), with oversized S sides split into several items.
// ---------------------------------------------------------------------------
constexpr int PLAN_THREADS = 1024;

__device__ void plan_bases(const uint32_t *hist, uint64_t *base, uint64_t n, int P,
                           unsigned long long *maxp, uint64_t *scratch) {
    const int C = (P + PLAN_THREADS - 1) / PLAN_THREADS;
    const int lo = min(P, (int)threadIdx.x * C), hi = min(P, lo + C);
    uint64_t sum = 0;
    uint32_t mx = 0;
    for (int f = lo; f < hi; f++) {
        sum += hist[f];
        mx = max(mx, hist[f]);
    }
    uint64_t total;
    uint64_t run = block_excl_scan<PLAN_THREADS>(sum, &total, scratch);
    for (int f = lo; f < hi; f++) {
        base[f] = run;
        run += hist[f];
    }
    if (threadIdx.x == 0) base[P] = n;
    unsigned wmax = warp_max_u32(mx);
    if ((threadIdx.x & 31) == 0 && wmax) atomicMax(maxp, (unsigned long long)wmax);
}

__global__ void __launch_bounds__(PLAN_THREADS) k_plan(PlanArgs a) {
    __shared__ uint64_t scratch[PLAN_THREADS / 32 + 1];
    const int P = 1 << a.P_log2;
    plan_bases(a.r.hist, a.r.base, a.nR, P, &a.ctrl->max_part_R, scratch);
    plan_bases(a.s.hist, a.s.base, a.nS, P, &a.ctrl->max_part_S, scratch);
    __syncthreads();  // bases visible block-wide

    // pass-2 segments: pass-1 partition p1 = final partitions [p1 << b2, (p1+1) << b2)
    if (a.passes == 2) {
        const int F1 = 1 << a.b1;
        for (int rel = 0; rel < 2; rel++) {
            const RelPlan &rp = rel ? a.s : a.r;
            const uint64_t n = rel ? a.nS : a.nR;
            uint32_t tiles = 0;
            const int p1 = threadIdx.x;
            uint64_t st = 0;
            if (p1 < F1) {
                st = rp.base[(uint64_t)p1 << a.b2];
                uint64_t en = rp.base[(uint64_t)(p1 + 1) << a.b2];
                tiles = (uint32_t)((en - st + SCATTER_TILE - 1) / SCATTER_TILE);
            }
            uint64_t total;
            uint64_t ex = block_excl_scan<PLAN_THREADS>(tiles, &total, scratch);
            if (p1 < F1) {
                rp.seg_start[p1] = st;
                rp.seg_tile[p1] = (uint32_t)ex;
            }
            if (threadIdx.x == 0) {
                rp.seg_start[F1] = n;
                rp.seg_tile[F1] = (uint32_t)total;
            }
        }
    }

    // join work items
    const int C = (P + PLAN_THREADS - 1) / PLAN_THREADS;
    const int lo = min(P, (int)threadIdx.x * C), hi = min(P, lo + C);
    uint64_t cnt = 0, nonempty = 0;
    for (int f = lo; f < hi; f++) {
        uint32_t hr = a.r.hist[f], hs = a.s.hist[f];
        if (hr == 0 || hs == 0) continue;
        uint64_t nrc = (hr + (uint64_t)a.capR - 1) / a.capR;
        uint64_t nsc = (nrc == 1 && a.capS) ? (hs + a.capS - 1) / a.capS : 1;
        cnt += nrc * nsc;
        nonempty++;
    }
    uint64_t total;
    uint64_t off = block_excl_scan<PLAN_THREADS>(cnt, &total, scratch);
    if (total > a.item_cap) {  // cannot happen with the host's bound; guard anyway
        if (threadIdx.x == 0) {
            atomicCAS(&a.ctrl->error, 0u, (unsigned)TBG_ERR_CAPACITY);
            a.ctrl->nitems = 0;
        }
        return;
    }
    for (int f = lo; f < hi; f++) {
        uint32_t hr = a.r.hist[f], hs = a.s.hist[f];
        if (hr == 0 || hs == 0) continue;
        uint64_t nrc = (hr + (uint64_t)a.capR - 1) / a.capR;
        uint64_t nsc = (nrc == 1 && a.capS) ? (hs + a.capS - 1) / a.capS : 1;
        uint64_t sstep = (hs + nsc - 1) / nsc;
        for (uint64_t rc = 0; rc < nrc; rc++) {
            for (uint64_t sc = 0; sc < nsc; sc++) {
                Item it;
                it.part = (uint32_t)f;
                it.r_off = a.r.base[f] + rc * (uint64_t)a.capR;
                it.r_len = (uint32_t)umin64((uint64_t)a.capR, hr - rc * (uint64_t)a.capR);
                it.s_off = a.s.base[f] + sc * sstep;
                it.s_len = umin64(sstep, hs - sc * sstep);
                a.items[off++] = it;
            }
        }
    }
    unsigned long long ne = warp_sum_u64(nonempty);
    if ((threadIdx.x & 31) == 0 && ne) atomicAdd(&a.ctrl->nonempty, ne);
    if (threadIdx.x == 0) a.ctrl->nitems = (unsigned)total;
}

cudaError_t launch_plan(const PlanArgs &a, cudaStream_t st) {
    k_plan<<<1, PLAN_THREADS, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K3 stable scatter, one tile of SCATTER_TILE rows per CTA ticket.
//
//  1. rows are loaded warp-striped: warp w owns a contiguous sub-tile, so the
//     order (warp, item, lane) is the input order (needed for stability);
//  2. each row is ranked inside its warp with __match_any_sync against a
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
        unsigned peers = __match_any_sync(0xffffffffu, d[i]);
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
        cudaError_t e = cudaFuncSetAttribute(k_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_done = true;
    }
    k_scatter<<<(unsigned)max_tiles, SCATTER_THREADS, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
