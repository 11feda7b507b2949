// Radix partitioning for sm_100a without inter-CTA waits.
//
// Replaces the reference's two partitioning passes (Joins/radix_join.c:630-703
// parallel_radix_partition, :525-562 radix_cluster, :573-619
// serial_radix_partition, the SWWC variant :734-827) and the task queues that
// feed them (Include/task_queue.h).  The reference's own structure -- every
// thread histograms a contiguous chunk, a prefix over (thread, digit) gives
// each thread exact write cursors, then each thread scatters its chunk -- is
// kept, with a CTA in the role of a thread:
//
//   K1 hist   CTA c histograms chunk c over all final partitions f (2^bits
//             bins in shared memory) -> hist[c][f];
//   K2 scan   column prefix over chunks -> pre[c][f], totals[f];
//   K3 plan   exclusive scan of totals -> base[f], join work items;
//   K4 pass 1 CTA c scatters chunk c by the pass-1 digit d1 = f >> b2 to
//             cursor[d1] = base[d1 << b2] + sum_{d2} pre[c][(d1 << b2) | d2];
//   K5 pass 2 unit (c, s) = the rows chunk c wrote to pass-1 partition s;
//             scattered by d2 to cursor[d2] = base[(s << b2) | d2] + pre[c][...].
//
// One histogram read gives every cursor of both passes, so the traffic is
// 8 (hist) + 16 (pass 1) + 16 (pass 2) bytes per row, and no CTA ever waits
// for another.  Each pass stages a tile digit-sorted in shared memory and
// writes runs with consecutive threads on consecutive addresses (coalesced).
#include "part_dev.cuh"

namespace tbg {

// Threads per CTA of the two passes (tiles of THREADS * PART_ITEMS rows).
#ifndef TBG_PASS1_THREADS
#define TBG_PASS1_THREADS 512
#endif
#ifndef TBG_PASS2_THREADS
#define TBG_PASS2_THREADS 512
#endif
constexpr int PASS1_THREADS = TBG_PASS1_THREADS;
constexpr int PASS2_THREADS = TBG_PASS2_THREADS;
// Tile buffers per CTA of the two passes (bulk copies run NBUF - 1 tiles ahead).
#ifndef TBG_PASS_NBUF
#define TBG_PASS_NBUF 3
#endif
constexpr int PASS_NBUF = TBG_PASS_NBUF;
template <int THREADS>
using PassSmem = PartSmem<THREADS, PASS_NBUF>;

// ---------------------------------------------------------------------------
// K1 per-chunk histogram over the final partition index f
// ---------------------------------------------------------------------------
constexpr int HIST_THREADS = 1024;

// With `oor` set, keys whose key - rf.sub exceeds range_max are also
// counted into *oor (the histogram of a relation binned by another's key
// range: a non-zero count means the bins are not valid).
__global__ void __launch_bounds__(HIST_THREADS) k_hist_chunks(const Row *__restrict__ in, uint64_t n,
                                                             uint64_t chunk, uint32_t *__restrict__ hist,
                                                             int nbins, RadixF rf, unsigned long long *oor,
                                                             uint32_t range_max) {
    unsigned outside = 0;
    extern __shared__ uint32_t sh[];
    for (int i = threadIdx.x; i < nbins; i += HIST_THREADS) sh[i] = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * chunk;
    const uint64_t hi = umin64(n, lo + chunk);
    if (lo < hi) {
        const uint64_t head = ((reinterpret_cast<uintptr_t>(in + lo) & 15) != 0) ? 1 : 0;
        const uint64_t body = hi - lo - head;
        const uint64_t nv = body / 2;
        const uint4 *v = reinterpret_cast<const uint4 *>(in + lo + head);
        // warp-uniform trip count: every lane reaches the shuffles
        const uint64_t per = (uint64_t)HIST_THREADS * 4;
        for (uint64_t base = 0; base < nv; base += per) {
            uint4 x[4];
            bool ok[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                uint64_t i = base + (uint64_t)u * HIST_THREADS + threadIdx.x;
                ok[u] = i < nv;
                if (ok[u]) x[u] = ldg_stream(v + i);
            }
            uint32_t f[8];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                f[2 * u] = ok[u] ? radix_f(rf, x[u].x) : 0;
                f[2 * u + 1] = ok[u] ? radix_f(rf, x[u].z) : 0;
                if (oor && ok[u]) outside += (x[u].x - rf.sub > range_max) + (x[u].z - rf.sub > range_max);
            }
            const bool dup = warp_has_dups(f[0], ok[0]);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                hist_add_warp(sh, f[2 * u], ok[u], dup);
                hist_add_warp(sh, f[2 * u + 1], ok[u], dup);
            }
        }
        if (threadIdx.x == 0) {
            if (head) {
                atomicAdd(&sh[radix_f(rf, in[lo].key)], 1u);
                outside += oor && in[lo].key - rf.sub > range_max;
            }
            if (body & 1) {
                atomicAdd(&sh[radix_f(rf, in[hi - 1].key)], 1u);
                outside += oor && in[hi - 1].key - rf.sub > range_max;
            }
        }
    }
    if (oor) {
        const unsigned long long wo = warp_sum_u64((unsigned long long)outside);
        if ((threadIdx.x & 31) == 0 && wo) atomicAdd(oor, wo);
    }
    __syncthreads();
    uint32_t *dst = hist + (uint64_t)blockIdx.x * nbins;
    for (int i = threadIdx.x; i < nbins; i += HIST_THREADS) dst[i] = sh[i];
}

// ---------------------------------------------------------------------------
// K2 column prefix over chunks (in place) and per-partition totals.  A CTA
// owns 32 consecutive partitions (threadIdx.x, coalesced) and splits the
// chunks into 32 segments (threadIdx.y): segment sums, a prefix over the
// segments, then each segment rewritten with running prefixes.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) k_colscan(uint32_t *__restrict__ hist, int G, int P,
                                                  uint32_t *__restrict__ totals) {
    __shared__ uint32_t seg[32][33];
    const int f = blockIdx.x * 32 + threadIdx.x;
    const int per = (G + 31) / 32;
    const int c0 = min(G, (int)threadIdx.y * per), c1 = min(G, c0 + per);
    uint32_t *col = hist + f;
    uint32_t sum = 0;
    if (f < P) {
        int c = c0;
        for (; c + 8 <= c1; c += 8) {  // eight independent loads in flight
            uint32_t x[8];
#pragma unroll
            for (int u = 0; u < 8; u++) x[u] = col[(uint64_t)(c + u) * P];
#pragma unroll
            for (int u = 0; u < 8; u++) sum += x[u];
        }
        for (; c < c1; c++) sum += col[(uint64_t)c * P];
    }
    seg[threadIdx.y][threadIdx.x] = sum;
    __syncthreads();
    if (threadIdx.y == 0) {
        uint32_t run = 0;
        for (int y = 0; y < 32; y++) {
            const uint32_t v = seg[y][threadIdx.x];
            seg[y][threadIdx.x] = run;
            run += v;
        }
        if (f < P) totals[f] = run;
    }
    __syncthreads();
    if (f < P) {
        uint32_t run = seg[threadIdx.y][threadIdx.x];
        int c = c0;
        for (; c + 8 <= c1; c += 8) {
            uint32_t x[8];
#pragma unroll
            for (int u = 0; u < 8; u++) x[u] = col[(uint64_t)(c + u) * P];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                col[(uint64_t)(c + u) * P] = run;
                run += x[u];
            }
        }
        for (; c < c1; c++) {
            const uint32_t v = col[(uint64_t)c * P];
            col[(uint64_t)c * P] = run;
            run += v;
        }
    }
}

// ---------------------------------------------------------------------------
// K3 planner (one CTA): partition bases and join work items.  Replaces the
// task creation of Joins/radix_join.c:946-1000 and :609-617 (pairs with both
// sides non-empty); oversized S sides are split into several items.
// ---------------------------------------------------------------------------
constexpr int PLAN_THREADS = 1024;

// Shared-memory index of entry i when every thread scans 32 consecutive
// entries: one word of padding per 32 keeps those reads conflict-free.
__device__ __forceinline__ uint32_t skew32(uint32_t i) { return i + (i >> 5); }

// Exclusive scan of hist[0..P) into base[0..P], base[P] = total, and the
// largest entry into *maxp.  The counts are staged through shared memory
// (`sh`, P + P / 32 words) so global reads and writes are coalesced.
__device__ void plan_bases(const uint32_t *hist, uint64_t *base, int P, unsigned long long *maxp, uint64_t *scratch,
                           uint32_t *sh) {
    const int tid = threadIdx.x;
    for (int i = tid; i < P; i += PLAN_THREADS) sh[skew32(i)] = hist[i];
    __syncthreads();
    const int C = (P + PLAN_THREADS - 1) / PLAN_THREADS;
    const int lo = min(P, tid * C), hi = min(P, lo + C);
    uint64_t sum = 0;
    uint32_t mx = 0;
    for (int f = lo; f < hi; f++) {
        const uint32_t x = sh[skew32(f)];
        sum += x;
        mx = max(mx, x);
    }
    uint64_t total;
    uint64_t run = block_excl_scan<PLAN_THREADS>(sum, &total, scratch);
    for (int f = lo; f < hi; f++) {  // prefixes fit 32 bits: a relation holds < 2^32 rows
        const uint32_t x = sh[skew32(f)];
        sh[skew32(f)] = (uint32_t)run;
        run += x;
    }
    __syncthreads();
    for (int i = tid; i < P; i += PLAN_THREADS) base[i] = sh[skew32(i)];
    if (tid == 0) base[P] = total;  // rows counted (n unless rows were bypassed)
    unsigned wmax = warp_max_u32(mx);
    if ((tid & 31) == 0 && wmax) atomicMax(maxp, (unsigned long long)wmax);
}

__global__ void __launch_bounds__(PLAN_THREADS) k_plan_bases(const uint32_t *totals, uint64_t *base, int P_log2,
                                                            unsigned long long *maxp) {
    extern __shared__ uint32_t sh[];
    __shared__ uint64_t scratch[PLAN_THREADS / 32 + 1];
    plan_bases(totals, base, 1 << P_log2, maxp, scratch, sh);
}

// Join work items from both relations' totals and bases (written by
// k_plan_bases), planned by P / PLAN_THREADS CTAs.  Every CTA first counts
// the items of all partitions (one coalesced read of both totals, from L2) to
// take the same split decision; then thread t of CTA c plans partition
// c * PLAN_THREADS + t, and each warp reserves its items with one atomic on
// ctrl->nitems (zeroed by the launcher).  The item list is in reservation
// order, not sorted by partition.
__global__ void __launch_bounds__(PLAN_THREADS) k_plan(PlanArgs a) {
    __shared__ uint64_t scratch[PLAN_THREADS / 32 + 1];
    const int P = 1 << a.P_log2;
    // S sides larger than capS are split (skew) for every R chunk of the
    // partition; if that would overflow the item buffer, partitions whose R
    // side needs several chunks keep S whole
    auto s_chunks = [&](uint32_t hs, uint64_t nrc, bool split_all) -> uint64_t {
        if (!a.capS || (nrc > 1 && !split_all)) return 1;
        return (hs + a.capS - 1) / a.capS;
    };
    uint64_t cnt_all = 0;
    for (int f = threadIdx.x; f < P; f += PLAN_THREADS) {
        const uint32_t hr = a.r.hist[f], hs = a.s.hist[f];
        if (hr == 0 || hs == 0) continue;
        const uint64_t nrc = (hr + (uint64_t)a.capR - 1) / a.capR;
        cnt_all += nrc * s_chunks(hs, nrc, true);
    }
    uint64_t total_all;
    block_excl_scan<PLAN_THREADS>(cnt_all, &total_all, scratch);
    const bool split_all = total_all <= a.item_cap;
    const int f = blockIdx.x * PLAN_THREADS + threadIdx.x;
    const int lane = threadIdx.x & 31;
    uint32_t hr = 0, hs = 0;
    uint64_t nrc = 0, nsc = 0;
    if (f < P) {
        hr = a.r.hist[f];
        hs = a.s.hist[f];
        if (hr && hs) {
            nrc = (hr + (uint64_t)a.capR - 1) / a.capR;
            nsc = s_chunks(hs, nrc, split_all);
        }
    }
    const uint64_t mine = nrc * nsc;
    // warp prefix of the item counts, one reservation per warp
    uint64_t inc = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    const uint64_t wtot = __shfl_sync(0xffffffffu, inc, 31);
    unsigned wb = 0;
    if (lane == 31 && wtot) wb = atomicAdd(&a.ctrl->nitems, (unsigned)wtot);
    wb = __shfl_sync(0xffffffffu, wb, 31);
    uint64_t off = (uint64_t)wb + inc - mine;
    const bool fits = off + mine <= a.item_cap;  // always, with the host's bound; guarded anyway
    if (mine && !fits) atomicCAS(&a.ctrl->error, 0u, (unsigned)TBG_ERR_CAPACITY);
    if (mine && fits) {
        const uint64_t sstep = (hs + nsc - 1) / nsc;
        const uint64_t rb = a.r.base[f], sb = a.s.base[f];
        for (uint64_t rc = 0; rc < nrc; rc++) {
            for (uint64_t sc = 0; sc < nsc; sc++) {
                Item it;
                it.part = (uint32_t)f;
                it.r_off = rb + rc * (uint64_t)a.capR;
                it.r_len = (uint32_t)umin64((uint64_t)a.capR, hr - rc * (uint64_t)a.capR);
                it.s_off = sb + sc * sstep;
                it.s_len = umin64(sstep, hs - sc * sstep);
                a.items[off++] = it;
            }
        }
    }
    const unsigned ne = __popc(__ballot_sync(0xffffffffu, mine != 0));
    if (lane == 0 && ne) atomicAdd(&a.ctrl->nonempty, (unsigned long long)ne);
}

// ---------------------------------------------------------------------------
// K4 pass 1: CTA c scatters chunk c by d1.  With one pass, d1 is f itself.
// ---------------------------------------------------------------------------
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_part_pass1(PartArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto &sm = *reinterpret_cast<PassSmem<THREADS> *>(smem_raw);
    const int c = blockIdx.x, tid = threadIdx.x;
    const int P = 1 << (a.b1 + a.b2);
    const int F = 1 << a.b1;
    const uint32_t *pre = a.pre + (uint64_t)c * P;
    const uint32_t *nxt = c + 1 < a.G ? a.pre + (uint64_t)(c + 1) * P : a.totals;
    // cursors: sum the chunk's prefix over each pass-1 digit's final partitions
    // (delta[0] holds the chunk's row count per pass-1 digit until the scatter)
    uint32_t *rows1 = sm.delta[0];
    for (int i = tid; i < F; i += THREADS) {
        sm.cursor[i] = 0;
        rows1[i] = 0;
    }
    __syncthreads();
    {
        // each thread sums a contiguous run of f (one pass-1 digit per flush)
        const int per = P >= THREADS ? P / THREADS : 1;
        const int f0 = tid * per;
        uint32_t acc_c = 0, acc_t = 0;
        int cur_s = -1;
        for (int f = f0; f < f0 + per && f < P; f++) {
            const int s = f >> a.b2;
            if (s != cur_s) {
                if (cur_s >= 0) {
                    atomicAdd(&sm.cursor[cur_s], acc_c);
                    atomicAdd(&rows1[cur_s], acc_t);
                }
                cur_s = s;
                acc_c = acc_t = 0;
            }
            acc_c += pre[f];
            acc_t += nxt[f] - pre[f];
        }
        if (cur_s >= 0) {
            atomicAdd(&sm.cursor[cur_s], acc_c);
            atomicAdd(&rows1[cur_s], acc_t);
        }
    }
    __syncthreads();
    for (int s = tid; s < F; s += THREADS) {
        const uint32_t cur = (uint32_t)a.base[(uint64_t)s << a.b2] + sm.cursor[s];
        sm.cursor[s] = cur;
        if (a.off1) {
            a.off1[(uint64_t)c * F + s] = cur;
            a.cnt1[(uint64_t)c * F + s] = rows1[s];
        }
    }
    __syncthreads();
    const uint64_t lo = (uint64_t)c * a.chunk;
    const uint64_t hi = a.chunk_len ? lo + a.chunk_len[c] : umin64(a.n, lo + a.chunk);
    part_range<THREADS>(a.in, lo, hi, a.n, a.out, (uint32_t)a.n, a.d1, F, sm, a.err);
}

// ---------------------------------------------------------------------------
// K5 pass 2: unit (c, s), s-major, scatters by d2 within pass-1 partition s.
// ---------------------------------------------------------------------------
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_part_pass2(PartArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto &sm = *reinterpret_cast<PassSmem<THREADS> *>(smem_raw);
    const int F1 = 1 << a.b1, F2 = 1 << a.b2;
    const int P = F1 * F2;
    const int ngroups = (a.G + a.group - 1) / a.group;
    const uint64_t unit = blockIdx.x;
    const int s = (int)(unit / ngroups), g = (int)(unit % ngroups);
    const int c0 = g * a.group, c1 = min(a.G, c0 + a.group) - 1;
    // chunk c's rows of partition s follow chunk c-1's in the pass-1 output,
    // so a group of chunks is one contiguous range with one cursor per digit
    const uint64_t lo = a.off1[(uint64_t)c0 * F1 + s];
    const uint64_t hi = (uint64_t)a.off1[(uint64_t)c1 * F1 + s] + a.cnt1[(uint64_t)c1 * F1 + s];
    if (lo >= hi) return;
    for (int d = threadIdx.x; d < F2; d += THREADS) {
        const uint64_t f = ((uint64_t)s << a.b2) | d;
        sm.cursor[d] = (uint32_t)a.base[f] + a.pre[(uint64_t)c0 * P + f];
    }
    __syncthreads();
    part_range<THREADS>(a.in, lo, hi, a.n, a.out, (uint32_t)a.n, a.d2, F2, sm, a.err);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
int hist_ctas_per_sm(int P_log2) {
    const size_t smem = ((size_t)1 << P_log2) * 4;
    int n = 0;
    smem_limit((const void *)k_hist_chunks, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_hist_chunks, HIST_THREADS, smem);
    return n < 1 ? 1 : n;
}

cudaError_t launch_hist_chunks(const Row *in, uint64_t n, uint64_t chunk, int G, uint32_t *hist,
                               int P_log2, RadixF rf, cudaStream_t st, unsigned long long *oor, uint32_t range_max) {
    const int nbins = 1 << P_log2;
    const size_t smem = (size_t)nbins * 4;
    cudaError_t e = smem_limit((const void *)k_hist_chunks, smem);
    if (e != cudaSuccess) return e;
    k_hist_chunks<<<G, HIST_THREADS, smem, st>>>(in, n, chunk, hist, nbins, rf, oor, range_max);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_colscan(uint32_t *hist, int G, int P, uint32_t *totals, cudaStream_t st) {
    k_colscan<<<(P + 31) / 32, dim3(32, 32), 0, st>>>(hist, G, P, totals);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_plan_bases(const uint32_t *totals, uint64_t *base, int P_log2, unsigned long long *maxp,
                              cudaStream_t st) {
    const int P = 1 << P_log2;
    const size_t smem = (size_t)(P + P / 32 + 1) * sizeof(uint32_t);
    cudaError_t e = smem_limit((const void *)k_plan_bases, smem);
    if (e != cudaSuccess) return e;
    k_plan_bases<<<1, PLAN_THREADS, smem, st>>>(totals, base, P_log2, maxp);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_plan(const PlanArgs &a, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(&a.ctrl->nitems, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    const int P = 1 << a.P_log2;
    k_plan<<<(P + PLAN_THREADS - 1) / PLAN_THREADS, PLAN_THREADS, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_part_pass1(const PartArgs &a, cudaStream_t st) {
    constexpr int T = PASS1_THREADS;
    const size_t smem = sizeof(PassSmem<T>);
    cudaError_t e = smem_limit((const void *)k_part_pass1<T>, smem);
    if (e != cudaSuccess) return e;
    k_part_pass1<T><<<a.G, T, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_part_pass2(const PartArgs &a, cudaStream_t st) {
    constexpr int T = PASS2_THREADS;
    const size_t smem = sizeof(PassSmem<T>);
    cudaError_t e = smem_limit((const void *)k_part_pass2<T>, smem);
    if (e != cudaSuccess) return e;
    const uint64_t units = (uint64_t)((a.G + a.group - 1) / a.group) << a.b1;
    k_part_pass2<T><<<(unsigned)units, T, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
