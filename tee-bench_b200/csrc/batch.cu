// Batched joins in one persistent launch.
//
// Every CTA pulls tickets from one counter; the ticket ranges are, in order,
//   hist     one chunk (`chunk` rows) of R_i or S_i: shared-memory histogram
//            over the join's P = 2^B partitions (low key bits);
//   scan     one join: column prefix of its chunk histograms (in place),
//            partition bases, join work items (S_p split every capS rows);
//   scatter  one chunk: the TMA-fed digit-sorting tile scatter of the
//            single-join partitioner, cursors = base[f] + prefix[chunk][f];
//   join     one worker of a partitioned join (pulls that join's items) or
//            one S slice of a direct join (B = 0, R_i loaded whole);
// build/probe runs out of shared memory as in the single-join kernel.  A
// ticket waits only on tickets handed out before it (per-join counters with
// acquire/release), so there is no grid-wide barrier and no co-residency
// requirement.  Data written earlier in the launch (histograms, bases,
// items, partitioned rows) is read with L2-only loads.
//
// Each join's count equals the reference's RHO count on that join
// (Joins/radix_join.c:1558-1561, join_init_run :1237-1396; bucket
// chaining :187-244, histogram join :374-440).
#include <algorithm>

#include "batch.h"
#include "join_dev.cuh"
#include "part_dev.cuh"

namespace tbg {

namespace {

using BPart = PartSmem<BATCH_THREADS>;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 waits until *flag >= target (bounded: records TBG_ERR_TIMEOUT and
// gives up), then the whole CTA proceeds.
__device__ void cta_wait(const unsigned *flag, unsigned target, unsigned *err) {
    if (threadIdx.x == 0) {
        unsigned ns = 32;
        for (uint32_t it = 0; ld_acquire_u32(flag) < target; it++) {
            if (it >= BATCH_SPIN_LIMIT) {
                atomicCAS(err, 0u, (unsigned)TBG_ERR_TIMEOUT);
                break;
            }
            __nanosleep(ns);
            if (ns < 512) ns <<= 1;
        }
        __threadfence();
    }
    __syncthreads();
}

// Publishes every write of this CTA, then *flag += 1.
__device__ void cta_signal(unsigned *flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(flag, 1u);
    }
}

__device__ __forceinline__ int ilog2(uint32_t p) { return 31 - __clz(p); }

// ---------------------------------------------------------------------------
// hist: chunk histogram over the join's partitions
// ---------------------------------------------------------------------------
// Per-warp sub-histograms (P <= 256 bins each): with so few bins nearly every
// warp holds repeated digits, so each row pays one shared atomic on its
// warp's own bins instead of a match-based aggregation; the warps' bins are
// summed at the end of the chunk.
__device__ void hist_chunk(const BatchArgs &a, uint32_t c, uint32_t *bins) {
    constexpr int NW = BATCH_THREADS / 32;
    const uint2 ch = a.chunks[c];
    const BatchJoin &J = a.joins[ch.x];
    const int rel = ch.y >> 31;
    const uint32_t idx = ch.y & 0x7fffffffu;
    const Row *in = rel ? J.S : J.R;
    const uint64_t n = rel ? J.nS : J.nR;
    const uint32_t P = J.P, mask = P - 1;
    const int tid = threadIdx.x;
    uint32_t *wb = bins + (tid >> 5) * BATCH_FMAX;  // this warp's bins
    for (uint32_t i = tid; i < NW * BATCH_FMAX; i += BATCH_THREADS) bins[i] = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)idx * J.chunk;
    const uint64_t hi = umin64(n, lo + J.chunk);
    const uint64_t head = ((reinterpret_cast<uintptr_t>(in + lo) & 15) != 0) ? 1 : 0;
    const uint64_t body = hi - lo - head;
    const uint64_t nv = body / 2;
    const uint4 *v = reinterpret_cast<const uint4 *>(in + lo + head);
    const uint64_t per = (uint64_t)BATCH_THREADS * 4;
    for (uint64_t base = 0; base < nv; base += per) {
        uint4 x[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t i = base + (uint64_t)u * BATCH_THREADS + tid;
            ok[u] = i < nv;
            if (ok[u]) x[u] = ldg_stream(v + i);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (ok[u]) {
                atomicAdd(&wb[x[u].x & mask], 1u);
                atomicAdd(&wb[x[u].z & mask], 1u);
            }
        }
    }
    if (tid == 0) {
        if (head) atomicAdd(&wb[in[lo].key & mask], 1u);
        if (body & 1) atomicAdd(&wb[in[hi - 1].key & mask], 1u);
    }
    __syncthreads();
    uint32_t *dst = (rel ? J.histS : J.histR) + (uint64_t)idx * P;
    for (uint32_t f = tid; f < P; f += BATCH_THREADS) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) t += bins[w * BATCH_FMAX + f];
        __stcg(dst + f, t);
    }
    cta_signal(&a.sync[ch.x].hist_done);
}

// ---------------------------------------------------------------------------
// scan: column prefix, bases, items
// ---------------------------------------------------------------------------

// In place: h[c][f] <- sum_{c' < c} h[c'][f]; tot[f] <- column total.
// Thread (z, f) owns chunk segment z of column f.
__device__ void column_prefix(uint32_t *h, uint32_t G, uint32_t P, uint32_t *part, uint32_t *tot) {
    const int tid = threadIdx.x;
    const int lp = ilog2(P);
    const uint32_t Z = BATCH_THREADS >> lp;
    const uint32_t f = tid & (P - 1), z = tid >> lp;
    const uint32_t seg = (G + Z - 1) / Z;
    const uint32_t c0 = min(G, z * seg), c1 = min(G, c0 + seg);
    uint32_t s = 0;
    uint32_t c = c0;
    for (; c + 8 <= c1; c += 8) {
        uint32_t x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = __ldcg(h + (uint64_t)(c + u) * P + f);
#pragma unroll
        for (int u = 0; u < 8; u++) s += x[u];
    }
    for (; c < c1; c++) s += __ldcg(h + (uint64_t)c * P + f);
    part[tid] = s;
    __syncthreads();
    uint32_t run = 0;
    for (uint32_t zz = 0; zz < z; zz++) run += part[zz * P + f];
    if (z == 0) {
        uint32_t t = 0;
        for (uint32_t zz = 0; zz < Z; zz++) t += part[zz * P + f];
        tot[f] = t;
    }
    c = c0;
    for (; c + 8 <= c1; c += 8) {
        uint32_t x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = __ldcg(h + (uint64_t)(c + u) * P + f);
#pragma unroll
        for (int u = 0; u < 8; u++) {
            __stcg(h + (uint64_t)(c + u) * P + f, run);
            run += x[u];
        }
    }
    for (; c < c1; c++) {
        const uint32_t x = __ldcg(h + (uint64_t)c * P + f);
        __stcg(h + (uint64_t)c * P + f, run);
        run += x;
    }
    __syncthreads();
}

__device__ void scan_join(const BatchArgs &a, uint32_t q, uint32_t *sm, uint64_t *scratch) {
    const uint32_t j = a.scans[q];
    const BatchJoin &J = a.joins[j];
    cta_wait(&a.sync[j].hist_done, J.GR + J.GS, a.err);
    const int tid = threadIdx.x;
    const uint32_t P = J.P;
    uint32_t *part = sm;                          // [BATCH_THREADS]
    uint32_t *tot = part + BATCH_THREADS;         // [2][BATCH_FMAX]
    uint32_t *base = tot + 2 * BATCH_FMAX;        // [2][BATCH_FMAX]
    column_prefix(J.histR, J.GR, P, part, tot);
    column_prefix(J.histS, J.GS, P, part, tot + BATCH_FMAX);
    bool ok = true;
    for (int rel = 0; rel < 2; rel++) {
        uint64_t total;
        const uint32_t x = (uint32_t)tid < P ? tot[rel * BATCH_FMAX + tid] : 0;
        const uint64_t b = block_excl_scan<BATCH_THREADS>(x, &total, scratch);
        if ((uint32_t)tid < P) {
            base[rel * BATCH_FMAX + tid] = (uint32_t)b;
            __stcg((rel ? J.baseS : J.baseR) + tid, (uint32_t)b);
        }
        // every chunk histogram landed exactly once: totals add up to |rel|
        ok = ok && total == (rel ? J.nS : J.nR);
    }
    __syncthreads();
    uint32_t rl = 0, sl = 0, ns = 0;
    if ((uint32_t)tid < P) {
        rl = tot[tid];
        sl = tot[BATCH_FMAX + tid];
        ns = (rl && sl) ? (sl + J.capS - 1) / J.capS : 0;
    }
    uint64_t nit;
    const uint64_t pos = block_excl_scan<BATCH_THREADS>(ns, &nit, scratch);
    if (!ok || nit > J.item_cap) {
        // only reachable after a wait above gave up
        if (tid == 0) atomicCAS(a.err, 0u, (unsigned)TBG_ERR_TIMEOUT);
        nit = 0;
    } else {
        for (uint32_t k = 0; k < ns; k++) {
            Item m;
            m.r_off = base[tid];
            m.r_len = rl;
            m.s_off = (uint64_t)base[BATCH_FMAX + tid] + (uint64_t)k * J.capS;
            m.s_len = min(J.capS, sl - k * J.capS);
            m.part = tid;
            J.items[pos + k] = m;
        }
    }
    if (tid == 0) __stcg(&a.sync[j].nitems, (unsigned)nit);
    cta_signal(&a.sync[j].scan_done);
}

// ---------------------------------------------------------------------------
// scatter: one chunk into its join's partitions
// ---------------------------------------------------------------------------
__device__ void scatter_chunk(const BatchArgs &a, uint32_t c, BPart &sm, uint64_t *mbar, uint32_t &kseq) {
    const uint2 ch = a.chunks[c];
    const BatchJoin &J = a.joins[ch.x];
    cta_wait(&a.sync[ch.x].scan_done, 1, a.err);
    const int rel = ch.y >> 31;
    const uint32_t idx = ch.y & 0x7fffffffu;
    const uint32_t P = J.P;
    const uint32_t *base = rel ? J.baseS : J.baseR;
    const uint32_t *pre = (rel ? J.histS : J.histR) + (uint64_t)idx * P;
    for (uint32_t f = threadIdx.x; f < P; f += BATCH_THREADS) sm.cursor[f] = __ldcg(base + f) + __ldcg(pre + f);
    const Row *in = rel ? J.S : J.R;
    const uint64_t n = rel ? J.nS : J.nR;
    const uint64_t lo = (uint64_t)idx * J.chunk;
    const uint64_t hi = umin64(n, lo + J.chunk);
    part_tiles<BATCH_THREADS>(in, lo, hi, n, rel ? J.Sp : J.Rp, (uint32_t)n, DigitOp{0u, P - 1}, (int)P, sm, mbar,
                              kseq, a.err);
    cta_signal(&a.sync[ch.x].scat_done);
}

// ---------------------------------------------------------------------------
// join: build/probe
// ---------------------------------------------------------------------------
template <bool CG>
__device__ unsigned long long pair_count(Table &t, const Row *R, uint64_t rn, const Row *S, uint64_t sn,
                                         uint32_t capR, uint64_t *scratch) {
    unsigned long long c = 0;
    for (uint64_t r0 = 0; r0 < rn; r0 += capR) {
        build_table<BATCH_THREADS, CG>(t, R, r0, (uint32_t)umin64(capR, rn - r0), scratch);
        c += probe_count<BATCH_THREADS, CG>(t, S, sn);
        __syncthreads();  // table rebuilt by the next R slice
    }
    return c;
}

__device__ void join_ticket(const BatchArgs &a, uint32_t q, unsigned char *smem, uint64_t *scratch,
                            uint32_t *s_item) {
    const uint2 jt = a.jt[q];
    const BatchJoin &J = a.joins[jt.x];
    const uint32_t capR = a.capR;
    Table t;
    t.key = reinterpret_cast<uint32_t *>(smem);
    t.pay = t.key + capR;
    t.heads = t.pay + capR;
    t.next = reinterpret_cast<uint16_t *>(t.heads + capR + 2);
    t.head64 = nullptr;
    if (J.layout == 0) {  // counts only: keys, packed heads (capR * 4 is a multiple of 8), links
        t.head64 = reinterpret_cast<uint64_t *>(t.key + capR);
        t.next = reinterpret_cast<uint16_t *>(t.head64 + floor_pow2(capR + 2));
    }
    t.hs = (int)J.B;
    t.layout = (int)J.layout;
    t.hcap = floor_pow2(capR + 2);
    unsigned long long local = 0;
    if (J.B == 0) {
        const uint64_t lo = (uint64_t)jt.y * J.capS;
        const uint64_t hi = umin64(J.nS, lo + J.capS);
        if (lo < hi) local = pair_count<false>(t, J.R, J.nR, J.S + lo, hi - lo, capR, scratch);
    } else {
        BatchSync &sy = a.sync[jt.x];
        cta_wait(&sy.scat_done, J.GR + J.GS, a.err);
        const unsigned nit = __ldcg(&sy.nitems);
        for (;;) {
            if (threadIdx.x == 0) *s_item = atomicAdd(&sy.item_ctr, 1u);
            __syncthreads();
            const unsigned i = *s_item;
            __syncthreads();
            if (i >= nit) break;
            const uint4 *mp = reinterpret_cast<const uint4 *>(J.items + i);
            const uint4 m0 = __ldcg(mp), m1 = __ldcg(mp + 1);
            const uint64_t r_off = (uint64_t)m0.x | ((uint64_t)m0.y << 32);
            const uint64_t s_off = (uint64_t)m0.z | ((uint64_t)m0.w << 32);
            const uint64_t s_len = (uint64_t)m1.x | ((uint64_t)m1.y << 32);
            const uint32_t r_len = m1.z;
            if (r_off + r_len <= J.nR && s_off + s_len <= J.nS)
                local += pair_count<true>(t, J.Rp + r_off, r_len, J.Sp + s_off, s_len, capR, scratch);
        }
    }
    const unsigned long long ws = warp_sum_u64(local);
    if ((threadIdx.x & 31) == 0 && ws) atomicAdd(a.counts + J.orig, ws);
}

static_assert(sizeof(Item) == 32, "join_ticket reads an item as two 16-byte words");

}  // namespace

__global__ void __launch_bounds__(BATCH_THREADS, 2) k_batch(BatchArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t mbar[PART_NBUF];
    __shared__ uint64_t scratch[BATCH_THREADS / 32 + 1];
    __shared__ uint32_t s_ticket, s_item;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int i = 0; i < PART_NBUF; i++) mbar_init(&mbar[i], 1);
        fence_mbar_init();
    }
    uint32_t kseq = 0;
    const uint32_t t_scan = a.n_chunks, t_scat = t_scan + a.n_scans, t_join = t_scat + a.n_chunks;
    const uint32_t t_end = t_join + a.n_jt;
    for (;;) {
        if (tid == 0) s_ticket = atomicAdd(a.ticket, 1u);
        __syncthreads();
        const uint32_t t = s_ticket;
        __syncthreads();
        if (t >= t_end) break;
        if (t < t_scan) hist_chunk(a, t, reinterpret_cast<uint32_t *>(smem));
        else if (t < t_scat) scan_join(a, t - t_scan, reinterpret_cast<uint32_t *>(smem), scratch);
        else if (t < t_join) scatter_chunk(a, t - t_scat, *reinterpret_cast<BPart *>(smem), mbar, kseq);
        else join_ticket(a, t - t_join, smem, scratch, &s_item);
        __syncthreads();  // shared memory is reused by the next ticket
    }
}

size_t batch_smem_bytes() {
    size_t s = sizeof(BPart);
    const size_t j = join_smem_bytes(BATCH_CAPR);
    if (j > s) s = j;
    const size_t sc = std::max<size_t>(BATCH_THREADS + 4 * BATCH_FMAX, BATCH_THREADS / 32 * BATCH_FMAX) * sizeof(uint32_t);
    if (sc > s) s = sc;
    return s;
}

cudaError_t batch_occupancy(int *per_sm) {
    const size_t smem = batch_smem_bytes();
    int n = 0;
    cudaError_t e = smem_limit((const void *)k_batch, smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch, BATCH_THREADS, smem);
    if (e != cudaSuccess) return e;
    *per_sm = n < 1 ? 1 : n;
    return cudaSuccess;
}

int batch_ctas_per_sm() {
    int n = 1;
    if (batch_occupancy(&n) != cudaSuccess) cudaGetLastError();
    return n;
}

// batch_ctas_per_sm() (called when a plan is made, outside any stream
// capture) sets the kernel's shared-memory attribute.
cudaError_t launch_batch(const BatchArgs &a, int grid, cudaStream_t st) {
    k_batch<<<grid, BATCH_THREADS, batch_smem_bytes(), st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
